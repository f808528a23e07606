"""The bookkeeping kernels (aero_record_history, aero_welford) through the solver-shaped seam
``aerolume_b200.ns3d.record.record`` against the reference's own _record / _welford."""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from _golden import GOLDEN

pytestmark = pytest.mark.gpu

Z = np.load(GOLDEN / "record3d.npz")
CAP = int(Z["capacity"])


def _dev(x, dt):
    return torch.as_tensor(np.ascontiguousarray(np.asarray(x))).to("cuda", dt)


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_record_matches_reference(tag):
    from aerolume_b200.ns3d.record import record
    dt = torch.float64 if tag == "f64" else torch.float32
    tol = 1e-12 if tag == "f64" else 1e-6
    shapes = {k: Z[f"{tag}_in0_field_{k}"].shape for k in "uvwpt"}
    heat = torch.zeros(2, device="cuda", dtype=dt)
    fans = SimpleNamespace(thrust=torch.zeros(1, device="cuda", dtype=dt), ud=torch.zeros(1, device="cuda", dtype=dt))
    avg = {"time": torch.zeros((), device="cuda", dtype=torch.float64),
           "pending": torch.zeros((), device="cuda", dtype=torch.float64)}
    for k, s in shapes.items():
        avg[k] = torch.zeros(s, device="cuda", dtype=dt)
        avg[k + "2"] = torch.zeros(s, device="cuda", dtype=dt)
    self = SimpleNamespace(dtype=dt, _body_c=torch.zeros(2, 6, device="cuda", dtype=dt),
                           _hist=torch.zeros(CAP, 7, device="cuda", dtype=dt),
                           _hist_n=torch.tensor(int(Z[f"{tag}_hist_n0"]), device="cuda", dtype=torch.int64),
                           _phist=torch.zeros(CAP, 5, device="cuda", dtype=dt), _phist_walls=False, _avg_on=True,
                           _avg=avg, _theta=None,
                           _phys=SimpleNamespace(thermal=SimpleNamespace(heat_rate=heat), fans=fans))
    for step in range(5):
        f = {k: _dev(Z[f"{tag}_in{step}_field_{k}"], dt) for k in "uvwpt"}
        self._theta = f["t"]
        ex = Z[f"{tag}_in{step}_extra"]
        heat.copy_(_dev(ex[:2], dt))
        fans.thrust.copy_(_dev(ex[2:3], dt))
        fans.ud.copy_(_dev(ex[3:4], dt))
        new = SimpleNamespace(u=f["u"], v=f["v"], w=f["w"], p=f["p"], t=_dev(Z[f"{tag}_in{step}_t"], dt),
                              dt=_dev(Z[f"{tag}_in{step}_dt"], dt))
        record(self, new, _dev(Z[f"{tag}_in{step}_bc"], dt), bool(Z[f"{tag}_in{step}_sample"]))
        torch.cuda.synchronize()
        rows = list(Z[f"{tag}_out{step}_hist_rows"])
        assert int(self._hist_n) == int(Z[f"{tag}_out{step}_hist_n"])
        assert np.abs(self._hist[rows].double().cpu().numpy() - Z[f"{tag}_out{step}_hist"]).max() <= tol * 10
        assert np.abs(self._phist[rows].double().cpu().numpy() - Z[f"{tag}_out{step}_phist"]).max() == 0
        assert np.abs(self._body_c.double().cpu().numpy() - Z[f"{tag}_out{step}_body_c"]).max() == 0
        assert float(avg["time"]) == float(Z[f"{tag}_out{step}_time"])
        assert float(avg["pending"]) == float(Z[f"{tag}_out{step}_pending"])
        for k in "uvwpt":
            for name, got in (("mean", avg[k]), ("m2", avg[k + "2"])):
                ref = Z[f"{tag}_out{step}_{name}_{k}"]
                err = np.abs(got.double().cpu().numpy() - ref).max() / max(np.abs(ref).max(), 1.0)
                assert err <= tol, (step, name, k, err)


def test_welford_unaligned_fields_match_aligned():
    """Fields off a 16-byte boundary take the scalar path and give the same means."""
    from aerolume_b200.ns3d.record import welford
    g = torch.Generator(device="cpu").manual_seed(3)
    x = torch.randn(1001, generator=g, dtype=torch.float32).cuda()
    buf = torch.zeros(1002, device="cuda")
    xu = buf[1:].view(1001)
    xu.copy_(x)
    outs = []
    for src in (x, xu):
        a = {"time": torch.tensor(0.5, device="cuda", dtype=torch.float64),
             "pending": torch.tensor(0.25, device="cuda", dtype=torch.float64),
             "u": torch.ones(1001, device="cuda"), "u2": torch.zeros(1001, device="cuda")}
        welford(None, a, [src])
        outs.append((a["u"].clone(), a["u2"].clone(), float(a["time"]), float(a["pending"])))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    assert outs[0][2] == 0.75 and outs[0][3] == 0.0
    r = np.float32(0.25 / 0.75)
    want = 1 + (x.cpu().numpy() - 1) * r
    assert np.abs(outs[0][0].cpu().numpy() - want).max() < 1e-6
