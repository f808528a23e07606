"""Golden vectors of the reference's per-step bookkeeping (run in the build container).

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_record.py

``FlowSolver3D._record`` and ``_welford`` (src/aerolume/solvers/ns3d/solver.py:706-744) are
called, unmodified, on an object carrying just the attributes they read: the history ring
(capacity 4096, seeded to wrap), the physics history, the running-mean buffers.  Five steps of
seeded states (u, v, w, p, theta on a 12 x 10 x 8 grid, two bodies' coefficients, heat rates,
fan thrust) go through them, every second step a Welford sample, in FP64 and FP32; the buffers
after every step go to ``record3d.npz``.
"""
from __future__ import annotations

import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

import make_golden as G  # noqa: E402,F401  (puts the reference on sys.path)
from aerolume.solvers.ns3d import solver as S  # noqa: E402


def _case(dtype, out, tag):
    dt = torch.float64 if dtype == "float64" else torch.float32
    g = torch.Generator().manual_seed(11 if dtype == "float64" else 12)
    nz, ny, nx = 8, 10, 12
    shapes = {"u": (nz, ny, nx + 1), "v": (nz, ny + 1, nx), "w": (nz + 1, ny, nx), "p": (nz, ny, nx),
              "t": (nz, ny, nx)}
    cap = S.HISTORY_CAPACITY
    self = SimpleNamespace(dtype=dt, _body_c=torch.zeros(2, 6, dtype=dt), _hist=torch.zeros(cap, 7, dtype=dt),
                           _hist_n=torch.tensor(cap - 2, dtype=torch.long), _phist=torch.zeros(cap, 5, dtype=dt),
                           _phist_walls=False, _avg_on=True, _theta=None)
    self._welford = lambda a, fields: S.FlowSolver3D._welford(self, a, fields)
    self._avg = {"time": torch.zeros((), dtype=torch.float64), "pending": torch.zeros((), dtype=torch.float64)}
    for name, sh in shapes.items():
        self._avg[name] = torch.zeros(sh, dtype=dt)
        self._avg[name + "2"] = torch.zeros(sh, dtype=dt)
    heat = torch.zeros(2, dtype=dt)
    fans = SimpleNamespace(thrust=torch.zeros(1, dtype=dt), ud=torch.zeros(1, dtype=dt))
    self._phys = SimpleNamespace(thermal=SimpleNamespace(heat_rate=heat), fans=fans)
    out[f"{tag}_hist_n0"] = self._hist_n.numpy().copy()
    t = 0.0
    for step in range(5):
        dts = 0.01 + 0.002 * step
        t += dts
        f = {k: torch.randn(sh, generator=g, dtype=torch.float64).to(dt) for k, sh in shapes.items()}
        self._theta = f["t"]
        bc = torch.randn(2, 6, generator=g, dtype=torch.float64).to(dt)
        heat.copy_(torch.randn(2, generator=g, dtype=torch.float64).to(dt))
        fans.thrust.copy_(torch.randn(1, generator=g, dtype=torch.float64).to(dt))
        fans.ud.copy_(torch.randn(1, generator=g, dtype=torch.float64).to(dt))
        new = SimpleNamespace(u=f["u"], v=f["v"], w=f["w"], p=f["p"], t=torch.tensor(t, dtype=dt),
                              dt=torch.tensor(dts, dtype=dt))
        sample = step % 2 == 1
        for k, x in f.items():
            out[f"{tag}_in{step}_field_{k}"] = x.numpy()
        out[f"{tag}_in{step}_bc"] = bc.numpy()
        out[f"{tag}_in{step}_extra"] = torch.cat([heat, fans.thrust, fans.ud]).numpy()
        out[f"{tag}_in{step}_t"] = new.t.numpy()
        out[f"{tag}_in{step}_dt"] = new.dt.numpy()
        out[f"{tag}_in{step}_sample"] = np.array(sample)
        S.FlowSolver3D._record(self, new, bc, sample)
        for k in shapes:
            out[f"{tag}_out{step}_mean_{k}"] = self._avg[k].numpy().copy()
            out[f"{tag}_out{step}_m2_{k}"] = self._avg[k + "2"].numpy().copy()
        out[f"{tag}_out{step}_time"] = self._avg["time"].numpy().copy()
        out[f"{tag}_out{step}_pending"] = self._avg["pending"].numpy().copy()
        n = int(self._hist_n)
        rows = [(n - 1 - q) % cap for q in range(min(step + 1, 3))]
        out[f"{tag}_out{step}_hist_rows"] = np.array(rows)
        out[f"{tag}_out{step}_hist"] = self._hist[rows].numpy().copy()
        out[f"{tag}_out{step}_phist"] = self._phist[rows].numpy().copy()
        out[f"{tag}_out{step}_hist_n"] = self._hist_n.numpy().copy()
        out[f"{tag}_out{step}_body_c"] = self._body_c.numpy().copy()


def main():
    torch.set_num_threads(4)
    out: dict = {}
    for dtype, tag in (("float64", "f64"), ("float32", "f32")):
        _case(dtype, out, tag)
    out["capacity"] = np.array(S.HISTORY_CAPACITY)
    np.savez_compressed(HERE / "record3d.npz", **out)
    print("wrote", HERE / "record3d.npz")


if __name__ == "__main__":
    main()
