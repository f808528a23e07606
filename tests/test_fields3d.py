"""3D field outputs (cell-centred velocity, speed, vorticity, Q-criterion, eddy viscosity) and
trilinear probes: the oracle against the reference's own values (fields3d.npz), and the CUDA
kernels through the C ABI against them."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from _golden import load_fields_case
from oracle import fields3d as F

TAGS = ["tunnel", "periodic"]
NAMES = ("uc", "vc", "wc", "speed", "vorticity", "q", "nut")
OFFS = {"c": (0.5, 0.5, 0.5), "u": (0.0, 0.5, 0.5), "v": (0.5, 0.0, 0.5), "w": (0.5, 0.5, 0.0)}


def _rel(a, b):
    a = a.detach().double().cpu().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.parametrize("tag", TAGS)
def test_oracle_fields_match_reference(tag):
    meta, ops, geom, arr = load_fields_case(tag)
    u, v, w, mask = arr["in_u"], arr["in_v"], arr["in_w"], arr["in_mask"]
    got = {"uc": F.centre_u(u), "vc": F.centre_v(v), "wc": F.centre_w(w), "speed": F.speed(u, v, w),
           "vorticity": F.gradient_field("vorticity", u, v, w, ops), "q": F.gradient_field("q", u, v, w, ops),
           "nut": F.gradient_field("nut", u, v, w, ops, mask=mask)}
    for k in NAMES:
        assert _rel(got[k], arr[f"out_{k}"]) < 1e-12, k
    for c, src in (("c", arr["out_speed"]), ("u", u), ("v", v), ("w", w)):
        p = F.trilinear(src, arr["in_pts"], meta["origin"], ops.h, OFFS[c])
        assert _rel(p, arr[f"probe_{c}"]) < 1e-12, c


def _dev(x):
    return torch.as_tensor(np.ascontiguousarray(x)).to("cuda", torch.float64).contiguous()


@pytest.mark.gpu
@pytest.mark.parametrize("tag", TAGS)
def test_cuda_fields_and_probes_match_reference(tag):
    from aerolume_b200.ns3d.plan import Ns3dPlan
    meta, ops, geom, arr = load_fields_case(tag)
    plan = Ns3dPlan(ops, geom)
    u, v, w = _dev(arr["in_u"]), _dev(arr["in_v"]), _dev(arr["in_w"])
    out = plan.fields(u, v, w, NAMES)
    torch.cuda.synchronize()
    for k in NAMES:
        assert _rel(out[k], arr[f"out_{k}"]) < 1e-10, k
    pts = _dev(arr["in_pts"])
    for c, src in (("c", out["speed"]), ("u", u), ("v", v), ("w", w)):
        p = plan.probe(src, pts, OFFS[c], origin=tuple(meta["origin"]))
        torch.cuda.synchronize()
        assert _rel(p, arr[f"probe_{c}"]) < 1e-10, c


@pytest.mark.gpu
def test_cuda_slice_interpolates_between_cell_planes():
    from aerolume_b200.ns3d.plan import Ns3dPlan
    meta, ops, geom, arr = load_fields_case("tunnel")
    plan = Ns3dPlan(ops, geom)
    u, v, w = _dev(arr["in_u"]), _dev(arr["in_v"]), _dev(arr["in_w"])
    q = arr["out_q"]
    h = ops.h
    for axis, dim, pos in (("x", 2, 7.3 * h), ("y", 1, 0.2 * h), ("z", 0, 99.0)):
        n = q.shape[dim]
        f = min(max(pos / h - 0.5, 0.0), n - 1.0)
        i0 = min(int(np.floor(f)), max(n - 2, 0))
        t = f - i0
        want = (1.0 - t) * np.take(q, i0, axis=dim) + t * np.take(q, min(i0 + 1, n - 1), axis=dim)
        got = plan.slice(u, v, w, "q", axis, pos)
        assert _rel(got, want) < 1e-10, axis
