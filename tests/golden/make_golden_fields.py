"""Golden vectors of the reference's 3D field outputs (run in the build container).

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_fields.py

Two seeded, projected states (the tunnel case with a box, WALE, and the periodic Vreman
box of make_golden.py) go through the reference's ``fields.gradient_field`` (vorticity, q,
nut with the body's solid fraction), the cell-centring of ``FlowSolver3D._centred`` (u, v,
w, speed) and ``fields.trilinear`` at seeded points for the centred field and each
staggered component.  Inputs, operators and outputs go to ``fields3d.npz``.
"""
from __future__ import annotations

import json
import math
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

import make_golden as G  # noqa: E402  (puts the reference on sys.path)
from aerolume.solvers.ns3d import core, fields  # noqa: E402
from aerolume.solvers.ns3d.config import ImmersedMesh, SolverConfig3D  # noqa: E402
from aerolume.solvers.ns3d.geometry import body_window3d, build_geometry3d  # noqa: E402

OFFS = {"c": (0.5, 0.5, 0.5), "u": (0.0, 0.5, 0.5), "v": (0.5, 0.0, 0.5), "w": (0.5, 0.5, 0.0)}


def case(tag, cfg_kw, seed, amp, out):
    cfg = SolverConfig3D(**{**cfg_kw, "dtype": "float64", "device": "cpu", "perturb": False})
    ops = core.make_operators3d(cfg)
    window = body_window3d([b.vertices_numpy() for b in cfg.bodies], ops) if cfg.bodies else (0, 0, 0, 0, 0, 0)
    geom = build_geometry3d(cfg.bodies, ops, window=window)
    u, v, w, _, _ = G._random_state(cfg, amp, seed)
    meta, arrays = G.extract(ops, geom, None, None)
    meta["origin"] = [ops.x0, ops.y0, ops.z0]
    mask = torch.zeros(cfg.nz, cfg.ny, cfg.nx, dtype=torch.float64)
    if not geom.empty:
        k0, k1, j0, j1, i0, i1 = geom.window
        mask[k0:k1, j0:j1, i0:i1] = geom.chi_c
    res = {"vorticity": fields.gradient_field("vorticity", u, v, w, ops),
           "q": fields.gradient_field("q", u, v, w, ops),
           "nut": fields.gradient_field("nut", u, v, w, ops, mask=mask),
           "uc": fields.centre_u(u), "vc": fields.centre_v(v), "wc": fields.centre_w(w)}
    res["speed"] = torch.sqrt(res["uc"] * res["uc"] + res["vc"] * res["vc"] + res["wc"] * res["wc"])
    g = torch.Generator().manual_seed(seed + 100)
    ext = torch.tensor([cfg.nx * cfg.h, cfg.ny * cfg.h, cfg.nz * cfg.h], dtype=torch.float64)
    org = torch.tensor([ops.x0, ops.y0, ops.z0], dtype=torch.float64)
    pts = org + (torch.rand(200, 3, generator=g, dtype=torch.float64) * 1.2 - 0.1) * ext   # some outside
    probes = {"c": fields.trilinear(res["speed"], pts, ops, OFFS["c"]), "u": fields.trilinear(u, pts, ops, OFFS["u"]),
              "v": fields.trilinear(v, pts, ops, OFFS["v"]), "w": fields.trilinear(w, pts, ops, OFFS["w"])}
    out[f"{tag}_meta"] = np.array(json.dumps(meta))
    for k, x in arrays.items():
        out[f"{tag}_{k}"] = np.asarray(x)
    for k, x in (("u", u), ("v", v), ("w", w), ("mask", mask), ("pts", pts)):
        out[f"{tag}_in_{k}"] = x.numpy()
    for k, x in res.items():
        out[f"{tag}_out_{k}"] = x.numpy()
    for k, x in probes.items():
        out[f"{tag}_probe_{k}"] = x.numpy()


def main():
    torch.set_num_threads(4)
    out = {}
    h = 1.0 / 6.0
    box = ImmersedMesh(*G.box_mesh(0.5, 0.5, 0.25, (1.25, 1.0, 0.125)), name="box")
    case("tunnel", {"nx": 24, "ny": 12, "nz": 10, "h": h, "x0": 0.0, "y0": 0.0, "z0": 0.0, "re": 1e4, "bodies": [box],
                    "bc_zmin": "moving", "ground_speed": 1.0, "turbulence": "wale", "ref_area": 0.125,
                    "moment_ref": (1.25, 1.0, 0.0)}, seed=11, amp=0.2, out=out)
    case("periodic", {"nx": 12, "ny": 10, "nz": 8, "h": 2 * math.pi / 12, "x0": 0.0, "y0": 0.0, "z0": 0.0,
                      "re": 2e3, "periodic": True, "turbulence": "vreman"}, seed=12, amp=0.5, out=out)
    np.savez_compressed(HERE / "fields3d.npz", **out)


if __name__ == "__main__":
    main()
