"""Golden vectors of the reference's 3D mask construction (run in the build container).

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_masks.py

Three configurations go through the reference's own ``build_geometry3d(..., use_shared=False)``
(its exact signed distance to the triangle meshes, geometry.py:126-262, 385-495): a box on the
floor of a tunnel (the window touches the floor, so the floor's w-faces are zeroed) in FP64 and
FP32, and, in a y-periodic box, a spinning icosphere overlapping a second box (two bodies:
shared force weights, solid velocity of the spin).  The meshes come from the reference's
validation/ns3d_cases.py.  ``mesh_signed_distance`` at the known-answer points of
tests/test_ns3d_core.py:264-273 is stored too.  Everything goes to ``masks3d.npz``.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

import make_golden as G  # noqa: E402  (puts the reference on sys.path)
from aerolume.solvers.ns3d import core  # noqa: E402
from aerolume.solvers.ns3d.config import ImmersedMesh, SolverConfig3D  # noqa: E402
from aerolume.solvers.ns3d.geometry import build_geometry3d, mesh_signed_distance  # noqa: E402

CASES = G.CASES


def _mesh_case(tag, cfg_kw, bodies, dtype, out, cases_meta):
    cfg = SolverConfig3D(**{**cfg_kw, "bodies": bodies, "dtype": dtype, "device": "cpu", "perturb": False,
                            "dye": False})
    ops = core.make_operators3d(cfg)
    geom = build_geometry3d(cfg.bodies, ops, use_shared=False)
    meta = {"nx": cfg.nx, "ny": cfg.ny, "nz": cfg.nz, "h": float(ops.h), "origin": [ops.x0, ops.y0, ops.z0],
            "periodic_axes": list(ops.periodic_axes), "moment_ref": list(ops.moment_ref),
            "mask_width": float(ops.mask_width), "mask_shift": float(ops.mask_shift), "dtype": dtype,
            "window": list(geom.window), "nbody": len(bodies),
            "bodies": [{"omega": b.omega, "center": list(b.center), "axis": list(b.axis)} for b in bodies]}
    for q, b in enumerate(bodies):
        out[f"{tag}_v{q}"] = np.asarray(b.vertices, np.float64)
        out[f"{tag}_f{q}"] = np.asarray(b.faces, np.int64)
    for name in ("chi_u", "chi_v", "chi_w", "chi_c", "a_u", "a_v", "a_w", "k_u", "k_v", "k_w"):
        out[f"{tag}_{name}"] = getattr(geom, name).detach().cpu().numpy()
    out[f"{tag}_meta"] = np.array(json.dumps(meta))
    cases_meta.append(tag)


def main():
    torch.set_num_threads(8)
    out: dict = {}
    tags: list = []
    box = CASES.box_mesh(1.0, 1.0, 0.5, center=(2.3, 2.0, 0.25), n=2)
    tunnel = dict(nx=48, ny=32, nz=16, h=0.125, x0=0.0, y0=0.0, z0=0.0, re=1000.0, bc_zmin="moving", moment_ref=(2.3, 2.0, 0.0))
    for dt in ("float64", "float32"):
        _mesh_case(f"box_floor_{dt[5:]}", tunnel, [ImmersedMesh(box[0], box[1], name="box")], dt, out, tags)
    sph = CASES.icosphere(1.0, 2, center=(1.5, 1.0, 1.0))
    cube = CASES.box_mesh(0.5, 0.6, 0.5, center=(2.15, 1.1, 1.0))
    two = dict(nx=32, ny=16, nz=16, h=0.125, x0=0.0, y0=0.0, z0=0.0, re=500.0, bc_y="periodic", moment_ref=(1.5, 1.0, 1.0))
    bodies = [ImmersedMesh(sph[0], sph[1], name="ball", omega=2.0, center=(1.5, 1.0, 1.0), axis=(0.0, 0.6, 0.8)),
              ImmersedMesh(cube[0], cube[1], name="cube")]
    _mesh_case("sphere_spin_box_64", two, bodies, "float64", out, tags)
    # known answers of the reference's own test (tests/test_ns3d_core.py:264-273)
    v, f = CASES.icosphere(2.0, 3)
    pts = np.array([[0, 0, 0], [0.5, 0, 0], [2.0, 0, 0], [0, -3.0, 0]], dtype=np.float64)
    out["ka_sphere_v"], out["ka_sphere_f"], out["ka_sphere_p"] = v, f, pts
    out["ka_sphere_d"] = mesh_signed_distance(torch.as_tensor(v), torch.as_tensor(f), torch.as_tensor(pts)).numpy()
    v, f = CASES.box_mesh(1.0, 2.0, 3.0, n=2)
    pts = np.array([[0, 0, 0], [0.6, 0, 0], [0, 1.25, 0], [0.75, 1.25, 0]], dtype=np.float64)
    out["ka_box_v"], out["ka_box_f"], out["ka_box_p"] = v, f, pts
    out["ka_box_d"] = mesh_signed_distance(torch.as_tensor(v), torch.as_tensor(f), torch.as_tensor(pts)).numpy()
    out["cases"] = np.array(json.dumps(tags))
    np.savez_compressed(HERE / "masks3d.npz", **out)
    print("wrote", HERE / "masks3d.npz", tags)


if __name__ == "__main__":
    main()
