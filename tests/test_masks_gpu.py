"""Mask construction on the GPU (aero_ns3d_build_masks, aero_mesh_signed_distance) against the
reference's own masks, the oracle, and the closed-form distance of a box at full size."""
from __future__ import annotations

import types

import numpy as np
import pytest
import torch

from _golden import load_masks, masks_case
from oracle import masks3d as M

pytestmark = pytest.mark.gpu

Z, TAGS = load_masks()
NAMES = ("chi_u", "chi_v", "chi_w", "chi_c", "a_u", "a_v", "a_w", "k_u", "k_v", "k_w")
# FP64: round-off of the distance arithmetic (FMA contraction); FP32: the field tolerance
TOL = {"float64": 1e-10, "float32": 1e-5}


def _cmp(got, ref, tol, name):
    got = got.detach().double().cpu().numpy()
    ref = np.asarray(ref, np.float64)
    assert got.shape == ref.shape, name
    err = np.abs(got - ref).max() / max(np.abs(ref).max(), 1.0)
    assert err <= tol, (name, err)


@pytest.mark.parametrize("tag", TAGS)
def test_masks_match_reference(tag):
    from aerolume_b200.ns3d.masks import build_geometry3d
    meta, ops, bodies = masks_case(Z, tag)
    g = build_geometry3d(bodies, ops, device="cuda")
    torch.cuda.synchronize()
    assert list(g.window) == meta["window"] and g.nbody == meta["nbody"]
    for n in NAMES:
        _cmp(getattr(g, n), Z[f"{tag}_{n}"], TOL[meta["dtype"]], n)


@pytest.mark.parametrize("name", ["sphere", "box"])
def test_signed_distance_known_answers(name):
    from aerolume_b200.ns3d.masks import mesh_signed_distance
    p = torch.as_tensor(Z[f"ka_{name}_p"]).cuda()
    d = mesh_signed_distance(Z[f"ka_{name}_v"], Z[f"ka_{name}_f"], p)
    assert np.abs(d.cpu().numpy() - Z[f"ka_{name}_d"]).max() < 1e-12


def test_signed_distance_survives_flipped_winding_and_matches_oracle():
    from aerolume_b200.ns3d.masks import mesh_signed_distance
    v, f = Z["ka_sphere_v"], Z["ka_sphere_f"]
    rng = np.random.default_rng(5)
    p = rng.uniform(-1.6, 1.6, size=(3000, 3))
    want = M.mesh_signed_distance(v, f, p, plane_zone=1e-3)
    got = mesh_signed_distance(v, f, torch.as_tensor(p).cuda(), plane_zone=1e-3).cpu().numpy()
    assert np.abs(got - want).max() < 1e-12
    flip = mesh_signed_distance(v, f[:, ::-1].copy(), torch.as_tensor(p).cuda()).cpu().numpy()
    assert np.array_equal(flip < 0, want < 0)


def test_masks_of_a_tilted_spinning_sphere_match_oracle():
    """A seeded attitude (pitch 7 deg, yaw 12 deg about the moment reference) of the level-2
    sphere, spinning, next to the floor of a bounded box: every output against the oracle."""
    from aerolume_b200.ns3d.masks import build_geometry3d, rotation_matrix
    v, f = Z["sphere_spin_box_64_v0"], Z["sphere_spin_box_64_f0"]
    ref = np.array([1.5, 1.0, 1.0])
    v = (v - ref) @ rotation_matrix(7.0, 12.0).T + ref + np.array([0.05, 0.02, -0.55])
    ops = types.SimpleNamespace(nx=40, ny=32, nz=24, h=1 / 16, x0=0.0, y0=0.0, z0=0.0,
                                periodic_axes=(False, False, False), moment_ref=(1.5, 1.0, 0.45), mask_width=1.0,
                                mask_shift=0.32, dtype="float64")
    body = types.SimpleNamespace(vertices=v, faces=f, omega=-1.5, center=(1.55, 1.02, 0.45), axis=(0.0, 1.0, 0.0))
    g = build_geometry3d([body], ops, device="cuda")
    mops = M.MaskOps(40, 32, 24, 1 / 16, moment_ref=(1.5, 1.0, 0.45))
    want = M.build_geometry3d([M.MeshBody(v, f, -1.5, (1.55, 1.02, 0.45), (0.0, 1.0, 0.0))], mops, np.float64)
    assert tuple(g.window) == want["window"] and g.window[0] == 0
    for n in NAMES:
        _cmp(getattr(g, n), want[n], 1e-10, n)


def _box_mesh(lo, hi):
    """Closed axis-aligned box, 12 triangles wound outward."""
    x = [lo[0], hi[0]]
    y = [lo[1], hi[1]]
    z = [lo[2], hi[2]]
    v = np.array([[x[i], y[j], z[k]] for k in range(2) for j in range(2) for i in range(2)], dtype=np.float64)
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    f = []
    for a, b, c, d in quads:
        f += [(a, b, c), (a, c, d)]
    return v, np.array(f, dtype=np.int64)


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_box_masks_at_bench_size_equal_closed_form(dtype):
    """The 1 x 1 x 0.5 box on the moving floor of the 256 x 128 x 128 tunnel: the masks from its
    12-triangle mesh equal those of the box's closed-form signed distance."""
    from aerolume_b200.ns3d.masks import build_geometry3d
    from aerolume_b200.ns3d.workloads import box_on_moving_floor
    ops, geom, _, _, boxes = box_on_moving_floor(256, 128, 128, dtype=dtype, seed=0)
    v, f = _box_mesh(*boxes[0].bounds)
    g = build_geometry3d([(v, f)], ops, device="cuda")
    assert tuple(g.window) == tuple(geom.window)
    for n in NAMES:
        _cmp(getattr(g, n), getattr(geom, n), TOL[dtype], n)


def test_bad_meshes_are_refused():
    """A face naming a vertex that does not exist, a mesh without faces and more than eight
    bodies raise before anything is launched."""
    from aerolume_b200.ns3d.masks import build_geometry3d, mesh_signed_distance
    meta, ops, bodies = masks_case(Z, "box_floor_64")
    v, f = bodies[0].vertices, bodies[0].faces
    bad = f.copy()
    bad[3, 1] = len(v)
    with pytest.raises(ValueError):
        build_geometry3d([(v, bad)], ops, device="cuda")
    with pytest.raises(ValueError):
        build_geometry3d([(v, f[:0])], ops, device="cuda")
    with pytest.raises(RuntimeError):
        build_geometry3d([(v, f)] * 9, ops, device="cuda")
    with pytest.raises(ValueError):
        mesh_signed_distance(v, bad, torch.zeros(4, 3, device="cuda", dtype=torch.float64))
