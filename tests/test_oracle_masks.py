"""The mask-construction oracle and the host-side window rule against the reference's own
masks (tests/golden/masks3d.npz, from build_geometry3d with its exact signed distance)."""
from __future__ import annotations

import numpy as np
import pytest

from _golden import load_masks, masks_case
from oracle import masks3d as M

Z, TAGS = load_masks()
NAMES = ("chi_u", "chi_v", "chi_w", "chi_c", "a_u", "a_v", "a_w", "k_u", "k_v", "k_w")


def _oracle(tag):
    meta, ops, bodies = masks_case(Z, tag)
    mops = M.MaskOps(ops.nx, ops.ny, ops.nz, ops.h, ops.x0, ops.y0, ops.z0, ops.periodic_axes, ops.moment_ref,
                     ops.mask_width, ops.mask_shift)
    mb = [M.MeshBody(b.vertices, b.faces, b.omega, b.center, b.axis) for b in bodies]
    dt = np.float64 if meta["dtype"] == "float64" else np.float32
    return meta, M.build_geometry3d(mb, mops, dt)


@pytest.mark.parametrize("tag", TAGS)
def test_oracle_masks_match_reference(tag):
    meta, out = _oracle(tag)
    assert list(out["window"]) == meta["window"]
    tol = 1e-12 if meta["dtype"] == "float64" else 1e-6
    for n in NAMES:
        ref = Z[f"{tag}_{n}"]
        assert out[n].shape == ref.shape, n
        assert np.abs(out[n].astype(np.float64) - ref).max() <= tol * max(np.abs(ref).max(), 1.0), n


def test_oracle_masks_are_not_vacuous():
    """The cases exercise what they claim: a solid core, zeroed floor faces, two bodies
    sharing faces, a spinning body's solid velocity."""
    assert Z["box_floor_64_chi_c"].max() == 1.0 and Z["box_floor_64_chi_c"].min() == 0.0
    assert np.all(Z["box_floor_64_chi_w"][0] == 0.0) and Z["box_floor_64_chi_w"][1].max() > 0.9
    k = Z["sphere_spin_box_64_k_u"]
    shared = (k[0, 0] > 0.05) & (k[1, 0] > 0.05)
    assert shared.any() and np.allclose((k[0, 0] + k[1, 0])[shared], 1.0)
    assert np.abs(Z["sphere_spin_box_64_a_u"]).max() > 0.1


@pytest.mark.parametrize("name", ["sphere", "box"])
def test_oracle_signed_distance_known_answers(name):
    d = M.mesh_signed_distance(Z[f"ka_{name}_v"], Z[f"ka_{name}_f"], Z[f"ka_{name}_p"])
    assert np.abs(d - Z[f"ka_{name}_d"]).max() < 1e-12


def test_oracle_sign_survives_flipped_winding():
    """tests/test_ns3d_core.py:276-285: a mesh wound the other way classifies alike."""
    v, f, p = Z["ka_sphere_v"], Z["ka_sphere_f"], Z["ka_sphere_p"]
    a = M.mesh_signed_distance(v, f, p)
    b = M.mesh_signed_distance(v, f[:, ::-1].copy(), p)
    assert np.array_equal(a < 0, b < 0)


@pytest.mark.parametrize("tag", TAGS)
def test_body_window_matches_reference(tag):
    """The product's window rule (host code) gives the reference's window."""
    from aerolume_b200.ns3d.masks import body_window3d
    meta, ops, bodies = masks_case(Z, tag)
    assert list(body_window3d([b.vertices for b in bodies], ops)) == meta["window"]


def test_body_window_covers_attitude_sweep():
    from aerolume_b200.ns3d.masks import body_window3d, rotation_matrix
    meta, ops, bodies = masks_case(Z, "box_floor_64")
    v = bodies[0].vertices
    wide = body_window3d([v], ops, pitch_deg=10.0, yaw_deg=15.0)
    ref = np.asarray(ops.moment_ref)
    for pa, ya in ((10.0, 15.0), (-10.0, 0.0), (0.0, -15.0)):
        rot = (v - ref) @ rotation_matrix(pa, ya).T + ref
        inner = body_window3d([rot], ops)
        assert all(wide[2 * a] <= inner[2 * a] and inner[2 * a + 1] <= wide[2 * a + 1] for a in range(3))
