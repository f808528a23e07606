"""The 2D mask construction (aerolume_b200.ns2d.setup) against the masks the reference built for
the golden cylinder case, and the sweep's airfoils (host logic, no GPU)."""
from __future__ import annotations

import numpy as np

from _golden import load_case2d
from aerolume_b200.ns2d.setup import build_geometry, make_ops
from aerolume_b200.ns2d.workloads import circle, naca4, sweep_instances


def test_cylinder_masks_match_reference():
    meta, ops, geom, arr = load_case2d("cylinder_upwind_f64")
    mine = make_ops(meta["nx"], meta["ny"], meta["h"], 1.0 / meta["nu"], force_ref=meta["force_ref"],
                    moment_ref=tuple(meta["moment_ref"]), dtype="float64", dye=True)
    g = build_geometry([circle(2.0, 2.0, 0.5, 64)], mine)
    assert g.window == tuple(meta["window"])
    for name in ("chi_u", "chi_v", "chi_c", "a_u", "a_v", "k_u", "k_v"):
        assert np.abs(getattr(g, name) - arr[name]).max() < 1e-12, name
    assert abs(mine.eta - meta["eta"]) < 1e-15
    assert np.array_equal(mine.dye_inlet, arr["dye_inlet"])


def test_two_body_masks_split_the_force_weights():
    meta, ops, geom, arr = load_case2d("tunnel_two_bodies_vreman_f64")
    a = circle(1.2, 1.1, 0.3, 48)
    b = np.array([[2.08, 1.18], [2.52, 1.18], [2.52, 1.62], [2.08, 1.62]])
    mine = make_ops(meta["nx"], meta["ny"], meta["h"], 1.0 / meta["nu"], moment_ref=tuple(meta["moment_ref"]),
                    inlet="parabolic", dtype="float64")
    g = build_geometry([a, b], mine)
    assert g.window == tuple(meta["window"])
    for name in ("chi_u", "chi_v", "k_u", "k_v"):
        assert np.abs(getattr(g, name) - arr[name]).max() < 1e-12, name
    assert np.abs(mine.u_inlet - arr["u_inlet"]).max() < 1e-15


def test_naca_outline_and_sweep_are_reproducible():
    pts = naca4(0.12, 0.0, 0.4, 0.0, pivot=(0.25, 0.0))
    assert abs(pts[:, 0].min()) < 1e-12 and abs(pts[:, 0].max() - 1.0) < 1e-12
    assert abs(pts[:, 1].max() - 0.06) < 2e-3 and abs(pts[:, 1].min() + 0.06) < 2e-3     # 12 % thick
    area = 0.5 * np.sum(pts[:, 0] * np.roll(pts[:, 1], -1) - np.roll(pts[:, 0], -1) * pts[:, 1])
    assert area > 0                                                                     # counter-clockwise
    a = sweep_instances(4, seed=3)
    b = sweep_instances(4, seed=3)
    assert [x[2] for x in a] == [x[2] for x in b]
    for ops, geom, prm in a:
        assert (ops.nx, ops.ny) == prm["grid"] and geom.nbody == 1 and not geom.empty
