"""The oracle against the reference's own outputs (golden vectors made by tests/golden/make_golden.py)."""
from __future__ import annotations

import numpy as np
import pytest

from _golden import CASES_3D, GOLDEN, load_case
from oracle import ns3d as O


def _run(name, steps=1):
    meta, ops, geom, th, src, arr = load_case(name)
    dt = np.float64 if meta["dtype"] == "float64" else np.float32
    ps = O.PoissonSolver3D(ops.nx, ops.ny, ops.nz, ops.h, ops.periodic_axes, dt)
    u, v, w, t = arr["in_u"], arr["in_v"], arr["in_w"], dt(arr["in_t"])
    theta = arr.get("in_theta")
    c = arr["in_dye"]
    outs = []
    for _ in range(steps):
        r = O.step3d_phys(u, v, w, t, geom, ops, ps, th=th, theta=theta)
        c = O.advect_dye3d(c, r.u, r.v, r.w, r.dt, ops)
        c = O.apply_solids_and_sources(c, r.t, geom, src)
        u, v, w, t, theta = r.u, r.v, r.w, r.t, r.theta
        r.dye = c
        outs.append(r)
    return meta, arr, outs


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.parametrize("name", CASES_3D)
def test_oracle_matches_reference_one_step(name):
    meta, arr, (r,) = _run(name)
    tol = 1e-12 if meta["dtype"] == "float64" else 2e-5
    for f in ("u", "v", "w", "p"):
        assert _rel(getattr(r, f), arr["out1_" + f]) < tol, f
    assert abs(float(r.dt) - float(arr["out1_dt"])) <= tol * float(arr["out1_dt"])
    assert abs(float(r.t) - float(arr["out1_t"])) <= tol * max(1.0, float(arr["out1_t"]))
    cref = arr["out1_coeffs"]
    assert cref.size == 0 or np.abs(r.coeffs - cref).max() <= (1e-10 if meta["dtype"] == "float64" else 1e-4) * max(1.0, np.abs(cref).max())
    if "out1_theta" in arr:
        assert _rel(r.theta, arr["out1_theta"]) < tol
        hr = arr["out1_heat_rate"]
        assert hr.size == 0 or np.abs(r.heat_rate - hr).max() <= (1e-10 if meta["dtype"] == "float64" else 1e-4) * max(1.0, np.abs(hr).max())
    assert _rel(r.dye, arr["out1_dye"]) < tol


@pytest.mark.parametrize("name", [n for n in CASES_3D if "tunnel" in n])
def test_oracle_matches_reference_three_steps(name):
    meta, arr, outs = _run(name, steps=3)
    r = outs[-1]
    tol = 1e-11 if meta["dtype"] == "float64" else 1e-4
    for f in ("u", "v", "w", "p", "theta"):
        assert _rel(getattr(r, f), arr["outN_" + f]) < tol, f
    assert _rel(r.dye, arr["outN_dye"]) < tol


def test_oracle_poisson_matches_reference():
    z = np.load(GOLDEN / "poisson3d.npz")
    h = float(z["h"])
    for n in range(int(z["count"])):
        nx, ny, nz, px, py, pz = (int(x) for x in z[f"meta{n}"])
        ps = O.PoissonSolver3D(nx, ny, nz, h, (bool(px), bool(py), bool(pz)), np.float64)
        psi = ps.solve(z[f"f{n}"])
        assert np.abs(psi - z[f"psi{n}"]).max() < 1e-12 * np.abs(z[f"psi{n}"]).max()
        # and the solve is exact: L psi = f (the reference's tests/test_ns3d_core.py:79-91)
        lap = ps.laplacian(psi, h, (bool(px), bool(py), bool(pz)))
        assert np.abs(lap - z[f"f{n}"]).max() < 1e-10 * np.abs(z[f"f{n}"]).max()
