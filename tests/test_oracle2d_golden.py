"""The 2D oracle against golden vectors produced by the reference itself (make_golden2d.py)."""
from __future__ import annotations

import numpy as np
import pytest

from _golden import CASES_2D, GOLDEN, load_case2d, placed2d_from_case, thermal2d_from_case
from oracle import ns2d as O2

# float64: the restatement agrees with the reference to round-off; float32: to the FP32 step
TOL = {"float64": 1e-12, "float32": 2e-6}


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _run(name, steps=1):
    meta, ops, geom, arr = load_case2d(name)
    dt = np.float64 if meta["dtype"] == "float64" else np.float32
    ps = O2.PoissonSolver2D(ops.nx, ops.ny, ops.h, ops.periodic, dt)
    u, v, t = arr["in_u"], arr["in_v"], arr["in_t"]
    dye = arr.get("in_dye")
    tp = thermal2d_from_case(meta, arr)
    pl = placed2d_from_case(meta, arr)
    theta = arr.get("in_theta")
    ctrl, dt_prev, extra = arr.get("in_ctrl"), 0.0, arr.get("in_dye_extra")
    outs = []
    for _ in range(steps):
        if pl is not None:
            r = O2.step2d_placed(u, v, t, geom, ops, ps, tp=tp, pl=pl, theta0=theta, dye=dye, dt_prev=dt_prev,
                                 ctrl=ctrl, dye_extra=extra)
            theta, ctrl, dt_prev, extra = r.theta, r.ctrl, float(r.dt), r.dye_extra
        elif tp is not None:
            r = O2.step2d_thermal(u, v, t, theta, geom, ops, ps, tp)
            theta = r.theta
        else:
            r = O2.step2d(u, v, t, geom, ops, ps, dye=dye)
        outs.append(r)
        u, v, t, dye = r.u, r.v, r.t, r.dye
    return meta, arr, outs


@pytest.mark.parametrize("name", CASES_2D)
def test_oracle2d_one_step_matches_reference(name):
    meta, arr, (r,) = _run(name)
    tol = TOL[meta["dtype"]]
    if ("thermal" in meta or "placed" in meta) and meta["dtype"] == "float32":
        tol = 1e-5  # numpy's FP32 sums and limiter against torch's: round-off of the FP32 step
    for k, got in (("u", r.u), ("v", r.v), ("p", r.p)):
        assert _rel(got, arr[f"out1_{k}"]) < tol, (k, _rel(got, arr[f"out1_{k}"]))
    assert _rel(r.dt, arr["out1_dt"]) < tol
    assert _rel(r.t, arr["out1_t"]) < tol
    if meta["nbody"]:
        assert _rel(r.coeffs, arr["out1_coeffs"]) < (1e-10 if meta["dtype"] == "float64" else 1e-4)
    if "out1_dye" in arr:
        assert _rel(r.dye, arr["out1_dye"]) < tol
    if "out1_dye_extra" in arr:
        assert _rel(r.dye_extra, arr["out1_dye_extra"]) < tol
    if "out1_theta" in arr:
        assert _rel(r.theta, arr["out1_theta"]) < tol, _rel(r.theta, arr["out1_theta"])
    for key in [k[len("out1_rep_"):] for k in arr if k.startswith("out1_rep_")]:
        ref = arr["out1_rep_" + key]
        err = np.abs(np.asarray(r.report[key], np.float64) - ref).max() / max(1.0, np.abs(ref).max())
        assert err < (1e-10 if meta["dtype"] == "float64" else 1e-4), (key, err)
    if "out1_ctrl" in arr:
        assert np.abs(np.asarray(r.ctrl, np.float64) - arr["out1_ctrl"]).max() < 10 * tol, (r.ctrl, arr["out1_ctrl"])


@pytest.mark.parametrize("name", [c for c in CASES_2D if c.startswith(("cylinder", "tunnel_fans", "cavity_heater",
                                                                        "tunnel_ports", "closed_jet",
                                                                        "tunnel_smoke", "closed_wall"))])
def test_oracle2d_three_steps_match_reference(name):
    meta, arr, outs = _run(name, steps=3)
    tol = 10 * TOL[meta["dtype"]]
    if "placed" in meta and meta["dtype"] == "float32":
        tol = 1e-4
    r = outs[-1]
    for k, got in (("u", r.u), ("v", r.v), ("p", r.p), ("dye", r.dye), ("theta", getattr(r, "theta", None)),
                   ("ctrl", getattr(r, "ctrl", None)), ("dt", r.dt), ("dye_extra", getattr(r, "dye_extra", None))):
        if f"outN_{k}" in arr:
            assert _rel(got, arr[f"outN_{k}"]) < tol, (k, _rel(got, arr[f"outN_{k}"]))


def test_poisson2d_matches_reference():
    z = np.load(GOLDEN / "poisson2d.npz")
    h = float(z["h"])
    for n in range(int(z["count"])):
        nx, ny, per = (int(x) for x in z[f"meta{n}"])
        ps = O2.PoissonSolver2D(nx, ny, h, bool(per), np.float64)
        assert _rel(ps.solve(z[f"f{n}"]), z[f"psi{n}"]) < 1e-12, n
