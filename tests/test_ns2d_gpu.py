"""The CUDA 2D step through the C ABI against the reference's golden vectors and the oracle."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from _golden import CASES_2D, GOLDEN, load_case2d, placed2d_from_case, thermal2d_from_case
from oracle import ns2d as O2

pytestmark = pytest.mark.gpu

# per-step tolerances relative to max |field|: FP64 agrees with the reference's FP64 step to
# round-off; FP32 to the stated 1e-5 of the FP32 step
TOL = {"float64": 1e-10, "float32": 1e-5}
TOL_COEFF = {"float64": 1e-9, "float32": 1e-4}


def _rel(a, b):
    a = a.detach().double().cpu().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _dev(x, dt):
    x = np.asarray(x)
    return torch.as_tensor(np.ascontiguousarray(x).reshape(x.shape)).to("cuda", dt).contiguous()


def _setup(name):
    from aerolume_b200.ns2d.plan import Ns2dPlan
    meta, ops, geom, arr = load_case2d(name)
    dt = torch.float64 if meta["dtype"] == "float64" else torch.float32
    plan = Ns2dPlan(ops, geom, dye="in_dye" in arr, thermal=thermal2d_from_case(meta, arr),
                    placed=placed2d_from_case(meta, arr))
    ins = {"u0": _dev(arr["in_u"], dt), "v0": _dev(arr["in_v"], dt), "t0": _dev(arr["in_t"], dt)}
    if "in_dye" in arr:
        ins["dye0"] = _dev(arr["in_dye"], dt)
    if "in_theta" in arr:
        ins["theta0"] = _dev(arr["in_theta"], dt)
    if "in_dye_extra" in arr:   # smoke channels 1..
        ins["dye_extra0"] = _dev(arr["in_dye_extra"], dt)
    if "in_ctrl" in arr:   # the controllers' memory and the previous step (0: the first)
        ins["ctrl0"] = _dev(arr["in_ctrl"], dt)
        ins["dt_prev"] = torch.zeros((), device="cuda", dtype=dt)
    return meta, plan, ins, arr


def _check_report(out, arr, meta):
    """The heat report against the reference's: each entry within TOL_COEFF of the larger of
    its own magnitude and the scale of the sums it is made of (heat storage is a difference
    of two sums over the grid, so its scale is sum |theta| h^2 / dt)."""
    tol = TOL_COEFF[meta["dtype"]]
    h2_dt = meta["h"] ** 2 / float(arr["out1_dt"])
    for key in ("heat", "theta_wall", "wall_heat", "heat_storage", "flow_heat"):
        ref_key = f"out1_rep_{key}"
        if ref_key not in arr:
            continue
        got = out[key].cpu().numpy()
        ref = np.asarray(arr[ref_key], np.float64)
        scale = max(np.abs(ref).max(), 1e-30)
        if key == "heat_storage":
            scale = max(scale, (np.abs(arr["in_theta"]).sum() + np.abs(arr["out1_theta"]).sum()) * h2_dt)
        assert got.shape == ref.shape, key
        assert np.abs(got - ref).max() <= tol * scale, (key, got, ref)


@pytest.mark.parametrize("name", CASES_2D)
def test_step2d_matches_reference(name):
    meta, plan, ins, arr = _setup(name)
    out = plan.step(**ins)
    torch.cuda.synchronize()
    tol = TOL[meta["dtype"]]
    for k in ("u", "v", "p"):
        assert _rel(out[k], arr[f"out1_{k}"]) < tol, (k, _rel(out[k], arr[f"out1_{k}"]))
    assert _rel(out["dt"], arr["out1_dt"]) < tol
    assert _rel(out["t"], arr["out1_t"]) < tol
    if meta["nbody"]:
        assert _rel(out["coeffs"], arr["out1_coeffs"]) < TOL_COEFF[meta["dtype"]]
    if "out1_dye" in arr:
        assert _rel(out["dye"], arr["out1_dye"]) < tol
    if "out1_dye_extra" in arr:
        assert _rel(out["dye_extra"], arr["out1_dye_extra"]) < tol
    if "out1_theta" in arr:
        assert _rel(out["theta"], arr["out1_theta"]) < tol, _rel(out["theta"], arr["out1_theta"])
        _check_report(out, arr, meta)
    # fans, paint and the controllers (core.py:998-1002, State.ctrl)
    for key, ref_key in (("fan_thrust", "out1_rep_fan_thrust"), ("fan_ud", "out1_rep_fan_ud"),
                         ("paint_force", "out1_rep_paint_force"), ("ctrl", "out1_ctrl"),
                         ("vent_heat", "out1_rep_vent_heat"), ("jet_heat", "out1_rep_jet_heat")):
        if ref_key in arr:
            ref = np.asarray(arr[ref_key], np.float64)
            got = out[key].double().cpu().numpy()
            assert np.abs(got - ref).max() <= TOL_COEFF[meta["dtype"]] * max(1.0, np.abs(ref).max()), (key, got, ref)
    assert plan.status() == 0 if hasattr(plan, "status") else True


@pytest.mark.parametrize("name", [c for c in CASES_2D if c.startswith(("cylinder", "tunnel_fans", "cavity_heater",
                                                                        "tunnel_ports", "closed_jet",
                                                                        "tunnel_smoke", "closed_wall"))
                                  or "heated" in c or "cold" in c])
def test_three_steps_in_place_match_reference(name):
    meta, plan, ins, arr = _setup(name)
    u, v, t, dye, theta = ins["u0"], ins["v0"], ins["t0"], ins.get("dye0"), ins.get("theta0")
    ctrl, dt_prev, extra = ins.get("ctrl0"), ins.get("dt_prev"), ins.get("dye_extra0")
    out = plan.empty_fields()
    for _ in range(3):
        out["u"], out["v"] = u, v             # in-place velocity update
        if theta is not None:
            out["theta"] = theta              # and theta in place
        res = plan.step(u, v, t, dye0=dye, theta0=theta, out=out, ctrl0=ctrl, dt_prev=dt_prev, dye_extra0=extra)
        t = res["t"].clone()
        if ctrl is not None:
            ctrl, dt_prev = res["ctrl"].clone(), res["dt"].clone()
        if dye is not None:
            dye, res["dye"] = res["dye"], dye  # ping-pong the dye
        if extra is not None:
            extra, res["dye_extra"] = res["dye_extra"], extra
    torch.cuda.synchronize()
    tol = 10 * TOL[meta["dtype"]]
    for k, got in (("u", u), ("v", v), ("p", res["p"]), ("t", t)):
        assert _rel(got, arr[f"outN_{k}"]) < tol, (k, _rel(got, arr[f"outN_{k}"]))
    if dye is not None:
        assert _rel(dye, arr["outN_dye"]) < tol
    if theta is not None:
        assert _rel(theta, arr["outN_theta"]) < tol, _rel(theta, arr["outN_theta"])
    if ctrl is not None:
        assert _rel(ctrl, arr["outN_ctrl"]) < tol and _rel(dt_prev, arr["outN_dt"]) < tol
    if extra is not None:
        assert _rel(extra, arr["outN_dye_extra"]) < tol


def _poisson_plan(nx, ny, h, periodic, dtype):
    from aerolume_b200.ns2d.plan import Ns2dPlan
    from aerolume_b200.ns2d.types import Geometry2D, Ops2D
    ops = Ops2D(nx=nx, ny=ny, h=h, periodic=periodic, u_inlet=np.ones(ny), dtype=dtype)
    return Ns2dPlan(ops, Geometry2D((0, 0, 0, 0)))


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_poisson2d_matches_reference(dtype):
    z = np.load(GOLDEN / "poisson2d.npz")
    h = float(z["h"])
    tdt = torch.float64 if dtype == "float64" else torch.float32
    for n in range(int(z["count"])):
        nx, ny, per = (int(x) for x in z[f"meta{n}"])
        if nx < 4 or ny < 4:
            continue
        plan = _poisson_plan(nx, ny, h, bool(per), dtype)
        psi = plan.poisson_solve(_dev(z[f"f{n}"], tdt))
        assert _rel(psi, z[f"psi{n}"]) < (1e-12 if dtype == "float64" else 2e-6), (n, _rel(psi, z[f"psi{n}"]))


@pytest.mark.parametrize("shape", [(64, 32), (256, 128), (128, 128), (96, 40)])
def test_poisson2d_solves_exactly(shape):
    nx, ny = shape
    for per in (False, True):
        plan = _poisson_plan(nx, ny, 0.05, per, "float64")
        f = torch.randn(ny, nx, dtype=torch.float64, generator=torch.Generator().manual_seed(3))
        f = (f - f.mean()).cuda()
        psi = plan.poisson_solve(f)
        lap = O2.PoissonSolver2D.laplacian(psi.cpu().numpy(), 0.05, per)
        assert np.abs(lap - f.cpu().numpy()).max() < 1e-9 * f.abs().max().item()


@pytest.mark.parametrize("name", ["cylinder_upwind_f64", "cylinder_heated_f64", "periodic_cold_body_f64"])
def test_given_dt_matches_oracle(name):
    """dt passed in (``step_full(..., dt)``): used as given, against the oracle's step with the
    same dt (with heat transfer its dt limits do not apply either)."""
    meta, plan, ins, arr = _setup(name)
    _, ops, geom, _ = load_case2d(name)
    tp = thermal2d_from_case(meta, arr)
    dt_val = 0.6 * float(arr["out1_dt"])
    out = plan.step(**ins, dt=torch.tensor(dt_val, device="cuda", dtype=torch.float64))
    torch.cuda.synchronize()
    ps = O2.PoissonSolver2D(ops.nx, ops.ny, ops.h, ops.periodic, np.float64)
    t0 = np.float64(arr["in_t"])
    if tp is None:
        r = O2.step2d(arr["in_u"], arr["in_v"], t0, geom, ops, ps, dye=arr.get("in_dye"), dt=np.float64(dt_val))
    else:
        r = O2.step2d_thermal(arr["in_u"], arr["in_v"], t0, arr["in_theta"], geom, ops, ps, tp, dt=np.float64(dt_val))
    assert float(out["dt"]) == dt_val
    for f, ref in (("u", r.u), ("v", r.v), ("p", r.p)):
        assert _rel(out[f], ref) < 1e-10, (f, _rel(out[f], ref))
    if tp is not None:
        assert _rel(out["theta"], r.theta) < 1e-10


def test_two_temperature_bodies_split_heat_like_oracle():
    """Two temperature bodies sharing the window (the heat split by their shares w_t,
    physics.py:733-757), built from the heated-cylinder case: theta and both bodies' heat
    against the oracle in FP64."""
    import dataclasses
    from aerolume_b200.ns2d.plan import Ns2dPlan
    meta, ops, geom, arr = load_case2d("cylinder_heated_f64")
    tp = thermal2d_from_case(meta, arr)
    wy, wx = tp.chi_t.shape
    share = np.linspace(0.2, 0.8, wx)[None, :] * np.ones((wy, 1))
    tp2 = dataclasses.replace(tp, temp_ids=(0, 1), w_t=np.stack([share, 1.0 - share]),
                              a_t=tp.chi_t * (0.5 + 0.5 * share))
    plan = Ns2dPlan(ops, geom, thermal=tp2)
    dt = torch.float64
    out = plan.step(_dev(arr["in_u"], dt), _dev(arr["in_v"], dt), _dev(arr["in_t"], dt),
                    theta0=_dev(arr["in_theta"], dt))
    torch.cuda.synchronize()
    ps = O2.PoissonSolver2D(ops.nx, ops.ny, ops.h, ops.periodic, np.float64)
    r = O2.step2d_thermal(arr["in_u"], arr["in_v"], np.float64(arr["in_t"]), arr["in_theta"], geom, ops, ps, tp2)
    assert _rel(out["theta"], r.theta) < 1e-10
    assert _rel(out["u"], r.u) < 1e-10
    ref = r.report["heat"]
    assert ref.shape == (2,) and np.abs(ref).min() > 0
    assert np.abs(out["heat"].cpu().numpy() - ref).max() <= 1e-9 * np.abs(ref).max()


def test_dye_with_heat_transfer_follows_the_step_velocity():
    """A plan with both dye and heat transfer: theta as without dye, and the dye advanced with
    the step's final velocity and dt and cleared in the solids (core.py:959-962)."""
    from aerolume_b200.ns2d.plan import Ns2dPlan
    meta, ops, geom, arr = load_case2d("cylinder_heated_f64")
    tp = thermal2d_from_case(meta, arr)
    ops.dye_inlet = np.linspace(0.0, 1.0, ops.ny)            # an inlet comb for the dye
    plan = Ns2dPlan(ops, geom, dye=True, thermal=tp)
    dt = torch.float64
    g = np.random.default_rng(7)
    dye0 = g.uniform(0.0, 1.0, (ops.ny, ops.nx))
    out = plan.step(_dev(arr["in_u"], dt), _dev(arr["in_v"], dt), _dev(arr["in_t"], dt),
                    dye0=_dev(dye0, dt), theta0=_dev(arr["in_theta"], dt))
    torch.cuda.synchronize()
    assert _rel(out["theta"], arr["out1_theta"]) < 1e-10
    u, v, step_dt = (out[k].cpu().numpy() for k in ("u", "v", "dt"))
    want = O2.zero_dye_in_solids(O2.advect_dye2d(dye0, u, v, step_dt, ops), geom)
    assert _rel(out["dye"], want) < 1e-12
