"""The reference-named seams (aerolume_b200.ns3d.fused, aerolume_b200.ns2d.step) called the way
the reference's solvers call them (ns3d/solver.py:583-595, 655-657; ns2d/solver.py:384-408)."""
from __future__ import annotations

import types

import numpy as np
import pytest
import torch

from _golden import load_case, load_case2d


def _rel(a, b):
    a = a.detach().double().cpu().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def test_load_kernels_refuses_a_cpu_device():
    from aerolume_b200.ns3d.fused import load_kernels
    with pytest.raises(RuntimeError):
        load_kernels("upwind3", torch.device("cpu"), torch.float32)


def test_step_full_refuses_diagnostics_and_placed_physics():
    from aerolume_b200.ns2d.step import State, step_full
    st = State(None, None, None, None, None, None)
    with pytest.raises(RuntimeError):
        step_full(st, None, None, diag=True)
    with pytest.raises(RuntimeError):
        step_full(st._replace(theta=1), None, None)


def test_thermal_from_physics_takes_heat_transfer():
    """The 2D plan reads heat transfer off the reference's Physics (fans, heaters, paint, jets
    and vents, smoke channels and the PID step are read by the plan itself) and returns None
    without heat transfer."""
    from aerolume_b200.ns2d.plan import thermal_from_physics
    from aerolume_b200.ns2d.types import Geometry2D
    geom = Geometry2D((2, 6, 3, 9), nbody=1)
    geom.thermal = types.SimpleNamespace(temp_ids=(0,), flux_ids=(), chi_t=np.ones((4, 6)), a_t=np.ones((4, 6)),
                                         w_t=np.ones((1, 4, 6)), ins_u=None, ins_v=None, q_skin=None, w_f=None,
                                         vol_u=None, vol_v=None)
    ph = types.SimpleNamespace(thermal=True, kappa=torch.tensor(0.01), ri=torch.tensor(0.5), prt=0.85,
                               gravity=(0.0, -1.0), eta_t=torch.tensor(0.005), theta_in=torch.tensor(0.0),
                               wall_modes=("inlet", "outlet", "adiabatic", "adiabatic"),
                               wall_values=torch.zeros(4), diff_coef=5.0, heat=None, ports=[], paint=False, nfan=0,
                               n_dye=0, comb=False, pid=False)
    th = thermal_from_physics(ph, geom)
    assert th.temp_ids == (0,) and th.wall_modes[0] == "inlet" and abs(th.kappa - 0.01) < 1e-9
    assert th.a_t is geom.thermal.a_t and th.wall_values == (0.0, 0.0, 0.0, 0.0)
    for name, val in (("nfan", 1), ("pid", True), ("paint", True), ("heat", torch.ones(2))):
        assert thermal_from_physics(types.SimpleNamespace(**{**vars(ph), name: val}), geom) is not None
    assert thermal_from_physics(types.SimpleNamespace(**{**vars(ph), "thermal": False}), geom) is None
    for name, val in (("ports", True), ("n_dye", 2), ("comb", True)):
        assert thermal_from_physics(types.SimpleNamespace(**{**vars(ph), name: val}), geom) is not None


def _dev(x, dt):
    x = np.asarray(x)
    return torch.as_tensor(np.ascontiguousarray(x).reshape(x.shape)).to("cuda", dt).contiguous()


@pytest.mark.gpu
def test_fast_step_phys_and_fast_dye_match_reference():
    from aerolume_b200.ns3d.fused import fast_dye, fast_step_phys, load_kernels
    from aerolume_b200.ns3d.types import State3D
    from oracle import ns3d as O
    meta, ops, geom, th, src, arr = load_case("tunnel_wale_heat_smoke_f64")
    dt = torch.float64
    kern = load_kernels(ops.advection, torch.device("cuda"), dt)
    phys = types.SimpleNamespace(thermal=th, fans=None, ports=None, paint=None, pid=None)
    nz, ny, nx = ops.nz, ops.ny, ops.nx
    state = State3D(_dev(arr["in_u"], dt), _dev(arr["in_v"], dt), _dev(arr["in_w"], dt),
                    torch.zeros(nz, ny, nx, device="cuda", dtype=dt), _dev(arr["in_t"], dt),
                    torch.zeros((), device="cuda", dtype=dt))
    out = fast_step_phys(state, geom, ops, kern, phys=phys, theta=_dev(arr["in_theta"], dt))
    torch.cuda.synchronize()
    for k, got in (("u", out.state.u), ("v", out.state.v), ("w", out.state.w), ("p", out.state.p),
                   ("theta", out.theta)):
        assert _rel(got, arr[f"out1_{k}"]) < 1e-10, k
    assert _rel(out.coeffs, arr["out1_coeffs"]) < 1e-9
    c = fast_dye(_dev(arr["in_dye"], dt), out.state.u, out.state.v, out.state.w, out.state.dt, ops, kern)
    want = O.advect_dye3d(arr["in_dye"], *(x.cpu().numpy() for x in (out.state.u, out.state.v, out.state.w)),
                          out.state.dt.cpu().numpy(), ops)
    assert _rel(c, want) < 1e-12


@pytest.mark.gpu
def test_step_full_matches_reference():
    from aerolume_b200.ns2d.step import State, step_full
    meta, ops, geom, arr = load_case2d("cylinder_upwind_f64")
    dt = torch.float64
    ny, nx = ops.ny, ops.nx
    st = State(_dev(arr["in_u"], dt), _dev(arr["in_v"], dt), torch.zeros(ny, nx, device="cuda", dtype=dt),
               _dev(arr["in_dye"], dt), _dev(arr["in_t"], dt), torch.zeros((), device="cuda", dtype=dt))
    new, coeffs = step_full(st, geom, ops, None)
    torch.cuda.synchronize()
    for k in ("u", "v", "p", "dye", "t", "dt"):
        assert _rel(getattr(new, k), arr[f"out1_{k}"]) < 1e-10, k
    assert _rel(coeffs, arr["out1_coeffs"]) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cavity_heated_wale_f64", "cylinder_heated_f64"])
def test_step_full_heat_matches_reference(name):
    """step_full with ops.phys carrying heat transfer (the attributes of the reference's 2D
    Physics) and geom.thermal: velocity, theta and the heat report in ``out``."""
    from _golden import thermal2d_from_case
    from aerolume_b200.ns2d.step import State, step_full
    meta, ops, geom, arr = load_case2d(name)
    th = thermal2d_from_case(meta, arr)
    dt = torch.float64
    ops.phys = types.SimpleNamespace(thermal=True, kappa=th.kappa, ri=th.ri, prt=th.prt, gravity=th.gravity,
                                     eta_t=th.eta_t, theta_in=th.theta_in, wall_modes=th.wall_modes,
                                     wall_values=th.wall_values, diff_coef=th.diff_coef, heat=None, ports=[],
                                     paint=False, nfan=0, n_dye=0, comb=False, pid=False)
    geom.thermal = th
    ny, nx = ops.ny, ops.nx
    st = State(_dev(arr["in_u"], dt), _dev(arr["in_v"], dt), torch.zeros(ny, nx, device="cuda", dtype=dt), None,
               _dev(arr["in_t"], dt), torch.zeros((), device="cuda", dtype=dt), _dev(arr["in_theta"], dt))
    out = {}
    new, coeffs = step_full(st, geom, ops, None, out=out)
    torch.cuda.synchronize()
    for k in ("u", "v", "p", "t", "dt", "theta"):
        assert _rel(getattr(new, k), arr[f"out1_{k}"]) < 1e-10, k
    assert _rel(coeffs, arr["out1_coeffs"]) < 1e-9
    for k in ("heat", "theta_wall", "wall_heat", "flow_heat"):
        assert (k in out) == (f"out1_rep_{k}" in arr), k
        if k in out:
            ref = arr[f"out1_rep_{k}"]
            assert np.abs(out[k].cpu().numpy() - ref).max() <= 1e-9 * max(np.abs(ref).max(), 1e-30), k


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["fans_swirl_f64", "ports_heat_f64", "tunnel_paint_pid_f64"])
def test_fast_step_phys_runs_the_placed_physics(name):
    """fast_step_phys with a Physics3D-shaped object carrying fans, jets / vents, paint and the
    PID controller: the step matches the reference and the objects' state tensors are the ones
    updated (FanSet.thrust, PidDt.dt_prev, ...), as the reference's solver expects."""
    from _golden import fan_items, port_items
    from aerolume_b200.ns3d.fused import fast_step_phys, load_kernels
    from aerolume_b200.ns3d.types import FanSet3D, PaintLayer3D, PidState3D, PortSet3D, State3D
    meta, ops, geom, th, src, arr = load_case(name)
    dt = torch.float64
    fans = ports = paint = pid = None
    if "fans" in meta:
        fm = meta["fans"]
        items = [{k: (_dev(x, dt) if k != "win" else x) for k, x in it.items()} for it in fan_items(meta, arr)]
        fans = FanSet3D(items, *(fm[k] for k in ("target", "kp", "ki", "tmax", "velocity_mode", "swirl")),
                        fm["any_swirl"], torch.tensor(fm["thrust"], device="cuda", dtype=dt),
                        *(torch.zeros(len(items), device="cuda", dtype=dt) for _ in range(3)))
    if "ports" in meta:
        ports = PortSet3D([{k: (_dev(x, dt) if isinstance(x, np.ndarray) else x) for k, x in it.items()}
                           for it in port_items(meta, arr)], meta["ports"]["mass_flux"], meta["ports"]["leak"])
    if "paint_u" in arr:
        paint = PaintLayer3D(*(_dev(arr["paint_" + g], dt) for g in "uvwc"))
    if "pid" in meta:
        pid = PidState3D(meta["pid"]["target"], *(torch.zeros((), device="cuda", dtype=dt) for _ in range(3)))
    phys = types.SimpleNamespace(thermal=th, fans=fans, ports=ports, paint=paint, pid=pid,
                                 u_floor=meta.get("u_floor", 0.0))
    kern = load_kernels(ops.advection, torch.device("cuda"), dt)
    nz, ny, nx = ops.nz, ops.ny, ops.nx
    state = State3D(_dev(arr["in_u"], dt), _dev(arr["in_v"], dt), _dev(arr["in_w"], dt),
                    torch.zeros(nz, ny, nx, device="cuda", dtype=dt), _dev(arr["in_t"], dt),
                    torch.zeros((), device="cuda", dtype=dt))
    theta = _dev(arr["in_theta"], dt) if "in_theta" in arr else None
    out = fast_step_phys(state, geom, ops, kern, phys=phys, theta=theta)
    torch.cuda.synchronize()
    for k, got in (("u", out.state.u), ("v", out.state.v), ("w", out.state.w), ("p", out.state.p)):
        assert _rel(got, arr[f"out1_{k}"]) < 1e-10, k
    if theta is not None:
        assert _rel(out.theta, arr["out1_theta"]) < 1e-10
    if fans is not None:
        got = np.stack([x.cpu().numpy() for x in (fans.thrust, fans.ud, fans.e_prev, fans.swirl_amp)])
        assert np.abs(got - arr["fans1"]).max() <= 1e-10 * max(1.0, np.abs(arr["fans1"]).max())
    if pid is not None:
        got = np.array([float(pid.dt_prev), float(pid.e1), float(pid.e2)])
        assert np.abs(got - arr["pid1"]).max() <= 1e-10 * max(1.0, np.abs(arr["pid1"]).max())


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tunnel_fans_pid_f64", "cavity_heater_paint_f64", "tunnel_ports_heat_f64",
                                  "closed_jet_paint_f64", "tunnel_smoke_channels_f64"])
def test_step_full_fans_heaters_paint_pid_match_reference(name):
    """step_full with ops.phys carrying fans and the PID step, or heaters and a paint layer (the
    reference's 2D Physics attribute names): three steps chained through State.ctrl and
    State.dt as the solver chains them, against the reference's own steps; the fans' and the
    paint's reports in ``out``."""
    from _golden import placed2d_from_case, thermal2d_from_case
    from aerolume_b200.ns2d.step import State, step_full
    meta, ops, geom, arr = load_case2d(name)
    dt = torch.float64
    th = thermal2d_from_case(meta, arr)
    pl = placed2d_from_case(meta, arr)
    ph = types.SimpleNamespace(**{k: getattr(pl, k) for k in vars(pl)}, comb=False, paint=pl.paint,
                               thermal=th is not None)
    if th is not None:
        for k in ("kappa", "ri", "prt", "gravity", "eta_t", "theta_in", "wall_modes", "wall_values", "diff_coef"):
            setattr(ph, k, getattr(th, k))
        geom.thermal = th
    ops.phys = ph
    ny, nx = ops.ny, ops.nx
    st = State(_dev(arr["in_u"], dt), _dev(arr["in_v"], dt), torch.zeros(ny, nx, device="cuda", dtype=dt),
               _dev(arr["in_dye"], dt) if "in_dye" in arr else None, _dev(arr["in_t"], dt),
               torch.zeros((), device="cuda", dtype=dt), _dev(arr["in_theta"], dt) if th is not None else None,
               _dev(arr["in_dye_extra"], dt) if "in_dye_extra" in arr else None,
               _dev(arr["in_ctrl"], dt) if "in_ctrl" in arr else None)
    out = {}
    new, _ = step_full(st, geom, ops, None, out=out)
    for key in ("fan_thrust", "fan_ud", "paint_force", "vent_heat", "jet_heat"):
        if f"out1_rep_{key}" in arr:
            ref = arr[f"out1_rep_{key}"]
            assert np.abs(out[key].cpu().numpy() - ref).max() <= 1e-9 * max(1.0, np.abs(ref).max()), key
    for _ in range(2):
        new, _ = step_full(new, geom, ops, None)
    torch.cuda.synchronize()
    for k in ("u", "v", "p", "t", "dt", "theta", "ctrl", "dye", "dye_extra"):
        if f"outN_{k}" in arr:
            assert _rel(getattr(new, k), arr[f"outN_{k}"]) < 1e-9, k
