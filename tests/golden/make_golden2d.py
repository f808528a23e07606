"""Generate the golden vectors that pin the 2D oracle to the reference (run in the build container).

Usage (the reference checkout is named by ``AEROLUME_REF``; it is read, never modified)::

    AEROLUME_REF=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden2d.py

Each case builds a configuration with the reference's own 2D API (``SolverConfig``,
``make_operators``, ``build_geometry``), starts from the reference's initial state plus seeded
noise, imposes the boundary values and projects in FP64 (the pattern of the reference's
tests/test_ns2d_core.py), then runs ``core.step_full`` on the CPU.  Every input the step reads
and every output it returns is written to ``ns2d_<case>.npz`` beside this script; scalar
parameters go into a JSON ``meta`` entry.  ``poisson2d.npz`` holds ``PoissonSolver.solve`` on
seeded right-hand sides.  Nothing at test time needs the reference.
"""
from __future__ import annotations

import json
import math
import os
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
if "AEROLUME_REF" not in os.environ:
    sys.exit("set AEROLUME_REF to the reference checkout (the directory holding src/aerolume)")
REF = Path(os.environ["AEROLUME_REF"])
sys.path.insert(0, str(REF / "src"))

from aerolume.solvers.ns2d import core  # noqa: E402
from aerolume.solvers.ns2d import physics as phx  # noqa: E402
from aerolume.solvers.ns2d.config import (EmitterSpec, FanSpec, HeatSourceSpec, ImmersedBody,  # noqa: E402
                                          PortSpec, SolverConfig, ThermalConfig, WallBC)
from aerolume.solvers.ns2d.geometry import build_geometry  # noqa: E402
from aerolume.solvers.ns2d.poisson import PoissonSolver  # noqa: E402


def circle(cx, cy, r, n):
    a = 2.0 * math.pi * np.arange(n) / n
    return np.stack([cx + r * np.cos(a), cy + r * np.sin(a)], axis=1)


def square(cx, cy, s):
    return np.array([[cx - s, cy - s], [cx + s, cy - s], [cx + s, cy + s], [cx - s, cy + s]])


def _np(t):
    return None if t is None else t.detach().cpu().numpy().copy()


def extract(ops, geom):
    meta = {
        "nx": ops.nx, "ny": ops.ny, "h": ops.h, "x0": ops.x0, "y0": ops.y0, "periodic": bool(ops.periodic),
        "closed": bool(ops.closed), "bc_top": ops.bc_top, "bc_bottom": ops.bc_bottom, "bc_left": ops.bc_left,
        "bc_right": ops.bc_right, "ground_speed": float(ops.ground_speed), "advection": ops.advection,
        "turbulence": ops.turbulence, "les_c": float(ops.les_c), "nu": float(ops.nu), "eta": float(ops.eta),
        "cfl": float(ops.cfl), "dt_fixed": ops.dt_fixed, "force_ref": float(ops.force_ref),
        "moment_ref": list(ops.moment_ref), "window": list(geom.window), "nbody": int(geom.nbody),
        "wall_model": bool(ops.wall_model),
        "forcing": list(ops.forcing) if ops.forcing is not None else None,
        "dtype": "float64" if ops.dtype == torch.float64 else "float32",
    }
    arrays = {"u_inlet": _np(ops.u_inlet)[:, 0]}
    if ops.dye_inlet is not None:
        arrays["dye_inlet"] = _np(ops.dye_inlet)[:, 0]
    if not geom.empty:
        for name in ("chi_u", "chi_v", "chi_c", "a_u", "a_v", "k_u", "k_v"):
            arrays[name] = _np(getattr(geom, name))
    ph = ops.phys
    if ph is not None and ph.thermal:
        meta["thermal"] = {"kappa": float(ph.kappa), "ri": float(ph.ri), "prt": ph.prt, "gravity": list(ph.gravity),
                           "eta_t": float(ph.eta_t), "theta_in": float(ph.theta_in),
                           "wall_modes": list(ph.wall_modes), "wall_values": [float(x) for x in ph.wall_values],
                           "diff_coef": ph.diff_coef}
        tg = geom.thermal
        if tg is not None and not geom.empty:
            meta["thermal"]["temp_ids"] = list(tg.temp_ids)
            meta["thermal"]["flux_ids"] = list(tg.flux_ids)
            for name in ("chi_t", "a_t", "w_t", "ins_u", "ins_v", "q_skin", "w_f", "vol_u", "vol_v"):
                val = getattr(tg, name)
                if val is not None:
                    arrays["th_" + name] = _np(val)
    if ph is not None:
        # the placed physics besides heat transfer: fans, heaters, paint, the PID step
        meta["placed"] = {"nfan": ph.nfan, "pid": bool(ph.pid), "paint": bool(ph.paint), "ctrl_size": ph.ctrl_size,
                          "u_floor": float(ph.u_floor), "heat": ph.heat is not None, "ports": bool(ph.ports)}
        if ph.ports:
            meta["placed"]["q_net"] = float(ph.q_net)
            for name in ("src", "src_neg", "pchi_u", "pa_u", "pchi_v", "pa_v"):
                arrays[name] = _np(getattr(ph, name))
            if ph.pt_chi is not None:
                arrays["pt_chi"], arrays["pt_a"] = _np(ph.pt_chi), _np(ph.pt_a)
        if ph.ports or ph.paint:
            for name in ("xchi_u", "xa_u", "xchi_v", "xa_v"):
                arrays[name] = _np(getattr(ph, name))
        if ph.n_dye:   # smoke channels with emitter groups and port smoke (physics.py:497-540)
            meta["placed"]["n_dye"] = ph.n_dye
            meta["placed"]["groups"] = [int(g.channel) for g in ph.groups]
            meta["placed"]["port_dye"] = sorted(int(c) for c in ph.port_dye)
            arrays["dye_inflow"] = _np(ph.dye_inflow)[..., 0]
            for q, g in enumerate(ph.groups):
                arrays[f"group{q}_w"], arrays[f"group{q}_target"] = _np(g.weight), _np(g.target)
                arrays[f"group{q}_timing"] = _np(g.timing)
            for c, w in ph.port_dye.items():
                arrays[f"port_dye{c}"] = _np(w)
        if ph.nfan:
            for name in ("fan_gu", "fan_gv", "fan_phi", "fan_dir", "fan_value", "fan_width", "fan_kp", "fan_ki",
                         "fan_dpmax", "fan_isvel", "fan_isthrust"):
                arrays[name] = _np(getattr(ph, name))
        if ph.heat is not None:
            arrays["heat"] = _np(ph.heat)
            meta["placed"]["heat_max"] = float(ph.heat_max)
        if ph.paint:
            for name in ("paint_c", "paint_u", "paint_v", "paint_wu", "paint_wv"):
                arrays[name] = _np(getattr(ph, name))
    return meta, arrays


def _paint(ops, sdf):
    """A painted obstacle ``sdf(x, y) < 0`` on the grid of ``ops`` (the app's brush,
    physics.py:542-575), then the combined penalisation it enters."""
    if ops.phys is None:
        ops.phys = phx.empty_physics(ops)
    phx.ensure_paint(ops.phys, ops)
    phx.paint_brush(ops.phys, ops, sdf, 1.5, False)
    phx.combine_penalisation(ops.phys)


def _run_case(name, cfg_kw, *, dtype="float64", amp=0.1, seed=1, steps=1, paint=None, forcing=None):
    cfg64 = SolverConfig(**{**cfg_kw, "dtype": "float64", "device": "cpu", "perturb": False})
    cfg = SolverConfig(**{**cfg_kw, "dtype": dtype, "device": "cpu", "perturb": False})
    ops64 = core.make_operators(cfg64)
    ops = core.make_operators(cfg)
    if forcing is not None:   # a uniform body force (the verification cases' ops.forcing)
        ops.forcing = tuple(forcing)
    if paint is not None:
        _paint(ops, paint)
    geom = build_geometry(cfg.bodies, ops)
    s64 = core.init_state(cfg64, ops64, perturb=False)
    g = torch.Generator().manual_seed(seed)
    u = s64.u + amp * torch.randn(s64.u.shape, generator=g, dtype=torch.float64)
    v = s64.v + amp * torch.randn(s64.v.shape, generator=g, dtype=torch.float64)
    u, v = core._apply_boundary_values(u, v, ops64)
    u, v, _ = core.project(u, v, ops64)
    tdt = ops.dtype
    dye = None
    dye_extra = None
    if cfg.dye or cfg.dye_channels:
        dye = torch.rand((cfg.ny, cfg.nx), generator=g, dtype=torch.float64)
        dye[dye < 0.3] = 0.0
        dye = dye.to(tdt)
        if cfg.dye_channels > 1:
            dye_extra = torch.rand((cfg.dye_channels - 1, cfg.ny, cfg.nx), generator=g, dtype=torch.float64)
            dye_extra[dye_extra < 0.5] = 0.0
            dye_extra = dye_extra.to(tdt)
    zero = torch.zeros((), dtype=tdt)
    theta = None
    if cfg.thermal is not None:
        theta = (0.3 * torch.randn((cfg.ny, cfg.nx), generator=g, dtype=torch.float64)).to(tdt)
    ctrl = None
    if ops.phys is not None and ops.phys.ctrl_size:
        ctrl = torch.zeros(ops.phys.ctrl_size, dtype=tdt)
        ctrl[:2] = (0.2 * torch.randn(2, generator=g, dtype=torch.float64)).to(tdt)   # PID memory e1, e2
    state = core.State(u.to(tdt), v.to(tdt), torch.zeros(cfg.ny, cfg.nx, dtype=tdt), dye,
                       torch.tensor(0.37, dtype=tdt), zero.clone(), theta, dye_extra, ctrl)
    meta, arrays = extract(ops, geom)
    arrays.update({"in_u": _np(state.u), "in_v": _np(state.v), "in_t": _np(state.t)})
    if ctrl is not None:
        arrays["in_ctrl"] = _np(ctrl)
    if dye_extra is not None:
        arrays["in_dye_extra"] = _np(dye_extra)
    if dye is not None:
        arrays["in_dye"] = _np(dye)
    if theta is not None:
        arrays["in_theta"] = _np(theta)
    st = state
    with torch.no_grad():
        for k in range(steps):
            rep = {}
            st, coeffs = core.step_full(st, geom, ops, out=rep)
            if k == 0:
                arrays.update({"out1_u": _np(st.u), "out1_v": _np(st.v), "out1_p": _np(st.p), "out1_t": _np(st.t),
                               "out1_dt": _np(st.dt), "out1_coeffs": _np(coeffs)})
                if st.dye is not None:
                    arrays["out1_dye"] = _np(st.dye)
                if st.theta is not None:
                    arrays["out1_theta"] = _np(st.theta)
                for key, val in rep.items():
                    arrays["out1_rep_" + key] = _np(val)
                if st.ctrl is not None:
                    arrays["out1_ctrl"] = _np(st.ctrl)
                if st.dye_extra is not None:
                    arrays["out1_dye_extra"] = _np(st.dye_extra)
    meta["steps"] = steps
    if steps > 1:
        arrays.update({"outN_u": _np(st.u), "outN_v": _np(st.v), "outN_p": _np(st.p), "outN_t": _np(st.t)})
        if st.dye is not None:
            arrays["outN_dye"] = _np(st.dye)
        if st.theta is not None:
            arrays["outN_theta"] = _np(st.theta)
        if st.ctrl is not None:
            arrays["outN_ctrl"] = _np(st.ctrl)
            arrays["outN_dt"] = _np(st.dt)
        if st.dye_extra is not None:
            arrays["outN_dye_extra"] = _np(st.dye_extra)
    store = {k: (np.asarray(x, dtype=np.float32) if dtype == "float32" and np.asarray(x).dtype == np.float64
                 else np.asarray(x)) for k, x in arrays.items()}
    np.savez_compressed(HERE / f"ns2d_{name}.npz", meta=np.array(json.dumps(meta)), **store)
    return meta


def poisson_cases():
    """Seeded right-hand sides and the reference's solutions (Neumann and periodic)."""
    out = {}
    g = torch.Generator().manual_seed(7)
    shapes = [(7, 5), (8, 6), (12, 9), (16, 12), (20, 10), (32, 16)]
    n = 0
    for (nx, ny) in shapes:
        for per in (False, True):
            ps = PoissonSolver(nx, ny, 0.3, periodic=per, device=torch.device("cpu"), dtype=torch.float64)
            f = torch.randn(ny, nx, generator=g, dtype=torch.float64)
            f = f - f.mean()
            out[f"f{n}"] = f.numpy()
            out[f"psi{n}"] = ps.solve(f).numpy()
            out[f"meta{n}"] = np.array([nx, ny, int(per)], dtype=np.int64)
            n += 1
    np.savez_compressed(HERE / "poisson2d.npz", h=np.array(0.3), count=np.array(n), **out)


def main():
    torch.set_num_threads(4)
    names = sys.argv[1:]

    def run_case(name, *a, **kw):
        if not names or name in names:
            _run_case(name, *a, **kw)
    # cylinder in a slip-walled tunnel (the shape of the 2D benchmark, coarser)
    cyl = ImmersedBody(circle(2.0, 2.0, 0.5, 64), name="cylinder")
    tunnel = {"nx": 64, "ny": 32, "h": 1.0 / 8.0, "x0": 0.0, "y0": 0.0, "re": 200.0, "bodies": [cyl],
              "force_ref": 0.5, "moment_ref": (2.0, 2.0), "dye": True}
    run_case("cylinder_upwind_f64", tunnel, dtype="float64", amp=0.05, seed=1, steps=3)
    run_case("cylinder_upwind_f32", tunnel, dtype="float32", amp=0.05, seed=1, steps=3)
    # periodic box, Smagorinsky, a spinning body
    spin = ImmersedBody(square(1.0, 1.2, 0.3), name="spinner", omega=1.5, center=(1.0, 1.2))
    run_case("periodic_smag_spin_f64", {"nx": 32, "ny": 24, "h": 2.5 / 32, "x0": 0.0, "y0": 0.0, "re": 800.0,
                                        "bodies": [spin], "periodic": True, "turbulence": "smagorinsky",
                                        "dye": True, "moment_ref": (1.0, 1.2)},
             dtype="float64", amp=0.3, seed=2)
    # closed cavity: moving bottom, slip left wall, WALE, a body
    block = ImmersedBody(square(1.6, 1.0, 0.25), name="block")
    run_case("closed_wale_f64", {"nx": 40, "ny": 24, "h": 0.1, "x0": 0.0, "y0": 0.0, "re": 2000.0,
                                 "bodies": [block], "domain": "closed", "bc_bottom": "moving", "ground_speed": 1.0,
                                 "bc_left": "slip", "bc_right": "noslip", "bc_top": "noslip",
                                 "turbulence": "wale", "dye": True, "moment_ref": (1.6, 1.0)},
             dtype="float64", amp=0.2, seed=3)
    # no-slip top, moving floor, parabolic inlet, central advection, Vreman, two bodies
    a = ImmersedBody(circle(1.2, 1.1, 0.3, 48), name="a")
    b = ImmersedBody(square(2.3, 1.4, 0.22), name="b")
    run_case("tunnel_two_bodies_vreman_f64", {"nx": 48, "ny": 24, "h": 0.1, "x0": 0.0, "y0": 0.0, "re": 500.0,
                                              "bodies": [a, b], "inlet": "parabolic", "bc_top": "noslip",
                                              "bc_bottom": "moving", "ground_speed": 0.5, "advection": "central",
                                              "turbulence": "vreman", "dye": False, "moment_ref": (1.5, 1.0)},
             dtype="float64", amp=0.05, seed=4)
    # heat transfer: a hot cylinder in a tunnel with buoyancy; a differentially heated cavity
    # with an insulated block, a heat-flux body and WALE; a periodic box with a cold body
    hot = ImmersedBody(circle(2.0, 2.0, 0.5, 64), name="hot", thermal="temperature", thermal_value=1.0)
    heated = dict(tunnel, bodies=[hot], dye=False, thermal=ThermalConfig(prandtl=0.71, richardson=0.5))
    run_case("cylinder_heated_f64", heated, dtype="float64", amp=0.05, seed=5, steps=3)
    run_case("cylinder_heated_f32", heated, dtype="float32", amp=0.05, seed=5, steps=3)
    ins = ImmersedBody(square(1.2, 1.2, 0.3), name="insulated", thermal="adiabatic")
    flux = ImmersedBody(circle(2.8, 1.0, 0.25, 48), name="flux", thermal="heat_flux", thermal_value=0.8)
    cavity = {"nx": 40, "ny": 24, "h": 0.1, "x0": 0.0, "y0": 0.0, "re": 1500.0, "bodies": [ins, flux],
              "domain": "closed", "bc_bottom": "noslip", "bc_left": "noslip", "bc_right": "noslip",
              "bc_top": "noslip", "turbulence": "wale", "dye": False, "moment_ref": (2.0, 1.2),
              "thermal": ThermalConfig(prandtl=0.9, richardson=1.0, gravity=(0.3, -1.0),
                                       walls=[WallBC("left", "temperature", 0.5), WallBC("right", "temperature", -0.5),
                                              WallBC("bottom", "heat_flux", 0.3)])}
    run_case("cavity_heated_wale_f64", cavity, dtype="float64", amp=0.1, seed=6, steps=3)
    cold = ImmersedBody(square(1.0, 1.2, 0.4), name="cold", thermal="temperature", thermal_value=-0.5)
    run_case("periodic_cold_body_f64", {"nx": 32, "ny": 24, "h": 2.5 / 32, "x0": 0.0, "y0": 0.0, "re": 600.0,
                                        "bodies": [cold], "periodic": True, "dye": False, "moment_ref": (1.0, 1.2),
                                        "thermal": ThermalConfig(prandtl=0.71, richardson=0.8)},
             dtype="float64", amp=0.2, seed=7, steps=3)
    # placed physics besides heat: a velocity-regulated fan and a thrust fan with the PID step in
    # the cylinder tunnel (three steps: the controller's first step, then two regulated ones)
    fans = [FanSpec((1.0, 1.2), direction=(1.0, 0.0), width=0.8, mode="velocity", value=1.3, name="reg"),
            FanSpec((5.5, 3.0), direction=(0.6, -0.8), width=0.6, mode="thrust", value=0.4, name="push")]
    fan_case = dict(tunnel, fans=fans, adaptive_dt="pid")
    run_case("tunnel_fans_pid_f64", fan_case, dtype="float64", amp=0.05, seed=8, steps=3)
    run_case("tunnel_fans_pid_f32", fan_case, dtype="float32", amp=0.05, seed=8, steps=3)
    # a heater and a painted obstacle in the heated cavity, with smoke (paint clears it)
    heaters = [HeatSourceSpec((2.8, 1.6), kind="rect", size=(0.4, 0.2), power=0.6, name="strip"),
               HeatSourceSpec((1.0, 0.5), kind="disc", size=(0.2,), power=-0.3, name="cooler")]
    heater_case = dict(cavity, bodies=[ins], heat_sources=heaters, dye=True)

    def block(x, y):
        return torch.maximum((x - 3.2).abs() - 0.25, (y - 0.8).abs() - 0.3)
    run_case("cavity_heater_paint_f64", heater_case, dtype="float64", amp=0.1, seed=9, steps=3, paint=block)
    run_case("cavity_heater_paint_f32", heater_case, dtype="float32", amp=0.1, seed=9, steps=3, paint=block)
    # jets and vents: a warm jet and a vent in the heated tunnel (the outlet balance takes the
    # net port flow); an unbalanced jet in a closed heated box with a painted block (the uniform
    # sink, the combined port / paint penalisation, the paint's force share)
    ports = [PortSpec((0.8, 3.2), direction=(1.0, -0.3), size=0.3, speed=1.5, kind="jet", theta=1.0, name="jet"),
             PortSpec((5.0, 0.7), direction=(0.0, -1.0), size=0.4, speed=0.6, kind="vent", name="vent")]
    port_case = dict(tunnel, bodies=[hot], ports=ports, dye=True, thermal=ThermalConfig(prandtl=0.71, richardson=0.3))
    run_case("tunnel_ports_heat_f64", port_case, dtype="float64", amp=0.05, seed=10, steps=3)
    run_case("tunnel_ports_heat_f32", port_case, dtype="float32", amp=0.05, seed=10, steps=3)
    box_jet = dict(cavity, bodies=[ins], ports=[PortSpec((0.4, 0.5), direction=(1.0, 0.2), size=0.25, speed=1.0,
                                                         kind="jet", theta=0.8, name="jet")], dye=True)
    run_case("closed_jet_paint_f64", box_jet, dtype="float64", amp=0.1, seed=11, steps=3, paint=block)
    # smoke channels: a pulsed rake on channel 0 beside the inlet comb, a line emitter on channel
    # 1 that switches on during the run, a smoking jet on channel 2 and a vent
    emitters = [EmitterSpec((1.0, 1.0), kind="rake", end=(1.0, 3.0), count=6, channel=0, rate=0.8, pulse_period=0.1,
                            pulse_duty=0.5),
                EmitterSpec((3.0, 3.2), kind="line", end=(4.5, 3.4), channel=1, rate=0.6, start=0.38),
                EmitterSpec((5.5, 1.0), kind="disc", size=(0.3,), channel=1, rate=1.0, stop=0.4)]
    smoke_ports = [PortSpec((0.8, 0.8), direction=(1.0, 0.4), size=0.3, speed=1.2, kind="jet", dye_channel=2),
                   PortSpec((6.0, 3.3), direction=(0.0, 1.0), size=0.4, speed=0.5, kind="vent")]
    smoke_case = dict(tunnel, emitters=emitters, ports=smoke_ports, dye=True)
    run_case("tunnel_smoke_channels_f64", smoke_case, dtype="float64", amp=0.05, seed=12, steps=3)
    run_case("tunnel_smoke_channels_f32", smoke_case, dtype="float32", amp=0.05, seed=12, steps=3)
    # the Werner-Wengle wall shear on a coarse closed room (a moving floor, no-slip sides and top)
    room = {"nx": 40, "ny": 24, "h": 0.1, "x0": 0.0, "y0": 0.0, "re": 20000.0,
            "bodies": [ImmersedBody(square(1.6, 1.0, 0.25), name="block")],
            "domain": "closed", "bc_bottom": "moving", "ground_speed": 1.0, "bc_left": "noslip", "bc_right": "noslip",
            "bc_top": "noslip", "turbulence": "wale", "dye": False, "moment_ref": (1.6, 1.0),
            "wall_model": "werner_wengle"}
    run_case("closed_wall_model_f64", room, dtype="float64", amp=0.5, seed=13, steps=3)
    run_case("closed_wall_model_f32", room, dtype="float32", amp=0.5, seed=13, steps=3)
    run_case("periodic_forced_f64", {"nx": 32, "ny": 24, "h": 2.5 / 32, "x0": 0.0, "y0": 0.0, "re": 400.0,
                                     "bodies": [spin], "periodic": True, "dye": False, "moment_ref": (1.0, 1.2)},
             dtype="float64", amp=0.3, seed=14, steps=3, forcing=(0.4, -0.2))
    if not names or "poisson" in names:
        poisson_cases()


if __name__ == "__main__":
    main()
