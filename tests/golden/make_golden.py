"""Generate the golden vectors that pin the oracle to the reference (run in the build container).

Usage (the reference checkout is named by ``AEROLUME_REF``; it is read, never modified)::

    AEROLUME_REF=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py [case ...]

(no case names: every case and the Poisson fixtures).

Each case builds a configuration with the reference's own API (``SolverConfig3D``,
``make_operators3d``, ``build_geometry3d``, ``Physics3D``, ``build_dye_sources``), starts
from a seeded, projected random state (the pattern of the reference's
tests/test_ns3d_core.py:66-72) and runs one step of ``core.step3d_phys`` plus the smoke
update of ``FlowSolver3D._advance_tracers`` (``advect_dye3d`` + ``apply_solids_and_sources``)
on the CPU.  Every input the step reads and every output it returns is written to
``ns3d_<case>.npz`` beside this script; scalar parameters go into a JSON ``meta`` entry.
The fixtures are committed; nothing at test time needs the reference.
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

from aerolume.solvers.ns3d import core  # noqa: E402
from aerolume.solvers.ns3d.config import (DyeRake, Fan3D, HeatSource3D, ImmersedMesh, Port3D,  # noqa: E402
                                          SolverConfig3D, ThermalConfig3D)
from aerolume.solvers.ns3d.dye import advect_dye3d, apply_solids_and_sources, build_dye_sources  # noqa: E402
from aerolume.solvers.ns3d.geometry import body_window3d, build_geometry3d  # noqa: E402
from aerolume.solvers.ns3d.physics import PaintLayer, Physics3D  # noqa: E402
from aerolume.solvers.ns3d.poisson import PoissonSolver3D  # noqa: E402


def _validation_cases():
    """The reference's validation/ns3d_cases.py (mesh helpers), loaded by path as its own
    tests do (tests/test_ns3d_core.py:33-47)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("ns3d_cases", REF / "validation" / "ns3d_cases.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ns3d_cases"] = mod
    spec.loader.exec_module(mod)
    return mod


CASES = _validation_cases()


def box_mesh(lx, ly, lz, center):
    return CASES.box_mesh(lx, ly, lz, center)


def _np(t):
    return None if t is None else t.detach().cpu().numpy().copy()


def _random_state(cfg64, amp, seed):
    """Seeded noise on the reference's initial state, boundary values and an FP64 projection."""
    ops = core.make_operators3d(cfg64)
    s = core.init_state3d(cfg64, ops, perturb=False)
    g = torch.Generator().manual_seed(seed)
    u, v, w = (x + amp * torch.randn(x.shape, generator=g, dtype=torch.float64) for x in (s.u, s.v, s.w))
    u, v, w = core.apply_boundary_values(u, v, w, ops)
    u, v, w, _ = core.project3d(u, v, w, ops)
    theta = 0.3 * torch.randn((cfg64.nz, cfg64.ny, cfg64.nx), generator=g, dtype=torch.float64)
    dye = torch.rand((cfg64.nz, cfg64.ny, cfg64.nx), generator=g, dtype=torch.float64)
    dye[dye < 0.3] = 0.0
    return u, v, w, theta, dye


def extract(ops, geom, phys, src):
    """Everything the step reads, as JSON scalars and numpy arrays."""
    meta = {
        "nx": ops.nx, "ny": ops.ny, "nz": ops.nz, "h": ops.h, "x0": ops.x0, "y0": ops.y0, "z0": ops.z0,
        "periodic_axes": list(ops.periodic_axes), "closed": bool(ops.closed), "symmetry": bool(ops.symmetry),
        "advection": ops.advection, "turbulence": ops.turbulence, "les_c": float(ops.les_c),
        "nu_value": float(ops.nu_value), "eta": float(ops.eta), "cfl": float(ops.cfl),
        "dt_fixed": ops.dt_fixed, "ghost": {k: [list(map(list, ax)) for ax in v] for k, v in ops.ghost.items()},
        "ref_area": ops.ref_area, "length_ref": ops.length_ref, "span_ref": ops.span_ref,
        "moment_ref": list(ops.moment_ref), "window": list(geom.window), "nbody": int(geom.nbody),
        "dtype": "float64" if ops.dtype == torch.float64 else "float32",
        "forcing": list(ops.forcing) if getattr(ops, "forcing", None) is not None else None,
    }
    arrays = {"u_inlet": _np(ops.u_inlet)[..., 0]}
    if not geom.empty:
        for name in ("chi_u", "chi_v", "chi_w", "chi_c", "a_u", "a_v", "a_w", "k_u", "k_v", "k_w"):
            arrays[name] = _np(getattr(geom, name))
    th = phys.thermal if phys is not None else None
    if th is not None:
        tg = th.geom
        meta["thermal"] = {
            "kappa": th.kappa, "pe": th.pe, "ri": th.ri, "prt": th.prt, "eta": float(th.eta),
            "side_kinds": list(th.side_kinds), "side_vals": [float(x) for x in th.side_vals],
            "t_index": list(tg.t_index), "flux_rate": [float(x) for x in tg.flux_rate],
            "heat_max": None if th.heat_max is None else float(th.heat_max),
        }
        for name in ("chi_t", "a_t", "w_t", "vol_w", "skin"):
            val = getattr(tg, name)
            if val is not None:
                arrays["th_" + name] = _np(val)
        if th.sources.items:
            meta["thermal"]["sources"] = [list(win) for win, _ in th.sources.items]
            for q, (_, dens) in enumerate(th.sources.items):
                arrays[f"th_src{q}"] = _np(dens)
        if tg.adia is not None:
            for n, a in zip("uvw", tg.adia):
                arrays["th_adia_" + n] = _np(a)
    if src is not None and not src.empty:
        meta["dye"] = {"window": list(src.window), "pulse": [float(x) for x in src.pulse]}
        arrays["dye_weight"] = _np(src.weight)
    if phys is not None and phys.pid is not None:
        meta["pid"] = {"target": phys.pid.target}
    if phys is not None:
        meta["u_floor"] = float(phys.u_floor)
    if phys is not None and phys.paint is not None:
        for g in "uvwc":
            arrays["paint_" + g] = _np(getattr(phys.paint, "chi_" + g))
    if phys is not None and phys.fans is not None:
        fs = phys.fans
        meta["fans"] = {"any_swirl": bool(fs.any_swirl), "win": [list(it["win"]) for it in fs.items],
                        **{k: [float(x) for x in getattr(fs, k).tolist()]
                           for k in ("target", "kp", "ki", "tmax", "swirl", "thrust")},
                        "velocity_mode": [bool(x) for x in fs.velocity_mode.tolist()]}
        for q, it in enumerate(fs.items):
            for kind in "fsm":
                for g in "uvw":
                    arrays[f"fan{q}_{kind}{g}"] = _np(it[kind + g])
    if phys is not None and phys.ports is not None:
        ps = phys.ports
        meta["ports"] = {"mass_flux": float(ps.mass_flux), "leak": float(ps.leak),
                         "items": [{"win": list(it["win"]), "kind": it["kind"], "theta": float(it["theta"])}
                                   for it in ps.items]}
        for q, it in enumerate(ps.items):
            arrays[f"port{q}_m"] = _np(it["m"])
            for g in "uvw":
                arrays[f"port{q}_f{g}"] = _np(it["f" + g])
    return meta, arrays


def _run_case(name, cfg_kw, *, dtype="float64", amp=0.1, seed=1, rake=None, steps=1, strokes=(), forcing=None):
    """One fixture; ``strokes`` are PaintLayer.stroke keyword sets (painted solids); ``forcing``
    a uniform body force (the verification cases' ``ops.forcing``)."""
    base = dict(cfg_kw)
    cfg64 = SolverConfig3D(**{**base, "dtype": "float64", "device": "cpu", "perturb": False})
    cfg = SolverConfig3D(**{**base, "dtype": dtype, "device": "cpu", "perturb": False})
    ops = core.make_operators3d(cfg)
    if forcing is not None:
        ops.forcing = tuple(forcing)
    window = body_window3d([b.vertices_numpy() for b in cfg.bodies], ops) if cfg.bodies else (0, 0, 0, 0, 0, 0)
    geom = build_geometry3d(cfg.bodies, ops, window=window)
    phys = Physics3D(cfg, ops, geom, cfg.bodies) if cfg.has_placed_physics else None
    if strokes:
        phys.paint = PaintLayer(ops)
        for kw in strokes:
            assert phys.paint.stroke(ops, **kw)
    src = build_dye_sources(rake, ops) if rake is not None else None
    u, v, w, theta, dye = _random_state(cfg64, amp, seed)
    tdt = ops.dtype
    state = core.State3D(u.to(tdt), v.to(tdt), w.to(tdt), torch.zeros(cfg.nz, cfg.ny, cfg.nx, dtype=tdt),
                         torch.tensor(0.37, dtype=tdt), torch.zeros((), dtype=tdt))
    th0 = theta.to(tdt) if (phys is not None and phys.thermal is not None) else None
    c0 = dye.to(tdt)
    meta, arrays = extract(ops, geom, phys, src)
    arrays.update({"in_u": _np(state.u), "in_v": _np(state.v), "in_w": _np(state.w), "in_t": _np(state.t),
                   "in_dye": _np(c0)})
    if th0 is not None:
        arrays["in_theta"] = _np(th0)
    st, th, c = state, th0, c0
    with torch.no_grad():
        for k in range(steps):
            out = core.step3d_phys(st, geom, ops, phys=phys, theta=th)
            new = out.state
            c = advect_dye3d(c, new.u, new.v, new.w, new.dt, ops)
            apply_solids_and_sources(c, new.t, geom, src)
            if phys is not None and phys.paint is not None:   # FlowSolver3D._solid_cleanup
                c.masked_fill_(phys.paint.chi_c > 0.5, 0.0)
            st, th = new, out.theta
            if phys is not None and phys.pid is not None:
                arrays[f"pid{k + 1}"] = np.array([float(phys.pid.dt_prev), float(phys.pid.e1), float(phys.pid.e2)])
            if phys is not None and phys.fans is not None:   # thrust, ud, e_prev, swirl_amp after the step
                f = phys.fans
                arrays[f"fans{k + 1}"] = np.stack([_np(x).astype(np.float64) for x in (f.thrust, f.ud, f.e_prev,
                                                                                       f.swirl_amp)])
            if k == 0:
                arrays.update({"out1_u": _np(new.u), "out1_v": _np(new.v), "out1_w": _np(new.w),
                               "out1_p": _np(new.p), "out1_t": _np(new.t), "out1_dt": _np(new.dt),
                               "out1_coeffs": _np(out.coeffs), "out1_dye": _np(c)})
                if th is not None:
                    arrays["out1_theta"] = _np(th)
                    arrays["out1_heat_rate"] = _np(phys.thermal.heat_rate)
    meta["steps"] = steps
    if steps > 1:
        arrays.update({"outN_u": _np(st.u), "outN_v": _np(st.v), "outN_w": _np(st.w), "outN_p": _np(st.p),
                       "outN_t": _np(st.t), "outN_dye": _np(c)})
        if th is not None:
            arrays["outN_theta"] = _np(th)
    store = {k: (np.asarray(v, dtype=np.float32) if dtype == "float32" and np.asarray(v).dtype == np.float64
                 else np.asarray(v)) for k, v in arrays.items()}
    np.savez_compressed(HERE / f"ns3d_{name}.npz", meta=np.array(json.dumps(meta)), **store)
    return meta


def poisson_cases():
    """Seeded right-hand sides and the reference's solutions for odd shapes and every BC mix
    (the shapes and mixes of the reference's tests/test_ns3d_core.py:79-91)."""
    out = {}
    g = torch.Generator().manual_seed(5)
    shapes = [(7, 6, 5), (8, 6, 5), (9, 5, 6), (12, 8, 6), (16, 12, 10)]
    mixes = [(False, False, False), (True, True, True), (False, True, False), (True, False, True)]
    for n, ((nx, ny, nz), per) in enumerate((s, p) for s in shapes for p in mixes):
        ps = PoissonSolver3D(nx, ny, nz, 0.3, periodic=per, device=torch.device("cpu"), dtype=torch.float64)
        f = torch.randn(nz, ny, nx, generator=g, dtype=torch.float64)
        f = f - f.mean()
        out[f"f{n}"] = f.numpy()
        out[f"psi{n}"] = ps.solve(f).numpy()
        out[f"meta{n}"] = np.array([nx, ny, nz, *per], dtype=np.int64)
    np.savez_compressed(HERE / "poisson3d.npz", h=np.array(0.3), count=np.array(len(shapes) * len(mixes)), **out)


def main():
    torch.set_num_threads(4)
    names = sys.argv[1:]

    def run_case(name, *a, **kw):
        if not names or name in names:
            _run_case(name, *a, **kw)
    h = 1.0 / 6.0
    box = ImmersedMesh(*box_mesh(0.5, 0.5, 0.25, (1.25, 1.0, 0.125)), name="box", thermal="temperature",
                       thermal_value=1.0)
    rake = DyeRake("rake", [(0.5, 0.6, 0.2), (0.5, 0.9, 0.25), (0.5, 1.2, 0.3), (0.5, 1.45, 0.5)], radius=1.25 * h)
    grid = {"nx": 24, "ny": 12, "nz": 10, "h": h, "x0": 0.0, "y0": 0.0, "z0": 0.0}
    tunnel = dict(grid, re=1e4, bodies=[box], bc_zmin="moving", ground_speed=1.0, turbulence="wale",
                  thermal=ThermalConfig3D(prandtl=0.71, richardson=0.2), ref_area=0.125, moment_ref=(1.25, 1.0, 0.0))
    run_case("tunnel_wale_heat_smoke_f64", tunnel, dtype="float64", rake=rake, steps=3)
    run_case("tunnel_wale_heat_smoke_f32", tunnel, dtype="float32", rake=rake, steps=3)
    # the same physics on a grid that the stage kernel splits into two z-chunks of 16 planes
    # and whose middle x-y tile (i0 = 32, j0 = 8) touches no domain side: 72 x 24 x 32, h = 1/8,
    # a 1 x 1 x 0.5 box on the moving floor, WALE, heat, a four-nozzle rake
    hm = 1.0 / 8.0
    mid_box = ImmersedMesh(*box_mesh(1.0, 1.0, 0.5, (2.5, 1.5, 0.25)), name="box", thermal="temperature",
                           thermal_value=1.0)
    mid_rake = DyeRake("rake", [(1.25, 0.9, 0.15), (1.25, 1.3, 0.3), (1.25, 1.7, 0.2), (1.25, 2.1, 0.4)],
                       radius=1.25 * hm)
    mid = {"nx": 72, "ny": 24, "nz": 32, "h": hm, "x0": 0.0, "y0": 0.0, "z0": 0.0, "re": 1e4, "bodies": [mid_box],
           "bc_zmin": "moving", "ground_speed": 1.0, "turbulence": "wale",
           "thermal": ThermalConfig3D(prandtl=0.71, richardson=0.2), "ref_area": 0.5, "moment_ref": (2.5, 1.5, 0.0)}
    run_case("tunnel_mid_f64", mid, dtype="float64", rake=mid_rake, seed=16, amp=0.05)
    run_case("tunnel_mid_f32", mid, dtype="float32", rake=mid_rake, seed=16, amp=0.05)

    adia = ImmersedMesh(*box_mesh(0.5, 0.5, 0.5, (1.25, 0.0, 0.75)), name="adia")
    sym = dict(grid, y0=0.0, re=5e3, bodies=[adia], bc_y="symmetry_ymin", bc_zmax="noslip", turbulence="smagorinsky",
               thermal=ThermalConfig3D(prandtl=0.9, richardson=0.5,
                                       walls={"bottom": ("temperature", 0.5), "top": ("heat_flux", 0.2)}),
               ref_area=0.25, moment_ref=(1.0, 0.0, 0.5))
    run_case("symmetry_smag_adiabatic_f64", sym, dtype="float64", seed=2, amp=0.2)

    per = {"nx": 12, "ny": 10, "nz": 8, "h": 2 * math.pi / 12, "x0": 0.0, "y0": 0.0, "z0": 0.0}
    run_case("periodic_vreman_f64", dict(per, re=2e3, periodic=True, turbulence="vreman",
                                         thermal=ThermalConfig3D(prandtl=0.71, richardson=1.0)),
             dtype="float64", seed=3, amp=0.5)
    # a uniform body force (the verification cases' forcing) in the periodic box
    run_case("periodic_forced_f64", dict(per, re=500.0, periodic=True), dtype="float64", seed=14, amp=0.5,
             forcing=(0.3, -0.1, 0.05))

    closed = dict(grid, nx=14, ny=10, nz=10, re=300.0, domain="closed", bc_x="noslip", bc_y="noslip",
                  bc_zmin="noslip", bc_zmax="noslip", advection="central",
                  thermal=ThermalConfig3D(prandtl=0.71, richardson=2.0,
                                          walls={"left": ("temperature", 1.0), "right": ("temperature", -1.0)}))
    run_case("closed_central_cavity_f64", closed, dtype="float64", seed=4, amp=0.2)

    flux_a = ImmersedMesh(*box_mesh(0.5, 0.5, 0.5, (1.0, 1.0, 0.8)), name="hot", thermal="heat_flux",
                          thermal_value=2.0)
    flux_b = ImmersedMesh(*box_mesh(0.34, 0.34, 0.34, (2.1, 1.0, 0.8)), name="cold", thermal="temperature",
                          thermal_value=-0.5, omega=1.5, center=(2.1, 1.0, 0.8), axis=(0.0, 1.0, 0.0))
    yper = dict(grid, re=800.0, bodies=[flux_a, flux_b], bc_y="periodic", bc_zmin="noslip",
                thermal=ThermalConfig3D(prandtl=1.0, richardson=0.3), ref_area=0.3, moment_ref=(1.5, 1.0, 0.8),
                length_ref=0.5, span_ref=0.5)
    run_case("yperiodic_two_bodies_heatflux_f64", yper, dtype="float64", seed=6, amp=0.1)
    run_case("plain_upwind_f64", dict(grid, re=200.0, bodies=[ImmersedMesh(*box_mesh(0.5, 0.5, 0.5, (1.2, 1.0, 0.8)))],
                                      ref_area=0.25), dtype="float64", seed=7, amp=0.1)
    # painted solids (a ball and a box, one of them across the body window) and the PID step
    # controller, over three steps so that the controller runs past its first step
    strokes = (dict(center=(2.6, 1.0, 0.6), radius=0.35), dict(center=(1.6, 1.3, 0.4), radius=0.2, shape="box",
                                                               size=(0.3, 0.4, 0.5)))
    paint_pid = dict(tunnel, adaptive_dt="pid", pid_target=0.7)
    run_case("tunnel_paint_pid_f64", paint_pid, dtype="float64", rake=rake, steps=3, strokes=strokes, seed=8)
    run_case("tunnel_paint_pid_f32", paint_pid, dtype="float32", rake=rake, steps=3, strokes=strokes, seed=8)
    plain_pid = dict(grid, re=500.0, adaptive_dt="pid", pid_target=0.9)
    run_case("plain_pid_paint_f64", plain_pid, dtype="float64", steps=3, seed=9, amp=0.3,
             strokes=(dict(center=(2.0, 1.0, 0.8), radius=0.4),))
    # two fans: a velocity-regulated one with swirl and a fixed-thrust one at an angle, three
    # steps so that the PI controller acts on its own output
    fans = [Fan3D(center=(1.1, 1.0, 0.85), direction=(1.0, 0.0, 0.0), diameter=0.9, mode="velocity", value=1.4,
                  swirl=0.5, name="a"),
            Fan3D(center=(2.7, 1.1, 0.8), direction=(0.6, 0.8, 0.0), diameter=0.7, mode="thrust", value=0.08, name="b")]
    fan_case = dict(grid, re=600.0, fans=fans, turbulence="wale")
    run_case("fans_swirl_f64", fan_case, dtype="float64", steps=3, seed=10, amp=0.1)
    run_case("fans_swirl_f32", fan_case, dtype="float32", steps=3, seed=10, amp=0.1)
    closed_fan = dict(grid, nx=14, ny=10, nz=10, re=300.0, domain="closed", bc_x="noslip", bc_y="noslip",
                      bc_zmin="noslip", bc_zmax="noslip",
                      fans=[Fan3D(center=(1.2, 0.8, 0.8), direction=(0.0, 0.0, 1.0), diameter=0.8,
                                  mode="pressure_jump", value=0.3, name="up")])
    run_case("closed_fan_pressure_f64", closed_fan, dtype="float64", steps=3, seed=11, amp=0.05)
    # jets and vents: a warm jet up from the floor and a vent downstream in the heated tunnel,
    # and an unbalanced jet in a closed heated box (its uniform leak carries heat out)
    ports = [Port3D(kind="jet", center=(1.0, 1.0, 0.35), direction=(0.0, 0.0, 1.0), diameter=0.6, speed=0.8,
                    theta=0.7, name="jet"),
             Port3D(kind="vent", center=(3.0, 0.9, 0.9), diameter=0.5, speed=0.5, name="vent")]
    port_case = dict(grid, re=800.0, ports=ports, turbulence="wale",
                     thermal=ThermalConfig3D(prandtl=0.71, richardson=0.2))
    run_case("ports_heat_f64", port_case, dtype="float64", steps=3, seed=12, amp=0.1)
    run_case("ports_heat_f32", port_case, dtype="float32", steps=3, seed=12, amp=0.1)
    closed_jet = dict(grid, nx=14, ny=10, nz=10, re=300.0, domain="closed", bc_x="noslip", bc_y="noslip",
                      bc_zmin="noslip", bc_zmax="noslip",
                      ports=[Port3D(kind="jet", center=(1.1, 0.8, 0.5), direction=(0.6, 0.0, 0.8), diameter=0.5,
                                    speed=0.6, theta=1.0, name="inflow")],
                      thermal=ThermalConfig3D(prandtl=0.71, richardson=0.5))
    run_case("closed_jet_leak_f64", closed_jet, dtype="float64", steps=3, seed=13, amp=0.05)
    # volumetric heaters: a box heater behind the heated body and a cooling ball in the tunnel,
    # and a box heater warming a still closed box (the heaters' step limit sets dt)
    heaters = [HeatSource3D(kind="box", center=(2.2, 1.0, 0.3), size=(0.5, 0.4, 0.3), power=2.0, name="heater"),
               HeatSource3D(kind="sphere", center=(3.0, 0.8, 0.9), size=(0.3, 0.3, 0.3), power=-1.5, name="cooler")]
    run_case("tunnel_heaters_f64", dict(tunnel, heat_sources=heaters), dtype="float64", steps=3, seed=14, amp=0.1)
    run_case("tunnel_heaters_f32", dict(tunnel, heat_sources=heaters), dtype="float32", steps=3, seed=14, amp=0.1)
    still = dict(grid, nx=14, ny=10, nz=10, re=300.0, domain="closed", bc_x="noslip", bc_y="noslip",
                 bc_zmin="noslip", bc_zmax="noslip", thermal=ThermalConfig3D(prandtl=0.71, richardson=1.0),
                 heat_sources=[HeatSource3D(kind="box", center=(1.2, 0.8, 0.4), size=(0.5, 0.5, 0.3), power=300.0)])
    run_case("closed_heater_still_f64", still, dtype="float64", steps=3, seed=15, amp=1e-4)
    if not names or "poisson" in names:
        poisson_cases()
    for p in sorted(HERE.glob("*.npz")):
        print(f"{p.name}: {p.stat().st_size / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
