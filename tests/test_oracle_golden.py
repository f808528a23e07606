"""The oracle against the reference's own outputs (golden vectors made by tests/golden/make_golden.py)."""
from __future__ import annotations

import numpy as np
import pytest

from _golden import CASES_3D, GOLDEN, fan_items, load_case, port_items
from oracle import ns3d as O


def _run(name, steps=1):
    meta, ops, geom, th, src, arr = load_case(name)
    dt = np.float64 if meta["dtype"] == "float64" else np.float32
    ps = O.PoissonSolver3D(ops.nx, ops.ny, ops.nz, ops.h, ops.periodic_axes, dt)
    u, v, w, t = arr["in_u"], arr["in_v"], arr["in_w"], dt(arr["in_t"])
    theta = arr.get("in_theta")
    c = arr["in_dye"]
    paint = tuple(arr["paint_" + g] for g in "uvw") if "paint_u" in arr else None
    pid = O.PidState(meta["pid"]["target"], dt) if "pid" in meta else None
    fans = None
    if "fans" in meta:
        fm = meta["fans"]
        items = [{"win": it["win"], "f": tuple(it["f" + g] for g in "uvw"), "s": tuple(it["s" + g] for g in "uvw"),
                  "m": tuple(it["m" + g] for g in "uvw")} for it in fan_items(meta, arr)]
        fans = O.FanState(items, fm["target"], fm["kp"], fm["ki"], fm["tmax"], fm["velocity_mode"], fm["swirl"],
                          fm["any_swirl"], fm["thrust"], dt)
    ports = None
    if "ports" in meta:
        items = [dict(it, f=tuple(it["f" + g] for g in "uvw")) for it in port_items(meta, arr)]
        ports = O.PortState(items, meta["ports"]["mass_flux"], meta["ports"]["leak"])
    outs = []
    for _ in range(steps):
        r = O.step3d_phys(u, v, w, t, geom, ops, ps, th=th, theta=theta, paint=paint, pid=pid,
                          u_floor=meta.get("u_floor", 0.0), fans=fans, ports=ports)
        c = O.advect_dye3d(c, r.u, r.v, r.w, r.dt, ops)
        c = O.apply_solids_and_sources(c, r.t, geom, src)
        if "paint_c" in arr:                         # painted cells hold no smoke
            c = np.where(arr["paint_c"] > 0.5, c.dtype.type(0.0), c)
        u, v, w, t, theta = r.u, r.v, r.w, r.t, r.theta
        r.dye = c
        r.pid = None if pid is None else np.array([float(pid.dt_prev), float(pid.e1), float(pid.e2)])
        r.fans = None if fans is None else np.stack([fans.thrust, fans.ud, fans.e_prev, fans.swirl_amp]).astype(np.float64)
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


@pytest.mark.parametrize("name", [n for n in CASES_3D if ("tunnel" in n or "pid" in n or "fan" in n or "port" in n
                                                           or "jet" in n) and "mid" not in n])
def test_oracle_matches_reference_three_steps(name):
    meta, arr, outs = _run(name, steps=3)
    r = outs[-1]
    tol = 1e-11 if meta["dtype"] == "float64" else 1e-4
    for f in ("u", "v", "w", "p", "theta"):
        if "outN_" + f in arr:
            assert _rel(getattr(r, f), arr["outN_" + f]) < tol, f
    assert _rel(r.dye, arr["outN_dye"]) < tol
    if "pid" in meta:  # the controller's state after every step: dt_prev, e1, e2
        for k, rk in enumerate(outs):
            ref = arr[f"pid{k + 1}"]
            assert np.abs(rk.pid - ref).max() <= (1e-12 if meta["dtype"] == "float64" else 1e-5) * max(1.0, np.abs(ref).max()), k
    if "fans" in meta:  # thrust, disc velocity, PI error, swirl amplitude after every step
        for k, rk in enumerate(outs):
            ref = arr[f"fans{k + 1}"]
            assert np.abs(rk.fans - ref).max() <= (1e-11 if meta["dtype"] == "float64" else 1e-5) * max(1.0, np.abs(ref).max()), k


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


def test_paint_and_pid_fixtures_exercise_both():
    """Leaving out the painted solids, or the controller, moves the step far outside the
    tolerances above: the fixtures pin both features, not a step they do not touch."""
    meta, ops, geom, th, src, arr = load_case("tunnel_paint_pid_f64")
    ps = O.PoissonSolver3D(ops.nx, ops.ny, ops.nz, ops.h, ops.periodic_axes, np.float64)
    paint = tuple(arr["paint_" + g] for g in "uvw")
    args = (arr["in_u"], arr["in_v"], arr["in_w"], np.float64(arr["in_t"]), geom, ops, ps)
    kw = dict(th=th, theta=arr["in_theta"])
    no_paint = O.step3d_phys(*args, **kw, pid=O.PidState(meta["pid"]["target"], np.float64))
    assert _rel(no_paint.u, arr["out1_u"]) > 1e-4
    no_pid = O.step3d_phys(*args, **kw, paint=paint)
    assert abs(float(no_pid.dt) - float(arr["out1_dt"])) > 1e-3 * float(arr["out1_dt"])


def test_fan_fixtures_exercise_the_fans():
    """The fans move the flow and the controller moves the thrust: leaving them out, or
    freezing the thrust, is far outside the tolerances."""
    meta, ops, geom, th, src, arr = load_case("fans_swirl_f64")
    ps = O.PoissonSolver3D(ops.nx, ops.ny, ops.nz, ops.h, ops.periodic_axes, np.float64)
    r = O.step3d_phys(arr["in_u"], arr["in_v"], arr["in_w"], np.float64(arr["in_t"]), geom, ops, ps,
                      u_floor=meta["u_floor"])
    assert _rel(r.u, arr["out1_u"]) > 1e-3
    thrust = arr["fans3"][0]
    assert abs(thrust[0] - meta["fans"]["thrust"][0]) > 1e-3 * abs(meta["fans"]["thrust"][0])  # regulated
    assert thrust[1] == meta["fans"]["thrust"][1]                                             # fixed


def test_port_fixtures_exercise_the_ports():
    """Leaving the jets and vents out moves the step far outside the tolerances, and the
    closed box's jet is unbalanced (its leak term is live)."""
    meta, ops, geom, th, src, arr = load_case("ports_heat_f64")
    ps = O.PoissonSolver3D(ops.nx, ops.ny, ops.nz, ops.h, ops.periodic_axes, np.float64)
    r = O.step3d_phys(arr["in_u"], arr["in_v"], arr["in_w"], np.float64(arr["in_t"]), geom, ops, ps, th=th,
                      theta=arr["in_theta"], u_floor=meta["u_floor"])
    assert _rel(r.u, arr["out1_u"]) > 1e-3
    assert _rel(r.theta, arr["out1_theta"]) > 1e-4
    meta, *_ = load_case("closed_jet_leak_f64")
    assert meta["ports"]["leak"] > 0


def test_heater_fixtures_exercise_the_heaters():
    """Leaving the volumetric heaters out moves theta well outside the tolerances, and in the
    still closed box the heaters' step limit sets dt (the CFL and diffusion limits are looser)."""
    import dataclasses
    meta, ops, geom, th, src, arr = load_case("tunnel_heaters_f64")
    ps = O.PoissonSolver3D(ops.nx, ops.ny, ops.nz, ops.h, ops.periodic_axes, np.float64)
    r = O.step3d_phys(arr["in_u"], arr["in_v"], arr["in_w"], np.float64(arr["in_t"]), geom, ops, ps,
                      th=dataclasses.replace(th, sources=()), theta=arr["in_theta"])
    assert len(th.sources) == 2
    assert _rel(r.theta, arr["out1_theta"]) > 1e-4          # 2e-4: far above 1e-10 (FP64), 1e-5 (FP32)
    meta, ops, geom, th, src, arr = load_case("closed_heater_still_f64")
    ps = O.PoissonSolver3D(ops.nx, ops.ny, ops.nz, ops.h, ops.periodic_axes, np.float64)
    r = O.step3d_phys(arr["in_u"], arr["in_v"], arr["in_w"], np.float64(arr["in_t"]), geom, ops, ps,
                      th=dataclasses.replace(th, heat_max=None, sources=()), theta=arr["in_theta"])
    assert float(r.dt) > 1.5 * float(arr["out1_dt"])
