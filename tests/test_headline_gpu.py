"""Parity at the sizes and on the code paths the benchmarks run.

The golden cases are small (up to 24 x 12 x 10 besides the 72 x 24 x 32 mid-size tunnel), so
these tests hold the CUDA step to the oracle on the benchmark grids themselves:

* the headline workload, the box on a moving floor at 256 x 128 x 128 FP32 (WALE, heat, smoke),
  one step and three chained in-place steps: seven z-chunks of the stage kernel and interior
  x-y tiles that skip the ghost fill;
* the same builders at 80 x 40 x 40 in FP64 and FP32 (two z-chunks, interior tiles);
* one step of each grid of the batched 2D sweep (384 x 192 ... 1024 x 512, the radix-3 transform
  path among them) against the 2D oracle, and the sweep's persistent schedules (grid barrier,
  per-instance counters, work queue) and its multi-stream schedule against the plain
  per-instance loop (bit-identical).
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest
import torch

from oracle import ns2d as O2
from oracle import ns3d as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.detach().double().cpu().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _geom_np(geom, npd):
    from aerolume_b200.ns3d.types import Geometry3D
    g = Geometry3D(geom.window, nbody=geom.nbody)
    for n in ("chi_u", "chi_v", "chi_w", "chi_c", "a_u", "a_v", "a_w", "k_u", "k_v", "k_w"):
        setattr(g, n, np.asarray(getattr(geom, n), npd))
    return g


def _box_case(nx, ny, nz, dtype, seed):
    """Plan, projected seeded state, theta, dye of the box-on-moving-floor builders."""
    from aerolume_b200.ns3d.plan import Ns3dPlan
    from aerolume_b200.ns3d.workloads import box_on_moving_floor, initial_state
    ops, geom, th, src, _ = box_on_moving_floor(nx, ny, nz, dtype=dtype, seed=seed)
    plan = Ns3dPlan(ops, geom, th, src, smoke=True)
    u, v, w = initial_state(ops, seed=seed, noise=0.05)
    plan.project(u, v, w)
    g = torch.Generator().manual_seed(seed + 1)
    theta = (0.2 * torch.randn(nz, ny, nx, generator=g, dtype=torch.float64)).to("cuda", u.dtype)
    dye = torch.rand(nz, ny, nx, generator=g, dtype=torch.float64).to("cuda", u.dtype)
    return ops, geom, th, src, plan, (u, v, w, theta, dye)


def _oracle_steps(ops, geom, th, src, state, steps, npd):
    """``steps`` oracle steps (with the smoke update) from the given device state."""
    c = lambda x: x.detach().cpu().numpy()   # noqa: E731
    u, v, w, theta, dye = (c(x) for x in state)
    t = npd(0.0)
    gnp = _geom_np(geom, npd)
    ps = O.PoissonSolver3D(ops.nx, ops.ny, ops.nz, ops.h, ops.periodic_axes, npd)
    outs = []
    for _ in range(steps):
        r = O.step3d_phys(u, v, w, t, gnp, ops, ps, th=th, theta=theta)
        dye = O.apply_solids_and_sources(O.advect_dye3d(dye, r.u, r.v, r.w, r.dt, ops), r.t, gnp, src)
        u, v, w, theta, t = r.u, r.v, r.w, r.theta, r.t
        outs.append((r, dye))
    return outs


def _np(a):
    return a.detach().double().cpu().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)


def _scales(r, dye_ref):
    """Velocity errors are measured against the flow's speed scale (max |u|, the stream), the
    other fields against their own max norm."""
    U = max(np.abs(_np(r.u)).max(), np.abs(_np(r.v)).max(), np.abs(_np(r.w)).max())
    return {"u": U, "v": U, "w": U, "p": np.abs(_np(r.p)).max(), "theta": np.abs(_np(r.theta)).max(),
            "dye": np.abs(_np(dye_ref)).max()}


def _check(out, r, dye_ref, tol, coeff_tol, tag):
    sc = _scales(r, dye_ref)
    for f, ref in (("u", r.u), ("v", r.v), ("w", r.w), ("p", r.p), ("theta", r.theta), ("dye", dye_ref)):
        err = np.abs(_np(out[f]) - _np(ref)).max() / max(sc[f], 1e-30)
        assert err < tol, (tag, f, err)
    assert _rel(out["dt"], r.dt) < tol, tag
    got = out["coeffs"].double().cpu().numpy()
    assert np.abs(got - r.coeffs).max() <= coeff_tol * max(1.0, np.abs(r.coeffs).max()), (tag, got, r.coeffs)
    hr = out["heat_rate"].double().cpu().numpy()
    assert np.abs(hr - r.heat_rate).max() <= coeff_tol * max(1.0, np.abs(r.heat_rate).max()), (tag, hr, r.heat_rate)


def _check_fp32_level(out, r32, dye32, r64, dye64, tag):
    """Against the FP64 oracle step from the same inputs, the CUDA FP32 step is as close as the
    oracle's own FP32 step (twice its error, or 2e-6 of the scale, whichever is larger)."""
    sc = _scales(r64, dye64)
    for f, a32, a64 in (("u", r32.u, r64.u), ("v", r32.v, r64.v), ("w", r32.w, r64.w), ("p", r32.p, r64.p),
                        ("theta", r32.theta, r64.theta), ("dye", dye32, dye64)):
        e_cuda = np.abs(_np(out[f]) - _np(a64)).max() / max(sc[f], 1e-30)
        e_o32 = np.abs(_np(a32) - _np(a64)).max() / max(sc[f], 1e-30)
        assert e_cuda <= max(2.0 * e_o32, 2e-6), (tag, f, e_cuda, e_o32)


def _chained(plan, state, steps):
    """``steps`` steps updating u, v, w, theta in place (the solver's static buffers)."""
    u, v, w, theta, dye = (x.clone() for x in state)
    t = torch.zeros((), device="cuda", dtype=u.dtype)
    out = plan.empty_fields()
    res = []
    for _ in range(steps):
        out["u"], out["v"], out["w"], out["theta"] = u, v, w, theta
        r = plan.step(u, v, w, t, theta0=theta, dye0=dye, out=out)
        t = r["t"].clone()
        dye = r["dye"].clone()
        res.append({k: (x.clone() if torch.is_tensor(x) else x) for k, x in r.items()})
    torch.cuda.synchronize()
    return res


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_box_case_80x40x40_two_chunks_and_interior_tiles(dtype):
    """80 x 40 x 40: two 20-plane z-chunks of the stage kernel (the plane ring restarts and the
    z-carries begin again at the chunk boundary), x tiles 0, 32, 64 and y tiles 0..32 of which
    the inner ones skip the ghost fill.  One step and three chained steps against the oracle."""
    npd = np.float64 if dtype == "float64" else np.float32
    tol = 1e-10 if dtype == "float64" else 1e-5
    ctol = 1e-9 if dtype == "float64" else 2e-4
    ops, geom, th, src, plan, state = _box_case(80, 40, 40, dtype, seed=5)
    res = _chained(plan, state, 3)
    refs = _oracle_steps(ops, geom, th, src, state, 3, npd)
    _check(res[0], refs[0][0], refs[0][1], tol, ctol, "step 1")
    _check(res[2], refs[2][0], refs[2][1], 10 * tol, 10 * ctol, "step 3")
    assert plan.status() == 0


def test_headline_box_case_256x128x128_matches_oracle():
    """The benchmark workload itself, 256 x 128 x 128 FP32: one step within 1e-5 of max |field|
    of the oracle's FP32 step (the per-step tolerance of the FP32 reference), and after three
    chained in-place steps within 1e-4 (FP32 rounding of two different summation orders
    compounds over the steps)."""
    ops, geom, th, src, plan, state = _box_case(256, 128, 128, "float32", seed=0)
    res = _chained(plan, state, 3)
    refs = _oracle_steps(ops, geom, th, src, state, 3, np.float32)
    _check(res[0], refs[0][0], refs[0][1], 1e-5, 2e-4, "step 1")
    _check(res[2], refs[2][0], refs[2][1], 1e-4, 2e-3, "step 3")
    # the same first step of the oracle in FP64 (from the same FP32 inputs, WALE, heat, smoke)
    ops64 = dataclasses.replace(ops, dtype="float64")
    th64 = dataclasses.replace(th)
    st64 = tuple(x.double() for x in state)
    r64, d64 = _oracle_steps(ops64, geom, th64, src, st64, 1, np.float64)[0]
    _check_fp32_level(res[0], refs[0][0], refs[0][1], r64, d64, "step 1 vs FP64")
    assert plan.status() == 0


def _sweep_by_grid():
    from aerolume_b200.ns2d.workloads import sweep_instances
    first = {}
    for ops, geom, prm in sweep_instances(64, seed=0):
        first.setdefault((ops.nx, ops.ny), (ops, geom, prm))
    return first


@pytest.mark.parametrize("grid", [(256, 128), (384, 192), (512, 256), (768, 384), (1024, 512)])
def test_sweep_grid_step_matches_oracle(grid):
    """The first sweep instance of each grid size: one FP32 step against the 2D oracle's FP32
    step from the same projected state (384 and 768 take the radix-3 transform path)."""
    from aerolume_b200.ns2d.plan import Ns2dPlan
    from aerolume_b200.ns2d.workloads import initial_state
    inst = _sweep_by_grid()
    if grid not in inst:
        pytest.skip(f"no sweep instance on {grid}")
    ops, geom, prm = inst[grid]
    plan = Ns2dPlan(ops, geom)
    u, v = initial_state(ops, plan, seed=11, noise=1e-2)
    t0 = torch.zeros((), device="cuda", dtype=u.dtype)
    out = plan.step(u, v, t0)
    torch.cuda.synchronize()
    ps = O2.PoissonSolver2D(ops.nx, ops.ny, ops.h, ops.periodic, np.float32)
    r = O2.step2d(u.cpu().numpy(), v.cpu().numpy(), np.float32(0.0), geom, ops, ps)
    ops64 = dataclasses.replace(ops, dtype="float64")
    ps64 = O2.PoissonSolver2D(ops.nx, ops.ny, ops.h, ops.periodic, np.float64)
    g64 = dataclasses.replace(geom)
    for n in ("chi_u", "chi_v", "chi_c", "a_u", "a_v", "k_u", "k_v"):
        setattr(g64, n, np.asarray(getattr(geom, n), np.float64))
    r64 = O2.step2d(_np(u), _np(v), np.float64(0.0), g64, ops64, ps64)
    U = max(np.abs(r.u).max(), np.abs(r.v).max())
    for f, ref, ref64, sc in (("u", r.u, r64.u, U), ("v", r.v, r64.v, U), ("p", r.p, r64.p, np.abs(r.p).max())):
        err = np.abs(_np(out[f]) - ref).max() / sc
        assert err < 1e-5, (grid, f, err)
        e_cuda, e_o32 = np.abs(_np(out[f]) - ref64).max() / sc, np.abs(ref - ref64).max() / sc
        assert e_cuda <= max(2.0 * e_o32, 2e-6), (grid, f, e_cuda, e_o32)
    assert _rel(out["dt"], r.dt) < 1e-6
    got = out["coeffs"].double().cpu().numpy()
    assert np.abs(got - r.coeffs).max() <= 1e-4 * max(1.0, np.abs(r.coeffs).max()), (got, r.coeffs)


def _run(sw, snap, schedule, steps, graph):
    sw.restore(snap)
    if graph:
        g = sw.capture(steps, schedule)
        g.replay()
    else:
        for _ in range(steps):
            sw.step(schedule)
    torch.cuda.synchronize()
    return [(s["u"].clone(), s["v"].clone(), s["t"].clone(), s["out"]["coeffs"].clone()) for s in sw.states]


def test_sweep_schedules_equal_the_per_instance_loop():
    """The batched sweep (64 seeded NACA instances on five grid sizes) as one persistent launch
    per step -- with a grid barrier per phase, with per-instance counters of finished items
    (items dealt round robin, or taken from a queue), and the shape the autotuner picks, in and
    out of a CUDA graph -- and spread over 16 streams give every instance exactly what its own
    plan gives when the instances are stepped one after another: fields, time and coefficients
    bit for bit after five steps."""
    from aerolume_b200.ns2d.sweep import Sweep2D
    from aerolume_b200.ns2d.workloads import sweep_instances
    sw = Sweep2D(sweep_instances(64, seed=0))
    snap = sw.snapshot()
    ref = _run(sw, snap, "loop", 5, graph=False)

    def check(schedule, graph, tag):
        got = _run(sw, snap, schedule, 5, graph)
        for k, (a, b) in enumerate(zip(got, ref)):
            for x, y in zip(a, b):
                assert torch.equal(x, y), (tag, graph, k)
        if schedule == "persistent":
            assert sw.status() == 0, tag

    for cand in ((2, 2, 1, "barrier", 1), (3, 3, 0, "counters", 2), (2, 4, 1, "queue", 4)):
        sw.use_persistent(*cand)
        check("persistent", True, cand)
    table = sw.tune(candidates=[(3, 2, 1, "barrier", 2), (2, 2, 1, "counters", 1), (3, 1, 0, "queue", 4)], steps=2)
    assert sw.tuning is not None and any(r[1] is not None for r in table)
    check("persistent", False, sw.tuning)
    check("streams", True, "streams")
    assert all(float(s["t"]) > 0 for s in sw.states)


def test_sweep_with_run_time_table_axes_equals_the_loop():
    """Instances whose axes the compile-time tiles do not take (288 x 144 and 432 x 216: 9 and 27
    divide them) beside a power-of-two one: the persistent kernel with the run-time-table
    transform body gives every instance exactly what its own plan gives, in every schedule."""
    import numpy as np
    from aerolume_b200.ns2d.sweep import Sweep2D
    from aerolume_b200.ns2d.workloads import build_geometry, make_ops, naca4
    insts = []
    for k, (nx, ny) in enumerate(((288, 144), (432, 216), (256, 128), (288, 144))):
        ops = make_ops(nx, ny, 8.0 / nx, 1500.0 + 700.0 * k, force_ref=1.0, moment_ref=(2.0, 2.0), dtype="float32")
        insts.append((ops, build_geometry([naca4(0.12, 0.02 * k, 0.4, 2.0 + 3.0 * k)], ops), {}))
    sw = Sweep2D(insts)
    snap = sw.snapshot()
    ref = _run(sw, snap, "loop", 4, graph=False)
    for cand in ((2, 3, 1, "barrier", 1), (3, 4, 0, "queue", 4), (2, 2, 1, "counters", 2)):
        sw.use_persistent(*cand)
        assert sw._persistent["info"]["operations"] > 0
        got = _run(sw, snap, "persistent", 4, graph=True)
        for k, (a, b) in enumerate(zip(got, ref)):
            for x, y in zip(a, b):
                assert torch.equal(x, y), (cand, k)
        assert sw.status() == 0, cand
    assert np.all([float(s["t"]) > 0 for s in sw.states])


@pytest.mark.parametrize("schedule", ["barrier", "counters", "queue"])
def test_sweep_barrier_gives_up_and_reports(schedule):
    """The persistent launch's waits for arrivals that never come (the test hook asks for one
    CTA more than the launch has at a grid barrier, or one finished item more than an instance
    has before every item): every CTA gives up after the bounded wait, the status word reports
    it, and the next launch with the bound restored runs normally and matches the per-instance
    loop."""
    from aerolume_b200.ns2d.sweep import Sweep2D
    from aerolume_b200.ns2d.workloads import sweep_instances
    insts = [i for i in sweep_instances(64, seed=0) if i[0].nx == 256][:2]
    sw = Sweep2D(insts)
    snap = sw.snapshot()
    sw.use_persistent(2, 1, 1, schedule)
    sw.set_barrier(2000, extra=1)
    sw.step("persistent")
    torch.cuda.synchronize()
    assert sw.status() & 1
    sw.set_barrier(1 << 26, extra=0)
    got = _run(sw, snap, "persistent", 3, graph=False)
    assert sw.status() == 0
    ref = _run(sw, snap, "loop", 3, graph=False)
    for a, b in zip(got, ref):
        for x, y in zip(a, b):
            assert torch.equal(x, y)
