"""Throughput of the B200 3D Navier-Stokes step (Mcell-steps/s) on the bluff-box workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 256 x 128 x 128 FP32 cells (4.19 M), box 1 x 1 x 0.5 on a moving floor, WALE LES,
Boussinesq temperature (body 10 K above the stream, Pr 0.71, Ri 0.1 on the body height),
one 16-nozzle smoke rake; seeded N(0, 1e-3) noise on a uniform stream, projected.  One
"step" is one SSP-RK3 time step with its three projections, the temperature stages, the
forces and heat rates, and the smoke update.

``value``: steps with the state resident in HBM, K steps captured in one CUDA graph and
replayed once between a barrier and ``torch.cuda.synchronize()``, timed with CUDA events
(max over ranks).  ``e2e``: the same step through the public plan API with host buffers --
every step copies the state in from pinned host memory and the new state, coefficients and
heat rates back out.  ``roofline``: the dominant kernel's algorithmic bytes per launch over
its event-timed mean duration against the measured HBM copy bandwidth.  ``cpu_baseline``:
the numpy oracle (a restatement of the reference's plain-torch step) on a bounded sample of
the same workload on this host.

``--workload cylinder2d`` measures the 2D step instead (a D = 0.5 cylinder at Re_D 100 in an
8 x 4 tunnel, 256 x 128 FP32, upwind3, CFL 0.5; ``heated2d``: the same with heat transfer,
the cylinder held at theta = 1, Pr 0.71, Ri 0.5) and ``--workload sweep2d`` the batched sweep
(64 NACA 4-digit airfoils on grids from 256 x 128 to 1024 x 512, all advanced by one CUDA
graph that spreads the instances over 16 streams; the same plans looped one after another on
a single stream are reported beside it).

``--workload fields3d`` measures the field outputs of the same 3D state (ns3d/solver.py:
1374-1416, fields.py:45-102): one pass writes all seven cell fields (centred u, v, w, speed,
vorticity magnitude, Q-criterion, eddy viscosity) from the staggered velocity, and a
million trilinear probes of the speed field are timed beside it.

``--workload placed3d`` measures the box case with the placed physics in the step (a swirling
velocity-regulated fan, a warm jet and a vent, a painted block, the PID step controller; no
smoke, which jets and vents leave to the caller), with the same plan without them beside it.

``--workload record3d`` measures the per-step bookkeeping (ns3d/solver.py:706-744): the history
row and a running-mean sample of u, v, w, p and theta on the 256 x 128 x 128 grid.

``--workload masks3d`` measures mask construction (ns3d/geometry.py:385-495 with the exact
signed distance): the masks, solid velocity and force weights of a closed 9024-triangle
sphere of diameter 1 at 32 cells per diameter, rebuilt as a live attitude edit does.

With ``--gpus N`` (N > 1, launched by torch.distributed.run) every rank advances its own
replica (no data-path collective: a single instance of this solver does not shard), and
``value`` is the total over ranks.  ``--impl reference`` times the reference arm: the
oracle's CPU step on rank 0 (other ranks exit without work).
"""
from __future__ import annotations

import argparse
import json
import re
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from aerolume_b200.replicas import gather_results, max_over_ranks, shard_instances  # noqa: E402

METRIC = "Mcell-steps/s on 1 B200: plain vs batched vs learned closure, at stated error"
UNIT = "Mcell-steps/s"
SHAPE = (256, 128, 128)


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _tensor_peak():
    """(bf16 dense TFLOP/s burst, kind): MEASURED_PEAKS.json's cuBLAS figure, else the fallback."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def run_closure(args, rank, world, local_rank):
    """The learned-closure step (the box case with the closure's eddy viscosity in place of WALE
    where it applies), K steps in one graph; and its dominant kernel, the closure's pass over the
    padded grid, timed alone against the tensor-core peak."""
    import ctypes as C

    import torch
    from aerolume_b200 import _lib
    from aerolume_b200.ns3d.closure import ClosureModel
    from aerolume_b200.ns3d.plan import Ns3dPlan
    from aerolume_b200.ns3d.workloads import box_on_moving_floor, initial_state
    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    nx, ny, nz = args.shape
    cells = nx * ny * nz
    ops, geom, th, src, _ = box_on_moving_floor(nx, ny, nz, dtype="float32", seed=0)
    model = ClosureModel(device=dev, seed=0)
    model.out_std[:] = 0.02      # an untrained network: outputs of the subgrid stress's size
    plan = Ns3dPlan(ops, geom, th, src, smoke=True, device=dev, closure=model)
    u, v, w = initial_state(ops, seed=rank, device=dev)
    plan.project(u, v, w)
    theta = torch.zeros(nz, ny, nx, device=dev)
    dyes = [torch.zeros(nz, ny, nx, device=dev), torch.zeros(nz, ny, nx, device=dev)]
    t = torch.zeros((), device=dev)
    out = plan.empty_fields()
    out["u"], out["v"], out["w"], out["theta"] = u, v, w, theta

    def step(j):
        out["dye"] = dyes[(j + 1) % 2]
        plan.step(u, v, w, t, theta0=theta, dye0=dyes[j % 2], out=out)
        t.copy_(out["t"])

    for j in range(args.warmup):
        step(j)
    torch.cuda.synchronize()
    K = args.steps
    s = torch.cuda.Stream(device=dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            for j in range(K):
                step(args.warmup + j)
    torch.cuda.current_stream(dev).wait_stream(s)
    ms, clk = _time_graph(g, dist, local_rank, rank, dev)
    ev, wale = plan.closure_counts()
    status = plan.status()
    # the closure's pass alone on the padded grid's worth of cells (seeded gradients)
    n = (nz + 2) * (ny + 2) * (nx + 2)
    gen = torch.Generator(device=dev).manual_seed(1)
    grad9 = torch.randn(9, n, device=dev, generator=gen)
    grad9[8] = 1.0
    nu0 = torch.zeros(n, device=dev)
    nu = torch.empty_like(nu0)
    st = torch.zeros(1, device=dev, dtype=torch.int32)
    m = model.cstruct()
    L = _lib.lib()
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    reps = 10

    def one():
        _lib.check(L.aero_closure_eddy_viscosity(C.byref(m), C.c_void_p(grad9.data_ptr()), n, float(ops.h),
                                                 C.c_void_p(nu.data_ptr()), None, None, C.c_void_p(st.data_ptr()),
                                                 stream), "aero_closure_eddy_viscosity")

    for _ in range(3):
        one()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        one()
    b.record()
    torch.cuda.synchronize()
    pass_ms = a.elapsed_time(b) / reps
    if rank != 0:
        return
    peak, peak_kind = _tensor_peak()
    flops = 2.0 * 36864 * n          # padded 16 -> 128 -> 128 -> 128 -> 16 layers, 2 FLOP per MAC
    line = {"metric": METRIC, "value": world * cells * K / (ms * 1e-3) / 1e6, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 step, bf16 MLP (fp32 accumulate)", "data": "synthetic",
            "config": _config(nx, ny, nz, {"plain_variant": "learned closure (WALE fallback per cell)",
                                           "graph": f"{K} steps, 1 replay",
                                           "network": "untrained (seeded) weights: the cost does not depend on them"}),
            "closure_cells_evaluated": ev, "closure_wale_fraction": wale / max(ev, 1),
            "roofline": {"bound": "tensor", "kernel": "closure_nu_kernel (the closure's pass, timed alone)",
                         "achieved": flops / (pass_ms * 1e-3) / 1e12, "peak": peak, "peak_kind": peak_kind,
                         "unit": "TFLOP/s", "frac": flops / (pass_ms * 1e-3) / 1e12 / peak, "traffic": None,
                         "flops_per_launch": flops, "ms_per_launch": pass_ms, "cells_per_launch": n},
            "cpu_baseline": None, "e2e": None, "gpu_launches": (launches_per_step(plan) + 3) * K, "clocks": clk,
            "status": status}
    print(json.dumps(line), flush=True)


def _config(nx, ny, nz, extra=None):
    cfg = {"workload": f"box on moving floor {nx}x{ny}x{nz} FP32, WALE, Boussinesq heat, 1 smoke rake",
           "cells": nx * ny * nz, "grid": [nx, ny, nz], "inputs_vs_l2": "working set ~1 GB > 126 MB L2 (no flush)",
           "parallelism": "replicas"}
    if extra:
        cfg.update(extra)
    return cfg


class Clocks:
    """nvidia-smi sampling during the timed region (median SM clock, throttle reasons); the
    samples come back through a pipe (about 100 bytes every 100 ms)."""

    def __init__(self, index):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            text, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            text, _ = self.proc.communicate()
        rows = [r.split(",") for r in (text or "").splitlines() if r.strip()]
        sm = [float(r[0]) for r in rows if r[0].strip().replace(".", "").isdigit()]
        if not sm:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 3 + i and r[3 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][1]), "reasons": reasons,
                "samples": len(sm)}


def oracle_sample(nx, ny, nz, steps, warm=1):
    """Wall time of ``steps`` oracle steps (after ``warm`` untimed steps) on the full workload."""
    from aerolume_b200.ns3d.workloads import box_on_moving_floor, initial_state
    from oracle import ns3d as O
    ops, geom, th, src, _ = box_on_moving_floor(nx, ny, nz, dtype="float32")
    u, v, w = (x.numpy() for x in initial_state(ops, device="cpu"))
    f32 = np.float32
    ps = O.PoissonSolver3D(nx, ny, nz, ops.h, ops.periodic_axes, f32)
    u, v, w, _ = O.project3d(u, v, w, ops, ps)
    theta = np.zeros((nz, ny, nx), f32)
    dye = np.zeros((nz, ny, nx), f32)
    t = f32(0.0)

    def one(u, v, w, t, theta, dye):
        r = O.step3d_phys(u, v, w, t, geom, ops, ps, th=th, theta=theta)
        c = O.apply_solids_and_sources(O.advect_dye3d(dye, r.u, r.v, r.w, r.dt, ops), r.t, geom, src)
        return r.u, r.v, r.w, r.t, r.theta, c

    for _ in range(warm):
        u, v, w, t, theta, dye = one(u, v, w, t, theta, dye)
    t0 = time.perf_counter()
    for _ in range(steps):
        u, v, w, t, theta, dye = one(u, v, w, t, theta, dye)
    return time.perf_counter() - t0


def _threads():
    try:
        from threadpoolctl import threadpool_info
        return max([i.get("num_threads", 1) for i in threadpool_info()] + [1])
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------------------
# The reference itself (Aerolume installed unmodified under baseline/_ref): its FlowSolver3D
# on the host cores (the CPU baseline) and on the GPU (the bar of the plain drop-in)
# ---------------------------------------------------------------------------------------

REF_DIR = ROOT / "baseline" / "_ref"


def _reference_api():
    """The reference's public 3D solver API from baseline/_ref (ImportError when absent)."""
    if not (REF_DIR / "aerolume" / "solvers" / "ns3d" / "solver.py").exists():
        raise ImportError("baseline/_ref holds no installed reference")
    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    from aerolume.solvers.ns3d.config import DyeRake, ImmersedMesh, SolverConfig3D, ThermalConfig3D
    from aerolume.solvers.ns3d.solver import FlowSolver3D
    return DyeRake, ImmersedMesh, SolverConfig3D, ThermalConfig3D, FlowSolver3D


def _box_mesh(size, center):
    """(vertices (8, 3), faces (12, 3)) of an axis-aligned box, wound outward."""
    lx, ly, lz = size
    cx, cy, cz = center
    v = np.array([[cx + sx * lx / 2, cy + sy * ly / 2, cz + sz * lz / 2]
                  for sz in (-1, 1) for sy in (-1, 1) for sx in (-1, 1)], dtype=np.float64)
    f = np.array([[0, 2, 1], [1, 2, 3], [4, 5, 6], [5, 7, 6], [0, 1, 4], [1, 5, 4],
                  [2, 6, 3], [3, 6, 7], [0, 4, 2], [2, 4, 6], [1, 3, 5], [3, 7, 5]], dtype=np.int64)
    return v, f


def reference_box_config(nx, ny, nz, device):
    """The reference's SolverConfig3D of the box-on-moving-floor workload (the same case that
    aerolume_b200.ns3d.workloads.box_on_moving_floor builds for the B200 step)."""
    DyeRake, ImmersedMesh, SolverConfig3D, ThermalConfig3D, _ = _reference_api()
    h = 8.0 / nx
    v, f = _box_mesh((1.0, 1.0, 0.5), (2.5, 2.0, 0.25))
    box = ImmersedMesh(v, f, name="box", thermal="temperature", thermal_value=1.0)
    rng = np.random.default_rng(0)
    ys = np.sort(rng.uniform(1.2, 2.8, 16))
    zs = rng.uniform(0.1, 0.45, 16)
    rake = DyeRake("rake", [(1.25, float(y), float(z)) for y, z in zip(ys, zs)], radius=1.25 * h)
    return SolverConfig3D(nx=nx, ny=ny, nz=nz, h=h, x0=0.0, y0=0.0, z0=0.0, re=1e4, bodies=[box], bc_zmin="moving",
                          ground_speed=1.0, turbulence="wale", thermal=ThermalConfig3D(prandtl=0.71, richardson=0.2),
                          dye=True, dye_rake=rake, ref_area=0.5, moment_ref=(2.5, 2.0, 0.0), dtype="float32",
                          device=device, perturb=False)


def time_reference_cpu(nx, ny, nz, steps, warm, threads=None, repeats=3):
    """Best-of-``repeats`` wall time per step of the reference's FlowSolver3D.advance on the host
    (device "cpu", FP32; advance flushes denormals itself, ns3d/solver.py:998), after ``warm``
    untimed steps: the method of validation/bench_ns3d.py:73-101."""
    import torch
    *_, FlowSolver3D = _reference_api()
    old = torch.get_num_threads()
    torch.set_num_threads(threads or os.cpu_count() or 1)
    try:
        s = FlowSolver3D(reference_box_config(nx, ny, nz, "cpu"))
        s.advance(warm)
        best = float("inf")
        for _ in range(repeats):
            t0 = time.perf_counter()
            s.advance(steps)
            best = min(best, (time.perf_counter() - t0) / steps)
        return best, torch.get_num_threads()
    finally:
        torch.set_num_threads(old)


def time_reference_gpu(nx, ny, nz, dev, steps=200, repeats=3):
    """The reference's own PyTorch CUDA step on this GPU (fused NVRTC kernels, cuBLAS Poisson,
    10-step CUDA graphs): best of ``repeats`` runs of ``advance(steps)`` after a 30-step warm-up
    (NVRTC compile, graph capture), as validation/bench_ns3d.py:73-101 times it, with CUDA
    events around each run.  Returns a dict for the bench line."""
    import torch
    try:
        *_, FlowSolver3D = _reference_api()
    except ImportError as exc:
        return {"unavailable": str(exc)}
    with torch.cuda.device(dev):
        s = FlowSolver3D(reference_box_config(nx, ny, nz, f"cuda:{dev.index}"))
        s.advance(30)
        torch.cuda.synchronize()
        clocks = Clocks(dev.index)
        time.sleep(0.3)
        best = float("inf")
        for _ in range(repeats):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record()
            s.advance(steps)
            b.record()
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b) / steps)
        clk = clocks.stop()
        out = {"value": nx * ny * nz / (best * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": best, "steps": steps,
               "repeats": repeats, "fused_kernels": bool(getattr(s, "uses_fused_kernels", False)),
               "cuda_graphs": bool(getattr(s, "uses_cuda_graphs", False)),
               "fused_error": getattr(s, "fused_error", None), "clocks": clk,
               "how": "reference FlowSolver3D.advance on this GPU (baseline/_ref, unmodified), best of "
                      f"{repeats} x {steps} steps after 30 warm-up steps, CUDA events"}
        del s
        import gc
        gc.collect()
        torch.cuda.empty_cache()
    return out


def run_reference(args, rank):
    """``--impl reference``: the reference's own CPU path (FlowSolver3D on the host cores)."""
    nx, ny, nz = args.shape
    if rank != 0:
        return
    steps = max(1, min(args.steps, 5))
    warm = max(1, min(args.warmup, 3))   # a reference CPU step takes about a second: both bounded
    try:
        per_step, cores = time_reference_cpu(nx, ny, nz, steps, warm)
    except ImportError as exc:
        print(json.dumps({"impl": "reference", "unavailable": f"reference not installed: {exc}"}), flush=True)
        return
    val = nx * ny * nz / per_step / 1e6
    sample = (f"best of 3 x {steps} full {nx}x{ny}x{nz} steps of the reference's FlowSolver3D.advance "
              f"(device cpu, FP32, {cores} threads) after {warm} untimed steps")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": 1e3 * per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": _config(nx, ny, nz),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def launches_per_step(plan):
    """Kernels one aero_ns3d_step launches (the sequence in csrc/capi.cu)."""
    c = plan.cfg
    tunnel = not c.periodic[0] and not c.closed
    les = c.les != 0
    n = 2                                           # u copy with max |u|; max |v|, |w| (|theta|) in one launch
    n += 1                                          # dt
    n += 1 if tunnel else 0                         # inlet / u0 outlet sums
    # a power-of-two x axis folds the divergence into the first transform pass and the
    # pressure accumulation into the last one (not with jets / vents, whose mass sources enter
    # the divergence in their own launch)
    fused = 8 <= c.nx <= 2048 and (c.nx & (c.nx - 1)) == 0 and c.nport == 0
    per_stage = 1 + (0 if fused else 1) + 5 + (0 if fused else 1) + 1 + (2 if tunnel else 0) + (1 if les else 0)
    per_stage += 1 if c.nport else 0                # div -= m of the jets and vents
    n += 3 * per_stage                              # [nu], [sums, corr], stage, [div], 5 transforms, [psi_w], correct
    n += 1 if c.nfan else 0                         # disc velocities and PI thrust, once per step
    n += 1 if c.smoke else 0
    n += 1 if (c.nbody * 9 + (c.n_tbody if c.thermal else 0)) > 0 else 0   # partial-sum reduction
    n += 1                                          # finalize
    return n


def run_ours(args, rank, world, local_rank):
    import torch
    from aerolume_b200.ns3d.plan import Ns3dPlan
    from aerolume_b200.ns3d.workloads import box_on_moving_floor, initial_state
    from aerolume_b200 import _lib
    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    nx, ny, nz = args.shape
    cells = nx * ny * nz
    ops, geom, th, src, _ = box_on_moving_floor(nx, ny, nz, dtype="float32", seed=0)
    plan = Ns3dPlan(ops, geom, th, src, smoke=True, device=dev)
    u, v, w = initial_state(ops, seed=rank, device=dev)
    plan.project(u, v, w)
    theta = torch.zeros(nz, ny, nx, device=dev)
    dyes = [torch.zeros(nz, ny, nx, device=dev), torch.zeros(nz, ny, nx, device=dev)]
    t = torch.zeros((), device=dev)
    out = plan.empty_fields()
    out["u"], out["v"], out["w"], out["theta"] = u, v, w, theta

    def step(j, events=None):
        out["dye"] = dyes[(j + 1) % 2]
        plan.step(u, v, w, t, theta0=theta, dye0=dyes[j % 2], out=out, events=events)
        t.copy_(out["t"])

    # ---- warm-up (eager), then capture exactly K steps with phase events in one graph
    for j in range(args.warmup):
        step(j)
    torch.cuda.synchronize()
    K = args.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(_lib.TRACE_EVENTS)] for _ in range(K)]
    for row in ev:                          # torch creates the CUDA event on its first record
        for e in row:
            e.record()
    torch.cuda.synchronize()
    s = torch.cuda.Stream(device=dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            for j in range(K):
                step(args.warmup + j, ev[j])
    torch.cuda.current_stream(dev).wait_stream(s)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = Clocks(local_rank) if rank == 0 else None
    time.sleep(0.3 if clocks else 0.0)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    start.record()
    g.replay()
    end.record()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ms = start.elapsed_time(end)
    clk = clocks.stop() if clocks else None
    status = plan.status()
    ms = max_over_ranks(ms, dist, dev)
    # ---- phase times from the events (mean over the K captured steps)
    def span(j, a, b):
        return ev[j][a].elapsed_time(ev[j][b])
    stage_ms = [span(j, 2 + 5 * st, 3 + 5 * st) for j in range(K) for st in range(3)]
    poisson_ms = [span(j, 4 + 5 * st, 5 + 5 * st) for j in range(K) for st in range(3)]
    phases = {
        "time_step": float(np.mean([span(j, 0, 1) for j in range(K)])),
        "outlet_corr": float(np.mean([span(j, 1 + 5 * st if st else 1, 2 + 5 * st) for j in range(K) for st in range(3)])),
        "stage_kernel": float(np.mean(stage_ms)),
        "divergence": float(np.mean([span(j, 3 + 5 * st, 4 + 5 * st) for j in range(K) for st in range(3)])),
        "poisson": float(np.mean(poisson_ms)),
        "correct": float(np.mean([span(j, 5 + 5 * st, 6 + 5 * st) for j in range(K) for st in range(3)])),
        "smoke": float(np.mean([span(j, 16, 17) for j in range(K)])),
        "finalize": float(np.mean([span(j, 17, 18) for j in range(K)])),
    }
    # ---- e2e through the public API with host buffers
    e2e = None
    if rank == 0 or world > 1:
        host_in = {k: torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
                   for k, x in (("u", u), ("v", v), ("w", w), ("theta", theta), ("dye", dyes[0]), ("t", t))}
        for k, x in (("u", u), ("v", v), ("w", w), ("theta", theta), ("dye", dyes[0]), ("t", t)):
            host_in[k].copy_(x)
        host_out = {k: torch.empty(x.shape, dtype=x.dtype, pin_memory=True) for k, x in out.items()}
        d_in = {k: torch.empty_like(x, device=dev) for k, x in host_in.items()}
        o2 = plan.empty_fields()
        h2d = sum(x.numel() * x.element_size() for x in host_in.values())
        d2h = sum(x.numel() * x.element_size() for x in host_out.values())
        torch.cuda.synchronize()
        ke = max(3, min(K, 10))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(ke):
            for k in host_in:
                d_in[k].copy_(host_in[k], non_blocking=True)
            plan.step(d_in["u"], d_in["v"], d_in["w"], d_in["t"], theta0=d_in["theta"], dye0=d_in["dye"], out=o2)
            for k in host_out:
                host_out[k].copy_(o2[k], non_blocking=True)
            # the next step starts from this step's result, as a host caller's loop would
            for k in ("u", "v", "w", "theta", "dye", "t"):
                host_in[k], host_out[k] = host_out[k], host_in[k]
        e1.record()
        torch.cuda.synchronize()
        ems_serial = max_over_ranks(e0.elapsed_time(e1) / ke, dist, dev)
        # pipelined: every step still copies its whole input state in from pinned host memory and
        # its whole result out, but the copies run on their own streams (the two directions on
        # separate copy engines) and overlap the neighbouring steps' compute; each step starts
        # from a host state of its own (a stream of independent states), double-buffered on the
        # device
        main = torch.cuda.current_stream(dev)
        s_in, s_out = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
        d_buf = [{k: torch.empty_like(x, device=dev) for k, x in host_in.items()} for _ in range(2)]
        o_buf = [plan.empty_fields() for _ in range(2)]
        h_out = [{k: torch.empty(x.shape, dtype=x.dtype, pin_memory=True) for k, x in o_buf[0].items()}
                 for _ in range(2)]
        ev_in = [torch.cuda.Event() for _ in range(2)]
        ev_done = [torch.cuda.Event() for _ in range(2)]
        ev_out = [torch.cuda.Event() for _ in range(2)]
        torch.cuda.synchronize()
        e0.record()
        for j in range(ke):
            b = j % 2
            with torch.cuda.stream(s_in):
                if j >= 2:
                    s_in.wait_event(ev_done[b])        # step j - 2 has finished reading d_buf[b]
                for k in host_in:
                    d_buf[b][k].copy_(host_in[k], non_blocking=True)
                ev_in[b].record(s_in)
            main.wait_event(ev_in[b])
            if j >= 2:
                main.wait_event(ev_out[b])              # o_buf[b] of step j - 2 is on the host
            db = d_buf[b]
            plan.step(db["u"], db["v"], db["w"], db["t"], theta0=db["theta"], dye0=db["dye"], out=o_buf[b])
            ev_done[b].record(main)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_done[b])
                for k in h_out[b]:
                    h_out[b][k].copy_(o_buf[b][k], non_blocking=True)
                ev_out[b].record(s_out)
        main.wait_stream(s_out)
        e1.record()
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1) / ke, dist, dev)
        e2e = {"value": world * cells / (ems * 1e-3) / 1e6, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": ems, "steps": ke,
               "how": "Ns3dPlan.step on host states, copies in and out on their own streams overlapping the "
                      "neighbouring steps (each step a fresh host state)",
               "serial": {"value": world * cells / (ems_serial * 1e-3) / 1e6, "ms_per_step": ems_serial,
                          "how": "copy in, step, copy out on one stream, the next step starting from this "
                                 "step's host result"}}
    if rank != 0:
        return
    peak, peak_kind = _peaks()
    # dominant kernel: the stage kernel.  Algorithmic bytes per launch, FP32 (4 B) per cell:
    # reads stage-start u, v, w (3) and theta (1), the step-start u, v, w (3) and theta (1)
    # at stages 2 and 3, writes the stage value u, v, w (3) and theta (1): 8, 12, 12 words.
    alg = 4 * cells * (8 + 12 + 12) / 3.0
    achieved = alg / (phases["stage_kernel"] * 1e-3) / 1e9
    ms_step = ms / K
    value = world * cells * K / (ms * 1e-3) / 1e6
    # the reference's own PyTorch CUDA step on this GPU, after our timed region
    ref_gpu = None if args.no_ref_gpu else time_reference_gpu(nx, ny, nz, dev)
    if ref_gpu and "value" in ref_gpu:
        ref_gpu["speedup_of_value"] = value / ref_gpu["value"]
        if e2e:
            ref_gpu["speedup_of_e2e"] = e2e["value"] / ref_gpu["value"]
    sample_steps = 2
    if args.no_cpu:
        cpu = None
    else:
        try:
            per_step, cores = time_reference_cpu(nx, ny, nz, sample_steps, 1)
            cpu = {"value": cells / per_step / 1e6, "unit": UNIT, "cores": cores, "kind": "reference",
                   "sample": f"best of 3 x {sample_steps} full {nx}x{ny}x{nz} steps of the reference's "
                             f"FlowSolver3D.advance (device cpu, FP32, {cores} threads) after 1 untimed step"}
        except ImportError:
            secs = oracle_sample(nx, ny, nz, sample_steps)
            cpu = {"value": cells * sample_steps / secs / 1e6, "unit": UNIT, "cores": _threads(), "kind": "port",
                   "sample": f"{sample_steps} full {nx}x{ny}x{nz} steps of the numpy oracle after 1 untimed step"}
    # DRAM bytes per stage_kernel launch (mean of the three stages) from the committed ncu
    # summary of this workload; None for other shapes
    traffic = None
    tp = ROOT / "profiles" / "stage_kernel_256x128x128_dram.md"
    if (nx, ny, nz) == SHAPE and tp.exists():
        m = re.search(r"^traffic_bytes_per_launch_mean:\s*(\d+)", tp.read_text(), re.M)
        traffic = int(m.group(1)) if m else None
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": _config(nx, ny, nz, {"plain_variant": "plain drop-in (WALE)", "graph": f"{K} steps, 1 replay"}),
            "roofline": {"bound": "hbm", "kernel": "stage_kernel", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "alg_bytes_per_launch": alg},
            "phases_ms": phases, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches_per_step(plan) * K,
            "clocks": clk, "status": status, "reference_gpu": ref_gpu}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# 2D workloads
# ---------------------------------------------------------------------------------------

def _launches_2d(plan):
    c = plan.cfg
    fused = 8 <= c.nx <= 2048 and (c.nx & (c.nx - 1)) == 0
    n = 0                                              # (dt is derived inside the first stage kernel)
    if not c.has_dt_fixed:
        n += 1 + (1 if c.les else 0)                   # |u| and |v| maxima (one launch), nu_t of u0
    n += 3 * (1 + 3 + (0 if fused else 2)) + 1         # stage, 3 transform passes, [div, psi_w]; one correct
    n += 1 if c.dye else 0
    n += 3 + 1 if c.thermal else 0                     # a theta stage per RK stage, the heat report
    return n + 1                                       # finalize


def _time_graph(g, dist, local_rank, rank, dev):
    import torch
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = Clocks(local_rank) if rank == 0 else None
    time.sleep(0.3 if clocks else 0.0)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    start.record()
    g.replay()
    end.record()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ms = start.elapsed_time(end)
    clk = clocks.stop() if clocks else None
    return max_over_ranks(ms, dist, dev), clk


def cpu_baseline_2d(workload, port_sample, cells, what):
    """The 2D lines' cpu_baseline: the reference's own 2D solver on the host cores (kind
    "reference"), or, when baseline/_ref holds no reference, the numpy oracle port."""
    try:
        steps = 10
        per_step, cores, ref_cells, _ = time_reference_cpu_2d(workload, steps, 2)
        return {"value": ref_cells / per_step / 1e6, "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": f"best of 3 x {steps} {what} of the reference's 2D FlowSolver.advance (device cpu, FP32) "
                          "after 2 untimed steps"}
    except ImportError:
        steps = 10
        secs = port_sample(steps)
        return {"value": cells * steps / secs / 1e6, "unit": UNIT, "cores": _threads(), "kind": "port",
                "sample": f"{steps} {what} of the numpy 2D oracle after 1 untimed step"}


def oracle2d_sample(ops, geom, steps, seed=0, thermal=None):
    """Wall time of ``steps`` 2D oracle steps (after one untimed step); with ``thermal`` the
    heat-transfer step, theta starting at 0."""
    from oracle import ns2d as O2
    f32 = np.float32
    rng = np.random.default_rng(seed)
    ps = O2.PoissonSolver2D(ops.nx, ops.ny, ops.h, ops.periodic, f32)
    u = (np.ones((ops.ny, ops.nx + 1)) + 1e-3 * rng.standard_normal((ops.ny, ops.nx + 1))).astype(f32)
    v = (1e-3 * rng.standard_normal((ops.ny + 1, ops.nx))).astype(f32)
    u, v = O2.apply_boundary_values(u, v, ops)
    u, v, _ = O2.project2d(u, v, ops, ps)
    geom32 = type(geom)(geom.window, *[None if x is None else np.asarray(x, f32) for x in
                                       (geom.chi_u, geom.chi_v, geom.chi_c, geom.a_u, geom.a_v, geom.k_u, geom.k_v)],
                        geom.nbody)
    t = f32(0.0)
    if thermal is not None:
        import dataclasses
        tp = O2.Thermal2D(**{f.name: getattr(thermal, f.name) for f in dataclasses.fields(O2.Thermal2D)})
        for f in ("chi_t", "a_t", "w_t", "ins_u", "ins_v", "q_skin", "w_f", "vol_u", "vol_v"):
            if getattr(tp, f) is not None:
                setattr(tp, f, np.asarray(getattr(tp, f), f32))
        theta = np.zeros((ops.ny, ops.nx), f32)
        r = O2.step2d_thermal(u, v, t, theta, geom32, ops, ps, tp)
        t0 = time.perf_counter()
        for _ in range(steps):
            r = O2.step2d_thermal(r.u, r.v, r.t, r.theta, geom32, ops, ps, tp)
        return time.perf_counter() - t0
    r = O2.step2d(u, v, t, geom32, ops, ps)
    t0 = time.perf_counter()
    for _ in range(steps):
        r = O2.step2d(r.u, r.v, r.t, geom32, ops, ps)
    return time.perf_counter() - t0


HEATED_2D = ("heated cylinder D=0.5 at (2,2) held at theta 1, 256x128 FP32, Re_D 100, Pr 0.71, Ri 0.5, "
             "slip adiabatic walls, upwind3, CFL 0.5")


def run_2d(args, rank, world, local_rank):
    import torch
    from aerolume_b200.ns2d.plan import Ns2dPlan
    from aerolume_b200.ns2d.workloads import cylinder_tunnel, heated_cylinder, initial_state
    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    nx, ny = 256, 128
    cells = nx * ny
    heated = args.workload == "heated2d"
    thermal = None
    if heated:
        ops, geom, thermal = heated_cylinder(nx, ny, "float32")
    else:
        ops, geom = cylinder_tunnel(nx, ny, "float32")
    plan = Ns2dPlan(ops, geom, thermal=thermal, device=dev)
    u, v = initial_state(ops, plan, seed=rank, noise=1e-3)
    t = torch.zeros((), device=dev)
    theta = torch.zeros(ny, nx, device=dev) if heated else None
    out = plan.empty_fields()
    out["u"], out["v"] = u, v
    if heated:
        out["theta"] = theta

    def step():
        plan.step(u, v, t, theta0=theta, out=out)
        t.copy_(out["t"])

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    K = args.steps
    s = torch.cuda.Stream(device=dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            for _ in range(K):
                step()
    torch.cuda.current_stream(dev).wait_stream(s)
    ms, clk = _time_graph(g, dist, local_rank, rank, dev)
    coeffs = out["coeffs"][0].tolist()
    # e2e: state in from pinned host memory, step, state / coefficients / time out, every step
    hu, hv = u.cpu().pin_memory(), v.cpu().pin_memory()
    hth = theta.cpu().pin_memory() if heated else None
    ho = {k: torch.empty(x.shape, dtype=x.dtype, pin_memory=True) for k, x in out.items()}
    du, dv = torch.empty_like(u), torch.empty_like(v)
    dth = torch.empty_like(theta) if heated else None
    o2 = plan.empty_fields()
    ke = max(10, min(K, 200))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(ke):
        du.copy_(hu, non_blocking=True)
        dv.copy_(hv, non_blocking=True)
        if heated:
            dth.copy_(hth, non_blocking=True)
        plan.step(du, dv, t, theta0=dth, out=o2)
        for k in ho:
            ho[k].copy_(o2[k], non_blocking=True)
        hu, ho["u"] = ho["u"], hu
        hv, ho["v"] = ho["v"], hv
        if heated:
            hth, ho["theta"] = ho["theta"], hth
    e1.record()
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1) / ke
    if rank != 0:
        return
    h2d = u.numel() * 4 + v.numel() * 4 + (theta.numel() * 4 if heated else 0)
    d2h = sum(x.numel() * x.element_size() for x in out.values())
    peak, peak_kind = _peaks()
    # compulsory bytes per 2D cell-step, FP32; heat transfer adds theta_p (3 stages), theta_0
    # (stages 2, 3) and the stage writes: 8 F
    alg = (228.0 + (32.0 if heated else 0.0)) * cells
    ms_step = ms / K
    cpu = None
    if not args.no_cpu:
        cpu = cpu_baseline_2d(args.workload, lambda n: oracle2d_sample(ops, geom, n, thermal=thermal), cells,
                              f"full {nx}x{ny} steps")
    line = {"metric": METRIC, "value": world * cells * K / (ms * 1e-3) / 1e6, "unit": UNIT, "n_gpus": world,
            "steps": K, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": HEATED_2D if heated else
                       "cylinder D=0.5 at (2,2), 256x128 FP32, Re_D 100, slip walls, upwind3, CFL 0.5",
                       "cells": cells, "grid": [nx, ny],
                       "inputs_vs_l2": "7.5 MB working set stays in the 126 MB L2 between steps (no flush)",
                       "parallelism": "replicas", "graph": f"{K} steps, 1 replay"},
            "roofline": {"bound": "hbm", "kernel": "whole step", "achieved": alg / (ms_step * 1e-3) / 1e9,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": alg / (ms_step * 1e-3) / 1e9 / peak, "traffic": None,
                         "alg_bytes_per_step": alg},
            "cpu_baseline": cpu,
            "e2e": {"value": cells / (ems * 1e-3) / 1e6, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": ems, "steps": ke},
            "gpu_launches": _launches_2d(plan) * K, "clocks": clk, "coeffs_last": coeffs}
    print(json.dumps(line), flush=True)


def run_sweep(args, rank, world, local_rank):
    """The batched sweep: 64 NACA instances advanced by one persistent launch per step (its launch
    shape picked by Sweep2D.tune), K steps in one CUDA graph; beside it the same plans spread over
    16 streams and looped one after another (each in its own graph), and the e2e figure with
    every instance's state copied in from and its time and coefficients out to host memory."""
    import torch
    from aerolume_b200.ns2d.sweep import Sweep2D
    from aerolume_b200.ns2d.workloads import sweep_instances
    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    all_insts = sweep_instances(args.instances, seed=0)
    if args.shard:  # the 64 instances split over the ranks (strong scaling), else every rank runs all 64
        mine = shard_instances([o.nx * o.ny for o, _, _ in all_insts], world)[rank]
    else:
        mine = list(range(len(all_insts)))
    insts = [all_insts[k] for k in mine]
    sw = Sweep2D(insts, device=dev, seeds=[1000 * rank + k for k in range(len(insts))])
    cells = sw.cells
    snap = sw.snapshot()
    if args.tuning:   # a given launch shape instead of the autotuner (lcap,ctas_per_sm,order,schedule,tiles)
        lcap, cps, order, sched, tiles = args.tuning.split(",")
        cand = (int(lcap), int(cps), int(order), sched, int(tiles))
        sw.use_persistent(*cand)
        tune_table = [(sw.tuning, None, "given")]
    else:
        tune_table = sw.tune()
    K = args.steps
    for _ in range(args.warmup):
        sw.step("persistent")
    torch.cuda.synchronize()
    g = sw.capture(K, "persistent")
    ms, clk = _time_graph(g, dist, local_rank, rank, dev)
    status = sw.status()
    coeffs = {mine[k]: [float(x) for x in sw.states[k]["out"]["coeffs"].reshape(-1)[:2].tolist()]
              for k in range(len(insts))}
    del g
    timings = {}
    for sched in ("streams", "loop"):
        sw.restore(snap)
        for _ in range(args.warmup):
            sw.step(sched)
        gs = sw.capture(K, sched)
        timings[sched], _ = _time_graph(gs, dist, local_rank, rank, dev)
        del gs
    # e2e: host state in, host results out, every step, through the sweep's public calls
    sw.restore(snap)
    host_in = [(s["u"].cpu().pin_memory(), s["v"].cpu().pin_memory(), s["t"].cpu().pin_memory()) for s in sw.states]
    host_out = [(torch.empty(s["t"].shape, dtype=s["t"].dtype).pin_memory(),
                 torch.empty(s["out"]["coeffs"].shape, dtype=s["out"]["coeffs"].dtype).pin_memory())
                for s in sw.states]
    h2d = sum(a.numel() * a.element_size() + b.numel() * b.element_size() + c.numel() * c.element_size()
              for a, b, c in host_in)
    d2h = sum(a.numel() * a.element_size() + b.numel() * b.element_size() for a, b in host_out)
    ke = max(3, min(K, 10))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(ke):
        for s, (hu, hv, ht) in zip(sw.states, host_in):
            s["u"].copy_(hu, non_blocking=True)
            s["v"].copy_(hv, non_blocking=True)
            s["t"].copy_(ht, non_blocking=True)
        sw.step("persistent")
        for s, (ht, hc) in zip(sw.states, host_out):
            ht.copy_(s["t"], non_blocking=True)
            hc.copy_(s["out"]["coeffs"], non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    ems = max_over_ranks(e0.elapsed_time(e1) / ke, dist, dev)
    coeffs = gather_results(coeffs, dist)
    total_cells = sum(o.nx * o.ny for o, _, _ in all_insts) if args.shard else world * cells
    if rank != 0:
        return
    peak, peak_kind = _peaks()
    alg = 228.0 * cells
    cpu = None
    if not args.no_cpu:
        ops0, geom0, _ = all_insts[0]
        cpu = cpu_baseline_2d("sweep2d", lambda n: oracle2d_sample(ops0, geom0, n), ops0.nx * ops0.ny,
                              f"steps of the sweep's first ({ops0.nx}x{ops0.ny}) instance")
    grids = {}
    for o, _, _ in insts:
        grids[f"{o.nx}x{o.ny}"] = grids.get(f"{o.nx}x{o.ny}", 0) + 1
    info = sw._persistent["info"]
    ref_loop = None
    if not args.no_ref_gpu and not args.shard:
        try:
            ref_ms, ref_cells = time_reference_gpu_sweep(dev, n=args.instances)
            ref_loop = {"ms_per_step": ref_ms, "value": ref_cells / (ref_ms * 1e-3) / 1e6, "unit": UNIT,
                        "speedup_of_persistent": ref_ms / (ms / K),
                        "how": "the reference's own 2D FlowSolver.advance (baseline/_ref, unmodified, its CUDA "
                               f"graphs) over the same {args.instances} instances one after another on this GPU, "
                               "10 steps each "
                               "after 3 warm-up steps, CUDA events; the sum of the per-instance step times"}
        except ImportError as exc:
            ref_loop = {"unavailable": f"reference not installed: {exc}"}
    line = {"metric": METRIC, "value": total_cells * K / (ms * 1e-3) / 1e6, "unit": UNIT, "n_gpus": world,
            "steps": K, "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True,
            "scaling": "strong" if args.shard else "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batched sweep: {args.instances} NACA 4-digit airfoils, seeded grids "
                                   "256x128..1024x512 FP32, "
                                   "upwind3, CFL 0.5, no LES", "cells": cells, "grids": grids,
                       "inputs_vs_l2": f"{cells * 4 * 10 / 1e6:.0f} MB of state + workspace > 126 MB L2 (no flush)",
                       "parallelism": "instances sharded over the ranks" if args.shard else "replicas",
                       "graph": f"{K} sweep steps, each one persistent launch, 1 replay"},
            "persistent": {"tuning": {"lcap": sw.tuning[0], "ctas_per_sm": sw.tuning[1],
                                      "order": "largest first" if sw.tuning[2] else "as given",
                                      "schedule": sw.tuning[3], "tiles_per_item": sw.tuning[4]},
                           "phases": info["phases"], "operations": info["operations"],
                           "work_items_per_step": info["items"], "ctas": info["ctas"],
                           "dynamic_smem": info["smem"], "status": status,
                           "autotuner": [{"lcap": c[0], "ctas_per_sm": c[1], "order": c[2], "schedule": c[3],
                                          "tiles": c[4], "ms_per_step": t}
                                         for c, t, _ in tune_table]},
            "instances": len(coeffs), "instances_per_rank": len(mine) if not args.shard else "size-balanced shard",
            "streams": {"value": total_cells * K / (timings["streams"] * 1e-3) / 1e6, "unit": UNIT,
                        "ms_per_step": timings["streams"] / K, "how": "each instance's own launches over 16 streams"},
            "looped": {"value": total_cells * K / (timings["loop"] * 1e-3) / 1e6, "unit": UNIT,
                       "ms_per_step": timings["loop"] / K,
                       "how": "the plain per-instance loop: the same plans one after another on one stream"},
            "speedup_vs_loop": timings["loop"] / ms,
            "reference_gpu_loop": ref_loop,
            "roofline": {"bound": "hbm", "kernel": "sweep2d_kernel (the whole sweep step)",
                         "achieved": alg / (ms / K * 1e-3) / 1e9, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": alg / (ms / K * 1e-3) / 1e9 / peak, "traffic": None, "alg_bytes_per_step": alg},
            "cpu_baseline": cpu,
            "e2e": {"value": total_cells / (ems * 1e-3) / 1e6, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": ems, "steps": ke},
            "gpu_launches": K, "clocks": clk}
    print(json.dumps(line), flush=True)


FIELDS_METRIC = "Mcell/s of field outputs (7 cell fields per pass) on 1 B200"
FIELDS_UNIT = "Mcell/s"


def _fields_oracle(u, v, w, ops, geom):
    """The oracle's seven fields of one state (chi_c on the body window as the eddy-viscosity mask)."""
    from oracle import fields3d as F
    mask = None
    if not geom.empty:
        k0, k1, j0, j1, i0, i1 = geom.window
        mask = np.zeros(u[..., 1:].shape, u.dtype)
        mask[k0:k1, j0:j1, i0:i1] = geom.chi_c
    return [F.centre_u(u), F.centre_v(v), F.centre_w(w), F.speed(u, v, w)] + \
        [F.gradient_field(n, u, v, w, ops, mask) for n in ("vorticity", "q", "nut")]


def _fields_setup(shape, device):
    from aerolume_b200.ns3d.workloads import box_on_moving_floor, initial_state
    nx, ny, nz = shape
    ops, geom, th, src, _ = box_on_moving_floor(nx, ny, nz, dtype="float32")
    u, v, w = initial_state(ops, device=device)
    return ops, geom, th, src, u, v, w


def run_fields(args, rank, world, local_rank):
    import torch
    from aerolume_b200 import _lib
    from aerolume_b200.ns3d.plan import Ns3dPlan
    dist = None
    if world > 1:
        import torch.distributed as dist
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    nx, ny, nz = args.shape
    cells = nx * ny * nz
    ops, geom, th, src, u, v, w = _fields_setup(args.shape, dev)
    plan = Ns3dPlan(ops, geom, th, src, smoke=True, device=dev)
    names = _lib.FIELD_NAMES
    for _ in range(args.warmup):
        plan.fields(u, v, w, names)
    torch.cuda.synchronize()
    K = args.steps
    s = torch.cuda.Stream(device=dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            for _ in range(K):
                plan.fields(u, v, w, names)
    torch.cuda.current_stream(dev).wait_stream(s)
    ms, clk = _time_graph(g, dist, local_rank, rank, dev)
    # probes: a million seeded points in the domain, trilinear samples of the speed field
    speed = plan.fields(u, v, w, ("speed",))["speed"]
    gen = torch.Generator(device="cpu").manual_seed(0)
    ext = torch.tensor([nx, ny, nz], dtype=torch.float32) * float(ops.h)
    pts = (torch.rand(1 << 20, 3, generator=gen) * ext).to(dev).contiguous()
    for _ in range(3):
        plan.probe(speed, pts)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(K):
        plan.probe(speed, pts)
    e1.record()
    torch.cuda.synchronize()
    probe_ms = e0.elapsed_time(e1) / K
    # e2e: state in from pinned host memory, the seven fields back out
    host_in = [torch.empty(x.shape, dtype=x.dtype, pin_memory=True).copy_(x) for x in (u, v, w)]
    host_out = [torch.empty((nz, ny, nx), dtype=u.dtype, pin_memory=True) for _ in names]
    d_in = [torch.empty_like(x) for x in (u, v, w)]
    torch.cuda.synchronize()
    ke = max(3, min(K, 10))
    e0.record()
    for _ in range(ke):
        for d, h in zip(d_in, host_in):
            d.copy_(h, non_blocking=True)
        res = plan.fields(*d_in, names)
        for h, n in zip(host_out, names):
            h.copy_(res[n], non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1) / ke
    if rank != 0:
        return
    peak, peak_kind = _peaks()
    # algorithmic bytes per pass, FP32: the three face arrays read once, seven cell fields written
    alg = 4 * (u.numel() + v.numel() + w.numel() + len(names) * cells)
    achieved = alg / (ms / K * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu:
        un, vn, wn = (x.cpu().numpy() for x in (u, v, w))
        _fields_oracle(un, vn, wn, ops, geom)
        t0 = time.perf_counter()
        _fields_oracle(un, vn, wn, ops, geom)
        secs = time.perf_counter() - t0
        cpu = {"value": cells / secs / 1e6, "unit": FIELDS_UNIT, "cores": _threads(), "kind": "port",
               "sample": f"one full {nx}x{ny}x{nz} pass of the numpy field oracle after 1 untimed pass"}
    line = {"metric": FIELDS_METRIC, "value": world * cells * K / (ms * 1e-3) / 1e6, "unit": FIELDS_UNIT,
            "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"field outputs of the box-on-moving-floor state {nx}x{ny}x{nz} FP32 (WALE)",
                       "fields": list(names), "inputs_vs_l2": "67 MB in + 117 MB out per pass > 126 MB L2",
                       "parallelism": "replicas", "graph": f"{K} passes, 1 replay"},
            "roofline": {"bound": "hbm", "kernel": "fields_kernel", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                         "alg_bytes_per_launch": alg},
            "probes": {"value": (1 << 20) / (probe_ms * 1e-3) / 1e6, "unit": "Mpoints/s", "ms": probe_ms,
                       "points": 1 << 20, "field": "speed"},
            "cpu_baseline": cpu,
            "e2e": {"value": world * cells / (ems * 1e-3) / 1e6, "unit": FIELDS_UNIT,
                    "h2d_bytes_per_step": int(sum(x.numel() * x.element_size() for x in host_in)),
                    "d2h_bytes_per_step": int(sum(x.numel() * x.element_size() for x in host_out)),
                    "ms_per_step": ems, "steps": ke},
            "gpu_launches": K, "clocks": clk, "status": plan.status()}
    print(json.dumps(line), flush=True)


def run_reference_fields(args, rank):
    if rank != 0:
        return
    nx, ny, nz = args.shape
    ops, geom, _, _, u, v, w = _fields_setup(args.shape, "cpu")
    un, vn, wn = (x.numpy() for x in (u, v, w))
    _fields_oracle(un, vn, wn, ops, geom)
    steps = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(steps):
        _fields_oracle(un, vn, wn, ops, geom)
    secs = time.perf_counter() - t0
    val = nx * ny * nz * steps / secs / 1e6
    line = {"impl": "reference", "metric": FIELDS_METRIC, "value": val, "unit": FIELDS_UNIT, "n_gpus": args.gpus,
            "steps": steps, "warmup": 1, "ms_per_step": 1e3 * secs / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"field outputs of the box-on-moving-floor state {nx}x{ny}x{nz} FP32 (WALE)"},
            "cpu_baseline": {"value": val, "unit": FIELDS_UNIT, "cores": _threads(), "kind": "port",
                             "sample": f"{steps} full passes of the numpy field oracle after 1 untimed pass"},
            "e2e": {"value": val, "unit": FIELDS_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)



# ---------------------------------------------------------------------------------------
# mask construction
# ---------------------------------------------------------------------------------------
MASKS_METRIC = "mask rebuilds/s of a 9024-triangle sphere on the 256x128x128 grid on 1 B200"
MASKS_UNIT = "rebuilds/s"
# FP32 operations of one point-triangle pair in the search kernel, counted from its source: the
# solid angle, which every pair needs (85: three norms, triple product, denominator, plus 3
# square roots and 1 atan2 counted as one each).  The squared distance (148 more: edges,
# normal, three edge-side tests, three segment distances) runs only for the triangles whose
# bounding ball does not rule them out, so this is a lower bound of the work done.
FLOP_PER_PAIR = 85 + 4
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12   # SMs x FP32 lanes x FMA x max clock


def _masks_setup(shape):
    from aerolume_b200.ns3d.masks import body_window3d
    from aerolume_b200.ns3d.workloads import box_on_moving_floor, sphere_mesh
    nx, ny, nz = shape
    ops = box_on_moving_floor(nx, ny, nz, dtype="float32")[0]
    v, f = sphere_mesh((2.5, 2.0, 1.0), 0.5)
    win = body_window3d([v], ops)
    wz, wy, wx = win[1] - win[0], win[3] - win[2], win[5] - win[4]
    npts = (wx + 1) * wy * wz + wx * (wy + 1) * wz + wx * wy * (wz + 1) + wx * wy * wz
    return ops, v, f, win, npts


def run_masks(args, rank, world, local_rank):
    import torch
    from aerolume_b200.ns3d.masks import build_geometry3d
    from aerolume_b200.ns3d.types import Geometry3D
    dist = None
    if world > 1:
        import torch.distributed as dist
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    ops, v, f, win, npts = _masks_setup(args.shape)
    pairs = npts * len(f)
    body = (torch.as_tensor(v, dtype=torch.float32).to(dev), f)     # vertices resident on the device
    # a live attitude edit keeps its window (and the graphs captured on it): pass it in
    for _ in range(args.warmup):
        build_geometry3d([body], ops, window=win, device=dev)
    torch.cuda.synchronize()
    K = args.steps
    mon = Clocks(local_rank)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(K):
        g = build_geometry3d([body], ops, window=win, device=dev)
    e1.record()
    torch.cuda.synchronize()
    clk = mon.stop()
    ms = e0.elapsed_time(e1) / K
    if dist is not None:
        from aerolume_b200.replicas import max_over_ranks
        ms = max_over_ranks(ms, dist, dev)
    # e2e: the mesh from host memory each time, the ten mask arrays back to pinned host memory
    names = [n for n in Geometry3D.__dataclass_fields__ if n.startswith(("chi_", "a_", "k_"))]
    host_out = {n: torch.empty(getattr(g, n).shape, dtype=g.chi_c.dtype, pin_memory=True) for n in names}
    ke = max(3, min(K, 10))
    torch.cuda.synchronize()
    e0.record()
    for _ in range(ke):
        gh = build_geometry3d([(v, f)], ops, window=win, device=dev)
        for n in names:
            host_out[n].copy_(getattr(gh, n), non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1) / ke
    if rank != 0:
        return
    achieved = pairs * FLOP_PER_PAIR / (ms * 1e-3) / 1e12
    cpu = None
    if not args.no_cpu:
        cpu = _masks_cpu_sample(v, f, ops, win, pairs)
    line = {"metric": MASKS_METRIC, "value": world * 1e3 / ms, "unit": MASKS_UNIT, "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "masks of a closed sphere D = 1 (48 x 96 latitude-longitude mesh, 9024 triangles) "
                                   "at 32 cells per diameter in the 256x128x128 tunnel, exact signed distance",
                       "window": list(win), "points": npts, "triangles": len(f), "pairs_per_rebuild": pairs,
                       "inputs_vs_l2": "compute-bound search; 0.1 MB mesh, 5 MB of masks", "parallelism": "replicas"},
            "pairs_per_s": pairs * 1e3 / ms,
            "roofline": {"bound": "fp32", "kernel": "sdf_search_kernel", "achieved": achieved,
                         "peak": FP32_NOMINAL_TFLOPS, "peak_kind": "nominal FP32 CUDA-core rate", "unit": "TFLOP/s",
                         "frac": achieved / FP32_NOMINAL_TFLOPS, "traffic": None,
                         "flop_per_pair": FLOP_PER_PAIR},
            "cpu_baseline": cpu,
            "e2e": {"value": world * 1e3 / ems, "unit": MASKS_UNIT,
                    "h2d_bytes_per_step": int(v.size * 4 + f.size * 4),
                    "d2h_bytes_per_step": int(sum(x.numel() * x.element_size() for x in host_out.values())),
                    "ms_per_step": ems, "steps": ke},
            "gpu_launches": K * 16, "clocks": clk}
    print(json.dumps(line), flush=True)


def _masks_cpu_sample(v, f, ops, win, pairs, npoint=4096):
    """The numpy oracle's signed distance at npoint seeded window points (rebuilds/s scaled by
    the pairs of a full rebuild)."""
    from oracle import masks3d as M
    rng = np.random.default_rng(0)
    k0, k1, j0, j1, i0, i1 = win
    lo = np.array([ops.x0 + i0 * ops.h, ops.y0 + j0 * ops.h, ops.z0 + k0 * ops.h])
    hi = np.array([ops.x0 + i1 * ops.h, ops.y0 + j1 * ops.h, ops.z0 + k1 * ops.h])
    p = rng.uniform(lo, hi, size=(npoint, 3)).astype(np.float32)
    vf = v.astype(np.float32)
    M.mesh_signed_distance(vf, f, p[:256], chunk=128)
    t0 = time.perf_counter()
    M.mesh_signed_distance(vf, f, p, chunk=128)
    secs = time.perf_counter() - t0
    rate = npoint * len(f) / secs
    return {"value": rate / pairs, "unit": MASKS_UNIT, "cores": _threads(), "kind": "port",
            "sample": f"numpy signed distance of {npoint} seeded window points to the {len(f)} triangles "
                      f"({npoint * len(f) / 1e6:.0f} M pairs), scaled to a full rebuild of {pairs / 1e9:.2f} G pairs"}


def run_reference_masks(args, rank):
    if rank != 0:
        return
    ops, v, f, win, npts = _masks_setup(args.shape)
    cpu = _masks_cpu_sample(v, f, ops, win, npts * len(f))
    val = cpu["value"]
    line = {"impl": "reference", "metric": MASKS_METRIC, "value": val, "unit": MASKS_UNIT, "n_gpus": args.gpus,
            "steps": 1, "warmup": 1, "ms_per_step": 1e3 / val, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "masks of a closed sphere D = 1 (9024 triangles) at 32 cells per diameter in the "
                                   "256x128x128 tunnel, exact signed distance"},
            "cpu_baseline": cpu,
            "e2e": {"value": val, "unit": MASKS_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)



# ---------------------------------------------------------------------------------------
# placed physics in the 3D step
# ---------------------------------------------------------------------------------------
PLACED_DESC = ("box on moving floor {}x{}x{} FP32, WALE, Boussinesq heat, with a swirling velocity-regulated fan, "
               "a warm jet and a vent, a painted block and the PID step controller (no smoke)")


def _placed_cpu(shape, steps=1):
    """Seconds of ``steps`` oracle steps (after one untimed step) of the placed-physics case."""
    from aerolume_b200.ns3d.workloads import placed_box
    from oracle import ns3d as O
    nx, ny, nz = shape
    f32 = np.float32
    ops, geom, th, fans, ports, paint, pid_target, u_floor = placed_box(nx, ny, nz, dtype="float32")
    g32 = type(geom)(geom.window, nbody=geom.nbody)
    for n in ("chi_u", "chi_v", "chi_w", "chi_c", "a_u", "a_v", "a_w", "k_u", "k_v", "k_w"):
        setattr(g32, n, np.asarray(getattr(geom, n), f32))
    items = [{"win": it["win"], "f": tuple(np.asarray(it["f" + g], f32) for g in "uvw"),
              "s": tuple(np.asarray(it["s" + g], f32) for g in "uvw"),
              "m": tuple(np.asarray(it["m" + g], f32) for g in "uvw")} for it in fans["items"]]
    fs = O.FanState(items, fans["target"], fans["kp"], fans["ki"], fans["tmax"], fans["velocity_mode"], fans["swirl"],
                    fans["any_swirl"], fans["thrust"], f32)
    pitems = [{"win": it["win"], "kind": it["kind"], "theta": it["theta"], "m": np.asarray(it["m"], f32),
               "f": tuple(np.asarray(it["f" + g], f32) for g in "uvw")} for it in ports["items"]]
    ps_ = O.PortState(pitems, ports["mass_flux"], ports["leak"])
    pnt = tuple(np.asarray(paint[g], f32) for g in "uvw")
    pid = O.PidState(pid_target, f32)
    ps = O.PoissonSolver3D(nx, ny, nz, ops.h, ops.periodic_axes, f32)
    rng = np.random.default_rng(0)
    u = (np.ones((nz, ny, nx + 1)) + 1e-3 * rng.standard_normal((nz, ny, nx + 1))).astype(f32)
    v = (1e-3 * rng.standard_normal((nz, ny + 1, nx))).astype(f32)
    w = (1e-3 * rng.standard_normal((nz + 1, ny, nx))).astype(f32)
    theta = np.zeros((nz, ny, nx), f32)
    kw = dict(th=th, paint=pnt, pid=pid, u_floor=u_floor, fans=fs, ports=ps_)
    r = O.step3d_phys(u, v, w, f32(0), g32, ops, ps, theta=theta, **kw)
    t0 = time.perf_counter()
    for _ in range(steps):
        r = O.step3d_phys(r.u, r.v, r.w, r.t, g32, ops, ps, theta=r.theta, **kw)
    return time.perf_counter() - t0


def run_reference_placed(args, rank):
    if rank != 0:
        return
    nx, ny, nz = args.shape
    steps = max(1, min(args.steps, 2))
    secs = _placed_cpu(args.shape, steps)
    val = nx * ny * nz * steps / secs / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "warmup": 1, "ms_per_step": 1e3 * secs / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": PLACED_DESC.format(nx, ny, nz)},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": _threads(), "kind": "port",
                             "sample": f"{steps} full steps of the numpy oracle after 1 untimed step"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_placed(args, rank, world, local_rank):
    import torch
    from aerolume_b200.ns3d.plan import Ns3dPlan
    from aerolume_b200.ns3d.workloads import initial_state, placed_box, placed_state
    dist = None
    if world > 1:
        import torch.distributed as dist
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    nx, ny, nz = args.shape
    cells = nx * ny * nz
    ops, geom, th, fans, ports, paint, pid_target, u_floor = placed_box(nx, ny, nz, dtype="float32")
    fs, ps, pl, pid = placed_state(fans, ports, paint, pid_target, dev, "float32")
    plan = Ns3dPlan(ops, geom, th, None, device=dev, paint=pl, pid=pid, u_floor=u_floor, fans=fs, ports=ps)
    plain = Ns3dPlan(ops, geom, th, None, device=dev)
    u, v, w = initial_state(ops, seed=rank, device=dev)
    plan.project(u, v, w)
    theta = torch.zeros(nz, ny, nx, device=dev)
    t = torch.zeros((), device=dev)
    state0 = [x.clone() for x in (u, v, w, theta)]

    def runner(pl_):
        out = pl_.empty_fields()
        out["u"], out["v"], out["w"], out["theta"] = u, v, w, theta

        def step():
            pl_.step(u, v, w, t, theta0=theta, out=out)
            t.copy_(out["t"])
        return step, out

    res = {}
    for name, pl_ in (("placed", plan), ("plain", plain)):
        for x, x0 in zip((u, v, w, theta), state0):
            x.copy_(x0)
        step, out = runner(pl_)
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        K = args.steps
        s_ = torch.cuda.Stream(device=dev)
        s_.wait_stream(torch.cuda.current_stream(dev))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s_):
            with torch.cuda.graph(g, stream=s_):
                for _ in range(K):
                    step()
        torch.cuda.current_stream(dev).wait_stream(s_)
        ms, clk = _time_graph(g, dist, local_rank, rank, dev)
        res[name] = (ms / K, clk, pl_.status())
        del g
    # e2e of the placed step: state in from pinned host memory, state and coefficients out
    host_in = {k: x.cpu().pin_memory() for k, x in (("u", u), ("v", v), ("w", w), ("theta", theta), ("t", t))}
    o2 = plan.empty_fields()
    host_out = {k: torch.empty(x.shape, dtype=x.dtype, pin_memory=True) for k, x in o2.items()}
    d_in = {k: torch.empty_like(x, device=dev) for k, x in host_in.items()}
    ke = max(3, min(args.steps, 10))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(ke):
        for k in host_in:
            d_in[k].copy_(host_in[k], non_blocking=True)
        plan.step(d_in["u"], d_in["v"], d_in["w"], d_in["t"], theta0=d_in["theta"], out=o2)
        for k in host_out:
            host_out[k].copy_(o2[k], non_blocking=True)
        for k in ("u", "v", "w", "theta", "t"):
            host_in[k], host_out[k] = host_out[k], host_in[k]
    e1.record()
    torch.cuda.synchronize()
    ems = max_over_ranks(e0.elapsed_time(e1) / ke, dist, dev)
    if rank != 0:
        return
    ms_step, clk, status = res["placed"]
    peak, peak_kind = _peaks()
    cpu = None
    if not args.no_cpu:
        secs = _placed_cpu(args.shape, 1)
        cpu = {"value": cells / secs / 1e6, "unit": UNIT, "cores": _threads(), "kind": "port",
               "sample": f"1 full {nx}x{ny}x{nz} step of the numpy oracle after 1 untimed step"}
    # compulsory bytes per cell-step, FP32: plain 284 + theta 32 + LES pre-pass 12, and the
    # painted solid fractions read once per stage (4 arrays, 48 B)
    alg = (284.0 + 32.0 + 12.0 + 48.0) * cells
    line = {"metric": METRIC, "value": world * cells / (ms_step * 1e-3) / 1e6, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": PLACED_DESC.format(nx, ny, nz), "cells": cells,
                       "inputs_vs_l2": "working set ~1 GB > 126 MB L2 (no flush)", "parallelism": "replicas",
                       "graph": f"{args.steps} steps, 1 replay"},
            "plain_same_case": {"ms_per_step": res["plain"][0],
                                "value": cells / (res["plain"][0] * 1e-3) / 1e6, "status": res["plain"][2]},
            "roofline": {"bound": "hbm", "kernel": "whole step", "achieved": alg / (ms_step * 1e-3) / 1e9,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": alg / (ms_step * 1e-3) / 1e9 / peak, "traffic": None, "alg_bytes_per_step": alg},
            "cpu_baseline": cpu,
            "e2e": {"value": world * cells / (ems * 1e-3) / 1e6, "unit": UNIT,
                    "h2d_bytes_per_step": int(sum(x.numel() * x.element_size() for x in host_in.values())),
                    "d2h_bytes_per_step": int(sum(x.numel() * x.element_size() for x in host_out.values())),
                    "ms_per_step": ems, "steps": ke},
            "gpu_launches": launches_per_step(plan) * args.steps, "clocks": clk, "status": status}
    print(json.dumps(line), flush=True)



# ---------------------------------------------------------------------------------------
# per-step bookkeeping (history rows, running means)
# ---------------------------------------------------------------------------------------
RECORD_METRIC = "Mcell-samples/s of the running-mean update (u, v, w, p, theta) on 1 B200"
RECORD_UNIT = "Mcell/s"


def _record_state(shape, device, dtype="float32"):
    import torch
    from types import SimpleNamespace
    nx, ny, nz = shape
    tdt = torch.float64 if dtype == "float64" else torch.float32
    g = torch.Generator(device="cpu").manual_seed(5)
    shapes = {"u": (nz, ny, nx + 1), "v": (nz, ny + 1, nx), "w": (nz + 1, ny, nx), "p": (nz, ny, nx),
              "t": (nz, ny, nx)}
    f = {k: torch.randn(sh, generator=g).to(device, tdt) for k, sh in shapes.items()}
    avg = {"time": torch.zeros((), device=device, dtype=torch.float64),
           "pending": torch.zeros((), device=device, dtype=torch.float64)}
    for k, sh in shapes.items():
        avg[k] = torch.zeros(sh, device=device, dtype=tdt)
        avg[k + "2"] = torch.zeros(sh, device=device, dtype=tdt)
    self = SimpleNamespace(dtype=tdt, _body_c=torch.zeros(1, 6, device=device, dtype=tdt),
                           _hist=torch.zeros(4096, 7, device=device, dtype=tdt),
                           _hist_n=torch.zeros((), device=device, dtype=torch.int64), _phist=None,
                           _phist_walls=False, _avg_on=True, _avg=avg, _theta=f["t"], _phys=None)
    new = SimpleNamespace(u=f["u"], v=f["v"], w=f["w"], p=f["p"], t=torch.ones((), device=device, dtype=tdt),
                          dt=torch.full((), 0.01, device=device, dtype=tdt))
    bc = torch.zeros(1, 6, device=device, dtype=tdt)
    return self, new, bc, f, avg


def run_record(args, rank, world, local_rank):
    import torch
    from aerolume_b200.ns3d.record import record
    dist = None
    if world > 1:
        import torch.distributed as dist
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    nx, ny, nz = args.shape
    cells = nx * ny * nz
    self, new, bc, f, avg = _record_state(args.shape, dev)
    for _ in range(args.warmup):
        record(self, new, bc, True)
    torch.cuda.synchronize()
    K = args.steps
    s_ = torch.cuda.Stream(device=dev)
    s_.wait_stream(torch.cuda.current_stream(dev))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s_):
        with torch.cuda.graph(g, stream=s_):
            for _ in range(K):
                record(self, new, bc, True)
    torch.cuda.current_stream(dev).wait_stream(s_)
    ms, clk = _time_graph(g, dist, local_rank, rank, dev)
    if rank != 0:
        return
    peak, peak_kind = _peaks()
    # compulsory bytes of one sample: each field read once and its mean and second moment read
    # and written once (5 words per element), FP32
    elems = sum(x.numel() for x in f.values())
    alg = 4.0 * 5 * elems
    achieved = alg / (ms / K * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu:
        cpu = _record_cpu(args.shape)
    line = {"metric": RECORD_METRIC, "value": world * cells * K / (ms * 1e-3) / 1e6, "unit": RECORD_UNIT,
            "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"history row and running-mean sample of u, v, w, p, theta at {nx}x{ny}x{nz} FP32",
                       "inputs_vs_l2": f"{alg / 1e6:.0f} MB per sample > 126 MB L2", "parallelism": "replicas",
                       "graph": f"{K} samples, 1 replay"},
            "roofline": {"bound": "hbm", "kernel": "welford_kernel", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                         "alg_bytes_per_launch": alg},
            "cpu_baseline": cpu,
            "e2e": None, "gpu_launches": 3 * K, "clocks": clk}
    print(json.dumps(line), flush=True)


def _record_cpu(shape):
    """The numpy oracle's sample (history row + Welford of five fields) on the full grid."""
    from oracle import record3d as R
    nx, ny, nz = shape
    rng = np.random.default_rng(5)
    shapes = {"u": (nz, ny, nx + 1), "v": (nz, ny + 1, nx), "w": (nz + 1, ny, nx), "p": (nz, ny, nx),
              "t": (nz, ny, nx)}
    f = {k: rng.standard_normal(sh).astype(np.float32) for k, sh in shapes.items()}
    avg = {"time": np.float64(0), "pending": np.float64(0)}
    for k, sh in shapes.items():
        avg[k], avg[k + "2"] = np.zeros(sh, np.float32), np.zeros(sh, np.float32)
    buf = {"hist": np.zeros((4096, 7), np.float32), "hist_n": 0, "body_c": np.zeros((1, 6), np.float32),
           "phist": None, "avg": avg}
    bc = np.zeros((1, 6), np.float32)
    R.record(buf, 1.0, 0.01, bc, True, fields=f)
    t0 = time.perf_counter()
    R.record(buf, 1.0, 0.01, bc, True, fields=f)
    secs = time.perf_counter() - t0
    return {"value": nx * ny * nz / secs / 1e6, "unit": RECORD_UNIT, "cores": _threads(), "kind": "port",
            "sample": f"one full {nx}x{ny}x{nz} sample of the numpy oracle after 1 untimed sample"}


def run_reference_record(args, rank):
    if rank != 0:
        return
    nx, ny, nz = args.shape
    cpu = _record_cpu(args.shape)
    val = cpu["value"]
    line = {"impl": "reference", "metric": RECORD_METRIC, "value": val, "unit": RECORD_UNIT, "n_gpus": args.gpus,
            "steps": 1, "warmup": 1, "ms_per_step": nx * ny * nz / val / 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"history row and running-mean sample of u, v, w, p, theta at {nx}x{ny}x{nz} FP32"},
            "cpu_baseline": cpu, "e2e": {"value": val, "unit": RECORD_UNIT, "h2d_bytes_per_step": 0,
                                         "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def reference_2d_config(workload, device, instance=0):
    """The reference's 2D SolverConfig of a 2D bench workload: the cylinder tunnel (config [0]),
    the same with the cylinder held at theta = 1, or NACA instance ``instance`` of the sweep."""
    from aerolume_b200.ns2d.workloads import circle, naca4, sweep_instances
    _reference_api()                                  # baseline/_ref on the path (ImportError if absent)
    import aerolume.solvers.ns2d.config as C2
    kw = dict(bc_top="slip", bc_bottom="slip", advection="upwind3", cfl=0.5, dtype="float32", device=device,
              dye=False, perturb=False)
    if workload == "sweep2d":
        ops, _, prm = sweep_instances(max(64, instance + 1), seed=0)[instance]
        body = C2.ImmersedBody(naca4(prm["t"], prm["m"], prm["p"], prm["alpha"]), name="naca")
        return C2.SolverConfig(nx=ops.nx, ny=ops.ny, h=8.0 / ops.nx, x0=0.0, y0=0.0, re=prm["re"], bodies=[body],
                               force_ref=1.0, moment_ref=(2.0, 2.0), **kw), f"{ops.nx}x{ops.ny}"
    thermal = None
    cyl = C2.ImmersedBody(circle(2.0, 2.0, 0.25, 256), name="cylinder",
                          **({"thermal": "temperature", "thermal_value": 1.0} if workload == "heated2d" else {}))
    if workload == "heated2d":
        thermal = C2.ThermalConfig(prandtl=0.71, richardson=0.5)
    return C2.SolverConfig(nx=256, ny=128, h=1.0 / 32.0, x0=0.0, y0=0.0, re=200.0, bodies=[cyl], force_ref=0.5,
                           moment_ref=(2.0, 2.0), thermal=thermal, **kw), "256x128"


def time_reference_gpu_sweep(dev, steps=10, warm=3, n=64):
    """The reference's own 2D solver (baseline/_ref, unmodified, FlowSolver.advance with its CUDA
    graphs) looping over the sweep's 64 instances on this GPU: each instance built, warmed up and
    timed on its own (CUDA events around ``steps`` steps); the loop's time per sweep step is the
    sum of the per-instance step times."""
    import torch
    _reference_api()
    import aerolume.solvers.ns2d.solver as S2
    total, cells = 0.0, 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for k in range(n):
        cfg, _ = reference_2d_config("sweep2d", str(dev), k)
        s = S2.FlowSolver(cfg)
        s.advance(warm)
        torch.cuda.synchronize()
        e0.record()
        s.advance(steps)
        e1.record()
        torch.cuda.synchronize()
        total += e0.elapsed_time(e1) / steps
        cells += cfg.nx * cfg.ny
        del s
    torch.cuda.empty_cache()
    return total, cells


def time_reference_cpu_2d(workload, steps, warm, repeats=3):
    """Best-of-``repeats`` wall time per step of the reference's 2D FlowSolver.advance on the
    host cores (device "cpu", FP32, all threads) after ``warm`` untimed steps."""
    import torch
    _reference_api()
    import aerolume.solvers.ns2d.solver as S2
    cfg, grid = reference_2d_config(workload, "cpu")
    old = torch.get_num_threads()
    torch.set_num_threads(os.cpu_count() or 1)
    try:
        s = S2.FlowSolver(cfg)
        s.advance(warm)
        best = float("inf")
        for _ in range(repeats):
            t0 = time.perf_counter()
            s.advance(steps)
            best = min(best, (time.perf_counter() - t0) / steps)
        return best, torch.get_num_threads(), cfg.nx * cfg.ny, grid
    finally:
        torch.set_num_threads(old)


def run_reference_2d(args, rank):
    """``--impl reference`` of the 2D workloads: the reference's own 2D solver on the host cores."""
    if rank != 0:
        return
    steps = max(1, min(args.steps, 50))
    try:
        per_step, cores, cells, grid = time_reference_cpu_2d(args.workload, steps, 2)
    except ImportError as exc:
        print(json.dumps({"impl": "reference", "unavailable": f"reference not installed: {exc}"}), flush=True)
        return
    desc = {"cylinder2d": "cylinder D=0.5 at (2,2), 256x128 FP32, Re_D 100, slip walls, upwind3, CFL 0.5",
            "heated2d": HEATED_2D}.get(args.workload, f"one {grid} instance of the batched NACA sweep")
    val = cells / per_step / 1e6
    sample = (f"best of 3 x {steps} steps of the reference's 2D FlowSolver.advance (device cpu, FP32, {cores} "
              f"threads) on {desc} after 2 untimed steps")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "warmup": 2, "ms_per_step": 1e3 * per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": {"workload": desc},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default 20; 400 for cylinder2d, "
                                                             "10 for sweep2d)")
    ap.add_argument("--workload", default="box3d",
                    choices=["box3d", "placed3d", "cylinder2d", "heated2d", "sweep2d", "fields3d", "masks3d",
                             "record3d", "closure3d"])
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--shape", type=int, nargs=3, default=list(SHAPE), help="nx ny nz (2:1:1)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip timing the reference's CUDA step")
    ap.add_argument("--tuning", default=None,
                    help="sweep2d: lcap,ctas_per_sm,order,schedule,tiles instead of the autotuner (e.g. 2,3,1,queue,4)")
    ap.add_argument("--instances", type=int, default=64,
                    help="sweep2d: instances of the sweep (the first n of the seeded 64; the headline uses 64)")
    ap.add_argument("--shard", action="store_true",
                    help="sweep2d with N > 1: split the 64 instances over the ranks instead of replicating them")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = {"box3d": 20, "placed3d": 20, "cylinder2d": 400, "heated2d": 400, "sweep2d": 10,
                      "fields3d": 20, "masks3d": 10, "record3d": 20, "closure3d": 20}[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if args.workload in ("box3d", "closure3d"):   # the reference has no learned closure: its WALE step
            run_reference(args, rank)
        elif args.workload == "fields3d":
            run_reference_fields(args, rank)
        elif args.workload == "masks3d":
            run_reference_masks(args, rank)
        elif args.workload == "placed3d":
            run_reference_placed(args, rank)
        elif args.workload == "record3d":
            run_reference_record(args, rank)
        else:
            run_reference_2d(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        {"box3d": run_ours, "placed3d": run_placed, "cylinder2d": run_2d, "heated2d": run_2d, "sweep2d": run_sweep,
         "fields3d": run_fields, "masks3d": run_masks, "record3d": run_record, "closure3d": run_closure}[args.workload](
            args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
