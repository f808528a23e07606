"""Long validation runs of the B200 step against the reference's own solvers (one JSON line each).

    python validate.py --case cylinder2d [--steps 4000]
    python validate.py --case box3d [--steps 2000]
    python validate.py --case closure [--steps 4000]

``cylinder2d`` (the 2D plain configuration: 256 x 128 FP32, a D = 0.5 cylinder at (2, 2) in the
8 x 4 tunnel, Re_D 100, upwind3, CFL 0.5, uniform stream plus seeded N(0, 1e-3) noise on u and v):
the reference's FlowSolver (installed unmodified under baseline/_ref) on this GPU, the same solver
with its step function rebound to the B200 step (aerolume_b200.ns2d.step.step_full, the drop-in of
ns2d/solver.py:44-57, 384-408), and the reference in FP64, all from the same inputs.  Reported:
mean Cd, Cl RMS, Cl amplitude (half the peak-to-peak, the reference's Cl') and the Strouhal
number from the upward zero crossings of Cl (validation/ns2d_cases.py:87-95, restated below)
over the second half, each run's wall time, and the errors of the B200 run and of the reference's
FP32 run against the FP64 run.

``box3d`` (the 3D drop-in configuration: the box on the moving floor at 256 x 128 x 128 FP32, WALE,
heat, smoke): the reference's FlowSolver3D with and without the B200 seam
(aerolume_b200.ns3d.fused in place of its fused module) and in FP64.  Reported: mean Cd and the
mean Nusselt number of the heated body over the second half, the divergence max |div u| h / U at
the end, wall times.

``closure``: the learned closure end to end -- training pairs from decaying turbulence at 384^3
(filtered 4x to 96^3), tensor-core training, then the box case at 256 x 128 x 128 with the closure
beside the plain WALE run at the same grid and the plain 512 x 256 x 256 run over the same
simulated time: mean Cd, mean heat rate, the dominant wake frequency, wall times.
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402  (the reference's install and the box case of the benchmark)


def strouhal(t, cl, length):
    """Shedding frequency from the upward zero crossings of Cl - mean (the first crossing
    skipped, at least four needed) times the reference length (validation/ns2d_cases.py:87-95)."""
    x = cl - cl.mean()
    idx = np.where((x[:-1] < 0) & (x[1:] >= 0))[0]
    if len(idx) < 4:
        return None
    tc = t[idx] - x[idx] * (t[idx + 1] - t[idx]) / (x[idx + 1] - x[idx])
    return float(length / np.mean(np.diff(tc[1:])))


def _sync():
    import torch
    torch.cuda.synchronize()


def _rel(a, b):
    if a is None or b is None:
        return None
    return abs(a - b) / max(abs(b), 1e-30)


# ---------------------------------------------------------------------------------------
# 2D: config [0]
# ---------------------------------------------------------------------------------------

def _ref2d():
    bench._reference_api()                      # puts baseline/_ref on the path (ImportError if absent)
    import aerolume.solvers.ns2d.config as C2
    import aerolume.solvers.ns2d.solver as S2
    return C2, S2


def _cylinder_config(C2, dtype):
    from aerolume_b200.ns2d.workloads import circle
    return C2.SolverConfig(nx=256, ny=128, h=1.0 / 32.0, x0=0.0, y0=0.0, re=200.0,
                           bodies=[C2.ImmersedBody(circle(2.0, 2.0, 0.25, 256), name="cylinder")], bc_top="slip",
                           bc_bottom="slip", advection="upwind3", cfl=0.5, dtype=dtype, device="cuda",
                           force_ref=0.5, moment_ref=(2.0, 2.0), dye=False, perturb=False)


def _noise2d(s, seed=0, amp=1e-3):
    import torch
    g = torch.Generator().manual_seed(seed)
    st = s._state
    with torch.no_grad():
        for x in (st.u, st.v):
            x.add_((amp * torch.randn(tuple(x.shape), generator=g, dtype=torch.float64)).to(x.device, x.dtype))


def _run2d(s, steps, chunk=200):
    _sync()
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        s.advance(k)
        done += k
    _sync()
    wall = time.perf_counter() - t0
    h = s.history()
    t, cd, cl = h["t"], h["cd"], h["cl"]
    m = t >= 0.5 * t[-1]
    return {"cd_mean": float(cd[m].mean()), "cl_rms": float(cl[m].std()), "cl_amp": float(0.5 * (cl[m].max() - cl[m].min())),
            "st": strouhal(t[m], cl[m], 0.5), "t_end": float(t[-1]), "steps": int(steps), "wall_s": wall}


def cylinder2d(steps):
    from aerolume_b200.ns2d import step as seam
    C2, S2 = _ref2d()
    out = {"case": "cylinder2d", "config": "256x128 FP32, D = 0.5 at (2, 2), Re_D 100, upwind3, CFL 0.5, "
                                           "slip walls, uniform stream + N(0, 1e-3) noise (seed 0)"}
    runs = {}
    for tag, dtype, ours in (("reference_f64", "float64", False), ("reference_f32", "float32", False),
                             ("b200_f32", "float32", True)):
        orig = S2.step_full
        try:
            if ours:
                S2.step_full = seam.step_full
            s = S2.FlowSolver(_cylinder_config(C2, dtype))
            _noise2d(s, 0)
            runs[tag] = _run2d(s, steps)
            runs[tag]["graphs"] = bool(getattr(s, "uses_cuda_graphs", False))
        finally:
            S2.step_full = orig
        del s
    r64 = runs["reference_f64"]
    for tag in ("reference_f32", "b200_f32"):
        r = runs[tag]
        r["err_vs_f64"] = {k: _rel(r[k], r64[k]) for k in ("cd_mean", "cl_rms", "cl_amp", "st")}
    b, r32 = runs["b200_f32"], runs["reference_f32"]
    b["err_vs_reference_f32"] = {k: _rel(b[k], r32[k]) for k in ("cd_mean", "cl_rms", "cl_amp", "st")}
    b["speedup_vs_reference_f32"] = r32["wall_s"] / b["wall_s"]
    out["runs"] = runs
    out["bands_32_cells_per_D"] = {"cd": [1.30, 1.42], "cl_amp": [0.30, 0.36], "st": [0.160, 0.172],
                                   "note": "tests/test_ns2d_validation.py:64-70, at 5 % blockage; this case has 12.5 %"}
    return out


# ---------------------------------------------------------------------------------------
# 3D: config [1]
# ---------------------------------------------------------------------------------------

def _noise3d(s, seed=0, amp=1e-3):
    import torch
    g = torch.Generator().manual_seed(seed)
    st = s._state
    with torch.no_grad():
        for x in (st.u, st.v, st.w):
            x.add_((amp * torch.randn(tuple(x.shape), generator=g, dtype=torch.float64)).to(x.device, x.dtype))


def _run3d(s, steps, chunk=100):
    import torch
    _sync()
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        s.advance(k)
        done += k
    _sync()
    wall = time.perf_counter() - t0
    h = s.history()
    ph = s.physics_history()
    t, cd = h["t"], h["cd"]
    m = t >= 0.5 * t[-1]
    nu = ph.get("nu")
    st = s._state
    with torch.no_grad():
        div = ((st.u[..., 1:] - st.u[..., :-1]) + (st.v[:, 1:] - st.v[:, :-1]) + (st.w[1:] - st.w[:-1]))
        div_h = float(div.abs().max()) / float(max(st.u.abs().max(), 1e-30))
    return {"cd_mean": float(cd[m].mean()), "nu_mean": float(np.nanmean(nu[m])) if nu is not None else None,
            "div_max_h_over_U": div_h, "t_end": float(t[-1]), "steps": int(steps), "wall_s": wall}


def box3d(steps):
    import aerolume_b200.ns3d.fused as B
    bench._reference_api()
    import aerolume.solvers.ns3d.fused as F
    import aerolume.solvers.ns3d.solver as S3
    names = ("load_kernels", "fast_step", "fast_step_phys", "fast_dye", "check_dye_kernels", "check_theta_kernels")
    out = {"case": "box3d", "config": "box 1 x 1 x 0.5 on a moving floor, 256x128x128 FP32, Re_H 5000, WALE, "
                                      "heat (Pr 0.71, Ri_H 0.1), 16-nozzle smoke rake, uniform + N(0, 1e-3)"}
    runs = {}
    for tag, dtype, ours in (("reference_f64", "float64", False), ("reference_f32", "float32", False),
                             ("b200_f32", "float32", True)):
        saved = {n: getattr(F, n) for n in names}
        try:
            if ours:
                for n in names:
                    setattr(F, n, getattr(B, n))
            import dataclasses
            cfg = dataclasses.replace(bench.reference_box_config(256, 128, 128, "cuda"), dtype=dtype)
            s = S3.FlowSolver3D(cfg)
            if ours:
                assert isinstance(s._kern, B.B200Kernels)
            _noise3d(s, 0)
            runs[tag] = _run3d(s, steps)
        finally:
            for n, f in saved.items():
                setattr(F, n, f)
        del s
    r64 = runs["reference_f64"]
    for tag in ("reference_f32", "b200_f32"):
        r = runs[tag]
        r["err_vs_f64"] = {k: _rel(r[k], r64[k]) for k in ("cd_mean", "nu_mean")}
    b, r32 = runs["b200_f32"], runs["reference_f32"]
    b["err_vs_reference_f32"] = {k: _rel(b[k], r32[k]) for k in ("cd_mean", "nu_mean")}
    b["speedup_vs_reference_f32"] = r32["wall_s"] / b["wall_s"]
    out["runs"] = runs
    out["reference_divergence_level"] = "4.0e-7 (docs/theory_ns3d.md:345)"
    return out


# ---------------------------------------------------------------------------------------
# the learned closure: configs [3] and [4]
# ---------------------------------------------------------------------------------------

def _box_run(nx, ny, nz, t_end, closure=None, probe=(3.75, 2.0, 0.5), max_steps=20000):
    """Our plan on the box case until t_end: (mean Cd, mean heat rate over the second half),
    the wake's dominant frequency (vertical velocity at the probe), steps, wall time."""
    import torch
    from aerolume_b200.ns3d.plan import Ns3dPlan
    from aerolume_b200.ns3d.workloads import box_on_moving_floor, initial_state
    ops, geom, th, src, _ = box_on_moving_floor(nx, ny, nz, dtype="float32", seed=0)
    plan = Ns3dPlan(ops, geom, th, src, smoke=True, closure=closure)
    u, v, w = initial_state(ops, seed=0)
    plan.project(u, v, w)
    theta = torch.zeros(nz, ny, nx, device="cuda")
    dyes = [torch.zeros(nz, ny, nx, device="cuda"), torch.zeros(nz, ny, nx, device="cuda")]
    t = torch.zeros((), device="cuda")
    out = plan.empty_fields()
    out["u"], out["v"], out["w"], out["theta"] = u, v, w, theta
    h = ops.h
    pk, pj, pi = int(probe[2] / h), int(probe[1] / h), int(probe[0] / h)
    chunk = 200
    rec = torch.zeros(max_steps, 4, device="cuda", dtype=torch.float64)   # t, Cd, heat rate, probe w
    _sync()
    t0 = time.perf_counter()
    k = 0
    while k < max_steps:
        for _ in range(chunk):
            out["dye"] = dyes[(k + 1) % 2]
            plan.step(u, v, w, t, theta0=theta, dye0=dyes[k % 2], out=out)
            t.copy_(out["t"])
            rec[k, 0] = out["t"]
            rec[k, 1] = out["coeffs"][0, 0]
            rec[k, 2] = out["heat_rate"].sum()
            rec[k, 3] = w[pk, pj, pi]
            k += 1
        if float(t) >= t_end:
            break
    _sync()
    wall = time.perf_counter() - t0
    r = rec[:k].cpu().numpy()
    m = r[:, 0] >= 0.5 * r[-1, 0]
    tt, sig = r[m, 0], r[m, 3] - r[m, 3].mean()
    # dominant frequency of the probe signal on a uniform resampling (the steps' dt varies)
    tu = np.linspace(tt[0], tt[-1], len(tt))
    su = np.interp(tu, tt, sig)
    spec = np.abs(np.fft.rfft(su * np.hanning(len(su)))) ** 2
    freq = np.fft.rfftfreq(len(su), tu[1] - tu[0])
    f_peak = float(freq[1 + np.argmax(spec[1:])]) if len(spec) > 2 else None
    res = {"grid": [nx, ny, nz], "cd_mean": float(r[m, 1].mean()), "heat_rate_mean": float(r[m, 2].mean()),
           "nusselt_mean": float(r[m, 2].mean() / 3.0), "wake_peak_frequency": f_peak,
           "strouhal_H": f_peak * 0.5 if f_peak else None, "steps": k, "t_end": float(r[-1, 0]), "wall_s": wall,
           "status": plan.status()}
    if closure is not None:
        ev, wale = plan.closure_counts()
        res["closure_cells"] = ev
        res["closure_wale_fraction"] = wale / max(ev, 1)
    return res


def closure(steps, hit_n=384, snapshots=8, train_steps=3000):
    import torch
    from aerolume_b200.ns3d.closure import ClosureModel, make_pairs
    out = {"case": "closure"}
    # config [3]: training pairs from decaying turbulence, filtered 4x
    _sync()
    t0 = time.perf_counter()
    feat, target, valid, record = make_pairs(hit_n, factor=4, re=1500.0, seed=0, spinup=400, snapshots=snapshots,
                                             every=50)
    _sync()
    out["data"] = {"grid": hit_n, "pairs": int(valid.sum().item()), "snapshots": snapshots, "every": 50,
                   "spinup_steps": 400, "wall_s": time.perf_counter() - t0, "kinetic_energy": record}
    model = ClosureModel(seed=0)
    model.fit_normalisation(feat, target, valid)
    ok = valid.bool()
    x, t = model.normalise(feat[ok].contiguous(), target[ok].contiguous())
    del feat, target
    n_hold = x.shape[0] // 10
    xtr, ttr, xte, tte = x[n_hold:], t[n_hold:], x[:n_hold], t[:n_hold]
    _sync()
    t0 = time.perf_counter()
    hist = model.train(xtr, ttr, train_steps, batch=65536, lr=1e-3, seed=1, log_every=100)
    _sync()
    wall = time.perf_counter() - t0
    yte = model.forward(xte)
    mse = float(((yte - tte) ** 2).mean().item())
    flops = 3 * 2 * 36864 * 65536 * train_steps          # forward + backward, padded MACs
    out["training"] = {"steps": train_steps, "batch": 65536, "lr": 1e-3, "wall_s": wall,
                       "tflops_achieved": flops / wall / 1e12, "mse_first": hist[0][1], "mse_last": hist[-1][1],
                       "mse_held_out": mse, "variance_of_targets": 1.0}
    # config [4]: the bluff-body case with the closure, plain WALE, and the 2x finer plain run
    coarse_c = _box_run(256, 128, 128, t_end=1e9, closure=model, max_steps=steps)
    t_end = coarse_c["t_end"]
    coarse_w = _box_run(256, 128, 128, t_end=t_end, max_steps=steps + 400)
    fine = _box_run(512, 256, 256, t_end=t_end, max_steps=4 * steps)
    out["deployed"] = {"closure_256": coarse_c, "wale_256": coarse_w, "plain_512": fine}
    out["judge"] = {"cd_error_closure_vs_512": _rel(coarse_c["cd_mean"], fine["cd_mean"]),
                    "cd_error_wale_vs_512": _rel(coarse_w["cd_mean"], fine["cd_mean"]),
                    "heat_error_closure_vs_512": _rel(coarse_c["heat_rate_mean"], fine["heat_rate_mean"]),
                    "heat_error_wale_vs_512": _rel(coarse_w["heat_rate_mean"], fine["heat_rate_mean"]),
                    "wall_ratio_512_over_closure": fine["wall_s"] / coarse_c["wall_s"],
                    "target": "mean Cd within 2 % of the 512 run in >= 4x less wall time"}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", required=True, choices=["cylinder2d", "box3d", "closure"])
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--hit-n", type=int, default=384)
    ap.add_argument("--snapshots", type=int, default=8)
    ap.add_argument("--train-steps", type=int, default=3000)
    a = ap.parse_args()
    if a.case == "cylinder2d":
        res = cylinder2d(a.steps or 4000)
    elif a.case == "box3d":
        res = box3d(a.steps or 2000)
    else:
        res = closure(a.steps or 4000, a.hit_n, a.snapshots, a.train_steps)
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
