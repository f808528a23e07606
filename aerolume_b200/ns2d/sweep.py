"""A batched sweep of independent 2D solves of uneven grid size, advanced together.

The reference has no batched form: a sweep there is :class:`FlowSolver` looped over the
instances (src/aerolume/solvers/ns2d/solver.py:489 ``advance`` per instance, each step
``core.step_full`` of ns2d/core.py:815-969).  :class:`Sweep2D` owns one plan and one state per
instance and advances all of them by one step per call, each instance with its own CFL dt;
the result of every instance is the one its own plan gives alone (the tests hold every schedule
to the per-instance loop bit for bit).

Schedules:

* ``"persistent"`` -- one persistent launch per sweep step (``aero_ns2d_sweep_step``): the
  co-resident CTAs take the work items of all instances' operations, numbered phase by phase
  (phase p: operation p of every instance's step).  Between them either a grid barrier per
  phase or, without barriers, a per-instance count of finished items that each item waits on
  (its own instance's earlier operations only); every wait is bounded (it gives up and reports
  instead of spinning forever).  :meth:`tune` picks the schedule, tile width, CTAs per SM and
  instance order by timing them.
* ``"streams"`` -- each instance's own launches, the instances spread over ``nstream`` CUDA
  streams (largest first, round robin).
* ``"loop"`` -- the plain per-instance loop on the caller's stream.

Any schedule can be captured in a CUDA graph (:meth:`capture`).
"""
from __future__ import annotations

import ctypes as C
import itertools

import torch

from .. import _lib
from .._lib import check
from .plan import Ns2dPlan


class Sweep2D:
    """Plans and states of the instances [(ops, geom), ...] on one device."""

    def __init__(self, instances, *, device=None, nstream: int = 16, seeds=None, noise: float = 1e-3):
        from .workloads import initial_state
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.plans, self.states = [], []
        for k, inst in enumerate(instances):
            ops, geom = inst[0], inst[1]
            plan = Ns2dPlan(ops, geom, device=self.device)
            u, v = initial_state(ops, plan, seed=k if seeds is None else seeds[k], noise=noise)
            out = plan.empty_fields()
            out["u"], out["v"] = u, v
            t = torch.zeros((), device=self.device, dtype=u.dtype)
            out["t"] = t                       # t advances in place (t_out = t0 + dt)
            self.plans.append(plan)
            self.states.append({"u": u, "v": v, "t": t, "out": out})
        self.cells = sum(p.shape[0] * p.shape[1] for p in self.plans)
        order = sorted(range(len(self.plans)), key=lambda k: -self.plans[k].shape[0] * self.plans[k].shape[1])
        self.nstream = max(1, min(int(nstream), len(self.plans)))
        self.lanes = [order[q::self.nstream] for q in range(self.nstream)]
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(self.nstream)]
        self._persistent = None
        self.tuning = None
        self.tuning_table = []

    # ------------------------------------------------------------------ per-instance launches
    def _one(self, k):
        s = self.states[k]
        self.plans[k].step(s["u"], s["v"], s["t"], out=s["out"])

    # ------------------------------------------------------------------ the persistent launch
    def _fields(self, k):
        s = self.states[k]
        f = _lib.Ns2dFields()
        out = s["out"]
        f.u0, f.v0, f.t0 = s["u"].data_ptr(), s["v"].data_ptr(), s["t"].data_ptr()
        for name in ("u", "v", "p", "t", "dt"):
            setattr(f, name, out[name].data_ptr())
        plan = self.plans[k]
        if plan.nbody and plan.has_win:
            f.coeffs = out["coeffs"].data_ptr()
        return f

    SCHEDULES = {"barrier": 0, "counters": 1, "queue": 2}

    def build_persistent(self, lcap=2, ctas_per_sm=3, order=1, schedule="counters", tiles=1):
        """The persistent launch of the current instances with these launch choices (schedule:
        "barrier", "counters" or "queue"; tiles: stage or transform tiles per work item)."""
        L = _lib.lib()
        n = len(self.plans)
        plans = (C.c_void_p * n)(*[p._handle.value for p in self.plans])
        fields = (_lib.Ns2dFields * n)(*[self._fields(k) for k in range(n)])
        geoms = (_lib.Ns2dGeom * n)(*[p.geom_c for p in self.plans])
        wss = (C.c_void_p * n)(*[p.ws_ptr for p in self.plans])
        tun = _lib.SweepTuning(int(lcap), int(ctas_per_sm), int(order), self.SCHEDULES[schedule], int(tiles))
        handle = C.c_void_p()
        check(L.aero_ns2d_sweep_create(n, plans, fields, geoms, wss, C.byref(tun), C.byref(handle)),
              "aero_ns2d_sweep_create")
        nbytes = L.aero_ns2d_sweep_workspace_bytes(handle)
        raw = torch.empty(nbytes + 256, dtype=torch.uint8, device=self.device)
        ptr = (raw.data_ptr() + 255) & ~255
        check(L.aero_ns2d_sweep_init(handle, C.c_void_p(ptr), self._stream()), "aero_ns2d_sweep_init")
        info = (C.c_int64 * 6)()
        check(L.aero_ns2d_sweep_info(handle, info), "aero_ns2d_sweep_info")
        return {"handle": handle, "raw": raw, "ptr": ptr,
                "tuning": (int(lcap), int(ctas_per_sm), int(order), schedule, int(tiles)),
                "info": dict(zip(("phases", "operations", "items", "ctas", "smem", "lcap"), list(info)))}

    def use_persistent(self, lcap=2, ctas_per_sm=3, order=1, schedule="counters", tiles=1):
        self._release()
        self._persistent = self.build_persistent(lcap, ctas_per_sm, order, schedule, tiles)
        self.tuning = self._persistent["tuning"]
        return self._persistent["info"]

    def _release(self, obj=None):
        obj = obj if obj is not None else self._persistent
        if obj is not None and obj.get("handle") is not None:
            _lib.lib().aero_ns2d_sweep_destroy(obj["handle"])
            obj["handle"] = None
        if obj is self._persistent:
            self._persistent = None

    def __del__(self):
        try:
            self._release()
        except Exception:  # pragma: no cover - interpreter shutdown
            pass

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _persistent_step(self, obj=None):
        obj = obj or self._persistent
        if obj is None:
            self.use_persistent()
            obj = self._persistent
        check(_lib.lib().aero_ns2d_sweep_step(obj["handle"], C.c_void_p(obj["ptr"]), self._stream()),
              "aero_ns2d_sweep_step")

    def status(self, obj=None):
        """The persistent launch's status word since the last read (bit 0: a grid barrier ran out)."""
        obj = obj or self._persistent
        st = C.c_int32()
        check(_lib.lib().aero_ns2d_sweep_read_status(obj["handle"], C.c_void_p(obj["ptr"]), C.byref(st),
                                                     self._stream()), "aero_ns2d_sweep_read_status")
        return int(st.value)

    def set_barrier(self, spin_limit, extra=0):
        """Bound of the persistent launch's grid barrier; extra > 0 (a test of the bound) waits
        for arrivals that never come."""
        check(_lib.lib().aero_ns2d_sweep_set_barrier(self._persistent["handle"], int(spin_limit), int(extra)),
              "aero_ns2d_sweep_set_barrier")

    # ------------------------------------------------------------------ stepping
    def step(self, schedule: str = "persistent"):
        """Advance every instance by one step (in place: u, v, t of each state)."""
        if schedule == "persistent":
            self._persistent_step()
            return
        main = torch.cuda.current_stream(self.device)
        if schedule == "loop":
            for k in range(len(self.plans)):
                self._one(k)
            return
        if schedule != "streams":
            raise ValueError(f"unknown schedule {schedule!r}")
        for s in self.streams:
            s.wait_stream(main)
        for lane, s in zip(self.lanes, self.streams):
            with torch.cuda.stream(s):
                for k in lane:
                    self._one(k)
        for s in self.streams:
            main.wait_stream(s)

    def capture(self, steps: int, schedule: str = "persistent"):
        """A CUDA graph of ``steps`` sweep steps (replay with ``g.replay()``)."""
        if schedule == "persistent" and self._persistent is None:
            self.use_persistent()
        main = torch.cuda.current_stream(self.device)
        side = torch.cuda.Stream(device=self.device)
        side.wait_stream(main)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            with torch.cuda.graph(g, stream=side):
                for _ in range(steps):
                    self.step(schedule)
        main.wait_stream(side)
        return g

    # ------------------------------------------------------------------ the autotuner
    def tune(self, candidates=None, steps=3, warmup=1):
        """Time each candidate (lcap, ctas_per_sm, order, schedule, tiles) of the persistent launch over ``steps``
        sweep steps (CUDA events, after ``warmup``), keep the fastest, and put every instance's
        state back as it was.  Returns the table of (candidate, ms per step)."""
        if candidates is None:
            candidates = list(itertools.product((2, 3), (3, 4), (0, 1), ("barrier", "queue"), (4, 8, 16)))
        snap = self.snapshot()
        table = []
        for cand in candidates:
            try:
                obj = self.build_persistent(*cand)
            except RuntimeError as exc:          # a launch shape that does not fit is skipped
                table.append((cand, None, str(exc)))
                continue
            cand = obj["tuning"]                 # every choice spelled out
            for _ in range(warmup):
                self._persistent_step(obj)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(steps):
                self._persistent_step(obj)
            b.record()
            torch.cuda.synchronize()
            st = self.status(obj)
            self._release(obj)
            self.restore(snap)
            table.append((cand, a.elapsed_time(b) / steps if st == 0 else None, obj["info"]))
        ok = [r for r in table if r[1] is not None]
        if not ok:
            raise RuntimeError("no launch shape of the persistent sweep ran")
        best = min(ok, key=lambda r: r[1])[0]
        self.use_persistent(*best)
        self.tuning_table = table
        return table

    # ------------------------------------------------------------------ results
    def coefficients(self):
        """[(nbody, 3) coefficients of each instance's last step] (device tensors)."""
        return [s["out"]["coeffs"] for s in self.states]

    def snapshot(self):
        """Copies of every instance's (u, v, t)."""
        return [(s["u"].clone(), s["v"].clone(), s["t"].clone()) for s in self.states]

    def restore(self, snap):
        for s, (u, v, t) in zip(self.states, snap):
            s["u"].copy_(u)
            s["v"].copy_(v)
            s["t"].copy_(t)


__all__ = ["Sweep2D"]
