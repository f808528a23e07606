"""A batched sweep of independent 2D solves of uneven grid size, advanced together.

The reference has no batched form: a sweep there is :class:`FlowSolver` looped over the
instances (src/aerolume/solvers/ns2d/solver.py:489 ``advance`` per instance, each step
``core.step_full`` of ns2d/core.py:815-969).  :class:`Sweep2D` owns one plan and one state per
instance and advances all of them by one step per call, each instance with its own CFL dt;
the result of every instance is the one its own plan gives alone (the tests hold the sweep to
the per-instance loop bit for bit).

``schedule="streams"`` spreads the instances over ``nstream`` CUDA streams (largest first,
round robin) so that the small instances' launches overlap the large ones'; ``"loop"`` runs
them one after another on the caller's stream (the plain per-instance loop).  Either can be
captured in a CUDA graph (:meth:`capture`).
"""
from __future__ import annotations

import torch

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
            self.plans.append(plan)
            self.states.append({"u": u, "v": v, "t": torch.zeros((), device=self.device, dtype=u.dtype), "out": out})
        self.cells = sum(p.shape[0] * p.shape[1] for p in self.plans)
        order = sorted(range(len(self.plans)), key=lambda k: -self.plans[k].shape[0] * self.plans[k].shape[1])
        self.nstream = max(1, min(int(nstream), len(self.plans)))
        self.lanes = [order[q::self.nstream] for q in range(self.nstream)]
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(self.nstream)]

    def _one(self, k):
        s = self.states[k]
        self.plans[k].step(s["u"], s["v"], s["t"], out=s["out"])
        s["t"].copy_(s["out"]["t"])

    def step(self, schedule: str = "streams"):
        """Advance every instance by one step (in place: u, v, t of each state)."""
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

    def capture(self, steps: int, schedule: str = "streams"):
        """A CUDA graph of ``steps`` sweep steps (replay with ``g.replay()``)."""
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
