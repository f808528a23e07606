"""The reference's 2D step function (src/aerolume/solvers/ns2d/core.py:815 ``step_full``),
served by the B200 step.

``FlowSolver`` imports ``step_full`` at module import (ns2d/solver.py:44-57) and calls it as
``step_full(state, geom, ops, None, out=..., diag=...)`` (solver.py:384-408); rebinding
``aerolume.solvers.ns2d.solver.step_full`` to this function swaps the step.  It returns
``(State, coeffs (nbody, 3))`` of new tensors like the reference.  With heat transfer theta
advances too and ``out`` receives the heat report of core.py:974-995; fans, heaters, painted
obstacles, jets and vents, smoke channels with emitters and the PID step of ``ops.phys`` run in
the step, ``state.ctrl`` carries the controllers' memory, ``state.dye_extra`` the smoke
channels after the first, and ``out`` receives ``fan_thrust``, ``fan_ud``, ``paint_force``,
``vent_heat`` and ``jet_heat`` as core.py:987-1002 fills them.  The wall model, diagnostics rows
and traces raise instead of being computed differently.
"""
from __future__ import annotations

import weakref
from typing import Any, NamedTuple

import torch

from .plan import Ns2dPlan


class State(NamedTuple):
    """The reference's 2D state (core.py:111-130)."""
    u: Any
    v: Any
    p: Any
    dye: Any
    t: Any
    dt: Any
    theta: Any = None
    dye_extra: Any = None
    ctrl: Any = None


_PLANS: dict = {}   # id(ops) -> {(id(geom), dye): (plan, geom)}, most recent last
_KEEP = 2


def _plan_for(ops, geom, dye, device):
    """The plan of (ops, geom, dye).  A plan reads the reference's device scalars ops.nu,
    ops.eta, phys.kappa and phys.eta_t at every launch, so an in-place ``set_reynolds``
    (core.py:167-176) needs no new plan and a captured graph stays valid, as in the reference;
    a ``set_bodies`` that builds a new geometry (and re-captures, solver.py:1050-1080) gets a
    new plan.  Each solver's ``ops`` keeps its ``_KEEP`` most recent plans; older ones are
    dropped with their device workspace, and all of them when ``ops`` itself is collected."""
    bucket = _PLANS.get(id(ops))
    if bucket is None:
        bucket = _PLANS[id(ops)] = {}
        try:
            weakref.finalize(ops, _PLANS.pop, id(ops), None)
        except TypeError:        # not weak-referenceable: its bucket stays bounded by _KEEP
            pass
    ph = getattr(ops, "phys", None)
    # the paint layer appears with the first stroke (physics.py:542-549): a new plan then
    key = (id(geom), dye, id(getattr(ph, "paint_u", None)) if ph is not None else 0)
    entry = bucket.pop(key, None)
    if entry is None:
        entry = (Ns2dPlan(ops, geom, dye=dye, device=device), geom)   # the entry keeps geom alive
    bucket[key] = entry
    while len(bucket) > _KEEP:
        del bucket[next(iter(bucket))]
    return entry[0]


def step_full(state, geom, ops, dt=None, *, out=None, diag=False, trace=None):
    """One SSP-RK3 step (plus the dye update when the state carries dye)."""
    if diag or trace is not None:
        raise RuntimeError("diagnostics rows and stage traces are not produced by the B200 step")
    theta = getattr(state, "theta", None)
    if theta is not None and getattr(ops, "phys", None) is None:
        raise RuntimeError("state.theta without heat transfer in ops.phys")
    plan = _plan_for(ops, geom, state.dye is not None, state.u.device)
    if (plan.thermal is None) != (theta is None):
        raise RuntimeError("state.theta must be given exactly when ops.phys has heat transfer")
    ctrl = getattr(state, "ctrl", None)
    if (ctrl is None) != (plan.ctrl_size == 0):
        raise RuntimeError("state.ctrl must be given exactly when ops.phys has fans or the PID step")
    if dt is not None and not torch.is_tensor(dt):
        dt = torch.tensor(float(dt), device=state.u.device, dtype=state.u.dtype)
    extra = getattr(state, "dye_extra", None)
    if (extra is not None) != (plan.dye_channels > 1):
        raise RuntimeError("state.dye_extra must be given exactly when ops.phys has several smoke channels")
    res = plan.step(state.u, state.v, state.t, dye0=state.dye, theta0=theta, dt=dt, ctrl0=ctrl,
                    dt_prev=state.dt if ctrl is not None else None, dye_extra0=extra)
    new = State(res["u"], res["v"], res["p"], res.get("dye"), res["t"], res["dt"], res.get("theta"),
                res.get("dye_extra"), res.get("ctrl"))
    if out is not None and plan.thermal is not None:
        keys = (["heat"] if plan.n_temp else []) + (["theta_wall"] if plan.n_flux else []) + [
            "wall_heat", "heat_storage", "flow_heat"]
        for k in keys:
            out[k] = res[k].to(state.u.dtype)
    if out is not None:
        for k in ("fan_thrust", "fan_ud", "paint_force", "vent_heat", "jet_heat"):
            if k in res:
                out[k] = res[k]
    coeffs = res["coeffs"] if plan.nbody and plan.has_win else torch.zeros(0, 3, device=state.u.device,
                                                                          dtype=state.u.dtype)
    return new, coeffs
