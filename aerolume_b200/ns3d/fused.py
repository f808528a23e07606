"""The reference's fused-kernel seam of ``FlowSolver3D`` (src/aerolume/solvers/ns3d/fused.py),
served by the B200 step.

Same names, arguments and results as the reference module, so ``ns3d/solver.py`` can import
these instead (solver.py:161-166 ``load_kernels``; solver.py:583-595 ``fast_step`` /
``fast_step_phys``; solver.py:655-657 ``fast_dye``):

* ``load_kernels(scheme, device, dtype)`` raises ``RuntimeError`` when the B200 library or a
  CUDA device is missing (fused.py:226-235 raises the same way, so the solver records
  ``fused_error``); it returns a handle that caches one plan per configuration.
* ``fast_step`` / ``fast_step_phys`` return ``(State3D, coeffs)`` / ``StepOut3D`` of new
  tensors, as fused.py:371 / 378-502 do.
* ``fast_dye`` is the MUSCL advection of one smoke channel (fused.py:553-565).

Heat transfer with its volumetric heaters, fans, jets and vents, painted solids and the PID
step controller run in the step; with ``diag`` the step also leaves the squared norm of the last
stage's projection right-hand side in ``phys.div_pre`` (physics.py:1303-1305), which the
solver's diagnostics row reads.
"""
from __future__ import annotations

import torch

from .plan import Ns3dPlan
from .types import Geometry3D, State3D, StepOut3D


def _live_key(ops, thermal):
    """The plan constants that the reference changes in place on a live edit, as host values:
    ``set_reynolds`` (core.py:140-144) writes ``ops.nu_value`` (and ``ops.nu`` / ``ops.eta`` from
    the same Re), ``ThermalOps.set_reynolds`` (physics.py:580-586) writes ``pe`` / ``kappa`` (and
    the thermal eta from the same Pe), and ``FlowSolver3D.set_bodies`` (solver.py:1659-1700) may
    swap ``thermal.geom``.  Host attributes only: reading a device tensor here would synchronise
    the stream, which a graph capture forbids."""
    key = (float(ops.nu_value),)
    if thermal is not None:
        key += (float(thermal.kappa), float(thermal.pe), id(getattr(thermal, "geom", None)))
    return key


class B200Kernels:
    """What ``load_kernels`` returns: the scheme plus the plans of the latest configurations.

    A plan holds its constants from creation, so a plan is looked up by the identities of the
    objects it was built from and by :func:`_live_key`: after ``set_inflow`` or a ``set_bodies``
    that replaces the thermal masks the next step builds a new plan (the reference re-captures
    its graphs on both, solver.py:1656, :1699).  At most ``keep`` plans of each kind stay
    cached; older ones are dropped with their device workspace."""

    keep = 2

    def __init__(self, scheme, device, dtype):
        self.scheme, self.device, self.dtype = scheme, device, dtype
        self._plans = {}
        # the learned subgrid closure (a trained ClosureModel) for WALE steps, or None; set it
        # on the handle the solver holds (``solver._kern.closure = model``): the next step
        # builds its plan with it
        self.closure = None

    def _remember(self, key, entry):
        same = [k for k in self._plans if k[0] == key[0]]
        for k in same[: max(0, len(same) - self.keep + 1)]:
            del self._plans[k]
        self._plans[key] = entry

    def plan_for(self, geom, ops, phys=None):
        thermal = getattr(phys, "thermal", None) if phys is not None else None
        paint = getattr(phys, "paint", None) if phys is not None else None
        pid = getattr(phys, "pid", None) if phys is not None else None
        fans = getattr(phys, "fans", None) if phys is not None else None
        ports = getattr(phys, "ports", None) if phys is not None else None
        closure = self.closure if getattr(ops, "turbulence", None) == "wale" else None
        key = ("step", id(geom), id(ops), id(thermal), id(paint), id(pid), id(fans), id(ports),
               id(closure)) + _live_key(ops, thermal)
        entry = self._plans.get(key)
        if entry is None:
            plan = Ns3dPlan(ops, geom, thermal, None, device=self.device, paint=paint, pid=pid, fans=fans, ports=ports,
                            u_floor=float(getattr(phys, "u_floor", 0.0) or 0.0) if phys is not None else 0.0,
                            closure=closure)
            entry = (plan, geom, ops, thermal, paint, pid, fans, ports)   # the objects stay alive with their plan
            self._remember(key, entry)
        return entry[0]

    def dye_plan_for(self, ops, shape=None):
        """The smoke-only plan of ``ops`` (or, for an ``ops`` that carries no grid, as the
        reference's kernel self-test passes, of the field shape (nz, ny, nx))."""
        key = ("dye", id(ops), shape)
        entry = self._plans.get(key)
        if entry is None:
            grid_ops = ops if hasattr(ops, "ghost") else _smoke_ops(ops, shape, self.dtype)
            plan = Ns3dPlan(grid_ops, Geometry3D((0, 0, 0, 0, 0, 0)), None, None, smoke=True, device=self.device)
            entry = (plan, ops)
            self._remember(key, entry)
        return entry[0]


def _smoke_ops(ops, shape, dtype):
    """Operators of a smoke-only plan from the attributes the smoke update reads (cell size and
    periodic axes) and the field shape."""
    from .setup import make_ops
    nz, ny, nx = shape
    o = make_ops(nx, ny, nz, float(ops.h), re=1.0, dtype="float64" if dtype == torch.float64 else "float32")
    o.periodic_axes = tuple(bool(x) for x in getattr(ops, "periodic_axes", (False, False, False)))
    return o


def load_kernels(scheme: str, device: torch.device, dtype: torch.dtype) -> B200Kernels:
    """The B200 kernels for ``scheme`` on ``device`` / ``dtype`` (raises when unavailable)."""
    device = torch.device(device)
    if device.type != "cuda":
        raise RuntimeError("the B200 kernels need a CUDA device")
    if not torch.cuda.is_available():
        raise RuntimeError("CUDA is not available")
    if scheme not in ("upwind3", "central"):
        raise RuntimeError(f"unknown advection scheme {scheme!r}")
    from .. import _lib
    _lib.lib()                                           # raises when libaero_b200.so is missing
    return B200Kernels(scheme, device, dtype)


def _dt_arg(dt, like):
    if dt is None or torch.is_tensor(dt):
        return dt
    return torch.tensor(float(dt), device=like.device, dtype=like.dtype)


def fast_step(state, geom, ops, kern):
    """One plain step: (State3D, coeffs (nbody, 6)) of new tensors."""
    out = kern.plan_for(geom, ops).step(state.u, state.v, state.w, state.t)
    return State3D(out["u"], out["v"], out["w"], out["p"], out["t"], out["dt"]), out["coeffs"]


def fast_step_phys(state, geom, ops, kern, dt=None, *, phys=None, theta=None, diag=False, theta_kernels=True):
    """One step with the placed physics the B200 step implements (heat transfer, fans, jets and
    vents, painted solids, the PID step controller); ``diag`` records the last stage's
    projection right-hand side norm in ``phys.div_pre`` as fused.py:480-482 does."""
    plan = kern.plan_for(geom, ops, phys)
    thermal = plan.thermal is not None and theta is not None
    div_sq = getattr(phys, "div_pre", None) if diag and phys is not None else None
    out = plan.step(state.u, state.v, state.w, state.t, theta0=theta if thermal else None,
                    dt=_dt_arg(dt, state.t), div_sq=div_sq)
    if thermal and torch.is_tensor(getattr(plan.thermal, "heat_rate", None)):
        plan.thermal.heat_rate.copy_(out["heat_rate"])  # the reference leaves the rates there
    new = State3D(out["u"], out["v"], out["w"], out["p"], out["t"], out["dt"])
    return StepOut3D(new, out["coeffs"], out.get("theta") if thermal else None)


def fast_dye(c, u, v, w, dt, ops, kern):
    """MUSCL / van Leer advection of one smoke channel with the step's velocity and dt."""
    dt = _dt_arg(dt, c)
    return kern.dye_plan_for(ops, tuple(c.shape)).smoke_step(c, u, v, w, dt, dt, solids=False, sources=False)


def check_dye_kernels(kern, device, dtype):
    """The reference's self-test hook of the smoke kernels (fused.py:528-550): runs the B200
    smoke update once on a small random field and raises RuntimeError when the library fails or
    gives a non-finite or unbounded result (the solver then keeps its own smoke scheme)."""
    from types import SimpleNamespace
    try:
        g = torch.Generator(device=device).manual_seed(7)
        c = torch.rand((6, 5, 7), generator=g, device=device, dtype=dtype)
        u = torch.randn((6, 5, 8), generator=g, device=device, dtype=dtype) * 0.1
        v = torch.randn((6, 6, 7), generator=g, device=device, dtype=dtype) * 0.1
        w = torch.randn((7, 5, 7), generator=g, device=device, dtype=dtype) * 0.1
        out = fast_dye(c, u, v, w, torch.tensor(0.05, device=device, dtype=dtype),
                       SimpleNamespace(periodic_axes=(False, False, False), h=0.1), kern)
    except Exception as exc:
        raise RuntimeError(f"B200 smoke kernels unavailable ({type(exc).__name__}: {exc})") from exc
    if not (bool(torch.isfinite(out).all()) and float(out.max()) <= 1.0 and float(out.min()) >= 0.0):
        raise RuntimeError("B200 smoke kernel self-test gave an out-of-range result")


def check_theta_kernels(kern, device, dtype):
    """The reference's self-test hook of the heat-equation kernels (fused.py:505-525): the B200
    step advances theta inside ``fast_step_phys``, so this only checks that the library loads."""
    from .. import _lib
    _lib.lib()
