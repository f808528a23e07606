"""Host-side containers of the 3D step, with the reference's attribute names.

The drop-in step (:mod:`aerolume_b200.ns3d.fused`) reads its inputs by attribute, so it
accepts either these containers or the reference's own objects:

* :class:`Ops3D`      -- ``aerolume.solvers.ns3d.core.Ops3D`` (core.py:61-108)
* :class:`Geometry3D` -- ``aerolume.solvers.ns3d.geometry.Geometry3D`` (geometry.py:275-303)
* :class:`ThermalOps` / :class:`ThermalGeometry` -- the parts of
  ``aerolume.solvers.ns3d.physics.ThermalOps`` / ``ThermalGeometry`` the step reads
  (physics.py:314-461, 494-560)
* :class:`DyeSources` -- ``aerolume.solvers.ns3d.dye.DyeSources`` (dye.py:140-151)
* :class:`PaintLayer3D` / :class:`PidState3D` / :class:`FanSet3D` / :class:`PortSet3D` -- the
  parts of ``aerolume.solvers.ns3d.physics.PaintLayer`` / ``PidDt`` / ``FanSet`` / ``PortSet``
  the step reads and updates (physics.py:831-1181)
* :class:`State3D`, :class:`StepOut3D` -- core.py:111-119, 745-750

Arrays may be numpy arrays or torch tensors; the step uploads what is not already on the
device once per plan.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, NamedTuple


class State3D(NamedTuple):
    """u (nz, ny, nx+1), v (nz, ny+1, nx), w (nz+1, ny, nx), p (nz, ny, nx), t, dt (0-d)."""
    u: Any
    v: Any
    w: Any
    p: Any
    t: Any
    dt: Any


class StepOut3D(NamedTuple):
    """New state, per-body coefficients (nbody, 6) and the new temperature (or None)."""
    state: State3D
    coeffs: Any
    theta: Any


@dataclass
class Ops3D:
    """Grid, boundary rules and numerics of one 3D solve (core.py:61-108).

    ``ghost`` maps "u", "v", "w" to per-axis ``((kind, value), (kind, value))`` rules of
    core.py:147-181; ``u_inlet`` is the (nz, ny) inlet profile.
    """
    nx: int
    ny: int
    nz: int
    h: float
    x0: float = 0.0
    y0: float = 0.0
    z0: float = 0.0
    periodic_axes: tuple = (False, False, False)
    closed: bool = False
    symmetry: bool = False
    advection: str = "upwind3"
    turbulence: str = "none"
    les_c: float = 0.0
    nu_value: float = 1e-3
    eta: float = 1.0
    cfl: float = 0.5
    dt_fixed: float | None = None
    ghost: dict = field(default_factory=dict)
    u_inlet: Any = None
    ref_area: float = 1.0
    length_ref: float = 1.0
    span_ref: float = 1.0
    moment_ref: tuple = (0.0, 0.0, 0.0)
    dtype: str = "float32"
    forcing: Any = None          # uniform body force (fx, fy, fz) of the verification cases (core.py:106)

    @property
    def periodic(self) -> bool:
        return all(self.periodic_axes)


@dataclass
class Geometry3D:
    """Masks on the cell window ``(k0, k1, j0, j1, i0, i1)`` (geometry.py:275-303)."""
    window: tuple
    chi_u: Any = None
    chi_v: Any = None
    chi_w: Any = None
    chi_c: Any = None
    a_u: Any = None
    a_v: Any = None
    a_w: Any = None
    k_u: Any = None
    k_v: Any = None
    k_w: Any = None
    nbody: int = 0

    @property
    def empty(self) -> bool:
        k0, k1, j0, j1, i0, i1 = self.window
        return k1 <= k0 or j1 <= j0 or i1 <= i0


@dataclass
class ThermalGeometry:
    """Thermal masks on the momentum window (physics.py:314-461)."""
    window: tuple
    nbody: int = 0
    chi_t: Any = None
    a_t: Any = None
    w_t: Any = None
    t_index: list = field(default_factory=list)
    adia: Any = None
    vol_w: Any = None
    skin: Any = None
    flux_rate: Any = None


@dataclass
class ThermalOps:
    """Heat-equation constants the step reads (physics.py:494-560).

    ``side_kinds`` / ``side_vals`` follow WALL_SIDES order (left, right, front, back,
    bottom, top); kinds are "periodic", "outflow", "adiabatic", "inflow", "temperature",
    "heat_flux".
    """
    kappa: float
    pe: float
    ri: float
    prt: float
    eta: float
    side_kinds: tuple
    side_vals: tuple
    geom: ThermalGeometry
    h: float
    symmetry: bool = False
    heat_max: float | None = None
    sources: tuple = ()          # volumetric heaters: (cell window, density (wz, wy, wx)) pairs


@dataclass
class DyeSources:
    """Smoke nozzles: weights on a cell window and the pulse [t_on, period] (dye.py:140-151)."""
    window: tuple
    weight: Any
    pulse: tuple = (2.0, 1.0)

    @property
    def empty(self) -> bool:
        k0, k1, j0, j1, i0, i1 = self.window
        return k1 <= k0 or j1 <= j0 or i1 <= i0


@dataclass
class PaintLayer3D:
    """Painted solid fractions on the whole grid (physics.py:1074-1141): chi_u (nz, ny, nx+1),
    chi_v (nz, ny+1, nx), chi_w (nz+1, ny, nx), chi_c (nz, ny, nx), device tensors of the
    plan's dtype.  The step reads them at every call, so edits in place take effect."""
    chi_u: Any
    chi_v: Any
    chi_w: Any
    chi_c: Any


@dataclass
class PidState3D:
    """The PID step controller (physics.py:1144-1181): the target fraction of the stability
    limit and its state, 0-d device tensors dt_prev (<= 0: no step yet), e1, e2 that the
    step updates in place."""
    target: float
    dt_prev: Any
    e1: Any
    e2: Any


@dataclass
class FanSet3D:
    """Actuator discs (physics.py:831-979), the attributes the step reads and updates.

    ``items[q]``: ``win`` (the fan's cell window) and its weights on the window's faces,
    ``fu / fv / fw`` (force), ``su / sv / sw`` (swirl), ``mu / mv / mw`` (disc average).
    Per-fan constants ``target, kp, ki, tmax, swirl`` and ``velocity_mode`` (nfan,), and the
    state tensors ``thrust, ud, e_prev, swirl_amp`` (nfan,) on the device, updated in place.
    """
    items: list
    target: Any
    kp: Any
    ki: Any
    tmax: Any
    velocity_mode: Any
    swirl: Any
    any_swirl: bool
    thrust: Any
    ud: Any
    e_prev: Any
    swirl_amp: Any

    def __len__(self) -> int:
        return len(self.items)


@dataclass
class PortSet3D:
    """Jets and vents (physics.py:981-1072), the attributes the step reads.

    ``items[q]``: ``win`` (cell window), ``kind`` ("jet" / "vent"), ``m`` (mass source on the
    window's cells), ``fu / fv / fw`` (momentum weights on its faces; a vent's are multiplied
    by the local velocity), ``theta`` (a jet's temperature).  ``mass_flux``: the net source in
    outlet-face units; ``leak``: the uniform scalar leak of an unbalanced closed box."""
    items: list
    mass_flux: Any
    leak: float = 0.0

    def __len__(self) -> int:
        return len(self.items)
