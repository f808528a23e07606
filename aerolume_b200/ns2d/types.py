"""Plain containers with the attribute names of the reference's 2D objects.

``Ns2dPlan`` and the oracle read these attributes only, so the reference's own ``Ops`` /
``Geometry`` (src/aerolume/solvers/ns2d/core.py:67-108, geometry.py:160-197) work as well.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Any, NamedTuple


class State2D(NamedTuple):
    """Evolving state (core.py:111-130 without placed physics)."""
    u: Any
    v: Any
    p: Any
    dye: Any
    t: Any
    dt: Any


@dataclass
class Ops2D:
    """Grid, boundaries and numerics of a 2D solve (core.py:67-108)."""
    nx: int
    ny: int
    h: float
    x0: float = 0.0
    y0: float = 0.0
    periodic: bool = False
    closed: bool = False
    bc_top: str = "slip"
    bc_bottom: str = "slip"
    bc_left: str = "noslip"
    bc_right: str = "noslip"
    ground_speed: float = 1.0
    advection: str = "upwind3"
    turbulence: str = "none"
    les_c: float = 0.0
    nu: float = 1e-3
    eta: float = 1.0
    cfl: float = 0.5
    dt_fixed: float | None = None
    u_inlet: Any = None          # (ny,) inlet u profile
    dye_inlet: Any = None        # (ny,) inlet dye comb, or None without dye
    force_ref: float = 1.0
    moment_ref: tuple = (0.25, 0.0)
    dtype: str = "float32"
    wall_model: bool = False     # the Werner-Wengle shear on the no-slip domain walls (core.py:505-564)
    forcing: Any = None          # uniform body force (fx, fy) of the verification cases (core.py:102)


@dataclass
class Geometry2D:
    """Body masks on the cell window (j0, j1, i0, i1) (geometry.py:160-182)."""
    window: tuple
    chi_u: Any = None            # (wy, wx + 1)
    chi_v: Any = None            # (wy + 1, wx)
    chi_c: Any = None            # (wy, wx)
    a_u: Any = None
    a_v: Any = None
    k_u: Any = None              # (nb, 2, wy, wx + 1): [Fx weight, moment weight]
    k_v: Any = None              # (nb, 2, wy + 1, wx)
    nbody: int = 0

    @property
    def empty(self) -> bool:
        return self.window[1] <= self.window[0] or self.window[3] <= self.window[2]


@dataclass
class Thermal2D:
    """Heat transfer of a 2D solve: the thermal part of the reference's ``Physics``
    (src/aerolume/solvers/ns2d/physics.py:305-322) with the bodies' ``ThermalGeometry``
    (geometry.py:120-158) on the body window.  ``wall_modes`` are the side modes of
    scalar.py:96-146 (left, right, bottom, top); ``temp_ids`` / ``flux_ids`` only count the
    temperature and heat-flux bodies."""
    kappa: float
    ri: float
    prt: float
    gravity: tuple
    eta_t: float
    theta_in: float
    wall_modes: tuple
    wall_values: tuple
    diff_coef: float
    temp_ids: tuple = ()
    flux_ids: tuple = ()
    chi_t: Any = None            # (wy, wx) temperature-body mask
    a_t: Any = None              # (wy, wx) chi_t * body temperature
    w_t: Any = None              # (n_temp, wy, wx) heat shares
    ins_u: Any = None            # (wy, wx + 1) insulation factors of the x-faces
    ins_v: Any = None            # (wy + 1, wx)
    q_skin: Any = None           # (wy, wx) heat-flux skin source / kappa
    w_f: Any = None              # (n_flux, wy, wx) wall-temperature weights
    vol_u: Any = None            # (wy, wx + 1) solid area fractions for the buoyancy share
    vol_v: Any = None            # (wy + 1, wx)


@dataclass
class Placed2D:
    """Fans, heaters, painted obstacles and the PID step of a 2D solve: the fields of the
    reference's ``Physics`` with the same names (src/aerolume/solvers/ns2d/physics.py:70-140),
    full-grid arrays.  The reference's own ``ops.phys`` serves as well (its tensors are then
    read in place at every step, so strokes of the paint brush and live fan settings apply)."""
    nfan: int = 0
    fan_gu: Any = None           # (nfan, ny, nx + 1) force per unit thrust on the u faces
    fan_gv: Any = None           # (nfan, ny + 1, nx)
    fan_phi: Any = None          # (nfan, ny, nx) disc-averaging weight
    fan_dir: Any = None          # (nfan, 2)
    fan_value: Any = None        # (nfan,) thrust / pressure jump / target speed
    fan_width: Any = None
    fan_kp: Any = None
    fan_ki: Any = None
    fan_dpmax: Any = None
    fan_isvel: Any = None
    fan_isthrust: Any = None
    u_floor: Any = 0.0           # the sources' speed scale
    heat: Any = None             # (ny, nx) heater density (heat transfer only)
    heat_max: Any = None
    paint: bool = False
    paint_c: Any = None          # (ny, nx), (ny, nx + 1), (ny + 1, nx) solid fractions
    paint_u: Any = None
    paint_v: Any = None
    paint_wu: Any = None         # the paint's force weights on the faces
    paint_wv: Any = None
    pid: bool = False
    ports: bool = False          # jets and vents: the combined port / paint penalisation on the
    xchi_u: Any = None           # faces, the ports' mass source, the vents' sinks, the net
    xa_u: Any = None             # volume flow and the jets' temperature penalisation
    xchi_v: Any = None
    xa_v: Any = None
    src: Any = None
    src_neg: Any = None
    q_net: Any = 0.0
    pt_chi: Any = None
    pt_a: Any = None
    n_dye: int = 0               # smoke channels (0: the single comb channel of the plain step)
    dye_inflow: Any = None       # (n_dye, ny) the channels' inlet values
    groups: Any = None           # emitter groups: (channel, weight, target, timing) or DyeGroup
    port_dye: Any = None         # {channel: (ny, nx) smoking jets' weight}
