"""Host-side set-up of a 3D case: operators, box-body masks, heat transfer and smoke nozzles.

This is the not-timed input side of the step (mask construction runs once per
configuration).  Each builder restates the reference's rule so that a case built here
matches one the reference builds from the same description:

* :func:`ghost_rules`      core.py:147-181
* :func:`make_ops`         core.py:135-137, 184-203 (auto eta, LES constants ns2d/core.py:51-61)
* :func:`box_geometry`     geometry.py:265-268 (smooth step), 323-356 (window), 385-495 (masks);
                           the signed distance of an axis-aligned box is exact in closed form,
                           where the reference evaluates it from the box's triangle mesh
* :func:`thermal_ops`      physics.py:290-294 (thermal eta), 314-461 (masks), 494-560 (sides)
* :func:`rake_sources`     dye.py:154-213 (nozzle weights)

Arrays are numpy float64 until :class:`~aerolume_b200.ns3d.plan.Ns3dPlan` uploads them
in the field dtype.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .types import DyeSources, Geometry3D, Ops3D, ThermalGeometry, ThermalOps

ETA_PER_H = 0.05            # ns2d/core.py:56
STIFFNESS_MIN = 60.0        # ns2d/core.py:57
MASK_SHIFT = 0.32           # ns2d/core.py:61
LES_CONSTANTS = {"smagorinsky": 0.17, "wale": 0.5, "vreman": 0.07}   # ns2d/core.py:51
NOZZLE_DEPTH_CELLS = 1.0    # dye.py:69
WALL_SIDES = ("left", "right", "front", "back", "bottom", "top")


def ghost_rules(*, periodic=False, bc_y="slip", bc_zmin="slip", bc_zmax="slip", ground_speed=1.0, closed=False,
                bc_x="noslip"):
    """Ghost rule per component and axis (core.py:147-181)."""
    px, py, pz = (True, True, True) if periodic else (False, bc_y == "periodic", False)
    pc, pf = ("periodic_cell", 0.0), ("periodic_face", 0.0)
    even, odd, edge, fodd = ("even", 0.0), ("odd", 0.0), ("edge", 0.0), ("face_odd", 0.0)
    zlo_tan = {"slip": even, "noslip": odd, "moving": ("affine", float(ground_speed))}[bc_zmin]
    zlo_v = {"slip": even, "noslip": odd, "moving": odd}[bc_zmin]
    zhi = {"slip": even, "noslip": odd}[bc_zmax]
    y_tan = odd if bc_y == "noslip" else even
    if closed:
        x_tan = odd if bc_x == "noslip" else even
        ux, vx = (fodd, fodd), (x_tan, x_tan)
    else:
        ux, vx = (edge, edge), (odd, edge)
    u = ((pf, pf) if px else ux, (pc, pc) if py else (y_tan, y_tan), (pc, pc) if pz else (zlo_tan, zhi))
    v = ((pc, pc) if px else vx, (pf, pf) if py else (fodd, fodd), (pc, pc) if pz else (zlo_v, zhi))
    w = ((pc, pc) if px else vx, (pc, pc) if py else (y_tan, y_tan), (pf, pf) if pz else (fodd, fodd))
    return {"u": u, "v": v, "w": w}


def auto_eta(h, re):
    """Brinkman permeability rule (core.py:135-137)."""
    return min(ETA_PER_H * h, h * h * re / STIFFNESS_MIN)


def make_ops(nx, ny, nz, h, *, re, x0=0.0, y0=0.0, z0=0.0, periodic=False, bc_y="slip", bc_zmin="slip",
             bc_zmax="slip", ground_speed=1.0, domain="tunnel", bc_x="noslip", advection="upwind3",
             turbulence="none", cfl=0.5, dt=None, eta=None, les_constant=None, ref_area=1.0, length_ref=1.0,
             span_ref=1.0, moment_ref=(0.0, 0.0, 0.0), dtype="float32") -> Ops3D:
    """Operators of one configuration (core.py:184-203)."""
    closed = domain == "closed"
    pax = (True, True, True) if periodic else (False, bc_y == "periodic", False)
    les_c = les_constant if les_constant is not None else LES_CONSTANTS.get(turbulence, 0.0)
    return Ops3D(nx=nx, ny=ny, nz=nz, h=h, x0=x0, y0=y0, z0=z0, periodic_axes=pax, closed=closed,
                 symmetry=(bc_y == "symmetry_ymin" and not periodic), advection=advection, turbulence=turbulence,
                 les_c=les_c, nu_value=1.0 / re, eta=eta if eta is not None else auto_eta(h, re), cfl=cfl,
                 dt_fixed=dt, ghost=ghost_rules(periodic=periodic, bc_y=bc_y, bc_zmin=bc_zmin, bc_zmax=bc_zmax,
                                                ground_speed=ground_speed, closed=closed, bc_x=bc_x),
                 u_inlet=np.ones((nz, ny)), ref_area=ref_area, length_ref=length_ref, span_ref=span_ref,
                 moment_ref=tuple(moment_ref), dtype=dtype)


@dataclass
class Box:
    """An axis-aligned box body: extents, centre and heat-transfer mode (ImmersedMesh's
    ``thermal`` / ``thermal_value``, config.py:80-140)."""
    size: tuple
    center: tuple
    thermal: str = "adiabatic"
    thermal_value: float = 0.0

    @property
    def bounds(self):
        c = np.asarray(self.center, float)
        half = 0.5 * np.asarray(self.size, float)
        return c - half, c + half


def box_sdf(box: Box, X, Y, Z):
    """Exact signed distance to the box surface (negative inside)."""
    c = np.asarray(box.center, float)
    half = 0.5 * np.asarray(box.size, float)
    qx, qy, qz = np.abs(X - c[0]) - half[0], np.abs(Y - c[1]) - half[1], np.abs(Z - c[2]) - half[2]
    outside = np.sqrt(np.maximum(qx, 0.0) ** 2 + np.maximum(qy, 0.0) ** 2 + np.maximum(qz, 0.0) ** 2)
    inside = np.minimum(np.maximum(np.maximum(qx, qy), qz), 0.0)
    return outside + inside


def smooth_step(d, w):
    """Compact C1 solid fraction (geometry.py:265-268)."""
    s = np.clip(d / w, -1.0, 1.0)
    return 0.5 - 0.5 * np.sin(0.5 * math.pi * s)


def body_window(boxes, ops, mask_width=1.0):
    """Cell window of the bodies plus a margin, clipped (geometry.py:323-356)."""
    if not boxes:
        return (0, 0, 0, 0, 0, 0)
    lo = np.min([b.bounds[0] for b in boxes], axis=0)
    hi = np.max([b.bounds[1] for b in boxes], axis=0)
    margin = mask_width + 3.0 + abs(MASK_SHIFT)
    h = ops.h
    i0 = math.floor((lo[0] - ops.x0) / h - margin)
    i1 = math.ceil((hi[0] - ops.x0) / h + margin)
    j0 = math.floor((lo[1] - ops.y0) / h - margin)
    j1 = math.ceil((hi[1] - ops.y0) / h + margin)
    k0 = math.floor((lo[2] - ops.z0) / h - margin)
    k1 = math.ceil((hi[2] - ops.z0) / h + margin)
    return (max(k0, 0), min(k1, ops.nz), max(j0, 0), min(j1, ops.ny), max(i0, 0), min(i1, ops.nx))


def _grid_coords(ops, win, g):
    """Broadcastable (Z, Y, X) of grid g ("u", "v", "w", "c") over a cell window."""
    k0, k1, j0, j1, i0, i1 = win
    h = ops.h
    xs = ops.x0 + (np.arange(i0, i1 + 1) * h if g == "u" else (np.arange(i0, i1) + 0.5) * h)
    ys = ops.y0 + (np.arange(j0, j1 + 1) * h if g == "v" else (np.arange(j0, j1) + 0.5) * h)
    zs = ops.z0 + (np.arange(k0, k1 + 1) * h if g == "w" else (np.arange(k0, k1) + 0.5) * h)
    return zs[:, None, None], ys[None, :, None], xs[None, None, :]


def _zero_boundary(arr, win, ops, g):
    """Faces on non-periodic domain boundaries carry boundary conditions (geometry.py:416-439)."""
    k0, k1, j0, j1, i0, i1 = win
    px, py, pz = ops.periodic_axes
    arr = arr.copy()
    if g == "u" and not px:
        if i0 == 0:
            arr[..., 0] = 0.0
        if i1 == ops.nx:
            arr[..., -1] = 0.0
    if g == "v" and not py:
        if j0 == 0:
            arr[:, 0] = 0.0
        if j1 == ops.ny:
            arr[:, -1] = 0.0
    if g == "w" and not pz:
        if k0 == 0:
            arr[0] = 0.0
        if k1 == ops.nz:
            arr[-1] = 0.0
    return arr


def box_geometry(boxes, ops, mask_width=1.0, window=None):
    """Masks, (zero) solid velocities and force weights of box bodies (geometry.py:385-495)."""
    nb = len(boxes)
    win = body_window(boxes, ops, mask_width) if window is None else tuple(window)
    k0, k1, j0, j1, i0, i1 = win
    if nb == 0 or k1 <= k0 or j1 <= j0 or i1 <= i0:
        return Geometry3D((0, 0, 0, 0, 0, 0), nbody=nb)
    h = ops.h
    w, shift = mask_width * h, MASK_SHIFT * h
    chis = {}
    for g in ("u", "v", "w", "c"):
        Z, Y, X = _grid_coords(ops, win, g)
        per = np.stack([smooth_step(box_sdf(b, X, Y, Z) + shift, w) for b in boxes])
        if g != "c":
            per = np.stack([_zero_boundary(p, win, ops, g) for p in per])
        chis[g] = per
    cu, cv, cw, cc = chis["u"], chis["v"], chis["w"], chis["c"]
    chi_u, chi_v, chi_w, chi_c = (np.minimum(x.sum(0), 1.0) for x in (cu, cv, cw, cc))
    if nb == 1:
        wu, wv, ww = np.ones_like(cu), np.ones_like(cv), np.ones_like(cw)
    else:
        wu, wv, ww = (x / (x.sum(0, keepdims=True) + 1e-30) for x in (cu, cv, cw))
    xr, yr, zr = ops.moment_ref
    zu, yu, _ = _grid_coords(ops, win, "u")
    zv, _, xv = _grid_coords(ops, win, "v")
    _, yw, xw = _grid_coords(ops, win, "w")
    k_u = np.stack([wu * np.ones_like(chi_u), wu * (zu - zr), -wu * (yu - yr)], axis=1)
    k_v = np.stack([wv * np.ones_like(chi_v), -wv * (zv - zr), wv * (xv - xr)], axis=1)
    k_w = np.stack([ww * np.ones_like(chi_w), ww * (yw - yr), -ww * (xw - xr)], axis=1)
    return Geometry3D(win, chi_u=chi_u, chi_v=chi_v, chi_w=chi_w, chi_c=chi_c, a_u=np.zeros_like(chi_u),
                      a_v=np.zeros_like(chi_v), a_w=np.zeros_like(chi_w), k_u=k_u, k_v=k_v, k_w=k_w, nbody=nb)


def auto_eta_thermal(h, pe):
    """physics.py:290-294."""
    return min(ETA_PER_H * h, h * h * pe / STIFFNESS_MIN)


def thermal_ops(ops, geom, boxes, *, re, prandtl=0.71, richardson=0.0, prandtl_turbulent=0.85, walls=None,
                theta_inlet=0.0, side_walls=None, mask_width=1.0, eta=None) -> ThermalOps:
    """Heat-equation constants, side conditions and body masks (physics.py:314-560).

    ``side_walls`` gives the velocity condition per side (config.py ``side_walls``); ``walls``
    maps a side to (mode, value) for walls ("adiabatic" when unlisted)."""
    walls = walls or {}
    pe = re * prandtl
    if side_walls is None:
        side_walls = dict(zip(WALL_SIDES, ("inflow", "outflow", "slip", "slip", "slip", "slip")))
    kinds, vals = [], []
    for side in WALL_SIDES:
        vel = side_walls[side]
        if vel == "periodic":
            kind, val = "periodic", 0.0
        elif vel == "inflow":
            kind, val = "inflow", theta_inlet
        elif vel == "outflow":
            kind, val = "outflow", 0.0
        elif vel == "symmetry":
            kind, val = "adiabatic", 0.0
        else:
            kind, val = walls.get(side, ("adiabatic", 0.0))
        kinds.append(kind)
        vals.append(float(val))
    win = geom.window
    nb = len(boxes)
    tg = ThermalGeometry(win, nbody=nb, flux_rate=np.zeros(nb))
    if not geom.empty:
        h = ops.h
        w, shift = mask_width * h, MASK_SHIFT * h
        t_index = [b for b, box in enumerate(boxes) if box.thermal == "temperature"]
        if any(box.thermal == "heat_flux" for box in boxes):
            raise NotImplementedError("heat-flux box bodies are not built here (pass the reference's masks)")
        tg.t_index = t_index
        Zc, Yc, Xc = _grid_coords(ops, win, "c")
        if t_index:
            cc = np.stack([smooth_step(box_sdf(boxes[b], Xc, Yc, Zc) + shift, w) for b in t_index])
            tg.chi_t = np.minimum(cc.sum(0), 1.0)
            theta = np.array([boxes[b].thermal_value for b in t_index])
            tg.a_t = (cc * theta[:, None, None, None]).sum(0)
            tg.w_t = np.ones_like(cc) if len(t_index) == 1 else cc / (cc.sum(0, keepdims=True) + 1e-30)
        adia = [b for b, box in enumerate(boxes) if box.thermal == "adiabatic"]
        if adia:
            fr = []
            for g in ("u", "v", "w"):
                Z, Y, X = _grid_coords(ops, win, g)
                chi = np.minimum(np.stack([smooth_step(box_sdf(boxes[b], X, Y, Z) + shift, w) for b in adia]).sum(0), 1.0)
                fr.append(_zero_boundary(chi, win, ops, g))
            tg.adia = tuple(fr)
        Z, Y, X = _grid_coords(ops, win, "w")
        vol = np.minimum(np.stack([smooth_step(box_sdf(b, X, Y, Z), w) for b in boxes]).sum(0), 1.0)
        tg.vol_w = _zero_boundary(vol, win, ops, "w")
    return ThermalOps(kappa=1.0 / pe, pe=pe, ri=float(richardson), prt=float(prandtl_turbulent),
                      eta=eta if eta is not None else auto_eta_thermal(ops.h, pe), side_kinds=tuple(kinds),
                      side_vals=tuple(vals), geom=tg, h=ops.h, symmetry=ops.symmetry)


def _ramp(d, edge, h):
    return np.clip((edge + 0.5 * h - d) / h, 0.0, 1.0)


def rake_sources(positions, ops, radius=None) -> DyeSources:
    """Nozzle weights of a rake of round nozzles (dye.py:154-213, kind "rake")."""
    h = ops.h
    pos = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    r = radius if radius else 1.25 * h
    depth = NOZZLE_DEPTH_CELLS * h
    lo = pos.min(axis=0) - np.array([depth, r, r]) - h
    hi = pos.max(axis=0) + np.array([depth, r, r]) + h
    i0, j0, k0 = (math.floor((lo[a] - o) / h) for a, o in ((0, ops.x0), (1, ops.y0), (2, ops.z0)))
    i1, j1, k1 = (math.ceil((hi[a] - o) / h) for a, o in ((0, ops.x0), (1, ops.y0), (2, ops.z0)))
    i0, i1 = max(i0, 0), min(i1, ops.nx)
    j0, j1 = max(j0, 0), min(j1, ops.ny)
    k0, k1 = max(k0, 0), min(k1, ops.nz)
    if i1 <= i0 or j1 <= j0 or k1 <= k0:
        return DyeSources((0, 0, 0, 0, 0, 0), np.zeros((0, 0, 0)))
    Z, Y, X = _grid_coords(ops, (k0, k1, j0, j1, i0, i1), "c")
    w = np.zeros(np.broadcast_shapes(Z.shape, Y.shape, X.shape))
    for px, py, pz in pos:
        rr = np.sqrt((Y - py) ** 2 + (Z - pz) ** 2)
        w = np.maximum(w, _ramp(rr, r, h) * _ramp(np.abs(X - px), depth, h))
    return DyeSources((k0, k1, j0, j1, i0, i1), w, (2.0, 1.0))


__all__ = ["Box", "auto_eta", "auto_eta_thermal", "body_window", "box_geometry", "box_sdf", "ghost_rules", "make_ops",
           "rake_sources", "smooth_step", "thermal_ops"]
