"""Host-side construction of 2D operators and body masks for the workloads and tests.

Restates the reference's set-up (not timed, not on the GPU): ``make_ops`` follows
src/aerolume/solvers/ns2d/core.py:145-213 (inlet profile, dye comb, automatic Brinkman
permeability, LES constants) and ``build_geometry`` follows ns2d/geometry.py:61-124 and
200-340 (exact polygon signed distance, the compact half-sine mask shifted 0.32 h inside the
surface, the body window, zeroed boundary faces, rigid-rotation targets and the per-body
force / moment weights).  The step itself only consumes the resulting arrays.
"""
from __future__ import annotations

import math

import numpy as np

from .types import Geometry2D, Ops2D

ETA_PER_H = 0.05           # core.py:55
STIFFNESS_MIN = 60.0       # core.py:56
MASK_SHIFT = 0.32          # core.py:59
LES_CONSTANTS = {"smagorinsky": 0.17, "wale": 0.5, "vreman": 0.07}   # core.py:51


def auto_eta(h, re):
    """min(ETA_PER_H h, h^2 Re / STIFFNESS_MIN) (core.py:172-174)."""
    return min(ETA_PER_H * h, h * h * re / STIFFNESS_MIN)


def inlet_profile(ny, kind="uniform"):
    """1, or a parabola with discrete mean exactly 1 (core.py:145-151)."""
    if kind == "uniform":
        return np.ones(ny)
    eta = (np.arange(ny) + 0.5) / ny
    prof = 6.0 * eta * (1.0 - eta)
    return prof / prof.mean()


def dye_comb(ny):
    """Thin inlet streaks every few cells (core.py:154-159)."""
    spacing = max(6, ny // 40)
    width = max(1, spacing // 4)
    j = np.arange(ny)
    return (((j + spacing // 2) % spacing) < width).astype(np.float64)


def make_ops(nx, ny, h, re, *, x0=0.0, y0=0.0, periodic=False, closed=False, bc_top="slip", bc_bottom="slip",
             bc_left="noslip", bc_right="noslip", ground_speed=1.0, advection="upwind3", turbulence="none",
             les_constant=None, cfl=0.5, dt=None, force_ref=1.0, moment_ref=(0.25, 0.0), inlet="uniform",
             dye=False, eta=None, dtype="float32"):
    les_c = les_constant if les_constant is not None else LES_CONSTANTS.get(turbulence, 0.0)
    comb = dye and not closed
    return Ops2D(nx=nx, ny=ny, h=h, x0=x0, y0=y0, periodic=periodic, closed=closed, bc_top=bc_top,
                 bc_bottom=bc_bottom, bc_left=bc_left, bc_right=bc_right, ground_speed=ground_speed,
                 advection=advection, turbulence=turbulence, les_c=les_c, nu=1.0 / re,
                 eta=eta if eta is not None else auto_eta(h, re), cfl=cfl, dt_fixed=dt,
                 u_inlet=inlet_profile(ny, inlet), dye_inlet=(dye_comb(ny) if comb else np.zeros(ny)) if dye else None,
                 force_ref=force_ref, moment_ref=tuple(moment_ref), dtype=dtype)


def polygon_sdf(poly, x, y):
    """Signed distance to a closed polygon, negative inside: exact edge distance, even-odd
    sign (geometry.py:61-98)."""
    a = np.asarray(poly, np.float64)
    b = np.roll(a, -1, axis=0)
    ab = b - a
    ab2 = np.maximum((ab * ab).sum(-1), 1e-30)
    px, py = x.reshape(-1, 1), y.reshape(-1, 1)
    apx, apy = px - a[None, :, 0], py - a[None, :, 1]
    t = np.clip((apx * ab[None, :, 0] + apy * ab[None, :, 1]) / ab2[None], 0.0, 1.0)
    dx, dy = apx - t * ab[None, :, 0], apy - t * ab[None, :, 1]
    d2 = (dx * dx + dy * dy).min(axis=1)
    ay, by = a[None, :, 1], b[None, :, 1]
    straddle = (ay > py) != (by > py)
    xcross = a[None, :, 0] + (py - ay) * ab[None, :, 0] / np.where(by != ay, by - ay, 1e-30)
    crossings = (straddle & (px < xcross)).sum(axis=1)
    sign = 1.0 - 2.0 * (crossings % 2)
    return (sign * np.sqrt(np.maximum(d2, 1e-24))).reshape(x.shape)


def smooth_step(d, w):
    """Compact C1 solid fraction of a signed distance (geometry.py:115-118)."""
    s = np.clip(d / w, -1.0, 1.0)
    return 0.5 - 0.5 * np.sin(0.5 * math.pi * s)


def body_window(polys, ops, margin=None, mask_width=1.0):
    """Cell window covering the polygons plus a margin, clipped to the domain (geometry.py:206-223)."""
    if not polys:
        return (0, 0, 0, 0)
    pts = np.vstack([np.asarray(p, np.float64).reshape(-1, 2) for p in polys])
    m = (mask_width + 3.0 + abs(MASK_SHIFT)) if margin is None else margin
    h = ops.h
    i0 = math.floor((pts[:, 0].min() - ops.x0) / h - m)
    i1 = math.ceil((pts[:, 0].max() - ops.x0) / h + m)
    j0 = math.floor((pts[:, 1].min() - ops.y0) / h - m)
    j1 = math.ceil((pts[:, 1].max() - ops.y0) / h + m)
    i0, i1 = max(i0, 0), min(i1, ops.nx)
    j0, j1 = max(j0, 0), min(j1, ops.ny)
    if i1 <= i0 or j1 <= j0:
        return (0, 0, 0, 0)
    return (j0, j1, i0, i1)


def build_geometry(polys, ops, *, omegas=None, centers=None, mask_width=1.0):
    """Masks, solid velocities and force weights on the window (geometry.py:226-340)."""
    nb = len(polys)
    window = body_window(polys, ops, mask_width=mask_width)
    j0, j1, i0, i1 = window
    wy, wx = j1 - j0, i1 - i0
    if nb == 0 or wy <= 0 or wx <= 0:
        return Geometry2D((0, 0, 0, 0), nbody=nb)
    h = ops.h
    omegas = [0.0] * nb if omegas is None else list(omegas)
    centers = [(0.0, 0.0)] * nb if centers is None else list(centers)

    def grid(nr, nc, xoff, yoff):
        ys = ops.y0 + (np.arange(nr) + j0 + yoff) * h
        xs = ops.x0 + (np.arange(nc) + i0 + xoff) * h
        return np.meshgrid(ys, xs, indexing="ij")

    yu, xu = grid(wy, wx + 1, 0.0, 0.5)
    yv, xv = grid(wy + 1, wx, 0.5, 0.0)
    yc, xc = grid(wy, wx, 0.5, 0.5)
    w = mask_width * h
    shift = MASK_SHIFT * h
    cu = np.stack([smooth_step(polygon_sdf(p, xu, yu) + shift, w) for p in polys])
    cv = np.stack([smooth_step(polygon_sdf(p, xv, yv) + shift, w) for p in polys])
    cc = np.stack([smooth_step(polygon_sdf(p, xc, yc) + shift, w) for p in polys])
    if not ops.periodic:  # boundary faces carry boundary conditions, never penalisation
        fu = np.ones(wx + 1)
        if i0 == 0:
            fu[0] = 0.0
        if i1 == ops.nx:
            fu[-1] = 0.0
        fv = np.ones(wy + 1)
        if j0 == 0:
            fv[0] = 0.0
        if j1 == ops.ny:
            fv[-1] = 0.0
        cu = cu * fu[None, None, :]
        cv = cv * fv[None, :, None]
    chi_u = np.minimum(cu.sum(0), 1.0)
    chi_v = np.minimum(cv.sum(0), 1.0)
    chi_c = np.minimum(cc.sum(0), 1.0)
    om = np.asarray(omegas, np.float64)[:, None, None]
    cx = np.asarray([c[0] for c in centers], np.float64)[:, None, None]
    cy = np.asarray([c[1] for c in centers], np.float64)[:, None, None]
    a_u = (cu * (-om * (yu[None] - cy))).sum(0)
    a_v = (cv * (om * (xv[None] - cx))).sum(0)
    if nb == 1:
        wu, wv = np.ones_like(cu), np.ones_like(cv)
    else:
        wu = cu / (cu.sum(0, keepdims=True) + 1e-30)
        wv = cv / (cv.sum(0, keepdims=True) + 1e-30)
    xr, yr = ops.moment_ref
    k_u = np.stack([wu, wu * (yu[None] - yr)], axis=1)
    k_v = np.stack([wv, -wv * (xv[None] - xr)], axis=1)
    return Geometry2D(window, chi_u, chi_v, chi_c, a_u, a_v, k_u, k_v, nb)
