"""CPU oracle for the 2D staggered-grid Navier-Stokes step -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``, ``__graft_entry__.smoke()``
and the CPU legs of ``bench.py`` may import it.  The CUDA path in ``aerolume_b200`` never
calls into it.

It restates, in numpy, the reference's plain 2D step (Aerolume ``src/aerolume/solvers/ns2d``)
for the configurations the sm_100a kernels implement (tunnel, closed and periodic domains,
slip / no-slip / moving walls, upwind3 or central advection, Smagorinsky / WALE / Vreman,
immersed bodies, inlet-comb dye) and heat transfer (no other placed physics):

* ``step2d``            core.py:815-969   SSP-RK3 with a projection after every stage
* ``pad_u`` / ``pad_v`` core.py:284-325   two ghost layers
* ``inlet_outlet``      core.py:328-359   inlet profile and outlet mass balance
* ``advection2d``       core.py:366-414   upwind3 / central conservative advection
* ``add_diffusion``     core.py:417-424
* ``sgs_divergence2d``  core.py:427-520   eddy viscosity and div(2 nu_t S)
* ``momentum_rhs2d``    core.py:571-613   tendencies with the boundary rows
* ``project2d``         core.py:620-660   divergence, Poisson solve, u - grad psi
* ``penalise2d``        core.py:663-682
* ``cfl_dt2d``          core.py:685-696
* ``advect_dye2d``      core.py:703-735, 779-792
* ``PoissonSolver2D``   poisson.py:93-144 (the same exact solve in the orthonormal eigenbases)
* heat transfer         physics.py:623-639, 696-794, 833-923; scalar.py:34-183; core.py:774-813,
                        974-1000: bounded theta transport, diffusion with wall modes, insulated and
                        heat-flux bodies, temperature-body penalisation, buoyancy, dt limit, report

Parity is pinned: ``tests/test_oracle2d_golden.py`` checks this module against golden
vectors that ``tests/golden/make_golden2d.py`` produced by running the reference itself.

Inputs are duck-typed objects with the reference's attribute names (see
``aerolume_b200.ns2d.types``); arrays are numpy, C order ``(ny, nx)`` with the staggered
shapes of core.py:9-12: u (ny, nx + 1), v (ny + 1, nx), p (ny, nx).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .ns3d import FORCE_WEIGHTS, SSP_RK3, face_flux, lerp, neumann_basis, periodic_basis

_SQRT_EPS = 1e-30                                                  # ns2d/core.py:466
DYE_ZERO = 1e-6                                                    # ns2d/core.py:735


# ---------------------------------------------------------------------------
# boundary conditions (core.py:271-359)
# ---------------------------------------------------------------------------

def _wall_ghost(rows, kind, speed):
    if kind == "slip":
        return rows
    if kind == "noslip":
        return -rows
    return rows.dtype.type(2.0 * speed) - rows


def pad_u(u, ops):
    """(ny + 4, nx + 5): padded [j + 2, i + 2] = u[j, i] (core.py:284-305)."""
    if ops.periodic:
        up = u[:, :-1]
        up = np.concatenate([up[:, -2:], up, up[:, :3]], axis=1)
        return np.concatenate([up[-2:], up, up[:2]], axis=0)
    if ops.closed:
        ux = np.concatenate([-u[:, 1:3][:, ::-1], u, -u[:, -3:-1][:, ::-1]], axis=1)
    else:
        ux = np.concatenate([np.repeat(u[:, :1], 2, axis=1), u, np.repeat(u[:, -1:], 2, axis=1)], axis=1)
    bot = _wall_ghost(ux[:2][::-1], ops.bc_bottom, ops.ground_speed)
    top = _wall_ghost(ux[-2:][::-1], ops.bc_top, 0.0)
    return np.concatenate([bot, ux, top], axis=0)


def pad_v(v, ops):
    """(ny + 5, nx + 4): padded [j + 2, i + 2] = v[j, i] (core.py:308-325)."""
    if ops.periodic:
        vp = v[:-1]
        vp = np.concatenate([vp[-2:], vp, vp[:3]], axis=0)
        return np.concatenate([vp[:, -2:], vp, vp[:, :2]], axis=1)
    vy = np.concatenate([-v[1:3][::-1], v, -v[-3:-1][::-1]], axis=0)
    if ops.closed:
        sl = -1.0 if ops.bc_left == "noslip" else 1.0
        sr = -1.0 if ops.bc_right == "noslip" else 1.0
        T = v.dtype.type
        return np.concatenate([T(sl) * vy[:, :2][:, ::-1], vy, T(sr) * vy[:, -2:][:, ::-1]], axis=1)
    return np.concatenate([-vy[:, :2][:, ::-1], vy, np.repeat(vy[:, -1:], 2, axis=1)], axis=1)


def inlet_outlet(u, ops):
    """Inlet profile, outlet shifted so outflow = inflow (core.py:337-359)."""
    u = u.copy()
    if ops.closed:
        u[:, 0] = 0
        u[:, -1] = 0
        return u
    T = u.dtype.type
    corr = (np.asarray(ops.u_inlet, dtype=u.dtype).sum(dtype=u.dtype) - u[:, -1].sum(dtype=u.dtype)) / T(ops.ny)
    u[:, 0] = np.asarray(ops.u_inlet, dtype=u.dtype)
    u[:, -1] = u[:, -1] + corr
    return u


def apply_boundary_values(u, v, ops):
    """Dirichlet values and outlet balance; periodic duplicates (core.py:328-334)."""
    if ops.periodic:
        u = u.copy()
        v = v.copy()
        u[:, -1] = u[:, 0]
        v[-1] = v[0]
        return u, v
    u = inlet_outlet(u, ops)
    v = v.copy()
    v[0] = 0
    v[-1] = 0
    return u, v


# ---------------------------------------------------------------------------
# right-hand side (core.py:366-613)
# ---------------------------------------------------------------------------

def advection_scale(ops):
    return (7.0 / 24.0 if ops.advection == "upwind3" else 0.25) / ops.h       # core.py:369


def advection2d(U, V, ops):
    """-div(u u) at the u- and v-faces (core.py:366-383)."""
    ny, nx = ops.ny, ops.nx
    up = ops.advection == "upwind3"
    k = U.dtype.type(advection_scale(ops))
    fx = face_flux(None, U[2:-2, 0:nx + 2], U[2:-2, 1:nx + 3], U[2:-2, 2:nx + 4], U[2:-2, 3:nx + 5], up)
    vs = V[2:ny + 3, 1:nx + 2] + V[2:ny + 3, 2:nx + 3]
    gy = face_flux(vs, U[0:ny + 1, 2:-2], U[1:ny + 2, 2:-2], U[2:ny + 3, 2:-2], U[3:ny + 4, 2:-2], up)
    au = (((fx[:, :-1] - fx[:, 1:]) + gy[:-1]) - gy[1:]) * k
    us = U[1:ny + 2, 2:-2] + U[2:ny + 3, 2:-2]
    fx = face_flux(us, V[2:-2, 0:nx + 1], V[2:-2, 1:nx + 2], V[2:-2, 2:nx + 3], V[2:-2, 3:nx + 4], up)
    gy = face_flux(None, V[0:ny + 2, 2:-2], V[1:ny + 3, 2:-2], V[2:ny + 4, 2:-2], V[3:ny + 5, 2:-2], up)
    av = (((fx[:, :-1] - fx[:, 1:]) + gy[:-1]) - gy[1:]) * k
    return au, av


def add_diffusion(acc, P, nu_h2):
    """acc + nu / h^2 * 5-point Laplacian (core.py:417-424)."""
    ring = (((P[2:-2, 3:-1] + P[2:-2, 1:-3]) + P[3:-1, 2:-2]) + P[1:-3, 2:-2])
    ring = ring + P.dtype.type(-4.0) * P[2:-2, 2:-2]
    return acc + ring * nu_h2


def gradients2d(U, V, ops):
    """(g11, g12, g21, g22) at cells -1..ny x -1..nx, shear at corners (core.py:427-444)."""
    ny, nx = ops.ny, ops.nx
    inv_h = U.dtype.type(1.0 / ops.h)
    g11 = (U[1:ny + 3, 2:nx + 4] - U[1:ny + 3, 1:nx + 3]) * inv_h
    g22 = (V[2:ny + 4, 1:nx + 3] - V[1:ny + 3, 1:nx + 3]) * inv_h
    dudy = (U[1:ny + 4, 1:nx + 4] - U[0:ny + 3, 1:nx + 4]) * inv_h
    dvdx = (V[1:ny + 4, 1:nx + 4] - V[1:ny + 4, 0:nx + 3]) * inv_h
    q = U.dtype.type(0.25)

    def avg(a):
        return (((a[:-1, :-1] + a[1:, :-1]) + a[:-1, 1:]) + a[1:, 1:]) * q
    return g11, avg(dudy), avg(dvdx), g22, dudy + dvdx


def eddy_viscosity2d(g11, g12, g21, g22, ops):
    """Smagorinsky / WALE / Vreman in 2D (core.py:469-500)."""
    T = g11.dtype.type
    delta2 = ops.h * ops.h
    c = ops.les_c
    s12 = T(0.5) * (g12 + g21)
    ss = (g11 * g11 + g22 * g22) + T(2.0) * s12 * s12
    if ops.turbulence == "smagorinsky":
        return T(c * c * delta2) * np.sqrt(T(2.0) * ss + T(_SQRT_EPS))
    if ops.turbulence == "wale":
        q11 = g11 * g11 + g12 * g21
        q22 = g21 * g12 + g22 * g22
        q12 = T(0.5) * (((g11 * g12 + g12 * g22) + g21 * g11) + g22 * g21)
        tr3 = (q11 + q22) * T(1.0 / 3.0)
        sd = (((q11 - tr3) ** 2 + (q22 - tr3) ** 2) + T(2.0) * q12 * q12) + tr3 * tr3
        num = np.maximum(sd, T(0)) ** T(1.5)
        den = (np.maximum(ss, T(0)) ** T(2.5) + np.maximum(sd, T(0)) ** T(1.25)) + T(1e-30)
        return T(c * c * delta2) * num / den
    if ops.turbulence == "vreman":
        b11 = g11 * g11 + g12 * g12
        b22 = g21 * g21 + g22 * g22
        b12 = g11 * g21 + g12 * g22
        bb = np.maximum(b11 * b22 - b12 * b12, T(0))
        aa = ((g11 * g11 + g12 * g12) + g21 * g21) + g22 * g22
        return T(c * delta2) * np.sqrt(bb / (aa + T(1e-30)) + T(_SQRT_EPS))
    raise ValueError(ops.turbulence)


def sgs_divergence2d(U, V, geom, ops):
    """div(2 nu_t S) at u- and v-faces and max nu_t (core.py:503-525)."""
    ny, nx = ops.ny, ops.nx
    T = U.dtype.type
    inv_h = T(1.0 / ops.h)
    g11, g12, g21, g22, shear_k = gradients2d(U, V, ops)
    nut = eddy_viscosity2d(g11, g12, g21, g22, ops)
    if not geom.empty:
        j0, j1, i0, i1 = geom.window
        nut = nut.copy()
        nut[j0 + 1:j1 + 1, i0 + 1:i1 + 1] = nut[j0 + 1:j1 + 1, i0 + 1:i1 + 1] * (T(1.0) - geom.chi_c)
    q = T(0.25)
    sgs_divergence2d.nut = nut                     # the field, for the heat equation's diffusivity
    nut_k = (((nut[:-1, :-1] + nut[1:, :-1]) + nut[:-1, 1:]) + nut[1:, 1:]) * q
    txx = T(2.0) * nut[1:ny + 1] * g11[1:ny + 1]
    tyy = T(2.0) * nut[:, 1:nx + 1] * g22[:, 1:nx + 1]
    txy = nut_k * shear_k[1:ny + 2, 1:nx + 2]
    fu = (((txx[:, 1:] - txx[:, :-1]) + txy[1:]) - txy[:-1]) * inv_h
    fv = (((txy[:, 1:] - txy[:, :-1]) + tyy[1:]) - tyy[:-1]) * inv_h
    return fu, fv, nut.max()


WW_A, WW_B = 8.3, 1.0 / 7.0                                        # core.py:510-511


def wall_shear_excess2d(us, y, nu):
    """core.py:517-533: the Werner-Wengle shear above the resolved one, signed like us."""
    T = us.dtype.type
    a = np.abs(us)
    tau_lam = a * T(T(nu) / T(y))
    tau_ww = (a * (T(T(nu) / T(y)) ** T(WW_B)) * T(1.0 / WW_A)) ** T(2.0 / (1.0 + WW_B))
    return np.sign(us) * np.maximum(tau_ww - tau_lam, T(0.0))


def wall_model_force2d(u, v, ops):
    """core.py:536-564: the excess shear on the face rows next to the no-slip domain walls."""
    T = u.dtype.type
    y = 0.5 * ops.h
    inv_h = T(1.0 / ops.h)
    fu = np.zeros_like(u)
    if ops.bc_bottom in ("noslip", "moving"):
        us = u[:1] - T(ops.ground_speed) if ops.bc_bottom == "moving" else u[:1]
        fu[:1] = -wall_shear_excess2d(us, y, ops.nu) * inv_h
    if ops.bc_top == "noslip":
        fu[-1:] = -wall_shear_excess2d(u[-1:], y, ops.nu) * inv_h
    if not ops.closed or (ops.bc_left != "noslip" and ops.bc_right != "noslip"):
        return fu, None
    fv = np.zeros_like(v)
    if ops.bc_left == "noslip":
        fv[:, :1] = -wall_shear_excess2d(v[:, :1], y, ops.nu) * inv_h
    if ops.bc_right == "noslip":
        fv[:, -1:] = -wall_shear_excess2d(v[:, -1:], y, ops.nu) * inv_h
    return fu, fv


def momentum_rhs2d(u, v, geom, ops):
    """(Lu, Lv, nut_max) with the boundary rows / columns set (core.py:571-613)."""
    T = u.dtype.type
    U, V = pad_u(u, ops), pad_v(v, ops)
    au, av = advection2d(U, V, ops)
    nu_h2 = T(ops.nu) * T(1.0 / ops.h ** 2)
    lu = add_diffusion(au, U, nu_h2)
    lv = add_diffusion(av, V, nu_h2)
    nut_max = None
    if ops.turbulence != "none":
        fu, fv, nut_max = sgs_divergence2d(U, V, geom, ops)
        lu = lu + fu
        lv = lv + fv
    if getattr(ops, "forcing", None) is not None:   # the verification cases' uniform body force
        lu = lu + T(ops.forcing[0])
        lv = lv + T(ops.forcing[1])
    if getattr(ops, "wall_model", False):
        wu, wv = wall_model_force2d(u, v, ops)
        lu = lu + wu
        if wv is not None:
            lv = lv + wv
    if ops.periodic:
        return lu, lv, nut_max
    lu = lu.copy()
    lv = lv.copy()
    lu[:, 0] = 0
    lu[:, -1] = 0 if ops.closed else (u[:, -2] - u[:, -1]) * T(1.0 / ops.h)
    lv[0] = 0
    lv[-1] = 0
    return lu, lv, nut_max


# ---------------------------------------------------------------------------
# projection, penalisation, time step (core.py:620-696)
# ---------------------------------------------------------------------------

def divergence2d(u, v, h):
    """((u_{i+1} - u_i) + v_{j+1}) - v_j, over h (core.py:620-622)."""
    return (((u[:, 1:] - u[:, :-1]) + v[1:]) - v[:-1]) * u.dtype.type(1.0 / h)


class PoissonSolver2D:
    """Exact ``L psi = f`` with zero mean (poisson.py:93-144), in the orthonormal DCT-II /
    Hartley eigenbases (the same solution as the reference's packed real FFTs)."""

    def __init__(self, nx, ny, h, periodic, dtype):
        qx, lx = periodic_basis(nx) if periodic else neumann_basis(nx)
        qy, ly = periodic_basis(ny) if periodic else neumann_basis(ny)
        self.qx, self.qy = qx.astype(dtype), qy.astype(dtype)
        lam = ly[:, None] / (h * h) + lx[None, :] / (h * h)
        inv = np.where(lam != 0, 1.0 / np.where(lam != 0, lam, 1.0), 0.0)
        inv[0, 0] = 0.0
        self.inv_lam = inv.astype(dtype)

    def solve(self, f):
        a = f @ self.qx.T
        a = self.qy @ a
        a = a * self.inv_lam
        a = self.qy.T @ a
        return a @ self.qx

    @staticmethod
    def laplacian(psi, h, periodic):
        """The discrete operator (poisson.py:136-144)."""
        if periodic:
            pe = np.concatenate([psi[:, -1:], psi, psi[:, :1]], axis=1)
            pe = np.concatenate([pe[-1:], pe, pe[:1]], axis=0)
        else:
            pe = np.concatenate([psi[:, :1], psi, psi[:, -1:]], axis=1)
            pe = np.concatenate([pe[:1], pe, pe[-1:]], axis=0)
        return (pe[1:-1, 2:] + pe[1:-1, :-2] + pe[2:, 1:-1] + pe[:-2, 1:-1] - 4 * pe[1:-1, 1:-1]) / (h * h)


def correct2d(u, v, psi, ops):
    """u - grad psi; boundary-normal faces untouched (core.py:643-660)."""
    T = psi.dtype.type
    inv_h = T(1.0 / ops.h)
    if ops.periodic:
        gx = (psi - np.roll(psi, 1, axis=1)) * inv_h
        gy = (psi - np.roll(psi, 1, axis=0)) * inv_h
        return u - np.concatenate([gx, gx[:, :1]], axis=1), v - np.concatenate([gy, gy[:1]], axis=0)
    gx = (psi[:, 1:] - psi[:, :-1]) * inv_h
    gy = (psi[1:] - psi[:-1]) * inv_h
    zc = np.zeros_like(psi[:, :1])
    zr = np.zeros_like(psi[:1])
    return u - np.concatenate([zc, gx, zc], axis=1), v - np.concatenate([zr, gy, zr], axis=0)


def project2d(u, v, ops, poisson):
    psi = poisson.solve(divergence2d(u, v, ops.h))
    un, vn = correct2d(u, v, psi, ops)
    return un, vn, psi


def penalise2d(u, v, geom, ops, bdt):
    """Implicit Brinkman on the window; returns (u, v, du, dv) (core.py:663-682)."""
    T = u.dtype.type
    j0, j1, i0, i1 = geom.window
    k = bdt / T(ops.eta)
    u = u.copy()
    v = v.copy()
    uw = u[j0:j1, i0:i1 + 1]
    vw = v[j0:j1 + 1, i0:i1]
    un = (uw + k * geom.a_u) / (T(1.0) + k * geom.chi_u)
    vn = (vw + k * geom.a_v) / (T(1.0) + k * geom.chi_v)
    du, dv = un - uw, vn - vw
    u[j0:j1, i0:i1 + 1] = un
    v[j0:j1 + 1, i0:i1] = vn
    return u, v, du, dv


def cfl_dt2d(u, v, ops, nut_max=None):
    """min(cfl h / (max|u| + max|v|), 0.25 h^2 / (nu + max nu_t)) (core.py:685-696)."""
    T = u.dtype.type
    umax = max(np.abs(u).max() + np.abs(v).max(), T(1e-6))
    dt = T(ops.cfl * ops.h) / umax
    nu = T(ops.nu) if nut_max is None else T(ops.nu) + nut_max
    return min(dt, T(0.25 * ops.h * ops.h) / nu)


# ---------------------------------------------------------------------------
# dye (core.py:703-735, 779-792)
# ---------------------------------------------------------------------------

def _van_leer(a, b):
    ab = a * b
    s = a + b
    out = np.zeros_like(ab)
    m = ab > 0
    out[m] = a.dtype.type(2.0) * ab[m] / s[m]
    return out


def advect_dye2d(c, u, v, dt, ops):
    """Forward-Euler MUSCL / van Leer step of the dye, cut below 1e-6, clamped at 1."""
    T = c.dtype.type
    if ops.periodic:
        cx = np.concatenate([c[:, -2:], c, c[:, :2]], axis=1)
        cy = np.concatenate([c[-2:], c, c[:2]], axis=0)
    else:
        inlet = np.asarray(ops.dye_inlet, dtype=c.dtype).reshape(-1, 1)
        cx = np.concatenate([np.repeat(inlet, 2, axis=1), c, np.repeat(c[:, -1:], 2, axis=1)], axis=1)
        cy = np.concatenate([np.repeat(c[:1], 2, axis=0), c, np.repeat(c[-1:], 2, axis=0)], axis=0)
    half = T(0.5)
    s = _van_leer(cx[:, 1:-1] - cx[:, :-2], cx[:, 2:] - cx[:, 1:-1])
    left = cx[:, 1:-2] + half * s[:, :-1]
    right = cx[:, 2:-1] - half * s[:, 1:]
    fx = u * np.where(u > 0, left, right)
    s = _van_leer(cy[1:-1] - cy[:-2], cy[2:] - cy[1:-1])
    low = cy[1:-2] + half * s[:-1]
    high = cy[2:-1] - half * s[1:]
    fy = v * np.where(v > 0, low, high)
    c = c - (dt * T(1.0 / ops.h)) * (((fx[:, 1:] - fx[:, :-1]) + fy[1:]) - fy[:-1])
    c = np.where(c > T(DYE_ZERO), c, T(0))
    return np.minimum(c, T(1.0))


def zero_dye_in_solids(c, geom):
    if geom.empty:
        return c
    c = c.copy()
    j0, j1, i0, i1 = geom.window
    c[j0:j1, i0:i1] = c[j0:j1, i0:i1] * (geom.chi_c <= 0.5).astype(c.dtype)
    return c


# ---------------------------------------------------------------------------
# the step (core.py:815-969)
# ---------------------------------------------------------------------------

def force_coefficients2d(acc_u, acc_v, geom, ops, dt):
    """[Cd, Cl, Cm] per body (core.py:943-949), reduced in float64."""
    if geom.empty:
        return np.zeros((geom.nbody, 3))
    denom = float(dt * dt.dtype.type(0.5) * dt.dtype.type(ops.force_ref))
    scale = -(ops.h * ops.h) / denom
    ku = np.asarray(geom.k_u, np.float64)
    kv = np.asarray(geom.k_v, np.float64)
    ru = np.einsum("bkij,ij->bk", ku, np.asarray(acc_u, np.float64))
    rv = np.einsum("bkij,ij->bk", kv, np.asarray(acc_v, np.float64))
    return np.stack([ru[:, 0], rv[:, 0], ru[:, 1] + rv[:, 1]], axis=1) * scale


@dataclass
class StepResult2D:
    u: np.ndarray
    v: np.ndarray
    p: np.ndarray
    t: np.ndarray
    dt: np.ndarray
    coeffs: np.ndarray
    dye: np.ndarray | None = None


def step2d(u0, v0, t, geom, ops, poisson, *, dye=None, dt=None):
    """One SSP-RK3 step (core.py:815-969 without placed physics)."""
    T = u0.dtype.type
    up, vp = u0, v0
    acc_u = acc_v = psi_w = None
    for s, ((a, b), w) in enumerate(zip(SSP_RK3, FORCE_WEIGHTS)):
        lu, lv, nut_max = momentum_rhs2d(up, vp, geom, ops)
        if s == 0 and dt is None:
            dt = T(ops.dt_fixed) if ops.dt_fixed is not None else cfl_dt2d(u0, v0, ops, nut_max)
        dt = T(dt)
        bdt = dt * T(b)
        if a == 0.0:
            uh = up + lu * bdt
            vh = vp + lv * bdt
        else:
            uh = lerp(up, u0, a) + lu * bdt
            vh = lerp(vp, v0, a) + lv * bdt
        if not ops.periodic:
            uh = inlet_outlet(uh, ops)
        if not geom.empty:
            uh, vh, du, dv = penalise2d(uh, vh, geom, ops, bdt)
            acc_u = du * T(w) if acc_u is None else acc_u + du * T(w)
            acc_v = dv * T(w) if acc_v is None else acc_v + dv * T(w)
            if ops.periodic:
                uh, vh = apply_boundary_values(uh, vh, ops)
        up, vp, psi = project2d(uh, vh, ops, poisson)
        psi_w = psi * T(w) if psi_w is None else psi_w + T(w) * psi
    p = psi_w * (T(1.0) / dt)
    coeffs = force_coefficients2d(acc_u, acc_v, geom, ops, dt)
    new_dye = None
    if dye is not None:
        new_dye = zero_dye_in_solids(advect_dye2d(dye, up, vp, dt, ops), geom)
    return StepResult2D(up, vp, p, np.asarray(t + dt, dtype=u0.dtype), np.asarray(dt, dtype=u0.dtype), coeffs,
                        new_dye)


# ---------------------------------------------------------------------------
# heat transfer (physics.py:623-923, scalar.py:34-183, core.py:774-1000)
# ---------------------------------------------------------------------------

@dataclass
class Thermal2D:
    """The thermal part of the reference's 2D ``Physics`` (physics.py:305-322) and the
    bodies' ``ThermalGeometry`` (geometry.py:120-158); arrays on the body window."""
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
    chi_t: np.ndarray | None = None
    a_t: np.ndarray | None = None
    w_t: np.ndarray | None = None
    ins_u: np.ndarray | None = None
    ins_v: np.ndarray | None = None
    q_skin: np.ndarray | None = None
    w_f: np.ndarray | None = None
    vol_u: np.ndarray | None = None
    vol_v: np.ndarray | None = None


def _van_leer_scalar(a, b):
    """scalar.py:34-39: 2ab / (a + b) where ab > 0, else 0."""
    ab = a * b
    out = np.zeros_like(ab)
    m = ab > 0
    out[m] = a.dtype.type(2.0) * ab[m] / (a + b)[m]
    return out


def tvd_fluxes(c, u, v, ops, inflow):
    """MUSCL / van Leer advective fluxes u c, v c (scalar.py:63-84)."""
    T = c.dtype.type
    half = T(0.5)
    if ops.periodic:
        cx = np.concatenate([c[:, -2:], c, c[:, :2]], axis=1)
        cy = np.concatenate([c[-2:], c, c[:2]], axis=0)
    else:
        right = np.repeat(c[:, -1:], 2, axis=1)
        left = np.repeat(c[:, :1], 2, axis=1) if ops.closed else np.full_like(right, T(inflow))
        cx = np.concatenate([left, c, right], axis=1)
        cy = np.concatenate([np.repeat(c[:1], 2, axis=0), c, np.repeat(c[-1:], 2, axis=0)], axis=0)
    s = _van_leer_scalar(cx[:, 1:-1] - cx[:, :-2], cx[:, 2:] - cx[:, 1:-1])
    left = cx[:, 1:-2] + half * s[:, :-1]
    right = cx[:, 2:-1] - half * s[:, 1:]
    fx = u * np.where(u > 0, left, right)
    s = _van_leer_scalar(cy[1:-1] - cy[:-2], cy[2:] - cy[1:-1])
    low = cy[1:-2] + half * s[:-1]
    high = cy[2:-1] - half * s[1:]
    fy = v * np.where(v > 0, low, high)
    return fx, fy


def flux_divergence(fx, fy, h):
    """-(div F) at the cells (scalar.py:87-89)."""
    return (((fx[:, :-1] - fx[:, 1:]) + fy[:-1]) - fy[1:]) * fx.dtype.type(1.0 / h)


def face_average_x(q, ops):
    T = q.dtype.type
    mid = T(0.5) * (q[:, 1:] + q[:, :-1])
    if ops.periodic:
        w = T(0.5) * (q[:, :1] + q[:, -1:])
        return np.concatenate([w, mid, w], axis=1)
    return np.concatenate([q[:, :1], mid, q[:, -1:]], axis=1)


def face_average_y(q, ops):
    T = q.dtype.type
    mid = T(0.5) * (q[1:] + q[:-1])
    if ops.periodic:
        w = T(0.5) * (q[:1] + q[-1:])
        return np.concatenate([w, mid, w], axis=0)
    return np.concatenate([q[:1], mid, q[-1:]], axis=0)


def diffusive_fluxes(c, kx, ky, ops, modes, values):
    """F = -kappa grad c with the wall conditions on the boundary faces (scalar.py:100-146)."""
    T = c.dtype.type
    inv_h, inv_half = T(1.0 / ops.h), T(2.0 / ops.h)
    kx_a, ky_a = np.ndim(kx) > 0, np.ndim(ky) > 0
    kxi = kx[:, 1:-1] if kx_a else kx
    kyi = ky[1:-1] if ky_a else ky
    fxi = -(kxi * (c[:, 1:] - c[:, :-1])) * inv_h
    fyi = -(kyi * (c[1:] - c[:-1])) * inv_h
    kl = kx[:, :1] if kx_a else kx
    kr = kx[:, -1:] if kx_a else kx
    kb = ky[:1] if ky_a else ky
    kt = ky[-1:] if ky_a else ky
    first_x, last_x, first_y, last_y = c[:, :1], c[:, -1:], c[:1], c[-1:]

    def side(mode, k, inner, value, sign, wrap):
        if mode in ("temperature", "inlet"):
            return (T(-sign) * inv_half) * k * (inner - T(value))
        if mode == "heat_flux":
            return (T(sign) * k) * T(value) * np.ones_like(inner)
        if mode == "periodic":
            return wrap
        return np.zeros_like(inner)

    wrap_x = -(kl * (first_x - last_x)) * inv_h if modes[0] == "periodic" else None
    wrap_y = -(kb * (first_y - last_y)) * inv_h if modes[2] == "periodic" else None
    fl = side(modes[0], kl, first_x, values[0], 1.0, wrap_x)
    fr = side(modes[1], kr, last_x, values[1], -1.0, wrap_x)
    fb = side(modes[2], kb, first_y, values[2], 1.0, wrap_y)
    ft = side(modes[3], kt, last_y, values[3], -1.0, wrap_y)
    fl, fr = (np.broadcast_to(x, (c.shape[0], 1)) for x in (fl, fr))
    fb, ft = (np.broadcast_to(x, (1, c.shape[1])) for x in (fb, ft))
    return np.concatenate([fl, fxi, fr], axis=1), np.concatenate([fb, fyi, ft], axis=0)


def theta_rhs2d(th, u, v, nut, geom, tp, ops):
    """Tendency of theta: bounded advection, diffusion with kappa (+ nu_t / Pr_t), insulated
    bodies, wall conditions, heat-flux skins (physics.py:696-730, without heaters or vents)."""
    T = th.dtype.type
    ny, nx = th.shape
    fx, fy = tvd_fluxes(th, u, v, ops, tp.theta_in)
    lt = flux_divergence(fx, fy, ops.h)
    kappa = T(tp.kappa)
    insulated = tp.ins_u is not None and not geom.empty
    if nut is not None:
        nc = nut[1:-1, 1:-1] * T(1.0 / tp.prt)
        kx = kappa + face_average_x(nc, ops)
        ky = kappa + face_average_y(nc, ops)
    elif insulated:
        kx = np.full((ny, nx + 1), kappa, dtype=th.dtype)
        ky = np.full((ny + 1, nx), kappa, dtype=th.dtype)
    else:
        kx = ky = kappa
    if insulated:
        j0, j1, i0, i1 = geom.window
        kx = kx.copy()
        ky = ky.copy()
        kx[j0:j1, i0:i1 + 1] = kx[j0:j1, i0:i1 + 1] * tp.ins_u
        ky[j0:j1 + 1, i0:i1] = ky[j0:j1 + 1, i0:i1] * tp.ins_v
    Fx, Fy = diffusive_fluxes(th, kx, ky, ops, tp.wall_modes, tp.wall_values)
    lt = lt + flux_divergence(Fx, Fy, ops.h)
    if tp.flux_ids and not geom.empty:
        j0, j1, i0, i1 = geom.window
        lt = lt.copy()
        lt[j0:j1, i0:i1] = lt[j0:j1, i0:i1] + kappa * tp.q_skin
    return lt


def penalise_theta2d(th, geom, tp, bdt):
    """Implicit penalisation toward the temperature bodies; their heat (physics.py:733-757)."""
    T = th.dtype.type
    if not tp.temp_ids or geom.empty:
        return th, None
    k = T(bdt / T(tp.eta_t))
    j0, j1, i0, i1 = geom.window
    tw = th[j0:j1, i0:i1]
    tn = (tw + k * tp.a_t) / (T(1.0) + k * tp.chi_t)
    heat = np.einsum("bij,ij->b", tp.w_t.astype(np.float64), (tn - tw).astype(np.float64))
    th = th.copy()
    th[j0:j1, i0:i1] = tn
    return th, heat


def buoyancy2d(theta, tp, ops):
    """-Ri theta g on the faces, zero on the boundary faces of a bounded domain (physics.py:623-637)."""
    T = theta.dtype.type
    gx, gy = tp.gravity
    fu = fv = None
    if gy != 0.0:
        tv = face_average_y(theta, ops)
        if not ops.periodic:
            tv = tv.copy()
            tv[0] = 0
            tv[-1] = 0
        fv = tv * T(T(tp.ri) * T(-gy))
    if gx != 0.0:
        tu = face_average_x(theta, ops)
        if not ops.periodic:
            tu = tu.copy()
            tu[:, 0] = 0
            tu[:, -1] = 0
        fu = tu * T(T(tp.ri) * T(-gx))
    return fu, fv


def physics_dt_limit2d(dt, u, v, theta, nut_max, tp, ops):
    """The bounded temperature step and the buoyant free-fall limit (physics.py:851-884)."""
    T = u.dtype.type
    kap = T(tp.kappa) if nut_max is None else T(tp.kappa) + nut_max * T(1.0 / tp.prt)
    speed = max(np.abs(u).max() + np.abs(v).max(), T(0.0))
    rate = speed * T(2.0 / ops.h) + kap * T(tp.diff_coef / (ops.h * ops.h))
    dt = min(dt, T(1.0) / rate)
    acc = T(abs(tp.ri)) * np.abs(theta).max()
    return min(dt, T(ops.cfl) * np.sqrt(T(ops.h) / max(acc, T(1e-12))))


def heat_report2d(old_theta, new_theta, new_u, heat_acc, geom, tp, ops, dt):
    """The step's heat outputs (core.py:974-995, physics.py:760-794)."""
    T = new_theta.dtype.type
    h = ops.h
    h2 = T(h * h)
    out = {}
    if tp.temp_ids and not geom.empty:
        out["heat"] = heat_acc * float(h2 / dt)
    if tp.flux_ids and not geom.empty:
        j0, j1, i0, i1 = geom.window
        out["theta_wall"] = np.einsum("bij,ij->b", tp.w_f.astype(np.float64), new_theta[j0:j1, i0:i1].astype(np.float64))
    k = T(tp.kappa)
    first = (new_theta[:, 0], new_theta[:, -1], new_theta[0, :], new_theta[-1, :])
    rates = []
    for i, mode in enumerate(tp.wall_modes):
        if mode in ("temperature", "inlet"):
            rates.append(float((T(2.0) * k) * (T(tp.wall_values[i]) - first[i]).sum()))
        elif mode == "heat_flux":
            rates.append(float(k * T(tp.wall_values[i]) * T(first[i].size * h)))
        else:
            rates.append(0.0)
    out["wall_heat"] = np.array(rates)
    out["heat_storage"] = np.array([float((new_theta.sum() - old_theta.sum()) * (h2 / dt))])
    if ops.periodic or ops.closed:
        out["flow_heat"] = np.zeros(2)
    else:
        out["flow_heat"] = np.array([float((new_u[:, 0] * T(tp.theta_in)).sum() * T(h)),
                                     float((new_u[:, -1] * new_theta[:, -1]).sum() * T(h))])
    return out


def step2d_thermal(u0, v0, t, theta0, geom, ops, poisson, tp, *, dt=None):
    """One SSP-RK3 step with heat transfer (core.py:815-969 with a thermal Physics): the
    momentum of step2d plus theta transport, buoyancy after the penalisation (its solid share
    booked against the body force), theta penalisation, and the heat report."""
    T = u0.dtype.type
    up, vp, thp = u0, v0, theta0
    acc_u = acc_v = psi_w = heat_acc = None
    les = ops.turbulence != "none"
    for s, ((a, b), w) in enumerate(zip(SSP_RK3, FORCE_WEIGHTS)):
        lu, lv, nut_max = momentum_rhs2d(up, vp, geom, ops)
        nut = sgs_divergence2d.nut if les else None
        if s == 0 and dt is None:
            if ops.dt_fixed is not None:
                dt = T(ops.dt_fixed)
            else:
                dt = cfl_dt2d(u0, v0, ops, nut_max)
                dt = physics_dt_limit2d(dt, u0, v0, theta0, nut_max, tp, ops)
        dt = T(dt)
        lt = theta_rhs2d(thp, up, vp, nut, geom, tp, ops)
        bdt = dt * T(b)
        if a == 0.0:
            uh = up + lu * bdt
            vh = vp + lv * bdt
            thh = thp + lt * bdt
        else:
            uh = lerp(up, u0, a) + lu * bdt
            vh = lerp(vp, v0, a) + lv * bdt
            thh = lerp(thp, theta0, a) + lt * bdt
        if not ops.periodic:
            uh = inlet_outlet(uh, ops)
        if not geom.empty:
            uh, vh, du, dv = penalise2d(uh, vh, geom, ops, bdt)
            acc_u = du * T(w) if acc_u is None else acc_u + du * T(w)
            acc_v = dv * T(w) if acc_v is None else acc_v + dv * T(w)
        if tp.ri != 0.0:  # core.py:774-813
            fu, fv = buoyancy2d(thp, tp, ops)
            if fu is not None:
                uh = uh + bdt * fu
            if fv is not None:
                vh = vh + bdt * fv
            if not geom.empty:
                j0, j1, i0, i1 = geom.window
                vu = tp.vol_u if tp.vol_u is not None else geom.chi_u
                vv = tp.vol_v if tp.vol_v is not None else geom.chi_v
                if fu is not None:
                    acc_u = acc_u + fu[j0:j1, i0:i1 + 1] * vu * T(bdt * T(w))
                if fv is not None:
                    acc_v = acc_v + fv[j0:j1 + 1, i0:i1] * vv * T(bdt * T(w))
        if ops.periodic and not geom.empty:
            uh, vh = apply_boundary_values(uh, vh, ops)
        thh, heat = penalise_theta2d(thh, geom, tp, bdt)
        if heat is not None:
            heat_acc = heat * float(T(w)) if heat_acc is None else heat_acc + heat * float(T(w))
        thp = thh
        up, vp, psi = project2d(uh, vh, ops, poisson)
        psi_w = psi * T(w) if psi_w is None else psi_w + T(w) * psi
    p = psi_w * (T(1.0) / dt)
    coeffs = force_coefficients2d(acc_u, acc_v, geom, ops, dt)
    res = StepResult2D(up, vp, p, np.asarray(t + dt, dtype=u0.dtype), np.asarray(dt, dtype=u0.dtype), coeffs)
    res.theta = thp
    res.report = heat_report2d(theta0, thp, up, heat_acc, geom, tp, ops, dt)
    return res


# ---------------------------------------------------------------------------
# placed physics besides heat: fans, heaters, painted obstacles, the PID step
# (physics.py:434-496, 578-694, 696-730, 805-884; diagnostics.py:104-124; core.py:815-1003)
# ---------------------------------------------------------------------------

PID_TARGET, PID_GAINS, PID_MAX_GROWTH = 0.9, (0.10, 0.25, 0.02), 1.03    # diagnostics.py:46-48
FAN_CTRL_OFFSET = 2                                                     # physics.py:140


@dataclass
class Placed2D:
    """The reference's 2D ``Physics`` fields of fans, heaters, paint and the PID step
    (physics.py:70-140), as numpy arrays of the step's dtype."""
    nfan: int = 0
    fan_gu: np.ndarray | None = None        # (nf, ny, nx + 1) force per unit thrust
    fan_gv: np.ndarray | None = None        # (nf, ny + 1, nx)
    fan_phi: np.ndarray | None = None       # (nf, ny, nx) averaging weight
    fan_dir: np.ndarray | None = None       # (nf, 2)
    fan_value: np.ndarray | None = None
    fan_width: np.ndarray | None = None
    fan_kp: np.ndarray | None = None
    fan_ki: np.ndarray | None = None
    fan_dpmax: np.ndarray | None = None
    fan_isvel: np.ndarray | None = None
    fan_isthrust: np.ndarray | None = None
    pid: bool = False
    u_floor: float = 0.0
    heat: np.ndarray | None = None          # (ny, nx) heat-rate density
    heat_max: float | None = None
    paint_c: np.ndarray | None = None
    paint_u: np.ndarray | None = None
    paint_v: np.ndarray | None = None
    paint_wu: np.ndarray | None = None
    paint_wv: np.ndarray | None = None
    # jets and vents (physics.py:362-433): the combined port / paint penalisation (xchi, xa on
    # the faces), the mass source of the projection, the vents' sinks (with the uniform leak of
    # a closed box), the net volume flow, the jets' temperature penalisation
    ports: bool = False
    xchi_u: np.ndarray | None = None
    xa_u: np.ndarray | None = None
    xchi_v: np.ndarray | None = None
    xa_v: np.ndarray | None = None
    src: np.ndarray | None = None
    src_neg: np.ndarray | None = None
    q_net: float = 0.0
    pt_chi: np.ndarray | None = None
    pt_a: np.ndarray | None = None
    # smoke channels (physics.py:497-540, 795-830): the channels' inlet values (n, ny), the
    # emitter groups [(channel, weight, target, timing)] in the reference's sorted order and the
    # smoking jets' weights {channel: (ny, nx)}
    n_dye: int = 0
    dye_inflow: np.ndarray | None = None
    groups: list = None
    port_dye: dict = None

    @property
    def paint(self):
        return self.paint_u is not None


def pid_dt2d(dt_limit, dt_prev, ctrl):
    """diagnostics.py:104-124: the PID-controlled step and the new controller memory."""
    T = type(dt_limit)
    kp, ki, kd = (T(g) for g in PID_GAINS)
    target = T(PID_TARGET) * dt_limit
    first = dt_prev <= 0
    safe_prev = target if first else T(dt_prev)
    e = np.log(T(target / safe_prev))
    e1, e2 = ctrl[0], ctrl[1]
    step = ki * e + kp * (e - e1) + kd * ((e - T(2.0) * e1) + e2)
    grow = np.exp(min(step, T(np.log(PID_MAX_GROWTH))))
    dt = target if first else min(safe_prev * grow, dt_limit)
    e = T(0.0) if first else e
    new = ctrl.copy()
    new[0], new[1] = e, e1
    return T(dt), new


def fan_control2d(u, v, ctrl, dt, pl):
    """physics.py:640-672: disc velocities, the PI controller, the thrusts and the new memory."""
    T = u.dtype.type
    uc = T(0.5) * (u[:, 1:] + u[:, :-1])
    vc = T(0.5) * (v[1:] + v[:-1])
    ua = np.einsum("kij,ij->k", pl.fan_phi, uc)
    va = np.einsum("kij,ij->k", pl.fan_phi, vc)
    ud = ua * pl.fan_dir[:, 0] + va * pl.fan_dir[:, 1]
    o = FAN_CTRL_OFFSET
    integ = ctrl[o::2]
    err = pl.fan_value - ud
    ilim = pl.fan_dpmax / pl.fan_ki
    integ_new = np.maximum(np.minimum(integ + err * T(dt) * pl.fan_isvel, ilim), -ilim)
    dp_pi = np.maximum(np.minimum(pl.fan_kp * err + pl.fan_ki * integ_new, pl.fan_dpmax), -pl.fan_dpmax)
    thrust_fixed = np.where(pl.fan_isthrust > 0, pl.fan_value, pl.fan_value * pl.fan_width)
    thrust = np.where(pl.fan_isvel > 0, dp_pi * pl.fan_width, thrust_fixed)
    dp = thrust / pl.fan_width
    new = np.concatenate([ctrl[:o], np.stack([integ_new, dp], axis=1).reshape(-1)]).astype(u.dtype)
    return thrust.astype(u.dtype), new, ud.astype(u.dtype)


def placed_dt_limit2d(dt, u, v, theta, nut_max, tp, pl, ops):
    """physics.py:851-884 with the sources' speed floor and the heaters' bounds."""
    T = u.dtype.type
    if pl is not None and (pl.nfan or pl.ports):
        dt = min(dt, T(ops.cfl) * T(ops.h) / max(T(pl.u_floor), T(1e-6)))
    if tp is not None and theta is not None:
        kap = T(tp.kappa) if nut_max is None else T(tp.kappa) + nut_max * T(1.0 / tp.prt)
        u_floor = T(pl.u_floor) if pl is not None else T(0.0)
        speed = max(np.abs(u).max() + np.abs(v).max(), u_floor)
        rate = speed * T(2.0 / ops.h) + kap * T(tp.diff_coef / (ops.h * ops.h))
        dt = min(dt, T(1.0) / rate)
        acc = T(abs(tp.ri)) * np.abs(theta).max()
        dt = min(dt, T(ops.cfl) * np.sqrt(T(ops.h) / max(acc, T(1e-12))))
        if pl is not None and pl.heat_max is not None:
            s_max = max(T(pl.heat_max), T(1e-12))
            dt = min(dt, T(1.0) / s_max)
            dt = min(dt, (T(6.0 * ops.cfl * ops.h) / max(T(abs(tp.ri)) * s_max, T(1e-12))) ** T(1.0 / 3.0))
    return T(dt)


def theta_rhs2d_placed(th, u, v, nut, geom, tp, pl, ops):
    """physics.py:696-730 with the heaters and the paint's insulation."""
    T = th.dtype.type
    ny, nx = th.shape
    fx, fy = tvd_fluxes(th, u, v, ops, tp.theta_in)
    lt = flux_divergence(fx, fy, ops.h)
    kappa = T(tp.kappa)
    insulated = tp.ins_u is not None and not geom.empty
    paint = pl is not None and pl.paint
    if nut is not None:
        nc = nut[1:-1, 1:-1] * T(1.0 / tp.prt)
        kx = kappa + face_average_x(nc, ops)
        ky = kappa + face_average_y(nc, ops)
    elif paint or insulated:
        kx = np.full((ny, nx + 1), kappa, dtype=th.dtype)
        ky = np.full((ny + 1, nx), kappa, dtype=th.dtype)
    else:
        kx = ky = kappa
    if paint:
        kx = kx * (T(1.0) - pl.paint_u)
        ky = ky * (T(1.0) - pl.paint_v)
    if insulated:
        j0, j1, i0, i1 = geom.window
        kx = kx.copy()
        ky = ky.copy()
        kx[j0:j1, i0:i1 + 1] = kx[j0:j1, i0:i1 + 1] * tp.ins_u
        ky[j0:j1 + 1, i0:i1] = ky[j0:j1 + 1, i0:i1] * tp.ins_v
    Fx, Fy = diffusive_fluxes(th, kx, ky, ops, tp.wall_modes, tp.wall_values)
    lt = lt + flux_divergence(Fx, Fy, ops.h)
    if pl is not None and pl.heat is not None:
        lt = lt + pl.heat
    if tp.flux_ids and not geom.empty:
        j0, j1, i0, i1 = geom.window
        lt = lt.copy()
        lt[j0:j1, i0:i1] = lt[j0:j1, i0:i1] + kappa * tp.q_skin
    if pl is not None and pl.ports:
        lt = lt + pl.src_neg * th                 # fluid leaving through a vent takes its heat along
    return lt


def emitter_on2d(t, timing):
    """physics.py:795-802: 1 while an emitter group releases at time t."""
    T = type(t)
    start, stop, period, duty = (T(x) for x in timing)
    active = (t >= start) and (t < stop)
    safe = period if period > 0 else T(1.0)
    r = np.fmod(T(t - start), safe)
    if r != 0 and ((safe < 0) != (r < 0)):
        r = r + safe
    phase = T(r / safe)
    return T(1.0) if (active and (period <= 0 or phase < duty)) else T(0.0)


def _dye_fluxes2d(c, u, v, ops, inflow):
    """scalar.py:42-83 for one channel: the limited (van Leer) face values with the inlet
    value left of a tunnel (inflow: (ny,)), replicated cells elsewhere, wrap when periodic."""
    T = c.dtype.type
    ny, nx = c.shape
    if ops.periodic:
        cx = np.concatenate([c[:, -2:], c, c[:, :2]], axis=1)
        cy = np.concatenate([c[-2:], c, c[:2]], axis=0)
    else:
        right = np.repeat(c[:, -1:], 2, axis=1)
        left = np.repeat(c[:, :1], 2, axis=1) if ops.closed else np.repeat(inflow.reshape(ny, 1), 2, axis=1)
        cx = np.concatenate([left, c, right], axis=1)
        cy = np.concatenate([np.repeat(c[:1], 2, axis=0), c, np.repeat(c[-1:], 2, axis=0)], axis=0)
    s = _van_leer_scalar(cx[:, 1:-1] - cx[:, :-2], cx[:, 2:] - cx[:, 1:-1])
    left_v = cx[:, 1:-2] + T(0.5) * s[:, :-1]
    right_v = cx[:, 2:-1] - T(0.5) * s[:, 1:]
    fx = u * np.where(u > 0, left_v, right_v)
    s = _van_leer_scalar(cy[1:-1] - cy[:-2], cy[2:] - cy[1:-1])
    low = cy[1:-2] + T(0.5) * s[:-1]
    high = cy[2:-1] - T(0.5) * s[1:]
    fy = v * np.where(v > 0, low, high)
    return fx, fy


def update_dye2d(chans, u, v, dt, t, geom, pl, ops):
    """physics.py:805-830: every smoke channel one forward-Euler step with the end-of-step
    velocity, the vents' sink, the emitter groups and smoking jets, solids and paint, the floor."""
    T = u.dtype.type
    out = []
    for ch, c in enumerate(chans):
        fx, fy = _dye_fluxes2d(c, u, v, ops, pl.dye_inflow[ch].astype(c.dtype))
        c = c + T(dt) * flux_divergence(fx, fy, ops.h)
        if pl.ports:
            c = c + (T(dt) * pl.src_neg) * c
        out.append(c)
    for ch, w, target, timing in pl.groups or []:
        on = emitter_on2d(T(t), timing)
        out[ch] = out[ch] + (w * on) * (target - out[ch])
    for ch, w in (pl.port_dye or {}).items():
        out[ch] = out[ch] + w * (T(1.0) - out[ch])
    res = []
    for c in out:
        c = zero_dye_in_solids(c, geom) if not geom.empty else c
        if pl.paint:
            c = c * (pl.paint_c <= 0.5).astype(c.dtype)
        res.append(np.minimum(np.where(c > T(1e-6), c, T(0.0)), T(1.0)))
    return res


def step2d_placed(u0, v0, t, geom, ops, poisson, *, tp=None, pl=None, theta0=None, dye=None, dt_prev=0.0,
                  ctrl=None, dt=None, dye_extra=None):
    """One SSP-RK3 step (core.py:815-969) with heat transfer (``tp``), fans, heaters, painted
    obstacles and the PID step (``pl``); ``ctrl`` is the controller memory (PID errors, then
    (integral, pressure jump) per fan) and ``dt_prev`` the previous step (0: first)."""
    T = u0.dtype.type
    up, vp = u0, v0
    thermal = tp is not None and theta0 is not None
    thp = theta0
    acc_u = acc_v = psi_w = heat_acc = paint_acc = jet_acc = None
    fan_f = fan_thrust = fan_ud = None
    les = ops.turbulence != "none"
    paint = pl is not None and pl.paint
    ports = pl is not None and pl.ports
    for s, ((a, b), w) in enumerate(zip(SSP_RK3, FORCE_WEIGHTS)):
        lu, lv, nut_max = momentum_rhs2d(up, vp, geom, ops)
        nut = sgs_divergence2d.nut if (les and thermal) else None
        if s == 0:
            if dt is None:
                if ops.dt_fixed is not None:
                    dt = T(ops.dt_fixed)
                else:
                    dt = cfl_dt2d(u0, v0, ops, nut_max)
                    if pl is not None or thermal:
                        dt = placed_dt_limit2d(dt, u0, v0, theta0, nut_max, tp if thermal else None, pl, ops)
                    if pl is not None and pl.pid:
                        dt, ctrl = pid_dt2d(T(dt), dt_prev, ctrl)
            dt = T(dt)
            if pl is not None and pl.nfan:
                fan_thrust, ctrl, fan_ud = fan_control2d(u0, v0, ctrl, dt, pl)
                fan_f = (np.einsum("k,kij->ij", fan_thrust, pl.fan_gu), np.einsum("k,kij->ij", fan_thrust, pl.fan_gv))
        if fan_f is not None:
            lu = lu + fan_f[0]
            lv = lv + fan_f[1]
        lt = theta_rhs2d_placed(thp, up, vp, nut, geom, tp, pl, ops) if thermal else None
        bdt = dt * T(b)
        if a == 0.0:
            uh = up + lu * bdt
            vh = vp + lv * bdt
        else:
            uh = lerp(up, u0, a) + lu * bdt
            vh = lerp(vp, v0, a) + lv * bdt
        if lt is not None:
            thh = (thp if a == 0.0 else lerp(thp, theta0, a)) + lt * bdt
        if not ops.periodic:
            if ports and not ops.closed:   # core.py:352-356: the outflow also carries the ports' net flow
                T_ = uh.dtype.type
                uh = uh.copy()
                corr = ((np.asarray(ops.u_inlet, dtype=uh.dtype).sum(dtype=uh.dtype) + T_(pl.q_net) * T_(1.0 / ops.h))
                        - uh[:, -1].sum(dtype=uh.dtype)) / T_(ops.ny)
                uh[:, 0] = np.asarray(ops.u_inlet, dtype=uh.dtype)
                uh[:, -1] = uh[:, -1] + corr
            else:
                uh = inlet_outlet(uh, ops)
        if not geom.empty:
            uh, vh, du, dv = penalise2d(uh, vh, geom, ops, bdt)
            acc_u = du * T(w) if acc_u is None else acc_u + du * T(w)
            acc_v = dv * T(w) if acc_v is None else acc_v + dv * T(w)
        if paint or ports:   # physics.py:675-683: the combined penalisation, the paint's impulse
            k = T(bdt / T(ops.eta))
            if ports:
                un = (uh + k * pl.xa_u) / (T(1.0) + k * pl.xchi_u)
                vn = (vh + k * pl.xa_v) / (T(1.0) + k * pl.xchi_v)
            else:
                un = uh / (T(1.0) + k * pl.paint_u)
                vn = vh / (T(1.0) + k * pl.paint_v)
            if paint:
                imp = np.array([((un - uh) * pl.paint_wu).sum(), ((vn - vh) * pl.paint_wv).sum()], dtype=np.float64)
                paint_acc = imp * float(T(w)) if paint_acc is None else paint_acc + imp * float(T(w))
            uh, vh = un, vn
        if thermal and tp.ri != 0.0:  # core.py:774-813
            fu, fv = buoyancy2d(thp, tp, ops)
            if fu is not None:
                uh = uh + bdt * fu
            if fv is not None:
                vh = vh + bdt * fv
            if not geom.empty:
                j0, j1, i0, i1 = geom.window
                vu = tp.vol_u if tp.vol_u is not None else geom.chi_u
                vv = tp.vol_v if tp.vol_v is not None else geom.chi_v
                if fu is not None:
                    acc_u = acc_u + fu[j0:j1, i0:i1 + 1] * vu * T(bdt * T(w))
                if fv is not None:
                    acc_v = acc_v + fv[j0:j1 + 1, i0:i1] * vv * T(bdt * T(w))
            if paint and paint_acc is not None:
                su = float((fu * pl.paint_u * pl.paint_wu).sum()) if fu is not None else 0.0
                sv = float((fv * pl.paint_v * pl.paint_wv).sum()) if fv is not None else 0.0
                paint_acc = paint_acc + np.array([su, sv]) * float(bdt * T(w))
        if ops.periodic and (paint or ports or not geom.empty):
            uh, vh = apply_boundary_values(uh, vh, ops)
        if lt is not None:
            thh, heat = penalise_theta2d(thh, geom, tp, bdt)
            if heat is not None:
                heat_acc = heat * float(T(w)) if heat_acc is None else heat_acc + heat * float(T(w))
            if ports and pl.pt_chi is not None:   # physics.py:753-756: the jets' temperature
                kt = T(bdt / T(tp.eta_t))
                tn = (thh + kt * pl.pt_a) / (T(1.0) + kt * pl.pt_chi)
                jh = float((tn - thh).astype(np.float64).sum())
                jet_acc = jh * float(T(w)) if jet_acc is None else jet_acc + jh * float(T(w))
                thh = tn
            thp = thh
        if ports:   # core.py:626-642: div u = the ports' mass source
            psi = poisson.solve(divergence2d(uh, vh, ops.h) - pl.src)
            up, vp = correct2d(uh, vh, psi, ops)
        else:
            up, vp, psi = project2d(uh, vh, ops, poisson)
        psi_w = psi * T(w) if psi_w is None else psi_w + T(w) * psi
    p = psi_w * (T(1.0) / dt)
    coeffs = force_coefficients2d(acc_u, acc_v, geom, ops, dt)
    new_dye = new_extra = None
    if dye is not None and pl is not None and pl.n_dye:
        chans = [dye] + (list(dye_extra) if dye_extra is not None else [])
        res_ch = update_dye2d(chans, up, vp, dt, T(t + dt), geom, pl, ops)
        new_dye = res_ch[0]
        new_extra = np.stack(res_ch[1:]) if len(res_ch) > 1 else None
    elif dye is not None:
        new_dye = zero_dye_in_solids(advect_dye2d(dye, up, vp, dt, ops), geom)
        if paint:
            new_dye = new_dye * (pl.paint_c <= 0.5).astype(new_dye.dtype)
    res = StepResult2D(up, vp, p, np.asarray(t + dt, dtype=u0.dtype), np.asarray(dt, dtype=u0.dtype), coeffs,
                       new_dye)
    res.dye_extra = new_extra
    res.theta = thp if thermal else None
    res.ctrl = ctrl
    res.report = heat_report2d(theta0, thp, up, heat_acc, geom, tp, ops, dt) if thermal else {}
    if thermal and ports:
        h2 = ops.h * ops.h
        res.report["vent_heat"] = np.array([-float((pl.src_neg * thp).astype(np.float64).sum()) * h2])
        if jet_acc is not None:
            res.report["jet_heat"] = np.array([jet_acc * h2 / float(dt)])
    if fan_thrust is not None:
        res.report["fan_thrust"] = fan_thrust
        res.report["fan_ud"] = fan_ud
    if paint_acc is not None:
        res.report["paint_force"] = paint_acc * float(-(ops.h * ops.h) / (float(dt) * 0.5 * ops.force_ref))
    return res
