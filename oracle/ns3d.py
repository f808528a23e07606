"""CPU oracle for the 3D staggered-grid Navier-Stokes step -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it.  The
CUDA path in ``aerolume_b200`` never calls into it.

It restates, in numpy, the reference's plain-torch 3D step with the placed physics that
the sm_100a kernels implement (Aerolume ``src/aerolume/solvers/ns3d``):

* ``step3d_phys``        core.py:765-883   SSP-RK3 with a projection after every stage
* ``pad3``/ghost rules   core.py:147-272   two ghost layers, rules composed axis by axis
* ``advection3``         core.py:331-390   upwind3 / central conservative advection
* ``sgs_divergence3d``   core.py:400-524   Smagorinsky / WALE / Vreman eddy viscosity
* ``penalise3d``         core.py:615-634   implicit Brinkman penalisation on the window
* ``force_coefficients`` core.py:653-678
* ``PoissonSolver3D``    poisson.py:74-157 exact solve in the per-axis eigenbases
* ``ThermalOps``         physics.py:494-790 heat equation, buoyancy, heat rates
* ``Physics3D.dt_rule``  physics.py:1230-1262 (with the sources' speed floor and ``PidDt``,
                         physics.py:1144-1181)
* ``PaintLayer``         physics.py:1074-1141 painted solids, penalised after the bodies
* ``FanSet``             physics.py:831-979 actuator discs: disc velocity, PI thrust, forces
* ``PortSet``            physics.py:981-1072 jets and vents: forces, mass sources, theta sources
* smoke                  dye.py:232-312    MUSCL / van Leer advection, solids, nozzles

Parity is pinned: ``tests/test_oracle_golden.py`` checks this module against golden
vectors that ``tests/golden/make_golden.py`` produced by running the reference itself
(float64 to 1e-12, float32 to round-off).

Inputs are duck-typed objects with the reference's attribute names (see
``aerolume_b200.ns3d`` for the concrete containers); arrays are numpy, C order
``(nz, ny, nx)`` with the staggered shapes of core.py:11-14.
"""
from __future__ import annotations

import math

import numpy as np

SSP_RK3 = ((0.0, 1.0), (0.75, 0.25), (1.0 / 3.0, 2.0 / 3.0))     # ns2d/core.py:47
FORCE_WEIGHTS = (1.0 / 6.0, 2.0 / 3.0, 1.0)                       # ns2d/core.py:49
VISCOUS_DT = 1.0 / 6.0                                            # ns3d/core.py:51
THETA_COURANT_MAX = 0.5                                           # ns3d/physics.py:82
DYE_FLOOR = 1e-8                                                  # ns3d/dye.py:63
_SQRT_EPS = 1e-30                                                 # ns3d/core.py:54


def lerp(start, end, weight):
    """torch.lerp's two-branch formula (the reference's RK stage blend, core.py:823)."""
    T = start.dtype.type
    if weight < 0.5:
        return start + T(weight) * (end - start)
    return end - (end - start) * T(1.0 - weight)


def _narrow(x, dim, start, length):
    sl = [slice(None)] * x.ndim
    sl[dim] = slice(start, start + length)
    return x[tuple(sl)]


# ---------------------------------------------------------------------------
# ghost cells (core.py:223-278)
# ---------------------------------------------------------------------------

def _ghost_slabs(x, dim, lo, hi):
    """The two ghost layers below and above ``x`` along ``dim`` (core.py:223-246)."""
    n = x.shape[dim]

    def make(rule, side):
        kind, val = rule
        low = side == "lo"
        if kind == "edge":
            return _narrow(x, dim, 0 if low else n - 1, 1)
        if kind in ("even", "odd", "affine"):
            m = np.flip(_narrow(x, dim, 0 if low else n - 2, 2), dim)
            if kind == "even":
                return m
            if kind == "odd":
                return -m
            return x.dtype.type(2.0 * val) - m
        if kind == "face_odd":
            return -np.flip(_narrow(x, dim, 1 if low else n - 3, 2), dim)
        if kind == "periodic_cell":
            return _narrow(x, dim, n - 2 if low else 0, 2)
        if kind == "periodic_face":
            return _narrow(x, dim, n - 3 if low else 1, 2)
        raise ValueError(kind)

    return make(lo, "lo"), make(hi, "hi")


def pad3(x, rules):
    """``x`` with two ghost layers per side, x first, then y, then z (core.py:249-272)."""
    nz, ny, nx = x.shape
    out = np.empty((nz + 4, ny + 4, nx + 4), dtype=x.dtype)
    rx, ry, rz = rules
    lo, hi = _ghost_slabs(x, 2, *rx)
    out[2:-2, 2:-2, 2:-2] = x
    out[2:-2, 2:-2, 0:2] = lo
    out[2:-2, 2:-2, nx + 2:] = hi
    mid = out[2:-2]
    lo, hi = _ghost_slabs(mid[:, 2:-2], 1, *ry)
    out[2:-2, 0:2] = lo
    out[2:-2, ny + 2:] = hi
    lo, hi = _ghost_slabs(out[2:-2], 0, *rz)
    out[0:2] = lo
    out[nz + 2:] = hi
    return out


def pad_velocity(u, v, w, ops):
    g = ops.ghost
    return pad3(u, g["u"]), pad3(v, g["v"]), pad3(w, g["w"])


def inlet_outlet(u, ops, source=None):
    """Inlet profile and outlet mass balance (core.py:281-297); ``source`` is the ports' net
    mass flux in outlet-face units (or None)."""
    u = u.copy()
    if ops.closed:
        u[..., 0] = 0.0
        u[..., -1] = 0.0
        return u
    T = u.dtype.type
    corr = (ops.u_inlet.sum(dtype=u.dtype) - u[..., -1].sum(dtype=u.dtype)) * T(1.0 / (ops.nz * ops.ny))
    if source is not None:
        corr = T(corr + T(T(source) * T(1.0 / (ops.nz * ops.ny))))
    u[..., -1] = u[..., -1] + corr
    u[..., 0] = ops.u_inlet
    return u


def sync_periodic(u, v, w, ops):
    """Duplicate faces of periodic axes (core.py:300-309)."""
    px, py, pz = ops.periodic_axes
    if px:
        u = u.copy()
        u[..., -1] = u[..., 0]
    if py:
        v = v.copy()
        v[:, -1] = v[:, 0]
    if pz:
        w = w.copy()
        w[-1] = w[0]
    return u, v, w


def apply_boundary_values(u, v, w, ops):
    """All Dirichlet values (core.py:312-324)."""
    px, py, pz = ops.periodic_axes
    if not px:
        u = inlet_outlet(u, ops)
    if not py:
        v = v.copy()
        v[:, 0] = 0.0
        v[:, -1] = 0.0
    if not pz:
        w = w.copy()
        w[0] = 0.0
        w[-1] = 0.0
    return sync_periodic(u, v, w, ops)


# ---------------------------------------------------------------------------
# right-hand side (core.py:331-570)
# ---------------------------------------------------------------------------

def face_flux(vsum, a, b, c, d, upwind):
    """Scaled upwind3 / central flux through the b|c face (core.py:331-345)."""
    T = b.dtype.type
    s = b + c
    vsum = s if vsum is None else vsum
    if not upwind:
        return vsum * s
    cen = s + T(-1.0 / 7.0) * (a + d)
    dis = (b - c) + T(-1.0 / 3.0) * (a - d)
    return vsum * cen + T(3.0 / 7.0) * np.abs(vsum) * dis


def advection_scale(ops):
    return (7.0 / 24.0 if ops.advection == "upwind3" else 0.25) / ops.h        # core.py:348-350


def advection3(U, V, W, ops):
    """-div(u u) at the u-, v- and w-faces (core.py:353-390)."""
    nz, ny, nx = ops.nz, ops.ny, ops.nx
    up = ops.advection == "upwind3"
    k = U.dtype.type(advection_scale(ops))
    m = slice(2, -2)
    fx = face_flux(None, U[m, m, 0:nx + 2], U[m, m, 1:nx + 3], U[m, m, 2:nx + 4], U[m, m, 3:nx + 5], up)
    au = fx[..., :-1] - fx[..., 1:]
    vs = V[m, 2:ny + 3, 1:nx + 2] + V[m, 2:ny + 3, 2:nx + 3]
    g = face_flux(vs, U[m, 0:ny + 1, m], U[m, 1:ny + 2, m], U[m, 2:ny + 3, m], U[m, 3:ny + 4, m], up)
    au = au + (g[:, :-1] - g[:, 1:])
    ws = W[2:nz + 3, m, 1:nx + 2] + W[2:nz + 3, m, 2:nx + 3]
    g = face_flux(ws, U[0:nz + 1, m, m], U[1:nz + 2, m, m], U[2:nz + 3, m, m], U[3:nz + 4, m, m], up)
    au = (au + (g[:-1] - g[1:])) * k
    us = U[m, 1:ny + 2, m] + U[m, 2:ny + 3, m]
    g = face_flux(us, V[m, m, 0:nx + 1], V[m, m, 1:nx + 2], V[m, m, 2:nx + 3], V[m, m, 3:nx + 4], up)
    av = g[..., :-1] - g[..., 1:]
    g = face_flux(None, V[m, 0:ny + 2, m], V[m, 1:ny + 3, m], V[m, 2:ny + 4, m], V[m, 3:ny + 5, m], up)
    av = av + (g[:, :-1] - g[:, 1:])
    ws = W[2:nz + 3, 1:ny + 2, m] + W[2:nz + 3, 2:ny + 3, m]
    g = face_flux(ws, V[0:nz + 1, m, m], V[1:nz + 2, m, m], V[2:nz + 3, m, m], V[3:nz + 4, m, m], up)
    av = (av + (g[:-1] - g[1:])) * k
    us = U[1:nz + 2, m, m] + U[2:nz + 3, m, m]
    g = face_flux(us, W[m, m, 0:nx + 1], W[m, m, 1:nx + 2], W[m, m, 2:nx + 3], W[m, m, 3:nx + 4], up)
    aw = g[..., :-1] - g[..., 1:]
    vs = V[1:nz + 2, m, m] + V[2:nz + 3, m, m]
    g = face_flux(vs, W[m, 0:ny + 1, m], W[m, 1:ny + 2, m], W[m, 2:ny + 3, m], W[m, 3:ny + 4, m], up)
    aw = aw + (g[:, :-1] - g[:, 1:])
    g = face_flux(None, W[0:nz + 2, m, m], W[1:nz + 3, m, m], W[2:nz + 4, m, m], W[3:nz + 5, m, m], up)
    aw = (aw + (g[:-1] - g[1:])) * k
    return au, av, aw


def laplacian_padded(P):
    """h^2 times the 7-point Laplacian on the interior (core.py:393-397)."""
    m = slice(2, -2)
    ring = (P[m, m, 3:-1] + P[m, m, 1:-3]) + (P[m, 3:-1, m] + P[m, 1:-3, m]) + (P[3:-1, m, m] + P[1:-3, m, m])
    return ring - P.dtype.type(6.0) * P[m, m, m]


def velocity_gradient(U, V, W, h):
    """Gradient tensor at centres -1..n and edge shears (core.py:400-434)."""
    nz, ny, nx = U.shape[0] - 4, U.shape[1] - 4, U.shape[2] - 5
    inv = U.dtype.type(1.0 / h)
    q = U.dtype.type(0.25)
    g11 = (U[1:nz + 3, 1:ny + 3, 2:nx + 4] - U[1:nz + 3, 1:ny + 3, 1:nx + 3]) * inv
    g22 = (V[1:nz + 3, 2:ny + 4, 1:nx + 3] - V[1:nz + 3, 1:ny + 3, 1:nx + 3]) * inv
    g33 = (W[2:nz + 4, 1:ny + 3, 1:nx + 3] - W[1:nz + 3, 1:ny + 3, 1:nx + 3]) * inv
    dudy = (U[1:nz + 3, 1:ny + 4, 1:nx + 4] - U[1:nz + 3, 0:ny + 3, 1:nx + 4]) * inv
    dvdx = (V[1:nz + 3, 1:ny + 4, 1:nx + 4] - V[1:nz + 3, 1:ny + 4, 0:nx + 3]) * inv
    dudz = (U[1:nz + 4, 1:ny + 3, 1:nx + 4] - U[0:nz + 3, 1:ny + 3, 1:nx + 4]) * inv
    dwdx = (W[1:nz + 4, 1:ny + 3, 1:nx + 4] - W[1:nz + 4, 1:ny + 3, 0:nx + 3]) * inv
    dvdz = (V[1:nz + 4, 1:ny + 4, 1:nx + 3] - V[0:nz + 3, 1:ny + 4, 1:nx + 3]) * inv
    dwdy = (W[1:nz + 4, 1:ny + 4, 1:nx + 3] - W[1:nz + 4, 0:ny + 3, 1:nx + 3]) * inv

    def a_xy(t):
        return (t[:, :-1, :-1] + t[:, 1:, :-1] + t[:, :-1, 1:] + t[:, 1:, 1:]) * q

    def a_xz(t):
        return (t[:-1, :, :-1] + t[1:, :, :-1] + t[:-1, :, 1:] + t[1:, :, 1:]) * q

    def a_yz(t):
        return (t[:-1, :-1] + t[1:, :-1] + t[:-1, 1:] + t[1:, 1:]) * q

    g = ((g11, a_xy(dudy), a_xz(dudz)),
         (a_xy(dvdx), g22, a_yz(dvdz)),
         (a_xz(dwdx), a_yz(dwdy), g33))
    return {"g": g, "sxy": dudy + dvdx, "sxz": dudz + dwdx, "syz": dvdz + dwdy}


def traceless(g):
    """g33 := -(g11 + g22) (core.py:437-445)."""
    return (g[0], g[1], (g[2][0], g[2][1], -(g[0][0] + g[1][1])))


def eddy_viscosity3d(g, ops):
    """Smagorinsky / WALE / Vreman eddy viscosity (core.py:448-482)."""
    T = g[0][0].dtype.type
    delta2 = ops.h * ops.h
    c = ops.les_c
    s = [[T(0.5) * (g[i][j] + g[j][i]) for j in range(3)] for i in range(3)]
    ss = 0
    for i in range(3):
        for j in range(3):
            ss = ss + s[i][j] * s[i][j]
    if ops.turbulence == "smagorinsky":
        return T(c * c * delta2) * np.sqrt(T(2.0) * ss + T(_SQRT_EPS))
    if ops.turbulence == "wale":
        g2 = [[sum(g[i][k] * g[k][j] for k in range(3)) for j in range(3)] for i in range(3)]
        tr3 = (g2[0][0] + g2[1][1] + g2[2][2]) * T(1.0 / 3.0)
        sd = T(0.0)
        for i in range(3):
            for j in range(3):
                sdij = T(0.5) * (g2[i][j] + g2[j][i])
                if i == j:
                    sdij = sdij - tr3
                sd = sd + sdij * sdij
        sdp = np.maximum(sd, T(0.0))
        num = sdp ** T(1.5)
        den = np.maximum(ss, T(0.0)) ** T(2.5) + sdp ** T(1.25) + T(1e-30)
        return T(c * c * delta2) * num / den
    if ops.turbulence == "vreman":
        b = [[sum(g[i][m] * g[j][m] for m in range(3)) for j in range(3)] for i in range(3)]
        bb = np.maximum(b[0][0] * b[1][1] - b[0][1] * b[0][1] + b[0][0] * b[2][2] - b[0][2] * b[0][2]
                        + b[1][1] * b[2][2] - b[1][2] * b[1][2], T(0.0))
        aa = 0
        for i in range(3):
            for j in range(3):
                aa = aa + g[i][j] * g[i][j]
        return T(c * delta2) * np.sqrt(bb / (aa + T(1e-30)) + T(_SQRT_EPS))
    raise ValueError(ops.turbulence)


def sgs_divergence3d(U, V, W, geom, ops):
    """div(2 nu_t S) on the faces, nu_t (with ghost ring) and its max (core.py:485-524)."""
    nz, ny, nx = ops.nz, ops.ny, ops.nx
    T = U.dtype.type
    inv = T(1.0 / ops.h)
    gr = velocity_gradient(U, V, W, ops.h)
    g = gr["g"]
    nut = eddy_viscosity3d(traceless(g), ops)
    if not geom.empty:
        k0, k1, j0, j1, i0, i1 = geom.window
        nut = nut.copy()
        nut[k0 + 1:k1 + 1, j0 + 1:j1 + 1, i0 + 1:i1 + 1] *= (T(1.0) - geom.chi_c)
    i = slice(1, -1)
    q = T(0.25)
    n_xy = nut[i]
    n_xy = (n_xy[:, :-1, :-1] + n_xy[:, 1:, :-1] + n_xy[:, :-1, 1:] + n_xy[:, 1:, 1:]) * q
    n_xz = nut[:, i]
    n_xz = (n_xz[:-1, :, :-1] + n_xz[1:, :, :-1] + n_xz[:-1, :, 1:] + n_xz[1:, :, 1:]) * q
    n_yz = nut[:, :, i]
    n_yz = (n_yz[:-1, :-1] + n_yz[1:, :-1] + n_yz[:-1, 1:] + n_yz[1:, 1:]) * q
    t12 = n_xy * gr["sxy"][1:nz + 1, 1:ny + 2, 1:nx + 2]
    t13 = n_xz * gr["sxz"][1:nz + 2, 1:ny + 1, 1:nx + 2]
    t23 = n_yz * gr["syz"][1:nz + 2, 1:ny + 2, 1:nx + 1]
    two = T(2.0)
    t11 = two * nut[i, i] * g[0][0][i, i]
    t22 = two * nut[i, :, i] * g[1][1][i, :, i]
    t33 = two * nut[:, i, i] * g[2][2][:, i, i]
    fu = (t11[..., 1:] - t11[..., :-1] + t12[:, 1:] - t12[:, :-1] + t13[1:] - t13[:-1]) * inv
    fv = (t12[..., 1:] - t12[..., :-1] + t22[:, 1:] - t22[:, :-1] + t23[1:] - t23[:-1]) * inv
    fw = (t13[..., 1:] - t13[..., :-1] + t23[:, 1:] - t23[:, :-1] + t33[1:] - t33[:-1]) * inv
    return fu, fv, fw, nut, nut.max()


def boundary_tendencies(u, lu, lv, lw, ops):
    """Inlet 0, convective outlet, walls 0 (core.py:527-543)."""
    px, py, pz = ops.periodic_axes
    T = u.dtype.type
    lu, lv, lw = lu.copy(), lv.copy(), lw.copy()
    if not px:
        out = (u[..., -2] - u[..., -1]) * T(1.0 / ops.h)
        if ops.closed:
            out = np.zeros_like(out)
        lu[..., 0] = 0.0
        lu[..., -1] = out
    if not py:
        lv[:, 0] = 0.0
        lv[:, -1] = 0.0
    if not pz:
        lw[0] = 0.0
        lw[-1] = 0.0
    return lu, lv, lw


def momentum_rhs3d(u, v, w, geom, ops, sources=None):
    """Explicit tendencies, nu_t field and max (core.py:546-570); ``sources`` (lu, lv, lw) ->
    (lu, lv, lw) adds the placed physics' forces before the boundary tendencies."""
    T = u.dtype.type
    U, V, W = pad_velocity(u, v, w, ops)
    au, av, aw = advection3(U, V, W, ops)
    nu_h2 = T(T(ops.nu_value) * T(1.0 / ops.h ** 2))
    lu = au + nu_h2 * laplacian_padded(U)
    lv = av + nu_h2 * laplacian_padded(V)
    lw = aw + nu_h2 * laplacian_padded(W)
    nut = nut_max = None
    if ops.turbulence != "none":
        fu, fv, fw, nut, nut_max = sgs_divergence3d(U, V, W, geom, ops)
        lu, lv, lw = lu + fu, lv + fv, lw + fw
    if getattr(ops, "forcing", None) is not None:   # the verification cases' uniform body force
        lu, lv, lw = lu + T(ops.forcing[0]), lv + T(ops.forcing[1]), lw + T(ops.forcing[2])
    if sources is not None:
        lu, lv, lw = sources(lu, lv, lw)
    lu, lv, lw = boundary_tendencies(u, lu, lv, lw, ops)
    return lu, lv, lw, nut, nut_max


# ---------------------------------------------------------------------------
# projection (core.py:577-612; poisson.py:74-157)
# ---------------------------------------------------------------------------

def divergence3d(u, v, w, h):
    return ((u[..., 1:] - u[..., :-1]) + (v[:, 1:] - v[:, :-1]) + (w[1:] - w[:-1])) * u.dtype.type(1.0 / h)


def neumann_basis(n):
    """Orthonormal DCT-II matrix and eigenvalues for h = 1 (poisson.py:74-81)."""
    k = np.arange(n, dtype=np.float64)[:, None]
    j = np.arange(n, dtype=np.float64)[None, :]
    q = np.cos(math.pi * k * (j + 0.5) / n) * math.sqrt(2.0 / n)
    q[0] *= math.sqrt(0.5)
    lam = 2.0 * np.cos(math.pi * np.arange(n, dtype=np.float64) / n) - 2.0
    return q, lam


def periodic_basis(n):
    """Orthonormal discrete Hartley matrix and periodic eigenvalues (poisson.py:84-90)."""
    k = np.arange(n, dtype=np.float64)
    ang = 2.0 * math.pi * k[:, None] * k[None, :] / n
    q = (np.cos(ang) + np.sin(ang)) / math.sqrt(n)
    lam = 2.0 * np.cos(2.0 * math.pi * k / n) - 2.0
    return q, lam


class PoissonSolver3D:
    """Exact ``L psi = f`` with zero mean (poisson.py:93-157)."""

    def __init__(self, nx, ny, nz, h, periodic, dtype):
        self.shape = (nz, ny, nx)
        mats, lams = [], []
        for n, per in zip((nx, ny, nz), periodic):
            q, lam = periodic_basis(n) if per else neumann_basis(n)
            mats.append(q.astype(dtype))
            lams.append(lam / (h * h))
        self.qx, self.qy, self.qz = mats
        lx, ly, lz = lams
        lam = lz[:, None, None] + ly[None, :, None] + lx[None, None, :]
        inv = np.where(lam != 0, 1.0 / np.where(lam != 0, lam, 1.0), 0.0)
        inv[0, 0, 0] = 0.0
        self.inv_lam = inv.astype(dtype)

    def solve(self, f):
        nz, ny, nx = f.shape
        a = (f.reshape(-1, nx) @ self.qx.T).reshape(nz, ny, nx)
        a = np.matmul(self.qy, a)
        a = (self.qz @ a.reshape(nz, -1)).reshape(nz, ny, nx)
        a = a * self.inv_lam
        a = (self.qz.T @ a.reshape(nz, -1)).reshape(nz, ny, nx)
        a = np.matmul(self.qy.T, a)
        return (a.reshape(-1, nx) @ self.qx).reshape(nz, ny, nx)

    def laplacian(self, psi, h, periodic):
        """The discrete operator itself (poisson.py:160-173)."""
        pe = psi
        for dim, per in zip((2, 1, 0), periodic):
            n = pe.shape[dim]
            if per:
                lo, hi = _narrow(pe, dim, n - 1, 1), _narrow(pe, dim, 0, 1)
            else:
                lo, hi = _narrow(pe, dim, 0, 1), _narrow(pe, dim, n - 1, 1)
            pe = np.concatenate([lo, pe, hi], axis=dim)
        c = pe[1:-1, 1:-1, 1:-1]
        ring = (pe[1:-1, 1:-1, 2:] + pe[1:-1, 1:-1, :-2] + pe[1:-1, 2:, 1:-1] + pe[1:-1, :-2, 1:-1]
                + pe[2:, 1:-1, 1:-1] + pe[:-2, 1:-1, 1:-1])
        return (ring - 6.0 * c) / (h * h)


def pressure_gradient(psi, ops):
    """grad psi on every face, zero on non-periodic boundary faces (core.py:582-601)."""
    T = psi.dtype.type
    inv = T(1.0 / ops.h)
    px, py, pz = ops.periodic_axes
    nz, ny, nx = psi.shape
    if px:
        gx = (psi - np.roll(psi, 1, axis=2)) * inv
        gx = np.concatenate([gx, gx[..., :1]], axis=2)
    else:
        gx = np.zeros((nz, ny, nx + 1), psi.dtype)
        gx[..., 1:-1] = (psi[..., 1:] - psi[..., :-1]) * inv
    if py:
        gy = (psi - np.roll(psi, 1, axis=1)) * inv
        gy = np.concatenate([gy, gy[:, :1]], axis=1)
    else:
        gy = np.zeros((nz, ny + 1, nx), psi.dtype)
        gy[:, 1:-1] = (psi[:, 1:] - psi[:, :-1]) * inv
    if pz:
        gz = (psi - np.roll(psi, 1, axis=0)) * inv
        gz = np.concatenate([gz, gz[:1]], axis=0)
    else:
        gz = np.zeros((nz + 1, ny, nx), psi.dtype)
        gz[1:-1] = (psi[1:] - psi[:-1]) * inv
    return gx, gy, gz


def project3d(u, v, w, ops, poisson):
    psi = poisson.solve(divergence3d(u, v, w, ops.h))
    gx, gy, gz = pressure_gradient(psi, ops)
    return u - gx, v - gy, w - gz, psi


# ---------------------------------------------------------------------------
# penalisation, dt, forces (core.py:615-678)
# ---------------------------------------------------------------------------

def penalise3d(u, v, w, geom, ops, bdt):
    """Implicit Brinkman on the window; returns fields and increments (core.py:615-634)."""
    T = u.dtype.type
    k0, k1, j0, j1, i0, i1 = geom.window
    k = T(bdt / T(ops.eta))
    u, v, w = u.copy(), v.copy(), w.copy()
    uw = u[k0:k1, j0:j1, i0:i1 + 1]
    vw = v[k0:k1, j0:j1 + 1, i0:i1]
    ww = w[k0:k1 + 1, j0:j1, i0:i1]
    un = (uw + k * geom.a_u) / (T(1.0) + k * geom.chi_u)
    vn = (vw + k * geom.a_v) / (T(1.0) + k * geom.chi_v)
    wn = (ww + k * geom.a_w) / (T(1.0) + k * geom.chi_w)
    du, dv, dw = un - uw, vn - vw, wn - ww
    u[k0:k1, j0:j1, i0:i1 + 1] = un
    v[k0:k1, j0:j1 + 1, i0:i1] = vn
    w[k0:k1 + 1, j0:j1, i0:i1] = wn
    return u, v, w, du, dv, dw


def speed_sum(u, v, w):
    return max(float(np.abs(u).max()) + float(np.abs(v).max()) + float(np.abs(w).max()), 1e-6)


def cfl_dt3d(u, v, w, ops, nut_max=None):
    """CFL and viscous limit (core.py:637-646)."""
    T = u.dtype.type
    umax = np.maximum(np.abs(u).max() + np.abs(v).max() + np.abs(w).max(), T(1e-6))
    dt = T(ops.cfl * ops.h) / umax
    nu = T(ops.nu_value) if nut_max is None else T(ops.nu_value) + nut_max
    return np.minimum(dt, T(VISCOUS_DT * ops.h * ops.h) / nu), umax


def force_coefficients(acc, geom, ops, dt):
    """[CD, CS, CL, C_roll, Cm, Cn] per body (core.py:653-678); sums in float64."""
    acc_u, acc_v, acc_w = (a.astype(np.float64) for a in acc)
    scale = -(ops.h ** 3) / float(dt)
    ru = np.einsum("bkzyx,zyx->bk", geom.k_u.astype(np.float64), acc_u) * scale
    rv = np.einsum("bkzyx,zyx->bk", geom.k_v.astype(np.float64), acc_v) * scale
    rw = np.einsum("bkzyx,zyx->bk", geom.k_w.astype(np.float64), acc_w) * scale
    fx, fy, fz = ru[:, 0], rv[:, 0], rw[:, 0]
    mx, my, mz = rv[:, 1] + rw[:, 1], ru[:, 1] + rw[:, 2], ru[:, 2] + rv[:, 2]
    if ops.symmetry:
        dy = ops.moment_ref[1] - ops.y0
        fx, fz, my = 2.0 * fx, 2.0 * fz, 2.0 * my
        fy = np.zeros_like(fy)
        mx = -dy * fz
        mz = dy * fx
    q_a = 0.5 * ops.ref_area
    return np.stack([fx / q_a, fy / q_a, fz / q_a, mx / (q_a * ops.span_ref), my / (q_a * ops.length_ref),
                     mz / (q_a * ops.span_ref)], axis=1)


# ---------------------------------------------------------------------------
# heat equation (physics.py:494-790)
# ---------------------------------------------------------------------------

def _theta_ghosts(th, c, dim, side):
    """Ghost layers of one domain side (physics.py:589-607)."""
    n = c.shape[dim]
    lo = side % 2 == 0
    kind = th.side_kinds[side]
    T = c.dtype.type
    if kind == "periodic":
        return _narrow(c, dim, n - 2, 2) if lo else _narrow(c, dim, 0, 2)
    if kind == "outflow":
        e = _narrow(c, dim, 0 if lo else n - 1, 1)
        return np.concatenate([e, e], axis=dim)
    mirror = np.flip(_narrow(c, dim, 0, 2), dim) if lo else np.flip(_narrow(c, dim, n - 2, 2), dim)
    if kind == "adiabatic":
        return mirror
    val = T(th.side_vals[side])
    if kind == "inflow":
        return np.zeros_like(mirror) + val
    if kind == "temperature":
        return T(2.0) * val - mirror
    wts = np.array([3.0, 1.0] if lo else [1.0, 3.0]) * th.h
    shape = [1, 1, 1]
    shape[dim] = 2
    return mirror + val * wts.astype(c.dtype).reshape(shape)          # heat flux (physics.py:541-548)


def theta_pad(th, c):
    """Two ghost layers on the six faces (physics.py:609-621)."""
    nz, ny, nx = c.shape
    P = np.zeros((nz + 4, ny + 4, nx + 4), dtype=c.dtype)
    m = slice(2, -2)
    P[m, m, m] = c
    P[m, m, 0:2] = _theta_ghosts(th, c, 2, 0)
    P[m, m, nx + 2:] = _theta_ghosts(th, c, 2, 1)
    P[m, 0:2, m] = _theta_ghosts(th, c, 1, 2)
    P[m, ny + 2:, m] = _theta_ghosts(th, c, 1, 3)
    P[0:2, m, m] = _theta_ghosts(th, c, 0, 4)
    P[nz + 2:, m, m] = _theta_ghosts(th, c, 0, 5)
    return P


def _van_leer(p, q):
    """dye.py:266-270."""
    T = p.dtype.type
    pq = p * q
    pos = pq > 0
    return np.where(pos, T(2.0) * pq / np.where(pos, p + q, T(1.0)), T(0.0))


def muscl_flux(a, b, c, d, vel):
    """Upwind MUSCL / van Leer face flux (dye.py:273-277)."""
    T = b.dtype.type
    up = b + T(0.5) * _van_leer(b - a, c - b)
    dn = c - T(0.5) * _van_leer(c - b, d - c)
    return vel * np.where(vel > 0, up, dn)


def face_kappa(th, nut, ops, dtype):
    """kappa / h on the faces, with nu_t / Pr_t when LES is on (physics.py:624-645)."""
    T = dtype.type
    kh = T(th.kappa / ops.h)
    if nut is None:
        return kh, kh, kh
    c = T(0.5 / (th.prt * ops.h))
    m = slice(1, -1)
    kx = kh + c * (nut[m, m, :-1] + nut[m, m, 1:])
    ky = kh + c * (nut[m, :-1, m] + nut[m, 1:, m])
    kz = kh + c * (nut[:-1, m, m] + nut[1:, m, m])
    px, py, pz = ops.periodic_axes
    if not px:
        kx[..., 0] = kh
        kx[..., -1] = kh
    if not py:
        ky[:, 0] = kh
        ky[:, -1] = kh
    if not pz:
        kz[0] = kh
        kz[-1] = kh
    return kx, ky, kz


def _face_slices(win, g):
    k0, k1, j0, j1, i0, i1 = win
    return (slice(k0, k1 + (1 if g == "w" else 0)), slice(j0, j1 + (1 if g == "v" else 0)),
            slice(i0, i1 + (1 if g == "u" else 0)))


def theta_fluxes(th, c, u, v, w, ops, nut):
    """Advective minus diffusive theta fluxes on every face (physics.py:647-676)."""
    nz, ny, nx = c.shape
    P = theta_pad(th, c)
    m = slice(2, -2)
    kx, ky, kz = face_kappa(th, nut, ops, c.dtype)
    sx = (P[m, m, 0:nx + 1], P[m, m, 1:nx + 2], P[m, m, 2:nx + 3], P[m, m, 3:nx + 4])
    sy = (P[m, 0:ny + 1, m], P[m, 1:ny + 2, m], P[m, 2:ny + 3, m], P[m, 3:ny + 4, m])
    sz = (P[0:nz + 1, m, m], P[1:nz + 2, m, m], P[2:nz + 3, m, m], P[3:nz + 4, m, m])
    out = []
    for st, vel, kf in ((sx, u, kx), (sy, v, ky), (sz, w, kz)):
        out.append(muscl_flux(*st, vel) - kf * (st[2] - st[1]))
    g = th.geom
    if g.adia is not None:
        k0, k1, j0, j1, i0, i1 = g.window
        K, J, I = slice(k0 + 2, k1 + 2), slice(j0 + 2, j1 + 2), slice(i0 + 2, i1 + 2)
        cu, cv, cw = g.adia
        dx = P[K, J, i0 + 2:i1 + 3] - P[K, J, i0 + 1:i1 + 2]
        dy = P[K, j0 + 2:j1 + 3, I] - P[K, j0 + 1:j1 + 2, I]
        dz = P[k0 + 2:k1 + 3, J, I] - P[k0 + 1:k1 + 2, J, I]
        for f, kf, d, chi, gg in ((out[0], kx, dx, cu, "u"), (out[1], ky, dy, cv, "v"), (out[2], kz, dz, cw, "w")):
            sl = _face_slices(g.window, gg)
            kw = kf if np.ndim(kf) == 0 else kf[sl]
            f[sl] += kw * chi * d
    return out


def theta_stage(th, c_prev, c0, up, vp, wp, a, bdt, wgt, ops, nut, heat_acc, ports=None):
    """One RK stage of theta with the ports' sources and the body penalisation
    (physics.py:678-708)."""
    T = c_prev.dtype.type
    fx, fy, fz = theta_fluxes(th, c_prev, up, vp, wp, ops, nut)
    D = ((fx[..., 1:] - fx[..., :-1]) + (fy[:, 1:] - fy[:, :-1]) + (fz[1:] - fz[:-1])) * T(1.0 / ops.h)
    base = c_prev if a == 0.0 else lerp(c_prev, c0, a)
    ch = base - bdt * D
    bk = T(bdt * T(th.kappa))
    for win, q in getattr(th, "sources", ()) or ():   # volumetric heaters (physics.py:693-694)
        ch[_face_slices(win, "c")] += bk * q
    g = th.geom
    if g.skin is not None:
        ch[_face_slices(g.window, "c")] += bk * g.skin
    if ports is not None:
        ch = port_scalar_sources(ports, ch, c_prev, bdt)
    if g.chi_t is not None:
        sl = _face_slices(g.window, "c")
        win = ch[sl]
        k = T(bdt / T(th.eta))
        new = (win + k * g.a_t) / (T(1.0) + k * g.chi_t)
        inc = (new - win) * T(wgt)
        ch[sl] = new
        contrib = np.einsum("bzyx,zyx->b", g.w_t.astype(np.float64), inc.astype(np.float64))
        for n, b in enumerate(g.t_index):
            heat_acc[b] += contrib[n]
    return ch


def add_buoyancy(th, wh, theta, bdt, wgt, geom, ops):
    """Buoyancy after the penalisation and the solids' share (physics.py:744-790)."""
    T = wh.dtype.type
    if th.ri == 0.0 or theta is None:
        return wh, None
    wh = wh.copy()
    tf = T(0.5) * (theta[1:] + theta[:-1])
    wh[1:-1] = wh[1:-1] + tf * T(bdt * T(th.ri))
    if ops.periodic_axes[2]:
        edge = (theta[:1] + theta[-1:]) * T(0.5 * th.ri) * bdt
        wh[:1] = wh[:1] + edge
        wh[-1:] = wh[-1:] + edge
    if geom.empty:
        return wh, None
    k0, k1, j0, j1, i0, i1 = geom.window
    lo, hi = max(k0 - 1, 0), min(k1, ops.nz - 1)
    tc = theta[lo:hi + 1, j0:j1, i0:i1]
    pz = ops.periodic_axes[2]
    if k0 == 0:
        tc = np.concatenate([theta[-1:, j0:j1, i0:i1] if pz else tc[:1], tc], axis=0)
    if k1 == ops.nz:
        tc = np.concatenate([tc, theta[:1, j0:j1, i0:i1] if pz else tc[-1:]], axis=0)
    tw = T(0.5) * (tc[1:] + tc[:-1])
    vol = th.geom.vol_w if th.geom.vol_w is not None else geom.chi_w
    share = (tw * vol) * T(bdt * T(th.ri * wgt))
    return wh, share


def thermal_dt_limit(th, nut_max, ops, umax):
    """Combined advection-diffusion bound (physics.py:723-742)."""
    T = umax.dtype.type
    kap = T(th.kappa) if nut_max is None else T(th.kappa) + nut_max / T(th.prt)
    diff_rate = kap / T(VISCOUS_DT * ops.h * ops.h)
    return T(1.0) / (umax * T(1.0 / (THETA_COURANT_MAX * ops.h)) + diff_rate)


PID_GAINS = (0.3, 0.4, 0.05)                                      # ns3d/physics.py:79 (kI, kP, kD)
PID_LIMITS = (0.5, 1.2)                                           # ns3d/physics.py:81


class PidState:
    """The PID controller's state (physics.py:1144-1181): 0-d arrays dt_prev, e1, e2
    (dt_prev <= 0: no step yet) and the target fraction of the limit."""

    def __init__(self, target, dtype):
        self.target = float(target)
        self.dt_prev, self.e1, self.e2 = (np.zeros((), dtype) for _ in range(3))


def pid_dt(pid, dt_cap):
    """PidDt.__call__ (physics.py:1161-1173): updates the state, returns dt."""
    T = np.asarray(dt_cap).dtype.type
    ki, kp, kd = PID_GAINS
    want = T(dt_cap * T(pid.target))
    first = pid.dt_prev <= 0
    prev = want if first else T(pid.dt_prev)
    with np.errstate(all="ignore"):
        e = T(np.log(T(want / prev)))
        fac = T(np.exp(T(T(T(T(ki) * e) + T(T(kp) * T(e - pid.e1))) + T(T(kd) * T(T(e - T(2.0) * pid.e1) + pid.e2)))))
    fac = T(min(max(fac, T(PID_LIMITS[0])), T(PID_LIMITS[1])))
    dt = T(np.minimum(want if first else T(prev * fac), dt_cap))
    pid.e2 = np.asarray(pid.e1).copy()
    pid.e1 = np.asarray(T(0.0) if first else e)
    pid.dt_prev = np.asarray(dt)
    return dt


class FanState:
    """FanSet (physics.py:831-979) in numpy.  ``items[q]``: ``win`` and the weight triples
    ``f`` (force), ``s`` (swirl), ``m`` (disc average) on the window's u, v, w faces;
    per-fan constants (nfan,) and the state ``thrust, ud, e_prev, swirl_amp`` (nfan,)."""

    def __init__(self, items, target, kp, ki, tmax, velocity_mode, swirl, any_swirl, thrust, dtype):
        T = np.dtype(dtype).type
        self.items = items
        self.target, self.kp, self.ki, self.tmax, self.swirl = (np.asarray(x, dtype) for x in
                                                                 (target, kp, ki, tmax, swirl))
        self.velocity_mode = np.asarray(velocity_mode, bool)
        self.any_swirl = bool(any_swirl)
        self.thrust = np.asarray(thrust, dtype).copy()
        self.ud, self.e_prev, self.swirl_amp = (np.zeros(len(items), dtype) for _ in range(3))
        self.T = T


def fan_begin_step(fans, u0, v0, w0, dt):
    """FanSet.measure + begin_step (physics.py:922-942)."""
    T = fans.T
    ud = np.array([T(T(T(np.sum(it["m"][0] * u0[_face_slices(it["win"], "u")])) +
                       T(np.sum(it["m"][1] * v0[_face_slices(it["win"], "v")]))) +
                     T(np.sum(it["m"][2] * w0[_face_slices(it["win"], "w")]))) for it in fans.items], fans.thrust.dtype)
    fans.ud = ud
    e = fans.target - ud
    new = (fans.thrust + fans.kp * (e - fans.e_prev)) + (fans.ki * T(dt)) * e
    new = np.maximum(np.minimum(new, fans.tmax), -fans.tmax)
    fans.thrust = np.where(fans.velocity_mode, new, fans.thrust)
    fans.e_prev = np.where(fans.velocity_mode, e, fans.e_prev)
    if fans.any_swirl:
        fans.swirl_amp = (fans.swirl * ud) * np.abs(ud)


class PortState:
    """PortSet (physics.py:981-1072) in numpy: ``items[q]`` with ``win``, ``kind`` ("jet" /
    "vent"), ``m`` (cells), ``f`` (the u, v, w face weights) and ``theta``; the net mass flux
    in outlet-face units and the uniform leak of an unbalanced closed box."""

    def __init__(self, items, mass_flux, leak):
        self.items, self.mass_flux, self.leak = items, mass_flux, float(leak)


def port_forces(ports, lu, lv, lw, u, v, w):
    """PortSet.add_forces (physics.py:1033-1041): + f (jet) or + f u (vent)."""
    out = [lu.copy(), lv.copy(), lw.copy()]
    for it in ports.items:
        for c, (g, vel) in enumerate(zip("uvw", (u, v, w))):
            sl = _face_slices(it["win"], g)
            out[c][sl] = out[c][sl] + (it["f"][c] if it["kind"] == "jet" else it["f"][c] * vel[sl])
    return tuple(out)


def port_continuity(ports, div):
    """PortSet.continuity (physics.py:1043-1047): div - m on each port's cells."""
    div = div.copy()
    for it in ports.items:
        sl = _face_slices(it["win"], "c")
        div[sl] = div[sl] - it["m"]
    return div


def port_scalar_sources(ports, ch, c_prev, bdt):
    """PortSet.scalar_sources for theta (physics.py:1049-1072)."""
    T = ch.dtype.type
    ch = ch.copy()
    for it in ports.items:
        sl = _face_slices(it["win"], "c")
        if it["kind"] == "vent":
            ch[sl] = ch[sl] + (bdt * it["m"]) * c_prev[sl]
            continue
        val = float(it.get("theta", 0.0) or 0.0)
        if val != 0.0:
            ch[sl] = ch[sl] + T(bdt * T(val)) * it["m"]
    if ports.leak:
        ch = ch - c_prev * T(bdt * T(ports.leak))
    return ch


def fan_forces(fans, lu, lv, lw):
    """FanSet.add_forces (physics.py:944-952): + f T (+ s amp) on each fan's faces."""
    out = [lu.copy(), lv.copy(), lw.copy()]
    for q, it in enumerate(fans.items):
        for c, g in enumerate("uvw"):
            sl = _face_slices(it["win"], g)
            out[c][sl] = out[c][sl] + it["f"][c] * fans.thrust[q]
            if fans.any_swirl:
                out[c][sl] = out[c][sl] + it["s"][c] * fans.swirl_amp[q]
    return tuple(out)


def dt_rule(u0, v0, w0, ops, nut_max, th, theta, u_floor=0.0, pid=None):
    """Physics3D.dt_rule without fans and ports (physics.py:1230-1262); ``u_floor`` is the
    sources' speed scale, ``pid`` a :class:`PidState` (or None)."""
    T = u0.dtype.type
    dt, umax = cfl_dt3d(u0, v0, w0, ops, nut_max)
    if u_floor > 0.0:
        dt = np.minimum(dt, T(ops.cfl * ops.h / u_floor))
        umax = np.maximum(umax, T(u_floor))
    if th is not None:
        dt = np.minimum(dt, thermal_dt_limit(th, nut_max, ops, umax))
        if th.ri != 0.0 and theta is not None:
            acc = np.maximum(T(abs(th.ri)) * np.abs(theta).max(), T(1e-12))
            dt = np.minimum(dt, T(ops.cfl) * np.sqrt(T(ops.h) / acc))
        if getattr(th, "heat_max", None) is not None:
            s_max = max(T(th.heat_max), T(1e-12))
            dt = np.minimum(dt, T(1.0) / s_max)
            if th.ri != 0.0:
                dt = np.minimum(dt, (T(6.0 * ops.cfl * ops.h) / (T(abs(th.ri)) * s_max)) ** T(1.0 / 3.0))
    if pid is not None:
        dt = pid_dt(pid, T(dt))
    return T(dt)


# ---------------------------------------------------------------------------
# the step (core.py:765-883)
# ---------------------------------------------------------------------------

class StepResult:
    """What one step returns: new u, v, w, p, t, dt, per-body coefficients (nb, 6),
    theta (or None), heat rates (nb) (or None), the per-stage traces, and div_pre, the sum of
    squares of the last stage's projection right-hand side (the diagnostics row's input)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)


def step3d_phys(u0, v0, w0, t, geom, ops, poisson, *, th=None, theta=None, dt=None, trace=False, paint=None,
                pid=None, u_floor=0.0, fans=None, ports=None):
    """One SSP-RK3 step (core.py:765-883) with heat transfer, buoyancy, painted solids
    (``paint``: (chi_u, chi_v, chi_w) on the whole grid), the PID / speed-floor dt rule and
    fans (a :class:`FanState`, updated in place) and jets / vents (a :class:`PortState`)."""
    T = u0.dtype.type
    up, vp, wp = u0, v0, w0
    acc = None
    psi_w = None
    thermal = th is not None and theta is not None
    t0 = tp = theta
    heat_acc = np.zeros(geom.nbody if not geom.empty else max(geom.nbody, 0), dtype=np.float64)
    stages = []
    nut_stage1 = None
    placed = th is not None or pid is not None or u_floor > 0.0 or fans is not None or ports is not None

    def sources(lu_, lv_, lw_):  # Physics3D.momentum_sources: fans, then jets and vents
        if fans is not None:
            lu_, lv_, lw_ = fan_forces(fans, lu_, lv_, lw_)
        if ports is not None:
            lu_, lv_, lw_ = port_forces(ports, lu_, lv_, lw_, up, vp, wp)
        return lu_, lv_, lw_
    for s, ((a, b), wgt) in enumerate(zip(SSP_RK3, FORCE_WEIGHTS)):
        if s == 0:
            # the dt rule and the fans' controllers act before any source is evaluated
            lu, lv, lw, nut, nut_max = momentum_rhs3d(up, vp, wp, geom, ops)
            nut_stage1 = nut
            if dt is None:
                if ops.dt_fixed is not None:
                    dt = T(ops.dt_fixed)
                elif placed:
                    dt = dt_rule(u0, v0, w0, ops, nut_max, th, t0, u_floor, pid)
                else:
                    dt = cfl_dt3d(u0, v0, w0, ops, nut_max)[0]
            dt = T(dt)
            if fans is not None:
                fan_begin_step(fans, u0, v0, w0, dt)
        if s > 0 or fans is not None or ports is not None:
            lu, lv, lw, nut, nut_max = momentum_rhs3d(
                up, vp, wp, geom, ops, sources=None if fans is None and ports is None else sources)
        bdt = T(dt * T(b))
        if a == 0.0:
            uh, vh, wh = up + lu * bdt, vp + lv * bdt, wp + lw * bdt
        else:
            uh = lerp(up, u0, a) + lu * bdt
            vh = lerp(vp, v0, a) + lv * bdt
            wh = lerp(wp, w0, a) + lw * bdt
        if not ops.periodic_axes[0]:
            uh = inlet_outlet(uh, ops, None if ports is None else ports.mass_flux)
        if not geom.empty:
            uh, vh, wh, du, dv, dw = penalise3d(uh, vh, wh, geom, ops, bdt)
            wg = T(wgt)
            acc = [du * wg, dv * wg, dw * wg] if acc is None else [acc[0] + du * wg, acc[1] + dv * wg,
                                                                    acc[2] + dw * wg]
            if any(ops.periodic_axes):
                uh, vh, wh = sync_periodic(uh, vh, wh, ops)
        if paint is not None:  # PaintLayer.penalise (physics.py:1132-1137), after the bodies
            k = T(bdt / T(ops.eta))
            uh, vh, wh = (x / (T(1.0) + k * chi) for x, chi in zip((uh, vh, wh), paint))
            if any(ops.periodic_axes):
                uh, vh, wh = sync_periodic(uh, vh, wh, ops)
        if thermal and th.ri != 0.0:
            wh, share = add_buoyancy(th, wh, tp, bdt, wgt, geom, ops)
            if share is not None:
                acc[2] = acc[2] + share
        if thermal:
            tp_new = theta_stage(th, tp, t0, up, vp, wp, a, bdt, wgt, ops,
                                 nut if ops.turbulence != "none" else None, heat_acc, ports)
        div = divergence3d(uh, vh, wh, ops.h)
        if ports is not None:
            div = port_continuity(ports, div)
        if s == 2:   # Physics3D.record_divergence (physics.py:1303-1305), fused.py:480-482
            div_pre = float(np.sum(np.asarray(div, np.float64) ** 2))
        psi = poisson.solve(div)
        gx, gy, gz = pressure_gradient(psi, ops)
        if trace:
            stages.append({"lu": lu, "lv": lv, "lw": lw, "uh": uh, "vh": vh, "wh": wh, "div": div, "psi": psi})
        up, vp, wp = uh - gx, vh - gy, wh - gz
        if thermal:
            tp = tp_new
        psi_w = psi * T(wgt) if psi_w is None else psi_w + T(wgt) * psi
    p = psi_w * T(T(1.0) / dt)
    if geom.empty:
        coeffs = np.zeros((geom.nbody, 6))
    else:
        coeffs = force_coefficients(acc, geom, ops, dt)
    heat_rate = None
    if thermal:
        scale = (2.0 if ops.symmetry else 1.0) * ops.h ** 3 * th.pe
        heat_rate = heat_acc * (scale / float(dt))
        if getattr(th.geom, "flux_rate", None) is not None:
            heat_rate = heat_rate + np.asarray(th.geom.flux_rate, np.float64) * (2.0 if ops.symmetry else 1.0)
    return StepResult(u=up, v=vp, w=wp, p=p, t=T(t + dt), dt=dt, coeffs=coeffs, theta=tp if thermal else None,
                      heat_rate=heat_rate, stages=stages, nut_stage1=nut_stage1, div_pre=div_pre)


# ---------------------------------------------------------------------------
# smoke (dye.py:232-312)
# ---------------------------------------------------------------------------

def pad_dye(c, ops):
    """dye.py:232-263 (edges and corners left at zero: never read)."""
    nz, ny, nx = c.shape
    P = np.zeros((nz + 4, ny + 4, nx + 4), dtype=c.dtype)
    P[2:-2, 2:-2, 2:-2] = c
    px, py, pz = ops.periodic_axes
    m = slice(2, -2)
    if px:
        P[m, m, 0:2] = c[..., nx - 2:]
        P[m, m, nx + 2:] = c[..., :2]
    else:
        P[m, m, 0:2] = 0.0
        P[m, m, nx + 2:] = c[..., nx - 1:]
    if py:
        P[m, 0:2, m] = c[:, ny - 2:]
        P[m, ny + 2:, m] = c[:, :2]
    else:
        P[m, 0:2, m] = np.flip(c[:, :2], 1)
        P[m, ny + 2:, m] = np.flip(c[:, ny - 2:], 1)
    if pz:
        P[0:2, m, m] = c[nz - 2:]
        P[nz + 2:, m, m] = c[:2]
    else:
        P[0:2, m, m] = np.flip(c[:2], 0)
        P[nz + 2:, m, m] = np.flip(c[nz - 2:], 0)
    return P


def advect_dye3d(c, u, v, w, dt, ops):
    """Forward Euler MUSCL step, clipped and floored (dye.py:280-298)."""
    T = c.dtype.type
    nz, ny, nx = c.shape
    P = pad_dye(c, ops)
    m = slice(2, -2)
    fx = muscl_flux(P[m, m, 0:nx + 1], P[m, m, 1:nx + 2], P[m, m, 2:nx + 3], P[m, m, 3:nx + 4], u)
    fy = muscl_flux(P[m, 0:ny + 1, m], P[m, 1:ny + 2, m], P[m, 2:ny + 3, m], P[m, 3:ny + 4, m], v)
    fz = muscl_flux(P[0:nz + 1, m, m], P[1:nz + 2, m, m], P[2:nz + 3, m, m], P[3:nz + 4, m, m], w)
    k = T(dt * T(1.0 / ops.h))
    r = c - k * ((fx[..., 1:] - fx[..., :-1]) + (fy[:, 1:] - fy[:, :-1]) + (fz[1:] - fz[:-1]))
    r = np.minimum(r, T(1.0))
    return np.where(r < T(DYE_FLOOR), T(0.0), r)


def apply_solids_and_sources(c, t, geom, src):
    """Solid cells cleared, nozzles relaxed to 1 (dye.py:301-312)."""
    T = c.dtype.type
    c = c.copy()
    if geom is not None and not geom.empty:
        k0, k1, j0, j1, i0, i1 = geom.window
        win = c[k0:k1, j0:j1, i0:i1]
        win[geom.chi_c > 0.5] = 0.0
    if src is not None and not src.empty:
        k0, k1, j0, j1, i0, i1 = src.window
        win = c[k0:k1, j0:j1, i0:i1]
        on = T(1.0) if float(np.remainder(T(t), T(src.pulse[1]))) < float(T(src.pulse[0])) else T(0.0)
        win += src.weight * on * (T(1.0) - win)
    return c
