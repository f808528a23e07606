"""CPU oracle for the 3D field outputs -- TEST INFRASTRUCTURE ONLY.

Restates, in numpy, the reference's derived fields and point sampling
(src/aerolume/solvers/ns3d/fields.py and the cell-centring of solver.py:1374-1416):

* ``centre_u`` / ``centre_v`` / ``centre_w`` / ``speed``  fields.py:24-34, solver.py:1382-1384
* ``gradient_field``  fields.py:45-75  vorticity |curl u|, Q = -g_ij g_ji / 2, eddy viscosity
* ``trilinear``       fields.py:78-102 interpolation of a staggered field at points

Pinned by ``tests/test_fields3d.py`` against ``tests/golden/fields3d.npz``, which
``tests/golden/make_golden_fields.py`` produced with the reference itself.
"""
from __future__ import annotations

import numpy as np

from .ns3d import eddy_viscosity3d, pad_velocity, traceless, velocity_gradient


def centre_u(u):
    return u.dtype.type(0.5) * (u[..., 1:] + u[..., :-1])


def centre_v(v):
    return v.dtype.type(0.5) * (v[:, 1:] + v[:, :-1])


def centre_w(w):
    return w.dtype.type(0.5) * (w[1:] + w[:-1])


def speed(u, v, w):
    uc, vc, wc = centre_u(u), centre_v(v), centre_w(w)
    return np.sqrt(uc * uc + vc * vc + wc * wc)


def gradient_field(name, u, v, w, ops, mask=None):
    """"vorticity", "q" or "nut" on every cell; ``mask`` is the cell-centred solid fraction."""
    T = u.dtype.type
    U, V, W = pad_velocity(u, v, w, ops)
    g = velocity_gradient(U, V, W, ops.h)["g"]
    g = [[g[i][j][1:-1, 1:-1, 1:-1] for j in range(3)] for i in range(3)]
    if name == "q":
        return T(-0.5) * sum(g[i][j] * g[j][i] for i in range(3) for j in range(3))
    if name == "vorticity":
        ox, oy, oz = g[2][1] - g[1][2], g[0][2] - g[2][0], g[1][0] - g[0][1]
        return np.sqrt(ox * ox + oy * oy + oz * oz)
    if ops.turbulence == "none":
        return np.zeros_like(g[0][0])
    f = eddy_viscosity3d(traceless(g), ops)
    if mask is not None:
        f = f * (T(1.0) - mask)
    return f


def trilinear(field, pts, origin, h, off=(0.5, 0.5, 0.5)):
    """Field value at points (P, 3) = (x, y, z); field[k, j, i] sits at
    origin + ((i, j, k) + off) h; points outside are clamped to the edge."""
    T = field.dtype.type
    nz, ny, nx = field.shape
    pts = np.asarray(pts, dtype=field.dtype)
    idx = []
    for c, n in ((0, nx), (1, ny), (2, nz)):
        f = np.clip((pts[:, c] - T(origin[c])) / T(h) - T(off[c]), T(0.0), T(max(n - 1.0, 0.0)))
        i0 = np.minimum(np.floor(f), max(n - 2, 0)).astype(np.int64)
        idx.append((i0, (f - i0).astype(field.dtype), min(1, n - 1)))
    (i0, tx, sx), (j0, ty, sy), (k0, tz, sz) = idx
    one = T(1.0)

    def at(dk, dj, di):
        return field[k0 + dk * sz, j0 + dj * sy, i0 + di * sx]
    c00 = at(0, 0, 0) * (one - tx) + at(0, 0, 1) * tx
    c01 = at(0, 1, 0) * (one - tx) + at(0, 1, 1) * tx
    c10 = at(1, 0, 0) * (one - tx) + at(1, 0, 1) * tx
    c11 = at(1, 1, 0) * (one - tx) + at(1, 1, 1) * tx
    return (c00 * (one - ty) + c01 * ty) * (one - tz) + (c10 * (one - ty) + c11 * ty) * tz
