"""CPU restatement of the reference's 3D mask construction with its exact signed distance.

TEST INFRASTRUCTURE ONLY: tests, the smoke check and the bench's CPU leg use this module as
the checker; nothing in the product path imports it.

Follows src/aerolume/solvers/ns3d/geometry.py:
  _tri_d2                geometry.py:68-109   squared point-triangle distance
  _solid_angle           geometry.py:112-123  van Oosterom & Strackee signed solid angle
  mesh_signed_distance   geometry.py:126-196  nearest triangle, winding-number sign, the face
                                              plane distance near a face (plane_zone)
  grid_signed_distance   geometry.py:229-262  at the centres of a staggered grid (the private
                                              path: use_shared=False)
  smooth_step            geometry.py:265-268
  body_window3d          geometry.py:323-356
  build_geometry3d       geometry.py:385-495  masks, solid velocity, force / moment weights
numpy in the working dtype, brute force over all point-triangle pairs: small cases only.
Pinned by tests/golden/masks3d.npz (the reference's own build_geometry3d with
use_shared=False, and its signed distance at the known-answer points of
tests/test_ns3d_core.py:264-273).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def _tri_d2(px, py, pz, a, b, c):
    """Squared point-triangle distance on broadcasting coordinate arrays (geometry.py:68-109);
    a, b, c are (x, y, z) tuples."""
    T = np.asarray(px).dtype.type
    tiny = T(np.finfo(np.asarray(px).dtype).tiny)
    ax, ay, az = a
    bx, by, bz = b
    cx, cy, cz = c
    e0 = (bx - ax, by - ay, bz - az)
    e1 = (cx - bx, cy - by, cz - bz)
    e2 = (ax - cx, ay - cy, az - cz)
    nx = e0[1] * (-e2[2]) - e0[2] * (-e2[1])
    ny = e0[2] * (-e2[0]) - e0[0] * (-e2[2])
    nz = e0[0] * (-e2[1]) - e0[1] * (-e2[0])
    nn = nx * nx + ny * ny + nz * nz
    w0 = (px - ax, py - ay, pz - az)
    w1 = (px - bx, py - by, pz - bz)
    w2 = (px - cx, py - cy, pz - cz)

    def side(e, w):
        cxp = e[1] * w[2] - e[2] * w[1]
        cyp = e[2] * w[0] - e[0] * w[2]
        czp = e[0] * w[1] - e[1] * w[0]
        return nx * cxp + ny * cyp + nz * czp

    inside = (side(e0, w0) >= 0) & (side(e1, w1) >= 0) & (side(e2, w2) >= 0) & (nn > tiny)
    pd = nx * w0[0] + ny * w0[1] + nz * w0[2]
    plane = pd * pd / np.maximum(nn, tiny)

    def seg(e, w):
        ee = np.maximum(e[0] * e[0] + e[1] * e[1] + e[2] * e[2], tiny)
        t = np.clip((w[0] * e[0] + w[1] * e[1] + w[2] * e[2]) / ee, T(0.0), T(1.0))
        dx, dy, dz = w[0] - t * e[0], w[1] - t * e[1], w[2] - t * e[2]
        return dx * dx + dy * dy + dz * dz

    edge = np.minimum(np.minimum(seg(e0, w0), seg(e1, w1)), seg(e2, w2))
    return np.where(inside, plane, edge)


def tri_d2(p, a, b, c):
    """Squared distance of points p (P, 3) to triangles a, b, c (T, 3): (P, T)."""
    return _tri_d2(p[:, 0:1], p[:, 1:2], p[:, 2:3], *(tuple(x[None, :, k] for k in range(3)) for x in (a, b, c)))


def tri_d2_rows(p, a, b, c):
    """Squared distance of each point p[k] to its own triangle a[k], b[k], c[k]: (P,)."""
    return _tri_d2(p[:, 0], p[:, 1], p[:, 2], *(tuple(x[:, k] for k in range(3)) for x in (a, b, c)))


def solid_angle(p, a, b, c):
    """Signed solid angle (P, T) of the triangles seen from the points."""
    T = p.dtype.type
    px, py, pz = (p[:, k:k + 1] for k in range(3))
    ax, ay, az = a[None, :, 0] - px, a[None, :, 1] - py, a[None, :, 2] - pz
    bx, by, bz = b[None, :, 0] - px, b[None, :, 1] - py, b[None, :, 2] - pz
    cx, cy, cz = c[None, :, 0] - px, c[None, :, 1] - py, c[None, :, 2] - pz
    la = np.sqrt(ax * ax + ay * ay + az * az)
    lb = np.sqrt(bx * bx + by * by + bz * bz)
    lc = np.sqrt(cx * cx + cy * cy + cz * cz)
    det = ax * (by * cz - bz * cy) + ay * (bz * cx - bx * cz) + az * (bx * cy - by * cx)
    den = la * lb * lc + (ax * bx + ay * by + az * bz) * lc + (bx * cx + by * cy + bz * cz) * la \
        + (cx * ax + cy * ay + cz * az) * lb
    return T(2.0) * np.arctan2(det, den)


def mesh_signed_distance(vertices, faces, points, plane_zone=0.0, chunk=4096):
    """Exact signed distance (negative inside) of points to a triangle soup."""
    p = np.asarray(points)
    dt = p.dtype
    T = dt.type
    v = np.asarray(vertices, dtype=dt)
    f = np.asarray(faces, dtype=np.int64)
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    npt, nt = p.shape[0], f.shape[0]
    best = np.zeros(npt, dtype=np.int64)
    gwn = np.zeros(npt, dtype=dt)
    for s in range(0, npt, chunk):
        q = p[s:s + chunk]
        d2 = tri_d2(q, a, b, c)
        best[s:s + chunk] = d2.argmin(axis=1)                    # first index of the minimum
        gwn[s:s + chunk] = solid_angle(q, a, b, c).sum(axis=1)
    inside = np.abs(gwn) > T(2.0 * math.pi)
    A, B, C = a[best], b[best], c[best]
    d2 = tri_d2_rows(p, A, B, C)
    d = np.sqrt(np.maximum(d2, T(1e-24)))
    sig = np.where(inside, T(-1.0), T(1.0))
    e0 = B - A
    e1 = C - A
    n = np.stack([e0[:, 1] * e1[:, 2] - e0[:, 2] * e1[:, 1], e0[:, 2] * e1[:, 0] - e0[:, 0] * e1[:, 2],
                  e0[:, 0] * e1[:, 1] - e0[:, 1] * e1[:, 0]], axis=1)
    nn = np.maximum(n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1] + n[:, 2] * n[:, 2], T(np.finfo(dt).tiny))
    w = p - A
    dp = (n[:, 0] * w[:, 0] + n[:, 1] * w[:, 1] + n[:, 2] * w[:, 2]) / np.sqrt(nn)
    in_plane = (d2 - dp * dp) <= T(1e-18) + T(1e-12) * d2
    vote = in_plane & (np.abs(dp) > T(plane_zone)) & (dp != 0)
    votes = np.zeros(nt, dtype=np.float64)
    np.add.at(votes, best[vote], (sig * np.sign(dp))[vote].astype(np.float64))
    orient = np.sign((a.astype(np.float64) * np.cross(b.astype(np.float64), c.astype(np.float64))).sum())
    side = np.where(votes != 0, np.sign(votes), orient)[best].astype(dt)
    on = in_plane & (np.abs(dp) <= T(plane_zone)) & (side != 0)
    return np.where(on, side * dp, sig * d).astype(dt)


def grid_points(grid, dtype):
    """(P, 3) centres of grid = (nx, ny, nz, h, x0, y0, z0), z slowest (geometry.py:253-257)."""
    nx, ny, nz, h, x0, y0, z0 = grid
    T = np.dtype(dtype).type
    zs = T(z0) + (np.arange(nz, dtype=dtype) + T(0.5)) * T(h)
    ys = T(y0) + (np.arange(ny, dtype=dtype) + T(0.5)) * T(h)
    xs = T(x0) + (np.arange(nx, dtype=dtype) + T(0.5)) * T(h)
    zz, yy, xx = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.stack([xx.reshape(-1), yy.reshape(-1), zz.reshape(-1)], axis=1)


def grid_signed_distance(vertices, faces, grid, dtype):
    """The private path of grid_signed_distance (plane_zone 0.02 h), shape (nz, ny, nx)."""
    nx, ny, nz, h = grid[:4]
    d = mesh_signed_distance(np.asarray(vertices, dtype=dtype), faces, grid_points(grid, dtype), plane_zone=0.02 * h)
    return d.reshape(nz, ny, nx)


def smooth_step(d, w):
    T = d.dtype.type
    s = np.clip(d / T(w), T(-1.0), T(1.0))
    return T(0.5) - T(0.5) * np.sin(T(0.5 * math.pi) * s)


@dataclass
class MaskOps:
    """The operator fields build_geometry3d reads (core.py:61-108)."""
    nx: int
    ny: int
    nz: int
    h: float
    x0: float = 0.0
    y0: float = 0.0
    z0: float = 0.0
    periodic_axes: tuple = (False, False, False)
    moment_ref: tuple = (0.0, 0.0, 0.0)
    mask_width: float = 1.0
    mask_shift: float = 0.32


@dataclass
class MeshBody:
    """One immersed mesh (config.py:81-117): vertices, faces, rigid spin."""
    vertices: np.ndarray
    faces: np.ndarray
    omega: float = 0.0
    center: tuple = (0.0, 0.0, 0.0)
    axis: tuple = (0.0, 1.0, 0.0)


def body_window3d(vertex_sets, ops):
    """Cell window of all vertices plus the mask margin, clipped (geometry.py:323-356)."""
    pts = np.vstack([np.asarray(v, np.float64).reshape(-1, 3) for v in vertex_sets if len(v)])
    margin = ops.mask_width + 3.0 + abs(ops.mask_shift)
    h = ops.h
    lo, hi = pts.min(axis=0), pts.max(axis=0)
    i0, i1 = math.floor((lo[0] - ops.x0) / h - margin), math.ceil((hi[0] - ops.x0) / h + margin)
    j0, j1 = math.floor((lo[1] - ops.y0) / h - margin), math.ceil((hi[1] - ops.y0) / h + margin)
    k0, k1 = math.floor((lo[2] - ops.z0) / h - margin), math.ceil((hi[2] - ops.z0) / h + margin)
    i0, i1 = max(i0, 0), min(i1, ops.nx)
    j0, j1 = max(j0, 0), min(j1, ops.ny)
    k0, k1 = max(k0, 0), min(k1, ops.nz)
    if i1 <= i0 or j1 <= j0 or k1 <= k0:
        return (0, 0, 0, 0, 0, 0)
    return (k0, k1, j0, j1, i0, i1)


def build_geometry3d(bodies, ops, dtype, window=None):
    """dict of chi_u/v/w/c, a_u/v/w, k_u/v/w and the window (geometry.py:385-495)."""
    T = np.dtype(dtype).type
    nb = len(bodies)
    if window is None:
        window = body_window3d([b.vertices for b in bodies], ops)
    k0, k1, j0, j1, i0, i1 = window
    wz, wy, wx = k1 - k0, j1 - j0, i1 - i0
    if nb == 0 or wz <= 0 or wy <= 0 or wx <= 0:
        return {"window": (0, 0, 0, 0, 0, 0)}
    h = ops.h
    w = ops.mask_width * h
    shift = ops.mask_shift * h
    X0, Y0, Z0 = ops.x0 + i0 * h, ops.y0 + j0 * h, ops.z0 + k0 * h
    grids = {"u": (wx + 1, wy, wz, h, X0 - 0.5 * h, Y0, Z0), "v": (wx, wy + 1, wz, h, X0, Y0 - 0.5 * h, Z0),
             "w": (wx, wy, wz + 1, h, X0, Y0, Z0 - 0.5 * h), "c": (wx, wy, wz, h, X0, Y0, Z0)}
    chis = {k: [] for k in grids}
    for b in bodies:
        for key, g in grids.items():
            d = grid_signed_distance(b.vertices, b.faces, g, dtype)
            chis[key].append(smooth_step(d + T(shift), w))
    cu, cv, cw, cc = (np.stack(chis[k]) for k in ("u", "v", "w", "c"))
    px, py, pz = ops.periodic_axes
    if not px:
        fu = np.ones(wx + 1, dtype=dtype)
        if i0 == 0:
            fu[0] = 0
        if i1 == ops.nx:
            fu[-1] = 0
        cu = cu * fu
    if not py:
        fv = np.ones(wy + 1, dtype=dtype)
        if j0 == 0:
            fv[0] = 0
        if j1 == ops.ny:
            fv[-1] = 0
        cv = cv * fv[:, None]
    if not pz:
        fw = np.ones(wz + 1, dtype=dtype)
        if k0 == 0:
            fw[0] = 0
        if k1 == ops.nz:
            fw[-1] = 0
        cw = cw * fw[:, None, None]
    out = {"window": tuple(window)}
    for name, x in (("chi_u", cu), ("chi_v", cv), ("chi_w", cw), ("chi_c", cc)):
        out[name] = np.minimum(x.sum(0), T(1.0))

    def coords(g):
        nx_, ny_, nz_, _, gx, gy, gz = g
        zs = T(gz) + (np.arange(nz_, dtype=dtype) + T(0.5)) * T(h)
        ys = T(gy) + (np.arange(ny_, dtype=dtype) + T(0.5)) * T(h)
        xs = T(gx) + (np.arange(nx_, dtype=dtype) + T(0.5)) * T(h)
        return zs[:, None, None], ys[None, :, None], xs[None, None, :]

    zu, yu, _ = coords(grids["u"])
    zv, _, xv = coords(grids["v"])
    _, yw, xw = coords(grids["w"])
    a_u, a_v, a_w = (np.zeros_like(out[k]) for k in ("chi_u", "chi_v", "chi_w"))
    for b, body in enumerate(bodies):
        om = body.omega
        if om == 0.0:
            continue
        cx, cy, cz = (T(x) for x in body.center)
        axx, axy, axz = (T(x) for x in body.axis)
        om = T(om)
        a_u = a_u + cu[b] * (om * (axy * (zu - cz) - axz * (yu - cy)))
        a_v = a_v + cv[b] * (om * (axz * (xv - cx) - axx * (zv - cz)))
        a_w = a_w + cw[b] * (om * (axx * (yw - cy) - axy * (xw - cx)))
    out.update(a_u=a_u, a_v=a_v, a_w=a_w)
    if nb == 1:
        wu, wv, ww = np.ones_like(cu), np.ones_like(cv), np.ones_like(cw)
    else:
        wu, wv, ww = (x / (x.sum(0, keepdims=True) + T(1e-30)) for x in (cu, cv, cw))
    xr, yr, zr = (T(x) for x in ops.moment_ref)
    out["k_u"] = np.stack([wu * np.ones_like(out["chi_u"]), wu * (zu - zr), -wu * (yu - yr)], axis=1)
    out["k_v"] = np.stack([wv * np.ones_like(out["chi_v"]), -wv * (zv - zr), wv * (xv - xr)], axis=1)
    out["k_w"] = np.stack([ww * np.ones_like(out["chi_w"]), ww * (yw - yr), -ww * (xw - xr)], axis=1)
    return out
