"""Synthetic 3D workloads (seeded inputs with the shapes of the benchmark configurations).

``box_on_moving_floor``: a 1 x 1 x 0.5 bluff box on a floor moving at the free-stream
speed, in an 8 x 4 x 4 tunnel at 256 x 128 x 128 cells (4.2 M, h = 1/32); Re = 5000 on the
box height (1e4 per unit length), WALE LES, Boussinesq temperature with the body held at
theta = 1 (10 K above the stream), Pr = 0.71, Ri = 0.1 on the body height (0.2 per unit
length), one smoke rake of 16 seeded nozzles upstream; initial field uniform U = 1 plus
seeded N(0, 1e-3) noise on u, v, w, made divergence-free by the step's own projection.

``placed_box``: the same box case with the placed physics in the step (a fan disc with swirl,
a warm jet and a vent, a painted block, the PID step controller).

``sphere_mesh``: a closed latitude-longitude triangulation of a sphere, wound outward, the
body of the mask-construction workload (a live attitude edit rebuilds its masks).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .setup import Box, box_geometry, make_ops, rake_sources, thermal_ops


def box_on_moving_floor(nx=256, ny=128, nz=128, *, dtype="float32", seed=0, noise=1e-3):
    """(ops, geom, thermal, dye_sources, boxes) of the bluff-box case, scaled to nx x ny x nz."""
    lx, ly, lz = 8.0, 4.0, 4.0
    h = lx / nx
    if abs(ly / ny - h) > 1e-12 or abs(lz / nz - h) > 1e-12:
        raise ValueError("the box case needs cubic cells: nx : ny : nz = 2 : 1 : 1")
    H = 0.5
    re = 5000.0 / H                          # Re 5000 on the body height
    ri = 0.1 / H                             # Ri 0.1 on the body height -> per unit length
    box = Box(size=(1.0, 1.0, H), center=(2.5, 2.0, 0.5 * H), thermal="temperature", thermal_value=1.0)
    ops = make_ops(nx, ny, nz, h, re=re, bc_zmin="moving", ground_speed=1.0, turbulence="wale",
                   ref_area=1.0 * H, moment_ref=(2.5, 2.0, 0.0), dtype=dtype)
    geom = box_geometry([box], ops)
    sides = {"left": "inflow", "right": "outflow", "front": "slip", "back": "slip", "bottom": "moving", "top": "slip"}
    th = thermal_ops(ops, geom, [box], re=re, prandtl=0.71, richardson=ri, side_walls=sides)
    rng = np.random.default_rng(seed)
    x = 1.25
    ys = np.sort(rng.uniform(1.2, 2.8, 16))
    zs = rng.uniform(0.1, 0.45, 16)
    src = rake_sources([(x, y, z) for y, z in zip(ys, zs)], ops)
    return ops, geom, th, src, [box]


def initial_state(ops, *, seed=0, noise=1e-3, device="cuda"):
    """Uniform inflow plus seeded N(0, noise) on u, v, w (torch float64 on the CPU generator),
    cast to the case dtype on ``device``; boundary values applied, not yet projected."""
    nx, ny, nz = ops.nx, ops.ny, ops.nz
    g = torch.Generator().manual_seed(seed)
    u = torch.ones(nz, ny, nx + 1, dtype=torch.float64) + noise * torch.randn(nz, ny, nx + 1, generator=g,
                                                                             dtype=torch.float64)
    v = noise * torch.randn(nz, ny + 1, nx, generator=g, dtype=torch.float64)
    w = noise * torch.randn(nz + 1, ny, nx, generator=g, dtype=torch.float64)
    u[..., 0] = 1.0
    u[..., -1] = u[..., -1] + (ny * nz - u[..., -1].sum()) / (ny * nz)
    v[:, 0] = 0.0
    v[:, -1] = 0.0
    w[0] = 0.0
    w[-1] = 0.0
    dt = torch.float64 if ops.dtype in ("float64", torch.float64) else torch.float32
    return tuple(a.to(device=device, dtype=dt).contiguous() for a in (u, v, w))


__all__ = ["box_on_moving_floor", "initial_state"]


def sphere_mesh(center, radius, n_lat=48, n_lon=96):
    """(vertices (N, 3) float64, faces (M, 3) int64) of a closed sphere: two poles and
    n_lat - 1 rings of n_lon vertices, 2 n_lon (n_lat - 1) triangles wound outward."""
    c = np.asarray(center, dtype=np.float64)
    th = np.pi * np.arange(1, n_lat) / n_lat                    # polar angle of each ring
    ph = 2.0 * np.pi * np.arange(n_lon) / n_lon
    st, ct = np.sin(th)[:, None], np.cos(th)[:, None]
    ring = np.stack([st * np.cos(ph)[None, :], st * np.sin(ph)[None, :], np.broadcast_to(ct, (n_lat - 1, n_lon))],
                    axis=-1).reshape(-1, 3)
    v = np.vstack([[0.0, 0.0, 1.0], ring, [0.0, 0.0, -1.0]]) * radius + c
    south = len(v) - 1
    idx = lambda r, k: 1 + r * n_lon + (k % n_lon)              # noqa: E731
    f = []
    for k in range(n_lon):
        f.append((0, idx(0, k), idx(0, k + 1)))
        f.append((south, idx(n_lat - 2, k + 1), idx(n_lat - 2, k)))
        for r in range(n_lat - 2):
            a, b, c2, d = idx(r, k), idx(r, k + 1), idx(r + 1, k + 1), idx(r + 1, k)
            f.append((a, d, c2))
            f.append((a, c2, b))
    return v, np.asarray(f, dtype=np.int64)


def _disc_weights(ops, win, g, center, radius, half_len, axis=0):
    """Indicator of the staggered grid g's points of window win inside a cylinder of the given
    radius and half length along the axis through center (numpy float64, window shape)."""
    from .setup import _grid_coords
    Z, Y, X = _grid_coords(ops, win, g)
    c = np.asarray(center, float)
    pts = [X - c[0], Y - c[1], Z - c[2]]
    along = np.abs(pts[axis])
    r2 = sum(p * p for q, p in enumerate(pts) if q != axis)
    return ((along <= half_len) & (r2 <= radius * radius)).astype(np.float64)


def placed_box(nx=256, ny=128, nz=128, *, dtype="float32"):
    """The box on the moving floor with the placed physics of physics.py:831-1262 in the step
    (no smoke: jets and vents leave it to the caller): a velocity-regulated fan disc with swirl
    upstream of the box (radius 0.4, two cells thick, PI thrust towards U = 1.3), a warm jet
    rising from the floor behind the box and a vent in the ceiling, a painted block on the
    floor downstream, and the PID step controller (target 0.85 of the stability limit).
    Returns (ops, geom, thermal, fans, ports, paint, pid, u_floor) with numpy weights; the
    fan and controller state tensors are created on the device by :func:`placed_state`."""
    from .setup import _grid_coords, box_sdf, smooth_step, MASK_SHIFT
    ops, geom, th, _, boxes = box_on_moving_floor(nx, ny, nz, dtype=dtype)
    h = ops.h
    # fan: disc at x = 1.0 about the axis through (y, z) = (2.0, 0.9)
    fc, R = (1.0, 2.0, 0.9), 0.4
    fwin = (max(int((fc[2] - R) / h) - 2, 0), min(int((fc[2] + R) / h) + 3, nz),
            max(int((fc[1] - R) / h) - 2, 0), min(int((fc[1] + R) / h) + 3, ny),
            max(int((fc[0] - 2 * h) / h) - 1, 0), min(int((fc[0] + 2 * h) / h) + 2, nx))
    wu = _disc_weights(ops, fwin, "u", fc, R, h)
    fan = {"win": fwin, "fu": wu / (wu.sum() * h ** 3), "mu": wu / wu.sum()}
    # swirl: tangential weights about the fan axis on the v- and w-faces, zero net force
    for g, comp in (("v", "sv"), ("w", "sw")):
        Z, Y, X = _grid_coords(ops, fwin, g)
        wg = _disc_weights(ops, fwin, g, fc, R, h)
        dy, dz = Y - fc[1], Z - fc[2]
        r = np.sqrt(dy * dy + dz * dz) + 1e-12
        tang = (-dz / r) if g == "v" else (dy / r)
        s = wg * tang
        fan[comp] = (s - wg * (s.sum() / max(wg.sum(), 1.0))) / (max(wg.sum(), 1.0) * h ** 3)
    k0, k1, j0, j1, i0, i1 = fwin
    shapes = {"u": (k1 - k0, j1 - j0, i1 - i0 + 1), "v": (k1 - k0, j1 - j0 + 1, i1 - i0),
              "w": (k1 - k0 + 1, j1 - j0, i1 - i0)}
    for kind in "fsm":                       # the step takes every weight array, zeros included
        for g in "uvw":
            fan.setdefault(kind + g, np.zeros(shapes[g]))
    fans = {"items": [fan], "target": [1.3], "kp": [1.1], "ki": [0.9], "tmax": [60.0], "velocity_mode": [True],
            "swirl": [0.3], "any_swirl": True, "thrust": [0.5]}
    # jet: a disc of radius 0.15 in the floor at x = 4.2 blowing up at 0.8 with theta = 0.7;
    # vent: radius 0.2 in the ceiling at x = 6.5 drawing 0.5 of the jet's volume flow
    jc, jr, vc, vr = (4.2, 2.0, 0.0), 0.15, (6.5, 2.0, nz * h), 0.2
    jwin = (0, 3, int((jc[1] - jr) / h) - 1, int((jc[1] + jr) / h) + 2, int((jc[0] - jr) / h) - 1,
            int((jc[0] + jr) / h) + 2)
    jm = _disc_weights(ops, jwin, "c", jc, jr, 2 * h, axis=2)
    q_jet = 0.8 * math.pi * jr * jr
    m = jm * (q_jet / (jm.sum() * h ** 3))
    jw = np.concatenate([m, np.zeros_like(m[:1])], axis=0) * 0.8
    jet = {"win": jwin, "kind": "jet", "theta": 0.7, "m": m, "fu": np.zeros((3, jwin[3] - jwin[2], jwin[5] - jwin[4] + 1)),
           "fv": np.zeros((3, jwin[3] - jwin[2] + 1, jwin[5] - jwin[4])), "fw": jw}
    vwin = (nz - 3, nz, int((vc[1] - vr) / h) - 1, int((vc[1] + vr) / h) + 2, int((vc[0] - vr) / h) - 1,
            int((vc[0] + vr) / h) + 2)
    vm = _disc_weights(ops, vwin, "c", vc, vr, 2 * h, axis=2)
    mv = -vm * (0.5 * q_jet / (vm.sum() * h ** 3))
    pad = lambda a, ax: np.concatenate([a, a.take([-1], axis=ax)], axis=ax)   # noqa: E731
    vent = {"win": vwin, "kind": "vent", "theta": 0.0, "m": mv, "fu": pad(mv, 2), "fv": pad(mv, 1), "fw": pad(mv, 0)}
    mass_flux = (m.sum() + mv.sum()) * h ** 3 / h ** 2
    ports = {"items": [jet, vent], "mass_flux": mass_flux, "leak": 0.0}
    # paint: a 0.5 x 0.5 x 0.6 block on the floor at x = 5.6, smoothed like the bodies
    from .setup import Box
    blk = Box(size=(0.5, 0.5, 0.6), center=(5.6, 1.4, 0.3))
    full = (0, nz, 0, ny, 0, nx)
    paint = {}
    for g in ("u", "v", "w", "c"):
        Z, Y, X = _grid_coords(ops, full, g)
        paint[g] = smooth_step(box_sdf(blk, X, Y, Z) + MASK_SHIFT * h, h)
    return ops, geom, th, fans, ports, paint, 0.85, 1.3


def placed_state(fans, ports, paint, pid_target, device, dtype):
    """Device-side FanSet3D / PortSet3D / PaintLayer3D / PidState3D of :func:`placed_box`."""
    import torch

    from .types import FanSet3D, PaintLayer3D, PidState3D, PortSet3D
    tdt = torch.float64 if str(dtype) == "float64" else torch.float32
    dev = lambda a: torch.as_tensor(np.asarray(a)).to(device, tdt).contiguous()   # noqa: E731
    items = [{k: (dev(v) if isinstance(v, np.ndarray) else v) for k, v in it.items()} for it in fans["items"]]
    fs = FanSet3D(items, fans["target"], fans["kp"], fans["ki"], fans["tmax"], fans["velocity_mode"], fans["swirl"],
                  fans["any_swirl"], dev(fans["thrust"]), *(torch.zeros(len(items), device=device, dtype=tdt)
                                                           for _ in range(3)))
    ps = PortSet3D([{k: (dev(v) if isinstance(v, np.ndarray) else v) for k, v in it.items()} for it in ports["items"]],
                   ports["mass_flux"], ports["leak"])
    pl = PaintLayer3D(*(dev(paint[g]) for g in ("u", "v", "w", "c")))
    pid = PidState3D(pid_target, *(torch.zeros((), device=device, dtype=tdt) for _ in range(3)))
    return fs, ps, pl, pid
