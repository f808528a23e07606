"""Synthetic 3D workloads (seeded inputs with the shapes of the benchmark configurations).

``box_on_moving_floor``: a 1 x 1 x 0.5 bluff box on a floor moving at the free-stream
speed, in an 8 x 4 x 4 tunnel at 256 x 128 x 128 cells (4.2 M, h = 1/32); Re = 5000 on the
box height (1e4 per unit length), WALE LES, Boussinesq temperature with the body held at
theta = 1 (10 K above the stream), Pr = 0.71, Ri = 0.1 on the body height (0.2 per unit
length), one smoke rake of 16 seeded nozzles upstream; initial field uniform U = 1 plus
seeded N(0, 1e-3) noise on u, v, w, made divergence-free by the step's own projection.

``sphere_mesh``: a closed latitude-longitude triangulation of a sphere, wound outward, the
body of the mask-construction workload (a live attitude edit rebuilds its masks).
"""
from __future__ import annotations

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
