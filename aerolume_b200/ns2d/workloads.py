"""Seeded synthetic 2D workloads: the cylinder wake (256 x 128) and the batched NACA sweep.

Both follow the benchmark configurations: a circular cylinder of diameter 0.5 at (2, 2) in an
8 x 4 slip-walled tunnel at Re_D = 100 (Re = 200 on the unit length), upwind3, CFL 0.5, no
LES, no dye; and 64 NACA 4-digit airfoils (chord 1, quarter chord at (2, 2)) on grids drawn
from {256x128, 384x192, 512x256, 768x384, 1024x512} with seeded thickness, camber, camber
position, angle of attack and Reynolds number.  Initial fields: the inlet profile plus seeded
N(0, noise) on u and v, boundary values imposed, then projected.

``heated_cylinder`` is the cylinder wake with heat transfer: the cylinder held at theta = 1
in a stream at theta = 0, Pr 0.71, Ri 0.5 with gravity along -y, inlet / outlet temperature
sides and adiabatic walls (the reference's heated-cylinder validation set-up).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .setup import build_geometry, make_ops, polygon_sdf, smooth_step
from .types import Thermal2D

SWEEP_GRIDS = ((256, 128), (384, 192), (512, 256), (768, 384), (1024, 512))


def circle(cx, cy, r, n):
    a = 2.0 * math.pi * np.arange(n) / n
    return np.stack([cx + r * np.cos(a), cy + r * np.sin(a)], axis=1)


def cylinder_tunnel(nx=256, ny=128, dtype="float32", vertices=256):
    """Cylinder D = 0.5 at (2, 2) in the 8 x 4 tunnel, Re_D = 100."""
    h = 8.0 / nx
    ops = make_ops(nx, ny, h, 200.0, force_ref=0.5, moment_ref=(2.0, 2.0), dtype=dtype)
    geom = build_geometry([circle(2.0, 2.0, 0.25, vertices)], ops)
    return ops, geom


def naca4(t, m, p, alpha_deg, n=160, pivot=(2.0, 2.0)):
    """NACA 4-digit outline (thickness t, camber m at p; Jacobs' published equations, closed
    trailing edge), chord 1, counter-clockwise, rotated nose-up by alpha about the quarter
    chord placed at ``pivot``."""
    beta = np.linspace(0.0, math.pi, n // 2 + 1)
    x = 0.5 * (1.0 - np.cos(beta))
    yt = 5.0 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)
    if m > 0 and 0 < p < 1:
        yc = np.where(x < p, m / p ** 2 * (2 * p * x - x ** 2), m / (1 - p) ** 2 * ((1 - 2 * p) + 2 * p * x - x ** 2))
        dyc = np.where(x < p, 2 * m / p ** 2 * (p - x), 2 * m / (1 - p) ** 2 * (p - x))
    else:
        yc = np.zeros_like(x)
        dyc = np.zeros_like(x)
    th = np.arctan(dyc)
    xu, yu = x - yt * np.sin(th), yc + yt * np.cos(th)
    xl, yl = x + yt * np.sin(th), yc - yt * np.cos(th)
    # trailing edge -> upper surface -> leading edge -> lower surface (counter-clockwise from
    # the trailing edge going over the top is clockwise; reverse to keep the outline CCW)
    px = np.concatenate([xl[::-1][:-1], xu[:-1]])
    py = np.concatenate([yl[::-1][:-1], yu[:-1]])
    pts = np.stack([px, py], axis=1)[::-1]
    qc = np.array([0.25, float(np.interp(0.25, x, yc))])
    a = -math.radians(alpha_deg)          # nose up for flow along +x
    rot = np.array([[math.cos(a), -math.sin(a)], [math.sin(a), math.cos(a)]])
    return (pts - qc) @ rot.T + np.asarray(pivot)


def sweep_instances(n=64, seed=0, dtype="float32"):
    """The batched sweep's instances: [(ops, geom, params)] in a seeded, reproducible order."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx, ny = SWEEP_GRIDS[int(rng.integers(len(SWEEP_GRIDS)))]
        t, m, p = rng.uniform(0.06, 0.18), rng.uniform(0.0, 0.06), rng.uniform(0.3, 0.5)
        alpha = rng.uniform(-4.0, 16.0)
        re = float(10.0 ** rng.uniform(3.0, 4.0))
        ops = make_ops(nx, ny, 8.0 / nx, re, force_ref=1.0, moment_ref=(2.0, 2.0), dtype=dtype)
        geom = build_geometry([naca4(t, m, p, alpha)], ops)
        out.append((ops, geom, {"grid": (nx, ny), "t": t, "m": m, "p": p, "alpha": alpha, "re": re}))
    return out


def initial_state(ops, plan, seed=0, noise=1e-3):
    """Inlet profile + seeded N(0, noise) on u and v, boundary values, projection (on the
    plan's device, with its Poisson solve)."""
    ny, nx = ops.ny, ops.nx
    g = torch.Generator().manual_seed(seed)
    inlet = torch.as_tensor(np.asarray(ops.u_inlet, np.float64))
    u = inlet.reshape(ny, 1).expand(ny, nx + 1).clone() + noise * torch.randn(ny, nx + 1, generator=g, dtype=torch.float64)
    v = noise * torch.randn(ny + 1, nx, generator=g, dtype=torch.float64)
    u[:, 0] = inlet
    u[:, -1] = u[:, -1] + (inlet.sum() - u[:, -1].sum()) / ny
    v[0] = 0.0
    v[-1] = 0.0
    dev, dt = plan.device, plan.dtype
    u, v = u.to(dev, dt), v.to(dev, dt)
    div = ((u[:, 1:] - u[:, :-1]) + v[1:] - v[:-1]) * (1.0 / ops.h)
    psi = plan.poisson_solve(div.contiguous())
    u[:, 1:-1] -= (psi[:, 1:] - psi[:, :-1]) * (1.0 / ops.h)
    v[1:-1] -= (psi[1:] - psi[:-1]) * (1.0 / ops.h)
    return u.contiguous(), v.contiguous()


def heated_cylinder(nx=256, ny=128, dtype="float32", vertices=256, prandtl=0.71, richardson=0.5):
    """(ops, geom, thermal) of the cylinder tunnel with the cylinder held at theta = 1: the
    thermal masks of ns2d/geometry.py:385-419 for one temperature body (chi_t = the cell
    mask, a_t = chi_t, unit share, no insulated or heat-flux body) and the face area
    fractions without the wall offset for the buoyancy share; kappa = 1 / (Re Pr), the
    thermal permeability and diffusion coefficient of physics.py:263-288, 833-848."""
    ops, geom = cylinder_tunnel(nx, ny, dtype, vertices)
    h = ops.h
    poly = circle(2.0, 2.0, 0.25, vertices)
    j0, j1, i0, i1 = geom.window
    wy, wx = j1 - j0, i1 - i0

    def grid(nr, nc, xoff, yoff):
        ys = ops.y0 + (np.arange(nr) + j0 + yoff) * h
        xs = ops.x0 + (np.arange(nc) + i0 + xoff) * h
        return np.meshgrid(ys, xs, indexing="ij")

    yu, xu = grid(wy, wx + 1, 0.0, 0.5)
    yv, xv = grid(wy + 1, wx, 0.5, 0.0)
    vol_u = smooth_step(polygon_sdf(poly, xu, yu), h)
    vol_v = smooth_step(polygon_sdf(poly, xv, yv), h)
    chi_t = np.asarray(geom.chi_c, np.float64)
    pe = 200.0 * prandtl                                   # Re 200 per unit length
    eta_t = min(0.05 * h, h * h * pe / 60.0)
    th = Thermal2D(kappa=1.0 / pe, ri=richardson, prt=0.85, gravity=(0.0, -1.0), eta_t=eta_t, theta_in=0.0,
                   wall_modes=("inlet", "outlet", "adiabatic", "adiabatic"), wall_values=(0.0, 0.0, 0.0, 0.0),
                   diff_coef=5.0, temp_ids=(0,), flux_ids=(), chi_t=chi_t, a_t=chi_t * 1.0,
                   w_t=np.ones((1, wy, wx)), ins_u=np.ones((wy, wx + 1)), ins_v=np.ones((wy + 1, wx)),
                   vol_u=vol_u, vol_v=vol_v)
    return ops, geom, th
