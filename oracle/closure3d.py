"""Oracle of the learned closure's non-network arithmetic (test infrastructure only: imported by
tests/ and nothing else).

The reference has no learned closure; these are restatements, in numpy float64, of the parts of
the closure that the library computes around the network:

* ``filter_pairs``: the box filter of a periodic staggered state onto coarse cells (the
  filtered cell-centred velocities' subgrid stress and the coarse face velocities) and the
  coarse gradient by the reference's velocity-gradient stencil (src/aerolume/solvers/ns3d/
  core.py:400-445: face differences on the diagonal, averages of four edge differences off
  it, g33 = -(g11 + g22)), periodic neighbours.
* ``features``: the network's ten inputs of a gradient and the scales around them.
* ``eddy_viscosity``: the closure's nu_t given the network's standardised outputs, with the
  fallback to the WALE value (the reference's core.py:448-482 model) where the learned
  dissipation is not positive or an input leaves the training range.
* ``mlp``: the network in float32 with its operands rounded to bfloat16 between layers and its
  SiLU, x (1 + tanh(x / 2)) / 2, rounded to bfloat16 at each operation (the precision the
  tensor-core kernels run at), for the kernels' tolerance checks.
"""
from __future__ import annotations

import numpy as np

SQRT6 = np.sqrt(6.0)


def filter_pairs(u, v, w, n, h, factor):
    """(g8 (8, m^3), tau (6, m^3)) of a periodic n^3 state, m = n / factor, float64."""
    u, v, w = (np.asarray(a, np.float64) for a in (u, v, w))
    m = n // factor
    uc = 0.5 * (u[:, :, :-1] + u[:, :, 1:])
    vc = 0.5 * (v[:, :-1, :] + v[:, 1:, :])
    wc = 0.5 * (w[:-1] + w[1:])

    def box(a):
        return a.reshape(m, factor, m, factor, m, factor).mean(axis=(1, 3, 5))

    mu, mv, mw = box(uc), box(vc), box(wc)
    tau = np.stack([box(uc * uc) - mu * mu, box(vc * vc) - mv * mv, box(wc * wc) - mw * mw,
                    box(uc * vc) - mu * mv, box(uc * wc) - mu * mw, box(vc * wc) - mv * mw])
    # coarse faces: the factor x factor fine faces on each coarse face averaged
    U = u[:, :, :-1][:, :, ::factor].reshape(m, factor, m, factor, m).mean(axis=(1, 3))
    V = v[:, :-1, :][:, ::factor, :].reshape(m, factor, m, m, factor).mean(axis=(1, 4))
    W = w[:-1][::factor].reshape(m, m, factor, m, factor).mean(axis=(2, 4))
    d = 1.0 / (factor * h)

    def sh(a, dk=0, dj=0, di=0):
        return np.roll(a, shift=(-dk, -dj, -di), axis=(0, 1, 2))

    q = 0.25
    g11 = (sh(U, di=1) - U) * d
    g22 = (sh(V, dj=1) - V) * d
    g12 = ((((U - sh(U, dj=-1)) * d + (sh(U, dj=1) - U) * d) + (sh(U, di=1) - sh(U, dj=-1, di=1)) * d)
           + (sh(U, dj=1, di=1) - sh(U, di=1)) * d) * q
    g13 = ((((U - sh(U, dk=-1)) * d + (sh(U, dk=1) - U) * d) + (sh(U, di=1) - sh(U, dk=-1, di=1)) * d)
           + (sh(U, dk=1, di=1) - sh(U, di=1)) * d) * q
    g21 = ((((V - sh(V, di=-1)) * d + (sh(V, dj=1) - sh(V, dj=1, di=-1)) * d) + (sh(V, di=1) - V) * d)
           + (sh(V, dj=1, di=1) - sh(V, dj=1)) * d) * q
    g23 = ((((V - sh(V, dk=-1)) * d + (sh(V, dk=1) - V) * d) + (sh(V, dj=1) - sh(V, dk=-1, dj=1)) * d)
           + (sh(V, dk=1, dj=1) - sh(V, dj=1)) * d) * q
    g31 = ((((W - sh(W, di=-1)) * d + (sh(W, dk=1) - sh(W, dk=1, di=-1)) * d) + (sh(W, di=1) - W) * d)
           + (sh(W, dk=1, di=1) - sh(W, dk=1)) * d) * q
    g32 = ((((W - sh(W, dj=-1)) * d + (sh(W, dk=1) - sh(W, dk=1, dj=-1)) * d) + (sh(W, dj=1) - W) * d)
           + (sh(W, dk=1, dj=1) - sh(W, dk=1)) * d) * q
    g8 = np.stack([g11, g12, g13, g21, g22, g23, g31, g32]).reshape(8, -1)
    return g8, tau.reshape(6, -1)


def tensors(g8):
    """(g (n, 3, 3), S (n, 3, 3)) of traceless gradients g8 (8, n)."""
    g8 = np.asarray(g8, np.float64)
    n = g8.shape[1]
    g = np.zeros((n, 3, 3))
    g[:, 0, 0], g[:, 0, 1], g[:, 0, 2] = g8[0], g8[1], g8[2]
    g[:, 1, 0], g[:, 1, 1], g[:, 1, 2] = g8[3], g8[4], g8[5]
    g[:, 2, 0], g[:, 2, 1] = g8[6], g8[7]
    g[:, 2, 2] = -(g8[0] + g8[4])
    return g, 0.5 * (g + g.transpose(0, 2, 1))


def features(g8, delta, tau=None):
    """(feat (n, 10), scale (n), valid (n), target (n, 6) or None)."""
    g, S = tensors(g8)
    g2 = (g * g).sum((1, 2))
    s2 = (S * S).sum((1, 2))
    valid = (g2 > 1e-20) & (s2 > 1e-6 * g2)
    ig = np.where(valid, 1.0 / np.sqrt(np.where(valid, g2, 1.0)), 0.0)
    feat = np.zeros((g8.shape[1], 10))
    feat[:, :8] = np.asarray(g8, np.float64).T * ig[:, None]
    feat[:, 8] = np.where(valid, (g2 - 2.0 * s2) / np.where(valid, g2, 1.0), 0.0)
    t3 = np.einsum("nab,nbc,nca->n", S, S, S)
    feat[:, 9] = np.where(valid, SQRT6 * t3 / np.where(valid, s2 * np.sqrt(s2), 1.0), 0.0)
    scale = delta * delta * g2
    target = None
    if tau is not None:
        target = np.where(valid[:, None], np.asarray(tau, np.float64).T / scale[:, None], 0.0)
    return feat, scale, valid, target


def mlp(params, x, layout):
    """The network on standardised inputs x (n, 10) in float32 with bfloat16 operands: the
    weights and each layer's input rounded to bfloat16, FP32 accumulation, SiLU."""
    import torch
    p = torch.as_tensor(np.asarray(params, np.float32))
    views, off = {}, 0
    for name, shape in layout:
        k = int(np.prod(shape))
        views[name] = p[off:off + k].view(*shape)
        off += k
    bf = lambda a: a.to(torch.bfloat16).to(torch.float32)   # noqa: E731
    h = bf(torch.as_tensor(np.asarray(x, np.float32)))
    for q in (1, 2, 3):
        z = h @ bf(views[f"w{q}"]).T + views[f"b{q}"]
        z = bf(z)
        h = bf(z * bf(0.5 * bf(torch.tanh(0.5 * z)) + 0.5))   # SiLU in BF16 arithmetic
    y = h @ bf(views["w4"]).T + views["b4"]
    return y.numpy().astype(np.float64)


def eddy_viscosity(y, g8, fac, nu_wale, delta, out_mean, out_std, in_lo, in_hi, feat=None):
    """(nu_t, used) of the closure: y (n, 6) the network's standardised outputs."""
    g, S = tensors(g8)
    f, scale, valid, _ = features(g8, delta)
    inside = valid & np.all((f >= np.asarray(in_lo)) & (f <= np.asarray(in_hi)), axis=1)
    tau = scale[:, None] * (np.asarray(y, np.float64) * np.asarray(out_std) + np.asarray(out_mean))
    eps = -((tau[:, 0] * S[:, 0, 0] + tau[:, 1] * S[:, 1, 1] + tau[:, 2] * S[:, 2, 2])
            + 2.0 * ((tau[:, 3] * S[:, 0, 1] + tau[:, 4] * S[:, 0, 2]) + tau[:, 5] * S[:, 1, 2]))
    s2 = (S * S).sum((1, 2))
    used = inside & (eps > 0)
    safe = 2.0 * np.where(used, s2, 1.0)
    nu = np.where(used, np.asarray(fac) * eps / safe, np.asarray(nu_wale, np.float64))
    # the size of the dissipation's terms, sum |tau_ij S_ij|, as an eddy viscosity: the scale of
    # the rounding error of nu (eps is a sum of terms of either sign)
    terms = (np.abs(tau[:, 0] * S[:, 0, 0]) + np.abs(tau[:, 1] * S[:, 1, 1]) + np.abs(tau[:, 2] * S[:, 2, 2])
             + 2.0 * (np.abs(tau[:, 3] * S[:, 0, 1]) + np.abs(tau[:, 4] * S[:, 0, 2]) + np.abs(tau[:, 5] * S[:, 1, 2])))
    return nu, used, np.asarray(fac) * terms / safe
