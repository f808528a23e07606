"""CPU restatement of the reference's smoke emitters (field sources).

TEST INFRASTRUCTURE ONLY: tests use this module as the checker; nothing in the product path
imports it.

Follows src/aerolume/solvers/ns3d/emitters.py:
  release_switch       emitters.py:83-87    1 while t is past the start, before the stop and
                                            in the on part of the pulse period (the float
                                            remainder of torch, exact through fmod)
  apply_smoke_sources  emitters.py:200-210  each emitter in turn relaxes its channel towards
                                            its rate inside its window: c += w on (rate - c)
Pinned by tests/golden/emitters3d.npz (the reference's own function on seeded channels).
"""
from __future__ import annotations

import numpy as np


def release_switch(t, params):
    T = params.dtype.type
    since = T(t) - params[1]
    rem = np.fmod(since, params[3])
    if rem != 0 and (params[3] < 0) != (rem < 0):
        rem = rem + params[3]
    on = since >= 0 and T(t) < params[2] and rem < params[4]
    return T(1.0) if on else T(0.0)


def apply_smoke_sources(channels, t, sources):
    """In place; ``sources`` items: (window, weight, params, channel)."""
    for win, w, p, ch in sources:
        k0, k1, j0, j1, i0, i1 = win
        c = channels[ch][k0:k1, j0:j1, i0:i1]
        on = release_switch(t, p)
        c[...] = c + (w * on) * (p[0] - c)
