"""CPU restatement of the reference's per-step bookkeeping of the 3D solver.

TEST INFRASTRUCTURE ONLY: tests and the bench's CPU leg use this module as the checker;
nothing in the product path imports it.

Follows src/aerolume/solvers/ns3d/solver.py:
  record   solver.py:706-730  the history ring row (t, the bodies' coefficients summed), the
                              physics history row, the ring counter, the pending averaging time
  welford  solver.py:732-744  the time-weighted Welford update of the running means and second
                              moments with the weight of the time elapsed since the last sample
numpy in the working dtype; the averaging clock (time, pending) is FP64 as in the reference.
Pinned by tests/golden/record3d.npz (the reference's own methods on seeded steps).
"""
from __future__ import annotations

import numpy as np


def record(buf, t, dt, bc, sample, fields=None, extra=None):
    """One step's bookkeeping, in place on ``buf`` (dict: hist (cap, 7), hist_n (int), body_c
    (nb, 6), phist (cap, 1 + n_extra) or None, avg (dict: time, pending, u, u2, ...) or None)."""
    T = buf["hist"].dtype.type
    bc = np.asarray(bc)
    if bc.shape[0]:
        buf["body_c"][...] = bc
    cap = buf["hist"].shape[0]
    slot = buf["hist_n"] % cap
    buf["hist"][slot] = np.concatenate([[T(t)], bc.sum(axis=0).astype(buf["hist"].dtype)])
    if buf.get("phist") is not None:
        buf["phist"][slot] = np.concatenate([[T(t)], np.asarray(extra, buf["hist"].dtype)])
    buf["hist_n"] += 1
    a = buf.get("avg")
    if a is not None:
        a["pending"] = a["pending"] + np.float64(T(dt))
        if sample:
            welford(a, fields, buf["hist"].dtype)


def welford(a, fields, dtype):
    """Fold the fields (name -> array) into the running means (solver.py:732-744)."""
    T = np.dtype(dtype).type
    w = np.float64(a["pending"])
    a["time"] = np.float64(a["time"]) + w
    r = T(w / a["time"])
    wf = T(w)
    for name, x in fields.items():
        mean, m2 = a[name], a[name + "2"]
        d = x - mean
        mean[...] = mean + d * r
        m2[...] = m2 + (d * (x - mean)) * wf
    a["pending"] = np.float64(0.0)
