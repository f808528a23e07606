"""The 3D solver's per-step bookkeeping on the device (src/aerolume/solvers/ns3d/solver.py:706-744).

:func:`record` has the signature of ``FlowSolver3D._record(self, new, bc, sample)`` and reads
the same solver attributes (``_body_c``, ``_hist``, ``_hist_n``, ``_phist``, ``_phys``,
``_phist_walls``, ``_avg_on``, ``_avg``, ``_theta``), so binding it as the method swaps the
bookkeeping: the history ring row and the physics-history row in one launch
(``aero_record_history``), and on sampling steps the time-weighted Welford update of u, v, w,
p (and theta) in one launch over all fields (``aero_welford``).  :func:`welford` is the
sampling update alone (``FlowSolver3D._welford``).  Everything stays on the caller's current
stream; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import torch

from .. import _lib
from .._lib import F32, F64, check


def _code(dtype):
    if dtype == torch.float64:
        return F64
    if dtype == torch.float32:
        return F32
    raise RuntimeError(f"unsupported dtype {dtype}")


def _stream(t):
    if not torch.is_tensor(t) or t.device.type != "cuda":
        raise RuntimeError("the bookkeeping runs on CUDA tensors only (no CPU fallback)")
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _physics_parts(self, new):
    """The physics-history row after t, as the reference builds it (solver.py:713-720)."""
    ph = self._phys
    parts = []
    if ph.thermal is not None:
        parts.append(ph.thermal.heat_rate)
        if self._phist_walls:
            parts.append(ph.thermal.geom.wall_theta(self._theta))
    if ph.fans is not None:
        parts += [ph.fans.thrust, ph.fans.ud]
    return torch.cat([p.reshape(-1) for p in parts]).to(self.dtype) if parts else None


def record(self, new, bc, sample) -> None:
    """One step's bookkeeping (FlowSolver3D._record): the history rows, the averaging clock and,
    when ``sample``, the Welford update of the running means."""
    hist, hist_n = self._hist, self._hist_n
    st = _stream(hist)
    dt_code = _code(hist.dtype)
    for name, x in (("hist", hist), ("bc", bc), ("t", new.t)):
        if not x.is_contiguous() or x.dtype != hist.dtype:
            raise RuntimeError(f"{name} must be a contiguous {hist.dtype} tensor")
    if hist_n.dtype != torch.int64:
        raise RuntimeError("the ring counter must be an int64 tensor")
    phist = getattr(self, "_phist", None)
    extra = _physics_parts(self, new) if phist is not None else None
    if phist is not None and (extra is None or phist.shape[1] != 1 + extra.numel()):
        raise RuntimeError("the physics-history row does not match its ring")
    avg = self._avg if getattr(self, "_avg_on", False) else None
    nb = int(bc.shape[0])
    dt_t = new.dt.to(hist.dtype).contiguous() if avg is not None else None
    check(_lib.lib().aero_record_history(
        dt_code, _ptr(new.t), _ptr(dt_t), _ptr(bc) if nb else None, nb, _ptr(self._body_c) if nb else None,
        _ptr(hist), hist.shape[0], _ptr(hist_n), _ptr(extra), 0 if extra is None else extra.numel(), _ptr(phist),
        _ptr(avg["pending"]) if avg is not None else None, st), "aero_record_history")
    if avg is not None and sample:
        fields = [new.u, new.v, new.w, new.p]
        if "t" in avg and self._theta is not None:
            fields.append(self._theta)
        welford(self, avg, fields)


def welford(self, a: dict, fields) -> None:
    """The time-weighted Welford update (FlowSolver3D._welford), all fields in one launch."""
    names = "uvwpt"[:len(fields)]
    xs, means, m2s, counts = [], [], [], []
    for name, x in zip(names, fields):
        m, s = a[name], a[name + "2"]
        for t in (x, m, s):
            if not t.is_contiguous() or t.dtype != x.dtype or t.shape != x.shape:
                raise RuntimeError("fields and running means must be contiguous, of one dtype and shape")
        xs.append(x.data_ptr())
        means.append(m.data_ptr())
        m2s.append(s.data_ptr())
        counts.append(x.numel())
    for k in ("pending", "time"):
        if a[k].dtype != torch.float64:
            raise RuntimeError("the averaging clock must be float64")
    n = len(xs)
    arr = lambda v: (C.c_void_p * n)(*v)   # noqa: E731
    check(_lib.lib().aero_welford(_code(fields[0].dtype), n, arr(xs), arr(means), arr(m2s), (C.c_int64 * n)(*counts),
                                  _ptr(a["pending"]), _ptr(a["time"]), _stream(fields[0])), "aero_welford")
