"""The smoke emitters' per-step release on the device (src/aerolume/solvers/ns3d/emitters.py:200-210).

:func:`apply_smoke_sources` has the reference's signature and reads its ``EmitterSource``
items (``window``, ``weight``, ``params``, ``channel``) as they are, so the solver's tracer
update can call it in place of the reference's function: each emitter in turn relaxes its
channel towards its rate inside its window while its release switch is on
(``aero_smoke_emitters``).  The footprints themselves (``build_smoke_sources``) stay with the
caller: they are set up once.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import torch

from .. import _lib
from .._lib import F32, F64, check


def apply_smoke_sources(channels, t, sources) -> None:
    """In place on the device channels: c += w on (rate - c) inside each emitter's window."""
    items = [s for s in sources if not (s.window[1] <= s.window[0] or s.window[3] <= s.window[2]
                                        or s.window[5] <= s.window[4])]
    if not items:
        return
    c0 = channels[0]
    if not torch.is_tensor(c0) or c0.device.type != "cuda":
        raise RuntimeError("smoke channels must be CUDA tensors (no CPU fallback)")
    dt = c0.dtype
    for c in channels:
        if not c.is_contiguous() or c.dtype != dt or c.shape != c0.shape:
            raise RuntimeError("smoke channels must be contiguous, of one dtype and shape")
    t = t if torch.is_tensor(t) else torch.tensor(float(t), device=c0.device, dtype=dt)
    t = t.to(device=c0.device, dtype=dt).contiguous()
    arr = (_lib.SmokeEmitter * len(items))()
    keep = [t]
    for q, s in enumerate(items):
        w = s.weight.to(device=c0.device, dtype=dt).contiguous()
        p = s.params.to(device=c0.device, dtype=dt).contiguous()
        keep += [w, p]
        for e in range(6):
            arr[q].window[e] = int(s.window[e])
        arr[q].channel = int(s.channel)
        arr[q].weight, arr[q].params = w.data_ptr(), p.data_ptr()
    ptrs = (C.c_void_p * len(channels))(*[c.data_ptr() for c in channels])
    nz, ny, nx = c0.shape
    stream = C.c_void_p(torch.cuda.current_stream(c0.device).cuda_stream)
    check(_lib.lib().aero_smoke_emitters(F64 if dt == torch.float64 else F32, nz, ny, nx, ptrs, len(channels), arr,
                                         len(items), C.c_void_p(t.data_ptr()), stream), "aero_smoke_emitters")
    del keep
