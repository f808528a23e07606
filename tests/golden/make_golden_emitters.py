"""Golden vectors of the reference's smoke emitters (run in the build container).

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_emitters.py

The reference's own ``apply_smoke_sources`` (src/aerolume/solvers/ns3d/emitters.py:200-210,
with ``release_switch`` 83-87 and ``emitter_params`` 70-80) runs, unmodified, on seeded smoke
channels (two channels of 8 x 10 x 12) with four emitters: always on (the legacy rake), pulsed
(on and off phases), not started yet, and stopped -- two of them on the same channel with
overlapping windows -- at three times, in FP64 and FP32.  Inputs and outputs go to
``emitters3d.npz``.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

import make_golden as G  # noqa: E402,F401  (puts the reference on sys.path)
from aerolume.solvers.ns3d import emitters as E  # noqa: E402


def main():
    out: dict = {}
    specs = [  # window, channel, emitter (None: the legacy rake)
        ((1, 5, 2, 7, 0, 3), 0, None),
        ((2, 6, 3, 8, 2, 6), 0, SimpleNamespace(stop=None, pulse_period=0.4, pulse_duty=0.5, rate=0.8, enabled=True,
                                                start=0.1)),
        ((0, 3, 0, 4, 5, 9), 1, SimpleNamespace(stop=None, pulse_period=0.0, pulse_duty=0.0, rate=1.0, enabled=True,
                                                start=5.0)),
        ((4, 8, 5, 10, 7, 12), 1, SimpleNamespace(stop=0.3, pulse_period=0.0, pulse_duty=0.0, rate=0.6, enabled=True,
                                                  start=0.0)),
    ]
    times = (0.2, 0.45, 0.62)
    for dtype, tag in ((torch.float64, "f64"), (torch.float32, "f32")):
        g = torch.Generator().manual_seed(21)
        chans = [torch.rand(8, 10, 12, generator=g, dtype=torch.float64).to(dtype) for _ in range(2)]
        sources = []
        for q, (win, ch, e) in enumerate(specs):
            k0, k1, j0, j1, i0, i1 = win
            w = (0.9 * torch.rand(k1 - k0, j1 - j0, i1 - i0, generator=g, dtype=torch.float64)).to(dtype)
            params = E.emitter_params(e, "cpu", dtype)
            sources.append(E.EmitterSource(win, w, params, ch))
            out[f"{tag}_w{q}"] = w.numpy()
            out[f"{tag}_p{q}"] = params.numpy()
        for c in range(2):
            out[f"{tag}_in_c{c}"] = chans[c].numpy().copy()
        for s, t in enumerate(times):
            E.apply_smoke_sources(chans, torch.tensor(t, dtype=dtype), sources)
            for c in range(2):
                out[f"{tag}_out{s}_c{c}"] = chans[c].numpy().copy()
    out["meta"] = np.array(json.dumps({"windows": [list(w) for w, _, _ in specs], "channels": [c for _, c, _ in specs],
                                       "times": list(times)}))
    np.savez_compressed(HERE / "emitters3d.npz", **out)
    print("wrote", HERE / "emitters3d.npz")


if __name__ == "__main__":
    main()
