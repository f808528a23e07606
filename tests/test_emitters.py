"""Smoke emitters: the oracle (CPU) and the CUDA kernel behind the reference-named seam (GPU)
against the reference's own apply_smoke_sources (tests/golden/emitters3d.npz)."""
from __future__ import annotations

import json
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from _golden import GOLDEN
from oracle import emitters3d as E

Z = np.load(GOLDEN / "emitters3d.npz")
META = json.loads(str(Z["meta"]))


def _sources(tag):
    return [(tuple(META["windows"][q]), Z[f"{tag}_w{q}"], Z[f"{tag}_p{q}"], META["channels"][q]) for q in range(4)]


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_oracle_emitters_match_reference(tag):
    ch = [Z[f"{tag}_in_c{c}"].copy() for c in range(2)]
    for s, t in enumerate(META["times"]):
        E.apply_smoke_sources(ch, ch[0].dtype.type(t), _sources(tag))
        for c in range(2):
            assert np.array_equal(ch[c], Z[f"{tag}_out{s}_c{c}"]), (s, c)


def test_fixture_covers_every_switch_state():
    """On, pulsed on and off, not started, stopped; overlapping windows on one channel."""
    assert not np.array_equal(Z["f64_out0_c1"], Z["f64_in_c1"])       # the stopping emitter ran
    assert np.array_equal(Z["f64_out1_c1"], Z["f64_out0_c1"])         # stopped; the other not started
    a, b = META["windows"][0], META["windows"][1]
    assert META["channels"][0] == META["channels"][1] and all(max(a[2 * k], b[2 * k]) < min(a[2 * k + 1], b[2 * k + 1])
                                                              for k in range(3))


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_emitters_on_gpu_match_reference(tag):
    from aerolume_b200.ns3d.emitters import apply_smoke_sources
    dt = torch.float64 if tag == "f64" else torch.float32
    ch = [torch.as_tensor(Z[f"{tag}_in_c{c}"]).cuda() for c in range(2)]
    src = [SimpleNamespace(window=w, weight=torch.as_tensor(wt).cuda(), params=torch.as_tensor(p).cuda(), channel=c)
           for w, wt, p, c in _sources(tag)]
    for s, t in enumerate(META["times"]):
        apply_smoke_sources(ch, torch.tensor(t, device="cuda", dtype=dt), src)
        torch.cuda.synchronize()
        for c in range(2):
            ref = Z[f"{tag}_out{s}_c{c}"]
            assert np.abs(ch[c].cpu().numpy() - ref).max() <= (1e-15 if tag == "f64" else 1e-7), (s, c)
