"""The bookkeeping oracle against the reference's own FlowSolver3D._record / _welford
(tests/golden/record3d.npz: five seeded steps, the history ring wrapping, FP64 and FP32)."""
from __future__ import annotations

import numpy as np
import pytest

from _golden import GOLDEN
from oracle import record3d as R

Z = np.load(GOLDEN / "record3d.npz")
CAP = int(Z["capacity"])


def _buffers(tag, dt):
    shapes = {k: Z[f"{tag}_in0_field_{k}"].shape for k in "uvwpt"}
    avg = {"time": np.float64(0), "pending": np.float64(0)}
    for k, s in shapes.items():
        avg[k], avg[k + "2"] = np.zeros(s, dt), np.zeros(s, dt)
    return {"hist": np.zeros((CAP, 7), dt), "hist_n": int(Z[f"{tag}_hist_n0"]), "body_c": np.zeros((2, 6), dt),
            "phist": np.zeros((CAP, 5), dt), "avg": avg}


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_oracle_bookkeeping_matches_reference(tag):
    dt = np.float64 if tag == "f64" else np.float32
    tol = 1e-14 if tag == "f64" else 1e-6
    buf = _buffers(tag, dt)
    for step in range(5):
        f = {k: Z[f"{tag}_in{step}_field_{k}"] for k in "uvwpt"}
        R.record(buf, Z[f"{tag}_in{step}_t"], Z[f"{tag}_in{step}_dt"], Z[f"{tag}_in{step}_bc"],
                 bool(Z[f"{tag}_in{step}_sample"]), fields=f, extra=Z[f"{tag}_in{step}_extra"])
        rows = Z[f"{tag}_out{step}_hist_rows"]
        assert buf["hist_n"] == int(Z[f"{tag}_out{step}_hist_n"])
        assert np.abs(buf["hist"][rows] - Z[f"{tag}_out{step}_hist"]).max() <= tol * 10
        assert np.abs(buf["phist"][rows] - Z[f"{tag}_out{step}_phist"]).max() == 0
        assert buf["avg"]["time"] == float(Z[f"{tag}_out{step}_time"])
        assert buf["avg"]["pending"] == float(Z[f"{tag}_out{step}_pending"])
        for k in "uvwpt":
            for name, got in (("mean", buf["avg"][k]), ("m2", buf["avg"][k + "2"])):
                ref = Z[f"{tag}_out{step}_{name}_{k}"]
                assert np.abs(got - ref).max() <= tol * max(np.abs(ref).max(), 1.0), (step, name, k)


def test_fixture_wraps_the_ring_and_samples():
    """The fixture exercises the wrap (counter from capacity - 2) and both kinds of step."""
    assert int(Z["f64_hist_n0"]) == CAP - 2 and int(Z["f64_out4_hist_n"]) == CAP + 3
    assert list(Z["f64_out4_hist_rows"]) == [2, 1, 0]
    assert [bool(Z[f"f64_in{s}_sample"]) for s in range(5)] == [False, True, False, True, False]
    assert np.abs(Z["f64_out1_mean_u"]).max() > 0 and float(Z["f64_out4_pending"]) > 0
