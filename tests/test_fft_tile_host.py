"""The Poisson solve's compile-time FFT tile (aerolume_b200/csrc/fft_tile.cuh; lengths 2^a and
3 * 2^a) executed on the CPU through tests/native/fft_tile_host.cpp -- the same phases the GPU
runs, thread by thread -- against scipy's orthonormal DCT-II / DCT-III and the discrete Hartley transform
that Aerolume's Poisson bases define (ns3d/poisson.py:74-90)."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest
import scipy.fft as sf

ROOT = Path(__file__).resolve().parents[1]
SRC = Path(__file__).resolve().parent / "native" / "fft_tile_host.cpp"

# relative to max |output|: FP64 to round-off, FP32 to the solver's FP32 tolerance
TOL = {"f64": 1e-13, "f32": 2e-6}


def _lines(n, e):
    l = (48 * 1024) // (3 * e * n)
    l = min(64, max(2, l))
    return 1 << (l.bit_length() - 1)


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ is not available")
    exe = tmp_path_factory.mktemp("fft") / "fft_tile_host"
    subprocess.run([gxx, "-std=c++17", "-O2", "-I", str(ROOT / "aerolume_b200" / "csrc"), str(SRC), "-o", str(exe)],
                   check=True)
    return exe


def _run(exe, prec, n, kind, inverse, x, narrow=False):
    r = subprocess.run([str(exe), prec, str(n), str(kind), str(int(inverse)), str(int(narrow))],
                       input=x.astype(np.float64).tobytes(), capture_output=True, check=True)
    return np.frombuffer(r.stdout, dtype=np.float64).reshape(x.shape)


def _want(x, kind, inverse):
    if kind == 0:
        return sf.idct(x, type=2, norm="ortho", axis=0) if inverse else sf.dct(x, type=2, norm="ortho", axis=0)
    f = np.fft.fft(x, axis=0)
    return (f.real - f.imag) / np.sqrt(x.shape[0])


@pytest.mark.parametrize("narrow", [False, True], ids=["wide", "two_lines"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("n", [8, 16, 32, 64, 128, 256, 512, 1024, 2048, 12, 24, 48, 96, 192, 384, 768, 1536])
def test_tile_transform_matches_orthonormal_bases(harness, prec, n, narrow):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, 2 if narrow else _lines(n, 8 if prec == "f64" else 4)))
    if prec == "f32":
        x = x.astype(np.float32).astype(np.float64)
    for kind in (0, 1):
        for inverse in (False, True):
            got = _run(harness, prec, n, kind, inverse, x, narrow)
            want = _want(x, kind, inverse)
            err = np.abs(got - want).max() / np.abs(want).max()
            assert err < TOL[prec], (n, kind, inverse, err)
