"""The C-ABI library loads and exports every symbol include/aero_b200.h declares (no GPU needed)."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import pytest

from aerolume_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    text = (ROOT / "include" / "aero_b200.h").read_text()
    return sorted(set(re.findall(r"\b(aero_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert sorted(_lib.EXPORTS) == _declared()


def test_library_loads_and_exports_everything():
    L = _lib.lib()
    for name in _declared():
        assert hasattr(L, name), name
    assert L.aero_abi_version() == _lib.ABI_VERSION


def test_plan_validation_errors_are_reported():
    L = _lib.lib()
    cfg = _lib.Ns3dConfig()
    cfg.abi_version = _lib.ABI_VERSION
    cfg.nx, cfg.ny, cfg.nz, cfg.h = 2, 8, 8, 0.1                 # too small
    h = C.c_void_p()
    rc = L.aero_ns3d_plan_create(C.byref(cfg), C.byref(h))
    assert rc == -1 and b"4 x 4 x 4" in L.aero_last_error()
    cfg.nx = 16
    cfg.eta, cfg.nbody = 1.0, 9
    rc = L.aero_ns3d_plan_create(C.byref(cfg), C.byref(h))
    assert rc == -2 and b"bodies" in L.aero_last_error()
    with pytest.raises(RuntimeError, match="unsupported"):
        _lib.check(rc, "plan")


def test_plan_create_and_workspace_size_on_host():
    """Plan creation is host-only: a valid config gives a plan and a workspace size."""
    from aerolume_b200.ns3d.setup import make_ops
    L = _lib.lib()
    cfg = _lib.Ns3dConfig()
    cfg.abi_version = _lib.ABI_VERSION
    cfg.nx, cfg.ny, cfg.nz, cfg.h, cfg.eta, cfg.cfl, cfg.nu = 24, 12, 10, 1 / 6, 0.01, 0.5, 1e-3
    ops = make_ops(24, 12, 10, 1 / 6, re=1e3)
    for c, comp in enumerate("uvw"):
        for a in range(3):
            for s in range(2):
                cfg.ghost_kind[c][a][s] = _lib.GHOST[ops.ghost[comp][a][s][0]]
    h = C.c_void_p()
    assert L.aero_ns3d_plan_create(C.byref(cfg), C.byref(h)) == 0
    n = L.aero_ns3d_workspace_bytes(h)
    cells = 24 * 12 * 10
    assert n > 6 * cells * 4
    L.aero_ns3d_plan_destroy(h)
