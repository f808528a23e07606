"""aero_ns3d_poisson_solve_static (the allocation-free Poisson solve whose transform tables live
in a static device array) against aero_ns3d_poisson_solve with a workspace, through the C ABI.

Named so that pytest collects it last; it passes alone in a fresh process as well, where its
first call is the one that looks up the static array's device address."""
from __future__ import annotations

import ctypes as C

import pytest
import torch

pytestmark = pytest.mark.gpu

# the Poisson tolerances of the golden tests, relative to max |psi|
TOL = {torch.float64: 1e-12, torch.float32: 2e-6}


def _plan(nx, ny, nz, h, per, dtype):
    from aerolume_b200.ns3d.plan import Ns3dPlan
    from aerolume_b200.ns3d.setup import make_ops
    from aerolume_b200.ns3d.types import Geometry3D
    ops = make_ops(nx, ny, nz, h, re=100.0, periodic=all(per), bc_y="periodic" if per[1] and not all(per) else "slip",
                   dtype=dtype)
    ops.periodic_axes = tuple(per)
    return Ns3dPlan(ops, Geometry3D((0, 0, 0, 0, 0, 0)))


def _static_solve(plan, f):
    from aerolume_b200 import _lib
    psi = torch.full_like(f, float("nan"))
    rc = _lib.lib().aero_ns3d_poisson_solve_static(plan._handle, C.c_void_p(f.data_ptr()), C.c_void_p(psi.data_ptr()),
                                                   C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc, psi


def _rhs(shape, dtype, seed):
    f = torch.randn(*shape, dtype=torch.float64, generator=torch.Generator().manual_seed(seed))
    return (f - f.mean()).to("cuda", dtype)


def test_static_scratch_solve_matches_workspace_solve_on_two_calls_in_a_row():
    # two different grids, precisions and boundary mixes back to back: the second call must
    # not see anything the first one left in the shared static array
    cases = [((64, 32, 32), (False, True, False), "float64", 1),
             ((48, 40, 36), (True, False, False), "float32", 2)]
    for (nx, ny, nz), per, dtype, seed in cases:
        plan = _plan(nx, ny, nz, 0.05, per, dtype)
        f = _rhs((nz, ny, nx), plan.dtype, seed)
        want = plan.poisson_solve(f)
        rc, got = _static_solve(plan, f)
        torch.cuda.synchronize()
        assert rc == 0, rc
        assert torch.isfinite(got).all()
        err = ((got - want).abs().max() / want.abs().max()).item()
        assert err < TOL[plan.dtype], ((nx, ny, nz), dtype, err)


def test_static_scratch_matches_the_reference_solves():
    """The reference's own Poisson solves (tests/golden/poisson3d.npz: odd shapes, every
    boundary mix, dense and FFT axes) through the static-scratch entry point."""
    import numpy as np
    from pathlib import Path
    z = np.load(Path(__file__).resolve().parent / "golden" / "poisson3d.npz")
    h = float(z["h"])
    for dtype, tdt in (("float64", torch.float64), ("float32", torch.float32)):
        for n in range(int(z["count"])):
            nx, ny, nz, px, py, pz = (int(x) for x in z[f"meta{n}"])
            plan = _plan(nx, ny, nz, h, (bool(px), bool(py), bool(pz)), dtype)
            rc, got = _static_solve(plan, torch.as_tensor(z[f"f{n}"]).to("cuda", tdt))
            torch.cuda.synchronize()
            assert rc == 0, rc
            ref = z[f"psi{n}"]
            err = np.abs(got.double().cpu().numpy() - ref).max() / np.abs(ref).max()
            assert err < TOL[tdt], (n, dtype, err)


def test_static_scratch_solve_with_tables_256_bytes_below_its_size():
    """A dense 358-cell x axis in FP64 (its 358 x 358 matrix and the other tables come to
    1,048,320 of the 1,048,576 bytes): the tables packed up to the array's end."""
    plan = _plan(358, 8, 8, 0.05, (False, False, False), "float64")
    f = _rhs((8, 8, 358), plan.dtype, 3)
    want = plan.poisson_solve(f)
    rc, got = _static_solve(plan, f)
    torch.cuda.synchronize()
    assert rc == 0, rc
    err = ((got - want).abs().max() / want.abs().max()).item()
    assert err < TOL[plan.dtype], err


def test_static_scratch_rejects_grids_beyond_its_size():
    from aerolume_b200 import _lib
    plan = _plan(1000, 8, 8, 0.05, (False, False, False), "float64")  # dense x axis: 8 MB of tables
    f = torch.zeros(8, 8, 1000, dtype=torch.float64, device="cuda")
    rc, _ = _static_solve(plan, f)
    assert rc == -1
    assert b"static scratch holds" in _lib.lib().aero_last_error()
