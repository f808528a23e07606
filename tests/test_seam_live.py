"""Live edits through the drop-in seams: a Reynolds-number change between steps reaches the
B200 step, in 3D through a new plan (the reference re-captures its graphs,
ns3d/solver.py:1643-1657) and in 2D through the device scalars the reference fills in place
under a live CUDA graph (ns2d/core.py:167-176, ns2d/solver.py:1040-1048); the plan caches stay
bounded."""
from __future__ import annotations

import dataclasses
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from _golden import load_case, load_case2d, thermal2d_from_case
from oracle import ns2d as O2
from oracle import ns3d as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.detach().double().cpu().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _dev(x, dt=torch.float64):
    x = np.asarray(x)
    return torch.as_tensor(np.ascontiguousarray(x).reshape(x.shape)).to("cuda", dt).contiguous()


def _set_re_3d(ops, th, re):
    """What set_reynolds (core.py:140-144) and ThermalOps.set_reynolds (physics.py:580-586)
    change, for the B200 containers: nu, eta, Pe, kappa, the thermal eta."""
    from aerolume_b200.ns3d.setup import auto_eta, auto_eta_thermal
    prandtl = th.pe * ops.nu_value          # Pr = Pe / Re
    ops.nu_value = 1.0 / re
    ops.eta = auto_eta(ops.h, re)
    th.pe = re * prandtl
    th.kappa = 1.0 / th.pe
    th.eta = auto_eta_thermal(ops.h, th.pe)


def test_3d_seam_follows_set_reynolds_between_steps():
    from aerolume_b200.ns3d.fused import fast_step_phys, load_kernels
    from aerolume_b200.ns3d.types import State3D
    meta, ops, geom, th, src, arr = load_case("tunnel_wale_heat_smoke_f64")
    kern = load_kernels("upwind3", torch.device("cuda"), torch.float64)
    phys = SimpleNamespace(thermal=th, paint=None, pid=None, fans=None, ports=None, u_floor=0.0)
    z = lambda shape: torch.zeros(shape, device="cuda", dtype=torch.float64)   # noqa: E731
    st = State3D(_dev(arr["in_u"]), _dev(arr["in_v"]), _dev(arr["in_w"]), z(arr["in_u"].shape[:2] + (ops.nx,)),
                 _dev(arr["in_t"]), z(()))
    theta = _dev(arr["in_theta"])
    first = fast_step_phys(st, geom, ops, kern, phys=phys, theta=theta)
    assert _rel(first.state.u, arr["out1_u"]) < 1e-10
    # live change of Re, then the next step from the same inputs: the oracle at the new Re
    ops_new, th_new = dataclasses.replace(ops), dataclasses.replace(th)
    _set_re_3d(ops_new, th_new, 2500.0)
    _set_re_3d(ops, th, 2500.0)
    second = fast_step_phys(st, geom, ops, kern, phys=phys, theta=theta)
    torch.cuda.synchronize()
    ps = O.PoissonSolver3D(ops.nx, ops.ny, ops.nz, ops.h, ops.periodic_axes, np.float64)
    r = O.step3d_phys(arr["in_u"], arr["in_v"], arr["in_w"], np.float64(arr["in_t"]), geom, ops_new, ps, th=th_new,
                      theta=arr["in_theta"])
    for f, ref in (("u", r.u), ("v", r.v), ("w", r.w), ("p", r.p)):
        assert _rel(getattr(second.state, f), ref) < 1e-10, f
    assert _rel(second.theta, r.theta) < 1e-10
    assert _rel(r.u, arr["out1_u"]) > 1e-6            # the change is visible at all
    # one more change and back: at most `keep` step plans stay cached
    _set_re_3d(ops, th, 4000.0)
    fast_step_phys(st, geom, ops, kern, phys=phys, theta=theta)
    assert sum(1 for k in kern._plans if k[0] == "step") <= kern.keep


def test_2d_seam_follows_set_reynolds_inside_a_captured_graph():
    """The reference's 2D solver keeps its graphs across set_inflow; the B200 step reads
    ops.nu, ops.eta, phys.kappa and phys.eta_t from the device at every launch, so the same
    captured graph replayed after the in-place change gives the step at the new Re."""
    from aerolume_b200.ns2d import step as seam
    meta, ops, geom, arr = load_case2d("cylinder_heated_f64")
    tp = thermal2d_from_case(meta, arr)
    dt = torch.float64
    # the reference's objects hold these as 0-d device tensors
    ops_dev = dataclasses.replace(ops)
    ops_dev.nu = torch.tensor(ops.nu, device="cuda", dtype=dt)
    ops_dev.eta = torch.tensor(ops.eta, device="cuda", dtype=dt)
    geom.thermal = SimpleNamespace(chi_t=tp.chi_t, a_t=tp.a_t, w_t=tp.w_t, ins_u=tp.ins_u, ins_v=tp.ins_v,
                                   q_skin=tp.q_skin, w_f=tp.w_f, vol_u=tp.vol_u, vol_v=tp.vol_v,
                                   temp_ids=tp.temp_ids, flux_ids=tp.flux_ids)
    ops_dev.phys = SimpleNamespace(thermal=True, kappa=torch.tensor(tp.kappa, device="cuda", dtype=dt), ri=tp.ri,
                                   prt=tp.prt, gravity=tp.gravity, eta_t=torch.tensor(tp.eta_t, device="cuda", dtype=dt),
                                   theta_in=tp.theta_in, wall_modes=tp.wall_modes, wall_values=tp.wall_values,
                                   diff_coef=tp.diff_coef, heat=None, ports=None, paint=False, nfan=0, n_dye=0,
                                   comb=False, pid=False)
    state = seam.State(_dev(arr["in_u"]), _dev(arr["in_v"]), None, None, _dev(arr["in_t"]), None,
                       _dev(arr["in_theta"]))
    seam.step_full(state, geom, ops_dev)            # warm-up (plan creation) outside the capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s), torch.cuda.graph(g, stream=s):
        new, coeffs = seam.step_full(state, geom, ops_dev)
    torch.cuda.current_stream().wait_stream(s)
    g.replay()
    torch.cuda.synchronize()
    assert _rel(new.u, arr["out1_u"]) < 1e-10
    # set_reynolds in place (core.py:167-176): nu, eta, kappa, eta_t
    re2, pr = 60.0, ops.nu / tp.kappa       # Pr = Pe / Re = nu / kappa
    nu2, eta2 = 1.0 / re2, 0.5 * ops.eta
    kappa2, eta_t2 = 1.0 / (re2 * pr), 0.7 * tp.eta_t
    ops_dev.nu.fill_(nu2)
    ops_dev.eta.fill_(eta2)
    ops_dev.phys.kappa.fill_(kappa2)
    ops_dev.phys.eta_t.fill_(eta_t2)
    g.replay()
    torch.cuda.synchronize()
    ops2 = dataclasses.replace(ops, nu=nu2, eta=eta2)
    tp2 = dataclasses.replace(tp, kappa=kappa2, eta_t=eta_t2)
    ps = O2.PoissonSolver2D(ops.nx, ops.ny, ops.h, ops.periodic, np.float64)
    r = O2.step2d_thermal(arr["in_u"], arr["in_v"], np.float64(arr["in_t"]), arr["in_theta"], geom, ops2, ps, tp2)
    for f, ref in (("u", r.u), ("v", r.v), ("p", r.p)):
        assert _rel(getattr(new, f), ref) < 1e-10, (f, _rel(getattr(new, f), ref))
    assert _rel(new.theta, r.theta) < 1e-10
    assert _rel(r.u, arr["out1_u"]) > 1e-6
    del g


def test_2d_seam_cache_is_bounded_per_solver():
    from aerolume_b200.ns2d import step as seam
    meta, ops, geom, arr = load_case2d("cylinder_upwind_f64")
    state = seam.State(_dev(arr["in_u"]), _dev(arr["in_v"]), None, None, _dev(arr["in_t"]), None)
    for _ in range(4):   # four set_bodies that each build a new geometry object
        seam.step_full(state, dataclasses.replace(geom), ops)
    assert len(seam._PLANS[id(ops)]) <= seam._KEEP
    key = id(ops)
    del ops
    import gc
    gc.collect()
    assert key not in seam._PLANS
