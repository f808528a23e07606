"""The learned closure's CUDA kernels against plain FP32 references: the tensor-core MLP forward
and backward against torch (the same network in FP32 with its operands rounded to BF16), the
filter and features against the numpy oracle, the closure's eddy viscosity against the oracle's
fallback logic, and the closure inside the 3D step."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import closure3d as OC

pytestmark = pytest.mark.gpu


def _model(seed=0):
    from aerolume_b200.ns3d.closure import ClosureModel
    return ClosureModel(seed=seed)


def _inputs(n, seed=1):
    g = torch.Generator().manual_seed(seed)
    x = torch.zeros(n, 16)
    x[:, :10] = torch.randn(n, 10, generator=g)
    return x.to("cuda", torch.bfloat16)


def _torch_mlp(params, x):
    """The network in FP32 with BF16 weights and layer inputs (differentiable)."""
    from aerolume_b200.ns3d.closure import param_views
    v = param_views(params)
    bf = lambda a: a.to(torch.bfloat16).to(torch.float32)   # noqa: E731
    h = x[:, :10].to(torch.float32)
    for q in (1, 2, 3):
        z = bf(h @ bf(v[f"w{q}"]).T + v[f"b{q}"])
        # SiLU in BF16 arithmetic, as the kernels form it: z (1 + tanh(z / 2)) / 2
        h = bf(z * bf(0.5 * bf(torch.tanh(0.5 * z)) + 0.5))
    return h @ bf(v["w4"]).T + v["b4"]


def test_mlp_forward_matches_fp32_reference():
    """n = 1000 rows (a partial last tile of 128): tcgen05 BF16 x BF16 -> FP32 against torch."""
    m = _model(3)
    x = _inputs(1000)
    y = m.forward(x)
    torch.cuda.synchronize()
    assert int(m.last_status.item()) == 0
    ref = _torch_mlp(m.params, x)
    err = (y - ref).abs().max().item() / ref.abs().max().item()
    assert err < 3e-2, err
    # the same rows in another tile position give the same outputs (row independence)
    y2 = m.forward(x[128:256].contiguous())
    assert torch.equal(y2, y[128:256])


def test_mlp_gradients_match_autograd():
    """Gradients of the batch's mean squared error, forward and backward on the tensor cores,
    against torch autograd of the FP32 reference (bias gradients through the ones columns of the
    weight-gradient GEMM, layer 4's with shuffles)."""
    from aerolume_b200.ns3d.closure import param_views
    m = _model(5)
    n, batch = 2048, 384
    x = _inputs(n, 7)
    gt = torch.Generator().manual_seed(8)
    t = torch.randn(n, 6, generator=gt).cuda()
    idx = torch.randint(0, n, (batch,), generator=torch.Generator().manual_seed(9), dtype=torch.int32).cuda()
    grad, loss = m.gradients(x, t, idx)
    torch.cuda.synchronize()
    assert int(m.last_status.item()) == 0
    p = m.params.clone().requires_grad_(True)
    y = _torch_mlp(p, x[idx.long()])
    ref_loss = ((y - t[idx.long()]) ** 2).mean()
    ref_loss.backward()
    assert abs(loss.item() / (batch * 6) - ref_loss.item()) <= 2e-2 * ref_loss.item()
    gv, rv = param_views(grad), param_views(p.grad)
    for name in ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4"):
        a, b = gv[name], rv[name]
        err = (a - b).abs().max().item() / max(b.abs().max().item(), 1e-12)
        assert err < 6e-2, (name, err)


def test_training_fits_a_smooth_map():
    """300 Adam steps on the tensor-core kernels bring the error of a smooth synthetic map well
    below its starting value."""
    m = _model(11)
    n = 65536
    g = torch.Generator().manual_seed(12)
    x = torch.zeros(n, 16)
    x[:, :10] = torch.rand(n, 10, generator=g) * 2 - 1
    A = torch.randn(6, 10, generator=g) / 3
    t = torch.tanh(x[:, :10] @ A.T) + 0.1 * torch.sin(3 * x[:, :1])
    x, t = x.to("cuda", torch.bfloat16), t.cuda()
    hist = m.train(x, t, 300, batch=4096, lr=2e-3, log_every=50)
    first, last = hist[0][1], hist[-1][1]
    assert last < 0.2 * first, hist
    assert np.isfinite(last)


def test_filter_pairs_and_features_match_oracle():
    from aerolume_b200.ns3d.closure import features, filter_pairs, hit_state
    n, F = 32, 4
    h = 2 * np.pi / n
    u, v, w = hit_state(n, seed=4)
    g8, tau = filter_pairs(u, v, w, n, h, F)
    torch.cuda.synchronize()
    rg, rt = OC.filter_pairs(u.cpu().numpy(), v.cpu().numpy(), w.cpu().numpy(), n, h, F)
    assert np.abs(g8.cpu().numpy() - rg).max() <= 1e-5 * np.abs(rg).max()
    assert np.abs(tau.cpu().numpy() - rt).max() <= 1e-5 * np.abs(rt).max()
    feat, scale, valid, target = features(g8, F * h, tau)
    rf, rs, rv, rtg = OC.features(g8.cpu().numpy(), F * h, tau.cpu().numpy())
    assert np.array_equal(valid.cpu().numpy().astype(bool), rv)
    assert np.abs(feat.cpu().numpy() - rf).max() <= 1e-5
    assert np.abs(scale.cpu().numpy() - rs).max() <= 1e-5 * rs.max()
    assert np.abs(target.cpu().numpy() - rtg)[rv].max() <= 1e-4 * np.abs(rtg[rv]).max()


def _grad_cells(n, seed):
    g = np.random.default_rng(seed)
    g8 = g.normal(size=(8, n)) * np.exp(g.normal(size=n))
    g8[:, :5] = 0.0                                        # |g| = 0: no features
    g8[:, 5:9] *= 1e-12
    fac = np.where(g.random(n) < 0.1, g.random(n), 1.0)
    return g8, fac


def test_closure_eddy_viscosity_matches_oracle():
    """The closure's pass: nu_t of the learned stress where the dissipation is positive and the
    inputs are inside the training range, WALE's value elsewhere, against the oracle with the
    FP32 reference network."""
    from aerolume_b200.ns3d.closure import features
    m = _model(21)
    n = 50_000
    g8, fac = _grad_cells(n, 22)
    grad9 = torch.as_tensor(np.vstack([g8, fac[None]]), dtype=torch.float32).cuda()
    nu_wale = torch.rand(n, generator=torch.Generator().manual_seed(23)).cuda() * 1e-3
    feat, _, valid, _ = features(grad9[:8].contiguous(), 0.05)
    m.fit_normalisation(feat, torch.zeros(n, 6, device="cuda"), valid)
    m.out_mean[:] = 0.0
    m.out_std[:] = 0.05
    # a tighter range on two inputs, so the range test is exercised
    m.in_lo[8], m.in_hi[8] = -0.5, 0.5
    nu, mx, counts = m.eddy_viscosity(grad9, nu_wale, 0.05)
    torch.cuda.synchronize()
    assert int(m.last_status.item()) == 0
    f, _, ok, _ = OC.features(g8.astype(np.float32).astype(np.float64), 0.05)
    x = np.where(ok[:, None], (f - m.in_mean) / m.in_std, 0.0)
    y = OC.mlp(m.params.cpu().numpy(), x, _layout())
    ref, used, scale = OC.eddy_viscosity(y, g8.astype(np.float32), fac.astype(np.float32), nu_wale.cpu().numpy(),
                                         0.05, m.out_mean, m.out_std, m.in_lo, m.in_hi)
    got = nu.cpu().numpy()
    kept = got == nu_wale.cpu().numpy()
    agree = (kept == ~used).mean()
    assert agree > 0.995, agree                            # borderline dissipation signs may flip
    both = used & ~kept
    assert both.sum() > 0.2 * n and (~used).sum() > 0.05 * n
    # BF16 operands: nu within a few per cent of the scale of the dissipation's terms (the
    # dissipation itself can be a small difference of them), and of nu itself at the median
    rel = np.abs(got[both] - ref[both]) / scale[both]
    assert np.quantile(rel, 0.99) < 5e-2, np.quantile(rel, 0.99)
    assert np.median(np.abs(got[both] - ref[both]) / np.abs(ref[both])) < 1e-2
    assert counts[0] == n and abs(counts[1] - int(kept.sum())) <= 0
    assert abs(mx - got.max()) <= 1e-6 * got.max()


def _layout():
    from aerolume_b200.ns3d.closure import LAYOUT
    return LAYOUT


def _box_plans(closure):
    from aerolume_b200.ns3d.plan import Ns3dPlan
    from aerolume_b200.ns3d.workloads import box_on_moving_floor, initial_state
    ops, geom, th, src, _ = box_on_moving_floor(80, 40, 40, dtype="float32", seed=5)
    plan_w = Ns3dPlan(ops, geom, th, src, smoke=True)
    plan_c = Ns3dPlan(ops, geom, th, src, smoke=True, closure=closure)
    u, v, w = initial_state(ops, seed=5, noise=0.05)
    plan_w.project(u, v, w)
    theta = torch.zeros(40, 40, 80, device="cuda")
    dye = torch.zeros(40, 40, 80, device="cuda")
    t0 = torch.zeros((), device="cuda")
    return plan_w, plan_c, (u, v, w, t0, theta, dye)


def test_closure_with_an_empty_training_range_is_the_wale_step():
    """A model whose input range is empty falls back everywhere: the closure step is the plain
    WALE step bit for bit, and the counts say every cell kept WALE."""
    m = _model(31)
    m.in_lo[:] = 1.0
    m.in_hi[:] = -1.0
    plan_w, plan_c, (u, v, w, t0, theta, dye) = _box_plans(m)
    a = plan_w.step(u, v, w, t0, theta0=theta, dye0=dye)
    b = plan_c.step(u, v, w, t0, theta0=theta, dye0=dye)
    torch.cuda.synchronize()
    for k in ("u", "v", "w", "p", "theta", "dye", "dt", "coeffs"):
        assert torch.equal(a[k], b[k]), k
    ev, wale = plan_c.closure_counts()
    assert ev == 3 * 82 * 42 * 42 and wale == ev
    assert plan_c.status() == 0


def test_closure_step_uses_the_model():
    """With a model whose range covers the flow, part of the cells take the learned nu_t: the
    step stays finite with a clean status and differs from the WALE step."""
    from aerolume_b200.ns3d.closure import ClosureModel
    m = ClosureModel(seed=41)
    m.out_std[:] = 0.02
    plan_w, plan_c, (u, v, w, t0, theta, dye) = _box_plans(m)
    a = plan_w.step(u, v, w, t0, theta0=theta, dye0=dye)
    b = plan_c.step(u, v, w, t0, theta0=theta, dye0=dye)
    torch.cuda.synchronize()
    assert plan_c.status() == 0
    for k in ("u", "v", "w", "p", "theta", "dye"):
        assert torch.isfinite(b[k]).all(), k
    ev, wale = plan_c.closure_counts()
    assert 0 < wale < ev
    assert not torch.equal(a["u"], b["u"])


def test_closure_through_the_seam():
    """The drop-in handle carries the model (``kern.closure``): its WALE step then runs the
    closure -- bit for bit the plain step when the model's range is empty, as above -- and a
    plan without it is kept apart in the cache."""
    from types import SimpleNamespace

    from aerolume_b200.ns3d.fused import fast_step_phys, load_kernels
    from aerolume_b200.ns3d.types import State3D
    from aerolume_b200.ns3d.workloads import box_on_moving_floor, initial_state
    ops, geom, th, _, _ = box_on_moving_floor(64, 32, 32, dtype="float32", seed=7)
    u, v, w = initial_state(ops, seed=7, noise=0.05)
    kern = load_kernels("upwind3", torch.device("cuda"), torch.float32)
    kern.plan_for(geom, ops, SimpleNamespace(thermal=th)).project(u, v, w)
    st = State3D(u, v, w, torch.zeros(32, 32, 64, device="cuda"), torch.zeros((), device="cuda"),
                 torch.zeros((), device="cuda"))
    theta = torch.zeros(32, 32, 64, device="cuda")
    phys = SimpleNamespace(thermal=th, paint=None, pid=None, fans=None, ports=None, u_floor=0.0)
    plain = fast_step_phys(st, geom, ops, kern, phys=phys, theta=theta)
    m = _model(51)
    m.in_lo[:] = 1.0
    m.in_hi[:] = -1.0
    kern.closure = m
    learned = fast_step_phys(st, geom, ops, kern, phys=phys, theta=theta)
    torch.cuda.synchronize()
    for a, b in ((plain.state.u, learned.state.u), (plain.state.p, learned.state.p), (plain.theta, learned.theta)):
        assert torch.equal(a, b)
    plan = kern.plan_for(geom, ops, phys)
    assert plan.closure is m
    ev, wale = plan.closure_counts()
    assert ev > 0 and wale == ev
