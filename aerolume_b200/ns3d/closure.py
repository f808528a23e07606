"""The learned subgrid closure: training data from the plain step's own filtered runs, training
on the tensor cores, and the model the 3D step runs in place of WALE where it applies.

The reference has no learned closure.  What it stands in for is the WALE eddy viscosity of
src/aerolume/solvers/ns3d/core.py:448-482 (``eddy_viscosity3d``; the fused kernel
ns3d/fused.py:102-132), which stays as the per-cell fallback.

* :func:`hit_state` -- a seeded, solenoidal, random-phase velocity field in a periodic 2 pi box
  with the energy spectrum E(k) ~ k^4 exp(-2 (k / k0)^2), scaled to u_rms = 1, sampled on the
  staggered faces (numpy, on the host), then projected by the step's own projection.
* :func:`make_pairs` -- the plain step (``Ns3dPlan`` on the periodic grid, no LES) advanced from
  that state; every ``every`` steps a ``factor``^3 box filter gives, per coarse cell, the
  filtered gradient (by the step's own stencil) and the subgrid stress (``aero_closure_pairs``),
  turned into standardised inputs and targets (``aero_closure_features`` /
  ``aero_closure_normalise``).
* :class:`ClosureModel` -- FP32 master parameters and their BF16 copy, the standardisation
  constants and the training range of the inputs; :meth:`ClosureModel.train` runs Adam steps
  whose forward and backward passes are the tensor-core kernels (``aero_mlp_train_step``).
* ``Ns3dPlan(..., closure=model)`` runs the model inside the step (``AeroNs3dConfig.closure``).

Every computation above runs in the library's CUDA kernels; torch supplies device memory and
random batch indices only.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from .. import _lib
from .._lib import CLOSURE_HIDDEN, CLOSURE_IN, CLOSURE_NPARAM, CLOSURE_OUT, check

# offsets of the flat parameter array (include/aero_b200.h AERO_CLOSURE_NPARAM)
LAYOUT = (("w1", (CLOSURE_HIDDEN, CLOSURE_IN)), ("b1", (CLOSURE_HIDDEN,)),
          ("w2", (CLOSURE_HIDDEN, CLOSURE_HIDDEN)), ("b2", (CLOSURE_HIDDEN,)),
          ("w3", (CLOSURE_HIDDEN, CLOSURE_HIDDEN)), ("b3", (CLOSURE_HIDDEN,)),
          ("w4", (CLOSURE_OUT, CLOSURE_HIDDEN)), ("b4", (CLOSURE_OUT,)))


def param_views(flat):
    """{name: view} of a flat parameter tensor in the library's layout."""
    out, off = {}, 0
    for name, shape in LAYOUT:
        n = int(np.prod(shape))
        out[name] = flat[off:off + n].view(*shape)
        off += n
    assert off == CLOSURE_NPARAM
    return out


def _stream(dev):
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class ClosureModel:
    """The MLP (10 -> 128 -> 128 -> 128 -> 6, SiLU) with its standardisation and input range."""

    def __init__(self, device="cuda", seed=0):
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("the learned closure runs on a CUDA device only (no CPU fallback)")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        g = torch.Generator().manual_seed(seed)
        flat = torch.zeros(CLOSURE_NPARAM, dtype=torch.float32)
        v = param_views(flat)
        for name, shape in LAYOUT:             # uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases
            if name.startswith("w"):
                bound = 1.0 / math.sqrt(shape[1])
                v[name].copy_((torch.rand(shape, generator=g) * 2 - 1) * bound)
        self.params = flat.to(self.device)
        self.params_bf16 = self.params.to(torch.bfloat16)
        self.in_mean = np.zeros(CLOSURE_IN, np.float32)
        self.in_std = np.ones(CLOSURE_IN, np.float32)
        self.in_lo = np.full(CLOSURE_IN, -np.inf, np.float32)
        self.in_hi = np.full(CLOSURE_IN, np.inf, np.float32)
        self.out_mean = np.zeros(CLOSURE_OUT, np.float32)
        self.out_std = np.ones(CLOSURE_OUT, np.float32)
        self.history = []
        self._adam = None
        self._step = 0

    # ------------------------------------------------------------------ ABI
    def cstruct(self):
        m = _lib.ClosureModel()
        m.params, m.params_bf16 = self.params.data_ptr(), self.params_bf16.data_ptr()
        for name in ("in_mean", "in_std", "in_lo", "in_hi", "out_mean", "out_std"):
            arr = getattr(self, name)
            dst = getattr(m, name)
            for q, x in enumerate(arr):
                dst[q] = float(x)
        return m

    def sync_bf16(self):
        """The BF16 copy of the FP32 master parameters (after editing ``params``)."""
        self.params_bf16.copy_(self.params.to(torch.bfloat16))

    # ------------------------------------------------------------------ data
    def fit_normalisation(self, feat, target, valid, sample=1 << 20, margin=0.0):
        """Standardisation constants and input range from (a strided sample of) raw pairs."""
        ok = valid.bool()
        stride = max(1, int(ok.sum().item()) // sample)
        f = feat[ok][::stride].double().cpu().numpy()
        t = target[ok][::stride].double().cpu().numpy()
        self.in_mean = f.mean(0).astype(np.float32)
        self.in_std = np.maximum(f.std(0), 1e-6).astype(np.float32)
        span = f.max(0) - f.min(0)
        self.in_lo = (f.min(0) - margin * span).astype(np.float32)
        self.in_hi = (f.max(0) + margin * span).astype(np.float32)
        self.out_mean = t.mean(0).astype(np.float32)
        self.out_std = np.maximum(t.std(0), 1e-9).astype(np.float32)

    def normalise(self, feat, target=None):
        """Standardised BF16 inputs (n, 16) and FP32 targets (n, 6) on the device."""
        n = feat.shape[0]
        x = torch.empty(n, 16, device=self.device, dtype=torch.bfloat16)
        t = torch.empty(n, CLOSURE_OUT, device=self.device, dtype=torch.float32) if target is not None else None
        m = self.cstruct()
        check(_lib.lib().aero_closure_normalise(n, _p(feat), _p(target), C.byref(m), _p(x), _p(t),
                                                _stream(self.device)), "aero_closure_normalise")
        return x, t

    # ------------------------------------------------------------------ compute
    def forward(self, x):
        """Standardised outputs (n, 6) of standardised BF16 inputs (n, 16), on the tensor cores."""
        n = x.shape[0]
        y = torch.empty(n, CLOSURE_OUT, device=self.device, dtype=torch.float32)
        status = torch.zeros(1, device=self.device, dtype=torch.int32)
        m = self.cstruct()
        check(_lib.lib().aero_mlp_forward(C.byref(m), _p(x), n, _p(y), _p(status), _stream(self.device)),
              "aero_mlp_forward")
        self.last_status = status
        return y

    def gradients(self, x, t, idx):
        """(grad (NPARAM FP32), loss sum) of the batch rows idx, on the tensor cores."""
        batch = int(idx.numel())
        grad = torch.zeros(CLOSURE_NPARAM, device=self.device, dtype=torch.float32)
        loss = torch.zeros(1, device=self.device, dtype=torch.float64)
        ws = self._workspace(batch)
        status = torch.zeros(1, device=self.device, dtype=torch.int32)
        check(_lib.lib().aero_mlp_gradients(_p(self.params), _p(self.params_bf16), _p(grad), _p(x), _p(t), _p(idx),
                                            batch, _p(loss), _p(ws), _p(status), _stream(self.device)),
              "aero_mlp_gradients")
        self.last_status = status
        return grad, loss

    def _workspace(self, batch):
        nb = _lib.lib().aero_mlp_train_workspace_bytes(batch)
        buf = getattr(self, "_ws", None)
        if buf is None or buf.numel() < nb + 256:
            self._ws = torch.empty(nb + 256, device=self.device, dtype=torch.uint8)
        base = self._ws.data_ptr()
        off = (-base) % 256
        return self._ws[off:off + nb]

    def train(self, x, t, steps, batch=65536, lr=1e-3, seed=0, log_every=100):
        """``steps`` Adam steps on random batches of the standardised pairs (x, t); the mean
        squared error of each logged step goes to ``history``."""
        if self._adam is None:
            self._adam = (torch.zeros_like(self.params), torch.zeros_like(self.params), torch.zeros_like(self.params))
        m, v, grad = self._adam
        n = x.shape[0]
        g = torch.Generator(device=self.device).manual_seed(seed)
        loss = torch.zeros(1, device=self.device, dtype=torch.float64)
        status = torch.zeros(1, device=self.device, dtype=torch.int32)
        ws = self._workspace(batch)
        L = _lib.lib()
        for k in range(steps):
            idx = torch.randint(0, n, (batch,), generator=g, device=self.device, dtype=torch.int32)
            self._step += 1
            check(L.aero_mlp_train_step(_p(self.params), _p(self.params_bf16), _p(m), _p(v), _p(grad), _p(x), _p(t),
                                        _p(idx), batch, self._step, float(lr), _p(loss), _p(ws), _p(status),
                                        _stream(self.device)), "aero_mlp_train_step")
            if log_every and (k + 1) % log_every == 0:
                self.history.append((self._step, float(loss.item()) / (log_every * batch * CLOSURE_OUT)))
                loss.zero_()
        if int(status.item()):
            raise RuntimeError(f"a tensor-core wait of the training kernels ran out (status {int(status.item())})")
        return self.history

    def eddy_viscosity(self, grad9, nu_wale, delta):
        """The closure's pass on flat cells: (nu_t, max nu_t, [evaluated, kept WALE])."""
        n = grad9.shape[1]
        nu = nu_wale.clone()
        mx = torch.zeros(1, device=self.device, dtype=torch.float64)
        counts = torch.zeros(2, device=self.device, dtype=torch.int64)
        status = torch.zeros(1, device=self.device, dtype=torch.int32)
        m = self.cstruct()
        check(_lib.lib().aero_closure_eddy_viscosity(C.byref(m), _p(grad9.contiguous()), n, float(delta), _p(nu),
                                                     _p(mx), _p(counts), _p(status), _stream(self.device)),
              "aero_closure_eddy_viscosity")
        self.last_status = status
        return nu, float(mx.item()), counts.tolist()

    # ------------------------------------------------------------------ persistence
    def state(self):
        return {"params": self.params.cpu().numpy(), **{k: getattr(self, k) for k in (
            "in_mean", "in_std", "in_lo", "in_hi", "out_mean", "out_std")}}

    def load(self, st):
        self.params.copy_(torch.as_tensor(np.asarray(st["params"], np.float32)))
        self.sync_bf16()
        for k in ("in_mean", "in_std", "in_lo", "in_hi", "out_mean", "out_std"):
            setattr(self, k, np.asarray(st[k], np.float32))
        return self


# ---------------------------------------------------------------------------------------
# training data
# ---------------------------------------------------------------------------------------

def hit_state(n, *, seed=0, k0=4.0, urms=1.0, device="cuda"):
    """Staggered (u (n, n, n+1), v (n, n+1, n), w (n+1, n, n)) FP32 velocity of decaying
    homogeneous turbulence in the periodic box [0, 2 pi)^3: random phases (seeded), solenoidal
    in the continuum, E(k) ~ k^4 exp(-2 (k / k0)^2), each face component sampled at its face by a
    phase shift, scaled to u_rms = urms (not yet projected onto the discrete divergence-free
    space: the plan's projection does that)."""
    rng = np.random.default_rng(seed)
    h = 2.0 * np.pi / n
    k1 = np.fft.fftfreq(n, 1.0 / n)
    kr = np.fft.rfftfreq(n, 1.0 / n)
    KZ, KY, KX = np.meshgrid(k1, k1, kr, indexing="ij")
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    k = np.sqrt(k2)
    amp = np.zeros_like(k)
    nz = k > 0
    # |u_hat|^2 summed over a shell of radius k (area 4 pi k^2) ~ E(k)
    amp[nz] = np.sqrt(k[nz] ** 4 * np.exp(-2.0 * (k[nz] / k0) ** 2) / (4.0 * np.pi * k2[nz]))
    comps = []
    for _ in range(3):
        comps.append(rng.standard_normal(k.shape) + 1j * rng.standard_normal(k.shape))
    a = np.stack(comps)                                          # (3, n, n, n//2+1)
    kv = np.stack([KX, KY, KZ])
    with np.errstate(invalid="ignore", divide="ignore"):
        proj = (a * kv).sum(0) / np.where(nz, k2, 1.0)
    a = (a - kv * proj) * amp                                    # solenoidal, shaped
    a[:, ~nz] = 0.0
    # face positions: u at (i h, (j + 1/2) h, (k + 1/2) h) etc. relative to the nodes
    shifts = {0: (0.0, 0.5, 0.5), 1: (0.5, 0.0, 0.5), 2: (0.5, 0.5, 0.0)}
    fields = []
    for c in range(3):
        sx, sy, sz = (s * h for s in shifts[c])
        ph = np.exp(1j * (KX * sx + KY * sy + KZ * sz))
        fields.append(np.fft.irfftn(a[c] * ph, s=(n, n, n), axes=(0, 1, 2)))
    rms = math.sqrt(sum(float((f ** 2).mean()) for f in fields) / 3.0)
    fields = [f * (urms / rms) for f in fields]
    u = np.concatenate([fields[0], fields[0][:, :, :1]], axis=2)   # duplicate periodic face
    v = np.concatenate([fields[1], fields[1][:, :1, :]], axis=1)
    w = np.concatenate([fields[2], fields[2][:1, :, :]], axis=0)
    dev = torch.device(device)
    return tuple(torch.as_tensor(np.ascontiguousarray(x, np.float32)).to(dev) for x in (u, v, w))


def hit_plan(n, re=1500.0, cfl=0.5, device="cuda"):
    """The plain step on the periodic 2 pi box, FP32, no LES (the training-data generator)."""
    from .plan import Ns3dPlan
    from .setup import make_ops
    from .types import Geometry3D
    ops = make_ops(n, n, n, 2.0 * np.pi / n, re=re, periodic=True, turbulence="none", cfl=cfl, dtype="float32")
    return ops, Ns3dPlan(ops, Geometry3D((0, 0, 0, 0, 0, 0)), device=device)


def filter_pairs(u, v, w, n, h, factor=4):
    """(g8 (8, m^3), tau (6, m^3)) of one periodic state, m = n / factor (CUDA)."""
    m = n // factor
    cells = m ** 3
    dev = u.device
    g8 = torch.empty(8, cells, device=dev, dtype=torch.float32)
    tau = torch.empty(6, cells, device=dev, dtype=torch.float32)
    work = torch.empty(3 * cells, device=dev, dtype=torch.float32)
    check(_lib.lib().aero_closure_pairs(n, factor, _p(u), _p(v), _p(w), float(h), _p(g8), _p(tau), _p(work),
                                        _stream(dev)), "aero_closure_pairs")
    return g8, tau


def features(g8, delta, tau=None):
    """(feat (n, 10), scale (n), valid (n) uint8, target (n, 6) or None) of gradients (CUDA)."""
    n = g8.shape[1]
    dev = g8.device
    feat = torch.empty(n, CLOSURE_IN, device=dev, dtype=torch.float32)
    scale = torch.empty(n, device=dev, dtype=torch.float32)
    valid = torch.empty(n, device=dev, dtype=torch.uint8)
    target = torch.empty(n, CLOSURE_OUT, device=dev, dtype=torch.float32) if tau is not None else None
    check(_lib.lib().aero_closure_features(n, _p(g8.contiguous()), float(delta), _p(tau), _p(feat), _p(scale),
                                           _p(valid), _p(target), _stream(dev)), "aero_closure_features")
    return feat, scale, valid, target


def make_pairs(n=384, *, factor=4, re=1500.0, seed=0, spinup=400, snapshots=8, every=50, device="cuda"):
    """Training pairs of the decaying-turbulence runs: (feat, target, valid) concatenated over
    the snapshots taken every ``every`` steps after ``spinup`` steps, plus the run's record."""
    ops, plan = hit_plan(n, re=re, device=device)
    u, v, w = hit_state(n, seed=seed, device=device)
    plan.project(u, v, w)
    t = torch.zeros((), device=plan.device, dtype=torch.float32)
    out = plan.empty_fields()
    out["u"], out["v"], out["w"] = u, v, w
    h = 2.0 * np.pi / n
    feats, targets, valids, record = [], [], [], []
    total = spinup + (snapshots - 1) * every
    for step in range(1, total + 1):
        plan.step(u, v, w, t, out=out)
        t.copy_(out["t"])
        if step >= spinup and (step - spinup) % every == 0:
            g8, tau = filter_pairs(u, v, w, n, h, factor)
            f, _, ok, tg = features(g8, factor * h, tau)
            feats.append(f)
            targets.append(tg)
            valids.append(ok)
            ke = 0.5 * float((u[..., :-1].double() ** 2).mean() + (v[:, :-1].double() ** 2).mean()
                             + (w[:-1].double() ** 2).mean())
            record.append({"step": step, "t": float(t), "kinetic_energy": ke})
    if plan.status():
        raise RuntimeError(f"the data-generation run reported status {plan.status()}")
    return torch.cat(feats), torch.cat(targets), torch.cat(valids), record


__all__ = ["ClosureModel", "features", "filter_pairs", "hit_plan", "hit_state", "make_pairs", "param_views"]
