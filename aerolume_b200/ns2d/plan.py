"""One 2D configuration bound to the C ABI: constants, device masks and the workspace.

:class:`Ns2dPlan` reads the reference's 2D objects by attribute (``Ops`` and ``Geometry`` of
src/aerolume/solvers/ns2d/core.py:67-108 and geometry.py:160-182, or the containers of
:mod:`aerolume_b200.ns2d.types`), turns the boundary types into the ghost-cell rules of
core.py:271-325, uploads the window masks once and owns the device workspace.  Heat
transfer comes from ``thermal=`` (a :class:`~aerolume_b200.ns2d.types.Thermal2D`) or from the
reference's ``ops.phys`` with ``geom.thermal``; fans, heaters, painted obstacles, jets and
vents, smoke channels with emitters and smoking jets and the PID step come from ``placed=`` (a
:class:`~aerolume_b200.ns2d.types.Placed2D`) or from ``ops.phys`` itself; ``ops.wall_model``
adds the Werner-Wengle wall shear and ``ops.forcing`` a uniform body force.  There is no
fallback to a CPU or plain-torch path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .. import _lib
from .._lib import ADV, F32, F64, GHOST, LES, MAX_BODIES, THETA2_MODE, check
from .types import Thermal2D

MAX_FANS = 4


def _f(x) -> float:
    return float(x.item() if torch.is_tensor(x) else x)


def _torch_dtype(ops):
    dt = getattr(ops, "dtype", "float32")
    if isinstance(dt, torch.dtype):
        return dt
    return torch.float64 if str(dt) in ("float64", "torch.float64") else torch.float32


def ghost_rules(ops):
    """[(u | v)][x | y][lo | hi] -> (kind, value): the padding of core.py:284-325."""
    if ops.periodic:
        # face arrays keep their duplicate entry (period n - 1), cell-centred ones wrap by n
        face = (("periodic_face", 0.0), ("periodic_face", 0.0))
        cell = (("periodic_cell", 0.0), ("periodic_cell", 0.0))
        return ((face, cell), (cell, face))

    def wall(kind, speed):
        if kind == "slip":
            return ("even", 0.0)
        if kind == "noslip":
            return ("odd", 0.0)
        return ("affine", float(speed))          # moving: u = speed on the wall

    uy = (wall(ops.bc_bottom, _f(ops.ground_speed)), wall(ops.bc_top, 0.0))
    vy = (("face_odd", 0.0), ("face_odd", 0.0))
    if ops.closed:
        ux = (("face_odd", 0.0), ("face_odd", 0.0))
        side = {"noslip": ("odd", 0.0), "slip": ("even", 0.0)}
        vx = (side[ops.bc_left], side[ops.bc_right])
    else:
        ux = (("edge", 0.0), ("edge", 0.0))
        vx = (("odd", 0.0), ("edge", 0.0))
    return ((ux, uy), (vx, vy))


def thermal_from_physics(ph, geom):
    """The heat transfer of the reference's 2D ``Physics`` (physics.py:291-345) and
    ``geom.thermal`` (None when it has none)."""
    if not getattr(ph, "thermal", False):
        return None
    tg = getattr(geom, "thermal", None)
    kw = {}
    if tg is not None and not geom.empty:
        kw = {n: getattr(tg, n, None) for n in ("chi_t", "a_t", "w_t", "ins_u", "ins_v", "q_skin", "w_f", "vol_u",
                                                 "vol_v")}
        kw["temp_ids"] = tuple(getattr(tg, "temp_ids", ()) or ())
        kw["flux_ids"] = tuple(getattr(tg, "flux_ids", ()) or ())
    vals = ph.wall_values
    vals = vals.detach().cpu().tolist() if torch.is_tensor(vals) else list(vals)
    return Thermal2D(kappa=_f(ph.kappa), ri=_f(ph.ri), prt=float(ph.prt), gravity=tuple(float(g) for g in ph.gravity),
                     eta_t=_f(ph.eta_t), theta_in=_f(ph.theta_in), wall_modes=tuple(ph.wall_modes),
                     wall_values=tuple(float(x) for x in vals), diff_coef=float(ph.diff_coef), **kw)


class Ns2dPlan:
    """Plan + device tensors for one 2D (ops, geom) configuration; ``dye`` turns on the dye
    update after each step, ``thermal`` (a :class:`Thermal2D`) heat transfer."""

    def __init__(self, ops, geom, *, dye: bool = False, thermal=None, placed=None, device=None):
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        if self.device.type != "cuda":
            raise RuntimeError("the B200 step runs on a CUDA device only (no CPU fallback)")
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA is not available: the B200 step has no CPU fallback")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        if getattr(ops, "phys", None) is not None:
            if thermal is not None or placed is not None:
                raise RuntimeError("placed physics comes either from ops.phys or from thermal= / placed=, not both")
            thermal = thermal_from_physics(ops.phys, geom)
            placed = ops.phys
        L = _lib.lib()
        self.dtype = _torch_dtype(ops)
        self.dye = bool(dye)
        nx, ny = int(ops.nx), int(ops.ny)
        self.shape = (ny, nx)
        cfg = _lib.Ns2dConfig()
        cfg.abi_version = _lib.ABI_VERSION
        cfg.dtype = F64 if self.dtype == torch.float64 else F32
        cfg.nx, cfg.ny = nx, ny
        cfg.h = float(ops.h)
        cfg.periodic = int(bool(ops.periodic))
        cfg.closed = int(bool(getattr(ops, "closed", False)))
        if ops.advection not in ADV:
            raise RuntimeError(f"unsupported advection scheme {ops.advection!r}")
        cfg.advection = ADV[ops.advection]
        if ops.turbulence not in LES:
            raise RuntimeError(f"unsupported turbulence model {ops.turbulence!r}")
        cfg.les = LES[ops.turbulence]
        cfg.les_c = float(ops.les_c)
        cfg.nu = _f(ops.nu)
        cfg.eta = _f(ops.eta)
        cfg.cfl = float(ops.cfl)
        if getattr(ops, "dt_fixed", None) is not None:
            cfg.has_dt_fixed = 1
            cfg.dt_fixed = float(ops.dt_fixed)
        for c, comp in enumerate(ghost_rules(ops)):
            for a in range(2):
                for s in range(2):
                    kind, val = comp[a][s]
                    cfg.ghost_kind[c][a][s] = GHOST[kind]
                    cfg.ghost_val[c][a][s] = val
        cfg.force_ref = float(ops.force_ref)
        self.nbody = int(geom.nbody)
        if self.nbody > MAX_BODIES:
            raise RuntimeError(f"the B200 step supports at most {MAX_BODIES} bodies")
        win = tuple(int(x) for x in geom.window)
        self.has_win = self.nbody > 0 and win[1] > win[0] and win[3] > win[2]
        for q in range(4):
            cfg.window[q] = win[q] if self.has_win else 0
        cfg.nbody = self.nbody if self.has_win else 0
        cfg.dye = int(self.dye)
        if getattr(ops, "forcing", None) is not None:   # the verification cases' uniform body force
            cfg.forcing = 1
            cfg.force[0], cfg.force[1] = _f(ops.forcing[0]), _f(ops.forcing[1])
        if getattr(ops, "wall_model", False):   # the Werner-Wengle shear (core.py:536-564)
            bits = 0
            if ops.bc_bottom in ("noslip", "moving"):
                bits |= 1
                if ops.bc_bottom == "moving":
                    cfg.wall_ground_speed = float(ops.ground_speed)
            if ops.bc_top == "noslip":
                bits |= 2
            if getattr(ops, "closed", False) and (ops.bc_left == "noslip" or ops.bc_right == "noslip"):
                bits |= (4 if ops.bc_left == "noslip" else 0) | (8 if ops.bc_right == "noslip" else 0)
            cfg.wall_model = bits
        self.thermal = thermal
        self.n_temp = self.n_flux = 0
        self._keep = []
        dev, dt = self.device, self.dtype

        def up(x, shape=None):
            t = torch.as_tensor(np.asarray(x) if not torch.is_tensor(x) else x)
            t = t.to(device=dev, dtype=dt)
            if shape is not None:
                t = t.reshape(shape)
            t = t.contiguous()
            self._keep.append(t)
            return t

        g = _lib.Ns2dGeom()
        if self.has_win:
            for name in ("chi_u", "chi_v", "chi_c", "a_u", "a_v", "k_u", "k_v"):
                setattr(g, name, up(getattr(geom, name)).data_ptr())
        u_in = getattr(ops, "u_inlet", None)
        if u_in is not None:
            g.u_inlet = up(u_in, (ny,)).data_ptr()
        d_in = getattr(ops, "dye_inlet", None)
        if self.dye and d_in is not None:
            g.dye_inlet = up(d_in, (ny,)).data_ptr()
        if thermal is not None:
            self._thermal_config(cfg, g, thermal, up)
        self.placed = placed
        self.nfan = 0
        self.pid = False
        self.dye_channels = 0
        if placed is not None:
            self._placed_config(cfg, g, placed, thermal is not None, up)

        def live(x):
            """The reference's 0-d device scalar itself (its set_reynolds fills it in place, so a
            captured step follows a live Re change), else None (the constant in cfg)."""
            ok = torch.is_tensor(x) and x.numel() == 1 and x.device == dev and x.dtype == dt and x.is_contiguous()
            if not ok:
                return None
            self._keep.append(x)          # held while the plan lives, whatever happens to ops
            return x.data_ptr()

        g.nu, g.eta = live(getattr(ops, "nu", None)), live(getattr(ops, "eta", None))
        ph = getattr(ops, "phys", None)
        if thermal is not None and ph is not None:
            g.kappa, g.eta_t = live(getattr(ph, "kappa", None)), live(getattr(ph, "eta_t", None))
        self.cfg = cfg
        self.geom_c = g
        handle = C.c_void_p()
        check(L.aero_ns2d_plan_create(C.byref(cfg), C.byref(handle)), "aero_ns2d_plan_create")
        self._handle = handle
        nbytes = L.aero_ns2d_workspace_bytes(handle)
        self._ws_raw = torch.empty(nbytes + 256, dtype=torch.uint8, device=dev)
        self.ws_ptr = (self._ws_raw.data_ptr() + 255) & ~255
        self.workspace_bytes = nbytes
        check(L.aero_ns2d_workspace_init(handle, C.c_void_p(self.ws_ptr), self._stream()), "aero_ns2d_workspace_init")

    def _thermal_config(self, cfg, g, th, up):
        cfg.thermal = 1
        cfg.kappa, cfg.ri, cfg.prt = float(th.kappa), float(th.ri), float(th.prt)
        cfg.gravity[0], cfg.gravity[1] = (float(x) for x in th.gravity)
        cfg.eta_t, cfg.theta_in = float(th.eta_t), float(th.theta_in)
        modes = tuple(th.wall_modes)
        if len(modes) != 4 or any(m not in THETA2_MODE for m in modes):
            raise RuntimeError(f"unsupported temperature boundary modes {modes!r}")
        for q in range(4):
            cfg.wall_mode[q] = THETA2_MODE[modes[q]]
            cfg.wall_value[q] = float(th.wall_values[q])
        cfg.diff_coef = float(th.diff_coef)
        if self.has_win:
            self.n_temp, self.n_flux = len(th.temp_ids), len(th.flux_ids)
            if self.n_temp > MAX_BODIES or self.n_flux > MAX_BODIES:
                raise RuntimeError(f"the B200 step supports at most {MAX_BODIES} temperature / heat-flux bodies")
            wy, wx = cfg.window[1] - cfg.window[0], cfg.window[3] - cfg.window[2]
            if self.n_temp:
                g.chi_t = up(th.chi_t, (wy, wx)).data_ptr()
                g.a_t = up(th.a_t, (wy, wx)).data_ptr()
                g.w_t = up(th.w_t, (self.n_temp, wy, wx)).data_ptr()
            if self.n_flux:
                g.q_skin = up(th.q_skin, (wy, wx)).data_ptr()
                g.w_f = up(th.w_f, (self.n_flux, wy, wx)).data_ptr()
            if th.ins_u is not None:
                cfg.has_ins = 1
                g.ins_u = up(th.ins_u, (wy, wx + 1)).data_ptr()
                g.ins_v = up(th.ins_v, (wy + 1, wx)).data_ptr()
            if th.vol_u is not None:
                cfg.has_vol = 1
                g.vol_u = up(th.vol_u, (wy, wx + 1)).data_ptr()
                g.vol_v = up(th.vol_v, (wy + 1, wx)).data_ptr()
        cfg.n_temp, cfg.n_flux = self.n_temp, self.n_flux

    def _placed_config(self, cfg, g, pl, thermal, up):
        """Fans, heaters, paint and the PID step (physics.py:70-140): the reference's tensors are
        used in place when they already live on the device in the plan's dtype (a live paint
        stroke or fan setting then reaches the next step), else uploaded."""
        ny, nx = self.shape
        dev, dt = self.device, self.dtype

        def arr(x, shape):
            if torch.is_tensor(x) and x.device == dev and x.dtype == dt and x.is_contiguous() and tuple(x.shape) == shape:
                self._keep.append(x)
                return x.data_ptr()
            return up(x, shape).data_ptr()

        nfan = int(getattr(pl, "nfan", 0) or 0)
        if nfan > MAX_FANS:
            raise RuntimeError(f"the B200 2D step supports at most {MAX_FANS} fans")
        self.nfan = cfg.nfan = nfan
        if nfan:
            g.fan_gu = arr(pl.fan_gu, (nfan, ny, nx + 1))
            g.fan_gv = arr(pl.fan_gv, (nfan, ny + 1, nx))
            g.fan_phi = arr(pl.fan_phi, (nfan, ny, nx))
            g.fan_dir = arr(pl.fan_dir, (nfan, 2))
            for name in ("fan_value", "fan_width", "fan_kp", "fan_ki", "fan_dpmax", "fan_isvel", "fan_isthrust"):
                setattr(g, name, arr(getattr(pl, name), (nfan,)))
        g.u_floor = arr(getattr(pl, "u_floor", 0.0) if getattr(pl, "u_floor", None) is not None else 0.0, ())
        if getattr(pl, "heat", None) is not None:
            if not thermal:
                raise RuntimeError("heaters need heat transfer")
            cfg.heaters = 1
            g.heat = arr(pl.heat, (ny, nx))
            g.heat_max = arr(pl.heat_max, ())
        if bool(getattr(pl, "paint", False)):
            cfg.paint = 1
            g.paint_c = arr(pl.paint_c, (ny, nx))
            for name, shape in (("paint_u", (ny, nx + 1)), ("paint_v", (ny + 1, nx)), ("paint_wu", (ny, nx + 1)),
                                ("paint_wv", (ny + 1, nx))):
                setattr(g, name, arr(getattr(pl, name), shape))
        self.pid = bool(getattr(pl, "pid", False))
        cfg.pid = int(self.pid)
        self.ports = bool(getattr(pl, "ports", False))
        if self.ports:   # jets and vents (physics.py:362-433) with the combined penalisation
            cfg.ports = 1
            for name, shape in (("xchi_u", (ny, nx + 1)), ("xa_u", (ny, nx + 1)), ("xchi_v", (ny + 1, nx)),
                                ("xa_v", (ny + 1, nx)), ("src", (ny, nx)), ("src_neg", (ny, nx))):
                setattr(g, name, arr(getattr(pl, name), shape))
            g.q_net = arr(getattr(pl, "q_net", 0.0), ())
            if thermal and getattr(pl, "pt_chi", None) is not None:
                g.pt_chi = arr(pl.pt_chi, (ny, nx))
                g.pt_a = arr(pl.pt_a, (ny, nx))
        n_dye = int(getattr(pl, "n_dye", 0) or 0)
        self.dye_channels = n_dye
        if n_dye:   # smoke channels with emitter groups and smoking jets (physics.py:497-540)
            if n_dye > 4:
                raise RuntimeError("the B200 2D step carries at most 4 smoke channels")
            if not self.dye:
                raise RuntimeError("smoke channels need the plan's dye")
            cfg.dye_channels = n_dye
            if getattr(pl, "dye_inflow", None) is not None:
                g.dye_inflow = arr(pl.dye_inflow, (n_dye, ny))
            groups = list(getattr(pl, "groups", None) or [])
            if len(groups) > 8:
                raise RuntimeError("the B200 2D step takes at most 8 emitter groups")
            cfg.n_groups = len(groups)
            for q, grp in enumerate(groups):
                ch, w, target, timing = grp if isinstance(grp, tuple) else (grp.channel, grp.weight, grp.target,
                                                                            grp.timing)
                cfg.group_channel[q] = int(ch)
                g.group_w[q] = arr(w, (ny, nx))
                g.group_target[q] = arr(target, (ny, nx))
                g.group_timing[q] = arr(timing, (4,))
            for ch, w in (getattr(pl, "port_dye", None) or {}).items():
                g.port_dye[int(ch)] = arr(w, (ny, nx))

    @property
    def ctrl_size(self):
        """Length of the controller memory (core.py State.ctrl): 0, or 2 + 2 nfan."""
        return 2 + 2 * self.nfan if (self.pid or self.nfan) else 0

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().aero_ns2d_plan_destroy(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self._handle = None

    def empty_fields(self):
        """Fresh device tensors for a step's outputs."""
        ny, nx = self.shape
        kw = dict(device=self.device, dtype=self.dtype)
        out = {"u": torch.empty(ny, nx + 1, **kw), "v": torch.empty(ny + 1, nx, **kw), "p": torch.empty(ny, nx, **kw),
               "t": torch.empty((), **kw), "dt": torch.empty((), **kw),
               "coeffs": torch.zeros(max(self.nbody, 1), 3, **kw)[: self.nbody]}
        if self.dye:
            out["dye"] = torch.empty(ny, nx, **kw)
            if self.dye_channels > 1:
                out["dye_extra"] = torch.empty(self.dye_channels - 1, ny, nx, **kw)
        if self.thermal is not None:
            d64 = dict(device=self.device, dtype=torch.float64)
            out.update(theta=torch.empty(ny, nx, **kw), heat=torch.zeros(self.n_temp, **d64),
                       theta_wall=torch.zeros(self.n_flux, **d64), wall_heat=torch.zeros(4, **d64),
                       heat_storage=torch.zeros(1, **d64), flow_heat=torch.zeros(2, **d64))
        if self.ctrl_size:
            out["ctrl"] = torch.zeros(self.ctrl_size, **kw)
        if self.nfan:
            out["fan_thrust"] = torch.zeros(self.nfan, **kw)
            out["fan_ud"] = torch.zeros(self.nfan, **kw)
        if self.cfg.paint:
            out["paint_force"] = torch.zeros(2, **kw)
        if self.cfg.ports and self.thermal is not None:
            d64 = dict(device=self.device, dtype=torch.float64)
            out["vent_heat"] = torch.zeros(1, **d64)
            if self.geom_c.pt_chi:
                out["jet_heat"] = torch.zeros(1, **d64)
        return out

    def _check(self, name, t, shape):
        if not (torch.is_tensor(t) and t.device == self.device and t.dtype == self.dtype and t.is_contiguous()):
            raise RuntimeError(f"{name} must be a contiguous {self.dtype} tensor on {self.device}")
        if tuple(t.shape) != tuple(shape):
            raise RuntimeError(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")

    def step(self, u0, v0, t0, *, dye0=None, theta0=None, out=None, dt=None, ctrl0=None, dt_prev=None,
             dye_extra0=None):
        """One step (plus the dye update when the plan has dye, theta and the heat report
        (float64: heat, theta_wall, wall_heat, heat_storage, flow_heat) with heat transfer);
        returns the output dict.  ``out`` may hold u0 / v0 / theta0 themselves (in-place
        update); ``dt`` is None (CFL rule on the device) or a 0-d device tensor.  With fans or
        the PID step, ``ctrl0`` is the controller memory (``ctrl_size``) and ``dt_prev`` the
        previous step (0-d; 0 on the first); ``out`` then also holds the new ``ctrl``, the
        fans' ``fan_thrust`` / ``fan_ud`` and the paint's ``paint_force``."""
        ny, nx = self.shape
        self._check("u0", u0, (ny, nx + 1))
        self._check("v0", v0, (ny + 1, nx))
        self._check("t0", t0, ())
        out = self.empty_fields() if out is None else out
        f = _lib.Ns2dFields()
        f.u0, f.v0, f.t0 = u0.data_ptr(), v0.data_ptr(), t0.data_ptr()
        for name in ("u", "v", "p", "t", "dt"):
            setattr(f, name, out[name].data_ptr())
        if self.nbody and self.has_win:
            f.coeffs = out["coeffs"].data_ptr()
        if self.dye:
            if dye0 is None:
                raise RuntimeError("this plan has dye: dye0 is required")
            self._check("dye0", dye0, (ny, nx))
            f.dye0, f.dye = dye0.data_ptr(), out["dye"].data_ptr()
            if self.dye_channels > 1:   # smoke channels 1.. (State.dye_extra)
                if dye_extra0 is None:
                    raise RuntimeError("this plan has several smoke channels: dye_extra0 is required")
                self._check("dye_extra0", dye_extra0, (self.dye_channels - 1, ny, nx))
                f.dye_extra0, f.dye_extra = dye_extra0.data_ptr(), out["dye_extra"].data_ptr()
        if self.thermal is not None:
            if theta0 is None:
                raise RuntimeError("this plan has heat transfer: theta0 is required")
            self._check("theta0", theta0, (ny, nx))
            f.theta0, f.theta = theta0.data_ptr(), out["theta"].data_ptr()
            for name in ("heat", "theta_wall", "wall_heat", "heat_storage", "flow_heat"):
                t = out[name]
                if not (t.device == self.device and t.dtype == torch.float64 and t.is_contiguous()):
                    raise RuntimeError(f"{name} must be a contiguous float64 tensor on {self.device}")
                if t.numel():
                    setattr(f, name, t.data_ptr())
        elif theta0 is not None:
            raise RuntimeError("theta0 given to a plan without heat transfer")
        if self.ctrl_size:
            if ctrl0 is None:
                raise RuntimeError("this plan has fans or the PID step: ctrl0 is required")
            self._check("ctrl0", ctrl0, (self.ctrl_size,))
            f.ctrl0, f.ctrl = ctrl0.data_ptr(), out["ctrl"].data_ptr()
            if dt_prev is None:
                dt_prev = torch.zeros((), device=self.device, dtype=self.dtype)
                self._keep_dt_prev = dt_prev
            self._check("dt_prev", dt_prev, ())
            f.dt_prev = dt_prev.data_ptr()
        if self.nfan:
            f.fan_thrust, f.fan_ud = out["fan_thrust"].data_ptr(), out["fan_ud"].data_ptr()
        if self.cfg.paint:
            f.paint_force = out["paint_force"].data_ptr()
        for name in ("vent_heat", "jet_heat"):
            if name in out:
                setattr(f, name, out[name].data_ptr())
        dtp = None
        if dt is not None:
            self._check("dt", dt, ())
            dtp = C.c_void_p(dt.data_ptr())
        check(_lib.lib().aero_ns2d_step(self._handle, C.byref(f), C.byref(self.geom_c), dtp, C.c_void_p(self.ws_ptr),
                                        self._stream()), "aero_ns2d_step")
        return out

    def poisson_solve(self, f, psi=None):
        self._check("f", f, self.shape)
        psi = torch.empty_like(f) if psi is None else psi
        check(_lib.lib().aero_ns2d_poisson_solve(self._handle, C.c_void_p(f.data_ptr()), C.c_void_p(psi.data_ptr()),
                                                 C.c_void_p(self.ws_ptr), self._stream()), "aero_ns2d_poisson_solve")
        return psi
