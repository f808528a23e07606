"""One 3D configuration bound to the C ABI: constants, device masks and the workspace.

:class:`Ns3dPlan` reads the reference's objects by attribute (``Ops3D``, ``Geometry3D``,
``ThermalOps``, ``DyeSources``: the containers of :mod:`aerolume_b200.ns3d.types` or the
reference's own), validates what the B200 step supports, uploads the window masks once
and owns the device workspace.  What the step does not support (more than eight bodies, four
fans, four jets / vents or four heaters; jets and vents together with the smoke update)
raises ``RuntimeError``: there is no fallback to a CPU or plain-torch path.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from .. import _lib
from .._lib import ADV, F32, F64, GHOST, LES, MAX_BODIES, MAX_FANS, MAX_PORTS, THETA_SIDE, check


def _f(x) -> float:
    return float(x.item() if torch.is_tensor(x) else x)


def _torch_dtype(ops):
    dt = getattr(ops, "dtype", "float32")
    if isinstance(dt, torch.dtype):
        return dt
    return torch.float64 if str(dt) in ("float64", "torch.float64") else torch.float32


def _window_empty(win) -> bool:
    k0, k1, j0, j1, i0, i1 = win
    return k1 <= k0 or j1 <= j0 or i1 <= i0


class Ns3dPlan:
    """Plan + device tensors for one (ops, geom, thermal, smoke) configuration.

    ``thermal`` is a ``ThermalOps`` (or None); ``dye_src`` a ``DyeSources`` (or None);
    ``smoke`` turns the smoke update on inside :meth:`step`.  ``paint`` (``chi_u / chi_v /
    chi_w / chi_c`` tensors, a ``PaintLayer``), ``pid`` (``target`` and the ``dt_prev / e1 /
    e2`` state tensors, a ``PidDt``), ``u_floor`` (the sources' speed scale) and ``fans`` (a
    ``FanSet``: actuator discs with their PI thrust state) and ``ports`` (a ``PortSet``: jets
    and vents) are the placed physics of physics.py:831-1262 the step runs.
    """

    def __init__(self, ops, geom, thermal=None, dye_src=None, *, smoke: bool = False, device=None, paint=None,
                 pid=None, u_floor: float = 0.0, fans=None, ports=None, closure=None):
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        if self.device.type != "cuda":
            raise RuntimeError("the B200 step runs on a CUDA device only (no CPU fallback)")
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA is not available: the B200 step has no CPU fallback")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        L = _lib.lib()
        self.dtype = _torch_dtype(ops)
        self.ops, self.geom, self.thermal, self.dye_src = ops, geom, thermal, dye_src
        self.smoke = bool(smoke)
        nx, ny, nz = int(ops.nx), int(ops.ny), int(ops.nz)
        self.shape = (nz, ny, nx)
        cfg = _lib.Ns3dConfig()
        cfg.abi_version = _lib.ABI_VERSION
        cfg.dtype = F64 if self.dtype == torch.float64 else F32
        cfg.nx, cfg.ny, cfg.nz = nx, ny, nz
        cfg.h = float(ops.h)
        px, py, pz = (bool(x) for x in ops.periodic_axes)
        cfg.periodic[0], cfg.periodic[1], cfg.periodic[2] = int(px), int(py), int(pz)
        cfg.closed = int(bool(getattr(ops, "closed", False)))
        cfg.symmetry = int(bool(getattr(ops, "symmetry", False)))
        if ops.advection not in ADV:
            raise RuntimeError(f"unsupported advection scheme {ops.advection!r}")
        cfg.advection = ADV[ops.advection]
        if ops.turbulence not in LES:
            raise RuntimeError(f"unsupported turbulence model {ops.turbulence!r}")
        cfg.les = LES[ops.turbulence]
        cfg.les_c = float(ops.les_c)
        cfg.nu = float(ops.nu_value)
        cfg.eta = _f(ops.eta)
        cfg.cfl = float(ops.cfl)
        if getattr(ops, "dt_fixed", None) is not None:
            cfg.has_dt_fixed = 1
            cfg.dt_fixed = float(ops.dt_fixed)
        for c, comp in enumerate("uvw"):
            for a in range(3):
                for s in range(2):
                    kind, val = ops.ghost[comp][a][s]
                    cfg.ghost_kind[c][a][s] = GHOST[kind]
                    cfg.ghost_val[c][a][s] = float(val)
        cfg.ref_area = float(ops.ref_area)
        cfg.length_ref = float(ops.length_ref)
        cfg.span_ref = float(ops.span_ref)
        for q in range(3):
            cfg.moment_ref[q] = float(ops.moment_ref[q])
        cfg.y0 = float(ops.y0)
        if getattr(ops, "forcing", None) is not None:   # the verification cases' uniform body force
            cfg.forcing = 1
            for q in range(3):
                cfg.force[q] = _f(ops.forcing[q])
        self.nbody = int(geom.nbody)
        win = tuple(int(x) for x in geom.window)
        self.has_win = not _window_empty(win) and self.nbody > 0
        if self.nbody > MAX_BODIES:
            raise RuntimeError(f"the B200 step supports at most {MAX_BODIES} bodies")
        for q in range(6):
            cfg.window[q] = win[q] if self.has_win else 0
        cfg.nbody = self.nbody
        self._keep = []
        dev, dt = self.device, self.dtype

        def up(x):
            if x is None:
                return None
            t = torch.as_tensor(np.asarray(x) if not torch.is_tensor(x) else x)
            t = t.to(device=dev, dtype=dt).contiguous()
            self._keep.append(t)
            return t

        g = _lib.Ns3dGeom()
        if self.has_win:
            for name in ("chi_u", "chi_v", "chi_w", "chi_c", "a_u", "a_v", "a_w", "k_u", "k_v", "k_w"):
                setattr(g, name, up(getattr(geom, name)).data_ptr())
        u_in = getattr(ops, "u_inlet", None)
        if u_in is not None:
            g.u_inlet = up(torch.as_tensor(np.asarray(u_in) if not torch.is_tensor(u_in) else u_in)
                           .reshape(nz, ny)).data_ptr()
        if thermal is not None:
            self._thermal_config(cfg, g, thermal, up)
        if self.smoke:
            cfg.smoke = 1
            if dye_src is not None and not _window_empty(dye_src.window):
                for q in range(6):
                    cfg.dye_window[q] = int(dye_src.window[q])
                g.dye_weight = up(dye_src.weight).data_ptr()
                pulse = [_f(x) for x in (dye_src.pulse if not torch.is_tensor(dye_src.pulse) else dye_src.pulse.tolist())]
                cfg.pulse_on, cfg.pulse_period = pulse[0], pulse[1]
            else:
                cfg.pulse_on, cfg.pulse_period = 2.0, 1.0
        self.paint, self.pid = paint, pid
        cfg.u_floor = float(u_floor)
        if pid is not None:
            cfg.pid, cfg.pid_target = 1, float(pid.target)
            for name in ("dt_prev", "e1", "e2"):
                self._check("pid." + name, getattr(pid, name), ())
        if paint is not None:
            cfg.paint = 1
            shapes = {"u": (nz, ny, nx + 1), "v": (nz, ny + 1, nx), "w": (nz + 1, ny, nx), "c": (nz, ny, nx)}
            for gname, shape in shapes.items():
                t = getattr(paint, "chi_" + gname)
                self._check("paint.chi_" + gname, t, shape)
                setattr(g, "paint_" + gname, t.data_ptr())
        self.fans = fans if fans is not None and len(fans) else None
        if self.fans is not None:
            self._fan_config(cfg, g, self.fans, up)
        self.ports = ports if ports is not None and len(ports) else None
        if self.ports is not None:
            self._port_config(cfg, g, self.ports, up)
        # the learned subgrid closure (a ClosureModel): its nu_t replaces WALE's where it applies;
        # the plan keeps the model's standardisation constants of this moment and reads its
        # parameters from the model's tensors at every step
        self.closure = closure
        if closure is not None:
            cfg.closure = 1
            self._closure_c = closure.cstruct()
            g.closure = C.addressof(self._closure_c)
            self._keep.extend([closure.params, closure.params_bf16])
        self.cfg = cfg
        self.geom_c = g
        handle = C.c_void_p()
        check(L.aero_ns3d_plan_create(C.byref(cfg), C.byref(handle)), "aero_ns3d_plan_create")
        self._handle = handle
        nbytes = L.aero_ns3d_workspace_bytes(handle)
        self._ws_raw = torch.empty(nbytes + 256, dtype=torch.uint8, device=dev)
        base = self._ws_raw.data_ptr()
        self.ws_ptr = (base + 255) & ~255
        self.workspace_bytes = nbytes
        check(L.aero_ns3d_workspace_init(handle, C.c_void_p(self.ws_ptr), self._stream()),
              "aero_ns3d_workspace_init")

    # -------------------------------------------------------------------- set-up
    def _thermal_config(self, cfg, g, th, up):
        srcs = getattr(th, "sources", None)
        items = list(getattr(srcs, "items", srcs) or [])   # a HeatSourceSet, or (window, density) pairs
        if len(items) > _lib.MAX_HEATERS:
            raise RuntimeError(f"the B200 step supports at most {_lib.MAX_HEATERS} volumetric heaters")
        if items:
            arr = (_lib.Ns3dHeater * len(items))()
            for q, (win, dens) in enumerate(items):
                win = tuple(int(x) for x in win)
                shape = (win[1] - win[0], win[3] - win[2], win[5] - win[4])
                t = up(dens)
                if tuple(t.shape) != shape:
                    raise RuntimeError(f"heater {q} density has shape {tuple(t.shape)}, expected {shape}")
                for e in range(6):
                    arr[q].window[e] = win[e]
                arr[q].q = t.data_ptr()
            cfg.nheat = len(items)
            self._heat_arr = arr
            g.heaters = C.cast(arr, C.c_void_p)
        cfg.thermal = 1
        cfg.kappa, cfg.pe, cfg.ri, cfg.prt = float(th.kappa), float(th.pe), float(th.ri), float(th.prt)
        cfg.eta_t = _f(th.eta)
        vals = th.side_vals.tolist() if torch.is_tensor(th.side_vals) else list(th.side_vals)
        for q in range(6):
            cfg.side_kind[q] = THETA_SIDE[th.side_kinds[q]]
            cfg.side_val[q] = float(vals[q])
        hm = getattr(th, "heat_max", None)
        if hm is not None:
            cfg.has_heat_max = 1
            cfg.heat_max = _f(hm)
        tg = th.geom
        t_index = list(getattr(tg, "t_index", []) or [])
        if self.has_win:
            cfg.n_tbody = len(t_index)
            for q, b in enumerate(t_index):
                cfg.t_index[q] = int(b)
            if tg.chi_t is not None:
                g.chi_t = up(tg.chi_t).data_ptr()
                g.a_t = up(tg.a_t).data_ptr()
                g.w_t = up(tg.w_t).data_ptr()
            if tg.adia is not None:
                cfg.has_adia = 1
                g.adia_u, g.adia_v, g.adia_w = (up(a).data_ptr() for a in tg.adia)
            if tg.vol_w is not None:
                g.vol_w = up(tg.vol_w).data_ptr()
            if getattr(tg, "skin", None) is not None:
                cfg.has_skin = 1
                g.skin = up(tg.skin).data_ptr()
        fr = getattr(tg, "flux_rate", None)
        if fr is not None:
            vals = fr.tolist() if torch.is_tensor(fr) else list(np.asarray(fr).reshape(-1))
            for q, x in enumerate(vals[:MAX_BODIES]):
                cfg.flux_rate[q] = float(x)

    def _fan_config(self, cfg, g, fans, up):
        n = len(fans.items)
        if n > MAX_FANS:
            raise RuntimeError(f"the B200 step supports at most {MAX_FANS} fans")

        def host(x):
            return [float(v) for v in (x.tolist() if torch.is_tensor(x) else np.asarray(x).reshape(-1))]
        consts = {name: host(getattr(fans, name)) for name in ("target", "kp", "ki", "tmax", "swirl")}
        vmode = host(fans.velocity_mode)
        cfg.nfan, cfg.fan_swirl = n, int(bool(fans.any_swirl))
        arr = (_lib.Ns3dFan * n)()
        nz, ny, nx = self.shape
        for q, it in enumerate(fans.items):
            d = arr[q]
            win = tuple(int(x) for x in it["win"])
            if _window_empty(win):
                raise RuntimeError("a fan window is empty")
            for e in range(6):
                d.window[e] = win[e]
            k0, k1, j0, j1, i0, i1 = win
            shapes = {"u": (k1 - k0, j1 - j0, i1 - i0 + 1), "v": (k1 - k0, j1 - j0 + 1, i1 - i0),
                      "w": (k1 - k0 + 1, j1 - j0, i1 - i0)}
            d.velocity_mode = int(bool(vmode[q]))
            for name in ("target", "kp", "ki", "tmax", "swirl"):
                setattr(d, name, consts[name][q])
            for kind in "fsm":
                for comp in "uvw":
                    a = it.get(kind + comp)
                    if a is None:
                        continue
                    t = up(a)
                    if tuple(t.shape) != shapes[comp]:
                        raise RuntimeError(f"fan {q} weights {kind}{comp} have shape {tuple(t.shape)}, "
                                           f"expected {shapes[comp]}")
                    setattr(d, f"{kind}_{comp}", t.data_ptr())
            for name in ("thrust", "ud", "e_prev", "swirl_amp"):
                t = getattr(fans, name)
                self._check("fans." + name, t, (n,))
                setattr(d, name, t.data_ptr() + q * t.element_size())
        self._fan_arr = arr
        g.fans = C.cast(arr, C.c_void_p)

    def _port_config(self, cfg, g, ports, up):
        n = len(ports.items)
        if n > MAX_PORTS:
            raise RuntimeError(f"the B200 step supports at most {MAX_PORTS} jets and vents")
        if self.smoke:
            raise RuntimeError("jets and vents: build the plan without smoke and apply their smoke sources after "
                               "smoke_step (as FlowSolver3D does)")
        mf = ports.mass_flux
        cfg.nport = n
        cfg.port_source = float(mf.item() if torch.is_tensor(mf) else mf)
        cfg.port_leak = float(getattr(ports, "leak", 0.0) or 0.0)
        arr = (_lib.Ns3dPort * n)()
        for q, it in enumerate(ports.items):
            d = arr[q]
            win = tuple(int(x) for x in it["win"])
            if _window_empty(win):
                raise RuntimeError("a port window is empty")
            for e in range(6):
                d.window[e] = win[e]
            k0, k1, j0, j1, i0, i1 = win
            d.vent = int(it["kind"] == "vent")
            d.theta = float(it.get("theta", 0.0) or 0.0)
            shapes = {"fu": ("f_u", (k1 - k0, j1 - j0, i1 - i0 + 1)), "fv": ("f_v", (k1 - k0, j1 - j0 + 1, i1 - i0)),
                      "fw": ("f_w", (k1 - k0 + 1, j1 - j0, i1 - i0)), "m": ("m", (k1 - k0, j1 - j0, i1 - i0))}
            for name, (field, shape) in shapes.items():
                t = up(it[name])
                if tuple(t.shape) != shape:
                    raise RuntimeError(f"port {q} weights {name} have shape {tuple(t.shape)}, expected {shape}")
                setattr(d, field, t.data_ptr())
        self._port_arr = arr
        g.ports = C.cast(arr, C.c_void_p)

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().aero_ns3d_plan_destroy(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self._handle = None

    # -------------------------------------------------------------------- buffers
    def empty_fields(self):
        """Fresh device tensors for a step's outputs."""
        nz, ny, nx = self.shape
        kw = {"device": self.device, "dtype": self.dtype}
        out = {"u": torch.empty(nz, ny, nx + 1, **kw), "v": torch.empty(nz, ny + 1, nx, **kw),
               "w": torch.empty(nz + 1, ny, nx, **kw), "p": torch.empty(nz, ny, nx, **kw),
               "t": torch.empty((), **kw), "dt": torch.empty((), **kw),
               "coeffs": torch.zeros(max(self.nbody, 0), 6, **kw)}
        if self.thermal is not None:
            out["theta"] = torch.empty(nz, ny, nx, **kw)
            out["heat_rate"] = torch.zeros(max(self.nbody, 0), **kw)
        if self.smoke:
            out["dye"] = torch.empty(nz, ny, nx, **kw)
        return out

    def _check(self, name, t, shape):
        if not torch.is_tensor(t) or t.device != self.device or t.dtype != self.dtype or not t.is_contiguous():
            raise RuntimeError(f"{name} must be a contiguous {self.dtype} tensor on {self.device}")
        if tuple(t.shape) != tuple(shape):
            raise RuntimeError(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")

    # -------------------------------------------------------------------- calls
    def step(self, u0, v0, w0, t0, *, theta0=None, dye0=None, out=None, dt=None, events=None, div_sq=None):
        """One step (plus the smoke update when the plan has smoke); returns the output dict.

        ``out`` (from :meth:`empty_fields`) may hold ``u0 / v0 / w0 / theta0`` themselves
        (in-place update); ``dt`` is None (CFL rule on the device) or a 0-d device tensor.
        ``events``: a list of ``torch.cuda.Event(enable_timing=True)`` recorded at the step's
        phase boundaries (``aero_ns3d_step_traced``).  ``div_sq``: a 0-d device tensor that
        receives the sum of squares of the last stage's projection right-hand side (the
        diagnostics row's ``poisson_residual`` denominator), or None."""
        nz, ny, nx = self.shape
        self._check("u0", u0, (nz, ny, nx + 1))
        self._check("v0", v0, (nz, ny + 1, nx))
        self._check("w0", w0, (nz + 1, ny, nx))
        self._check("t0", t0, ())
        out = self.empty_fields() if out is None else out
        f = _lib.Ns3dFields()
        f.u0, f.v0, f.w0, f.t0 = u0.data_ptr(), v0.data_ptr(), w0.data_ptr(), t0.data_ptr()
        for name in ("u", "v", "w", "p", "t", "dt", "coeffs"):
            setattr(f, name, out[name].data_ptr())
        if self.thermal is not None:
            if theta0 is None:
                raise RuntimeError("this plan has heat transfer: theta0 is required")
            self._check("theta0", theta0, (nz, ny, nx))
            f.theta0, f.theta, f.heat_rate = theta0.data_ptr(), out["theta"].data_ptr(), out["heat_rate"].data_ptr()
        if self.smoke:
            if dye0 is None:
                raise RuntimeError("this plan has smoke: dye0 is required")
            self._check("dye0", dye0, (nz, ny, nx))
            f.dye0, f.dye = dye0.data_ptr(), out["dye"].data_ptr()
        if self.pid is not None:
            f.pid_dt_prev, f.pid_e1, f.pid_e2 = (getattr(self.pid, n).data_ptr() for n in ("dt_prev", "e1", "e2"))
        if div_sq is not None:
            self._check("div_sq", div_sq, ())
            f.div_sq = div_sq.data_ptr()
        dtp = None
        if dt is not None:
            self._check("dt", dt, ())
            dtp = C.c_void_p(dt.data_ptr())
        L = _lib.lib()
        if events is None:
            check(L.aero_ns3d_step(self._handle, C.byref(f), C.byref(self.geom_c), dtp, C.c_void_p(self.ws_ptr),
                                   self._stream()), "aero_ns3d_step")
        else:
            arr = (C.c_void_p * len(events))(*[C.c_void_p(e.cuda_event) for e in events])
            check(L.aero_ns3d_step_traced(self._handle, C.byref(f), C.byref(self.geom_c), dtp, C.c_void_p(self.ws_ptr),
                                          self._stream(), arr, len(events)), "aero_ns3d_step_traced")
        return out

    def smoke_step(self, dye0, u, v, w, t_new, dt, out=None, *, solids=True, sources=True):
        """The smoke update alone with the given velocity, step and new time.  ``solids`` /
        ``sources`` False leave out the clearing inside bodies / the nozzles (advection,
        clipping and the floor only: the reference's fast_dye)."""
        if not self.smoke:
            raise RuntimeError("this plan was built without smoke")
        nz, ny, nx = self.shape
        self._check("dye0", dye0, (nz, ny, nx))
        out = torch.empty_like(dye0) if out is None else out
        f = _lib.Ns3dFields()
        f.dye0, f.dye = dye0.data_ptr(), out.data_ptr()
        f.u, f.v, f.w, f.t, f.dt = u.data_ptr(), v.data_ptr(), w.data_ptr(), t_new.data_ptr(), dt.data_ptr()
        g = self.geom_c
        if not (solids and sources):
            g = _lib.Ns3dGeom.from_buffer_copy(self.geom_c)
            if not solids:
                g.chi_c = None
                g.paint_c = None
            if not sources:
                g.dye_weight = None
        check(_lib.lib().aero_ns3d_smoke(self._handle, C.byref(f), C.byref(g), self._stream()), "aero_ns3d_smoke")
        return out

    def fields(self, u, v, w, names=_lib.FIELD_NAMES):
        """Cell-centred output fields of the state (u, v, w): any of "uc", "vc", "wc" (centred
        velocity), "speed", "vorticity", "q", "nut"; returns {name: (nz, ny, nx) tensor}."""
        nz, ny, nx = self.shape
        self._check("u", u, (nz, ny, nx + 1))
        self._check("v", v, (nz, ny + 1, nx))
        self._check("w", w, (nz + 1, ny, nx))
        res = {}
        ptrs = (C.c_void_p * len(_lib.FIELD_NAMES))()
        for q, name in enumerate(_lib.FIELD_NAMES):
            if name in names:
                res[name] = torch.empty(self.shape, device=self.device, dtype=self.dtype)
                ptrs[q] = res[name].data_ptr()
        unknown = set(names) - set(_lib.FIELD_NAMES)
        if unknown:
            raise KeyError(f"unknown fields {sorted(unknown)}; available: {', '.join(_lib.FIELD_NAMES)}")
        check(_lib.lib().aero_ns3d_fields(self._handle, C.c_void_p(u.data_ptr()), C.c_void_p(v.data_ptr()),
                                          C.c_void_p(w.data_ptr()), C.byref(self.geom_c), ptrs, self._stream()),
              "aero_ns3d_fields")
        return res

    def slice(self, u, v, w, name, axis, position):
        """A planar cut of an output field at ``position`` normal to ``axis`` ("x", "y", "z"):
        linear interpolation between the two nearest cell planes, clamped to the domain
        (ns3d/solver.py:1505-1540); (nz, nx) for "y", (ny, nx) for "z", (nz, ny) for "x"."""
        dim = {"z": 0, "y": 1, "x": 2}[axis]
        n = self.shape[dim]
        origin = float(getattr(self.ops, ("z0", "y0", "x0")[dim], 0.0))
        f = min(max((position - origin) / float(self.ops.h) - 0.5, 0.0), n - 1.0)
        i0 = min(math.floor(f), max(n - 2, 0))
        t = f - i0
        i1 = min(i0 + 1, n - 1)
        full = self.fields(u, v, w, (name,))[name]
        a, b = full.narrow(dim, i0, 1), full.narrow(dim, i1, 1)
        return ((1.0 - t) * a + t * b).squeeze(dim)

    def probe(self, field, pts, off=(0.5, 0.5, 0.5), origin=None):
        """Trilinear samples of ``field`` at points (P, 3) = (x, y, z); entry (k, j, i) of the
        field sits at origin + ((i, j, k) + off) h (off (0, .5, .5) for u-faces and so on)."""
        if origin is None:
            origin = (float(getattr(self.ops, "x0", 0.0)), float(getattr(self.ops, "y0", 0.0)),
                      float(getattr(self.ops, "z0", 0.0)))
        if not (torch.is_tensor(field) and field.device == self.device and field.dtype == self.dtype and field.dim() == 3
                and field.is_contiguous()):
            raise RuntimeError(f"field must be a contiguous 3D {self.dtype} tensor on {self.device}")
        self._check("pts", pts, (pts.shape[0], 3))
        out = torch.empty(pts.shape[0], device=self.device, dtype=self.dtype)
        shape = (C.c_int32 * 3)(*field.shape)
        o = (C.c_double * 3)(*origin)
        f = (C.c_double * 3)(*off)
        check(_lib.lib().aero_ns3d_probe(self._handle, C.c_void_p(field.data_ptr()), shape, o, f,
                                         C.c_void_p(pts.data_ptr()), pts.shape[0], C.c_void_p(out.data_ptr()),
                                         self._stream()), "aero_ns3d_probe")
        return out

    def poisson_solve(self, f, psi=None):
        self._check("f", f, self.shape)
        psi = torch.empty_like(f) if psi is None else psi
        check(_lib.lib().aero_ns3d_poisson_solve(self._handle, C.c_void_p(f.data_ptr()), C.c_void_p(psi.data_ptr()),
                                                 C.c_void_p(self.ws_ptr), self._stream()), "aero_ns3d_poisson_solve")
        return psi

    def project(self, u, v, w):
        """In place (u, v, w) <- projection; returns psi."""
        psi = torch.empty(self.shape, device=self.device, dtype=self.dtype)
        check(_lib.lib().aero_ns3d_project(self._handle, C.c_void_p(u.data_ptr()), C.c_void_p(v.data_ptr()),
                                           C.c_void_p(w.data_ptr()), C.c_void_p(psi.data_ptr()),
                                           C.c_void_p(self.ws_ptr), self._stream()), "aero_ns3d_project")
        return psi

    def closure_counts(self):
        """(cells evaluated, cells that kept WALE) of the closure passes since the workspace was
        initialised (synchronises)."""
        out = (C.c_uint64 * 2)()
        check(_lib.lib().aero_ns3d_closure_counts(self._handle, C.c_void_p(self.ws_ptr), out, self._stream()),
              "aero_ns3d_closure_counts")
        return int(out[0]), int(out[1])

    def status(self) -> int:
        """Device status word of the last step (synchronises): 0, or bit 0 = non-finite value,
        bit 1 = a plane load's wait ran out, bit 2 = a tensor-core wait of the closure ran out."""
        v = C.c_int32()
        check(_lib.lib().aero_ns3d_read_status(self._handle, C.c_void_p(self.ws_ptr), C.byref(v), self._stream()),
              "aero_ns3d_read_status")
        return int(v.value)

    def set_wait_bound(self, spin_limit: int = 0, test_extra_bytes: int = 0) -> None:
        """Polls of a plane wait before the kernel gives up (0: the default); test_extra_bytes > 0
        makes every plane wait for bytes that never arrive (tests of the bound only)."""
        check(_lib.lib().aero_ns3d_set_wait_bound(self._handle, int(spin_limit), int(test_extra_bytes)),
              "aero_ns3d_set_wait_bound")


__all__ = ["Ns3dPlan"]
