"""ctypes binding of ``libaero_b200.so`` (declarations in ``include/aero_b200.h``).

The library is built in-tree (``python -m aerolume_b200.build``).  There is no fallback:
:func:`lib` raises ``RuntimeError`` when the library is missing or cannot be loaded, and
every call that returns a negative status raises ``RuntimeError`` with the library's
message (``aero_last_error``).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import os

LIB_PATH = Path(__file__).resolve().parent / (
    "libaero_b200_checked.so" if os.environ.get("AERO_B200_CHECKED") == "1" else "libaero_b200.so")
ABI_VERSION = 6
MAX_BODIES = 8
MAX_FANS = 4
MAX_PORTS = 4
MAX_HEATERS = 4
TRACE_EVENTS = 19
# output fields of aero_ns3d_fields, in its order
FIELD_NAMES = ("uc", "vc", "wc", "speed", "vorticity", "q", "nut")

F32, F64 = 0, 1
ADV = {"upwind3": 0, "central": 1}
LES = {"none": 0, "laminar": 0, "smagorinsky": 1, "wale": 2, "vreman": 3}
GHOST = {"edge": 0, "even": 1, "odd": 2, "affine": 3, "face_odd": 4, "periodic_cell": 5, "periodic_face": 6}
THETA_SIDE = {"periodic": 0, "outflow": 1, "adiabatic": 2, "inflow": 3, "temperature": 4, "heat_flux": 5}
THETA2_MODE = {"adiabatic": 0, "temperature": 1, "heat_flux": 2, "inlet": 3, "outlet": 4, "periodic": 5}

# every symbol include/aero_b200.h declares
EXPORTS = ("aero_abi_version", "aero_last_error", "aero_ns3d_plan_create", "aero_ns3d_plan_destroy",
           "aero_ns3d_workspace_bytes", "aero_ns3d_workspace_init", "aero_ns3d_step", "aero_ns3d_step_traced",
           "aero_ns3d_smoke",
           "aero_ns3d_poisson_solve",
           "aero_ns3d_project", "aero_ns3d_read_status", "aero_debug_check", "aero_ns3d_poisson_solve_static",
           "aero_ns2d_plan_create", "aero_ns2d_plan_destroy", "aero_ns2d_workspace_bytes",
           "aero_ns2d_workspace_init", "aero_ns2d_step", "aero_ns2d_poisson_solve", "aero_ns3d_fields",
           "aero_ns3d_probe", "aero_ns3d_masks_workspace_bytes", "aero_ns3d_build_masks",
           "aero_mesh_sdf_workspace_bytes", "aero_mesh_signed_distance", "aero_record_history", "aero_welford",
           "aero_smoke_emitters", "aero_closure_pairs", "aero_closure_features", "aero_closure_normalise",
           "aero_mlp_forward", "aero_mlp_train_workspace_bytes", "aero_mlp_gradients", "aero_mlp_train_step",
           "aero_closure_eddy_viscosity", "aero_ns3d_closure_counts", "aero_ns2d_sweep_create",
           "aero_ns2d_sweep_destroy", "aero_ns2d_sweep_workspace_bytes", "aero_ns2d_sweep_init",
           "aero_ns2d_sweep_step", "aero_ns2d_sweep_read_status", "aero_ns2d_sweep_set_barrier",
           "aero_ns2d_sweep_info", "aero_ns3d_set_wait_bound")

CLOSURE_IN, CLOSURE_OUT, CLOSURE_HIDDEN, CLOSURE_NPARAM = 10, 6, 128, 35206


class Ns3dConfig(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("dtype", C.c_int32),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("h", C.c_double),
        ("periodic", C.c_int32 * 3), ("closed", C.c_int32), ("symmetry", C.c_int32),
        ("advection", C.c_int32), ("les", C.c_int32), ("les_c", C.c_double),
        ("nu", C.c_double), ("eta", C.c_double), ("cfl", C.c_double),
        ("has_dt_fixed", C.c_int32), ("dt_fixed", C.c_double),
        ("ghost_kind", ((C.c_int32 * 2) * 3) * 3), ("ghost_val", ((C.c_double * 2) * 3) * 3),
        ("ref_area", C.c_double), ("length_ref", C.c_double), ("span_ref", C.c_double),
        ("moment_ref", C.c_double * 3), ("y0", C.c_double),
        ("window", C.c_int32 * 6), ("nbody", C.c_int32),
        ("thermal", C.c_int32), ("kappa", C.c_double), ("pe", C.c_double), ("ri", C.c_double),
        ("prt", C.c_double), ("eta_t", C.c_double),
        ("side_kind", C.c_int32 * 6), ("side_val", C.c_double * 6),
        ("has_heat_max", C.c_int32), ("heat_max", C.c_double),
        ("n_tbody", C.c_int32), ("t_index", C.c_int32 * MAX_BODIES),
        ("has_adia", C.c_int32), ("has_skin", C.c_int32),
        ("flux_rate", C.c_double * MAX_BODIES),
        ("smoke", C.c_int32), ("dye_window", C.c_int32 * 6),
        ("pulse_on", C.c_double), ("pulse_period", C.c_double),
        ("u_floor", C.c_double), ("pid", C.c_int32), ("pid_target", C.c_double), ("paint", C.c_int32),
        ("nfan", C.c_int32), ("fan_swirl", C.c_int32),
        ("nport", C.c_int32), ("port_source", C.c_double), ("port_leak", C.c_double), ("nheat", C.c_int32),
        ("closure", C.c_int32), ("forcing", C.c_int32), ("force", C.c_double * 3),
    ]


class Ns3dFan(C.Structure):
    _fields_ = [("window", C.c_int32 * 6), ("velocity_mode", C.c_int32),
                ("target", C.c_double), ("kp", C.c_double), ("ki", C.c_double), ("tmax", C.c_double),
                ("swirl", C.c_double)] + [(n, C.c_void_p) for n in (
                    "f_u", "f_v", "f_w", "s_u", "s_v", "s_w", "m_u", "m_v", "m_w",
                    "thrust", "ud", "e_prev", "swirl_amp")]


class Ns3dPort(C.Structure):
    _fields_ = [("window", C.c_int32 * 6), ("vent", C.c_int32), ("theta", C.c_double)] + \
        [(n, C.c_void_p) for n in ("f_u", "f_v", "f_w", "m")]


class Ns3dHeater(C.Structure):
    _fields_ = [("window", C.c_int32 * 6), ("q", C.c_void_p)]


class Ns3dGeom(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "chi_u", "chi_v", "chi_w", "chi_c", "a_u", "a_v", "a_w", "k_u", "k_v", "k_w",
        "chi_t", "a_t", "w_t", "adia_u", "adia_v", "adia_w", "vol_w", "skin", "dye_weight", "u_inlet",
        "paint_u", "paint_v", "paint_w", "paint_c")] + \
        [("fans", C.c_void_p), ("ports", C.c_void_p), ("heaters", C.c_void_p), ("closure", C.c_void_p)]


class SweepTuning(C.Structure):
    _fields_ = [("lcap", C.c_int32), ("ctas_per_sm", C.c_int32), ("order", C.c_int32), ("schedule", C.c_int32),
                ("tiles", C.c_int32)]


class ClosureModel(C.Structure):
    _fields_ = [("params", C.c_void_p), ("params_bf16", C.c_void_p),
                ("in_mean", C.c_float * 10), ("in_std", C.c_float * 10), ("in_lo", C.c_float * 10),
                ("in_hi", C.c_float * 10), ("out_mean", C.c_float * 6), ("out_std", C.c_float * 6)]


class Ns3dFields(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "u0", "v0", "w0", "theta0", "dye0", "t0",
        "u", "v", "w", "p", "theta", "dye", "t", "dt", "coeffs", "heat_rate", "pid_dt_prev", "pid_e1", "pid_e2",
        "div_sq")]


class Ns2dConfig(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("dtype", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32),
        ("h", C.c_double), ("periodic", C.c_int32), ("closed", C.c_int32),
        ("advection", C.c_int32), ("les", C.c_int32), ("les_c", C.c_double),
        ("nu", C.c_double), ("eta", C.c_double), ("cfl", C.c_double),
        ("has_dt_fixed", C.c_int32), ("dt_fixed", C.c_double),
        ("ghost_kind", ((C.c_int32 * 2) * 2) * 2), ("ghost_val", ((C.c_double * 2) * 2) * 2),
        ("force_ref", C.c_double), ("window", C.c_int32 * 4), ("nbody", C.c_int32), ("dye", C.c_int32),
        ("thermal", C.c_int32), ("kappa", C.c_double), ("ri", C.c_double), ("prt", C.c_double),
        ("gravity", C.c_double * 2), ("eta_t", C.c_double), ("theta_in", C.c_double),
        ("wall_mode", C.c_int32 * 4), ("wall_value", C.c_double * 4), ("diff_coef", C.c_double),
        ("n_temp", C.c_int32), ("n_flux", C.c_int32), ("has_ins", C.c_int32), ("has_vol", C.c_int32),
        ("nfan", C.c_int32), ("heaters", C.c_int32), ("paint", C.c_int32), ("pid", C.c_int32),
        ("ports", C.c_int32), ("dye_channels", C.c_int32), ("n_groups", C.c_int32),
        ("group_channel", C.c_int32 * 8), ("wall_model", C.c_int32), ("wall_ground_speed", C.c_double),
        ("forcing", C.c_int32), ("force", C.c_double * 2),
    ]


class Ns2dGeom(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("chi_u", "chi_v", "chi_c", "a_u", "a_v", "k_u", "k_v", "u_inlet",
                                          "dye_inlet", "chi_t", "a_t", "w_t", "ins_u", "ins_v", "q_skin", "w_f",
                                          "vol_u", "vol_v", "nu", "eta", "kappa", "eta_t", "fan_gu", "fan_gv",
                                          "fan_phi", "fan_dir", "fan_value", "fan_width", "fan_kp", "fan_ki",
                                          "fan_dpmax", "fan_isvel", "fan_isthrust", "u_floor", "heat", "heat_max",
                                          "paint_c", "paint_u", "paint_v", "paint_wu", "paint_wv", "xchi_u", "xa_u",
                                          "xchi_v", "xa_v", "src", "src_neg", "q_net", "pt_chi", "pt_a",
                                          "dye_inflow")] + [
        ("group_w", C.c_void_p * 8), ("group_target", C.c_void_p * 8), ("group_timing", C.c_void_p * 8),
        ("port_dye", C.c_void_p * 4)]


class Ns2dFields(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("u0", "v0", "t0", "dye0", "u", "v", "p", "t", "dt", "dye", "coeffs",
                                          "theta0", "theta", "heat", "theta_wall", "wall_heat", "heat_storage",
                                          "flow_heat", "dt_prev", "ctrl0", "ctrl", "fan_thrust", "fan_ud",
                                          "paint_force", "jet_heat", "vent_heat", "dye_extra0", "dye_extra")]


class SmokeEmitter(C.Structure):
    _fields_ = [("window", C.c_int32 * 6), ("channel", C.c_int32), ("weight", C.c_void_p), ("params", C.c_void_p)]


class MaskConfig(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("dtype", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("h", C.c_double), ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double),
        ("periodic", C.c_int32 * 3), ("window", C.c_int32 * 6), ("mask_width", C.c_double),
        ("mask_shift", C.c_double), ("moment_ref", C.c_double * 3), ("nbody", C.c_int32),
    ]


class MaskBody(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("nvert", C.c_int32), ("faces", C.c_void_p), ("nface", C.c_int32),
                ("omega", C.c_double), ("center", C.c_double * 3), ("axis", C.c_double * 3)]


class MaskOut(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("chi_u", "chi_v", "chi_w", "chi_c", "a_u", "a_v", "a_w", "k_u", "k_v",
                                          "k_w")]


_LIB = None


def lib() -> C.CDLL:
    """The loaded library (raises RuntimeError when it is missing: no fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH.name} is not built; run `python -m aerolume_b200.build` "
                           "(the B200 step has no CPU fallback)")
    try:
        L = C.CDLL(str(LIB_PATH))
    except OSError as exc:
        raise RuntimeError(f"cannot load {LIB_PATH}: {exc}") from exc
    L.aero_abi_version.restype = C.c_int
    L.aero_last_error.restype = C.c_char_p
    L.aero_ns3d_plan_create.argtypes = [C.POINTER(Ns3dConfig), C.POINTER(C.c_void_p)]
    L.aero_ns3d_plan_destroy.argtypes = [C.c_void_p]
    L.aero_ns3d_plan_destroy.restype = None
    L.aero_ns3d_workspace_bytes.argtypes = [C.c_void_p]
    L.aero_ns3d_workspace_bytes.restype = C.c_size_t
    L.aero_ns3d_workspace_init.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.aero_ns3d_step.argtypes = [C.c_void_p, C.POINTER(Ns3dFields), C.POINTER(Ns3dGeom), C.c_void_p, C.c_void_p,
                                 C.c_void_p]
    L.aero_ns3d_step_traced.argtypes = [C.c_void_p, C.POINTER(Ns3dFields), C.POINTER(Ns3dGeom), C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p), C.c_int32]
    L.aero_ns3d_smoke.argtypes = [C.c_void_p, C.POINTER(Ns3dFields), C.POINTER(Ns3dGeom), C.c_void_p]
    L.aero_ns3d_poisson_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.aero_ns3d_project.argtypes = [C.c_void_p] + [C.c_void_p] * 6
    L.aero_ns3d_read_status.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.c_void_p]
    L.aero_debug_check.argtypes = [C.POINTER(C.c_int64)]
    L.aero_ns3d_poisson_solve_static.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.aero_ns2d_plan_create.argtypes = [C.POINTER(Ns2dConfig), C.POINTER(C.c_void_p)]
    L.aero_ns2d_plan_destroy.argtypes = [C.c_void_p]
    L.aero_ns2d_plan_destroy.restype = None
    L.aero_ns2d_workspace_bytes.argtypes = [C.c_void_p]
    L.aero_ns2d_workspace_bytes.restype = C.c_size_t
    L.aero_ns2d_workspace_init.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.aero_ns2d_step.argtypes = [C.c_void_p, C.POINTER(Ns2dFields), C.POINTER(Ns2dGeom), C.c_void_p, C.c_void_p,
                                 C.c_void_p]
    L.aero_ns2d_poisson_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.aero_ns3d_fields.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Ns3dGeom),
                                   C.POINTER(C.c_void_p), C.c_void_p]
    L.aero_ns3d_probe.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                  C.POINTER(C.c_double), C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    L.aero_ns3d_masks_workspace_bytes.argtypes = [C.POINTER(MaskConfig), C.POINTER(MaskBody)]
    L.aero_ns3d_masks_workspace_bytes.restype = C.c_size_t
    L.aero_ns3d_build_masks.argtypes = [C.POINTER(MaskConfig), C.POINTER(MaskBody), C.POINTER(MaskOut), C.c_void_p,
                                        C.c_void_p]
    L.aero_ns3d_build_masks.restype = C.c_int
    L.aero_mesh_sdf_workspace_bytes.argtypes = [C.c_int32, C.c_int32, C.c_int64]
    L.aero_mesh_sdf_workspace_bytes.restype = C.c_size_t
    L.aero_mesh_signed_distance.argtypes = [C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                                            C.c_int64, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    L.aero_mesh_signed_distance.restype = C.c_int
    L.aero_record_history.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                      C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                      C.c_void_p, C.c_void_p]
    L.aero_record_history.restype = C.c_int
    L.aero_welford.argtypes = [C.c_int32, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                               C.POINTER(C.c_void_p), C.POINTER(C.c_int64), C.c_void_p, C.c_void_p, C.c_void_p]
    L.aero_welford.restype = C.c_int
    L.aero_smoke_emitters.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_void_p), C.c_int32,
                                      C.POINTER(SmokeEmitter), C.c_int32, C.c_void_p, C.c_void_p]
    L.aero_smoke_emitters.restype = C.c_int
    L.aero_debug_check.restype = C.c_int
    vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int32
    L.aero_closure_pairs.argtypes = [i32, i32, vp, vp, vp, C.c_double, vp, vp, vp, vp]
    L.aero_closure_features.argtypes = [i64, vp, C.c_double, vp, vp, vp, vp, vp, vp]
    L.aero_closure_normalise.argtypes = [i64, vp, vp, C.POINTER(ClosureModel), vp, vp, vp]
    L.aero_mlp_forward.argtypes = [C.POINTER(ClosureModel), vp, i64, vp, vp, vp]
    L.aero_mlp_train_workspace_bytes.argtypes = [i32]
    L.aero_mlp_train_workspace_bytes.restype = C.c_size_t
    L.aero_mlp_train_step.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i32, i32, C.c_float, vp, vp, vp, vp]
    L.aero_ns3d_closure_counts.argtypes = [vp, vp, C.POINTER(C.c_uint64), vp]
    L.aero_mlp_gradients.argtypes = [vp, vp, vp, vp, vp, vp, i32, vp, vp, vp, vp]
    L.aero_closure_eddy_viscosity.argtypes = [C.POINTER(ClosureModel), vp, i64, C.c_double, vp, vp, vp, vp, vp]
    L.aero_ns2d_sweep_create.argtypes = [i32, C.POINTER(vp), C.POINTER(Ns2dFields), C.POINTER(Ns2dGeom),
                                         C.POINTER(vp), C.POINTER(SweepTuning), C.POINTER(vp)]
    L.aero_ns2d_sweep_destroy.argtypes = [vp]
    L.aero_ns2d_sweep_destroy.restype = None
    L.aero_ns2d_sweep_workspace_bytes.argtypes = [vp]
    L.aero_ns2d_sweep_workspace_bytes.restype = C.c_size_t
    L.aero_ns2d_sweep_init.argtypes = [vp, vp, vp]
    L.aero_ns2d_sweep_step.argtypes = [vp, vp, vp]
    L.aero_ns2d_sweep_read_status.argtypes = [vp, vp, C.POINTER(C.c_int32), vp]
    L.aero_ns2d_sweep_set_barrier.argtypes = [vp, i32, i32]
    L.aero_ns3d_set_wait_bound.argtypes = [vp, i32, i32]
    L.aero_ns3d_set_wait_bound.restype = C.c_int
    L.aero_ns2d_sweep_info.argtypes = [vp, C.POINTER(C.c_int64)]
    for name in ("aero_ns2d_sweep_create", "aero_ns2d_sweep_init", "aero_ns2d_sweep_step", "aero_ns2d_sweep_read_status",
                 "aero_ns2d_sweep_set_barrier", "aero_ns2d_sweep_info"):
        getattr(L, name).restype = C.c_int
    for name in ("aero_closure_pairs", "aero_closure_features", "aero_closure_normalise", "aero_mlp_forward",
                 "aero_mlp_gradients", "aero_mlp_train_step", "aero_closure_eddy_viscosity",
                 "aero_ns3d_closure_counts"):
        getattr(L, name).restype = C.c_int
    for name in ("aero_ns3d_plan_create", "aero_ns3d_workspace_init", "aero_ns3d_step", "aero_ns3d_step_traced",
                 "aero_ns3d_smoke",
                 "aero_ns3d_poisson_solve",
                 "aero_ns3d_project", "aero_ns3d_read_status", "aero_debug_check", "aero_ns3d_poisson_solve_static",
                 "aero_ns2d_plan_create", "aero_ns2d_workspace_init", "aero_ns2d_step", "aero_ns2d_poisson_solve",
                 "aero_ns3d_fields", "aero_ns3d_probe"):
        getattr(L, name).restype = C.c_int
    if L.aero_abi_version() != ABI_VERSION:
        raise RuntimeError(f"{LIB_PATH.name} has ABI {L.aero_abi_version()}, expected {ABI_VERSION}; rebuild it")
    _LIB = L
    return L


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib().aero_last_error().decode(errors="replace")
        kind = {-1: "invalid argument", -2: "unsupported", -3: "CUDA error"}.get(rc, f"error {rc}")
        raise RuntimeError(f"{what}: {kind}: {msg}")
