"""Mask construction of the 3D step on the GPU (src/aerolume/solvers/ns3d/geometry.py:323-495).

:func:`build_geometry3d` takes the reference's arguments -- ``ImmersedMesh`` items (or
``(vertices, faces)`` pairs) and an ``ops`` with the reference's attribute names -- and
returns a :class:`~aerolume_b200.ns3d.types.Geometry3D` of device tensors computed by
``aero_ns3d_build_masks``: the exact signed distance to each body's triangles
(``grid_signed_distance`` without the shared voxeliser, geometry.py:229-262), the smooth
solid fraction, boundary faces zeroed, the rigid-spin solid velocity and the force and
moment weights.  :func:`body_window3d` is the reference's window rule (with the pitch /
yaw sweep that keeps the window, and any captured graph, across live attitude edits);
:func:`mesh_signed_distance` is geometry.py:126 at arbitrary points.  There is no CPU
fallback: without the CUDA library every call raises.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from .. import _lib
from .._lib import F32, F64, MAX_BODIES, check
from .types import Geometry3D

MASK_SHIFT = 0.32           # ns2d/core.py:61, used by the 3D operators (ns3d/core.py:201)


def _torch_dtype(ops):
    dt = getattr(ops, "dtype", "float32")
    if isinstance(dt, torch.dtype):
        return dt
    return torch.float64 if str(dt) in ("float64", "torch.float64") else torch.float32


def _device(ops, device):
    dev = torch.device(device) if device is not None else torch.device(getattr(ops, "device", None) or "cuda")
    if dev.type != "cuda":
        raise RuntimeError("mask construction runs on a CUDA device only (no CPU fallback)")
    if not torch.cuda.is_available():
        raise RuntimeError("CUDA is not available: mask construction has no CPU fallback")
    return dev if dev.index is not None else torch.device("cuda", torch.cuda.current_device())


def _mesh(b):
    """(vertices (N, 3) float64 numpy or tensor, faces (M, 3) int numpy, omega, center, axis)."""
    if isinstance(b, (tuple, list)):
        v, f = b[0], b[1]
        rot = (0.0, (0.0, 0.0, 0.0), (0.0, 1.0, 0.0))
    else:
        v, f = b.vertices, b.faces
        rot = (float(getattr(b, "omega", 0.0)), tuple(getattr(b, "center", (0.0, 0.0, 0.0))),
               tuple(getattr(b, "axis", (0.0, 1.0, 0.0))))
    f = f.detach().cpu().numpy() if torch.is_tensor(f) else np.asarray(f)
    return v, np.asarray(f, dtype=np.int64).reshape(-1, 3), rot


def _vertices_numpy(v) -> np.ndarray:
    if torch.is_tensor(v):
        return v.detach().cpu().double().numpy().reshape(-1, 3)
    return np.asarray(v, dtype=np.float64).reshape(-1, 3)


def rotation_matrix(pitch_deg: float, yaw_deg: float) -> np.ndarray:
    """Yaw about +z by -yaw, then pitch about +y by +pitch (geometry.py:315-320)."""
    a, b = math.radians(pitch_deg), math.radians(-yaw_deg)
    ry = np.array([[math.cos(a), 0.0, math.sin(a)], [0.0, 1.0, 0.0], [-math.sin(a), 0.0, math.cos(a)]])
    rz = np.array([[math.cos(b), -math.sin(b), 0.0], [math.sin(b), math.cos(b), 0.0], [0.0, 0.0, 1.0]])
    return ry @ rz


def body_window3d(vertex_sets, ops, margin_cells=None, *, pitch_deg=0.0, yaw_deg=0.0):
    """Cell window (k0, k1, j0, j1, i0, i1) of the vertices plus a margin, clipped; with
    pitch / yaw it also covers the bodies rotated about the moment reference by up to
    those angles (geometry.py:323-356)."""
    sets = [_vertices_numpy(v) for v in vertex_sets if len(v)]
    if not sets:
        return (0, 0, 0, 0, 0, 0)
    pts = np.vstack(sets)
    if pitch_deg > 0 or yaw_deg > 0:
        ref = np.asarray(ops.moment_ref, dtype=np.float64)
        rot = []
        for pa in np.linspace(-pitch_deg, pitch_deg, 7 if pitch_deg > 0 else 1):
            for ya in np.linspace(-yaw_deg, yaw_deg, 7 if yaw_deg > 0 else 1):
                rot.append((pts - ref) @ rotation_matrix(pa, ya).T + ref)
        pts = np.vstack(rot)
    width = float(getattr(ops, "mask_width", 1.0))
    shift = float(getattr(ops, "mask_shift", MASK_SHIFT))
    margin = (width + 3.0 + abs(shift)) if margin_cells is None else margin_cells
    h = ops.h
    lo, hi = pts.min(axis=0), pts.max(axis=0)
    i0, i1 = math.floor((lo[0] - ops.x0) / h - margin), math.ceil((hi[0] - ops.x0) / h + margin)
    j0, j1 = math.floor((lo[1] - ops.y0) / h - margin), math.ceil((hi[1] - ops.y0) / h + margin)
    k0, k1 = math.floor((lo[2] - ops.z0) / h - margin), math.ceil((hi[2] - ops.z0) / h + margin)
    i0, i1 = max(i0, 0), min(i1, ops.nx)
    j0, j1 = max(j0, 0), min(j1, ops.ny)
    k0, k1 = max(k0, 0), min(k1, ops.nz)
    if i1 <= i0 or j1 <= j0 or k1 <= k0:
        return (0, 0, 0, 0, 0, 0)
    return (k0, k1, j0, j1, i0, i1)


def _upload_mesh(v, f, dev, dt):
    vt = (v.detach() if torch.is_tensor(v) else torch.as_tensor(_vertices_numpy(v)))
    vt = vt.reshape(-1, 3).to(device=dev, dtype=dt).contiguous()
    if len(f) and (f.min() < 0 or f.max() >= vt.shape[0]):
        raise ValueError("a face names a vertex that does not exist")
    ft = torch.as_tensor(f.astype(np.int32)).to(dev).contiguous()
    return vt, ft


def _workspace(nbytes, dev):
    raw = torch.empty(int(nbytes) + 256, dtype=torch.uint8, device=dev)
    return raw, (raw.data_ptr() + 255) & ~255


def build_geometry3d(bodies, ops, *, window=None, device=None) -> Geometry3D:
    """Masks, solid velocities and force weights of the immersed meshes on the device
    (geometry.py:385-495 with the exact signed distance)."""
    dev = _device(ops, device)
    dt = _torch_dtype(ops)
    nb = len(bodies)
    if nb > MAX_BODIES:
        raise RuntimeError(f"the B200 mask construction supports at most {MAX_BODIES} bodies")
    meshes = [_mesh(b) for b in bodies]
    if window is None:
        window = body_window3d([m[0] for m in meshes], ops)
    window = tuple(int(x) for x in window)
    k0, k1, j0, j1, i0, i1 = window
    wz, wy, wx = k1 - k0, j1 - j0, i1 - i0
    if nb == 0 or wz <= 0 or wy <= 0 or wx <= 0:
        z = torch.zeros(0, 0, 0, device=dev, dtype=dt)
        return Geometry3D((0, 0, 0, 0, 0, 0), z, z, z, z, z, z, z, z, z, z, nb)
    for v, f, _ in meshes:
        if len(f) == 0:
            raise ValueError("a body mesh without faces")
    cfg = _lib.MaskConfig()
    cfg.abi_version = _lib.ABI_VERSION
    cfg.dtype = F64 if dt == torch.float64 else F32
    cfg.nx, cfg.ny, cfg.nz = int(ops.nx), int(ops.ny), int(ops.nz)
    cfg.h, cfg.x0, cfg.y0, cfg.z0 = float(ops.h), float(ops.x0), float(ops.y0), float(ops.z0)
    for a, p in enumerate(getattr(ops, "periodic_axes", (False, False, False))):
        cfg.periodic[a] = int(bool(p))
    for q in range(6):
        cfg.window[q] = window[q]
    cfg.mask_width = float(getattr(ops, "mask_width", 1.0))
    cfg.mask_shift = float(getattr(ops, "mask_shift", MASK_SHIFT))
    for a in range(3):
        cfg.moment_ref[a] = float(ops.moment_ref[a])
    cfg.nbody = nb
    arr = (_lib.MaskBody * nb)()
    keep = []
    for b, (v, f, (om, cen, ax)) in enumerate(meshes):
        vt, ft = _upload_mesh(v, f, dev, dt)
        keep += [vt, ft]
        arr[b].vertices, arr[b].nvert = vt.data_ptr(), vt.shape[0]
        arr[b].faces, arr[b].nface = ft.data_ptr(), ft.shape[0]
        arr[b].omega = float(om)
        for a in range(3):
            arr[b].center[a] = float(cen[a])
            arr[b].axis[a] = float(ax[a])
    kw = dict(device=dev, dtype=dt)
    g = Geometry3D(window,
                   chi_u=torch.empty(wz, wy, wx + 1, **kw), chi_v=torch.empty(wz, wy + 1, wx, **kw),
                   chi_w=torch.empty(wz + 1, wy, wx, **kw), chi_c=torch.empty(wz, wy, wx, **kw),
                   a_u=torch.empty(wz, wy, wx + 1, **kw), a_v=torch.empty(wz, wy + 1, wx, **kw),
                   a_w=torch.empty(wz + 1, wy, wx, **kw),
                   k_u=torch.empty(nb, 3, wz, wy, wx + 1, **kw), k_v=torch.empty(nb, 3, wz, wy + 1, wx, **kw),
                   k_w=torch.empty(nb, 3, wz + 1, wy, wx, **kw), nbody=nb)
    out = _lib.MaskOut()
    for name in ("chi_u", "chi_v", "chi_w", "chi_c", "a_u", "a_v", "a_w", "k_u", "k_v", "k_w"):
        setattr(out, name, getattr(g, name).data_ptr())
    L = _lib.lib()
    nbytes = L.aero_ns3d_masks_workspace_bytes(C.byref(cfg), arr)
    if nbytes == 0:
        check(L.aero_ns3d_build_masks(C.byref(cfg), arr, C.byref(out), None, None), "aero_ns3d_build_masks")
    raw, ptr = _workspace(nbytes, dev)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    check(L.aero_ns3d_build_masks(C.byref(cfg), arr, C.byref(out), C.c_void_p(ptr), stream), "aero_ns3d_build_masks")
    # the uploaded meshes and the workspace go back to torch's stream-ordered allocator: later
    # work on this stream cannot reuse them before the construction has run
    del keep, raw
    return g


def mesh_signed_distance(vertices, faces, points, *, plane_zone: float = 0.0):
    """Exact signed distance (negative inside) of device points (P, 3) to a triangle soup
    (geometry.py:126-196), in the points' dtype, on their device."""
    if not torch.is_tensor(points) or points.device.type != "cuda":
        raise RuntimeError("points must be a CUDA tensor (no CPU fallback)")
    dt = points.dtype
    if dt not in (torch.float32, torch.float64):
        raise RuntimeError("points must be float32 or float64")
    dev = points.device
    f = faces.detach().cpu().numpy() if torch.is_tensor(faces) else np.asarray(faces)
    f = np.asarray(f, dtype=np.int64).reshape(-1, 3)
    if len(f) == 0:
        raise ValueError("a mesh without faces")
    vt, ft = _upload_mesh(vertices, f, dev, dt)
    p = points.detach().reshape(-1, 3).contiguous()
    out = torch.empty(p.shape[0], device=dev, dtype=dt)
    code = F64 if dt == torch.float64 else F32
    L = _lib.lib()
    raw, ptr = _workspace(L.aero_mesh_sdf_workspace_bytes(code, ft.shape[0], p.shape[0]), dev)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    check(L.aero_mesh_signed_distance(code, C.c_void_p(vt.data_ptr()), vt.shape[0], C.c_void_p(ft.data_ptr()),
                                      ft.shape[0], C.c_void_p(p.data_ptr()), p.shape[0], float(plane_zone),
                                      C.c_void_p(out.data_ptr()), C.c_void_p(ptr), stream), "aero_mesh_signed_distance")
    del raw, vt, ft
    return out
