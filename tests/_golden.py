"""Load the committed golden fixtures into the package's containers (test helper)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from aerolume_b200.ns3d.types import DyeSources, Geometry3D, Ops3D, ThermalGeometry, ThermalOps

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES_3D = sorted(p.stem[len("ns3d_"):] for p in GOLDEN.glob("ns3d_*.npz"))


def ops_from_meta(meta, arr):
    """The Ops3D and Geometry3D of a golden case's metadata and arrays."""
    dt = np.float64 if meta["dtype"] == "float64" else np.float32
    ghost = {k: tuple(tuple((r[0], float(r[1])) for r in ax) for ax in v) for k, v in meta["ghost"].items()}
    ops = Ops3D(nx=meta["nx"], ny=meta["ny"], nz=meta["nz"], h=meta["h"], x0=meta["x0"], y0=meta["y0"],
                z0=meta["z0"], periodic_axes=tuple(meta["periodic_axes"]), closed=meta["closed"],
                symmetry=meta["symmetry"], advection=meta["advection"], turbulence=meta["turbulence"],
                les_c=meta["les_c"], nu_value=meta["nu_value"], eta=meta["eta"], cfl=meta["cfl"],
                dt_fixed=meta["dt_fixed"], ghost=ghost, u_inlet=arr["u_inlet"].astype(dt),
                ref_area=meta["ref_area"], length_ref=meta["length_ref"], span_ref=meta["span_ref"],
                moment_ref=tuple(meta["moment_ref"]), dtype=meta["dtype"],
                forcing=tuple(meta["forcing"]) if meta.get("forcing") else None)
    win = tuple(meta["window"])
    geom = Geometry3D(win, nbody=meta["nbody"])
    if not geom.empty:
        for n in ("chi_u", "chi_v", "chi_w", "chi_c", "a_u", "a_v", "a_w", "k_u", "k_v", "k_w"):
            setattr(geom, n, arr[n].astype(dt))
    return ops, geom


def load_case(name):
    z = np.load(GOLDEN / f"ns3d_{name}.npz")
    meta = json.loads(str(z["meta"]))
    arr = {k: z[k] for k in z.files if k != "meta"}
    ops, geom = ops_from_meta(meta, arr)
    dt = np.float64 if meta["dtype"] == "float64" else np.float32
    win = tuple(meta["window"])
    th = None
    if "thermal" in meta:
        t = meta["thermal"]
        adia = tuple(arr["th_adia_" + c].astype(dt) for c in "uvw") if "th_adia_u" in arr else None
        tg = ThermalGeometry(win, nbody=meta["nbody"], chi_t=arr.get("th_chi_t"), a_t=arr.get("th_a_t"),
                             w_t=arr.get("th_w_t"), t_index=list(t["t_index"]), adia=adia,
                             vol_w=arr.get("th_vol_w"), skin=arr.get("th_skin"),
                             flux_rate=np.asarray(t["flux_rate"], np.float64))
        th = ThermalOps(kappa=t["kappa"], pe=t["pe"], ri=t["ri"], prt=t["prt"], eta=t["eta"],
                        side_kinds=tuple(t["side_kinds"]), side_vals=tuple(t["side_vals"]), geom=tg,
                        h=meta["h"], symmetry=meta["symmetry"], heat_max=t["heat_max"],
                        sources=tuple((tuple(w), arr[f"th_src{q}"].astype(dt)) for q, w in enumerate(t.get("sources", []))))
    src = None
    if "dye" in meta:
        src = DyeSources(tuple(meta["dye"]["window"]), arr["dye_weight"].astype(dt), tuple(meta["dye"]["pulse"]))
    return meta, ops, geom, th, src, arr


def fan_items(meta, arr):
    """Per-fan windows and weights of a golden case (numpy, the case dtype):
    [{"win", "fu".."fw", "su".."sw", "mu".."mw"}]."""
    dt = np.float64 if meta["dtype"] == "float64" else np.float32
    out = []
    for q, win in enumerate(meta["fans"]["win"]):
        it = {"win": tuple(win)}
        for kind in "fsm":
            for g in "uvw":
                it[kind + g] = arr[f"fan{q}_{kind}{g}"].astype(dt)
        out.append(it)
    return out


def port_items(meta, arr):
    """Per-port windows, kinds, temperatures and weights of a golden case (numpy, the case
    dtype): [{"win", "kind", "theta", "m", "fu", "fv", "fw"}]."""
    dt = np.float64 if meta["dtype"] == "float64" else np.float32
    out = []
    for q, it in enumerate(meta["ports"]["items"]):
        d = {"win": tuple(it["win"]), "kind": it["kind"], "theta": it["theta"], "m": arr[f"port{q}_m"].astype(dt)}
        for g in "uvw":
            d["f" + g] = arr[f"port{q}_f{g}"].astype(dt)
        out.append(d)
    return out


CASES_2D = sorted(p.stem[len("ns2d_"):] for p in GOLDEN.glob("ns2d_*.npz"))


def load_case2d(name):
    from aerolume_b200.ns2d.types import Geometry2D, Ops2D
    z = np.load(GOLDEN / f"ns2d_{name}.npz")
    meta = json.loads(str(z["meta"]))
    arr = {k: z[k] for k in z.files if k != "meta"}
    dt = np.float64 if meta["dtype"] == "float64" else np.float32
    ops = Ops2D(nx=meta["nx"], ny=meta["ny"], h=meta["h"], x0=meta["x0"], y0=meta["y0"], periodic=meta["periodic"],
                closed=meta["closed"], bc_top=meta["bc_top"], bc_bottom=meta["bc_bottom"], bc_left=meta["bc_left"],
                bc_right=meta["bc_right"], ground_speed=meta["ground_speed"], advection=meta["advection"],
                turbulence=meta["turbulence"], les_c=meta["les_c"], nu=meta["nu"], eta=meta["eta"], cfl=meta["cfl"],
                dt_fixed=meta["dt_fixed"], u_inlet=arr["u_inlet"].astype(dt),
                dye_inlet=arr["dye_inlet"].astype(dt) if "dye_inlet" in arr else None,
                force_ref=meta["force_ref"], moment_ref=tuple(meta["moment_ref"]), dtype=meta["dtype"],
                wall_model=bool(meta.get("wall_model", False)),
                forcing=tuple(meta["forcing"]) if meta.get("forcing") else None)
    geom = Geometry2D(tuple(meta["window"]), nbody=meta["nbody"])
    if not geom.empty:
        for n in ("chi_u", "chi_v", "chi_c", "a_u", "a_v", "k_u", "k_v"):
            setattr(geom, n, arr[n].astype(dt))
    return meta, ops, geom, arr


def load_fields_case(tag):
    """(ops, geom, arrays) of one case of fields3d.npz (arrays without the tag prefix)."""
    z = np.load(GOLDEN / "fields3d.npz")
    meta = json.loads(str(z[f"{tag}_meta"]))
    arr = {k[len(tag) + 1:]: z[k] for k in z.files if k.startswith(tag + "_") and k != f"{tag}_meta"}
    ops, geom = ops_from_meta(meta, arr)
    ops.x0, ops.y0, ops.z0 = meta["origin"]
    return meta, ops, geom, arr


def thermal2d_from_case(meta, arr):
    """The oracle's Thermal2D of a 2D golden case with heat transfer (None without)."""
    from oracle.ns2d import Thermal2D
    t = meta.get("thermal")
    if t is None:
        return None
    dt = np.float64 if meta["dtype"] == "float64" else np.float32
    g = {n: (arr["th_" + n].astype(dt) if "th_" + n in arr else None)
         for n in ("chi_t", "a_t", "w_t", "ins_u", "ins_v", "q_skin", "w_f", "vol_u", "vol_v")}
    return Thermal2D(kappa=t["kappa"], ri=t["ri"], prt=t["prt"], gravity=tuple(t["gravity"]), eta_t=t["eta_t"],
                     theta_in=t["theta_in"], wall_modes=tuple(t["wall_modes"]), wall_values=tuple(t["wall_values"]),
                     diff_coef=t["diff_coef"], temp_ids=tuple(t.get("temp_ids", ())),
                     flux_ids=tuple(t.get("flux_ids", ())), **g)


def placed2d_from_case(meta, arr):
    """The oracle's Placed2D (fans, heaters, paint, the PID step) of a 2D golden case, or None."""
    from oracle.ns2d import Placed2D
    pm = meta.get("placed")
    if pm is None or not (pm["nfan"] or pm["pid"] or pm["paint"] or pm["heat"] or pm.get("ports") or pm.get("n_dye")):
        return None
    dt = np.float64 if meta["dtype"] == "float64" else np.float32
    kw = {n: arr[n].astype(dt) for n in ("fan_gu", "fan_gv", "fan_phi", "fan_dir", "fan_value", "fan_width", "fan_kp",
                                         "fan_ki", "fan_dpmax", "fan_isvel", "fan_isthrust", "heat", "paint_c",
                                         "paint_u", "paint_v", "paint_wu", "paint_wv", "xchi_u", "xa_u", "xchi_v",
                                         "xa_v", "src", "src_neg", "pt_chi", "pt_a") if n in arr}
    pl = Placed2D(nfan=pm["nfan"], pid=pm["pid"], u_floor=pm["u_floor"], heat_max=pm.get("heat_max"),
                  ports=bool(pm.get("ports")), q_net=pm.get("q_net", 0.0), **kw)
    if pm.get("n_dye"):
        pl.n_dye = pm["n_dye"]
        pl.dye_inflow = arr["dye_inflow"].astype(dt)
        pl.groups = [(ch, arr[f"group{q}_w"].astype(dt), arr[f"group{q}_target"].astype(dt),
                      arr[f"group{q}_timing"].astype(dt)) for q, ch in enumerate(pm["groups"])]
        pl.port_dye = {c: arr[f"port_dye{c}"].astype(dt) for c in pm["port_dye"]}
    return pl


def load_masks():
    """(npz, case tags) of masks3d.npz."""
    z = np.load(GOLDEN / "masks3d.npz")
    return z, json.loads(str(z["cases"]))


def masks_case(z, tag):
    """(meta, ops namespace with the reference's attribute names, bodies) of one mask case."""
    from types import SimpleNamespace
    meta = json.loads(str(z[f"{tag}_meta"]))
    ops = SimpleNamespace(nx=meta["nx"], ny=meta["ny"], nz=meta["nz"], h=meta["h"], x0=meta["origin"][0],
                          y0=meta["origin"][1], z0=meta["origin"][2], periodic_axes=tuple(meta["periodic_axes"]),
                          moment_ref=tuple(meta["moment_ref"]), mask_width=meta["mask_width"],
                          mask_shift=meta["mask_shift"], dtype=meta["dtype"])
    bodies = [SimpleNamespace(vertices=z[f"{tag}_v{q}"], faces=z[f"{tag}_f{q}"], omega=b["omega"],
                              center=tuple(b["center"]), axis=tuple(b["axis"])) for q, b in enumerate(meta["bodies"])]
    return meta, ops, bodies
