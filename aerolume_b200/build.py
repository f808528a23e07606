"""Build ``libaero_b200.so`` in-tree with nvcc for sm_100a (the only target).

    python -m aerolume_b200.build            # incremental: rebuilds when a source is newer
    python -m aerolume_b200.build --force
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libaero_b200.so"
LIB_CHECKED = PKG / "libaero_b200_checked.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O3",
         "-Xptxas", "-O3"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found (CUDA 12.9+ with sm_100a support is required)")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def stale(lib: Path = LIB) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h")) + [Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> Path:
    """Compile the release library, or with ``checked`` the bounds-checked one
    (AERO_BOUNDS_CHECK: every instrumented index is checked on the device)."""
    lib = LIB_CHECKED if checked else LIB
    if not force and not stale(lib):
        return lib
    build_dir = PKG / ("_build_checked" if checked else "_build")
    build_dir.mkdir(exist_ok=True)
    cc = nvcc()
    cmds, objs = [], []
    for src in sources():
        obj = build_dir / (src.stem + ".o")
        cmd = [cc, *ARCH, *FLAGS, "-I", str(INCLUDE), "-dc", "-c", str(src), "-o", str(obj)]
        if checked:
            cmd.append("-DAERO_BOUNDS_CHECK=1")
        if verbose:
            cmd += ["-Xptxas", "-v"]
        cmds.append(cmd)
        objs.append(str(obj))
    # one nvcc per translation unit, in parallel
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c, capture_output=not verbose, text=True), cmds)):
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed: {' '.join(r.args)}\n{r.stdout or ''}{r.stderr or ''}")
    tmp = lib.with_suffix(".so.tmp")
    subprocess.run([cc, *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", str(tmp), "-lcudart"], check=True)
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true", help="print ptxas register / spill reports")
    ap.add_argument("--checked", action="store_true", help="build libaero_b200_checked.so (device bounds checks)")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, checked=a.checked))
    sys.exit(0)
