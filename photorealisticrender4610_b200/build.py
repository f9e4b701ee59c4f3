"""Builds libprr.so in-tree: host C++ with g++, kernels with nvcc for sm_100a.

Flags that matter for results:
  --fmad=false (device) and -ffp-contract=off (host): no multiply-add
    contraction, so every float op rounds where the reference's IEEE build
    rounds it (bit-exact slab tests, Möller-Trumbore, camera rays).
  default -prec-div / -prec-sqrt (no --use_fast_math): IEEE division and sqrt.
The library links the CUDA runtime statically and does not link torch.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libprr.so"
# the checked build: the same sources with -DPRR_CHECKED (device-side bounds
# tests on node, triangle, stack and queue indices, reported by prr_check_status)
BUILD_CHECKED = PKG / "_build_checked"
LIB_CHECKED = PKG / "libprr_checked.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr", "-I", str(INCLUDE)]
CXX = os.environ.get("CXX", "/usr/bin/g++")
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-pthread", "-Wall",
             "-Wno-unused-function", "-I", str(CUDA_HOME / "include"), "-I", str(INCLUDE)]


def _sources():
    cu = sorted(CSRC.glob("*.cu"))
    cpp = sorted(CSRC.glob("*.cpp"))
    headers = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))
    return cu, cpp, headers


def _stale(obj: Path, src: Path, headers) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in headers)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ... {cmd[-1]}")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(verbose: bool = False, ptxas_verbose: bool = False, jobs: int = 8,
          checked: bool = False) -> Path:
    """Compile every kernel and host unit and link libprr.so (checked=True:
    libprr_checked.so with -DPRR_CHECKED); returns its path."""
    if not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    out_dir, lib = (BUILD_CHECKED, LIB_CHECKED) if checked else (BUILD, LIB)
    define = ["-DPRR_CHECKED"] if checked else []
    out_dir.mkdir(exist_ok=True)
    cu, cpp, headers = _sources()
    cmds, objs = [], []
    for src in cu:
        obj = out_dir / (src.stem + ".cu.o")
        objs.append(obj)
        if _stale(obj, src, headers):
            extra = ["-Xptxas", "-v"] if ptxas_verbose else []
            cmds.append([NVCC, *ARCH, *NVCC_FLAGS, *define, *extra, "-c", str(src), "-o",
                         str(obj)])
    for src in cpp:
        obj = out_dir / (src.stem + ".o")
        objs.append(obj)
        if _stale(obj, src, headers):
            cmds.append([CXX, *CXX_FLAGS, *define, "-c", str(src), "-o", str(obj)])
    if cmds:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=jobs) as ex:
            list(ex.map(lambda c: _run(c, verbose), cmds))
    if cmds or not lib.exists() or any(o.stat().st_mtime > lib.stat().st_mtime for o in objs):
        tmp = lib.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs),
              "-Xcompiler", "-pthread", "-lz"], verbose)
        shutil.move(str(tmp), str(lib))
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_verbose="--ptxas" in sys.argv,
                checked="--checked" in sys.argv))
