"""Build recipe of the sm_100a library: nvcc compiles every csrc/*.cu for
compute_100a/sm_100a and links liblsmps_b200.so next to this file (in-tree,
so it travels with the repository snapshot).  --bounds-check builds the
checked variant liblsmps_b200_checked.so (-DLSMPS_BOUNDS_CHECK: every
neighbour table and PPE matrix is validated on the device before a kernel
reads it, and a bad entry is returned as LSMPS_INVALID_ARGUMENT).

    python lsmps-3d_b200/build.py [--force] [--ptxas-verbose] [--bounds-check]
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
OBJ_DIR = os.path.join(PKG_DIR, "_build")
LIB = os.path.join(PKG_DIR, "liblsmps_b200.so")
CHECKED_LIB = os.path.join(PKG_DIR, "liblsmps_b200_checked.so")
CHECKED_OBJ_DIR = os.path.join(PKG_DIR, "_build_checked")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
         "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC, "-DLSMPS_BUILDING_LIBRARY"]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps() -> list[str]:
    return sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(INCLUDE, "lsmps_b200.h"),
                                                                 os.path.abspath(__file__)]


def up_to_date(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(d) <= t for d in _deps())


def _compile(src: str, extra: list[str], obj_dir: str = OBJ_DIR) -> str:
    obj = os.path.join(obj_dir, os.path.basename(src)[:-3] + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and ("--resource-usage" in extra or "-Xptxas=-v" in extra):
        sys.stderr.write(r.stderr)
    return obj


def build_all(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False,
              bounds_check: bool = False) -> str:
    lib = CHECKED_LIB if bounds_check else LIB
    obj_dir = CHECKED_OBJ_DIR if bounds_check else OBJ_DIR
    if not force and not ptxas_verbose and up_to_date(lib):
        return lib
    os.makedirs(obj_dir, exist_ok=True)
    extra = ["-Xptxas=-v"] if ptxas_verbose else []
    if bounds_check:
        extra.append("-DLSMPS_BOUNDS_CHECK")
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra, obj_dir), sources()))
    tmp = lib + f".tmp{os.getpid()}"
    cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib)
    if verbose:
        print(f"built {lib}")
    return lib


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas-verbose" in sys.argv,
              bounds_check="--bounds-check" in sys.argv)
