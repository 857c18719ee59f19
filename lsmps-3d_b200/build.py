"""Build recipe of the sm_100a library: nvcc compiles every csrc/*.cu for
compute_100a/sm_100a and links liblsmps_b200.so next to this file (in-tree,
so it travels with the repository snapshot).

    python lsmps-3d_b200/build.py [--force] [--ptxas-verbose]
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


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def _compile(src: str, extra: list[str]) -> str:
    obj = os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and ("--resource-usage" in extra or "-Xptxas=-v" in extra):
        sys.stderr.write(r.stderr)
    return obj


def build_all(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    if not force and not ptxas_verbose and up_to_date():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    extra = ["-Xptxas=-v"] if ptxas_verbose else []
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), sources()))
    tmp = LIB + f".tmp{os.getpid()}"
    cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas-verbose" in sys.argv)
