"""TEST INFRASTRUCTURE: ctypes wrapper of the reference's own CUDA path
(oracle/_ref/libref_lsmps.so, built by `make -C oracle ref` from the reference
sources plus ref_harness.cu).

Used by the GPU parity tests to pin the oracle and the sm_100a path against
the reference's CUDA results on the same inputs, and by bench.py as the
reference timing arm.  The product path never imports it.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_float, c_int, c_longlong, c_size_t, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref_lsmps.so")


def available() -> bool:
    return os.path.exists(LIB)


_lib = None


def lib(abi):
    global _lib
    if _lib is not None:
        return _lib
    if not available():
        raise RuntimeError(f"{LIB} is missing: it is built from the reference sources by `make -C oracle ref`")
    L = ctypes.CDLL(LIB)
    P = POINTER
    sig = {
        "ref_create": (c_void_p, [P(abi.Params), c_size_t, c_size_t, c_size_t, c_size_t]),
        "ref_destroy": (None, [c_void_p]),
        "ref_workspace_bytes": (c_size_t, [c_void_p]),
        "ref_upload": (c_int, [c_void_p, P(abi.Fluid), P(abi.Walls)]),
        "ref_rebuild": (c_int, [c_void_p]),
        "ref_provision": (c_int, [c_void_p]),
        "ref_assemble_ppe": (c_int, [c_void_p]),
        "ref_correction": (c_int, [c_void_p]),
        "ref_steps": (c_int, [c_void_p, c_int, P(c_float)]),
        "ref_download_fluid": (c_int, [c_void_p, P(abi.Fluid)]),
        "ref_download_cells": (c_int, [c_void_p, c_int, P(abi.Cells)]),
        "ref_download_csr": (c_longlong, [c_void_p, c_int, P(abi.Csr)]),
        "ref_download_moment": (c_int, [c_void_p, c_int, P(abi.Moment)]),
        "ref_download_temporary": (c_int, [c_void_p, P(abi.Fluid), P(abi.Walls)]),
        "ref_download_ppe": (c_longlong, [c_void_p, P(abi.Ppe), c_size_t]),
        "ref_download_correction": (c_int, [c_void_p, P(abi.Vector), P(abi.Vector)]),
        "ref_virtual_light": (c_int, [c_void_p, c_void_p, c_void_p]),
        "ref_virtual_light_steps": (c_int, [c_void_p, c_int, P(c_float)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


class ReferencePath:
    """The reference CUDA path on one case, with results copied into a
    numpy-backed StepBuffers of the same shape."""

    def __init__(self, abi, case, host_buffers, max_fluid_neighbors=256, max_wall_neighbors=256):
        self.abi = abi
        self.L = lib(abi)
        self.case = case
        self.b = host_buffers
        self.h = self.L.ref_create(ctypes.byref(case.params), case.n_fluid, case.n_wall, max_fluid_neighbors,
                                   max_wall_neighbors)
        self.L.ref_upload(self.h, ctypes.byref(host_buffers.fluid_view()), ctypes.byref(host_buffers.walls_view()))

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rebuild(self):
        self.L.ref_rebuild(self.h)

    def provision(self):
        self.L.ref_provision(self.h)

    def assemble_ppe(self):
        self.L.ref_assemble_ppe(self.h)

    def correction(self):
        self.L.ref_correction(self.h)

    def steps(self, n: int) -> list[float]:
        ms = (c_float * max(n, 1))()
        self.L.ref_steps(self.h, n, ms)
        return [float(ms[i]) for i in range(n)]

    def workspace_bytes(self) -> int:
        return int(self.L.ref_workspace_bytes(self.h))

    # -- readback into self.b ------------------------------------------------
    def fetch_geometry(self):
        b = self.b
        self.L.ref_download_fluid(self.h, ctypes.byref(b.fluid_view()))
        self.L.ref_download_cells(self.h, 0, ctypes.byref(b.cells_view("fluid")))
        self.L.ref_download_cells(self.h, 1, ctypes.byref(b.cells_view("wall")))
        tf = self.L.ref_download_csr(self.h, 0, ctypes.byref(b.csr_view("fluid")))
        tw = self.L.ref_download_csr(self.h, 1, ctypes.byref(b.csr_view("wall")))
        return int(tf), int(tw)

    def fetch_moments(self, params):
        b = self.b
        b.params_for_moment = params
        for kind in (0, 1):
            self.L.ref_download_moment(self.h, kind, ctypes.byref(b.moment_view(kind)))

    def fetch_provision(self):
        self.L.ref_download_temporary(self.h, ctypes.byref(self.b.temporary_view()),
                                      ctypes.byref(self.b.temporary_walls_view()))

    def fetch_ppe(self, written: int) -> int:
        return int(self.L.ref_download_ppe(self.h, ctypes.byref(self.b.ppe_view()), written))

    def fetch_correction(self):
        b = self.b
        self.L.ref_download_fluid(self.h, ctypes.byref(b.fluid_view()))
        self.L.ref_download_correction(self.h, ctypes.byref(b.vector_view(b.pressure_gradient)),
                                       ctypes.byref(b.vector_view(b.ps_displacement)))

    def virtual_light(self):
        """compute_virtual_light_diagnostics of the reference on its current geometry:
        (open_direction_count int32[N], open_fraction float64[N])."""
        import numpy as np
        n = self.b.n_fluid
        count = np.zeros(n, dtype=np.int32)
        frac = np.zeros(n, dtype=np.float64)
        self.L.ref_virtual_light(self.h, count.ctypes.data, frac.ctypes.data)
        return count, frac

    def virtual_light_steps(self, n: int) -> list[float]:
        """n timed calls of the reference's compute_virtual_light_diagnostics (ms each)."""
        ms = (c_float * n)()
        self.L.ref_virtual_light_steps(self.h, n, ms)
        return [float(ms[i]) for i in range(n)]
