"""TEST INFRASTRUCTURE: ctypes wrapper of the CPU oracle (lsmps_oracle.cpp).

Only tests/, __graft_entry__.smoke() and the cpu_baseline / reference legs of
bench.py use this module, and only as the checker or the timed CPU baseline.
The product path never imports it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_size_t, c_uint64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "lsmps_oracle.cpp")
LIB = os.path.join(HERE, "_build", "liblsmps_oracle.so")
HEADER = os.path.join(ROOT, "include", "lsmps_b200.h")


def build(force: bool = False) -> str:
    """Compile the oracle (g++ -O3 -fopenmp -ffp-contract=off).  Generic
    x86-64 code: the library travels to other hosts."""
    newest = max(os.path.getmtime(SRC), os.path.getmtime(HEADER))
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    tmp = LIB + f".tmp{os.getpid()}"
    cmd = ["g++", "-std=c++17", "-O3", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
           "-I" + os.path.join(ROOT, "include"), SRC, "-o", tmp]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


_lib = None


def lib(abi):
    global _lib
    if _lib is not None:
        return _lib
    build()
    L = ctypes.CDLL(LIB)
    P = POINTER
    sig = {
        "oracle_build_cell_list": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t, P(abi.Grid), P(abi.Cells)]),
        "oracle_build_neighbor_lists": (c_int, [P(abi.Fluid), P(abi.Walls), P(abi.Params), P(abi.Cells),
                                                P(abi.Cells), P(abi.Csr), P(abi.Csr), P(c_uint64)]),
        "oracle_reference_number_density": (c_double, [c_double, c_double]),
        "oracle_classify_surface": (c_int, [P(abi.Fluid), P(abi.Walls), P(abi.Csr), P(abi.Csr), P(abi.Params),
                                            P(abi.SurfaceDiagnostics)]),
        "oracle_virtual_light": (c_int, [P(abi.Fluid), P(abi.Walls), P(abi.Csr), P(abi.Csr), P(abi.Params),
                                         c_void_p, c_void_p]),
        "oracle_prepare_moment": (c_int, [P(abi.Fluid), P(abi.Walls), P(abi.Csr), P(abi.Csr), P(abi.Params),
                                          P(abi.Moment)]),
        "oracle_velocity_laplacian": (c_int, [P(abi.Fluid), P(abi.Walls), P(abi.Csr), P(abi.Csr), P(abi.Moment),
                                              P(abi.Vector)]),
        "oracle_temporary_velocity": (c_int, [P(abi.Fluid), P(abi.Params), P(abi.Vector), P(abi.Fluid)]),
        "oracle_temporary_wall_velocity": (c_int, [P(abi.Walls), P(abi.Params), P(abi.Walls)]),
        "oracle_assemble_ppe": (c_int, [P(abi.Fluid), P(abi.Walls), P(abi.Params), P(abi.Csr), P(abi.Csr),
                                        P(abi.Fluid), P(abi.Walls), P(abi.Moment), P(abi.Moment), P(abi.Ppe)]),
        "oracle_clamp_pressure": (c_int, [P(abi.Fluid), c_void_p]),
        "oracle_pressure_gradient": (c_int, [P(abi.Fluid), P(abi.Walls), P(abi.Csr), P(abi.Csr), c_void_p,
                                             P(abi.Params), P(abi.Moment), P(abi.Vector)]),
        "oracle_particle_shifting": (c_int, [P(abi.Fluid), P(abi.Walls), P(abi.Csr), P(abi.Csr), P(abi.Params),
                                             P(abi.Vector)]),
        "oracle_update_velocity_position": (c_int, [P(abi.Fluid), P(abi.Fluid), P(abi.Params), P(abi.Vector),
                                                    P(abi.Vector)]),
        "oracle_anti_penetration": (c_int, [P(abi.Fluid), P(abi.Walls), P(abi.Csr), P(abi.Params)]),
        "oracle_smooth_velocity": (c_int, [P(abi.Fluid), P(abi.Csr), P(abi.Params), P(abi.Vector)]),
        "oracle_pressure_correction": (c_int, [P(abi.Fluid), P(abi.Walls), P(abi.Csr), P(abi.Csr), P(abi.Fluid),
                                               c_void_p, P(abi.Params), P(abi.Moment), P(abi.Vector),
                                               P(abi.Vector), P(abi.Vector)]),
        "oracle_step": (c_int, [P(abi.Params), P(abi.StepState), P(c_uint64)]),
        "oracle_solve_ppe": (c_int, [P(abi.CsrMatrix), c_void_p, c_void_p, P(abi.SolverOptions),
                                     P(abi.SolverReport)]),
        "oracle_advance_time": (c_int, [P(abi.Fluid), P(abi.TimeLimits), P(abi.TimeState)]),
        "oracle_max_threads": (c_int, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def r(x):
    return ctypes.byref(x)


class Oracle:
    """Oracle operations on a numpy-backed StepBuffers."""

    def __init__(self, abi):
        self.abi = abi
        self.L = lib(abi)

    def max_threads(self) -> int:
        return int(self.L.oracle_max_threads())

    def build_cell_list(self, x, y, z, grid, cells_view) -> int:
        return self.L.oracle_build_cell_list(x.ctypes.data, y.ctypes.data, z.ctypes.data, x.shape[0], r(grid),
                                             r(cells_view))

    def build_neighbor_lists(self, b, params):
        req = (c_uint64 * 2)()
        fv, wv = b.fluid_view(), b.walls_view()
        fc, wc = b.cells_view("fluid"), b.cells_view("wall")
        fn, wn = b.csr_view("fluid"), b.csr_view("wall")
        st = self.L.oracle_build_neighbor_lists(r(fv), r(wv), r(params), r(fc), r(wc), r(fn), r(wn), req)
        return st, (int(req[0]), int(req[1]))

    def reference_number_density(self, l0, re) -> float:
        return float(self.L.oracle_reference_number_density(l0, re))

    def classify_surface(self, b, params, diag=None) -> int:
        return self.L.oracle_classify_surface(r(b.fluid_view()), r(b.walls_view()), r(b.csr_view("fluid")),
                                              r(b.csr_view("wall")), r(params), r(diag) if diag is not None else None)

    def virtual_light(self, b, params, open_count=None, open_fraction=None) -> int:
        """open_count: int32 array, open_fraction: float64 array (numpy), either may be None."""
        return self.L.oracle_virtual_light(
            r(b.fluid_view()), r(b.walls_view()), r(b.csr_view("fluid")), r(b.csr_view("wall")), r(params),
            open_count.ctypes.data if open_count is not None else None,
            open_fraction.ctypes.data if open_fraction is not None else None)

    def prepare_moment(self, b, params, kind) -> int:
        b.params_for_moment = params
        return self.L.oracle_prepare_moment(r(b.fluid_view()), r(b.walls_view()), r(b.csr_view("fluid")),
                                            r(b.csr_view("wall")), r(params), r(b.moment_view(kind)))

    def provision(self, b, params) -> int:
        b.params_for_moment = params
        vm = b.moment_view(self.abi.VELOCITY_WALL_DIRICHLET_A)
        lap = b.vector_view(b.velocity_laplacian)
        st = self.L.oracle_velocity_laplacian(r(b.fluid_view()), r(b.walls_view()), r(b.csr_view("fluid")),
                                              r(b.csr_view("wall")), r(vm), r(lap))
        st |= self.L.oracle_temporary_velocity(r(b.fluid_view()), r(params), r(lap), r(b.temporary_view()))
        st |= self.L.oracle_temporary_wall_velocity(r(b.walls_view()), r(params), r(b.temporary_walls_view()))
        return st

    def assemble_ppe(self, b, params) -> int:
        b.params_for_moment = params
        return self.L.oracle_assemble_ppe(
            r(b.fluid_view()), r(b.walls_view()), r(params), r(b.csr_view("fluid")), r(b.csr_view("wall")),
            r(b.temporary_view()), r(b.temporary_walls_view()),
            r(b.moment_view(self.abi.VELOCITY_WALL_DIRICHLET_A)),
            r(b.moment_view(self.abi.PRESSURE_WALL_NEUMANN_A)), r(b.ppe_view()))

    def pressure_correction(self, b, params, pressure=None) -> int:
        b.params_for_moment = params
        pr = b.fluid["pressure"] if pressure is None else pressure
        return self.L.oracle_pressure_correction(
            r(b.fluid_view()), r(b.walls_view()), r(b.csr_view("fluid")), r(b.csr_view("wall")),
            r(b.temporary_view()), pr.ctypes.data, r(params), r(b.moment_view(self.abi.PRESSURE_WALL_NEUMANN_A)),
            r(b.vector_view(b.pressure_gradient)), r(b.vector_view(b.ps_displacement)),
            r(b.vector_view(b.smoothed_velocity)))

    def step(self, b, params):
        req = (c_uint64 * 2)()
        st = self.L.oracle_step(r(params), r(b.step_state(params)), req)
        return st, (int(req[0]), int(req[1]))

    def solve_ppe(self, row_offsets, col_indices, values, rhs, x, options):
        """GMRES on a host CSR system (numpy arrays); returns (status, SolverReport)."""
        A = self.abi.CsrMatrix(len(row_offsets) - 1, len(row_offsets) - 1, len(values), row_offsets.ctypes.data,
                               col_indices.ctypes.data, values.ctypes.data)
        rep = self.abi.SolverReport()
        st = self.L.oracle_solve_ppe(r(A), rhs.ctypes.data, x.ctypes.data, r(options), r(rep))
        return st, rep

    def advance_time(self, b, limits, state) -> int:
        """max |u| and the time manager's advance on a host TimeState (in place)."""
        return self.L.oracle_advance_time(r(b.fluid_view()), r(limits), r(state))
