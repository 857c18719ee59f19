"""ctypes mirror of include/lsmps_b200.h.

The structs are layout-identical to the C header (and therefore to the lsmps3D
reference views built with real = double).  Every pointer field is a plain
address (int): a torch CUDA tensor's ``data_ptr()`` for the product library, a
numpy array's ``ctypes.data`` for the host-side oracle.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, Structure, c_char_p, c_double, c_int, c_int32, c_size_t, c_uint64, c_void_p

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "liblsmps_b200.so"
CHECKED_LIB_NAME = "liblsmps_b200_checked.so"
# LSMPS_B200_LIBRARY selects another build of the same library, e.g. the
# bounds-checked one (build.py --bounds-check), for the whole process.
LIB_PATH = os.environ.get("LSMPS_B200_LIBRARY") or os.path.join(PKG_DIR, LIB_NAME)

# Status codes (lsmps_status).
OK = 0
CAPACITY_EXCEEDED = 1
INVALID_ARGUMENT = 2
NOT_PREPARED = 3
NON_SPD = 4
CUDA_ERROR = 5
INDEX_OVERFLOW = 6
NON_FINITE = 7
STATUS_NAMES = {
    0: "OK",
    1: "CAPACITY_EXCEEDED",
    2: "INVALID_ARGUMENT",
    3: "NOT_PREPARED",
    4: "NON_SPD",
    5: "CUDA_ERROR",
    6: "INDEX_OVERFLOW",
    7: "NON_FINITE",
}

PRECISION_PLAIN = 0
PRECISION_MIXED = 1

# Launch-shape knobs (lsmps_knob).
KNOB_MOMENT_OCCUPANCY = 0
KNOB_PPE_LANES = 1
KNOB_GATHER_LANES = 2
KNOB_COUNT = 3

# Particle limit of lsmps_build_cell_list_noalloc (its fixed scratch).
NOALLOC_MAX_PARTICLES = 524288

# Surface labels, include/lsmps3d/surface/surface_type.cuh:5-10.
INNER, NEAR_SURFACE, SURFACE, SPLASH = 0, 1, 2, 3

# Moment kinds, include/lsmps3d/moment_matrix/moment_matrix.cuh:39-44.
VELOCITY_WALL_DIRICHLET_A = 0
PRESSURE_WALL_NEUMANN_A = 1
PRESSURE_WALL_NEUMANN_B = 2
FLUID_ONLY_A = 3
MOMENT_SIZE = {0: 9, 1: 9, 2: 10, 3: 9}


class Fluid(Structure):
    _fields_ = [("count", c_size_t)] + [(n, c_void_p) for n in ("x", "y", "z", "vx", "vy", "vz", "pressure", "surface_type")]


class Walls(Structure):
    _fields_ = [("count", c_size_t)] + [
        (n, c_void_p) for n in ("x", "y", "z", "vx", "vy", "vz", "normal_x", "normal_y", "normal_z")
    ]


class Grid(Structure):
    _fields_ = [("origin", c_double * 3), ("cell_size", c_double), ("dims", c_int32 * 3)]


class Cells(Structure):
    _fields_ = [
        ("particle_count", c_size_t),
        ("cell_count", c_size_t),
        ("cell_ids", c_void_p),
        ("sorted_indices", c_void_p),
        ("cell_begin", c_void_p),
        ("cell_end", c_void_p),
    ]


class Csr(Structure):
    _fields_ = [("particle_count", c_size_t), ("neighbor_count", c_size_t), ("offsets", c_void_p), ("indices", c_void_p)]


class Vector(Structure):
    _fields_ = [("count", c_size_t), ("x", c_void_p), ("y", c_void_p), ("z", c_void_p)]


class SurfaceDiagnostics(Structure):
    _fields_ = [
        (n, c_void_p)
        for n in (
            "fluid_neighbor_count",
            "wall_neighbor_count",
            "number_density",
            "number_density_ratio",
            "anisotropy",
            "air_open_ratio",
            "air_anisotropy",
            "surface_normal_x",
            "surface_normal_y",
            "surface_normal_z",
        )
    ]


class Moment(Structure):
    _fields_ = [
        ("particle_count", c_size_t),
        ("matrix_size", c_int32),
        ("kind", c_int32),
        ("support_radius", c_double),
        ("wall_weight_scale", c_double),
        ("inverse_matrices", c_void_p),
        ("moment_trace", c_void_p),
        ("regularization_added", c_void_p),
        ("info", c_void_p),
        ("inversion_count", c_void_p),
    ]


class CsrMatrix(Structure):
    _fields_ = [
        ("rows", c_size_t),
        ("cols", c_size_t),
        ("nnz", c_size_t),
        ("row_offsets", c_void_p),
        ("col_indices", c_void_p),
        ("values", c_void_p),
    ]


class Ppe(Structure):
    _fields_ = [
        ("matrix", CsrMatrix),
        ("rhs", c_void_p),
        ("pressure", c_void_p),
        ("divergence", c_void_p),
        ("pressure_laplacian", c_void_p),
    ]


class SolverOptions(Structure):
    _fields_ = [
        ("max_iters", c_int32),
        ("restart", c_int32),
        ("tolerance", c_double),
        ("convergence", c_int32),
        ("preconditioner", c_int32),
        ("clamp_negative", c_int32),
        ("use_initial_guess", c_int32),
    ]


class SolverReport(Structure):
    _fields_ = [
        ("iterations", c_int32),
        ("converged", c_int32),
        ("initial_residual", c_double),
        ("final_residual", c_double),
    ]


class TimeLimits(Structure):
    _fields_ = [(n, c_double) for n in ("min_time_step", "max_time_step", "growth_factor", "cfl", "particle_spacing",
                                       "final_time")]


class TimeState(Structure):
    _fields_ = [("current_time", c_double), ("time_step", c_double), ("cfl_time_step", c_double),
                ("max_velocity", c_double), ("step_index", c_uint64)]


CONVERGENCE_RELATIVE_INITIAL = 0
CONVERGENCE_ABSOLUTE = 1
PRECONDITIONER_NONE = 0
PRECONDITIONER_JACOBI = 1


class Params(Structure):
    _fields_ = [
        ("particle_spacing", c_double),
        ("support_radius", c_double),
        ("near_surface_radius", c_double),
        ("grid", Grid),
        ("time_step", c_double),
        ("density", c_double),
        ("kinematic_viscosity", c_double),
        ("gravity", c_double * 3),
        ("splash_neighbor_threshold", c_int32),
        ("include_wall_neighbors", c_int32),
        ("number_density_ratio_threshold", c_double),
        ("air_open_ratio_threshold", c_double),
        ("air_anisotropy_threshold", c_double),
        ("wall_normal_independence_threshold", c_double),
        ("virtual_light_cone_cosine", c_double),
        ("lsmps_regularization", c_double),
        ("lsmps_wall_weight_scale", c_double),
        ("ps_displacement_scale", c_double),
        ("ps_min_distance_ratio", c_double),
        ("ps_max_displacement_ratio", c_double),
        ("wall_clearance_ratio", c_double),
        ("velocity_smoothing_strength", c_double),
    ]


class OperatorOut(Structure):
    _fields_ = [("count", c_size_t)] + [
        (n, c_void_p)
        for n in ("grad_x", "grad_y", "grad_z", "laplacian", "divergence", "ppe_row_offsets", "ppe_col_indices",
                  "ppe_values", "ppe_rhs")
    ]


class StepOperatorOut(Structure):
    _fields_ = [("count", c_size_t)] + [
        (n, c_void_p)
        for n in ("lap_x", "lap_y", "lap_z", "divergence", "grad_x", "grad_y", "grad_z", "ppe_row_offsets",
                  "ppe_col_indices", "ppe_values", "ppe_rhs", "wall_rhs")
    ]


class StepState(Structure):
    _fields_ = [
        ("fluid", Fluid),
        ("walls", Walls),
        ("fluid_cells", Cells),
        ("wall_cells", Cells),
        ("fluid_neighbors", Csr),
        ("wall_neighbors", Csr),
        ("temporary_velocity", Fluid),
        ("temporary_wall_velocity", Walls),
        ("velocity_laplacian", Vector),
        ("velocity_moment", Moment),
        ("pressure_moment", Moment),
        ("ppe", Ppe),
        ("pressure_gradient", Vector),
        ("ps_displacement", Vector),
        ("smoothed_velocity", Vector),
        ("pressure", c_void_p),
    ]


def default_solver_options() -> SolverOptions:
    """lsmps_solver_options_default: AMGX's GMRES configuration of the
    reference (src/ppe/ppe_matrix.cu:604-610) with AMGX's restart length 20."""
    return SolverOptions(max_iters=100, restart=20, tolerance=1e-6, convergence=CONVERGENCE_RELATIVE_INITIAL,
                         preconditioner=PRECONDITIONER_NONE, clamp_negative=1, use_initial_guess=0)


def default_params() -> Params:
    """SimulationConfig defaults (include/lsmps3d/core/config.hpp:12-60), as
    lsmps_params_default() fills them; kept in Python so the host side works
    without loading the CUDA library."""
    p = Params()
    p.particle_spacing = 0.01
    p.support_radius = 0.031
    p.near_surface_radius = 0.015
    p.grid.origin[:] = (0.0, 0.0, 0.0)
    p.grid.cell_size = 0.031
    p.grid.dims[:] = (1, 1, 1)
    p.time_step = 1.0e-4
    p.density = 1000.0
    p.kinematic_viscosity = 1.0e-6
    p.gravity[:] = (0.0, 0.0, -9.81)
    p.splash_neighbor_threshold = 4
    p.include_wall_neighbors = 1
    p.number_density_ratio_threshold = 0.85
    p.air_open_ratio_threshold = 0.33
    p.air_anisotropy_threshold = 0.033
    p.wall_normal_independence_threshold = 0.25
    p.virtual_light_cone_cosine = 0.8660254037844386
    p.lsmps_regularization = 1.0e-8
    p.lsmps_wall_weight_scale = 1.0
    p.ps_displacement_scale = 0.05
    p.ps_min_distance_ratio = 0.85
    p.ps_max_displacement_ratio = 0.2
    p.wall_clearance_ratio = 0.25
    p.velocity_smoothing_strength = 0.1
    return p


# Exported symbols of the product library with their ctypes signatures.  The
# test suite checks that this list and include/lsmps_b200.h agree.
P = POINTER
_SIGNATURES = {
    "lsmps_ctx_create": (c_int, [c_int, P(c_void_p)]),
    "lsmps_ctx_destroy": (None, [c_void_p]),
    "lsmps_ctx_set_stream": (c_int, [c_void_p, c_void_p]),
    "lsmps_ctx_stream": (c_void_p, [c_void_p]),
    "lsmps_ctx_set_precision": (c_int, [c_void_p, c_int]),
    "lsmps_ctx_set_synchronous": (c_int, [c_void_p, c_int]),
    "lsmps_ctx_reserve": (c_int, [c_void_p, c_size_t, c_size_t, c_size_t]),
    "lsmps_ctx_synchronize": (c_int, [c_void_p]),
    "lsmps_ctx_required": (c_uint64, [c_void_p]),
    "lsmps_ctx_launch_count": (c_uint64, [c_void_p]),
    "lsmps_ctx_set_profiling": (c_int, [c_void_p, c_int]),
    "lsmps_ctx_set_condition_threshold": (c_int, [c_void_p, c_double]),
    "lsmps_ctx_set_cell_order": (c_int, [c_void_p, c_int]),
    "lsmps_ctx_set_sorted_rows": (c_int, [c_void_p, c_int]),
    "lsmps_ctx_copy_sorted_rows": (c_int, [c_void_p, c_void_p, c_size_t]),
    "lsmps_ctx_set_adjoint_atomic": (c_int, [c_void_p, c_int]),
    "lsmps_ctx_fp64_fallbacks": (c_uint64, [c_void_p]),
    "lsmps_ctx_set_knob": (c_int, [c_void_p, c_int, c_int]),
    "lsmps_ctx_knob": (c_int, [c_void_p, c_int]),
    "lsmps_knob_variants": (c_int, [c_int]),
    "lsmps_autotune": (c_int, [c_void_p, P(Params), P(StepState), c_int, P(c_double)]),
    "lsmps_ctx_profile_report": (c_int, [c_void_p, ctypes.c_char_p, c_size_t, P(c_double), P(c_uint64), c_int]),
    "lsmps_ctx_last_error": (c_char_p, [c_void_p]),
    "lsmps_status_string": (c_char_p, [c_int]),
    "lsmps_params_default": (None, [P(Params)]),
    "lsmps_build_cell_list": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, P(Grid), P(Cells)]),
    "lsmps_build_cell_list_noalloc": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, P(Grid), P(Cells)]),
    "lsmps_build_neighbor_lists": (c_int, [c_void_p, P(Fluid), P(Walls), P(Params), P(Cells), P(Cells), P(Csr), P(Csr)]),
    "lsmps_reorder_fluid": (c_int, [c_void_p, P(Fluid), P(Cells), c_void_p]),
    "lsmps_reference_number_density": (c_double, [c_double, c_double]),
    "lsmps_classify_surface": (c_int, [c_void_p, P(Fluid), P(Walls), P(Csr), P(Csr), P(Params), P(SurfaceDiagnostics)]),
    "lsmps_virtual_light": (c_int, [c_void_p, P(Fluid), P(Walls), P(Csr), P(Csr), P(Params), c_void_p, c_void_p]),
    "lsmps_prepare_moments": (c_int, [c_void_p, P(Fluid), P(Walls), P(Csr), P(Csr), P(Params), P(Moment), c_int]),
    "lsmps_velocity_laplacian": (c_int, [c_void_p, P(Fluid), P(Walls), P(Csr), P(Csr), P(Moment), P(Vector)]),
    "lsmps_temporary_velocity": (c_int, [c_void_p, P(Fluid), P(Params), P(Vector), P(Fluid)]),
    "lsmps_temporary_wall_velocity": (c_int, [c_void_p, P(Walls), P(Params), P(Walls)]),
    "lsmps_assemble_ppe": (
        c_int,
        [c_void_p, P(Fluid), P(Walls), P(Params), P(Csr), P(Csr), P(Fluid), P(Walls), P(Moment), P(Moment), P(Ppe)],
    ),
    "lsmps_time_state_init": (None, [P(TimeLimits), c_double, P(TimeState)]),
    "lsmps_advance_time": (c_int, [c_void_p, P(Fluid), P(TimeLimits), c_void_p]),
    "lsmps_ctx_set_device_time_step": (c_int, [c_void_p, c_void_p]),
    "lsmps_solver_options_default": (None, [P(SolverOptions)]),
    "lsmps_solve_ppe": (c_int, [c_void_p, P(CsrMatrix), c_void_p, c_void_p, P(SolverOptions), P(SolverReport)]),
    "lsmps_clamp_particle_pressure": (c_int, [c_void_p, P(Fluid), c_void_p]),
    "lsmps_pressure_gradient": (
        c_int,
        [c_void_p, P(Fluid), P(Walls), P(Csr), P(Csr), c_void_p, P(Params), P(Moment), P(Vector)],
    ),
    "lsmps_particle_shifting": (c_int, [c_void_p, P(Fluid), P(Walls), P(Csr), P(Csr), P(Params), P(Vector)]),
    "lsmps_update_velocity_position": (c_int, [c_void_p, P(Fluid), P(Fluid), P(Params), P(Vector), P(Vector)]),
    "lsmps_anti_penetration": (c_int, [c_void_p, P(Fluid), P(Walls), P(Csr), P(Params)]),
    "lsmps_smooth_particle_velocity": (c_int, [c_void_p, P(Fluid), P(Csr), P(Params), P(Vector)]),
    "lsmps_pressure_correction": (
        c_int,
        [
            c_void_p,
            P(Fluid),
            P(Walls),
            P(Csr),
            P(Csr),
            P(Fluid),
            c_void_p,
            P(Params),
            P(Moment),
            P(Vector),
            P(Vector),
            P(Vector),
        ],
    ),
    "lsmps_step": (c_int, [c_void_p, P(Params), P(StepState)]),
    "lsmps_batch_create": (c_int, [c_int, c_int, P(c_void_p)]),
    "lsmps_batch_set_merged": (c_int, [c_void_p, c_int]),
    "lsmps_batch_merged": (c_int, [c_void_p]),
    "lsmps_batch_destroy": (None, [c_void_p]),
    "lsmps_batch_add": (c_int, [c_void_p, P(Params), P(StepState)]),
    "lsmps_batch_size": (c_int, [c_void_p]),
    "lsmps_batch_capture": (c_int, [c_void_p, c_int, c_int]),
    "lsmps_batch_launch": (c_int, [c_void_p, c_void_p]),
    "lsmps_batch_synchronize": (c_int, [c_void_p]),
    "lsmps_batch_stream": (c_void_p, [c_void_p]),
    "lsmps_batch_last_error": (c_char_p, [c_void_p]),
    "lsmps_operators_forward": (c_int, [c_void_p, P(Fluid), P(Csr), P(Params), c_void_p, P(Vector), P(OperatorOut),
                                        c_void_p]),
    "lsmps_operators_backward": (c_int, [c_void_p, P(Fluid), P(Csr), P(Params), c_void_p, P(Vector), P(OperatorOut),
                                         c_void_p, c_void_p, P(Vector), P(Vector)]),
    "lsmps_ctx_set_step_events": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "lsmps_step_operators_forward": (c_int, [c_void_p, P(Fluid), P(Walls), P(Csr), P(Csr), P(Params),
                                             P(StepOperatorOut)]),
    "lsmps_step_operators_backward": (c_int, [c_void_p, P(Fluid), P(Walls), P(Csr), P(Csr), P(Params),
                                              P(StepOperatorOut), P(Vector), c_void_p, P(Vector)]),
}


_LIB = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the CUDA library and attach signatures.  Raises if it is missing:
    the product has no CPU fallback."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build the CUDA extension first (lsmps-3d_b200/build.py or __graft_entry__.build())"
        )
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def exported_names() -> list[str]:
    return list(_SIGNATURES)
