"""Device API: a thin Python layer over the C ABI (include/lsmps_b200.h).

Every call goes through liblsmps_b200.so; there is no CPU fallback and the
module raises at import time if the library is missing.  Device memory comes
from torch (plumbing only), see buffers.TorchAlloc.

Errors: the reference exits the process on a failed check; here a non-OK
status raises LsmpsError carrying the status code and the library's message.
"""

from __future__ import annotations

import ctypes

from . import abi
from .buffers import StepBuffers, TorchAlloc

_lib = abi.load_library()


class LsmpsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


def r(x):
    return ctypes.byref(x)


def reference_number_density(particle_spacing: float, support_radius: float) -> float:
    """compute_uniform_reference_number_density (surface_detection.cuh:28)."""
    v = float(_lib.lsmps_reference_number_density(particle_spacing, support_radius))
    if v <= 0.0:
        raise LsmpsError(abi.INVALID_ARGUMENT, "Reference number density requires positive spacing and support radius")
    return v


class Context:
    """Owns one lsmps_ctx (stream, scratch, device status)."""

    def __init__(self, device: int = 0, precision: int = abi.PRECISION_PLAIN, synchronous: bool = True,
                 use_torch_stream: bool = True):
        import torch

        self.torch = torch
        self.device = device
        h = ctypes.c_void_p()
        st = _lib.lsmps_ctx_create(device, ctypes.byref(h))
        if st != abi.OK:
            raise LsmpsError(st, "lsmps_ctx_create failed")
        self.h = h
        if use_torch_stream:
            s = torch.cuda.current_stream(device)
            _lib.lsmps_ctx_set_stream(self.h, ctypes.c_void_p(s.cuda_stream))
        self.set_precision(precision)
        self.set_synchronous(synchronous)

    def close(self):
        if getattr(self, "h", None):
            _lib.lsmps_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- context controls ---------------------------------------------------
    def check(self, st: int) -> None:
        if st != abi.OK:
            msg = _lib.lsmps_ctx_last_error(self.h)
            raise LsmpsError(st, msg.decode() if msg else "")

    def set_precision(self, precision: int) -> None:
        self.check(_lib.lsmps_ctx_set_precision(self.h, precision))

    def set_synchronous(self, sync: bool) -> None:
        self.check(_lib.lsmps_ctx_set_synchronous(self.h, 1 if sync else 0))

    def set_stream(self, stream_handle: int | None) -> None:
        self.check(_lib.lsmps_ctx_set_stream(self.h, ctypes.c_void_p(stream_handle or 0)))

    def reserve(self, n_fluid: int, n_wall: int, n_cells: int) -> None:
        self.check(_lib.lsmps_ctx_reserve(self.h, n_fluid, n_wall, n_cells))

    def synchronize(self) -> None:
        self.check(_lib.lsmps_ctx_synchronize(self.h))

    def set_profiling(self, on: bool) -> None:
        self.check(_lib.lsmps_ctx_set_profiling(self.h, 1 if on else 0))

    def set_knob(self, knob: int, value: int) -> None:
        self.check(_lib.lsmps_ctx_set_knob(self.h, knob, value))

    def knob(self, knob: int) -> int:
        return int(_lib.lsmps_ctx_knob(self.h, knob))

    def autotune(self, b: StepBuffers, params: abi.Params, repeats: int = 3,
                 state: abi.StepState | None = None) -> dict[int, tuple[int, float]]:
        """lsmps_autotune on this state; returns {knob: (chosen variant, mean ms)}."""
        s = state if state is not None else b.step_state(params)
        ms = (ctypes.c_double * abi.KNOB_COUNT)()
        self.check(_lib.lsmps_autotune(self.h, r(params), r(s), repeats, ms))
        return {k: (self.knob(k), float(ms[k])) for k in range(abi.KNOB_COUNT)}

    def set_cell_order(self, on: bool) -> None:
        """lsmps_step visits the fluid in cell order (default) or index order."""
        self.check(_lib.lsmps_ctx_set_cell_order(self.h, 1 if on else 0))

    def sorted_rows(self, count: int):
        """The first `count` entries of the context's cell-sorted rows (numpy)."""
        import torch

        out = torch.empty(max(count, 1), dtype=torch.int32, device=f"cuda:{self.device}")
        self.check(_lib.lsmps_ctx_copy_sorted_rows(self.h, ctypes.c_void_p(out.data_ptr()), count))
        torch.cuda.synchronize()
        return out[:count].cpu().numpy()

    def set_sorted_rows(self, on: bool) -> None:
        """lsmps_step's gathers read cell-sorted rows and records (default)
        or the rows' indices and records in index order."""
        self.check(_lib.lsmps_ctx_set_sorted_rows(self.h, 1 if on else 0))

    def set_adjoint_atomic(self, on: bool) -> None:
        """Operator backward: scatter with FP64 atomics (True) or the
        deterministic transpose + gather (False, the default)."""
        self.check(_lib.lsmps_ctx_set_adjoint_atomic(self.h, 1 if on else 0))

    def set_condition_threshold(self, threshold: float) -> None:
        """Mixed form: condition estimate above which a moment matrix is
        factorised in FP64 (default 1e4)."""
        self.check(_lib.lsmps_ctx_set_condition_threshold(self.h, float(threshold)))

    @property
    def fp64_fallbacks(self) -> int:
        """Mixed form: moment matrices factorised in FP64 so far."""
        return int(_lib.lsmps_ctx_fp64_fallbacks(self.h))

    def profile_report(self, max_entries: int = 64) -> list[tuple[str, float, int]]:
        """(kernel name, total ms, launches) per kernel since profiling was
        switched on; clears the records."""
        names = ctypes.create_string_buffer(8192)
        ms = (ctypes.c_double * max_entries)()
        cnt = (ctypes.c_uint64 * max_entries)()
        n = _lib.lsmps_ctx_profile_report(self.h, names, len(names), ms, cnt, max_entries)
        if n < 0:
            raise LsmpsError(abi.CUDA_ERROR, "profile report failed")
        keys = names.value.decode().split("\n")[:n]
        return [(keys[i], float(ms[i]), int(cnt[i])) for i in range(n)]

    @property
    def required(self) -> int:
        return int(_lib.lsmps_ctx_required(self.h))

    @property
    def launch_count(self) -> int:
        return int(_lib.lsmps_ctx_launch_count(self.h))

    # -- hot-path operations on a StepBuffers --------------------------------
    def build_cell_list(self, x_ptr: int, y_ptr: int, z_ptr: int, count: int, grid: abi.Grid, cells: abi.Cells):
        self.check(_lib.lsmps_build_cell_list(self.h, x_ptr, y_ptr, z_ptr, count, r(grid), r(cells)))

    def build_neighbor_lists(self, b: StepBuffers, params: abi.Params) -> None:
        self.check(_lib.lsmps_build_neighbor_lists(
            self.h, r(b.fluid_view()), r(b.walls_view()), r(params), r(b.cells_view("fluid")),
            r(b.cells_view("wall")), r(b.csr_view("fluid")), r(b.csr_view("wall"))))

    def reorder_fluid(self, b: StepBuffers, permutation_ptr: int | None = None) -> None:
        """Renumber the fluid of `b` in its fluid cell-list order (lsmps_reorder_fluid); the
        neighbour lists must be rebuilt afterwards."""
        self.check(_lib.lsmps_reorder_fluid(self.h, r(b.fluid_view()), r(b.cells_view("fluid")),
                                            ctypes.c_void_p(permutation_ptr) if permutation_ptr else None))

    def classify_surface(self, b: StepBuffers, params: abi.Params, diagnostics: abi.SurfaceDiagnostics | None = None):
        self.check(_lib.lsmps_classify_surface(
            self.h, r(b.fluid_view()), r(b.walls_view()), r(b.csr_view("fluid")), r(b.csr_view("wall")),
            r(params), r(diagnostics) if diagnostics is not None else None))

    def virtual_light(self, b: StepBuffers, params: abi.Params, open_count_ptr: int | None,
                      open_fraction_ptr: int | None) -> None:
        """compute_virtual_light_diagnostics (surface_detection.cu:555-578): open-direction count
        (int32) and fraction (float64) per fluid particle into caller-owned device buffers."""
        self.check(_lib.lsmps_virtual_light(
            self.h, r(b.fluid_view()), r(b.walls_view()), r(b.csr_view("fluid")), r(b.csr_view("wall")),
            r(params), open_count_ptr, open_fraction_ptr))

    def prepare_moments(self, b: StepBuffers, params: abi.Params, kinds) -> None:
        b.params_for_moment = params
        arr = (abi.Moment * len(kinds))(*[b.moment_view(k) for k in kinds])
        self.check(_lib.lsmps_prepare_moments(self.h, r(b.fluid_view()), r(b.walls_view()), r(b.csr_view("fluid")),
                                              r(b.csr_view("wall")), r(params), arr, len(kinds)))

    def provision(self, b: StepBuffers, params: abi.Params) -> None:
        b.params_for_moment = params
        lap = b.vector_view(b.velocity_laplacian)
        self.check(_lib.lsmps_velocity_laplacian(
            self.h, r(b.fluid_view()), r(b.walls_view()), r(b.csr_view("fluid")), r(b.csr_view("wall")),
            r(b.moment_view(abi.VELOCITY_WALL_DIRICHLET_A)), r(lap)))
        self.check(_lib.lsmps_temporary_velocity(self.h, r(b.fluid_view()), r(params), r(lap), r(b.temporary_view())))
        self.check(_lib.lsmps_temporary_wall_velocity(self.h, r(b.walls_view()), r(params),
                                                      r(b.temporary_walls_view())))

    def assemble_ppe(self, b: StepBuffers, params: abi.Params) -> None:
        b.params_for_moment = params
        self.check(_lib.lsmps_assemble_ppe(
            self.h, r(b.fluid_view()), r(b.walls_view()), r(params), r(b.csr_view("fluid")), r(b.csr_view("wall")),
            r(b.temporary_view()), r(b.temporary_walls_view()), r(b.moment_view(abi.VELOCITY_WALL_DIRICHLET_A)),
            r(b.moment_view(abi.PRESSURE_WALL_NEUMANN_A)), r(b.ppe_view())))

    def pressure_correction(self, b: StepBuffers, params: abi.Params, pressure_ptr: int | None = None) -> None:
        b.params_for_moment = params
        p = pressure_ptr if pressure_ptr is not None else b.alloc.ptr(b.fluid["pressure"])
        self.check(_lib.lsmps_pressure_correction(
            self.h, r(b.fluid_view()), r(b.walls_view()), r(b.csr_view("fluid")), r(b.csr_view("wall")),
            r(b.temporary_view()), ctypes.c_void_p(p), r(params), r(b.moment_view(abi.PRESSURE_WALL_NEUMANN_A)),
            r(b.vector_view(b.pressure_gradient)), r(b.vector_view(b.ps_displacement)),
            r(b.vector_view(b.smoothed_velocity))))

    def solve_csr(self, matrix: abi.CsrMatrix, rhs_ptr: int, x_ptr: int,
                  options: abi.SolverOptions | None = None) -> abi.SolverReport:
        """lsmps_solve_ppe on any square device CSR system (AmgxPpeSolver::solve,
        src/ppe/ppe_matrix.cu:586-679): restarted GMRES from zero, then the clamp."""
        rep = abi.SolverReport()
        self.check(_lib.lsmps_solve_ppe(self.h, r(matrix), ctypes.c_void_p(rhs_ptr), ctypes.c_void_p(x_ptr),
                                        r(options) if options is not None else None, r(rep)))
        return rep

    def solve_ppe(self, b: StepBuffers, options: abi.SolverOptions | None = None) -> abi.SolverReport:
        """Solve the assembled PPE rows of `b` into b.ppe["pressure"]."""
        v = b.ppe_view()
        return self.solve_csr(v.matrix, v.rhs, v.pressure, options)

    def advance_time(self, b: StepBuffers, limits: abi.TimeLimits, state_ptr: int) -> None:
        """max |u| and SimulationTimeManager::advance on the device state at state_ptr
        (an abi.TimeState in device memory)."""
        self.check(_lib.lsmps_advance_time(self.h, r(b.fluid_view()), r(limits), ctypes.c_void_p(state_ptr)))

    def set_step_events(self, wall_event: int | None, input_event: int | None, output_event: int | None) -> None:
        """lsmps_ctx_set_step_events: raw cudaEvent_t handles (e.g. a recorded
        torch.cuda.Event's cuda_event), or None for an event not used."""
        self.check(_lib.lsmps_ctx_set_step_events(self.h, ctypes.c_void_p(wall_event or 0),
                                                  ctypes.c_void_p(input_event or 0),
                                                  ctypes.c_void_p(output_event or 0)))

    def set_device_time_step(self, ptr: int | None) -> None:
        """Kernels read dt from this device address (None: from the params)."""
        self.check(_lib.lsmps_ctx_set_device_time_step(self.h, ctypes.c_void_p(ptr) if ptr else None))

    def step(self, b: StepBuffers, params: abi.Params, state: abi.StepState | None = None) -> None:
        s = state if state is not None else b.step_state(params)
        self.check(_lib.lsmps_step(self.h, r(params), r(s)))


class Batch:
    """Independent boxes stepped by one captured CUDA graph (lsmps_batch_*).
    Keeps the boxes' StepBuffers, params and step states alive while the
    graph exists."""

    def __init__(self, device: int = 0, streams: int = 8):
        h = ctypes.c_void_p()
        st = _lib.lsmps_batch_create(device, streams, ctypes.byref(h))
        if st != abi.OK:
            raise LsmpsError(st, "lsmps_batch_create failed")
        self.h = h
        self.boxes = []

    def check(self, st: int) -> None:
        if st != abi.OK:
            msg = _lib.lsmps_batch_last_error(self.h)
            raise LsmpsError(st, msg.decode() if msg else "")

    def add(self, b: StepBuffers, params: abi.Params) -> None:
        state = b.step_state(params)
        self.boxes.append((b, params, state))
        self.check(_lib.lsmps_batch_add(self.h, r(params), r(state)))

    def set_merged(self, on: bool) -> None:
        """Merged form (all boxes as one particle set; the default) or one
        step per box on the worker streams; chosen before capture."""
        self.check(_lib.lsmps_batch_set_merged(self.h, 1 if on else 0))

    @property
    def merged(self) -> bool:
        """Whether the last capture used the merged form."""
        return bool(_lib.lsmps_batch_merged(self.h))

    def capture(self, precision: int = abi.PRECISION_MIXED, autotune_repeats: int = 0) -> None:
        self.check(_lib.lsmps_batch_capture(self.h, precision, autotune_repeats))

    def launch(self, stream_handle: int | None = None) -> None:
        self.check(_lib.lsmps_batch_launch(self.h, ctypes.c_void_p(stream_handle) if stream_handle else None))

    def synchronize(self) -> None:
        self.check(_lib.lsmps_batch_synchronize(self.h))

    @property
    def stream(self) -> int:
        return int(_lib.lsmps_batch_stream(self.h) or 0)

    def close(self):
        if getattr(self, "h", None):
            _lib.lsmps_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_buffers(case, max_fluid_neighbors: int = 256, max_wall_neighbors: int = 256, device="cuda") -> StepBuffers:
    """StepBuffers in device memory loaded with a synthetic case."""
    b = StepBuffers(TorchAlloc(device), case.n_fluid, case.n_wall, case.n_cells, max_fluid_neighbors,
                    max_wall_neighbors)
    b.load_case(case)
    return b
