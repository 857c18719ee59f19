"""Buffer sets for one LSMPS step, allocated by numpy (host) or torch (device),
and the C ABI views over them.

The layout follows the reference's owners: DeviceFluidParticles /
DeviceWallParticles (src/core/runtime.cu:113-199), DeviceNeighborList
(:225-248), DeviceCellList (:270-295), the moment caches
(src/moment_matrix/moment_matrix.cu:353-396), DevicePpeWorkspace
(src/ppe/ppe_matrix.cu:425-467) and DeviceCorrectionWorkspace
(src/correction/pressure_correction.cu:544-581).
"""

from __future__ import annotations

import numpy as np

from . import abi

FLUID_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "pressure")
WALL_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "normal_x", "normal_y", "normal_z")

# The reference driver's CSR capacity per fluid particle
# (src/app/simulation_driver.cu:29-30).
DEFAULT_MAX_NEIGHBORS = 256


class NumpyAlloc:
    """Host allocation; addresses are numpy data pointers."""

    device = "cpu"

    def zeros(self, n, dtype):
        return np.zeros(int(n), dtype=np.float64 if dtype == "f64" else np.int32)

    def full(self, n, value, dtype):
        a = self.zeros(n, dtype)
        a[:] = value
        return a

    @staticmethod
    def ptr(a) -> int:
        return int(a.ctypes.data) if a is not None and a.size else 0

    @staticmethod
    def to_numpy(a):
        return a

    def from_numpy(self, a, dtype):
        return np.ascontiguousarray(a, dtype=np.float64 if dtype == "f64" else np.int32).copy()

    @staticmethod
    def copy_(dst, src):
        dst[: src.shape[0]] = src


class TorchAlloc:
    """Device allocation through torch (plumbing only); addresses are
    data_ptr() values."""

    def __init__(self, device="cuda"):
        import torch

        self.torch = torch
        self.device = device

    def _dt(self, dtype):
        return self.torch.float64 if dtype == "f64" else self.torch.int32

    def zeros(self, n, dtype):
        return self.torch.zeros(max(int(n), 0), dtype=self._dt(dtype), device=self.device)

    def full(self, n, value, dtype):
        return self.torch.full((max(int(n), 0),), value, dtype=self._dt(dtype), device=self.device)

    @staticmethod
    def ptr(a) -> int:
        return int(a.data_ptr()) if a is not None and a.numel() else 0

    @staticmethod
    def to_numpy(a):
        return a.detach().cpu().numpy()

    def from_numpy(self, a, dtype):
        return self.torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64 if dtype == "f64" else np.int32)).to(
            self.device
        )

    def copy_(self, dst, src):
        dst[: src.shape[0]].copy_(self.torch.from_numpy(np.ascontiguousarray(src)).to(dst.device), non_blocking=False)


class StepBuffers:
    """Every buffer one step touches, with ABI views.  Capacities follow the
    reference driver: CSR capacity = max_neighbors * N_f per table, PPE nnz
    capacity = N_f + fluid CSR capacity (simulation_driver.cu:304-321)."""

    def __init__(self, alloc, n_fluid: int, n_wall: int, n_cells: int,
                 max_fluid_neighbors: int = DEFAULT_MAX_NEIGHBORS,
                 max_wall_neighbors: int = DEFAULT_MAX_NEIGHBORS,
                 fluid_capacity: int | None = None, wall_capacity: int | None = None):
        a = alloc
        self.alloc = a
        nf, nw, nc = int(n_fluid), int(n_wall), int(n_cells)
        self.n_fluid, self.n_wall, self.n_cells = nf, nw, nc
        self.cap_f = int(fluid_capacity) if fluid_capacity is not None else max_fluid_neighbors * nf
        self.cap_w = int(wall_capacity) if wall_capacity is not None else max_wall_neighbors * nf
        self.fluid = {k: a.zeros(nf, "f64") for k in FLUID_FIELDS}
        self.fluid["surface_type"] = a.zeros(nf, "i32")
        self.walls = {k: a.zeros(nw, "f64") for k in WALL_FIELDS}
        self.fluid_cells = {"cell_ids": a.zeros(nf, "i32"), "sorted_indices": a.zeros(nf, "i32"),
                            "cell_begin": a.zeros(nc, "i32"), "cell_end": a.zeros(nc, "i32")}
        self.wall_cells = {"cell_ids": a.zeros(nw, "i32"), "sorted_indices": a.zeros(nw, "i32"),
                           "cell_begin": a.zeros(nc, "i32"), "cell_end": a.zeros(nc, "i32")}
        self.fluid_neighbors = {"offsets": a.zeros(nf + 1, "i32"), "indices": a.zeros(self.cap_f, "i32")}
        self.wall_neighbors = {"offsets": a.zeros(nf + 1, "i32"), "indices": a.zeros(self.cap_w, "i32")}
        self.temporary_velocity = {k: a.zeros(nf, "f64") for k in ("vx", "vy", "vz")}
        self.temporary_wall_velocity = {k: a.zeros(nw, "f64") for k in ("vx", "vy", "vz")}
        self.velocity_laplacian = {k: a.zeros(nf, "f64") for k in ("x", "y", "z")}
        self.moments = {}
        for kind in (abi.VELOCITY_WALL_DIRICHLET_A, abi.PRESSURE_WALL_NEUMANN_A):
            self.moments[kind] = self._moment_arrays(kind, nf)
        self.nnz_cap = nf + self.cap_f
        self.ppe = {"row_offsets": a.zeros(nf + 1, "i32"), "col_indices": a.zeros(self.nnz_cap, "i32"),
                    "values": a.zeros(self.nnz_cap, "f64"), "rhs": a.zeros(nf, "f64"),
                    "pressure": a.zeros(nf, "f64"), "divergence": a.zeros(nf, "f64"),
                    "pressure_laplacian": a.zeros(nf, "f64")}
        self.pressure_gradient = {k: a.zeros(nf, "f64") for k in ("x", "y", "z")}
        self.ps_displacement = {k: a.zeros(nf, "f64") for k in ("x", "y", "z")}
        self.smoothed_velocity = {k: a.zeros(nf, "f64") for k in ("x", "y", "z")}

    # -- allocation helpers ------------------------------------------------
    def _moment_arrays(self, kind, n):
        m = abi.MOMENT_SIZE[kind]
        a = self.alloc
        return {"inverse_matrices": a.zeros(n * m * m, "f64"), "moment_trace": a.zeros(n, "f64"),
                "regularization_added": a.zeros(n, "f64"), "info": a.zeros(n, "i32"),
                "inversion_count": a.zeros(1, "i32")}

    def add_moment(self, kind):
        if kind not in self.moments:
            self.moments[kind] = self._moment_arrays(kind, self.n_fluid)
        return self.moments[kind]

    def load_case(self, case) -> None:
        for k in FLUID_FIELDS + ("surface_type",):
            self.alloc.copy_(self.fluid[k], case.fluid[k])
        for k in WALL_FIELDS:
            self.alloc.copy_(self.walls[k], case.walls[k])

    # -- views ---------------------------------------------------------------
    def fluid_view(self, count=None) -> abi.Fluid:
        p = self.alloc.ptr
        v = abi.Fluid()
        v.count = self.n_fluid if count is None else count
        for k in FLUID_FIELDS + ("surface_type",):
            setattr(v, k, p(self.fluid[k]))
        return v

    def walls_view(self) -> abi.Walls:
        p = self.alloc.ptr
        v = abi.Walls()
        v.count = self.n_wall
        for k in WALL_FIELDS:
            setattr(v, k, p(self.walls[k]))
        return v

    def cells_view(self, which: str) -> abi.Cells:
        d = self.fluid_cells if which == "fluid" else self.wall_cells
        p = self.alloc.ptr
        v = abi.Cells()
        v.particle_count = self.n_fluid if which == "fluid" else self.n_wall
        v.cell_count = self.n_cells
        for k in ("cell_ids", "sorted_indices", "cell_begin", "cell_end"):
            setattr(v, k, p(d[k]))
        return v

    def csr_view(self, which: str) -> abi.Csr:
        d = self.fluid_neighbors if which == "fluid" else self.wall_neighbors
        v = abi.Csr()
        v.particle_count = self.n_fluid
        v.neighbor_count = self.cap_f if which == "fluid" else self.cap_w
        v.offsets = self.alloc.ptr(d["offsets"])
        v.indices = self.alloc.ptr(d["indices"])
        return v

    def temporary_view(self) -> abi.Fluid:
        v = abi.Fluid()
        v.count = self.n_fluid
        for k in ("vx", "vy", "vz"):
            setattr(v, k, self.alloc.ptr(self.temporary_velocity[k]))
        return v

    def temporary_walls_view(self) -> abi.Walls:
        v = abi.Walls()
        v.count = self.n_wall
        for k in ("vx", "vy", "vz"):
            setattr(v, k, self.alloc.ptr(self.temporary_wall_velocity[k]))
        return v

    def vector_view(self, d) -> abi.Vector:
        v = abi.Vector()
        v.count = self.n_fluid
        v.x, v.y, v.z = (self.alloc.ptr(d[k]) for k in ("x", "y", "z"))
        return v

    def moment_view(self, kind) -> abi.Moment:
        d = self.add_moment(kind)
        p = self.params_for_moment
        v = abi.Moment()
        v.particle_count = self.n_fluid
        v.matrix_size = abi.MOMENT_SIZE[kind]
        v.kind = kind
        v.support_radius = p.support_radius if p is not None else 0.0
        v.wall_weight_scale = p.lsmps_wall_weight_scale if p is not None else 1.0
        for k in ("inverse_matrices", "moment_trace", "regularization_added", "info", "inversion_count"):
            setattr(v, k, self.alloc.ptr(d[k]))
        return v

    params_for_moment: abi.Params | None = None

    def ppe_view(self) -> abi.Ppe:
        v = abi.Ppe()
        v.matrix.rows = self.n_fluid
        v.matrix.cols = self.n_fluid
        v.matrix.nnz = self.nnz_cap
        p = self.alloc.ptr
        v.matrix.row_offsets = p(self.ppe["row_offsets"])
        v.matrix.col_indices = p(self.ppe["col_indices"])
        v.matrix.values = p(self.ppe["values"])
        for k in ("rhs", "pressure", "divergence", "pressure_laplacian"):
            setattr(v, k, p(self.ppe[k]))
        return v

    def step_state(self, params: abi.Params) -> abi.StepState:
        self.params_for_moment = params
        s = abi.StepState()
        s.fluid = self.fluid_view()
        s.walls = self.walls_view()
        s.fluid_cells = self.cells_view("fluid")
        s.wall_cells = self.cells_view("wall")
        s.fluid_neighbors = self.csr_view("fluid")
        s.wall_neighbors = self.csr_view("wall")
        s.temporary_velocity = self.temporary_view()
        s.temporary_wall_velocity = self.temporary_walls_view()
        s.velocity_laplacian = self.vector_view(self.velocity_laplacian)
        s.velocity_moment = self.moment_view(abi.VELOCITY_WALL_DIRICHLET_A)
        s.pressure_moment = self.moment_view(abi.PRESSURE_WALL_NEUMANN_A)
        s.ppe = self.ppe_view()
        s.pressure_gradient = self.vector_view(self.pressure_gradient)
        s.ps_displacement = self.vector_view(self.ps_displacement)
        s.smoothed_velocity = self.vector_view(self.smoothed_velocity)
        s.pressure = self.alloc.ptr(self.fluid["pressure"])
        return s

    # -- readback ------------------------------------------------------------
    def csr_rows(self, which: str):
        d = self.fluid_neighbors if which == "fluid" else self.wall_neighbors
        off = self.alloc.to_numpy(d["offsets"])[: self.n_fluid + 1].copy()
        total = int(off[-1]) if off.size else 0
        idx = self.alloc.to_numpy(d["indices"])[:total].copy()
        return off, idx

    def numpy(self, group: str) -> dict:
        d = getattr(self, group)
        return {k: self.alloc.to_numpy(v).copy() for k, v in d.items()}
