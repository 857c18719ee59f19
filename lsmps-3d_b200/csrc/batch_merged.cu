// batch_merged.cu - the merged form of a batch (lsmps_batch_set_merged): all
// boxes stepped as ONE particle set, so every stage of the step is one launch
// of the step's own kernels over the particles of all boxes (persistent,
// grid-stride kernels sized for the whole GPU) instead of one launch per box.
//
// The boxes share their parameters except the cell grid (checked at capture;
// otherwise the batch falls back to one step per box on worker streams).
// Merged numbering: box b's fluid particles are merged indices
// [fluid_base, fluid_base + n_b), its walls [wall_base, ...), its cells
// [cell_base, ...).  Every particle keeps its own box's coordinates: the cell
// hash and the neighbour search place each particle and cell on its box's
// grid (BoxGrid table, cells.cu / neighbors.cu), so a row holds only its own
// box's neighbours, in the order a solo step gives them; all other kernels
// are per particle and see one large set.  Each box's results therefore
// equal its solo lsmps_step bit for bit.
//
// One launch of the graph: gather the boxes' particle state (fluid SoA,
// labels, the pressure input, walls) into the merged buffers -> lsmps_step
// on the merged set -> scatter every output back into the boxes' own views
// (indices shifted back to the box's numbering).  The PPE rows need no
// scatter: the merged context writes each box's rows straight into the box's
// own matrix (lsmps_ctx::box_ppe, columns in the box's numbering); only
// their row offsets come from the merged set.  The merged neighbour
// tables and cell lists are the batch's own between launches: capture builds
// them from the boxes' current positions, and every launch ends with their
// rebuild, as a step does; the copies in the boxes' buffers are outputs.
#include <algorithm>
#include <cstring>
#include <vector>

#include "batch_impl.cuh"

namespace lsmps {
namespace {

constexpr int kThreads = 256;

// One box as the gather/scatter kernels see it.
struct BoxIO {
  lsmps_step_state s;
  index_t nf, nw, nc;
  index_t fb, wb, cb;
};

struct MergedArgs {
  const BoxIO* io;
  const BoxGrid* grids;
  int nbox;
  lsmps_step_state m;  // the merged views
  index_t nf, nw, nc;
  int full_inverse;    // plain form: the step wrote the 81-entry inverses
  DeviceStatus* status;  // the merged context's status word
};

MergedArgs merged_args(const MergedBatch& mb) {
  MergedArgs a{};
  a.io = static_cast<const BoxIO*>(mb.io);
  a.grids = mb.grids;
  a.nbox = mb.nbox;
  a.m = mb.state;
  a.nf = mb.nf;
  a.nw = mb.nw;
  a.nc = mb.nc;
  a.full_inverse = mb.precision == LSMPS_PRECISION_PLAIN ? 1 : 0;
  a.status = mb.ctx ? mb.ctx->d_status : nullptr;
  return a;
}

__device__ __forceinline__ int box_fluid(const MergedArgs& a, index_t t) { return box_of(a.grids, a.nbox, t, 1); }

__global__ void gather_kernel(MergedArgs a) {
  const index_t stride = gridDim.x * blockDim.x;
  for (index_t t = blockIdx.x * blockDim.x + threadIdx.x; t < a.nf; t += stride) {
    const BoxIO& b = a.io[box_fluid(a, t)];
    const index_t k = t - b.fb;
    const lsmps_fluid& f = b.s.fluid;
    a.m.fluid.x[t] = f.x[k];
    a.m.fluid.y[t] = f.y[k];
    a.m.fluid.z[t] = f.z[k];
    a.m.fluid.vx[t] = f.vx[k];
    a.m.fluid.vy[t] = f.vy[k];
    a.m.fluid.vz[t] = f.vz[k];
    a.m.fluid.pressure[t] = f.pressure[k];
    a.m.fluid.surface_type[t] = f.surface_type ? f.surface_type[k] : 0;
    a.m.pressure[t] = b.s.pressure[k];
  }
  for (index_t t = blockIdx.x * blockDim.x + threadIdx.x; t < a.nw; t += stride) {
    const BoxIO& b = a.io[box_of(a.grids, a.nbox, t, 2)];
    const index_t k = t - b.wb;
    const lsmps_walls& w = b.s.walls;
    a.m.walls.x[t] = w.x[k];
    a.m.walls.y[t] = w.y[k];
    a.m.walls.z[t] = w.z[k];
    a.m.walls.vx[t] = w.vx[k];
    a.m.walls.vy[t] = w.vy[k];
    a.m.walls.vz[t] = w.vz[k];
    a.m.walls.normal_x[t] = w.normal_x[k];
    a.m.walls.normal_y[t] = w.normal_y[k];
    a.m.walls.normal_z[t] = w.normal_z[k];
  }
}

__device__ __forceinline__ void copy3(const lsmps_vector& src, const lsmps_vector& dst, index_t t, index_t k) {
  dst.x[k] = src.x[t];
  dst.y[k] = src.y[t];
  dst.z[k] = src.z[t];
}

// Per merged fluid particle (and, for its box's last particle, the closing
// offsets): the particle state, the per-particle outputs, the fluid cell
// list entries at this sorted position, the CSR and PPE row offsets, the
// moment traces; the first particle of a box advances the box's inversion
// counters (one per kind and step, as a solo step does).
__global__ void scatter_particles_kernel(MergedArgs a) {
  const index_t stride = gridDim.x * blockDim.x;
  const lsmps_step_state& m = a.m;
  for (index_t t = blockIdx.x * blockDim.x + threadIdx.x; t < a.nf; t += stride) {
    const BoxIO& b = a.io[box_fluid(a, t)];
    const lsmps_step_state& s = b.s;
    const index_t k = t - b.fb;
    s.fluid.x[k] = m.fluid.x[t];
    s.fluid.y[k] = m.fluid.y[t];
    s.fluid.z[k] = m.fluid.z[t];
    s.fluid.vx[k] = m.fluid.vx[t];
    s.fluid.vy[k] = m.fluid.vy[t];
    s.fluid.vz[k] = m.fluid.vz[t];
    s.fluid.pressure[k] = m.fluid.pressure[t];
    if (s.fluid.surface_type) s.fluid.surface_type[k] = m.fluid.surface_type[t];
    s.pressure[k] = m.pressure[t];
    s.temporary_velocity.vx[k] = m.temporary_velocity.vx[t];
    s.temporary_velocity.vy[k] = m.temporary_velocity.vy[t];
    s.temporary_velocity.vz[k] = m.temporary_velocity.vz[t];
    copy3(m.velocity_laplacian, s.velocity_laplacian, t, k);
    copy3(m.pressure_gradient, s.pressure_gradient, t, k);
    copy3(m.ps_displacement, s.ps_displacement, t, k);
    copy3(m.smoothed_velocity, s.smoothed_velocity, t, k);
    s.ppe.rhs[k] = m.ppe.rhs[t];
    s.ppe.divergence[k] = m.ppe.divergence[t];
    if (s.ppe.pressure_laplacian) s.ppe.pressure_laplacian[k] = m.ppe.pressure_laplacian[t];
    const lsmps_moment* mk[2] = {&m.velocity_moment, &m.pressure_moment};
    const lsmps_moment* sk[2] = {&s.velocity_moment, &s.pressure_moment};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      sk[q]->moment_trace[k] = mk[q]->moment_trace[t];
      sk[q]->regularization_added[k] = mk[q]->regularization_added[t];
      sk[q]->info[k] = mk[q]->info[t];
      if (k == 0 && sk[q]->inversion_count) atomicAdd(sk[q]->inversion_count, 1);
    }
    // fluid cell list at sorted position t (box b's particles fill its range)
    s.fluid_cells.cell_ids[k] = m.fluid_cells.cell_ids[t] - b.cb;
    s.fluid_cells.sorted_indices[k] = m.fluid_cells.sorted_indices[t] - b.fb;
    // row offsets of both tables and of the PPE rows
    const index_t ef = m.fluid_neighbors.offsets[b.fb], ew = m.wall_neighbors.offsets[b.fb];
    // the box's first PPE slot (the PPE rows were assembled on the tables the
    // step started from, before its rebuild)
    const index_t rb = m.ppe.matrix.row_offsets[b.fb];
    s.fluid_neighbors.offsets[k] = m.fluid_neighbors.offsets[t] - ef;
    s.wall_neighbors.offsets[k] = m.wall_neighbors.offsets[t] - ew;
    s.ppe.matrix.row_offsets[k] = m.ppe.matrix.row_offsets[t] - rb;
    if (k + 1 == b.nf) {
      s.fluid_neighbors.offsets[b.nf] = m.fluid_neighbors.offsets[t + 1] - ef;
      s.wall_neighbors.offsets[b.nf] = m.wall_neighbors.offsets[t + 1] - ew;
      s.ppe.matrix.row_offsets[b.nf] = m.ppe.matrix.row_offsets[t + 1] - rb;
    }
  }
}

__global__ void scatter_walls_kernel(MergedArgs a) {
  const index_t stride = gridDim.x * blockDim.x;
  for (index_t t = blockIdx.x * blockDim.x + threadIdx.x; t < a.nw; t += stride) {
    const BoxIO& b = a.io[box_of(a.grids, a.nbox, t, 2)];
    const index_t k = t - b.wb;
    b.s.temporary_wall_velocity.vx[k] = a.m.temporary_wall_velocity.vx[t];
    b.s.temporary_wall_velocity.vy[k] = a.m.temporary_wall_velocity.vy[t];
    b.s.temporary_wall_velocity.vz[k] = a.m.temporary_wall_velocity.vz[t];
    b.s.wall_cells.cell_ids[k] = a.m.wall_cells.cell_ids[t] - b.cb;
    b.s.wall_cells.sorted_indices[k] = a.m.wall_cells.sorted_indices[t] - b.wb;
  }
}

__device__ __forceinline__ index_t shift_or_empty(index_t v, index_t base) { return v < 0 ? -1 : v - base; }

__global__ void scatter_cells_kernel(MergedArgs a) {
  const index_t stride = gridDim.x * blockDim.x;
  for (index_t c = blockIdx.x * blockDim.x + threadIdx.x; c < a.nc; c += stride) {
    const BoxIO& b = a.io[box_of(a.grids, a.nbox, c, 0)];
    const index_t k = c - b.cb;
    b.s.fluid_cells.cell_begin[k] = shift_or_empty(a.m.fluid_cells.cell_begin[c], b.fb);
    b.s.fluid_cells.cell_end[k] = shift_or_empty(a.m.fluid_cells.cell_end[c], b.fb);
    b.s.wall_cells.cell_begin[k] = shift_or_empty(a.m.wall_cells.cell_begin[c], b.wb);
    b.s.wall_cells.cell_end[k] = shift_or_empty(a.m.wall_cells.cell_end[c], b.wb);
  }
}

// The box holding entry e of a table whose rows are the merged fluid
// particles: the last box whose first row starts at or before e.
__device__ __forceinline__ int box_of_entry(const MergedArgs& a, const index_t* offsets, index_t e) {
  int lo = 0, hi = a.nbox - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const index_t fb = a.io[mid].fb;
    if (offsets[fb] <= e)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// The box of entry e for a thread whose entries only increase: one search
// for the first entry, then a walk forward past the boxes whose rows start
// at or before e (a grid-stride step crosses a box boundary rarely).
struct EntryCursor {
  const MergedArgs* a;
  const index_t* offsets;
  int b = -1;
  index_t next = 0;  // first entry of box b + 1 (INT32_MAX past the last box)
  __device__ index_t start_of(int k) const {
    return k < a->nbox ? offsets[a->io[k].fb] : static_cast<index_t>(0x7fffffff);
  }
  // Box b ends with start_of(b) <= e < start_of(b + 1): the last box whose
  // rows start at or before e (boxes without fluid share their successor's
  // start and are walked past).
  __device__ int box(index_t e) {
    if (b < 0) {
      b = box_of_entry(*a, offsets, e);
      next = start_of(b + 1);
    }
    while (e >= next) {
      ++b;
      next = start_of(b + 1);
    }
    return b;
  }
};

// Where a thread's current box sends entries of one table: the box's first
// merged entry, the index shift into the box's numbering, the box's own
// buffers and capacity; reloaded only when the cursor moves to another box.
struct EntryTarget {
  int box = -1;
  index_t start = 0;
  index_t shift = 0;
  unsigned long long cap = 0;
  index_t* idx = nullptr;
};

// Table T: 0 fluid rows, 1 wall rows.
template <int T>
__device__ __forceinline__ void load_target(const MergedArgs& a, const index_t* offsets, int bi, EntryTarget& g) {
  const BoxIO& b = a.io[bi];
  g.box = bi;
  g.start = offsets[b.fb];
  if (T == 0) {
    g.shift = b.fb;
    g.cap = b.s.fluid_neighbors.neighbor_count;
    g.idx = b.s.fluid_neighbors.indices;
  } else {
    g.shift = b.wb;
    g.cap = b.s.wall_neighbors.neighbor_count;
    g.idx = b.s.wall_neighbors.indices;
  }
}

// Entries [0, total) of table T into the boxes' buffers, kUnroll entries
// per thread and round, one grid stride apart (each load coalesced across
// the warp; the round's loads issued together).  A box's rows
// may fit the merged capacity (the sum of the boxes') but not its own: such
// entries are not copied and the capacity flag is raised with the box's
// required count, as a solo step would report.
template <int T>
__device__ void scatter_table(const MergedArgs& a, const index_t* offsets, const index_t* src_idx, index_t total) {
  constexpr int kUnroll = 4;
  const long long step = static_cast<long long>(gridDim.x) * blockDim.x;
  EntryCursor cur{&a, offsets};
  EntryTarget g;
  for (long long e0 = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e0 < total;
       e0 += step * kUnroll) {
    index_t v[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      if (e0 + u * step < total) {
        const index_t e = static_cast<index_t>(e0 + u * step);
        v[u] = src_idx[e];
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      if (e0 + u * step >= total) break;
      const index_t e = static_cast<index_t>(e0 + u * step);
      const int bi = cur.box(e);
      if (bi != g.box) load_target<T>(a, offsets, bi, g);
      const index_t eb = e - g.start;
      if (static_cast<unsigned long long>(eb) >= g.cap) {
        record_required(a.status, static_cast<unsigned long long>(eb) + 1);
        continue;
      }
      g.idx[eb] = v[u] - g.shift;
    }
  }
}

// The rows of both neighbour tables (indices shifted to the box's
// numbering).  A box with no fluid has no entries;
// the cursor walks past it because its first row starts where the next
// box's does.
__global__ void scatter_entries_kernel(MergedArgs a) {
  // the rebuilt totals, held to the merged capacities (beyond them the
  // rebuild wrote nothing and has raised the capacity flag)
  const index_t kf = static_cast<index_t>(min(static_cast<unsigned long long>(a.m.fluid_neighbors.offsets[a.nf]),
                                              static_cast<unsigned long long>(a.m.fluid_neighbors.neighbor_count)));
  const index_t kw = static_cast<index_t>(min(static_cast<unsigned long long>(a.m.wall_neighbors.offsets[a.nf]),
                                              static_cast<unsigned long long>(a.m.wall_neighbors.neighbor_count)));
  scatter_table<0>(a, a.m.fluid_neighbors.offsets, a.m.fluid_neighbors.indices, kf);
  scatter_table<1>(a, a.m.wall_neighbors.offsets, a.m.wall_neighbors.indices, kw);
  // (the PPE slots were written into the boxes' own matrices by the step)
}

// Plain form: the 81-entry inverses of both kinds.
__global__ void scatter_inverse_kernel(MergedArgs a) {
  const long long total = 81LL * a.nf;
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long v = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; v < total; v += stride) {
    const index_t t = static_cast<index_t>(v / 81);
    const BoxIO& b = a.io[box_fluid(a, t)];
    const long long dst = v - 81LL * b.fb;
    b.s.velocity_moment.inverse_matrices[dst] = a.m.velocity_moment.inverse_matrices[v];
    b.s.pressure_moment.inverse_matrices[dst] = a.m.pressure_moment.inverse_matrices[v];
  }
}

}  // namespace

void release_merged(MergedBatch& mb) {
  if (mb.ctx) lsmps_ctx_destroy(mb.ctx);
  for (void* p : mb.allocations) cudaFree(p);
  mb = MergedBatch{};
}

// True when every box has the first box's parameters apart from the grid
// origin and dims (the cell size must agree too).
bool boxes_mergeable(const std::vector<lsmps_params>& params) {
  if (params.empty()) return false;
  lsmps_params ref = params[0];
  std::memset(ref.grid.origin, 0, sizeof(ref.grid.origin));
  std::memset(ref.grid.dims, 0, sizeof(ref.grid.dims));
  for (const lsmps_params& p0 : params) {
    lsmps_params p = p0;
    std::memset(p.grid.origin, 0, sizeof(p.grid.origin));
    std::memset(p.grid.dims, 0, sizeof(p.grid.dims));
    if (std::memcmp(&p, &ref, sizeof(p)) != 0) return false;
  }
  return true;
}

lsmps_status prepare_merged(MergedBatch& mb, int device, cudaStream_t stream,
                            const std::vector<lsmps_params>& params, const std::vector<lsmps_step_state>& states,
                            int precision, int autotune_repeats, std::string& error) {
  release_merged(mb);
  const int nbox = static_cast<int>(states.size());
  std::vector<BoxGrid> grids(nbox);
  std::vector<BoxIO> io(nbox);
  long long nf = 0, nw = 0, nc = 0, capf = 0, capw = 0;
  for (int b = 0; b < nbox; ++b) {
    const lsmps_step_state& s = states[b];
    const lsmps_grid& g = params[b].grid;
    const long long cells = static_cast<long long>(g.dims[0]) * g.dims[1] * g.dims[2];
    if (s.fluid_cells.cell_count != static_cast<size_t>(cells) || s.wall_cells.cell_count != static_cast<size_t>(cells)) {
      error = "box " + std::to_string(b) + ": cell lists do not match its grid";
      return LSMPS_INVALID_ARGUMENT;
    }
    if (!s.fluid.surface_type || !s.pressure || !s.ppe.pressure_laplacian) {
      error = "box " + std::to_string(b) + ": the merged form needs labels, a pressure input and the wall rhs view";
      return LSMPS_INVALID_ARGUMENT;
    }
    for (int k = 0; k < 3; ++k) {
      grids[b].origin[k] = g.origin[k];
      grids[b].dims[k] = g.dims[k];
    }
    grids[b].cell_base = static_cast<index_t>(nc);
    grids[b].fluid_base = static_cast<index_t>(nf);
    grids[b].wall_base = static_cast<index_t>(nw);
    io[b].s = s;
    io[b].nf = static_cast<index_t>(s.fluid.count);
    io[b].nw = static_cast<index_t>(s.walls.count);
    io[b].nc = static_cast<index_t>(cells);
    io[b].fb = grids[b].fluid_base;
    io[b].wb = grids[b].wall_base;
    io[b].cb = grids[b].cell_base;
    nf += s.fluid.count;
    nw += s.walls.count;
    nc += cells;
    capf += static_cast<long long>(s.fluid_neighbors.neighbor_count);
    capw += static_cast<long long>(s.wall_neighbors.neighbor_count);
  }
  if (nf + capf > INT_MAX || nc > INT_MAX || nw > INT_MAX || capw > INT_MAX) {
    error = "the merged set exceeds the 32-bit index range";
    return LSMPS_INDEX_OVERFLOW;
  }
  if (cudaSetDevice(device) != cudaSuccess) return LSMPS_CUDA_ERROR;
  bool ok = true;
  auto alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (!ok || cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
      ok = false;
      return nullptr;
    }
    mb.allocations.push_back(p);
    return p;
  };
  auto d = [&](long long n) { return static_cast<double*>(alloc(static_cast<size_t>(n) * sizeof(double))); };
  auto i32 = [&](long long n) { return static_cast<int32_t*>(alloc(static_cast<size_t>(n) * sizeof(int32_t))); };
  lsmps_step_state m{};
  m.fluid.count = nf;
  m.fluid.x = d(nf), m.fluid.y = d(nf), m.fluid.z = d(nf);
  m.fluid.vx = d(nf), m.fluid.vy = d(nf), m.fluid.vz = d(nf);
  m.fluid.pressure = d(nf);
  m.fluid.surface_type = i32(nf);
  m.walls.count = nw;
  m.walls.x = d(nw), m.walls.y = d(nw), m.walls.z = d(nw);
  m.walls.vx = d(nw), m.walls.vy = d(nw), m.walls.vz = d(nw);
  m.walls.normal_x = d(nw), m.walls.normal_y = d(nw), m.walls.normal_z = d(nw);
  lsmps_cells* cls[2] = {&m.fluid_cells, &m.wall_cells};
  for (int q = 0; q < 2; ++q) {
    const long long np = q == 0 ? nf : nw;
    cls[q]->particle_count = np;
    cls[q]->cell_count = nc;
    cls[q]->cell_ids = i32(np);
    cls[q]->sorted_indices = i32(np);
    cls[q]->cell_begin = i32(nc);
    cls[q]->cell_end = i32(nc);
  }
  m.fluid_neighbors.particle_count = nf;
  m.fluid_neighbors.neighbor_count = capf;
  m.fluid_neighbors.offsets = i32(nf + 1);
  m.fluid_neighbors.indices = i32(capf);
  m.wall_neighbors.particle_count = nf;
  m.wall_neighbors.neighbor_count = capw;
  m.wall_neighbors.offsets = i32(nf + 1);
  m.wall_neighbors.indices = i32(capw);
  m.temporary_velocity.count = nf;
  m.temporary_velocity.vx = d(nf), m.temporary_velocity.vy = d(nf), m.temporary_velocity.vz = d(nf);
  m.temporary_wall_velocity.count = nw;
  m.temporary_wall_velocity.vx = d(nw), m.temporary_wall_velocity.vy = d(nw), m.temporary_wall_velocity.vz = d(nw);
  lsmps_vector* vecs[4] = {&m.velocity_laplacian, &m.pressure_gradient, &m.ps_displacement, &m.smoothed_velocity};
  for (lsmps_vector* v : vecs) {
    v->count = nf;
    v->x = d(nf), v->y = d(nf), v->z = d(nf);
  }
  lsmps_moment* mom[2] = {&m.velocity_moment, &m.pressure_moment};
  const lsmps_moment* box0[2] = {&states[0].velocity_moment, &states[0].pressure_moment};
  for (int q = 0; q < 2; ++q) {
    *mom[q] = *box0[q];
    mom[q]->particle_count = nf;
    mom[q]->inverse_matrices = d(81 * nf);
    mom[q]->moment_trace = d(nf);
    mom[q]->regularization_added = d(nf);
    mom[q]->info = i32(nf);
    mom[q]->inversion_count = i32(1);
  }
  m.ppe.matrix.rows = nf;
  m.ppe.matrix.cols = nf;
  m.ppe.matrix.nnz = nf + capf;
  m.ppe.matrix.row_offsets = i32(nf + 1);
  // The merged context writes every box's PPE rows straight into the box's
  // own matrix (lsmps_ctx::box_ppe), so the merged matrix holds only the
  // row offsets; its slot arrays are placeholders that are never written
  // (the view keeps the merged capacity, which the assembly checks).
  m.ppe.matrix.col_indices = i32(16);
  m.ppe.matrix.values = d(16);
  m.ppe.rhs = d(nf), m.ppe.pressure = d(nf), m.ppe.divergence = d(nf), m.ppe.pressure_laplacian = d(nf);
  m.pressure = d(nf);
  mb.grids = static_cast<BoxGrid*>(alloc(grids.size() * sizeof(BoxGrid)));
  std::vector<PpeBoxOut> ppe_out(nbox);
  for (int b = 0; b < nbox; ++b)
    ppe_out[b] = PpeBoxOut{states[b].ppe.matrix.col_indices, states[b].ppe.matrix.values,
                           static_cast<unsigned long long>(states[b].ppe.matrix.nnz)};
  mb.box_ppe = static_cast<PpeBoxOut*>(alloc(ppe_out.size() * sizeof(PpeBoxOut)));
  mb.io = alloc(io.size() * sizeof(BoxIO));
  if (!ok) {
    cudaGetLastError();
    release_merged(mb);
    error = "merged batch allocation failed";
    return LSMPS_CUDA_ERROR;
  }
  if (cudaMemcpy(mb.grids, grids.data(), grids.size() * sizeof(BoxGrid), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(mb.box_ppe, ppe_out.data(), ppe_out.size() * sizeof(PpeBoxOut), cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(mb.io, io.data(), io.size() * sizeof(BoxIO), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(mom[0]->inversion_count, 0, sizeof(int32_t)) != cudaSuccess ||
      cudaMemset(mom[1]->inversion_count, 0, sizeof(int32_t)) != cudaSuccess) {
    release_merged(mb);
    error = "merged batch set-up copies failed";
    return LSMPS_CUDA_ERROR;
  }
  mb.state = m;
  mb.nbox = nbox;
  mb.nf = static_cast<index_t>(nf);
  mb.nw = static_cast<index_t>(nw);
  mb.nc = static_cast<index_t>(nc);
  mb.params = params[0];
  mb.params.grid.dims[0] = static_cast<int>(nc);
  mb.params.grid.dims[1] = 1;
  mb.params.grid.dims[2] = 1;
  mb.precision = precision;
  lsmps_status st = lsmps_ctx_create(device, &mb.ctx);
  if (st) {
    release_merged(mb);
    error = "merged context creation failed";
    return st;
  }
  lsmps_ctx_set_stream(mb.ctx, stream);
  lsmps_ctx_set_precision(mb.ctx, precision);
  mb.ctx->boxes = mb.grids;
  mb.ctx->nbox = nbox;
  mb.ctx->box_ppe = mb.box_ppe;
  // The merged tables and labels from the boxes' current positions (as the
  // boxes' own tables were built), then the scratch for the step and,
  // optionally, the launch shapes tuned on the merged set.
  st = lsmps_ctx_reserve(mb.ctx, nf, nw, nc);
  if (!st) {
    MergedArgs a = merged_args(mb);
    gather_kernel<<<mb.ctx->sm_count * 8, kThreads, 0, stream>>>(a);
    st = lsmps_build_neighbor_lists(mb.ctx, &m.fluid, &m.walls, &mb.params, &m.fluid_cells, &m.wall_cells,
                                    &m.fluid_neighbors, &m.wall_neighbors);
  }
  if (!st) st = lsmps_classify_surface(mb.ctx, &m.fluid, &m.walls, &m.fluid_neighbors, &m.wall_neighbors, &mb.params,
                                       nullptr);
  if (!st && autotune_repeats > 0) st = lsmps_autotune(mb.ctx, &mb.params, &mb.state, autotune_repeats, nullptr);
  if (!st) st = lsmps_ctx_set_synchronous(mb.ctx, 0);
  if (st) {
    error = std::string("merged set-up: ") + lsmps_ctx_last_error(mb.ctx);
    release_merged(mb);
    return st;
  }
  return LSMPS_OK;
}

// One launch's work on the stream (recorded into the graph at capture).
lsmps_status queue_merged(MergedBatch& mb, cudaStream_t stream, std::string& error) {
  lsmps_ctx* ctx = mb.ctx;
  MergedArgs a = merged_args(mb);
  const int blocks = ctx->sm_count * 8;
  launch_named(ctx, "gather_kernel", gather_kernel, dim3(blocks), dim3(kThreads), 0, a);
  lsmps_status st = lsmps_step(ctx, &mb.params, &mb.state);
  if (st) {
    error = std::string("merged step: ") + lsmps_ctx_last_error(ctx);
    return st;
  }
  launch_named(ctx, "scatter_particles_kernel", scatter_particles_kernel, dim3(blocks), dim3(kThreads), 0, a);
  launch_named(ctx, "scatter_walls_kernel", scatter_walls_kernel, dim3(blocks), dim3(kThreads), 0, a);
  launch_named(ctx, "scatter_cells_kernel", scatter_cells_kernel, dim3(blocks), dim3(kThreads), 0, a);
  launch_named(ctx, "scatter_entries_kernel", scatter_entries_kernel, dim3(blocks), dim3(kThreads), 0, a);
  if (a.full_inverse)
    launch_named(ctx, "scatter_inverse_kernel", scatter_inverse_kernel, dim3(blocks), dim3(kThreads), 0, a);
  (void)stream;
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    error = std::string("merged scatter: ") + cudaGetErrorString(e);
    return LSMPS_CUDA_ERROR;
  }
  return LSMPS_OK;
}

}  // namespace lsmps
