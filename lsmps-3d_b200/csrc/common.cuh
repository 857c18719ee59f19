// common.cuh - shared internals of the sm_100a LSMPS hot path: the context,
// the device status word, launch bookkeeping and the per-neighbour formulas
// every gather kernel uses.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "lsmps_b200.h"

namespace lsmps {

using index_t = int32_t;

constexpr int kWarp = 32;

// Bits of DeviceStatus::flags.
constexpr unsigned kFlagCapacity = 1u;
constexpr unsigned kFlagNonFinite = 2u;
constexpr unsigned kFlagIndexOverflow = 4u;
constexpr unsigned kFlagNonSpd = 8u;
constexpr unsigned kFlagBadIndex = 16u;  // bounds-checked build: a table entry out of range

// Written by kernels, read back once per synchronous call (or per
// lsmps_ctx_synchronize in asynchronous mode).
struct DeviceStatus {
  unsigned int flags;
  unsigned int non_spd;
  unsigned long long required;
  unsigned int fallbacks;  // mixed form: moment matrices factorised in FP64
  unsigned int pad;
};

__device__ __forceinline__ void raise_flag(DeviceStatus* s, unsigned f) { atomicOr(&s->flags, f); }

__device__ __forceinline__ void record_required(DeviceStatus* s, unsigned long long required) {
  atomicOr(&s->flags, kFlagCapacity);
  atomicMax(&s->required, required);
}

// Linear kernel weight, identical in every reference module:
// surface_detection.cu:26-31, moment_matrix.cu:145-150,
// explicit_update.cu:121-126, ppe_matrix.cu:148-153.
__device__ __forceinline__ double lin_weight(double distance, double support_radius) {
  return distance >= support_radius ? 0.0 : 1.0 - distance / support_radius;
}

// correction_weight also rejects zero distance (pressure_correction.cu:127-132).
__device__ __forceinline__ double correction_weight(double distance, double support_radius) {
  return (distance >= support_radius || distance <= 0.0) ? 0.0 : 1.0 - distance / support_radius;
}

// The same weights with the division by r_e replaced by a multiplication with
// 1/r_e (one rounding instead of an IEEE division sequence on the FP64 pipe).
// The value differs from the reference's by at most one ulp of d/r_e; a
// distance within that ulp of r_e may get weight 0 instead of ~1e-16.  Used by
// the operator kernels, whose outputs are compared within a tolerance; the
// label kernel keeps the reference's exact expressions.
__device__ __forceinline__ double lin_weight_mul(double distance, double inv_re) {
  const double w = 1.0 - distance * inv_re;
  return w > 0.0 ? w : 0.0;
}

__device__ __forceinline__ double correction_weight_mul(double distance, double inv_re) {
  return distance <= 0.0 ? 0.0 : lin_weight_mul(distance, inv_re);
}

// Type-A quadratic basis of the r_e-scaled offset with the multiply-by-inverse
// form of explicit_update.cu:128-146 (ppe_matrix.cu:155-173 and
// pressure_correction.cu:138-156 are the same).
__device__ __forceinline__ void basis_a_mul(double dx, double dy, double dz, double inv_re, double b[9]) {
  const double sx = dx * inv_re, sy = dy * inv_re, sz = dz * inv_re;
  b[0] = sx;
  b[1] = sy;
  b[2] = sz;
  b[3] = sx * sx;
  b[4] = sy * sy;
  b[5] = sz * sz;
  b[6] = sx * sy;
  b[7] = sy * sz;
  b[8] = sz * sx;
}

// Wall Neumann vector q of moment_matrix.cu:177-201 (Type-A part).
__device__ __forceinline__ void neumann_a(double dx, double dy, double dz, double nx, double ny, double nz,
                                          double inv_re, double q[9]) {
  q[0] = nx;
  q[1] = ny;
  q[2] = nz;
  q[3] = 2.0 * dx * nx * inv_re;
  q[4] = 2.0 * dy * ny * inv_re;
  q[5] = 2.0 * dz * nz * inv_re;
  q[6] = (dy * nx + dx * ny) * inv_re;
  q[7] = (dz * ny + dy * nz) * inv_re;
  q[8] = (dx * nz + dz * nx) * inv_re;
}

inline int div_up(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

// One box of a merged batch (batch.cu): independent particle boxes stepped
// as one particle set, each with its own cell grid.  Box b's cells are the
// global cells [cell_base, cell_base + dims product), its fluid particles
// [fluid_base, next box's), its walls [wall_base, next box's).  The cell
// hash and the neighbour search of a merged set look each particle's or
// cell's box up in this table; every other kernel is per particle and needs
// nothing of it.
struct BoxGrid {
  double origin[3];
  int dims[3];
  index_t cell_base;
  index_t fluid_base;
  index_t wall_base;
};

// Where a merged batch's PPE rows go: box b's own matrix (its column and
// value arrays and their capacity), written by the PPE kernels directly so
// that the slots need no copy out of the merged matrix.
struct PpeBoxOut {
  index_t* col;
  double* val;
  unsigned long long cap;
};

// The box holding global cell c (or particle t, with field = the box's first
// index of that set): the last box whose base is <= the value.
__device__ __forceinline__ int box_of(const BoxGrid* __restrict__ boxes, int nbox, index_t v, int field) {
  int lo = 0, hi = nbox - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const index_t base = field == 0 ? boxes[mid].cell_base : field == 1 ? boxes[mid].fluid_base : boxes[mid].wall_base;
    if (base <= v)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Lane groups: G consecutive lanes of a warp (G a power of two dividing 32)
// share one particle.  group_mask names the calling thread's group only, so
// the shuffles stay valid when other groups of the warp have left.
template <int G>
__device__ __forceinline__ unsigned group_mask() {
  return ((G == 32) ? 0xffffffffu : ((1u << G) - 1u)) << ((threadIdx.x & (kWarp - 1)) & ~(G - 1));
}

// The particle a thread (or lane group) visits: its index in the context's
// visiting order (lsmps_ctx::order), or the index itself.
__device__ __forceinline__ index_t visit(const int32_t* __restrict__ order, index_t t) {
  return order ? order[t] : t;
}

// Where the particle visited at position t finds its own packed record: at t
// when the records are packed in cell-sorted (visiting) order, else at i.
__device__ __forceinline__ index_t self_of(int sorted, index_t t, index_t i) { return sorted ? t : i; }

// Sum over the lanes of a group; every lane of the group ends with the total.
template <int G>
__device__ __forceinline__ double group_sum(double v, unsigned mask) {
#pragma unroll
  for (int d = G / 2; d > 0; d >>= 1) v += __shfl_xor_sync(mask, v, d);
  return v;
}

}  // namespace lsmps

// Opaque context of the C ABI.
struct lsmps_ctx {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  int precision = LSMPS_PRECISION_PLAIN;
  bool synchronous = true;
  lsmps::DeviceStatus* d_status = nullptr;
  lsmps::DeviceStatus* h_status = nullptr;  // pinned mirror
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  size_t scratch_used = 0;
  unsigned long long launches = 0;
  unsigned long long required = 0;
  unsigned long long fallbacks = 0;
  std::string last_error;
  // Per-launch CUDA events while profiling is on (lsmps_ctx_set_profiling).
  struct ProfileRecord {
    const char* name;
    cudaEvent_t start;
    cudaEvent_t stop;
  };
  bool profiling = false;
  std::vector<ProfileRecord> profile;
  size_t profile_used = 0;
  // Launch-shape knobs (lsmps_knob).
  int knob[LSMPS_KNOB_COUNT] = {1, 1, 2};
  // Device-resident time step read by the kernels that use dt (provision
  // combine, PPE right-hand side, velocity/position update) instead of
  // lsmps_params::time_step, while set (lsmps_ctx_set_device_time_step).
  const double* device_dt = nullptr;
  // lsmps_ctx_set_step_events: waited for before the step's provision stage /
  // recorded after its pressure correction (cudaEvent_t, or NULL).
  void* step_wall_event = nullptr;
  void* step_input_event = nullptr;
  void* step_output_event = nullptr;
  // Set by lsmps_step around its moment stage (the step's wall event, or
  // NULL): the mixed moment stage waits for it right before it packs the
  // walls, after the fluid sums.
  void* walls_wait_event = nullptr;
  // Order in which the per-particle gather kernels of lsmps_step visit the
  // fluid (the fluid cell list's sorted indices: particles of one cell on
  // adjacent threads, so their neighbour records are shared in cache), or
  // NULL for index order.  Visiting order changes no result.
  const int32_t* order = nullptr;
  bool cell_order = true;
  // The fluid cell list this context built last (lsmps_build_neighbor_lists
  // or a step's rebuild): only such a list, known to hold a permutation of
  // the fluid, is used as a visiting order.
  const int32_t* built_order = nullptr;
  size_t built_order_count = 0;
  // Cell-sorted rows of the fluid table: for every CSR entry, the neighbour's
  // position in the fluid cell list (its sorted position) instead of its
  // index, written by this context's builds of the table next to the indices
  // (capacity: entries), and the table (offsets array), cell list and particle
  // count they describe (spos_table NULL: none valid).  While lsmps_step
  // visits the fluid in the order of that cell list, its gather kernels read
  // these rows and fluid records packed in cell-sorted order, so a home
  // cell's neighbours come from a few contiguous runs of records whatever
  // the caller's numbering (sorted_rows; results identical either way).
  // sorted_labels holds the labels in cell-sorted order for the NearSurface
  // expansion.
  int32_t* fluid_spos = nullptr;
  size_t fluid_spos_cap = 0;
  int32_t* sorted_labels = nullptr;
  size_t sorted_labels_cap = 0;
  const int32_t* spos_table = nullptr;
  const int32_t* spos_order = nullptr;
  size_t spos_count = 0;
  bool sorted_rows = true;
  // Inside lsmps_step (step_packs): which record packs already hold what a
  // later stage of the same step would pack again (bit 0: wall positions in
  // pack_wall[0], bit 1: wall normals in pack_wall[2], bit 2: fluid positions
  // in pack_fluid[0], packed in packs_fluid_order).  The walls do not move
  // during a step and the fluid does not move before the correction; any
  // other pack into those buffers clears its bit (packed.cu).
  bool step_packs = false;
  unsigned packs_ready = 0;
  const int32_t* packs_fluid_order = nullptr;
  // CSR count pass shape: false = warp per home cell, lane per home particle
  // (the fastest on a GPU the build has to itself); true = block per home
  // cell, warp per two home particles, which leaves the streams of a batched
  // graph running beside it faster (set for batch worker contexts).
  bool csr_cell_blocks = false;
  // 32-byte neighbour records (packed.cuh): two fluid and three wall arrays.
  double4* pack_fluid[2] = {nullptr, nullptr};
  double4* pack_wall[3] = {nullptr, nullptr, nullptr};
  size_t pack_fluid_cap = 0;
  size_t pack_wall_cap = 0;
  // Mixed form (LSMPS_PRECISION_MIXED): per fluid particle the 31 FP64 fluid
  // moment sums ([31][n]) and the compact FP32 operator rows of the velocity
  // and pressure inverses ([n][36]: Laplacian row, then rows 0, 1, 2), both
  // by visiting position (lsmps_ctx::order), as are the FP64 rows and flags.
  double* mixed_sums = nullptr;
  float* mixed_rows[2] = {nullptr, nullptr};
  double* mixed_rows64[2] = {nullptr, nullptr};  // rows of matrices factorised in FP64
  uint8_t* mixed_flag[2] = {nullptr, nullptr};   // 1: the particle's rows are in mixed_rows64
  // The particles whose rows are in mixed_rows64, per kind, listed by the
  // step's moment stage (mixed_count[kind] entries, in no particular order):
  // the FP32 consumer kernels skip them and an FP64 pass over the list
  // finishes them.
  int32_t* mixed_list[2] = {nullptr, nullptr};
  unsigned int* mixed_count = nullptr;  // [4]
  size_t mixed_cap = 0;
  // Condition-estimate threshold above which a moment matrix is factorised
  // in FP64 in the mixed form.  One FP64 refinement of an FP32 factor leaves
  // a relative error of about (kappa u)^2 (u = 2^-24): ~4e-7 at 1e4, ~4e-3 at
  // 1e6.
  double kappa_threshold = 1.0e4;
  // Operator forward/backward pair (adjoint.cu): fluid-only inverse, its
  // trace / regularisation / info, and the backward's per-particle stash.
  double* adj_inverse = nullptr;
  double* adj_trace = nullptr;
  double* adj_reg = nullptr;
  int32_t* adj_info = nullptr;
  int32_t* adj_count = nullptr;
  double* adj_stash = nullptr;
  size_t adj_cap = 0;
  // Backward form: false = transpose + gather (deterministic, the default),
  // true = scatter with FP64 atomics (lsmps_ctx_set_adjoint_atomic).
  bool adjoint_atomic = false;
  // Merged batch (batch.cu): the boxes' grid table in device memory while
  // this context steps a merged particle set, else NULL.
  const lsmps::BoxGrid* boxes = nullptr;
  int nbox = 0;
  // ... and where each box's PPE rows go (device table, nbox entries), or
  // NULL to write them into the matrix the call is given.
  const lsmps::PpeBoxOut* box_ppe = nullptr;
  // The step operator pair (step_adjoint.cu): inverses, traces,
  // regularisations, info and counts of the velocity Dirichlet-A and pressure
  // Neumann-A kinds, and the backward's stash.
  double* sop_inverse[2] = {nullptr, nullptr};
  double* sop_trace[2] = {nullptr, nullptr};
  double* sop_reg[2] = {nullptr, nullptr};
  int32_t* sop_info[2] = {nullptr, nullptr};
  int32_t* sop_count = nullptr;
  double* sop_stash = nullptr;
  size_t sop_cap = 0;
};

namespace lsmps {

// Bump allocator over the context's scratch; reset at the start of each API
// call.  Grows (outside stream capture) when a call needs more.
class Scratch {
 public:
  explicit Scratch(lsmps_ctx* ctx) : ctx_(ctx) { ctx_->scratch_used = 0; }
  // Ensure `bytes` of scratch in total for this call.
  bool reserve(size_t bytes);
  template <typename T>
  T* take(size_t count) {
    const size_t bytes = ((count * sizeof(T)) + 255) & ~size_t(255);
    if (ctx_->scratch_used + bytes > ctx_->scratch_bytes) return nullptr;
    T* p = reinterpret_cast<T*>(static_cast<char*>(ctx_->scratch) + ctx_->scratch_used);
    ctx_->scratch_used += bytes;
    return p;
  }

 private:
  lsmps_ctx* ctx_;
};

// Grow the pack arrays to hold nf fluid and nw wall records (outside stream
// capture; returns false if that is impossible).
bool ensure_packs(lsmps_ctx* ctx, size_t nf, size_t nw);
// The cell-sorted row array for `entries` fluid CSR entries and the sorted
// label array for nf particles (outside capture; false: not available).
bool ensure_sorted_rows(lsmps_ctx* ctx, size_t entries, size_t nf);
// Grow the mixed-form arrays to nf fluid particles (outside stream capture).
bool ensure_mixed(lsmps_ctx* ctx, size_t nf);
void free_mixed(lsmps_ctx* ctx);
// Grow / free the operator pair's scratch (adjoint.cu).
bool ensure_adjoint(lsmps_ctx* ctx, size_t n);
void free_adjoint(lsmps_ctx* ctx);
// Grow / free the step operator pair's scratch (step_adjoint.cu).
bool ensure_step_ops(lsmps_ctx* ctx, size_t n);
void free_step_ops(lsmps_ctx* ctx);

lsmps_status fail(lsmps_ctx* ctx, lsmps_status st, const char* what);
lsmps_status check_launch(lsmps_ctx* ctx, const char* what);
// Begin an API call: clear the device status in synchronous mode.
lsmps_status begin_call(lsmps_ctx* ctx);
// End an API call: in synchronous mode wait and fold the device status.
lsmps_status end_call(lsmps_ctx* ctx, lsmps_status st);
lsmps_status fold_status(lsmps_ctx* ctx);
// Bounds-checked build (bounds.cu): validate a CSR table (rows + 1 offsets,
// entries below `capacity`, indices below n_src) before kernels read it;
// returns LSMPS_INVALID_ARGUMENT with `what` when it is not valid.  A no-op
// in the normal build.
lsmps_status check_table(lsmps_ctx* ctx, const index_t* offsets, const index_t* indices, size_t rows,
                         unsigned long long capacity, size_t n_src, const char* what);
// The fluid table (indices into the fluid) and, if given, the wall table.
lsmps_status check_neighbor_tables(lsmps_ctx* ctx, size_t n_fluid, size_t n_wall, const lsmps_csr& fn,
                                   const lsmps_csr* wn);

// Event pair for the next profiled launch (grown on demand, reused across steps).
lsmps_ctx::ProfileRecord* profile_slot(lsmps_ctx* ctx, const char* name);

template <typename Kernel, typename... Args>
inline void launch_named(lsmps_ctx* ctx, const char* name, Kernel kernel, dim3 grid, dim3 block, size_t smem,
                         Args... args) {
  if (grid.x == 0 || grid.y == 0 || grid.z == 0) return;
  lsmps_ctx::ProfileRecord* rec = ctx->profiling ? profile_slot(ctx, name) : nullptr;
  if (rec) cudaEventRecord(rec->start, ctx->stream);
  kernel<<<grid, block, smem, ctx->stream>>>(args...);
  if (rec) cudaEventRecord(rec->stop, ctx->stream);
  ++ctx->launches;
}

#define launch(ctx, kernel, ...) launch_named(ctx, #kernel, kernel, __VA_ARGS__)

// NVTX range for the host-side span of one stage (what a timeline profiler
// shows as the stage's launch window).  NVTX is header-only: with no tool
// attached a push/pop costs a few nanoseconds.
struct StageRange {
  explicit StageRange(const char* name) { nvtxRangePushA(name); }
  ~StageRange() { nvtxRangePop(); }
  StageRange(const StageRange&) = delete;
  StageRange& operator=(const StageRange&) = delete;
};

// Scan helpers (scan.cu).  Exclusive scan of n int32 values into out (may
// alias in); values and partial sums are accumulated in 64 bits and any
// result above INT32_MAX raises kFlagIndexOverflow.  The grand total is
// written to *total and/or *total_i32 (device pointers) when they are non-null.
size_t scan_scratch_bytes(size_t n);
lsmps_status exclusive_scan_i32(lsmps_ctx* ctx, Scratch& scratch, const index_t* in, index_t* out, size_t n,
                                unsigned long long* total, index_t* total_i32);

// Cell-list build shared by lsmps_build_cell_list and the neighbour search
// (cells.cu).
size_t cell_list_scratch_bytes(size_t n, size_t ncell);
// boxes (a merged batch's device table, ctx->nbox entries): hash each
// particle on its box's grid (box_field 1: fluid ranges, 2: wall ranges);
// grid then only supplies the cell size and the total cell count
// (dims product).
lsmps_status build_cell_list_impl(lsmps_ctx* ctx, Scratch& scratch, const double* x, const double* y,
                                  const double* z, size_t count, const lsmps_grid& grid,
                                  const lsmps_cells& cells, const BoxGrid* boxes = nullptr,
                                  int box_field = 0);
lsmps_status validate_grid(lsmps_ctx* ctx, const lsmps_grid& grid);

}  // namespace lsmps
