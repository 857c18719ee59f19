// reorder.cu - fluid particles renumbered in cell order.
//
// The gather kernels read each neighbour's 32-byte record by particle
// index; when particle numbering follows space (particles of one cell
// consecutive, neighbouring cells close), the records of a row sit in a few
// cache lines and are shared by the rows of nearby particles.  Input whose
// numbering is unrelated to space (particles read from a file in arbitrary
// order, or mixed by long runs) scatters every row over the whole array.
// lsmps_reorder_fluid renumbers the fluid SoA in the order of the fluid cell
// list (cell id ascending, stable: equal cells keep their previous order) and
// returns the permutation, so a driver can renumber once, or every so many
// steps, and remap anything it keeps per particle.
//
// Because the cell list is stable and rows are written in sorted-position
// order inside each cell, the neighbour rows rebuilt after a renumbering
// list the same neighbours in the same order (under the new numbers): every
// sum of the step runs in the same order and the step's results are the
// same, renumbered, bit for bit.
#include "impl.cuh"

namespace lsmps {
namespace {

constexpr int kThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kThreads)
    gather_kernel(const T* __restrict__ src, const index_t* __restrict__ order, index_t n, T* __restrict__ dst) {
  for (index_t k = blockIdx.x * kThreads + threadIdx.x; k < n; k += gridDim.x * kThreads) dst[k] = src[order[k]];
}

template <typename T>
__global__ void __launch_bounds__(kThreads) copy_back_kernel(const T* __restrict__ src, index_t n, T* __restrict__ dst) {
  for (index_t k = blockIdx.x * kThreads + threadIdx.x; k < n; k += gridDim.x * kThreads) dst[k] = src[k];
}

}  // namespace

lsmps_status reorder_fluid_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_cells& cells, int32_t* permutation) {
  if (f.count == 0) return LSMPS_OK;
  if (cells.particle_count < f.count || !cells.sorted_indices)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "fluid cell list smaller than the fluid");
  if (f.count > static_cast<size_t>(INT32_MAX)) return fail(ctx, LSMPS_INDEX_OVERFLOW, "fluid count exceeds 32 bits");
  if (!f.x || !f.y || !f.z || !f.vx || !f.vy || !f.vz || !f.pressure || !f.surface_type)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "reordering needs every fluid array");
  const index_t n = static_cast<index_t>(f.count);
  Scratch scratch(ctx);
  if (!scratch.reserve(static_cast<size_t>(n) * (sizeof(double) + sizeof(index_t)) + 1024))
    return fail(ctx, LSMPS_CUDA_ERROR, "scratch allocation failed");
  double* tmp = scratch.take<double>(n);
  index_t* order = scratch.take<index_t>(n);
  if (!tmp || !order) return fail(ctx, LSMPS_CUDA_ERROR, "scratch exhausted");
  // The order is copied first: the cell list may be rebuilt by the caller
  // (and permutation may alias nothing of the fluid).
  if (cudaMemcpyAsync(order, cells.sorted_indices, static_cast<size_t>(n) * sizeof(index_t), cudaMemcpyDeviceToDevice,
                      ctx->stream) != cudaSuccess)
    return check_launch(ctx, "reorder");
  const dim3 grid(static_cast<unsigned>(std::min<long long>(div_up(static_cast<long long>(n), kThreads),
                                                            4LL * ctx->sm_count)));
  for (double* a : {f.x, f.y, f.z, f.vx, f.vy, f.vz, f.pressure}) {
    launch(ctx, gather_kernel<double>, grid, dim3(kThreads), 0, static_cast<const double*>(a),
           static_cast<const index_t*>(order), n, tmp);
    launch(ctx, copy_back_kernel<double>, grid, dim3(kThreads), 0, static_cast<const double*>(tmp), n, a);
  }
  int32_t* itmp = reinterpret_cast<int32_t*>(tmp);
  launch(ctx, gather_kernel<int32_t>, grid, dim3(kThreads), 0, static_cast<const int32_t*>(f.surface_type),
         static_cast<const index_t*>(order), n, itmp);
  launch(ctx, copy_back_kernel<int32_t>, grid, dim3(kThreads), 0, static_cast<const int32_t*>(itmp), n,
         f.surface_type);
  if (permutation &&
      cudaMemcpyAsync(permutation, order, static_cast<size_t>(n) * sizeof(index_t), cudaMemcpyDeviceToDevice,
                      ctx->stream) != cudaSuccess)
    return check_launch(ctx, "reorder");
  return check_launch(ctx, "reorder");
}

}  // namespace lsmps

using namespace lsmps;

extern "C" lsmps_status lsmps_reorder_fluid(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_cells* fluid_cells,
                                            int32_t* permutation) {
  if (!ctx || !fluid || !fluid_cells) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  st = reorder_fluid_impl(ctx, *fluid, *fluid_cells, permutation);
  return end_call(ctx, st);
}
