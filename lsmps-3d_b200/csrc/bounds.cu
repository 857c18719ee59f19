// bounds.cu - the table checks of the bounds-checked build (-DLSMPS_BOUNDS_CHECK,
// `python lsmps-3d_b200/build.py --bounds-check` -> liblsmps_b200_checked.so).
//
// The reference indexes its neighbour tables unchecked (neighbor_search.cu,
// and every gather after it).  In the checked build every implementation
// that reads a neighbour table (or the PPE CSR matrix) first validates it on
// the device -- offsets non-decreasing from 0 and within the capacity, every
// index inside the particle set it points into -- and returns
// LSMPS_INVALID_ARGUMENT before any kernel reads the table when it is not
// valid: a bad index becomes a status, never an out-of-bounds access, and
// nothing traps.  Each check waits for the context's stream (the checked
// build is for debugging and cannot be captured into a graph).  In the
// normal build the checks compile to nothing.
#include <algorithm>

#include "impl.cuh"

namespace lsmps {
#ifdef LSMPS_BOUNDS_CHECK
namespace {

__global__ void csr_check_kernel(const index_t* __restrict__ offsets, const index_t* __restrict__ indices, index_t n,
                                 unsigned long long capacity, long long n_src, DeviceStatus* __restrict__ status) {
  for (index_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const index_t b = offsets[i], e = offsets[i + 1];
    if (b < 0 || e < b || static_cast<unsigned long long>(e) > capacity || (i == 0 && b != 0)) {
      raise_flag(status, kFlagBadIndex);
      continue;
    }
    for (index_t o = b; o < e; ++o) {
      const index_t j = indices[o];
      if (j < 0 || j >= n_src) {
        raise_flag(status, kFlagBadIndex);
        break;
      }
    }
  }
}

}  // namespace
#endif

lsmps_status check_table(lsmps_ctx* ctx, const index_t* offsets, const index_t* indices, size_t rows,
                         unsigned long long capacity, size_t n_src, const char* what) {
#ifndef LSMPS_BOUNDS_CHECK
  (void)ctx, (void)offsets, (void)indices, (void)rows, (void)capacity, (void)n_src, (void)what;
  return LSMPS_OK;
#else
  if (rows == 0) return LSMPS_OK;
  if (!offsets || (capacity && !indices)) return fail(ctx, LSMPS_INVALID_ARGUMENT, what);
  if (cudaMemsetAsync(ctx->d_status, 0, sizeof(DeviceStatus), ctx->stream) != cudaSuccess)
    return check_launch(ctx, "bounds check");
  const int blocks = static_cast<int>(std::min<long long>(div_up(static_cast<long long>(rows), 256),
                                                          static_cast<long long>(ctx->sm_count) * 8));
  launch(ctx, csr_check_kernel, dim3(blocks), dim3(256), 0, offsets, indices, static_cast<index_t>(rows), capacity,
         static_cast<long long>(n_src), ctx->d_status);
  DeviceStatus h{};
  if (cudaMemcpyAsync(&h, ctx->d_status, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    return check_launch(ctx, "bounds check");
  if (h.flags & kFlagBadIndex) {
    cudaMemsetAsync(ctx->d_status, 0, sizeof(DeviceStatus), ctx->stream);
    return fail(ctx, LSMPS_INVALID_ARGUMENT, what);
  }
  return LSMPS_OK;
#endif
}

lsmps_status check_neighbor_tables(lsmps_ctx* ctx, size_t n_fluid, size_t n_wall, const lsmps_csr& fn,
                                   const lsmps_csr* wn) {
#ifdef LSMPS_BOUNDS_CHECK
  if (fn.particle_count < n_fluid || (wn && wn->particle_count < n_fluid))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "neighbour table smaller than the fluid");
#endif
  lsmps_status st = check_table(ctx, fn.offsets, fn.indices, n_fluid, fn.neighbor_count, n_fluid,
                                "fluid neighbour table: offset or index out of range");
  if (!st && wn)
    st = check_table(ctx, wn->offsets, wn->indices, n_fluid, wn->neighbor_count, n_wall,
                     "wall neighbour table: offset or index out of range");
  return st;
}

}  // namespace lsmps
