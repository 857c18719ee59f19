// cells.cu - cell list of one particle set: cell hash, stable LSD radix sort
// of (cell id, particle index), cell ranges.  Replaces build_cell_list_impl of
// src/neighbor/neighbor_search.cu:255-292, whose Thrust sort_by_key is a
// stable radix sort; this sort is stable too, so the particles of a cell keep
// ascending index order and cell_ids / sorted_indices / cell_begin / cell_end
// are identical to the reference's.
//
// The sort is reduce-then-scan per 8-bit digit: a per-tile digit histogram,
// one device-wide exclusive scan of the digit-major histogram table, and a
// scatter that ranks each key stably inside its tile with warp match masks.
// No block waits on another block.
#include <climits>
#include <cmath>

#include "cells.cuh"

namespace lsmps {
namespace {

// clamp_cell_index, neighbor_search.cu:36-46, with the float-to-int
// conversion of an out-of-range or NaN value made explicit.
__device__ __forceinline__ index_t cell_coord(double coordinate, double origin, double cell_size, index_t dim,
                                              bool& bad) {
  const double scaled = (coordinate - origin) / cell_size;
  if (!(scaled == scaled) || isinf(scaled)) {
    bad = true;
    return 0;
  }
  const double f = floor(scaled);
  if (f < 0.0) return 0;
  if (f >= static_cast<double>(dim)) return dim - 1;
  return static_cast<index_t>(f);
}

}  // namespace

// assign_cells_kernel (neighbor_search.cu:61-73) fused with the cell-range
// reset of reset_cell_ranges_kernel (:75-83).
__global__ void hash_kernel(const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, index_t n, lsmps_grid grid,
                            index_t* __restrict__ keys, index_t* __restrict__ vals,
                            index_t* __restrict__ cell_begin, index_t* __restrict__ cell_end, index_t ncell,
                            DeviceStatus* __restrict__ status) {
  const index_t total = n > ncell ? n : ncell;
  for (index_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    if (t < ncell) {
      cell_begin[t] = -1;
      cell_end[t] = -1;
    }
    if (t < n) {
      bool bad = false;
      const index_t ix = cell_coord(x[t], grid.origin[0], grid.cell_size, grid.dims[0], bad);
      const index_t iy = cell_coord(y[t], grid.origin[1], grid.cell_size, grid.dims[1], bad);
      const index_t iz = cell_coord(z[t], grid.origin[2], grid.cell_size, grid.dims[2], bad);
      if (bad) raise_flag(status, kFlagNonFinite);
      keys[t] = (iz * grid.dims[1] + iy) * grid.dims[0] + ix;  // flatten_cell, :32-34
      vals[t] = t;
    }
  }
}

// hash_kernel for a merged batch: particle t belongs to the box whose range
// of this set holds it (field 1: fluid, 2: walls) and is hashed on that box's
// grid (cell size shared), offset by the box's first global cell.
__global__ void hash_boxes_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                  const double* __restrict__ z, index_t n, const BoxGrid* __restrict__ boxes,
                                  int nbox, int field, double cell_size, index_t* __restrict__ keys,
                                  index_t* __restrict__ vals, index_t* __restrict__ cell_begin,
                                  index_t* __restrict__ cell_end, index_t ncell, DeviceStatus* __restrict__ status) {
  const index_t total = n > ncell ? n : ncell;
  for (index_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    if (t < ncell) {
      cell_begin[t] = -1;
      cell_end[t] = -1;
    }
    if (t < n) {
      const BoxGrid& g = boxes[box_of(boxes, nbox, t, field)];
      bool bad = false;
      const index_t ix = cell_coord(x[t], g.origin[0], cell_size, g.dims[0], bad);
      const index_t iy = cell_coord(y[t], g.origin[1], cell_size, g.dims[1], bad);
      const index_t iz = cell_coord(z[t], g.origin[2], cell_size, g.dims[2], bad);
      if (bad) raise_flag(status, kFlagNonFinite);
      keys[t] = g.cell_base + (iz * g.dims[1] + iy) * g.dims[0] + ix;
      vals[t] = t;
    }
  }
}

// Per-tile histogram of one digit, stored digit-major: hist[d * tiles + tile].
__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const index_t* __restrict__ keys, index_t n,
                                                                  int shift, index_t* __restrict__ hist,
                                                                  int tiles) {
  __shared__ unsigned int bins[kRadixBins];
  bins[threadIdx.x] = 0;
  __syncthreads();
  const size_t base = static_cast<size_t>(blockIdx.x) * kSortTile;
#pragma unroll 4
  for (int k = 0; k < kSortItems; ++k) {
    const size_t i = base + static_cast<size_t>(k) * kSortThreads + threadIdx.x;
    if (i < static_cast<size_t>(n)) atomicAdd(&bins[(keys[i] >> shift) & (kRadixBins - 1)], 1u);
  }
  __syncthreads();
  hist[static_cast<size_t>(threadIdx.x) * tiles + blockIdx.x] = static_cast<index_t>(bins[threadIdx.x]);
}

// Stable scatter of one digit.  The tile is walked in rounds of kSortThreads
// consecutive keys; inside a round, keys are ordered by warp then lane, so
// rank = tile base of the digit + keys of that digit in earlier rounds +
// keys in earlier warps of this round + lower lanes of this warp.
__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(
    const index_t* __restrict__ keys_in, const index_t* __restrict__ vals_in, index_t* __restrict__ keys_out,
    index_t* __restrict__ vals_out, index_t n, int shift, const index_t* __restrict__ hist_scanned, int tiles) {
  __shared__ unsigned int base[kRadixBins];
  __shared__ unsigned int warp_count[kSortWarps][kRadixBins];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  base[threadIdx.x] = static_cast<unsigned int>(hist_scanned[static_cast<size_t>(threadIdx.x) * tiles + blockIdx.x]);
  const unsigned lanemask_lt = (1u << lane) - 1u;
  const size_t tile_base = static_cast<size_t>(blockIdx.x) * kSortTile;
  for (int r = 0; r < kSortItems; ++r) {
    // Each warp clears its own counters for this round.
#pragma unroll
    for (int b = lane; b < kRadixBins; b += kWarp) warp_count[warp][b] = 0;
    __syncwarp();
    const size_t i = tile_base + static_cast<size_t>(r) * kSortThreads + threadIdx.x;
    const bool valid = i < static_cast<size_t>(n);
    index_t key = 0, val = 0;
    int digit = kRadixBins;  // invalid lanes form their own group
    if (valid) {
      key = keys_in[i];
      val = vals_in[i];
      digit = (key >> shift) & (kRadixBins - 1);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, digit);
    const unsigned rank_in_warp = __popc(peers & lanemask_lt);
    if (valid && rank_in_warp == 0) warp_count[warp][digit] = __popc(peers);
    __syncthreads();
    {
      // Thread t owns digit t: exclusive prefix over the warps of this round.
      unsigned running = base[threadIdx.x];
#pragma unroll
      for (int w = 0; w < kSortWarps; ++w) {
        const unsigned c = warp_count[w][threadIdx.x];
        warp_count[w][threadIdx.x] = running;
        running += c;
      }
      base[threadIdx.x] = running;
    }
    __syncthreads();
    if (valid) {
      const unsigned pos = warp_count[warp][digit] + rank_in_warp;
      keys_out[pos] = key;
      vals_out[pos] = val;
    }
    __syncthreads();
  }
}

// build_cell_ranges_kernel, neighbor_search.cu:85-98.
__global__ void ranges_kernel(const index_t* __restrict__ keys, index_t n, index_t* __restrict__ cell_begin,
                              index_t* __restrict__ cell_end) {
  for (index_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const index_t c = keys[p];
    if (p == 0 || keys[p - 1] != c) cell_begin[c] = p;
    if (p + 1 == n || keys[p + 1] != c) cell_end[c] = p + 1;
  }
}

int key_bits(long long ncell) {
  int bits = 0;
  while ((1LL << bits) < ncell) ++bits;
  return bits;
}

lsmps_status validate_grid(lsmps_ctx* ctx, const lsmps_grid& grid) {
  if (!(grid.cell_size > 0.0) || grid.dims[0] <= 0 || grid.dims[1] <= 0 || grid.dims[2] <= 0)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Invalid cell grid configuration");
  const long long ncell = static_cast<long long>(grid.dims[0]) * grid.dims[1] * grid.dims[2];
  if (ncell > INT_MAX) return fail(ctx, LSMPS_INDEX_OVERFLOW, "cell count exceeds the 32-bit index range");
  return LSMPS_OK;
}

size_t cell_list_scratch_bytes(size_t n, size_t ncell) {
  (void)ncell;
  const size_t tiles = (n + kSortTile - 1) / kSortTile + 1;
  // ping-pong keys and values, the histogram table, and one scan per pass
  return 2 * (n * sizeof(index_t) + 256) + tiles * kRadixBins * sizeof(index_t) + 256 +
         4 * scan_scratch_bytes(tiles * kRadixBins) + 4096;
}

lsmps_status build_cell_list_impl(lsmps_ctx* ctx, Scratch& scratch, const double* x, const double* y,
                                  const double* z, size_t count, const lsmps_grid& grid,
                                  const lsmps_cells& cells, const BoxGrid* boxes, int box_field) {
  lsmps_status st = validate_grid(ctx, grid);
  if (st) return st;
  const long long ncell = static_cast<long long>(grid.dims[0]) * grid.dims[1] * grid.dims[2];
  if (static_cast<size_t>(ncell) != cells.cell_count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Cell list capacity does not match grid cell count");
  if (count > cells.particle_count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Cell list particle capacity is smaller than particle count");
  if (count > static_cast<size_t>(INT_MAX))
    return fail(ctx, LSMPS_INDEX_OVERFLOW, "Particle count exceeds 32-bit index capacity");
  if (!cells.cell_begin || !cells.cell_end || (count && (!cells.cell_ids || !cells.sorted_indices || !x || !y || !z)))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "cell list buffers missing");
  const index_t n = static_cast<index_t>(count);
  const int passes = (key_bits(ncell) + kRadixBits - 1) / kRadixBits;
  const int tiles = n ? div_up(n, kSortTile) : 0;
  index_t* alt_keys = scratch.take<index_t>(n + 1);
  index_t* alt_vals = scratch.take<index_t>(n + 1);
  index_t* hist = scratch.take<index_t>(static_cast<size_t>(tiles) * kRadixBins + 1);
  if (!alt_keys || !alt_vals || !hist) return fail(ctx, LSMPS_CUDA_ERROR, "cell list scratch exhausted");
  // Ping-pong so that the last pass lands in the caller's arrays.
  index_t* k0 = (passes & 1) ? alt_keys : cells.cell_ids;
  index_t* v0 = (passes & 1) ? alt_vals : cells.sorted_indices;
  index_t* k1 = (passes & 1) ? cells.cell_ids : alt_keys;
  index_t* v1 = (passes & 1) ? cells.sorted_indices : alt_vals;
  const long long work = n > ncell ? n : ncell;
  const int hash_blocks = static_cast<int>(std::min<long long>(div_up(work, 256), ctx->sm_count * 8LL));
  if (boxes)
    launch(ctx, hash_boxes_kernel, dim3(hash_blocks), dim3(256), 0, x, y, z, n, boxes, ctx->nbox, box_field,
           grid.cell_size, k0, v0, cells.cell_begin, cells.cell_end, static_cast<index_t>(ncell), ctx->d_status);
  else
    launch(ctx, hash_kernel, dim3(hash_blocks), dim3(256), 0, x, y, z, n, grid, k0, v0, cells.cell_begin,
           cells.cell_end, static_cast<index_t>(ncell), ctx->d_status);
  if (n == 0) return check_launch(ctx, "cell hash");
  for (int p = 0; p < passes; ++p) {
    const int shift = p * kRadixBits;
    launch(ctx, radix_hist_kernel, dim3(tiles), dim3(kSortThreads), 0, static_cast<const index_t*>(k0), n, shift,
           hist, tiles);
    st = exclusive_scan_i32(ctx, scratch, hist, hist, static_cast<size_t>(tiles) * kRadixBins, nullptr, nullptr);
    if (st) return st;
    launch(ctx, radix_scatter_kernel, dim3(tiles), dim3(kSortThreads), 0, static_cast<const index_t*>(k0),
           static_cast<const index_t*>(v0), k1, v1, n, shift, static_cast<const index_t*>(hist), tiles);
    std::swap(k0, k1);
    std::swap(v0, v1);
  }
  const int range_blocks = static_cast<int>(std::min<long long>(div_up(n, 256), ctx->sm_count * 8LL));
  launch(ctx, ranges_kernel, dim3(range_blocks), dim3(256), 0, static_cast<const index_t*>(cells.cell_ids), n,
         cells.cell_begin, cells.cell_end);
  return check_launch(ctx, "cell list");
}

}  // namespace lsmps

using namespace lsmps;

extern "C" lsmps_status lsmps_build_cell_list(lsmps_ctx* ctx, const double* x, const double* y, const double* z,
                                              size_t count, const lsmps_grid* grid, const lsmps_cells* cells) {
  if (!ctx || !grid || !cells) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  Scratch scratch(ctx);
  if (!scratch.reserve(cell_list_scratch_bytes(count, cells->cell_count)))
    return fail(ctx, LSMPS_CUDA_ERROR, "scratch allocation failed");
  st = build_cell_list_impl(ctx, scratch, x, y, z, count, *grid, *cells);
  return end_call(ctx, st);
}
