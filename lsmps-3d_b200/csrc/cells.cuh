// cells.cuh - kernels of the cell-list build (cells.cu), shared by the
// context entry point and the allocation-free one (cells_noalloc.cu).
#pragma once

#include "common.cuh"

namespace lsmps {

constexpr int kRadixBits = 8;
constexpr int kRadixBins = 1 << kRadixBits;
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / kWarp;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;

// Cell id and identity value of every particle; resets cell_begin/cell_end
// to -1.  Raises kFlagNonFinite for a NaN or infinite coordinate.
__global__ void hash_kernel(const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, index_t n, lsmps_grid grid,
                            index_t* __restrict__ keys, index_t* __restrict__ vals,
                            index_t* __restrict__ cell_begin, index_t* __restrict__ cell_end, index_t ncell,
                            DeviceStatus* __restrict__ status);

// Per-tile histogram of one 8-bit digit, digit-major: hist[d * tiles + tile].
__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const index_t* __restrict__ keys, index_t n,
                                                                  int shift, index_t* __restrict__ hist,
                                                                  int tiles);

// Stable scatter of one digit given the exclusively scanned histogram table.
__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(
    const index_t* __restrict__ keys_in, const index_t* __restrict__ vals_in, index_t* __restrict__ keys_out,
    index_t* __restrict__ vals_out, index_t n, int shift, const index_t* __restrict__ hist_scanned, int tiles);

// cell_begin / cell_end from the sorted cell ids.
__global__ void ranges_kernel(const index_t* __restrict__ keys, index_t n, index_t* __restrict__ cell_begin,
                              index_t* __restrict__ cell_end);

// Bits needed for cell ids below ncell.
int key_bits(long long ncell);

}  // namespace lsmps
