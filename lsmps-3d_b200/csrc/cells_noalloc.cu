// cells_noalloc.cu - lsmps_build_cell_list_noalloc: the cell-list build of
// cells.cu (same kernels, same results) with its scratch in one fixed
// file-scope device array instead of context memory.
//
// Why it exists: lsmps_build_cell_list takes its ping-pong key/value arrays
// and histogram table from the context scratch, which grows with cudaMalloc
// (and frees the old block with cudaFree) the first time a call needs more.
// Some callers cannot allow that inside their loop: a host process whose
// device memory is handed out entirely by its own pool allocator (cudaMalloc
// then fails or fragments the pool), or a loop that must not take the
// implicit device-wide synchronisation of cudaFree.  For them this entry
// point needs no context and allocates nothing, for up to
// LSMPS_NOALLOC_MAX_PARTICLES particles.
//
// Scratch layout (g_scratch, 256-byte aligned):
//   [0, 256)                          DeviceStatus word
//   [256, 256 + 4 M)                  ping-pong cell ids      (M = max particles)
//   [256 + 4 M, 256 + 8 M)            ping-pong particle ids
//   [256 + 8 M, + 4 * tiles * 256)    digit-major histogram table
// Nothing in it has to start at zero: every call clears the status word
// itself and the sort writes keys, values and histograms before reading them.
#include <algorithm>
#include <climits>
#include <mutex>
#include <utility>

#include "cells.cuh"

namespace lsmps {
namespace {

constexpr size_t kMaxParticles = LSMPS_NOALLOC_MAX_PARTICLES;
constexpr int kMaxTiles = static_cast<int>((kMaxParticles + kSortTile - 1) / kSortTile);
constexpr size_t kHistEntries = static_cast<size_t>(kMaxTiles) * kRadixBins;
constexpr size_t kStatusBytes = 256;
constexpr size_t kKeysOffset = kStatusBytes;
constexpr size_t kValsOffset = kKeysOffset + kMaxParticles * sizeof(index_t);
constexpr size_t kHistOffset = kValsOffset + kMaxParticles * sizeof(index_t);
constexpr size_t kScratchBytes = kHistOffset + kHistEntries * sizeof(index_t);
static_assert(sizeof(DeviceStatus) <= kStatusBytes, "status word does not fit its slot");
static_assert(kValsOffset % 256 == 0 && kHistOffset % 256 == 0, "scratch slots must stay 256-byte aligned");

// About 4.1 MiB per device for 524,288 particles.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kScanThreads = 1024;

// Exclusive scan of the histogram table in one block: each thread owns a
// contiguous run of entries (at most kHistEntries / kScanThreads = 32).
__global__ void __launch_bounds__(kScanThreads) hist_scan_kernel(index_t* __restrict__ hist, int entries) {
  __shared__ index_t warp_total[kScanThreads / kWarp];
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x >> 5;
  const int per = (entries + kScanThreads - 1) / kScanThreads;
  const int begin = min(static_cast<int>(threadIdx.x) * per, entries);
  const int end = min(begin + per, entries);
  index_t own = 0;
  for (int k = begin; k < end; ++k) own += hist[k];
  index_t incl = own;
#pragma unroll
  for (int d = 1; d < kWarp; d <<= 1) {
    const index_t t = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += t;
  }
  if (lane == kWarp - 1) warp_total[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    index_t w = warp_total[lane];
#pragma unroll
    for (int d = 1; d < kWarp; d <<= 1) {
      const index_t t = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= d) w += t;
    }
    warp_total[lane] = w;
  }
  __syncthreads();
  index_t run = incl - own + (warp ? warp_total[warp - 1] : 0);
  for (int k = begin; k < end; ++k) {
    const index_t c = hist[k];
    hist[k] = run;
    run += c;
  }
}

// Per-device set-up, done once under the device's lock: the address of
// g_scratch on that device and the SM count for the grid sizes.  Each .cu
// file of the library is its own device module, and under lazy module loading
// (the CUDA runtime's default) a module is loaded on first use, which can
// allocate device memory.  Looking up g_scratch loads this file's module;
// querying the attributes of the sort kernels compiled in cells.cu loads
// that module too, so that no later call (count = 0 included) loads code.
constexpr int kMaxDevices = 64;
struct DeviceSlot {
  std::mutex lock;
  unsigned char* scratch = nullptr;
  int sm_count = 0;
};
DeviceSlot g_devices[kMaxDevices];

lsmps_status set_up(DeviceSlot& slot, int device) {
  if (slot.scratch) return LSMPS_OK;
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) return LSMPS_CUDA_ERROR;
  const void* kernels[] = {reinterpret_cast<const void*>(hash_kernel),
                           reinterpret_cast<const void*>(radix_hist_kernel),
                           reinterpret_cast<const void*>(radix_scatter_kernel),
                           reinterpret_cast<const void*>(ranges_kernel),
                           reinterpret_cast<const void*>(hist_scan_kernel)};
  for (const void* k : kernels) {
    cudaFuncAttributes attr;
    if (cudaFuncGetAttributes(&attr, k) != cudaSuccess) return LSMPS_CUDA_ERROR;
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0)
    return LSMPS_CUDA_ERROR;
  slot.sm_count = sms;
  slot.scratch = static_cast<unsigned char*>(p);
  return LSMPS_OK;
}

}  // namespace
}  // namespace lsmps

using namespace lsmps;

extern "C" lsmps_status lsmps_build_cell_list_noalloc(void* stream_handle, const double* x, const double* y,
                                                      const double* z, size_t count, const lsmps_grid* grid,
                                                      const lsmps_cells* cells) {
  if (!grid || !cells) return LSMPS_INVALID_ARGUMENT;
  if (!(grid->cell_size > 0.0) || grid->dims[0] <= 0 || grid->dims[1] <= 0 || grid->dims[2] <= 0)
    return LSMPS_INVALID_ARGUMENT;
  const long long ncell = static_cast<long long>(grid->dims[0]) * grid->dims[1] * grid->dims[2];
  if (ncell > INT_MAX) return LSMPS_INDEX_OVERFLOW;
  // The one size limit of the fixed scratch; checked before any device work.
  if (count > kMaxParticles) return LSMPS_CAPACITY_EXCEEDED;
  if (static_cast<size_t>(ncell) != cells->cell_count || count > cells->particle_count)
    return LSMPS_INVALID_ARGUMENT;
  if (!cells->cell_begin || !cells->cell_end ||
      (count && (!cells->cell_ids || !cells->sorted_indices || !x || !y || !z)))
    return LSMPS_INVALID_ARGUMENT;

  // An error left pending by earlier work of the caller is not this call's:
  // report it without clearing it and without queuing anything.
  if (cudaPeekAtLastError() != cudaSuccess) return LSMPS_CUDA_ERROR;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return LSMPS_CUDA_ERROR;
  if (device < 0 || device >= kMaxDevices) return LSMPS_INVALID_ARGUMENT;
  DeviceSlot& slot = g_devices[device];
  // One scratch per device: a second call on this device waits here until
  // the first one's kernels have finished (each call synchronises its stream
  // before it unlocks), since two sorts in flight on one scratch would race.
  std::lock_guard<std::mutex> guard(slot.lock);
  lsmps_status st = set_up(slot, device);
  if (st) return st;

  cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
  DeviceStatus* status = reinterpret_cast<DeviceStatus*>(slot.scratch);
  index_t* alt_keys = reinterpret_cast<index_t*>(slot.scratch + kKeysOffset);
  index_t* alt_vals = reinterpret_cast<index_t*>(slot.scratch + kValsOffset);
  index_t* hist = reinterpret_cast<index_t*>(slot.scratch + kHistOffset);
  if (cudaMemsetAsync(status, 0, sizeof(DeviceStatus), stream) != cudaSuccess) return LSMPS_CUDA_ERROR;

  const index_t n = static_cast<index_t>(count);
  const int passes = (key_bits(ncell) + kRadixBits - 1) / kRadixBits;
  const int tiles = n ? div_up(n, kSortTile) : 0;
  // Ping-pong so that the last pass lands in the caller's arrays.
  index_t* k0 = (passes & 1) ? alt_keys : cells->cell_ids;
  index_t* v0 = (passes & 1) ? alt_vals : cells->sorted_indices;
  index_t* k1 = (passes & 1) ? cells->cell_ids : alt_keys;
  index_t* v1 = (passes & 1) ? cells->sorted_indices : alt_vals;
  const long long work = n > ncell ? n : ncell;
  const int hash_blocks = static_cast<int>(std::min<long long>(div_up(work, 256), slot.sm_count * 8LL));
  hash_kernel<<<hash_blocks, 256, 0, stream>>>(x, y, z, n, *grid, k0, v0, cells->cell_begin, cells->cell_end,
                                               static_cast<index_t>(ncell), status);
  if (n > 0) {
    for (int p = 0; p < passes; ++p) {
      const int shift = p * kRadixBits;
      radix_hist_kernel<<<tiles, kSortThreads, 0, stream>>>(k0, n, shift, hist, tiles);
      hist_scan_kernel<<<1, kScanThreads, 0, stream>>>(hist, tiles * kRadixBins);
      radix_scatter_kernel<<<tiles, kSortThreads, 0, stream>>>(k0, v0, k1, v1, n, shift, hist, tiles);
      std::swap(k0, k1);
      std::swap(v0, v1);
    }
    const int range_blocks = static_cast<int>(std::min<long long>(div_up(n, 256), slot.sm_count * 8LL));
    ranges_kernel<<<range_blocks, 256, 0, stream>>>(cells->cell_ids, n, cells->cell_begin, cells->cell_end);
  }
  DeviceStatus h{};
  bool failed = cudaGetLastError() != cudaSuccess;
  if (!failed)
    failed = cudaMemcpyAsync(&h, status, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, stream) != cudaSuccess;
  // Always wait for what was queued before the lock is released: the next
  // call on this device reuses the same scratch.
  if (cudaStreamSynchronize(stream) != cudaSuccess || failed) return LSMPS_CUDA_ERROR;
  if (h.flags & kFlagNonFinite) return LSMPS_NON_FINITE;
  return LSMPS_OK;
}
