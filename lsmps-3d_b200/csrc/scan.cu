// scan.cu - device-wide exclusive scan of int32 counts (reduce-then-scan,
// three launches, no inter-block waiting).  Sums are carried in 64 bits so an
// overflow of the 32-bit index type is detected instead of wrapping.
#include <climits>

#include "common.cuh"

namespace lsmps {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const index_t* __restrict__ in, size_t n,
                                                                   long long* __restrict__ partials) {
  const size_t base = static_cast<size_t>(blockIdx.x) * kScanTile;
  long long sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const size_t i = base + static_cast<size_t>(k) * kScanThreads + threadIdx.x;
    if (i < n) sum += in[i];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  __shared__ long long warp_sum[kScanThreads / kWarp];
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
#pragma unroll
    for (int w = 0; w < kScanThreads / kWarp; ++w) t += warp_sum[w];
    partials[blockIdx.x] = t;
  }
}

// One block: exclusive scan of the per-tile sums in chunks of blockDim.
__global__ void __launch_bounds__(1024) scan_partials_kernel(long long* __restrict__ partials, int count,
                                                             unsigned long long* __restrict__ total,
                                                             index_t* __restrict__ total_i32,
                                                             DeviceStatus* __restrict__ status) {
  __shared__ long long warp_sum[32];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int base = 0; base < count; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const long long v = i < count ? partials[i] : 0;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      long long s = lane < nwarp ? warp_sum[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      if (lane < nwarp) warp_sum[lane] = s;
    }
    __syncthreads();
    const long long before = carry + (warp > 0 ? warp_sum[warp - 1] : 0) + x - v;
    if (i < count) partials[i] = before;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = before + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (total) *total = static_cast<unsigned long long>(carry);
    if (total_i32) {
      if (carry > INT_MAX) {
        raise_flag(status, kFlagIndexOverflow);
        *total_i32 = INT_MAX;
      } else {
        *total_i32 = static_cast<index_t>(carry);
      }
    }
  }
}

__global__ void __launch_bounds__(kScanThreads) scan_down_kernel(const index_t* in, index_t* out, size_t n,
                                                                 const long long* __restrict__ partials,
                                                                 DeviceStatus* __restrict__ status) {
  const size_t base = static_cast<size_t>(blockIdx.x) * kScanTile + static_cast<size_t>(threadIdx.x) * kScanItems;
  long long v[kScanItems];
  long long local = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const size_t i = base + k;
    v[k] = i < n ? in[i] : 0;
    local += v[k];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  long long x = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  __shared__ long long warp_sum[kScanThreads / kWarp];
  if (lane == 31) warp_sum[warp] = x;
  __syncthreads();
  long long before = partials[blockIdx.x] + x - local;
  for (int w = 0; w < warp; ++w) before += warp_sum[w];
  bool overflow = false;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const size_t i = base + k;
    if (i < n) {
      overflow |= before > INT_MAX;
      out[i] = static_cast<index_t>(before > INT_MAX ? INT_MAX : before);
    }
    before += v[k];
  }
  if (overflow) raise_flag(status, kFlagIndexOverflow);
}

}  // namespace

size_t scan_scratch_bytes(size_t n) {
  const size_t tiles = (n + kScanTile - 1) / kScanTile + 1;
  return tiles * sizeof(long long) + 512;
}

lsmps_status exclusive_scan_i32(lsmps_ctx* ctx, Scratch& scratch, const index_t* in, index_t* out, size_t n,
                                unsigned long long* total, index_t* total_i32) {
  const int tiles = n ? div_up(static_cast<long long>(n), kScanTile) : 0;
  long long* partials = scratch.take<long long>(tiles + 1);
  if (!partials) return fail(ctx, LSMPS_CUDA_ERROR, "scan scratch exhausted");
  if (tiles) launch(ctx, scan_reduce_kernel, dim3(tiles), dim3(kScanThreads), 0, in, n, partials);
  launch(ctx, scan_partials_kernel, dim3(1), dim3(1024), 0, partials, tiles, total, total_i32, ctx->d_status);
  if (tiles) launch(ctx, scan_down_kernel, dim3(tiles), dim3(kScanThreads), 0, in, out, n,
                    static_cast<const long long*>(partials), ctx->d_status);
  return check_launch(ctx, "exclusive scan");
}

}  // namespace lsmps
