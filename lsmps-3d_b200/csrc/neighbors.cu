// neighbors.cu - fluid-fluid and fluid-wall CSR neighbour tables.
// Replaces build_neighbor_lists / build_one_neighbor_list of
// src/neighbor/neighbor_search.cu:294-367 (count kernel :221-236, Thrust
// exclusive scan :319-320, host capacity check :323-328, write kernel
// :238-253).
//
// Layout of the work.  A home cell's candidates are the particles of the 27
// surrounding source cells in the reference's dz -> dy -> dx order, ascending
// sorted position inside a cell (its "sequence").  The count pass gives each
// home cell one warp and each home particle one lane: the warp stages the
// sequence in shared memory as cell-relative FP32 coordinates and every lane
// tests its particle against all of it through broadcast loads, keeping one
// 32-bit accept mask per 32 candidates.  After the scan of the counts, the
// write pass gives each home cell a block, stages the candidate indices and
// replays the masks, one warp per particle, compacting each 32-candidate
// chunk with a popcount: rows come out in exactly the reference's traversal
// order and the distance tests run once per table.
//
// Exactness: the FP32 distance is only a screen.  With coordinates scaled by
// 1/h and re-centred on the home cell, every component is at most 2 in
// magnitude for particles inside the grid, and the FP32 value of
// e = d^2 - lo2 (lo2 = (r/h)^2 - kScreenMargin, formed by three fused
// multiply-adds on the FP32 differences) is within a few hundred 2^-24 of the
// exact one, far inside kScreenMargin = 1e-4.  A candidate is accepted from
// FP32 when e < 0 and rejected when e >= 2 kScreenMargin; everything between,
// and every particle outside the +-2 window (clamped into an edge cell), is
// decided by the reference's own FP64 test dx*dx + dy*dy + dz*dz <= r^2
// (neighbor_search.cu:48-59).  The neighbour sets are therefore the FP64 ones.
#include <algorithm>
#include <climits>
#include <cmath>

#include "f32x2.cuh"
#include "impl.cuh"
#include "packed.cuh"

namespace lsmps {
namespace {

constexpr int kCsrThreads = 128;
constexpr int kCsrWarps = kCsrThreads / kWarp;
constexpr int kStageCap = 1024;
constexpr float kScreenMargin = 1.0e-4f;
constexpr float kFarLimit = 2.0f;
constexpr int kMaskWords = kStageCap / 32;
constexpr int kCountWarps = 2;               // warps (home cells) per block of the count pass
constexpr float kSentinel = 1.0e18f;         // far enough that d^2 stays finite and rejected
constexpr int kStageBatch = 8;               // candidate loads in flight per lane while staging

struct CsrArgs {
  const double* fx;
  const double* fy;
  const double* fz;
  const double* sx;
  const double* sy;
  const double* sz;
  const index_t* home_begin;
  const index_t* home_end;
  const index_t* home_sorted;
  const index_t* src_begin;
  const index_t* src_end;
  const index_t* src_sorted;
  lsmps_grid grid;
  double r2;
  double inv_h;
  float lo2;   // (r/h)^2 - kScreenMargin
  float band;  // a little over 2 kScreenMargin: FP32 rejects only e >= band
  index_t ncell;
  int exclude_self;
  index_t* offsets;  // count pass: per-particle counts; write pass: row offsets
  index_t* indices;
  // write pass, or NULL: each entry's sorted position (the position of the
  // neighbour in the source cell list) beside its index
  index_t* spos;
  unsigned long long capacity;
  const index_t* total;  // write pass: offsets[N]
  // Per home particle, one 32-bit accept mask per 32 staged candidates
  // (bits[i * kMaskWords + chunk]); written by the count pass, replayed by the
  // write pass.
  unsigned* bits;
  // Source positions in cell-sorted order (src_pos[k] = position of
  // src_sorted[k]), so that staging a cell reads one contiguous range.
  const double4* src_pos;
  DeviceStatus* status;
  // merged batch (batch.cu): every box's cells and grid, or NULL for one box
  // on a.grid; the cell size (a.grid.cell_size) is shared by all boxes
  const BoxGrid* boxes;
  int nbox;
};

// A home cell's place in its grid: its coordinates, the grid's dims and
// origin, and the box's first global cell (0 for one box).
struct CellFrame {
  int dims[3];
  int cx, cy, cz;
  index_t base;
  double origin[3];
};

__device__ __forceinline__ CellFrame frame_of(const CsrArgs& a, index_t c) {
  CellFrame f;
  if (a.boxes) {
    const BoxGrid& g = a.boxes[box_of(a.boxes, a.nbox, c, 0)];
    f.base = g.cell_base;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      f.dims[k] = g.dims[k];
      f.origin[k] = g.origin[k];
    }
  } else {
    f.base = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      f.dims[k] = a.grid.dims[k];
      f.origin[k] = a.grid.origin[k];
    }
  }
  const index_t lc = c - f.base;
  f.cx = lc % f.dims[0];
  f.cy = (lc / f.dims[0]) % f.dims[1];
  f.cz = lc / (f.dims[0] * f.dims[1]);
  return f;
}

// src_pos[k] = {x, y, z, 0} of particle sorted[k].
__global__ void sorted_positions_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                        const double* __restrict__ z, const index_t* __restrict__ sorted, index_t n,
                                        double4* __restrict__ out) {
  for (index_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const index_t j = sorted[k];
    out[k] = make_double4(x[j], y[j], z[j], 0.0);
  }
}

__device__ __forceinline__ bool within_radius(double ax, double ay, double az, double bx, double by, double bz,
                                              double r2) {
  const double dx = ax - bx;
  const double dy = ay - by;
  const double dz = az - bz;
  return dx * dx + dy * dy + dz * dz <= r2;
}

__device__ __forceinline__ float to_rel(double v, double centre, double inv_h) {
  const float r = static_cast<float>((v - centre) * inv_h);
  return fabsf(r) <= kFarLimit ? r : __int_as_float(0x7fc00000);  // NaN forces the exact test
}

// (acc << 1) | sign bit of the FP32 value in v's low (kHigh: high) half.
template <bool kHigh>
__device__ __forceinline__ unsigned shift_in_sign(unsigned acc, unsigned long long v) {
  return __funnelshift_l(static_cast<unsigned>(kHigh ? v >> 32 : v), acc, 1);
}

__device__ __forceinline__ index_t warp_sum(index_t v) {
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}

// Count pass: one warp per home cell, one lane per home particle.  The warp
// stages its 27-cell candidate sequence (cell-relative FP32 coordinates and
// the candidate's cell-sorted position) in shared memory, padded to whole
// 32-candidate chunks with far sentinels and laid out by candidate pairs
// ({x0, x1, y0, y1} and {z0, z1}: 12 bytes per candidate, so that more warps
// fit an SM; the rare FP64 test finds a candidate's sorted position from the
// cell starts), so that every lane walks the
// sequence with broadcast loads and tests two candidates per packed FP32
// instruction; the sign of e = d^2 - lo2 is shifted straight into the mask.
// Bit b of chunk c of a lane's mask is the candidate at sequence position
// 32c + b, the numbering the write pass replays.  In the fluid table the
// home cell is the centre source cell, so a particle's own bit sits at
// sequence position (start of the centre cell) + (its sorted position in the
// home cell) and is cleared after the tests (the reference skips j == i).
__global__ void __launch_bounds__(kCountWarps * kWarp) csr_count_kernel(CsrArgs a) {
  __shared__ float4 s_xy[kCountWarps][kStageCap / 2];  // pair p: {x_2p, x_2p+1, y_2p, y_2p+1}
  __shared__ float2 s_z[kCountWarps][kStageCap / 2];   // pair p: {z_2p, z_2p+1}
  __shared__ unsigned s_far[kCountWarps][kMaskWords];  // per chunk: candidates outside the window
  __shared__ index_t s_cb[kCountWarps][27];
  __shared__ index_t s_pre[kCountWarps][28];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  float4* sxy = s_xy[w];
  float2* sz = s_z[w];
  unsigned* far = s_far[w];
  index_t* cb = s_cb[w];
  index_t* pre = s_pre[w];
  for (index_t c = blockIdx.x * kCountWarps + w; c < a.ncell; c += gridDim.x * kCountWarps) {
    const index_t hb = a.home_begin[c];
    if (hb < 0) continue;  // uniform across the warp
    const index_t he = a.home_end[c];
    const CellFrame fr = frame_of(a, c);
    const int dimx = fr.dims[0], dimy = fr.dims[1], dimz = fr.dims[2];
    const int cx = fr.cx, cy = fr.cy, cz = fr.cz;
    index_t b = -1, n = 0;
    if (lane < 27) {
      const int nz = cz + lane / 9 - 1, ny = cy + (lane / 3) % 3 - 1, nx = cx + lane % 3 - 1;
      if (nz >= 0 && nz < dimz && ny >= 0 && ny < dimy && nx >= 0 && nx < dimx) {
        const index_t cell = fr.base + (nz * dimy + ny) * dimx + nx;
        b = a.src_begin[cell];
        const index_t e = a.src_end[cell];
        if (b >= 0 && e >= 0) n = e - b;
      }
    }
    index_t incl = n;
#pragma unroll
    for (int d = 1; d < kWarp; d <<= 1) {
      const index_t t = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += t;
    }
    const index_t nc = __shfl_sync(0xffffffffu, incl, 31);
    if (lane < 27) {
      cb[lane] = b;
      pre[lane] = incl - n;
    }
    if (lane == 0) pre[27] = nc;
    __syncwarp();
    if (nc == 0) {
      // no candidates (most home cells of the wall table): empty rows
      for (index_t h = hb + lane; h < he; h += kWarp) a.offsets[a.home_sorted[h]] = 0;
      continue;
    }
    if (nc > kStageCap) {
      // More candidates than the stage holds (overloaded edge cells): exact
      // tests straight from global memory; only the count is needed here.
      for (index_t h = hb; h < he; ++h) {
        const index_t i = a.home_sorted[h];
        const double xi = a.fx[i], yi = a.fy[i], zi = a.fz[i];
        index_t count = 0;
        for (int t = 0; t < 27; ++t) {
          const index_t b0 = cb[t], cnt = pre[t + 1] - pre[t];
          for (index_t k = lane; k < cnt; k += kWarp) {
            const index_t j = a.src_sorted[b0 + k];
            if (!(a.exclude_self && j == i) && within_radius(xi, yi, zi, a.sx[j], a.sy[j], a.sz[j], a.r2)) ++count;
          }
        }
        count = warp_sum(count);
        if (lane == 0) a.offsets[i] = count;
      }
      __syncwarp();
      continue;
    }
    const double ccx = fr.origin[0] + (cx + 0.5) * a.grid.cell_size;
    const double ccy = fr.origin[1] + (cy + 0.5) * a.grid.cell_size;
    const double ccz = fr.origin[2] + (cz + 0.5) * a.grid.cell_size;
    const int chunks = static_cast<int>((nc + kWarp - 1) / kWarp);
    {
      // kStageBatch loads in flight per lane: the staging is a chain of L2
      // round trips otherwise
      int t = 0;  // each lane's source cell only moves forward
      for (index_t k0 = lane; k0 < chunks * kWarp; k0 += kStageBatch * kWarp) {
        index_t pos[kStageBatch];
        double4 q[kStageBatch];
#pragma unroll
        for (int u = 0; u < kStageBatch; ++u) {
          const index_t k = k0 + u * kWarp;
          pos[u] = -1;
          if (k < nc) {
            while (pre[t + 1] <= k) ++t;
            pos[u] = cb[t] + (k - pre[t]);
          }
        }
#pragma unroll
        for (int u = 0; u < kStageBatch; ++u)
          if (pos[u] >= 0) q[u] = ld4(a.src_pos, pos[u]);
#pragma unroll
        for (int u = 0; u < kStageBatch; ++u) {
          const index_t k = k0 + u * kWarp;
          if (k >= chunks * kWarp) break;  // uniform: the lanes of one u share a chunk
          float x = kSentinel, y = kSentinel, z = kSentinel;
          if (pos[u] >= 0) {
            x = to_rel(q[u].x, ccx, a.inv_h);
            y = to_rel(q[u].y, ccy, a.inv_h);
            z = to_rel(q[u].z, ccz, a.inv_h);
          }
          float* xy = reinterpret_cast<float*>(sxy + (k >> 1)) + (k & 1);
          xy[0] = x;
          xy[2] = y;
          reinterpret_cast<float*>(sz + (k >> 1))[k & 1] = z;
          const unsigned outside = __ballot_sync(0xffffffffu, isnan(x) || isnan(y) || isnan(z));
          if (lane == 0) far[k >> 5] = outside;
        }
      }
    }
    __syncwarp();
    const index_t self_base = pre[13];
    for (index_t h0 = hb; h0 < he; h0 += kWarp) {
      const index_t h = h0 + lane;
      const bool live = h < he;
      index_t i = 0;
      double xi = 0.0, yi = 0.0, zi = 0.0;
      // idle lanes sit far from every candidate and from the sentinels
      float rx = -kSentinel, ry = -kSentinel, rz = -kSentinel;
      int self_chunk = -1;
      unsigned self_bit = 0u;
      bool home_far = false;
      if (live) {
        i = a.home_sorted[h];
        xi = a.fx[i];
        yi = a.fy[i];
        zi = a.fz[i];
        rx = to_rel(xi, ccx, a.inv_h);
        ry = to_rel(yi, ccy, a.inv_h);
        rz = to_rel(zi, ccz, a.inv_h);
        home_far = isnan(rx) || isnan(ry) || isnan(rz);
        if (a.exclude_self) {
          const index_t k = self_base + (h - hb);
          self_chunk = static_cast<int>(k >> 5);
          self_bit = 1u << (k & 31);
        }
      }
      const unsigned long long rxx = pack2(rx, rx), ryy = pack2(ry, ry), rzz = pack2(rz, rz);
      const unsigned long long nlo = pack2(-a.lo2, -a.lo2), band = pack2(a.band, a.band);
      index_t count = 0;
      for (int ch = 0; ch < chunks; ++ch) {
        const ulonglong2* qxy = reinterpret_cast<const ulonglong2*>(sxy + ch * (kWarp / 2));
        const unsigned long long* qz = reinterpret_cast<const unsigned long long*>(sz + ch * (kWarp / 2));
        // bit 31 - b: candidate b accepted from FP32 (e < 0) / not rejected (e < band)
        unsigned lo = 0u, near = 0u;
#pragma unroll
        for (int pr = 0; pr < kWarp / 2; ++pr) {
          const ulonglong2 xy = qxy[pr];
          const unsigned long long dx = sub2(rxx, xy.x), dy = sub2(ryy, xy.y), dz = sub2(rzz, qz[pr]);
          unsigned long long e = fma2(dx, dx, nlo);
          e = fma2(dy, dy, e);
          e = fma2(dz, dz, e);
          const unsigned long long f = sub2(e, band);
          lo = shift_in_sign<true>(shift_in_sign<false>(lo, e), e);
          near = shift_in_sign<true>(shift_in_sign<false>(near, f), f);
        }
        lo = __brev(lo);
        near = __brev(near);
        // between the thresholds, or a coordinate outside the window: FP64
        unsigned amb = (near & ~lo) | far[ch];
        if (home_far) amb = ~0u;
        for (; amb; amb &= amb - 1) {
          const int bit = __ffs(amb) - 1;
          const index_t k = static_cast<index_t>(ch) * kWarp + bit;
          index_t pos = -1;
          if (k < nc) {
            int t = 0;
            while (pre[t + 1] <= k) ++t;
            pos = cb[t] + (k - pre[t]);
          }
          bool in = false;
          if (pos >= 0) {
            const double4 sp = ld4(a.src_pos, pos);
            in = within_radius(xi, yi, zi, sp.x, sp.y, sp.z, a.r2);
          }
          lo = in ? (lo | (1u << bit)) : (lo & ~(1u << bit));
        }
        if (ch == self_chunk) lo &= ~self_bit;
        count += __popc(lo);
        // each lane fills its own particle's 128-byte mask line over the
        // chunks; the partial writes merge in L2
        if (live) a.bits[static_cast<size_t>(i) * kMaskWords + ch] = lo;
      }
      if (live) a.offsets[i] = count;
    }
  }
}

// The count pass in the shape the batched graphs use (lsmps_ctx::
// csr_cell_blocks): one block per home cell stages the sequence once as
// cell-relative FP32 coordinates (candidate index in s_idx), and each warp
// tests two home particles per staged 32-candidate chunk, one candidate per
// lane, with ballots into the same accept masks as csr_count_kernel.  The
// same screen (accept below lo2, FP64 test up to lo2 + band or for NaN).
__global__ void __launch_bounds__(kCsrThreads) csr_count_cell_kernel(CsrArgs a) {
  __shared__ float4 s_rel[kStageCap];
  __shared__ index_t s_idx[kStageCap];
  __shared__ index_t s_cb[27];
  __shared__ index_t s_cnt[27];
  __shared__ index_t s_pre[28];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float hi2 = a.lo2 + a.band;
  for (index_t c = blockIdx.x; c < a.ncell; c += gridDim.x) {
    const index_t hb = a.home_begin[c];
    if (hb < 0) continue;  // uniform across the block
    const index_t he = a.home_end[c];
    const CellFrame fr = frame_of(a, c);
    const int dimx = fr.dims[0], dimy = fr.dims[1], dimz = fr.dims[2];
    const int cx = fr.cx, cy = fr.cy, cz = fr.cz;
    if (warp == 0) {  // the 27 source cells and their starts, one warp scan
      index_t b = -1, n = 0;
      if (lane < 27) {
        const int nz = cz + lane / 9 - 1, ny = cy + (lane / 3) % 3 - 1, nx = cx + lane % 3 - 1;
        if (nz >= 0 && nz < dimz && ny >= 0 && ny < dimy && nx >= 0 && nx < dimx) {
          const index_t cell = fr.base + (nz * dimy + ny) * dimx + nx;
          b = a.src_begin[cell];
          const index_t e = a.src_end[cell];
          if (b >= 0 && e >= 0) n = e - b;
        }
      }
      index_t incl = n;
#pragma unroll
      for (int d = 1; d < kWarp; d <<= 1) {
        const index_t t = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += t;
      }
      if (lane < 27) {
        s_cb[lane] = b;
        s_cnt[lane] = n;
        s_pre[lane] = incl - n;
      }
      if (lane == kWarp - 1) s_pre[27] = incl;
    }
    __syncthreads();
    const index_t nc = s_pre[27];
    if (nc == 0) {
      // no candidates: empty rows (every thread has read nc before warp 0
      // moves on to the next cell)
      for (index_t h = hb + threadIdx.x; h < he; h += kCsrThreads) a.offsets[a.home_sorted[h]] = 0;
      __syncthreads();
      continue;
    }
    const double ccx = fr.origin[0] + (cx + 0.5) * a.grid.cell_size;
    const double ccy = fr.origin[1] + (cy + 0.5) * a.grid.cell_size;
    const double ccz = fr.origin[2] + (cz + 0.5) * a.grid.cell_size;
    if (nc <= kStageCap) {
      int t = 0;  // each thread's source cell only moves forward
      for (index_t k = threadIdx.x; k < nc; k += kCsrThreads) {
        while (s_pre[t + 1] <= k) ++t;
        const index_t pos = s_cb[t] + (k - s_pre[t]);
        s_idx[k] = a.src_sorted[pos];
        const double4 q = ld4(a.src_pos, pos);
        s_rel[k] = make_float4(to_rel(q.x, ccx, a.inv_h), to_rel(q.y, ccy, a.inv_h), to_rel(q.z, ccz, a.inv_h), 0.0f);
      }
      __syncthreads();
      for (index_t h = hb + 2 * warp; h < he; h += 2 * kCsrWarps) {
        const bool two = h + 1 < he;
        const index_t i0 = a.home_sorted[h];
        const index_t i1 = two ? a.home_sorted[h + 1] : i0;
        const double x0 = a.fx[i0], y0 = a.fy[i0], z0 = a.fz[i0];
        const double x1 = a.fx[i1], y1 = a.fy[i1], z1 = a.fz[i1];
        const float r0x = to_rel(x0, ccx, a.inv_h), r0y = to_rel(y0, ccy, a.inv_h), r0z = to_rel(z0, ccz, a.inv_h);
        const float r1x = to_rel(x1, ccx, a.inv_h), r1y = to_rel(y1, ccy, a.inv_h), r1z = to_rel(z1, ccz, a.inv_h);
        unsigned keep0 = 0u, keep1 = 0u;  // lane c keeps chunk c's masks
        index_t count0 = 0, count1 = 0;
        for (index_t base = 0; base < nc; base += kWarp) {
          const index_t k = base + lane;
          bool pass0 = false, pass1 = false;
          if (k < nc) {
            const index_t j = s_idx[k];
            const float4 q = s_rel[k];
            if (!(a.exclude_self && j == i0)) {
              const float dx = r0x - q.x, dy = r0y - q.y, dz = r0z - q.z;
              const float d2 = dx * dx + dy * dy + dz * dz;
              if (d2 < a.lo2) {
                pass0 = true;
              } else if (!(d2 > hi2)) {  // near the boundary, or NaN (outside the window)
                pass0 = within_radius(x0, y0, z0, a.sx[j], a.sy[j], a.sz[j], a.r2);
              }
            }
            if (two && !(a.exclude_self && j == i1)) {
              const float dx = r1x - q.x, dy = r1y - q.y, dz = r1z - q.z;
              const float d2 = dx * dx + dy * dy + dz * dz;
              if (d2 < a.lo2) {
                pass1 = true;
              } else if (!(d2 > hi2)) {
                pass1 = within_radius(x1, y1, z1, a.sx[j], a.sy[j], a.sz[j], a.r2);
              }
            }
          }
          const unsigned m0 = __ballot_sync(0xffffffffu, pass0);
          const unsigned m1 = __ballot_sync(0xffffffffu, pass1);
          if (lane == base / kWarp) {
            keep0 = m0;
            keep1 = m1;
          }
          count0 += __popc(m0);
          count1 += __popc(m1);
        }
        const int chunks = static_cast<int>((nc + kWarp - 1) / kWarp);
        if (lane < chunks) {
          a.bits[static_cast<size_t>(i0) * kMaskWords + lane] = keep0;
          if (two) a.bits[static_cast<size_t>(i1) * kMaskWords + lane] = keep1;
        }
        if (lane == 0) {
          a.offsets[i0] = count0;
          if (two) a.offsets[i1] = count1;
        }
      }
    } else {
      // More candidates than the stage holds: exact tests from global memory
      // (count only; the write pass keeps the order).
      for (index_t h = hb + warp; h < he; h += kCsrWarps) {
        const index_t i = a.home_sorted[h];
        const double xi = a.fx[i], yi = a.fy[i], zi = a.fz[i];
        index_t count = 0;
        for (int t = 0; t < 27; ++t) {
          const index_t b0 = s_cb[t], cnt = s_cnt[t];
          for (index_t k = lane; k < cnt; k += kWarp) {
            const index_t j = a.src_sorted[b0 + k];
            if (!(a.exclude_self && j == i) && within_radius(xi, yi, zi, a.sx[j], a.sy[j], a.sz[j], a.r2)) ++count;
          }
        }
        count = warp_sum(count);
        if (lane == 0) a.offsets[i] = count;
      }
    }
    __syncthreads();
  }
}

// Position of the n-th (from 0) set bit of w, n < popc(w): two halving steps
// down to a byte, then a table of the set-bit positions of every byte.
__device__ __forceinline__ int nth_set_bit(unsigned w, int n, const unsigned char* nth) {
  int pos = 0;
  int c = __popc(w & 0xffffu);
  if (n >= c) {
    n -= c;
    w >>= 16;
    pos = 16;
  }
  c = __popc(w & 0xffu);
  if (n >= c) {
    n -= c;
    w >>= 8;
    pos += 8;
  }
  return pos + nth[(w & 0xffu) * 8 + (n & 7)];
}

// Write pass: one block per home cell; the block stages the candidate indices
// of the 27-cell sequence, then each warp takes one home particle and replays
// its accept masks into the row (an exclusive scan of the chunk popcounts
// gives each chunk's base), so rows come out in the reference's order.
__global__ void __launch_bounds__(kCsrThreads) csr_write_kernel(CsrArgs a) {
  __shared__ index_t s_idx[kStageCap];
  __shared__ index_t s_sp[kStageCap];  // the candidates' sorted positions (a.spos only)
  __shared__ index_t s_cb[27];
  __shared__ index_t s_cnt[27];
  __shared__ index_t s_pre[28];
  __shared__ int s_list[kCsrWarps][kWarp];
  __shared__ unsigned char s_nth[256 * 8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lanemask_lt = (1u << lane) - 1u;
  for (int b = threadIdx.x; b < 256; b += kCsrThreads) {
    int k = 0;
    for (int bit = 0; bit < 8; ++bit)
      if ((b >> bit) & 1) s_nth[b * 8 + k++] = static_cast<unsigned char>(bit);
    for (; k < 8; ++k) s_nth[b * 8 + k] = 0;
  }
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x == 0 && static_cast<unsigned long long>(*a.total) > a.capacity)
    record_required(a.status, static_cast<unsigned long long>(*a.total));
  for (index_t c = blockIdx.x; c < a.ncell; c += gridDim.x) {
    const index_t hb = a.home_begin[c];
    if (hb < 0) continue;  // uniform across the block
    const index_t he = a.home_end[c];
    const CellFrame fr = frame_of(a, c);
    const int dimx = fr.dims[0], dimy = fr.dims[1], dimz = fr.dims[2];
    const int cx = fr.cx, cy = fr.cy, cz = fr.cz;
    if (warp == 0) {  // the 27 source cells and their starts, one warp scan
      index_t b = -1, n = 0;
      if (lane < 27) {
        const int nz = cz + lane / 9 - 1, ny = cy + (lane / 3) % 3 - 1, nx = cx + lane % 3 - 1;
        if (nz >= 0 && nz < dimz && ny >= 0 && ny < dimy && nx >= 0 && nx < dimx) {
          const index_t cell = fr.base + (nz * dimy + ny) * dimx + nx;
          b = a.src_begin[cell];
          const index_t e = a.src_end[cell];
          if (b >= 0 && e >= 0) n = e - b;
        }
      }
      index_t incl = n;
#pragma unroll
      for (int d = 1; d < kWarp; d <<= 1) {
        const index_t t = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += t;
      }
      if (lane < 27) {
        s_cb[lane] = b;
        s_cnt[lane] = n;
        s_pre[lane] = incl - n;
      }
      if (lane == kWarp - 1) s_pre[27] = incl;
    }
    __syncthreads();
    const index_t nc = s_pre[27];
    if (nc == 0) {
      // no candidates, so no rows to write (every thread has read nc before
      // warp 0 moves on to the next cell)
      __syncthreads();
      continue;
    }
    const bool staged = nc <= kStageCap;
    if (staged) {
      int t = 0;  // each thread's source cell only moves forward
      for (index_t k = threadIdx.x; k < nc; k += kCsrThreads) {
        while (s_pre[t + 1] <= k) ++t;
        const index_t pos = s_cb[t] + (k - s_pre[t]);
        s_idx[k] = a.src_sorted[pos];
        s_sp[k] = pos;
      }
    }
    __syncthreads();
    for (index_t h = hb + warp; h < he; h += kCsrWarps) {
      const index_t i = a.home_sorted[h];
      index_t out = a.offsets[i];
      if (staged) {
        const int chunks = (nc + kWarp - 1) / kWarp;
        const unsigned word = lane < chunks ? a.bits[static_cast<size_t>(i) * kMaskWords + lane] : 0u;
        const int pc = __popc(word);
        int incl = pc;
#pragma unroll
        for (int d = 1; d < kWarp; d <<= 1) {
          const int t = __shfl_up_sync(0xffffffffu, incl, d);
          if (lane >= d) incl += t;
        }
        const int base_mine = incl - pc;
        const int total = __shfl_sync(0xffffffffu, incl, kWarp - 1);
        // the non-empty chunks in order, so an entry finds its chunk by rank
        const unsigned nonempty = __ballot_sync(0xffffffffu, pc > 0);
        if (pc > 0) s_list[warp][__popc(nonempty & lanemask_lt)] = lane;
        __syncwarp();
        // 32 consecutive row entries per round, one per lane: coalesced stores
        for (int r0 = 0; r0 < total; r0 += kWarp) {
          const bool starts_here = pc > 0 && base_mine >= r0 && base_mine < r0 + kWarp;
          const unsigned starts = __reduce_or_sync(0xffffffffu, starts_here ? 1u << (base_mine - r0) : 0u);
          const int before = __popc(__ballot_sync(0xffffffffu, pc > 0 && base_mine < r0));
          const int e = r0 + lane;
          const int rank = before + __popc(starts & (0xffffffffu >> (kWarp - 1 - lane))) - 1;
          const int ch = s_list[warp][min(max(rank, 0), kWarp - 1)];
          const unsigned m = __shfl_sync(0xffffffffu, word, ch);
          const int cbase = __shfl_sync(0xffffffffu, base_mine, ch);
          if (e < total) {
            const unsigned long long pos = static_cast<unsigned long long>(out) + e;
            const int bit = nth_set_bit(m, e - cbase, s_nth);
            if (pos < a.capacity) {
              a.indices[pos] = s_idx[ch * kWarp + bit];
              if (a.spos) a.spos[pos] = s_sp[ch * kWarp + bit];
            }
          }
        }
        __syncwarp();
        continue;
      }
      // More candidates than the stage holds (overloaded edge cells): exact
      // tests straight from global memory, same order.
      const double xi = a.fx[i], yi = a.fy[i], zi = a.fz[i];
      for (int t = 0; t < 27; ++t) {
        const index_t cnt = s_cnt[t];
        const index_t b = s_cb[t];
        for (index_t base = 0; base < cnt; base += kWarp) {
          const index_t k = base + lane;
          bool pass = false;
          index_t j = 0;
          if (k < cnt) {
            j = a.src_sorted[b + k];
            if (!(a.exclude_self && j == i)) pass = within_radius(xi, yi, zi, a.sx[j], a.sy[j], a.sz[j], a.r2);
          }
          const unsigned m = __ballot_sync(0xffffffffu, pass);
          if (pass) {
            const unsigned long long pos = static_cast<unsigned long long>(out) + __popc(m & lanemask_lt);
            if (pos < a.capacity) {
              a.indices[pos] = j;
              if (a.spos) a.spos[pos] = b + k;
            }
          }
          out += __popc(m);
        }
      }
    }
    __syncthreads();
  }
}

lsmps_status one_neighbor_list(lsmps_ctx* ctx, Scratch& scratch, const lsmps_fluid& fluid, const double* sx,
                               const double* sy, const double* sz, const lsmps_cells& home, const lsmps_cells& src,
                               const lsmps_grid& grid, double radius, bool exclude_self, const lsmps_csr& out,
                               size_t n_src, unsigned* bits, double4* src_pos, index_t* spos) {
  if (fluid.count > out.particle_count || !out.offsets)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Neighbor list particle capacity is smaller than fluid count");
  const size_t n = fluid.count;
  CsrArgs a{};
  a.fx = fluid.x;
  a.fy = fluid.y;
  a.fz = fluid.z;
  a.sx = sx;
  a.sy = sy;
  a.sz = sz;
  a.home_begin = home.cell_begin;
  a.home_end = home.cell_end;
  a.home_sorted = home.sorted_indices;
  a.src_begin = src.cell_begin;
  a.src_end = src.cell_end;
  a.src_sorted = src.sorted_indices;
  a.grid = grid;
  a.r2 = radius * radius;
  a.inv_h = 1.0 / grid.cell_size;
  const double r2n = a.r2 * a.inv_h * a.inv_h;
  a.lo2 = static_cast<float>(r2n) - kScreenMargin;
  a.band = 2.0f * kScreenMargin * 1.001f;
  a.ncell = static_cast<index_t>(static_cast<long long>(grid.dims[0]) * grid.dims[1] * grid.dims[2]);
  a.boxes = ctx->boxes;
  a.nbox = ctx->nbox;
  a.exclude_self = exclude_self ? 1 : 0;
  // the count pass finds a particle's own bit through the home cell's place
  // in the source list, so the self-excluding table must use one cell list
  if (exclude_self && (home.sorted_indices != src.sorted_indices || home.cell_begin != src.cell_begin))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "self-excluding neighbour table needs one cell list");
  a.offsets = out.offsets;
  a.indices = out.indices;
  a.spos = spos;
  a.capacity = out.neighbor_count;
  a.total = out.offsets + n;
  a.bits = bits;
  a.src_pos = src_pos;
  a.status = ctx->d_status;
  // n_src is the source set's particle count (the cell list holds that many
  // sorted entries; its particle_count is only a capacity)
  if (n_src > src.particle_count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Cell list particle capacity is smaller than particle count");
  if (n_src > 0) {
    const int pb = static_cast<int>(std::min<long long>(div_up(static_cast<long long>(n_src), 256),
                                                        static_cast<long long>(ctx->sm_count) * 8));
    launch(ctx, sorted_positions_kernel, dim3(pb), dim3(256), 0, sx, sy, sz,
           static_cast<const index_t*>(src.sorted_indices), static_cast<index_t>(n_src), src_pos);
  }
  const int count_blocks = static_cast<int>(
      std::min<long long>(div_up(static_cast<long long>(a.ncell), kCountWarps), static_cast<long long>(ctx->sm_count) * 20));
  if (n && ctx->csr_cell_blocks)
    launch(ctx, csr_count_cell_kernel,
           dim3(static_cast<int>(std::min<long long>(a.ncell, static_cast<long long>(ctx->sm_count) * 16))),
           dim3(kCsrThreads), 0, a);
  else if (n)
    launch(ctx, csr_count_kernel, dim3(count_blocks), dim3(kCountWarps * kWarp), 0, a);
  lsmps_status st = exclusive_scan_i32(ctx, scratch, out.offsets, out.offsets, n, nullptr, out.offsets + n);
  if (st) return st;
  const int blocks = static_cast<int>(std::min<long long>(a.ncell, static_cast<long long>(ctx->sm_count) * 16));
  if (n) launch(ctx, csr_write_kernel, dim3(blocks), dim3(kCsrThreads), 0, a);
  return check_launch(ctx, "neighbour list");
}

}  // namespace

size_t neighbor_scratch_bytes(size_t n_fluid, size_t n_wall, size_t ncell) {
  const size_t nmax = n_fluid > n_wall ? n_fluid : n_wall;
  return 2 * cell_list_scratch_bytes(nmax, ncell) + 2 * scan_scratch_bytes(n_fluid + 1) +
         n_fluid * kMaskWords * sizeof(unsigned) + nmax * sizeof(double4) + 4096;
}

lsmps_status build_neighbor_lists_impl(lsmps_ctx* ctx, Scratch& scratch, const lsmps_fluid& fluid,
                                       const lsmps_walls& walls, const lsmps_params& p, const lsmps_cells& fc,
                                       const lsmps_cells& wc, const lsmps_csr& fn, const lsmps_csr& wn) {
  const double radius = p.support_radius;
  if (!(radius > 0.0)) return fail(ctx, LSMPS_INVALID_ARGUMENT, "Neighbor search radius must be positive");
  if (radius > p.grid.cell_size)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Neighbor search currently requires radius <= cell_size");
  unsigned* bits = scratch.take<unsigned>(fluid.count * kMaskWords + 1);
  double4* src_pos = scratch.take<double4>(std::max(fluid.count, walls.count) + 1);
  if (!bits || !src_pos) return fail(ctx, LSMPS_CUDA_ERROR, "neighbour scratch exhausted");
  ctx->built_order = nullptr;
  lsmps_status st =
      build_cell_list_impl(ctx, scratch, fluid.x, fluid.y, fluid.z, fluid.count, p.grid, fc, ctx->boxes, 1);
  if (!st) {
    ctx->built_order = fc.sorted_indices;
    ctx->built_order_count = fluid.count;
  }
  if (!st)
    st = build_cell_list_impl(ctx, scratch, walls.x, walls.y, walls.z, walls.count, p.grid, wc, ctx->boxes, 2);
  // The fluid table's cell-sorted rows go to the context's own array, where
  // they stay for the next step's gathers.
  ctx->spos_table = nullptr;
  index_t* spos = nullptr;
  if (ctx->sorted_rows && fluid.count > 0 && ensure_sorted_rows(ctx, fn.neighbor_count, fluid.count))
    spos = ctx->fluid_spos;
  // the two tables run one after the other on the stream and share the masks
  if (!st)
    st = one_neighbor_list(ctx, scratch, fluid, fluid.x, fluid.y, fluid.z, fc, fc, p.grid, radius, true, fn,
                           fluid.count, bits, src_pos, spos);
  if (!st && spos) {
    ctx->spos_table = fn.offsets;
    ctx->spos_order = fc.sorted_indices;
    ctx->spos_count = fluid.count;
  }
  if (!st)
    st = one_neighbor_list(ctx, scratch, fluid, walls.x, walls.y, walls.z, fc, wc, p.grid, radius, false, wn,
                           walls.count, bits, src_pos, nullptr);
  return st;
}

}  // namespace lsmps

using namespace lsmps;

extern "C" lsmps_status lsmps_build_neighbor_lists(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                                   const lsmps_walls* walls, const lsmps_params* params,
                                                   const lsmps_cells* fluid_cells, const lsmps_cells* wall_cells,
                                                   const lsmps_csr* fluid_neighbors,
                                                   const lsmps_csr* wall_neighbors) {
  if (!ctx || !fluid || !walls || !params || !fluid_cells || !wall_cells || !fluid_neighbors || !wall_neighbors)
    return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  Scratch scratch(ctx);
  if (!scratch.reserve(neighbor_scratch_bytes(fluid->count, walls->count, fluid_cells->cell_count)))
    return fail(ctx, LSMPS_CUDA_ERROR, "scratch allocation failed");
  st = build_neighbor_lists_impl(ctx, scratch, *fluid, *walls, *params, *fluid_cells, *wall_cells, *fluid_neighbors,
                                 *wall_neighbors);
  return end_call(ctx, st);
}
