// moment.cu - LSMPS moment matrices and their explicit inverses.
// Replaces DeviceMomentMatrix::prepare_matrices / ensure_matrix_internal of
// src/moment_matrix/moment_matrix.cu:398-476 and 615-654: the assembly kernel
// build_matrix_cache_kernel (:254-309) and the cuSOLVER batched potrf +
// potrs-per-identity-column inversion (:430-471).
//
// One thread owns one particle.  The moment sum is kept in registers as the
// 45 (Type-A) or 55 (Type-B) entries of the lower triangle, each accumulated
// as (w * b[r]) * b[c] in CSR row order like add_outer_product (:203-209).
// The kinds that share the Type-A fluid sum (velocity Dirichlet, pressure
// Neumann, fluid-only) are built from one pass over the fluid row: the
// fluid sum is parked in shared memory and each kind adds its own wall term.
// The inverse is computed in registers by the textbook Cholesky
// factorisation (Golub & Van Loan, Alg. 4.2.1), the in-place inverse of the
// triangular factor, and X = L^-T L^-1, then stored column-major and
// symmetric like the reference's inverse_matrices.
#include <cmath>
#include <utility>

#include "f32x2.cuh"
#include "impl.cuh"
#include "packed.cuh"

namespace lsmps {
namespace {

constexpr int kMomentThreads = 64;

__host__ __device__ constexpr int tri(int r, int c) { return r * (r + 1) / 2 + c; }

struct KindOut {
  int boundary;  // 0 none, 1 wall Dirichlet sample, 2 wall pressure Neumann (moment_matrix.cu:22-26)
  double* inverse;
  double* trace;
  double* reg;
  int32_t* info;
  int32_t* count;
};

struct MomentArgs {
  lsmps_fluid fluid;
  lsmps_walls walls;
  const index_t* fo;
  const index_t* fi;
  const index_t* wo;
  const index_t* wi;
  double re;
  double inv_re;
  double lambda;
  double wall_scale;
  KindOut k0;  // first kind (boundary given by the kernel's B0)
  KindOut k1;  // second kind when the kernel's B1 >= 0
  DeviceStatus* status;
};

// Type-A (N = 9) or Type-B (N = 10) monomial basis of basis_vector,
// moment_matrix.cu:152-175.
template <int N>
__device__ __forceinline__ void basis(double dx, double dy, double dz, double inv_re, double b[N]) {
  constexpr int o = N - 9;
  const double sx = dx * inv_re, sy = dy * inv_re, sz = dz * inv_re;
  if (o) b[0] = 1.0;
  b[o + 0] = sx;
  b[o + 1] = sy;
  b[o + 2] = sz;
  b[o + 3] = sx * sx;
  b[o + 4] = sy * sy;
  b[o + 5] = sz * sz;
  b[o + 6] = sx * sy;
  b[o + 7] = sy * sz;
  b[o + 8] = sz * sx;
}

// wall_neumann_vector, moment_matrix.cu:177-201.
template <int N>
__device__ __forceinline__ void neumann(double dx, double dy, double dz, double nx, double ny, double nz,
                                        double inv_re, double q[N]) {
  constexpr int o = N - 9;
  if (o) q[0] = 0.0;
  q[o + 0] = nx;
  q[o + 1] = ny;
  q[o + 2] = nz;
  q[o + 3] = 2.0 * dx * nx * inv_re;
  q[o + 4] = 2.0 * dy * ny * inv_re;
  q[o + 5] = 2.0 * dz * nz * inv_re;
  q[o + 6] = (dy * nx + dx * ny) * inv_re;
  q[o + 7] = (dz * ny + dy * nz) * inv_re;
  q[o + 8] = (dx * nz + dz * nx) * inv_re;
}

template <int N>
__device__ __forceinline__ void add_outer(double (&m)[N * (N + 1) / 2], const double v[N], double w) {
#pragma unroll
  for (int r = 0; r < N; ++r) {
    const double wr = w * v[r];
#pragma unroll
    for (int c = 0; c <= r; ++c) m[tri(r, c)] = fma(wr, v[c], m[tri(r, c)]);
  }
}

// Column J of the lower Cholesky factor, in place.  J is a template argument
// so that every index into the register array is a compile-time constant
// even though sqrt() keeps the compiler from unrolling a loop over columns.
// T is double for the plain form and float for the mixed form's first
// factorisation.
template <int N, int J, typename T>
__device__ __forceinline__ void cholesky_column(T (&a)[N * (N + 1) / 2], int& info) {
  T s = a[tri(J, J)];
#pragma unroll
  for (int k = 0; k < J; ++k) s = fma(-a[tri(J, k)], a[tri(J, k)], s);
  if (!(s > T(0)) && info == 0) info = J + 1;
  const T ljj = sqrt(s);
  a[tri(J, J)] = ljj;
  const T inv = T(1) / ljj;
#pragma unroll
  for (int i = J + 1; i < N; ++i) {
    T t = a[tri(i, J)];
#pragma unroll
    for (int k = 0; k < J; ++k) t = fma(-a[tri(i, k)], a[tri(J, k)], t);
    a[tri(i, J)] = t * inv;
  }
}

template <int N, typename T, int... J>
__device__ __forceinline__ void cholesky_columns(T (&a)[N * (N + 1) / 2], int& info,
                                                 std::integer_sequence<int, J...>) {
  (cholesky_column<N, J>(a, info), ...);
}

// Lower Cholesky in place; returns 0 or the 1-based order of the first
// non-positive pivot (the potrf info convention).
template <int N, typename T>
__device__ __forceinline__ int cholesky(T (&a)[N * (N + 1) / 2]) {
  int info = 0;
  cholesky_columns<N>(a, info, std::make_integer_sequence<int, N>{});
  return info;
}

// In-place inverse of the lower factor: column j, rows j..N-1 in order.
template <int N>
__device__ __forceinline__ void invert_lower(double (&a)[N * (N + 1) / 2]) {
  double dinv[N];
#pragma unroll
  for (int i = 0; i < N; ++i) dinv[i] = 1.0 / a[tri(i, i)];
#pragma unroll
  for (int j = 0; j < N; ++j) {
    a[tri(j, j)] = dinv[j];
#pragma unroll
    for (int i = j + 1; i < N; ++i) {
      double t = 0.0;
#pragma unroll
      for (int k = j; k < i; ++k) t = fma(a[tri(i, k)], a[tri(k, j)], t);
      a[tri(i, j)] = -t * dinv[i];
    }
  }
}

template <int N>
__device__ __forceinline__ void store_inverse(const double (&t)[N * (N + 1) / 2], double* __restrict__ out) {
#pragma unroll
  for (int c = 0; c < N; ++c) {
#pragma unroll
    for (int r = c; r < N; ++r) {
      double x = 0.0;
#pragma unroll
      for (int k = r; k < N; ++k) x = fma(t[tri(k, r)], t[tri(k, c)], x);
      out[r + c * N] = x;
      if (r != c) out[c + r * N] = x;
    }
  }
}

// The inverse X = L^-T L^-1 from the inverted factor t, written by the
// warp's active lanes together: in three passes of nine columns' 27 entries
// each lane stages its particle's entries in shared memory (stage: 27 rows
// of the warp's 32 lanes, `stride` doubles apart), then the warp writes them
// particle by particle, 27 consecutive
// doubles per store instruction, instead of 81 scattered 8-byte stores per
// lane.  The active lanes are the lowest ones (lanes past the particle count
// have left).  Same values as store_inverse (the same fused products in the
// same order); NaN where the factorisation failed (ok = false).
__device__ __forceinline__ void warp_store_inverse(const double (&t)[45], bool ok, double* out, double* stage,
                                                   int stride, unsigned active) {
  const int lane = threadIdx.x & (kWarp - 1);
  const int nact = __popc(active);
  const unsigned long long mine = reinterpret_cast<unsigned long long>(out);
#pragma unroll
  for (int pass = 0; pass < 3; ++pass) {
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
      const int c = 3 * pass + cc;
#pragma unroll
      for (int r = 0; r < 9; ++r) {
        const int lo = r > c ? r : c;
        double x = 0.0;
#pragma unroll
        for (int k = lo; k < 9; ++k) x = fma(t[tri(k, r)], t[tri(k, c)], x);
        stage[(cc * 9 + r) * stride + lane] = ok ? x : __longlong_as_double(0x7ff8000000000000LL);
      }
    }
    __syncwarp(active);
    for (unsigned rem = active; rem; rem &= rem - 1) {
      const int p = __ffs(rem) - 1;
      double* op = reinterpret_cast<double*>(__shfl_sync(active, mine, p));
      for (int e = lane; e < 27; e += nact) op[27 * pass + e] = stage[e * stride + p];
    }
    __syncwarp(active);
  }
}

// Adds the wall term of boundary kind B (0 none, 1 Dirichlet sample,
// 2 pressure Neumann) to m, regularises, inverts and stores one kind (with
// stage, by the warp's active lanes together: warp_store_inverse).
template <int N, int B>
__device__ __forceinline__ void finish_kind(double (&m)[N * (N + 1) / 2], const MomentArgs& a, const KindOut& ko,
                                            index_t i, double xi, double yi, double zi) {
  double b[N];
  if (B != 0) {
    const index_t we = a.wo[i + 1];
    for (index_t o = a.wo[i]; o < we; ++o) {
      const index_t j = a.wi[o];
      const double dx = a.walls.x[j] - xi, dy = a.walls.y[j] - yi, dz = a.walls.z[j] - zi;
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 <= 0.0) continue;
      const double w = a.wall_scale * (1.0 - sqrt(d2) * a.inv_re);
      if (w <= 0.0) continue;
      if (B == 2) {
        neumann<N>(dx, dy, dz, a.walls.normal_x[j], a.walls.normal_y[j], a.walls.normal_z[j], a.inv_re, b);
      } else {
        basis<N>(dx, dy, dz, a.inv_re, b);
      }
      add_outer<N>(m, b, w);
    }
  }
  // trace and regularisation, moment_matrix.cu:297-308
  double trace = 0.0;
#pragma unroll
  for (int r = 0; r < N; ++r) trace += m[tri(r, r)];
  const double reg = a.lambda * (trace > 0.0 ? trace / static_cast<double>(N) : 1.0);
#pragma unroll
  for (int r = 0; r < N; ++r) m[tri(r, r)] += reg;
  const int info = cholesky<N>(m);
  double* out = ko.inverse + static_cast<size_t>(i) * N * N;
  if (info == 0) {
    invert_lower<N>(m);
    store_inverse<N>(m, out);
  } else {
    for (int e = 0; e < N * N; ++e) out[e] = __longlong_as_double(0x7ff8000000000000LL);
    atomicAdd(&a.status->non_spd, 1u);
    raise_flag(a.status, kFlagNonSpd);
  }
  ko.trace[i] = trace;
  ko.reg[i] = reg;
  ko.info[i] = info;
}

// One or two kinds (B1 < 0: one) from one pass over the fluid row.
template <int N, int B0, int B1>
__global__ void __launch_bounds__(kMomentThreads) moment_kernel(MomentArgs a) {
  constexpr int E = N * (N + 1) / 2;
  extern __shared__ double s_fluid[];  // [E][kMomentThreads] when two kinds share the fluid sum
  const index_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (a.k0.count) atomicAdd(a.k0.count, 1);
    if (B1 >= 0 && a.k1.count) atomicAdd(a.k1.count, 1);
  }
  if (i >= static_cast<index_t>(a.fluid.count)) return;
  const double* __restrict__ fx = a.fluid.x;
  const double* __restrict__ fy = a.fluid.y;
  const double* __restrict__ fz = a.fluid.z;
  const double xi = fx[i], yi = fy[i], zi = fz[i];
  double m[E];
#pragma unroll
  for (int e = 0; e < E; ++e) m[e] = 0.0;
  double b[N];
  const index_t fe = a.fo[i + 1];
  for (index_t o = a.fo[i]; o < fe; ++o) {
    const index_t j = a.fi[o];
    const double dx = fx[j] - xi, dy = fy[j] - yi, dz = fz[j] - zi;
    const double d2 = dx * dx + dy * dy + dz * dz;
    if (d2 <= 0.0) continue;
    const double w = 1.0 - sqrt(d2) * a.inv_re;
    if (w <= 0.0) continue;
    basis<N>(dx, dy, dz, a.inv_re, b);
    add_outer<N>(m, b, w);
  }
  if (B1 >= 0) {
#pragma unroll
    for (int e = 0; e < E; ++e) s_fluid[e * kMomentThreads + threadIdx.x] = m[e];
  }
  finish_kind<N, B0>(m, a, a.k0, i, xi, yi, zi);
  if (B1 >= 0) {
#pragma unroll
    for (int e = 0; e < E; ++e) m[e] = s_fluid[e * kMomentThreads + threadIdx.x];
    finish_kind<N, (B1 < 0 ? 0 : B1)>(m, a, a.k1, i, xi, yi, zi);
  }
}

// ---------------------------------------------------------------------------
// Type-A through monomial sums.
//
// Every entry of sum_j w b b^T with b = (sx, sy, sz, sx^2, sy^2, sz^2, sx sy,
// sy sz, sz sx) is a weighted sum of one monomial of degree 2, 3 or 4 in
// (sx, sy, sz), and the 45 lower-triangle entries share 31 distinct
// monomials (6 + 10 + 15).  The hot loop accumulates those 31 sums
// (10 products and 31 FMAs per neighbour instead of 18 products and 45 FMAs)
// and the 45 entries are expanded once per particle.  Wall Dirichlet samples
// use the same basis and go into the same sums; the wall Neumann vectors have
// no such structure and are added to the expanded entries.
// ---------------------------------------------------------------------------
constexpr int kMonomials = 31;

// Exponent of axis (0 x, 1 y, 2 z) in Type-A basis entry r.
__host__ __device__ constexpr int basis_exponent(int r, int axis) {
  return r < 3 ? (r == axis ? 1 : 0)
       : r == 3 ? (axis == 0 ? 2 : 0)
       : r == 4 ? (axis == 1 ? 2 : 0)
       : r == 5 ? (axis == 2 ? 2 : 0)
       : r == 6 ? (axis == 0 || axis == 1 ? 1 : 0)
       : r == 7 ? (axis == 1 || axis == 2 ? 1 : 0)
                : (axis == 2 || axis == 0 ? 1 : 0);
}

// Slot of the monomial x^a y^b z^c in the 31 sums (layout of acc_monomials).
__host__ __device__ constexpr int monomial_slot(int a, int b, int c) {
  const int code = a * 25 + b * 5 + c;
  switch (code) {
    case 50: return 0;   // xx
    case 10: return 1;   // yy
    case 2: return 2;    // zz
    case 30: return 3;   // xy
    case 6: return 4;    // yz
    case 26: return 5;   // zx
    case 75: return 6;   // xxx
    case 15: return 7;   // yyy
    case 3: return 8;    // zzz
    case 55: return 9;   // xxy
    case 51: return 10;  // xxz
    case 35: return 11;  // xyy
    case 11: return 12;  // yyz
    case 27: return 13;  // xzz
    case 7: return 14;   // yzz
    case 31: return 15;  // xyz
    case 100: return 16; // xxxx
    case 20: return 17;  // yyyy
    case 4: return 18;   // zzzz
    case 80: return 19;  // xxxy
    case 76: return 20;  // xxxz
    case 40: return 21;  // xyyy
    case 16: return 22;  // yyyz
    case 28: return 23;  // xzzz
    case 8: return 24;   // yzzz
    case 60: return 25;  // xxyy
    case 12: return 26;  // yyzz
    case 52: return 27;  // xxzz
    case 56: return 28;  // xxyz
    case 36: return 29;  // xyyz
    case 32: return 30;  // xyzz
    default: return -1;
  }
}

__host__ __device__ constexpr int entry_slot(int r, int c) {
  return monomial_slot(basis_exponent(r, 0) + basis_exponent(c, 0), basis_exponent(r, 1) + basis_exponent(c, 1),
                       basis_exponent(r, 2) + basis_exponent(c, 2));
}

template <typename T>
__device__ __forceinline__ void acc_monomials(T (&s)[kMonomials], T sx, T sy, T sz, T w) {
  const T qxx = sx * sx, qyy = sy * sy, qzz = sz * sz;
  const T qxy = sx * sy, qyz = sy * sz, qzx = sz * sx;
  const T wxx = w * qxx, wyy = w * qyy, wzz = w * qzz, wxy = w * qxy;
  s[0] = fma(w, qxx, s[0]);
  s[1] = fma(w, qyy, s[1]);
  s[2] = fma(w, qzz, s[2]);
  s[3] = fma(w, qxy, s[3]);
  s[4] = fma(w, qyz, s[4]);
  s[5] = fma(w, qzx, s[5]);
  s[6] = fma(wxx, sx, s[6]);
  s[7] = fma(wyy, sy, s[7]);
  s[8] = fma(wzz, sz, s[8]);
  s[9] = fma(wxx, sy, s[9]);
  s[10] = fma(wxx, sz, s[10]);
  s[11] = fma(wyy, sx, s[11]);
  s[12] = fma(wyy, sz, s[12]);
  s[13] = fma(wzz, sx, s[13]);
  s[14] = fma(wzz, sy, s[14]);
  s[15] = fma(wxy, sz, s[15]);
  s[16] = fma(wxx, qxx, s[16]);
  s[17] = fma(wyy, qyy, s[17]);
  s[18] = fma(wzz, qzz, s[18]);
  s[19] = fma(wxx, qxy, s[19]);
  s[20] = fma(wxx, qzx, s[20]);
  s[21] = fma(wyy, qxy, s[21]);
  s[22] = fma(wyy, qyz, s[22]);
  s[23] = fma(wzz, qzx, s[23]);
  s[24] = fma(wzz, qyz, s[24]);
  s[25] = fma(wxx, qyy, s[25]);
  s[26] = fma(wyy, qzz, s[26]);
  s[27] = fma(wzz, qxx, s[27]);
  s[28] = fma(wxx, qyz, s[28]);
  s[29] = fma(wyy, qzx, s[29]);
  s[30] = fma(wzz, qxy, s[30]);
}

struct MomentPackedArgs {
  index_t n;
  const double4* fp;  // {x, y, z, -} fluid
  const double4* wp;  // {x, y, z, -} walls
  const double4* wn;  // {nx, ny, nz, -} walls
  const index_t* fo;
  const index_t* fi;
  const index_t* wo;
  const index_t* wi;
  double inv_re;
  double lambda;
  double wall_scale;
  KindOut k0;
  KindOut k1;
  DeviceStatus* status;
  const int32_t* order;  // visiting order (lsmps_ctx::order) or NULL
  int sorted;            // fi and fp in cell-sorted positions (sorted_rows_of)
};

template <int B>
__device__ __forceinline__ void finish_a(double (&s)[kMonomials], const MomentPackedArgs& a, const KindOut& ko,
                                         index_t i, const double4& pi, double* stage = nullptr,
                                         int stride = kWarp, unsigned active = 0u) {
  const index_t wb = a.wo[i], we = a.wo[i + 1];
  // The wall loops load the next wall's record(s) while this one is used,
  // with the index one further ahead.
  if (B == 1 && wb < we) {
    double4 qn = ld4(a.wp, a.wi[wb]);
    index_t jnn = wb + 1 < we ? a.wi[wb + 1] : 0;
    for (index_t o = wb; o < we; ++o) {
      const double4 q = qn;
      if (o + 1 < we) {
        qn = ld4(a.wp, jnn);
        if (o + 2 < we) jnn = a.wi[o + 2];
      }
      const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 <= 0.0) continue;
      const double w = a.wall_scale * (1.0 - sqrt(d2) * a.inv_re);
      if (w <= 0.0) continue;
      acc_monomials(s, dx * a.inv_re, dy * a.inv_re, dz * a.inv_re, w);
    }
  }
  double m[45];
#pragma unroll
  for (int r = 0; r < 9; ++r) {
#pragma unroll
    for (int c = 0; c <= r; ++c) m[tri(r, c)] = s[entry_slot(r, c)];
  }
  if (B == 2 && wb < we) {
    double q9[9];
    index_t jn = a.wi[wb];
    index_t jnn = wb + 1 < we ? a.wi[wb + 1] : 0;
    double4 qn = ld4(a.wp, jn), nn = ld4(a.wn, jn);
    for (index_t o = wb; o < we; ++o) {
      const double4 q = qn, nrm = nn;
      if (o + 1 < we) {
        jn = jnn;
        qn = ld4(a.wp, jn);
        nn = ld4(a.wn, jn);
        if (o + 2 < we) jnn = a.wi[o + 2];
      }
      const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 <= 0.0) continue;
      const double w = a.wall_scale * (1.0 - sqrt(d2) * a.inv_re);
      if (w <= 0.0) continue;
      neumann<9>(dx, dy, dz, nrm.x, nrm.y, nrm.z, a.inv_re, q9);
      add_outer<9>(m, q9, w);
    }
  }
  double trace = 0.0;
#pragma unroll
  for (int r = 0; r < 9; ++r) trace += m[tri(r, r)];
  const double reg = a.lambda * (trace > 0.0 ? trace / 9.0 : 1.0);
#pragma unroll
  for (int r = 0; r < 9; ++r) m[tri(r, r)] += reg;
  const int info = cholesky<9>(m);
  double* out = ko.inverse + static_cast<size_t>(i) * 81;
  if (info == 0) invert_lower<9>(m);
  if (stage) {
    warp_store_inverse(m, info == 0, out, stage, stride, active);
  } else if (info == 0) {
    store_inverse<9>(m, out);
  } else {
    for (int e = 0; e < 81; ++e) out[e] = __longlong_as_double(0x7ff8000000000000LL);
  }
  if (info != 0) {
    atomicAdd(&a.status->non_spd, 1u);
    raise_flag(a.status, kFlagNonSpd);
  }
  ko.trace[i] = trace;
  ko.reg[i] = reg;
  ko.info[i] = info;
}

// Type-A kinds B0 (and B1 >= 0) from one pass over the fluid row.  MinBlocks
// is the register budget variant (LSMPS_KNOB_MOMENT_OCCUPANCY).
// The last kind's inverses are written through shared memory by the warp
// (warp_store_inverse; the first of two kinds with scalar stores, its
// shared memory still holding the second kind's sums).
template <int B0, int B1, int MinBlocks>
__global__ void __launch_bounds__(kMomentThreads, MinBlocks) moment_a_kernel(MomentPackedArgs a) {
  // [kMonomials][kMomentThreads] when B1 >= 0, else [27][kMomentThreads]
  extern __shared__ double s_mono[];
  const index_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (a.k0.count) atomicAdd(a.k0.count, 1);
    if (B1 >= 0 && a.k1.count) atomicAdd(a.k1.count, 1);
  }
  const unsigned active = __ballot_sync(0xffffffffu, t < a.n);
  if (t >= a.n) return;
  double* stage = s_mono + (threadIdx.x & ~(kWarp - 1));
  const index_t i = visit(a.order, t);
  const double4 pi = ld4(a.fp, self_of(a.sorted, t, i));
  double s[kMonomials];
#pragma unroll
  for (int e = 0; e < kMonomials; ++e) s[e] = 0.0;
  // The next neighbour's record is loaded while this one is accumulated.
  const index_t fe = a.fo[i + 1];
  index_t o = a.fo[i];
  double4 qn = o < fe ? ld4(a.fp, a.fi[o]) : pi;
  for (; o < fe; ++o) {
    const double4 q = qn;
    if (o + 1 < fe) qn = ld4(a.fp, a.fi[o + 1]);
    const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
    const double d2 = dx * dx + dy * dy + dz * dz;
    if (d2 <= 0.0) continue;
    const double w = 1.0 - sqrt(d2) * a.inv_re;
    if (w <= 0.0) continue;
    acc_monomials(s, dx * a.inv_re, dy * a.inv_re, dz * a.inv_re, w);
  }
  if (B1 >= 0) {
#pragma unroll
    for (int e = 0; e < kMonomials; ++e) s_mono[e * kMomentThreads + threadIdx.x] = s[e];
  }
  if (B1 < 0) {
    finish_a<B0>(s, a, a.k0, i, pi, stage, kMomentThreads, active);
    return;
  }
  finish_a<B0>(s, a, a.k0, i, pi);
#pragma unroll
  for (int e = 0; e < kMonomials; ++e) s[e] = s_mono[e * kMomentThreads + threadIdx.x];
  finish_a<(B1 < 0 ? 0 : B1)>(s, a, a.k1, i, pi, stage, kMomentThreads, active);
}

// The velocity and pressure kinds with the two warps of a 64-thread block
// sharing 32 particles: warp h sums the even (h = 0) or odd (h = 1) entries of
// each row, the halves are exchanged through shared memory, then warp 0
// finishes the velocity kind and warp 1 the pressure kind, so neither the
// row sum nor the two factorisations run twice in one thread and no warp
// diverges between the kinds (LSMPS_KNOB_MOMENT_OCCUPANCY variant 2).
__global__ void __launch_bounds__(2 * kWarp, 8) moment_a_split_kernel(MomentPackedArgs a) {
  __shared__ double s_half[2][kMonomials][kWarp];
  const int lane = threadIdx.x & (kWarp - 1), half = threadIdx.x >> 5;
  const index_t t = blockIdx.x * kWarp + lane;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (a.k0.count) atomicAdd(a.k0.count, 1);
    if (a.k1.count) atomicAdd(a.k1.count, 1);
  }
  const bool live = t < a.n;
  const index_t i = live ? visit(a.order, t) : 0;
  const double4 pi = live ? ld4(a.fp, self_of(a.sorted, t, i)) : make_double4(0.0, 0.0, 0.0, 0.0);
  double s[kMonomials];
#pragma unroll
  for (int e = 0; e < kMonomials; ++e) s[e] = 0.0;
  if (live) {
    const index_t fe = a.fo[i + 1];
    index_t o = a.fo[i] + half;
    double4 qn = o < fe ? ld4(a.fp, a.fi[o]) : pi;
    index_t jnn = o + 2 < fe ? a.fi[o + 2] : i;  // the index after the next
    for (; o < fe; o += 2) {
      const double4 q = qn;
      if (o + 2 < fe) {
        qn = ld4(a.fp, jnn);
        if (o + 4 < fe) jnn = a.fi[o + 4];
      }
      const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 <= 0.0) continue;
      const double w = 1.0 - sqrt(d2) * a.inv_re;
      if (w <= 0.0) continue;
      acc_monomials(s, dx * a.inv_re, dy * a.inv_re, dz * a.inv_re, w);
    }
  }
#pragma unroll
  for (int e = 0; e < kMonomials; ++e) s_half[half][e][lane] = s[e];
  __syncthreads();
#pragma unroll
  for (int e = 0; e < kMonomials; ++e) s[e] = s_half[0][e][lane] + s_half[1][e][lane];
  // each warp then stages its kind's inverses in its half of s_half
  __syncthreads();
  const unsigned active = __ballot_sync(0xffffffffu, live);
  if (!live) return;
  double* stage = &s_half[half][0][0];
  static_assert(kMonomials >= 27, "the stage holds 27 x 32 doubles");
  if (half == 0)
    finish_a<1>(s, a, a.k0, i, pi, stage, kWarp, active);
  else
    finish_a<2>(s, a, a.k1, i, pi, stage, kWarp, active);
}

// ---------------------------------------------------------------------------
// Mixed form (LSMPS_PRECISION_MIXED).
//
// Stage 1 (moment_sums_kernel): the 31 fluid monomial sums of each particle.
// Each neighbour's r_e-scaled offset and weight are formed in FP32 from the
// FP64 coordinate difference, its 31 weighted monomials are formed in FP32,
// and each is added into its sum with Kahan's compensated summation (an FP32
// sum and an FP32 running compensation), so the summation adds no error
// beyond O(n u^2) to the rounding of the terms themselves.  The totals
// (sum minus compensation, in FP64) go to the context's mixed_sums array,
// monomial-major.
//
// Stage 2 (moment_rows_kernel, one thread per particle and kind): the kind's
// wall term (FP64; walls are few), trace and regularisation as in the plain
// form, then an FP32 Cholesky factorisation.  The operator rows the step
// consumes are y = M^-1 u for u = e3 + e4 + e5 (the Laplacian row) and
// u = e0, e1, e2 (the gradient rows; M^-1 is symmetric, so rows equal
// columns): each is solved with the FP32 factor and refined once in FP64,
// y1 = y0 + M^-1_f32 (u - M y0) with the residual u - M y0 formed against the
// FP64 matrix.  A matrix whose FP32 factorisation fails, or whose condition
// estimate (max L_ii / min L_ii)^2 exceeds the context's threshold (1e4 by
// default: ill-conditioned Surface and Splash particles), is factorised and
// solved in FP64 instead and counted in DeviceStatus::fallbacks.  The rows
// are stored as FP32, 36 per particle: [Laplacian row, row 0, row 1, row 2].
// With Full, all nine columns are solved and the full FP64 inverse is
// written to the moment view (lsmps_prepare_moments in the mixed form).

constexpr int kSumThreads = 128;
constexpr int kRowThreads = 64;

struct MixedSumArgs {
  index_t n;
  const double4* fp;
  const index_t* fo;
  const index_t* fi;
  double inv_re;
  double* sums;          // [kMonomials][n], by visiting position
  const int32_t* order;  // visiting order (lsmps_ctx::order) or NULL
  int sorted;            // fi and fp in cell-sorted positions (sorted_rows_of)
};

// Kahan step for the 31 weighted monomials of one neighbour (the same
// products as acc_monomials).
__device__ __forceinline__ void kahan_monomials(float (&s)[kMonomials], float (&c)[kMonomials], float sx, float sy,
                                                float sz, float w) {
  float t[kMonomials];
#pragma unroll
  for (int e = 0; e < kMonomials; ++e) t[e] = 0.0f;
  acc_monomials(t, sx, sy, sz, w);
#pragma unroll
  for (int e = 0; e < kMonomials; ++e) {
    const float y = t[e] - c[e];
    const float u = s[e] + y;
    c[e] = (u - s[e]) - y;
    s[e] = u;
  }
}

// The 31 weighted monomials as 16 packed pairs: pair p holds monomial
// sum_pair_lo(p) in its low half and sum_pair_hi(p) in its high half (-1:
// unused).  Every product is the scalar one of acc_monomials (one rounding of
// a two-factor product; wxx = w qxx etc.), two per instruction.
__host__ __device__ constexpr int sum_pair_lo(int p) {
  constexpr int lo[16] = {0, 2, 4, 6, 8, 9, 10, 13, 16, 18, 19, 20, 28, 24, 25, 27};
  return lo[p];
}
__host__ __device__ constexpr int sum_pair_hi(int p) {
  constexpr int hi[16] = {1, 3, 5, 7, 15, 11, 12, 14, 17, 30, 21, 29, 22, 23, 26, -1};
  return hi[p];
}

__device__ __forceinline__ void monomial_pairs(f32x2 (&t)[16], float sx, float sy, float sz, float w) {
  const f32x2 xy = pack2(sx, sy);
  const f32x2 q1 = mul2(xy, xy);                          // qxx, qyy
  const f32x2 q2 = mul2(pack2(sz, sx), pack2(sz, sy));    // qzz, qxy
  const f32x2 q3 = mul2(pack2(sy, sz), pack2(sz, sx));    // qyz, qzx
  const f32x2 ww = pack2(w, w);
  const f32x2 w1 = mul2(ww, q1);                          // wxx, wyy
  const f32x2 w2 = mul2(ww, q2);                          // wzz, wxy
  const f32x2 w3 = mul2(ww, q3);                          // w qyz, w qzx
  const float wzz = low_half(w2);
  const f32x2 zz = pack2(wzz, wzz);
  t[0] = w1;
  t[1] = w2;
  t[2] = w3;
  t[3] = mul2(w1, xy);                                    // wxx x, wyy y
  t[4] = mul2(w2, pack2(sz, sz));                         // wzz z, wxy z
  t[5] = mul2(w1, pack2(sy, sx));                         // wxx y, wyy x
  t[6] = mul2(w1, pack2(sz, sz));                         // wxx z, wyy z
  t[7] = mul2(zz, xy);                                    // wzz x, wzz y
  t[8] = mul2(w1, q1);                                    // wxx qxx, wyy qyy
  t[9] = mul2(zz, q2);                                    // wzz qzz, wzz qxy
  const float qxy = high_half(q2), qzx = high_half(q3), qyz = low_half(q3);
  t[10] = mul2(w1, pack2(qxy, qxy));                      // wxx qxy, wyy qxy
  t[11] = mul2(w1, pack2(qzx, qzx));                      // wxx qzx, wyy qzx
  t[12] = mul2(w1, pack2(qyz, qyz));                      // wxx qyz, wyy qyz
  t[13] = mul2(zz, q3);                                   // wzz qyz, wzz qzx
  t[14] = mul2(w1, pack2(high_half(q1), low_half(q2)));   // wxx qyy, wyy qzz
  t[15] = pack2(wzz * low_half(q1), 0.0f);                // wzz qxx
}

__global__ void __launch_bounds__(kSumThreads) moment_sums_kernel(MixedSumArgs a) {
  const index_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  const index_t i = visit(a.order, t);
  const double4 pi = ld4(a.fp, self_of(a.sorted, t, i));
  // Kahan sums and compensations, two monomials per register pair
  f32x2 sum[16], comp[16];
#pragma unroll
  for (int p = 0; p < 16; ++p) sum[p] = comp[p] = 0ull;
  const index_t fb = a.fo[i], fe = a.fo[i + 1];
  double4 qn = fb < fe ? ld4(a.fp, a.fi[fb]) : pi;
  index_t jnn = fb + 1 < fe ? a.fi[fb + 1] : i;  // the index after the next
  for (index_t o = fb; o < fe; ++o) {
    const double4 q = qn;
    if (o + 1 < fe) {
      qn = ld4(a.fp, jnn);
      if (o + 2 < fe) jnn = a.fi[o + 2];
    }
    const float sx = static_cast<float>((q.x - pi.x) * a.inv_re);
    const float sy = static_cast<float>((q.y - pi.y) * a.inv_re);
    const float sz = static_cast<float>((q.z - pi.z) * a.inv_re);
    const float d2 = sx * sx + sy * sy + sz * sz;
    if (d2 > 0.0f) {
      const float w = 1.0f - sqrtf(d2);
      if (w > 0.0f) {
        f32x2 tm[16];
        monomial_pairs(tm, sx, sy, sz, w);
#pragma unroll
        for (int p = 0; p < 16; ++p) {
          const f32x2 y = sub2(tm[p], comp[p]);
          const f32x2 u = add2(sum[p], y);
          comp[p] = sub2(sub2(u, sum[p]), y);
          sum[p] = u;
        }
      }
    }
  }
  const size_t n = static_cast<size_t>(a.n);
#pragma unroll
  for (int p = 0; p < 16; ++p) {
    a.sums[sum_pair_lo(p) * n + t] = static_cast<double>(low_half(sum[p])) - static_cast<double>(low_half(comp[p]));
    if (sum_pair_hi(p) >= 0)
      a.sums[sum_pair_hi(p) * n + t] =
          static_cast<double>(high_half(sum[p])) - static_cast<double>(high_half(comp[p]));
  }
}

struct MixedRowArgs {
  index_t n;
  const double* sums;
  const double4* fp;
  const double4* wp;
  const double4* wn;
  const index_t* fo;
  const index_t* fi;
  const index_t* wo;
  const index_t* wi;
  double inv_re;
  double lambda;
  double wall_scale;
  double kappa_threshold;
  KindOut k[2];       // velocity Dirichlet-A, pressure Neumann-A
  // compact rows per kind (unless Full), by visiting position: FP32, the
  // FP64 ones of the FP64-route particles, and 1 where rows64 holds them
  float* rows[2];
  double* rows64[2];
  uint8_t* flag[2];
  int32_t* list[2];   // the FP64-route particles' visiting positions, appended (unless Full)
  unsigned int* count;
  DeviceStatus* status;
  const int32_t* order;  // visiting order (the sums are stored by visiting position) or NULL
  int sorted;            // fi and fp in cell-sorted positions (sorted_rows_of)
};

// v <- L^-T L^-1 v with the packed lower factor and its reciprocal diagonal.
template <typename T>
__device__ __forceinline__ void chol_solve(const T (&l)[45], const T (&dinv)[9], T (&v)[9]) {
#pragma unroll
  for (int r = 0; r < 9; ++r) {
    T t = v[r];
#pragma unroll
    for (int k = 0; k < r; ++k) t = fma(-l[tri(r, k)], v[k], t);
    v[r] = t * dinv[r];
  }
#pragma unroll
  for (int r = 8; r >= 0; --r) {
    T t = v[r];
#pragma unroll
    for (int k = r + 1; k < 9; ++k) t = fma(-l[tri(k, r)], v[k], t);
    v[r] = t * dinv[r];
  }
}

// The same for G right-hand sides at once (independent chains interleaved).
template <typename T, int G>
__device__ __forceinline__ void chol_solve_group(const T (&l)[45], const T (&dinv)[9], T (&v)[G][9]) {
#pragma unroll
  for (int r = 0; r < 9; ++r) {
#pragma unroll
    for (int g = 0; g < G; ++g) {
      T t = v[g][r];
#pragma unroll
      for (int k = 0; k < r; ++k) t = fma(-l[tri(r, k)], v[g][k], t);
      v[g][r] = t * dinv[r];
    }
  }
#pragma unroll
  for (int r = 8; r >= 0; --r) {
#pragma unroll
    for (int g = 0; g < G; ++g) {
      T t = v[g][r];
#pragma unroll
      for (int k = r + 1; k < 9; ++k) t = fma(-l[tri(k, r)], v[g][k], t);
      v[g][r] = t * dinv[r];
    }
  }
}

// Estimate of ||M^-1||_1 from the FP32 factor by Hager's method with
// Higham's refinements (N. J. Higham, "FORTRAN codes for estimating the
// one-norm of a real or complex matrix", ACM TOMS 14 (1988); the iteration of
// LAPACK's xLACN2): x = e/n; repeat y = M^-1 x, z = M^-T sign(y) (= M^-1
// sign(y), M symmetric); stop when ||z||_inf <= z.x, else x = e_j at the
// largest |z_j|.  At most two rounds here, and the result is raised to
// Higham's alternative lower bound 2 ||M^-1 b||_1 / (3n) with
// b_i = (-1)^i (1 + i/(n-1)).  A lower bound of ||M^-1||_1, usually within a
// small factor of it.
__device__ __forceinline__ float inverse_norm1_estimate(const float (&l)[45], const float (&dinv)[9]) {
  float x[9], y[9], z[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) x[r] = 1.0f / 9.0f;
  float est = 0.0f;
#pragma unroll 1
  for (int round = 0; round < 2; ++round) {
#pragma unroll
    for (int r = 0; r < 9; ++r) y[r] = x[r];
    chol_solve(l, dinv, y);
    float ny = 0.0f;
#pragma unroll
    for (int r = 0; r < 9; ++r) ny += fabsf(y[r]);
    if (round > 0 && ny <= est) break;
    est = ny;
#pragma unroll
    for (int r = 0; r < 9; ++r) z[r] = y[r] >= 0.0f ? 1.0f : -1.0f;
    chol_solve(l, dinv, z);
    int jmax = 0;
    float zmax = fabsf(z[0]), zx = z[0] * x[0];
#pragma unroll
    for (int r = 1; r < 9; ++r) {
      zx = fmaf(z[r], x[r], zx);
      if (fabsf(z[r]) > zmax) {
        zmax = fabsf(z[r]);
        jmax = r;
      }
    }
    if (zmax <= zx) break;
#pragma unroll
    for (int r = 0; r < 9; ++r) x[r] = r == jmax ? 1.0f : 0.0f;
  }
#pragma unroll
  for (int r = 0; r < 9; ++r) y[r] = ((r & 1) ? -1.0f : 1.0f) * (1.0f + static_cast<float>(r) / 8.0f);
  chol_solve(l, dinv, y);
  float alt = 0.0f;
#pragma unroll
  for (int r = 0; r < 9; ++r) alt += fabsf(y[r]);
  alt *= 2.0f / 27.0f;
  return fmaxf(est, alt);
}

// Target t of the row set: t = 0 the Laplacian row (e3 + e4 + e5), t = 1..3
// rows 0..2; with Full, t = 0..8 is e_t.
template <bool Full>
__device__ __forceinline__ double target(int t, int r) {
  if (Full) return r == t ? 1.0 : 0.0;
  if (t == 0) return (r >= 3 && r <= 5) ? 1.0 : 0.0;
  return r == t - 1 ? 1.0 : 0.0;
}

template <bool Full>
__device__ __forceinline__ void store_target(const MixedRowArgs& a, int kind, index_t i, index_t vt, int t,
                                             const double (&y)[9], bool fp64) {
  if (Full) {
    double* out = a.k[kind].inverse + static_cast<size_t>(i) * 81;
#pragma unroll
    for (int r = 0; r < 9; ++r) {
      if (r < t) continue;
      out[r + t * 9] = y[r];
      out[t + r * 9] = y[r];
    }
  } else if (fp64) {
    double* out = a.rows64[kind] + static_cast<size_t>(vt) * 36 + t * 9;
#pragma unroll
    for (int r = 0; r < 9; ++r) out[r] = y[r];
  } else {
    float* out = a.rows[kind] + static_cast<size_t>(vt) * 36 + t * 9;
#pragma unroll
    for (int r = 0; r < 9; ++r) out[r] = static_cast<float>(y[r]);
  }
}

// The kind's matrix from the 31 fluid monomial totals s: the wall term (FP64;
// Dirichlet into s, Neumann as q q^T), expanded into the thread's column of
// shared memory m[e * kRowThreads], then trace and regularisation
// (moment_matrix.cu:286-308).  Returns the trace; *reg gets the shift.
__device__ __forceinline__ double assemble_kind(const MixedRowArgs& a, int kind, index_t i, const double4& pi,
                                                double (&s)[kMonomials], double* m, double* reg) {
  const index_t wb = a.wo[i], we = a.wo[i + 1];
  // The wall loops load the next wall's record(s) while this one is used,
  // with the index one further ahead.
  if (kind == 0 && wb < we) {
    double4 qn = ld4(a.wp, a.wi[wb]);
    index_t jnn = wb + 1 < we ? a.wi[wb + 1] : 0;
    for (index_t o = wb; o < we; ++o) {
      const double4 q = qn;
      if (o + 1 < we) {
        qn = ld4(a.wp, jnn);
        if (o + 2 < we) jnn = a.wi[o + 2];
      }
      const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 <= 0.0) continue;
      const double w = a.wall_scale * (1.0 - sqrt(d2) * a.inv_re);
      if (w <= 0.0) continue;
      acc_monomials(s, dx * a.inv_re, dy * a.inv_re, dz * a.inv_re, w);
    }
  }
#pragma unroll
  for (int r = 0; r < 9; ++r) {
#pragma unroll
    for (int c = 0; c <= r; ++c) m[tri(r, c) * kRowThreads] = s[entry_slot(r, c)];
  }
  if (kind == 1) {
    // The wall terms w q q^T in row order, two walls per pass over the 45
    // entries in shared memory (each entry gets the first wall's term, then
    // the second's: the same sums as one wall per pass, half the traffic).
    double qa[9], qb[9], wa = 0.0;
    bool held = false;
    index_t jn = wb < we ? a.wi[wb] : 0;
    index_t jnn = wb + 1 < we ? a.wi[wb + 1] : 0;
    double4 qn = make_double4(0.0, 0.0, 0.0, 0.0), nn = qn;
    if (wb < we) {
      qn = ld4(a.wp, jn);
      nn = ld4(a.wn, jn);
    }
    for (index_t o = wb; o < we; ++o) {
      const double4 q = qn, nrm = nn;
      if (o + 1 < we) {
        jn = jnn;
        qn = ld4(a.wp, jn);
        nn = ld4(a.wn, jn);
        if (o + 2 < we) jnn = a.wi[o + 2];
      }
      const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 <= 0.0) continue;
      const double w = a.wall_scale * (1.0 - sqrt(d2) * a.inv_re);
      if (w <= 0.0) continue;
      if (!held) {
        neumann<9>(dx, dy, dz, nrm.x, nrm.y, nrm.z, a.inv_re, qa);
        wa = w;
        held = true;
        continue;
      }
      neumann<9>(dx, dy, dz, nrm.x, nrm.y, nrm.z, a.inv_re, qb);
#pragma unroll
      for (int r = 0; r < 9; ++r) {
        const double war = wa * qa[r], wbr = w * qb[r];
#pragma unroll
        for (int c = 0; c <= r; ++c)
          m[tri(r, c) * kRowThreads] = fma(wbr, qb[c], fma(war, qa[c], m[tri(r, c) * kRowThreads]));
      }
      held = false;
    }
    if (held) {
#pragma unroll
      for (int r = 0; r < 9; ++r) {
        const double war = wa * qa[r];
#pragma unroll
        for (int c = 0; c <= r; ++c) m[tri(r, c) * kRowThreads] = fma(war, qa[c], m[tri(r, c) * kRowThreads]);
      }
    }
  }
  double trace = 0.0;
#pragma unroll
  for (int r = 0; r < 9; ++r) trace += m[tri(r, r) * kRowThreads];
  *reg = a.lambda * (trace > 0.0 ? trace / 9.0 : 1.0);
#pragma unroll
  for (int r = 0; r < 9; ++r) m[tri(r, r) * kRowThreads] += *reg;
  return trace;
}

// Stage 2 of one particle (index i, visiting position vt: what the FP64-route
// list records) and kind from its fluid monomial totals s (the thread's
// column of shared memory m holds the kind's matrix).
template <bool Full>
__device__ __forceinline__ void mixed_rows_of_particle(const MixedRowArgs& a, int kind, index_t vt, index_t i,
                                                       const double4& pi,
                                                       double (&s)[kMonomials], double* m) {
  const KindOut& ko = a.k[kind];
  constexpr int kTargets = Full ? 9 : 4;
  double reg = 0.0, trace = 0.0;
  trace = assemble_kind(a, kind, i, pi, s, m, &reg);
  float l[45];
#pragma unroll
  for (int e = 0; e < 45; ++e) l[e] = static_cast<float>(m[e * kRowThreads]);
  int info = cholesky<9>(l);
  bool fp64 = info != 0;
  float dinv[9];
  if (!fp64) {
    float lo = l[tri(0, 0)], hi = lo;
#pragma unroll
    for (int r = 1; r < 9; ++r) {
      lo = fminf(lo, l[tri(r, r)]);
      hi = fmaxf(hi, l[tri(r, r)]);
    }
#pragma unroll
    for (int r = 0; r < 9; ++r) dinv[r] = 1.0f / l[tri(r, r)];
    // Condition estimate: the larger of (max L_ii / min L_ii)^2 (a lower
    // bound of kappa_2) and kappa_1 = ||M||_1 * est(||M^-1||_1).
    const double ratio = static_cast<double>(hi) / static_cast<double>(lo);
    double norm1 = 0.0;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      double col = 0.0;
#pragma unroll
      for (int r = 0; r < 9; ++r) col += fabs(m[(r >= c ? tri(r, c) : tri(c, r)) * kRowThreads]);
      norm1 = fmax(norm1, col);
    }
    const double kappa1 = norm1 * static_cast<double>(inverse_norm1_estimate(l, dinv));
    const double kappa = fmax(ratio * ratio, kappa1);
    // NaN (an overflowed estimate) also takes the FP64 route
    fp64 = !(kappa <= a.kappa_threshold);
  }
  if (!fp64) {
    // The targets are solved in groups of kGroup so that their independent
    // substitution chains interleave.
    constexpr int kGroup = Full ? 3 : 2;  // divides kTargets
    static_assert(kTargets % kGroup == 0, "target groups must tile the targets");
    for (int t0 = 0; t0 < kTargets; t0 += kGroup) {
      float y0[kGroup][9], d[kGroup][9];
#pragma unroll
      for (int g = 0; g < kGroup; ++g) {
#pragma unroll
        for (int r = 0; r < 9; ++r) y0[g][r] = static_cast<float>(target<Full>(t0 + g, r));
      }
      chol_solve_group(l, dinv, y0);
      // one refinement step: residual against the FP64 matrix (each entry
      // read once for the group), correction through the FP32 factor
#pragma unroll
      for (int r = 0; r < 9; ++r) {
        double res[kGroup];
#pragma unroll
        for (int g = 0; g < kGroup; ++g) res[g] = target<Full>(t0 + g, r);
#pragma unroll
        for (int c = 0; c < 9; ++c) {
          const int e = r >= c ? tri(r, c) : tri(c, r);
          const double mv = m[e * kRowThreads];
#pragma unroll
          for (int g = 0; g < kGroup; ++g) res[g] = fma(-mv, static_cast<double>(y0[g][c]), res[g]);
        }
#pragma unroll
        for (int g = 0; g < kGroup; ++g) d[g][r] = static_cast<float>(res[g]);
      }
      chol_solve_group(l, dinv, d);
      if (Full) {
#pragma unroll
        for (int g = 0; g < kGroup; ++g) {
          double y[9];
#pragma unroll
          for (int r = 0; r < 9; ++r) y[r] = static_cast<double>(y0[g][r]) + static_cast<double>(d[g][r]);
          store_target<Full>(a, kind, i, vt, t0 + g, y, false);
        }
      } else {
        // The group's rows are adjacent in the particle's 36 floats (144
        // bytes) and start on 16 bytes (the first pair) or 8 bytes (the
        // second): written as float quadruples and pairs, fewer store
        // instructions than the scalar form, the same values.
        static_assert(Full || kGroup == 2, "row pairs");
        float f[kGroup * 9];
#pragma unroll
        for (int g = 0; g < kGroup; ++g) {
#pragma unroll
          for (int r = 0; r < 9; ++r)
            f[g * 9 + r] = static_cast<float>(static_cast<double>(y0[g][r]) + static_cast<double>(d[g][r]));
        }
        float* base = a.rows[kind] + static_cast<size_t>(vt) * 36 + t0 * 9;
        if (t0 == 0) {
          float4* out4 = reinterpret_cast<float4*>(base);
#pragma unroll
          for (int k = 0; k < 4; ++k) out4[k] = make_float4(f[4 * k], f[4 * k + 1], f[4 * k + 2], f[4 * k + 3]);
          reinterpret_cast<float2*>(base)[8] = make_float2(f[16], f[17]);
        } else {
          float2* out = reinterpret_cast<float2*>(base);
#pragma unroll
          for (int k = 0; k < kGroup * 9 / 2; ++k) out[k] = make_float2(f[2 * k], f[2 * k + 1]);
        }
      }
    }
    ko.trace[i] = trace;
    ko.reg[i] = reg;
    ko.info[i] = 0;
    if (!Full) a.flag[kind][vt] = 0;
    return;
  }
  // FP64 route: the matrix is re-assembled in FP64 from the particle's rows
  // (the FP32-rounded terms can leave a nearly rank-deficient matrix
  // indefinite) and factorised in FP64, as in the plain form.
  atomicAdd(&a.status->fallbacks, 1u);
  {
    double s[kMonomials];
#pragma unroll
    for (int e = 0; e < kMonomials; ++e) s[e] = 0.0;
    const index_t fe = a.fo[i + 1];
    for (index_t o = a.fo[i]; o < fe; ++o) {
      const double4 q = ld4(a.fp, a.fi[o]);
      const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 <= 0.0) continue;
      const double w = 1.0 - sqrt(d2) * a.inv_re;
      if (w <= 0.0) continue;
      acc_monomials(s, dx * a.inv_re, dy * a.inv_re, dz * a.inv_re, w);
    }
    trace = assemble_kind(a, kind, i, pi, s, m, &reg);
  }
  ko.trace[i] = trace;
  ko.reg[i] = reg;
  if (!Full) {
    a.flag[kind][vt] = 1;
    a.list[kind][atomicAdd(&a.count[kind], 1u)] = vt;
  }
  double l64[45];
#pragma unroll
  for (int e = 0; e < 45; ++e) l64[e] = m[e * kRowThreads];
  info = cholesky<9>(l64);
  ko.info[i] = info;
  if (info != 0) {
    double nan9[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) nan9[r] = __longlong_as_double(0x7ff8000000000000LL);
    for (int t = 0; t < kTargets; ++t) store_target<Full>(a, kind, i, vt, t, nan9, true);
    atomicAdd(&a.status->non_spd, 1u);
    raise_flag(a.status, kFlagNonSpd);
    return;
  }
  double dinv64[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) dinv64[r] = 1.0 / l64[tri(r, r)];
  for (int t = 0; t < kTargets; ++t) {
    double y[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) y[r] = target<Full>(t, r);
    chol_solve(l64, dinv64, y);
    store_target<Full>(a, kind, i, vt, t, y, true);
  }
}

template <bool Full>
__global__ void __launch_bounds__(kRowThreads, 6) moment_rows_kernel(MixedRowArgs a) {
  __shared__ double s_m[45 * kRowThreads];
  const int kind = blockIdx.y;
  const index_t t = blockIdx.x * kRowThreads + threadIdx.x;
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.k[kind].count) atomicAdd(a.k[kind].count, 1);
  if (t >= a.n) return;
  const index_t i = visit(a.order, t);
  const size_t n = static_cast<size_t>(a.n);
  double s[kMonomials];
#pragma unroll
  for (int e = 0; e < kMonomials; ++e) s[e] = a.sums[e * n + t];
  mixed_rows_of_particle<Full>(a, kind, t, i, ld4(a.fp, self_of(a.sorted, t, i)), s, s_m + threadIdx.x);
}

// Both stages in one kernel (the step's path): the two warps of a 64-thread
// block share 32 particles, each warp sums the even or odd entries of their
// rows (Kahan-compensated FP32), the halves meet in shared memory as FP64
// totals, then warp 0 finishes the velocity kind and warp 1 the pressure kind.
template <bool Full>
__global__ void __launch_bounds__(kRowThreads, 6) moment_mixed_split_kernel(MixedSumArgs sa, MixedRowArgs a) {
  static_assert(kRowThreads == 2 * kWarp, "two warps per block");
  __shared__ double s_m[45 * kRowThreads];
  __shared__ double s_half[2][kMonomials][kWarp];
  const int lane = threadIdx.x & (kWarp - 1), half = threadIdx.x >> 5;
  const index_t t = blockIdx.x * kWarp + lane;
  if (blockIdx.x == 0 && lane == 0 && a.k[half].count) atomicAdd(a.k[half].count, 1);
  const bool live = t < a.n;
  const index_t i = live ? visit(a.order, t) : 0;
  const double4 pi = live ? ld4(a.fp, self_of(a.sorted, t, i)) : make_double4(0.0, 0.0, 0.0, 0.0);
  {
    float sum[kMonomials], comp[kMonomials];
#pragma unroll
    for (int e = 0; e < kMonomials; ++e) sum[e] = comp[e] = 0.0f;
    if (live) {
      const index_t fe = sa.fo[i + 1];
      index_t o = sa.fo[i] + half;
      double4 qn = o < fe ? ld4(sa.fp, sa.fi[o]) : pi;
      for (; o < fe; o += 2) {
        const double4 q = qn;
        if (o + 2 < fe) qn = ld4(sa.fp, sa.fi[o + 2]);
        const float sx = static_cast<float>((q.x - pi.x) * sa.inv_re);
        const float sy = static_cast<float>((q.y - pi.y) * sa.inv_re);
        const float sz = static_cast<float>((q.z - pi.z) * sa.inv_re);
        const float d2 = sx * sx + sy * sy + sz * sz;
        if (d2 > 0.0f) {
          const float w = 1.0f - sqrtf(d2);
          if (w > 0.0f) kahan_monomials(sum, comp, sx, sy, sz, w);
        }
      }
    }
#pragma unroll
    for (int e = 0; e < kMonomials; ++e)
      s_half[half][e][lane] = static_cast<double>(sum[e]) - static_cast<double>(comp[e]);
  }
  __syncthreads();
  if (!live) return;
  double s[kMonomials];
#pragma unroll
  for (int e = 0; e < kMonomials; ++e) s[e] = s_half[0][e][lane] + s_half[1][e][lane];
  mixed_rows_of_particle<Full>(a, half, t, i, pi, s, s_m + threadIdx.x);
}

// make_matrix_request, moment_matrix.cu:494-538: boundary of each kind.
int boundary_of(int kind) {
  switch (kind) {
    case LSMPS_MOMENT_VELOCITY_WALL_DIRICHLET_A: return 1;
    case LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_A: return 2;
    case LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_B: return 2;
    default: return 0;
  }
}

// Queue the two mixed-form stages for the velocity (kv) and pressure (kp)
// Type-A kinds; positions are already packed into ctx->pack_fluid[0] and the
// wall packs.
// The walls' position and normal packs are made here, after the fluid sums
// (for the split kernel before it), once the context's walls_wait_event (a
// host-resident caller's wall copy, lsmps_step only) has been waited for.
lsmps_status launch_mixed(lsmps_ctx* ctx, index_t n, const lsmps_csr& fn, const lsmps_csr& wn,
                          const lsmps_params& p, const KindOut& kv, const KindOut& kp, bool full,
                          const lsmps_walls& walls) {
  if (!ensure_mixed(ctx, static_cast<size_t>(n))) return fail(ctx, LSMPS_CUDA_ERROR, "mixed-form allocation failed");
  const double inv_re = 1.0 / p.support_radius;
  const index_t* srows = sorted_rows_of(ctx, fn, static_cast<size_t>(n));
  const index_t* fi = srows ? srows : fn.indices;
  MixedSumArgs sa{n, ctx->pack_fluid[0], fn.offsets, fi, inv_re, ctx->mixed_sums, ctx->order, srows ? 1 : 0};
  const bool split = ctx->knob[LSMPS_KNOB_MOMENT_OCCUPANCY] == 2;
  MixedRowArgs ra{};
  ra.n = n;
  ra.sums = ctx->mixed_sums;
  ra.fp = ctx->pack_fluid[0];
  ra.wp = ctx->pack_wall[0];
  ra.wn = ctx->pack_wall[2];
  ra.wo = wn.offsets;
  ra.wi = wn.indices;
  ra.inv_re = inv_re;
  ra.lambda = p.lsmps_regularization;
  ra.wall_scale = p.lsmps_wall_weight_scale;
  ra.kappa_threshold = ctx->kappa_threshold;
  ra.k[0] = kv;
  ra.k[1] = kp;
  ra.fo = fn.offsets;
  ra.fi = fi;
  ra.sorted = srows ? 1 : 0;
  for (int k = 0; k < 2; ++k) {
    ra.rows[k] = ctx->mixed_rows[k];
    ra.rows64[k] = ctx->mixed_rows64[k];
    ra.flag[k] = ctx->mixed_flag[k];
    ra.list[k] = ctx->mixed_list[k];
  }
  ra.count = ctx->mixed_count;
  // the lists of FP64-route particles start empty every time
  cudaMemsetAsync(ctx->mixed_count, 0, 4 * sizeof(unsigned int), ctx->stream);
  ra.status = ctx->d_status;
  ra.order = ctx->order;
  auto pack_walls = [&]() {
    if (ctx->walls_wait_event)
      cudaStreamWaitEvent(ctx->stream, static_cast<cudaEvent_t>(ctx->walls_wait_event), 0);
    pack_wall_positions(ctx, walls);
    pack_wall_normals(ctx, walls);
  };
  if (split) {
    pack_walls();
    // one kernel: row halves on two warps, one kind per warp
    if (full)
      launch(ctx, moment_mixed_split_kernel<true>, dim3(div_up(n, kWarp)), dim3(kRowThreads), 0, sa, ra);
    else
      launch(ctx, moment_mixed_split_kernel<false>, dim3(div_up(n, kWarp)), dim3(kRowThreads), 0, sa, ra);
    return LSMPS_OK;
  }
  launch(ctx, moment_sums_kernel, dim3(div_up(n, kSumThreads)), dim3(kSumThreads), 0, sa);
  pack_walls();
  const dim3 grid(div_up(n, kRowThreads), 2);
  if (full)
    launch(ctx, moment_rows_kernel<true>, grid, dim3(kRowThreads), 0, ra);
  else
    launch(ctx, moment_rows_kernel<false>, grid, dim3(kRowThreads), 0, ra);
  return LSMPS_OK;
}

}  // namespace

lsmps_status mixed_step_moments_impl(lsmps_ctx* ctx, const lsmps_fluid& fluid, const lsmps_walls& walls,
                                     const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_params& p,
                                     const lsmps_moment& vm, const lsmps_moment& pm) {
  if (!(p.support_radius > 0.0)) return fail(ctx, LSMPS_INVALID_ARGUMENT, "Moment support radius must be positive");
  if (vm.kind != LSMPS_MOMENT_VELOCITY_WALL_DIRICHLET_A || pm.kind != LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_A ||
      vm.matrix_size != 9 || pm.matrix_size != 9 || vm.particle_count < fluid.count ||
      pm.particle_count < fluid.count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Invalid Moment matrix cache");
  if (fluid.count > fn.particle_count || fluid.count > wn.particle_count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Moment matrix neighbor lists are smaller than fluid particle count");
  const index_t n = static_cast<index_t>(fluid.count);
  if (n == 0) return LSMPS_OK;
  if (const lsmps_status cs = check_neighbor_tables(ctx, fluid.count, walls.count, fn, &wn)) return cs;
  if (!vm.moment_trace || !vm.regularization_added || !vm.info || !pm.moment_trace || !pm.regularization_added ||
      !pm.info)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Invalid Moment matrix cache buffers");
  if (!ensure_packs(ctx, fluid.count, walls.count)) return fail(ctx, LSMPS_CUDA_ERROR, "pack allocation failed");
  pack_fluid_positions(ctx, fluid, sorted_rows_of(ctx, fn, fluid.count) ? ctx->order : nullptr);
  const KindOut kv{1, vm.inverse_matrices, vm.moment_trace, vm.regularization_added, vm.info, vm.inversion_count};
  const KindOut kp{2, pm.inverse_matrices, pm.moment_trace, pm.regularization_added, pm.info, pm.inversion_count};
  lsmps_status st = launch_mixed(ctx, n, fn, wn, p, kv, kp, false, walls);
  if (st) return st;
  return check_launch(ctx, "mixed moment rows");
}

lsmps_status prepare_moments_impl(lsmps_ctx* ctx, const lsmps_fluid& fluid, const lsmps_walls& walls,
                                  const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_params& p,
                                  const lsmps_moment* kinds, int count) {
  if (!(p.support_radius > 0.0)) return fail(ctx, LSMPS_INVALID_ARGUMENT, "Moment support radius must be positive");
  if (p.lsmps_regularization < 0.0) return fail(ctx, LSMPS_INVALID_ARGUMENT, "Moment regularization must be non-negative");
  if (p.lsmps_wall_weight_scale < 0.0)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Moment wall weight scale must be non-negative");
  if (fluid.count > fn.particle_count || fluid.count > wn.particle_count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Moment matrix neighbor lists are smaller than fluid particle count");
  if (count < 0 || !kinds) return fail(ctx, LSMPS_INVALID_ARGUMENT, "moment kinds missing");
  // Group the Type-A kinds (one launch) and the Type-B kinds (one launch each).
  MomentArgs base{};
  base.fluid = fluid;
  base.walls = walls;
  base.fo = fn.offsets;
  base.fi = fn.indices;
  base.wo = wn.offsets;
  base.wi = wn.indices;
  base.re = p.support_radius;
  base.inv_re = 1.0 / p.support_radius;
  base.lambda = p.lsmps_regularization;
  base.wall_scale = p.lsmps_wall_weight_scale;
  base.status = ctx->d_status;
  const index_t n = static_cast<index_t>(fluid.count);
  int velocity_a = -1, pressure_a = -1;
  for (int k = 0; k < count; ++k) {
    const lsmps_moment& mk = kinds[k];
    const bool type_b = mk.kind == LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_B;
    if (mk.kind < 0 || mk.kind > 3) return fail(ctx, LSMPS_INVALID_ARGUMENT, "Unknown Moment matrix kind");
    if (mk.matrix_size != (type_b ? 10 : 9) || mk.particle_count < fluid.count)
      return fail(ctx, LSMPS_INVALID_ARGUMENT, "Invalid Moment matrix cache");
    if (n && (!mk.inverse_matrices || !mk.moment_trace || !mk.regularization_added || !mk.info))
      return fail(ctx, LSMPS_INVALID_ARGUMENT, "Invalid Moment matrix cache buffers");
    if (mk.kind == LSMPS_MOMENT_VELOCITY_WALL_DIRICHLET_A && velocity_a < 0) velocity_a = k;
    if (mk.kind == LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_A && pressure_a < 0) pressure_a = k;
  }
  if (n == 0) return LSMPS_OK;
  if (const lsmps_status cs = check_neighbor_tables(ctx, fluid.count, walls.count, fn, &wn)) return cs;
  auto out_of = [](const lsmps_moment& mk) {
    return KindOut{boundary_of(mk.kind), mk.inverse_matrices, mk.moment_trace, mk.regularization_added, mk.info,
                   mk.inversion_count};
  };
  const dim3 grid(div_up(n, kMomentThreads)), block(kMomentThreads);
  // single-kind launches: the warps' inverse staging (27 x kMomentThreads doubles)
  constexpr size_t kStageBytes = sizeof(double) * 27 * kMomentThreads;
  if (!ensure_packs(ctx, fluid.count, walls.count)) return fail(ctx, LSMPS_CUDA_ERROR, "pack allocation failed");
  const index_t* srows = sorted_rows_of(ctx, fn, fluid.count);
  pack_fluid_positions(ctx, fluid, srows ? ctx->order : nullptr);
  // (the mixed form packs the walls itself, after its fluid sums)
  const bool fused = velocity_a >= 0 && pressure_a >= 0;
  if (!(fused && ctx->precision == LSMPS_PRECISION_MIXED)) {
    pack_wall_positions(ctx, walls);
    pack_wall_normals(ctx, walls);
  }
  MomentPackedArgs pa{n, ctx->pack_fluid[0], ctx->pack_wall[0], ctx->pack_wall[2], fn.offsets,
                      srows ? srows : fn.indices, wn.offsets, wn.indices, base.inv_re, base.lambda,
                      base.wall_scale, KindOut{}, KindOut{}, ctx->d_status, ctx->order, srows ? 1 : 0};
  const bool capped = ctx->knob[LSMPS_KNOB_MOMENT_OCCUPANCY] == 1;
  const bool split = ctx->knob[LSMPS_KNOB_MOMENT_OCCUPANCY] == 2;
  if (fused && ctx->precision == LSMPS_PRECISION_MIXED) {
    // Mixed form: FP32 assembly and factorisation with FP64 refinement; the
    // full inverse is written (FP64) for the caller's views.
    lsmps_status st =
        launch_mixed(ctx, n, fn, wn, p, out_of(kinds[velocity_a]), out_of(kinds[pressure_a]), true, walls);
    if (st) return st;
  } else if (fused) {
    // The step's two kinds share the fluid sums: one pass over the rows.
    MomentPackedArgs a = pa;
    a.k0 = out_of(kinds[velocity_a]);
    a.k1 = out_of(kinds[pressure_a]);
    const size_t smem = sizeof(double) * kMonomials * kMomentThreads;
    if (split)
      launch_named(ctx, "moment_a_split_kernel", moment_a_split_kernel, dim3(div_up(n, kWarp)), dim3(2 * kWarp), 0, a);
    else if (capped)
      launch_named(ctx, "moment_a_kernel<V,P>", moment_a_kernel<1, 2, 8>, grid, block, smem, a);
    else
      launch_named(ctx, "moment_a_kernel<V,P>", moment_a_kernel<1, 2, 1>, grid, block, smem, a);
  }
  for (int k = 0; k < count; ++k) {
    if (fused && (k == velocity_a || k == pressure_a)) continue;
    MomentPackedArgs a = pa;
    a.k0 = out_of(kinds[k]);
    switch (kinds[k].kind) {
      case LSMPS_MOMENT_VELOCITY_WALL_DIRICHLET_A:
        launch_named(ctx, "moment_a_kernel<V>", moment_a_kernel<1, -1, 1>, grid, block, kStageBytes, a);
        break;
      case LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_A:
        launch_named(ctx, "moment_a_kernel<P>", moment_a_kernel<2, -1, 1>, grid, block, kStageBytes, a);
        break;
      case LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_B: {
        MomentArgs b = base;
        b.k0 = a.k0;
        launch_named(ctx, "moment_kernel<B>", moment_kernel<10, 2, -1>, grid, block, 0, b);
        break;
      }
      default:
        launch_named(ctx, "moment_a_kernel<F>", moment_a_kernel<0, -1, 1>, grid, block, kStageBytes, a);
        break;
    }
  }
  return check_launch(ctx, "moment matrices");
}

}  // namespace lsmps

using namespace lsmps;

extern "C" lsmps_status lsmps_prepare_moments(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_walls* walls,
                                              const lsmps_csr* fluid_neighbors, const lsmps_csr* wall_neighbors,
                                              const lsmps_params* params, const lsmps_moment* kinds, int count) {
  if (!ctx || !fluid || !walls || !fluid_neighbors || !wall_neighbors || !params) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  st = prepare_moments_impl(ctx, *fluid, *walls, *fluid_neighbors, *wall_neighbors, *params, kinds, count);
  return end_call(ctx, st);
}
