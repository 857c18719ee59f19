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

#include "impl.cuh"

namespace lsmps {
namespace {

constexpr int kMomentThreads = 64;
constexpr int kMaxKinds = 3;

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
template <int N, int J>
__device__ __forceinline__ void cholesky_column(double (&a)[N * (N + 1) / 2], int& info) {
  double s = a[tri(J, J)];
#pragma unroll
  for (int k = 0; k < J; ++k) s = fma(-a[tri(J, k)], a[tri(J, k)], s);
  if (!(s > 0.0) && info == 0) info = J + 1;
  const double ljj = sqrt(s);
  a[tri(J, J)] = ljj;
  const double inv = 1.0 / ljj;
#pragma unroll
  for (int i = J + 1; i < N; ++i) {
    double t = a[tri(i, J)];
#pragma unroll
    for (int k = 0; k < J; ++k) t = fma(-a[tri(i, k)], a[tri(J, k)], t);
    a[tri(i, J)] = t * inv;
  }
}

template <int N, int... J>
__device__ __forceinline__ void cholesky_columns(double (&a)[N * (N + 1) / 2], int& info,
                                                 std::integer_sequence<int, J...>) {
  (cholesky_column<N, J>(a, info), ...);
}

// Lower Cholesky in place; returns 0 or the 1-based order of the first
// non-positive pivot (the potrf info convention).
template <int N>
__device__ __forceinline__ int cholesky(double (&a)[N * (N + 1) / 2]) {
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

// Adds the wall term of boundary kind B (0 none, 1 Dirichlet sample,
// 2 pressure Neumann) to m, regularises, inverts and stores one kind.
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

// make_matrix_request, moment_matrix.cu:494-538: boundary of each kind.
int boundary_of(int kind) {
  switch (kind) {
    case LSMPS_MOMENT_VELOCITY_WALL_DIRICHLET_A: return 1;
    case LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_A: return 2;
    case LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_B: return 2;
    default: return 0;
  }
}

}  // namespace

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
  auto out_of = [](const lsmps_moment& mk) {
    return KindOut{boundary_of(mk.kind), mk.inverse_matrices, mk.moment_trace, mk.regularization_added, mk.info,
                   mk.inversion_count};
  };
  const dim3 grid(div_up(n, kMomentThreads)), block(kMomentThreads);
  const bool fused = velocity_a >= 0 && pressure_a >= 0;
  if (fused) {
    // The step's two kinds share the fluid sum: one pass over the rows.
    MomentArgs a = base;
    a.k0 = out_of(kinds[velocity_a]);
    a.k1 = out_of(kinds[pressure_a]);
    launch(ctx, moment_kernel<9, 1, 2>, grid, block, sizeof(double) * 45 * kMomentThreads, a);
  }
  for (int k = 0; k < count; ++k) {
    if (fused && (k == velocity_a || k == pressure_a)) continue;
    MomentArgs a = base;
    a.k0 = out_of(kinds[k]);
    switch (kinds[k].kind) {
      case LSMPS_MOMENT_VELOCITY_WALL_DIRICHLET_A: launch(ctx, moment_kernel<9, 1, -1>, grid, block, 0, a); break;
      case LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_A: launch(ctx, moment_kernel<9, 2, -1>, grid, block, 0, a); break;
      case LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_B: launch(ctx, moment_kernel<10, 2, -1>, grid, block, 0, a); break;
      default: launch(ctx, moment_kernel<9, 0, -1>, grid, block, 0, a); break;
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
