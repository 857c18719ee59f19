// solve.cu - the PPE solve on the device: restarted GMRES(m) over the PPE CSR
// rows, replacing AmgxPpeSolver::solve (src/ppe/ppe_matrix.cu:586-679).
//
// The reference hands the system to AMGX (a third-party library, linked only
// when found at configure time; no version is pinned in the tree) with
// AMGX's GMRES sample configuration (ppe_matrix.cu:604-610): GMRES, no
// preconditioner, at most 100 iterations, stop when the L2 norm of the
// residual falls to 1e-6 of the initial one (RELATIVE_INI), initial guess
// zero (:625), and clamps negative pressures to zero afterwards (:662).  AMGX
// copies the CSR to the host and back around every solve (:621-661); here
// the matrix stays where the assembly wrote it.
//
// Algorithm: GMRES(m) of Saad and Schultz (1986) with right preconditioning
// (none, or Jacobi: M = diag(A)).  Arnoldi uses classical Gram-Schmidt with
// one re-orthogonalisation (CGS2), so every projection is a batch of
// independent dot products; the Hessenberg column, its Givens rotations and
// the residual estimate |g_{j+1}| are kept on the host.  Each Arnoldi step is
// one SpMV (G lanes per CSR row, the vector read through L2), two batched
// dot-product passes and two update passes over the basis, and one 16-byte
// read-back.  All reductions go through per-block partials summed in a fixed
// order, so a solve is bitwise reproducible.
#include <cmath>
#include <vector>

#include "impl.cuh"

namespace lsmps {
namespace {

constexpr int kSolveThreads = 256;
constexpr int kSpmvLanes = 8;
constexpr int kMaxRestart = 64;

// y = A (s ∘ x) (s = NULL: y = A x); kSpmvLanes lanes per row.
template <int G>
__global__ void __launch_bounds__(kSolveThreads)
    spmv_kernel(index_t n, const index_t* __restrict__ ro, const index_t* __restrict__ ci,
                const double* __restrict__ va, const double* __restrict__ x, const double* __restrict__ s,
                double* __restrict__ y) {
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const index_t row = static_cast<index_t>(t / G);
  const int l = static_cast<int>(t % G);
  if (row >= n) return;  // the whole group
  double acc = 0.0;
  const index_t e = ro[row + 1];
  for (index_t k = ro[row] + l; k < e; k += G) {
    const index_t c = ci[k];
    acc += va[k] * (s ? s[c] * x[c] : x[c]);
  }
  acc = group_sum<G>(acc, group_mask<G>());
  if (l == 0) y[row] = acc;
}

// Per-block partial sums of a block-wide value, written to partial[blockIdx].
__device__ __forceinline__ void block_partial(double v, double* partial_out) {
  __shared__ double red[kSolveThreads / kWarp];
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  if ((threadIdx.x & (kWarp - 1)) == 0) red[threadIdx.x / kWarp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sum = 0.0;
    for (int w = 0; w < kSolveThreads / kWarp; ++w) sum += red[w];
    *partial_out = sum;
  }
}

// partial[k * gridDim.x + bx] = sum over this block's slice of v_k[i] * w[i],
// k = blockIdx.y.  V is [k][ldv].
__global__ void __launch_bounds__(kSolveThreads)
    dots_kernel(index_t n, const double* __restrict__ V, size_t ldv, const double* __restrict__ w,
                double* __restrict__ partial) {
  const double* v = V + blockIdx.y * ldv;
  double acc = 0.0;
  for (index_t i = blockIdx.x * kSolveThreads + threadIdx.x; i < n; i += gridDim.x * kSolveThreads)
    acc += v[i] * w[i];
  block_partial(acc, partial + static_cast<size_t>(blockIdx.y) * gridDim.x + blockIdx.x);
}

// out[k] (+)= sum of partial[k][0..nb) in order; one block per k.
__global__ void __launch_bounds__(kSolveThreads)
    reduce_kernel(const double* __restrict__ partial, int nb, double* __restrict__ out, int accumulate) {
  double acc = 0.0;
  for (int b = threadIdx.x; b < nb; b += kSolveThreads) acc += partial[static_cast<size_t>(blockIdx.x) * nb + b];
  __shared__ double red[kSolveThreads / kWarp];
  for (int d = 16; d > 0; d >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, d);
  if ((threadIdx.x & (kWarp - 1)) == 0) red[threadIdx.x / kWarp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sum = 0.0;
    for (int w = 0; w < kSolveThreads / kWarp; ++w) sum += red[w];
    out[blockIdx.x] = accumulate ? out[blockIdx.x] + sum : sum;
  }
}

// w -= sum_{k<kc} h[k] v_k; partial[bx] = this block's sum of w^2.
__global__ void __launch_bounds__(kSolveThreads)
    update_kernel(index_t n, const double* __restrict__ V, size_t ldv, int kc, const double* __restrict__ h,
                  double* __restrict__ w, double* __restrict__ partial) {
  __shared__ double sh[kMaxRestart + 1];
  for (int k = threadIdx.x; k < kc; k += kSolveThreads) sh[k] = h[k];
  __syncthreads();
  double acc = 0.0;
  for (index_t i = blockIdx.x * kSolveThreads + threadIdx.x; i < n; i += gridDim.x * kSolveThreads) {
    double wi = w[i];
    for (int k = 0; k < kc; ++k) wi -= sh[k] * V[k * ldv + i];
    w[i] = wi;
    acc += wi * wi;
  }
  block_partial(acc, partial + blockIdx.x);
}

// v = w * scale
__global__ void __launch_bounds__(kSolveThreads)
    scale_kernel(index_t n, const double* w, double scale, double* v) {  // v may alias w
  for (index_t i = blockIdx.x * kSolveThreads + threadIdx.x; i < n; i += gridDim.x * kSolveThreads)
    v[i] = w[i] * scale;
}

// x += s ∘ (sum_{k<kc} y[k] v_k)  (s = NULL: no scaling)
__global__ void __launch_bounds__(kSolveThreads)
    correct_kernel(index_t n, const double* __restrict__ V, size_t ldv, int kc, const double* __restrict__ y,
                   const double* __restrict__ s, double* __restrict__ x) {
  __shared__ double sy[kMaxRestart + 1];
  for (int k = threadIdx.x; k < kc; k += kSolveThreads) sy[k] = y[k];
  __syncthreads();
  for (index_t i = blockIdx.x * kSolveThreads + threadIdx.x; i < n; i += gridDim.x * kSolveThreads) {
    double u = 0.0;
    for (int k = 0; k < kc; ++k) u += sy[k] * V[k * ldv + i];
    x[i] += s ? s[i] * u : u;
  }
}

// r = b - Ax (Ax in r on entry), v0 = r; partial[bx] = block sum of r^2.
__global__ void __launch_bounds__(kSolveThreads)
    residual_kernel(index_t n, const double* __restrict__ b, double* __restrict__ r, double* __restrict__ partial) {
  double acc = 0.0;
  for (index_t i = blockIdx.x * kSolveThreads + threadIdx.x; i < n; i += gridDim.x * kSolveThreads) {
    const double ri = b[i] - r[i];
    r[i] = ri;
    acc += ri * ri;
  }
  block_partial(acc, partial + blockIdx.x);
}

// dinv[i] = 1 / a_ii (1 where the row has no non-zero diagonal entry).
__global__ void __launch_bounds__(kSolveThreads)
    jacobi_kernel(index_t n, const index_t* __restrict__ ro, const index_t* __restrict__ ci,
                  const double* __restrict__ va, double* __restrict__ dinv) {
  const index_t i = blockIdx.x * kSolveThreads + threadIdx.x;
  if (i >= n) return;
  double d = 0.0;
  for (index_t k = ro[i]; k < ro[i + 1]; ++k)
    if (ci[k] == i) d += va[k];
  dinv[i] = d != 0.0 ? 1.0 / d : 1.0;
}

// clamp_pressure_kernel, ppe_matrix.cu:373-379
__global__ void __launch_bounds__(kSolveThreads) clamp_kernel(index_t n, double* __restrict__ x) {
  const index_t i = blockIdx.x * kSolveThreads + threadIdx.x;
  if (i < n && x[i] < 0.0) x[i] = 0.0;
}

__global__ void __launch_bounds__(kSolveThreads) zero_kernel(index_t n, double* __restrict__ x) {
  const index_t i = blockIdx.x * kSolveThreads + threadIdx.x;
  if (i < n) x[i] = 0.0;
}

struct Solver {
  lsmps_ctx* ctx;
  index_t n;
  int nb;  // blocks of the streaming passes
  const lsmps_csr_matrix* A;
  const double* dinv;  // NULL without preconditioner
  double* V;
  size_t ldv;
  double* w;
  double* partial;  // [kMaxRestart + 1][nb]
  double* dev_h;    // [2 * (kMaxRestart + 1) + 1]: h (first pass), h (second pass), |w|^2
  double* host;     // pinned mirror of dev_h

  dim3 grid1() const { return dim3(nb); }

  void spmv(const double* x, double* y, bool precondition) {
    launch(ctx, spmv_kernel<kSpmvLanes>, dim3(div_up(static_cast<long long>(n) * kSpmvLanes, kSolveThreads)),
           dim3(kSolveThreads), 0, n, static_cast<const index_t*>(A->row_offsets),
           static_cast<const index_t*>(A->col_indices), static_cast<const double*>(A->values), x,
           precondition ? dinv : static_cast<const double*>(nullptr), y);
  }

  // |r|^2 of r = b - A x into dev_h[0] (and r), synchronously.
  bool residual(const double* b, const double* x, double* r, double& norm2) {
    spmv(x, r, false);
    launch(ctx, residual_kernel, grid1(), dim3(kSolveThreads), 0, n, b, r, partial);
    launch(ctx, reduce_kernel, dim3(1), dim3(kSolveThreads), 0, static_cast<const double*>(partial), nb, dev_h, 0);
    if (!read(1)) return false;
    norm2 = host[0];
    return true;
  }

  bool read(int count) {
    if (cudaMemcpyAsync(host, dev_h, count * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
      return false;
    return cudaStreamSynchronize(ctx->stream) == cudaSuccess;
  }
};

}  // namespace

void solver_options_default(lsmps_solver_options* o) {
  o->max_iters = 100;
  o->restart = 20;
  o->tolerance = 1.0e-6;
  o->convergence = LSMPS_CONVERGENCE_RELATIVE_INITIAL;
  o->preconditioner = LSMPS_PRECONDITIONER_NONE;
  o->clamp_negative = 1;
  o->use_initial_guess = 0;
}

lsmps_status solve_ppe_impl(lsmps_ctx* ctx, const lsmps_csr_matrix& A, const double* b, double* x,
                            const lsmps_solver_options& opt, lsmps_solver_report* report) {
  if (report) *report = lsmps_solver_report{0, 0, 0.0, 0.0};
  if (A.rows == 0) return LSMPS_OK;
  if (const lsmps_status cs = check_table(ctx, A.row_offsets, A.col_indices, A.rows, A.nnz, A.cols,
                                          "PPE matrix: row offset or column index out of range"))
    return cs;
  if (A.rows != A.cols || !A.row_offsets || !A.col_indices || !A.values || !b || !x)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "AMGX PPE solve requires a square CSR matrix, rhs, and solution buffer");
  if (A.rows > static_cast<size_t>(INT32_MAX)) return fail(ctx, LSMPS_INDEX_OVERFLOW, "PPE rows exceed 32-bit indices");
  if (opt.restart < 1 || opt.restart > kMaxRestart || opt.max_iters < 0 || !(opt.tolerance >= 0.0) ||
      (opt.convergence != LSMPS_CONVERGENCE_RELATIVE_INITIAL && opt.convergence != LSMPS_CONVERGENCE_ABSOLUTE) ||
      (opt.preconditioner != LSMPS_PRECONDITIONER_NONE && opt.preconditioner != LSMPS_PRECONDITIONER_JACOBI))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "invalid PPE solver options");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(ctx->stream, &cap);
  if (cap != cudaStreamCaptureStatusNone)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "the PPE solve reads residuals back and cannot be captured");

  const index_t n = static_cast<index_t>(A.rows);
  const int m = opt.restart;
  const int nb = static_cast<int>(std::min<long long>(div_up(static_cast<long long>(n), kSolveThreads),
                                                      4LL * ctx->sm_count));
  const size_t ldv = (static_cast<size_t>(n) + 31) & ~size_t(31);
  Scratch scratch(ctx);
  const size_t need = (static_cast<size_t>(m + 1) * ldv + 2 * ldv) * sizeof(double) +
                      static_cast<size_t>(kMaxRestart + 1) * nb * sizeof(double) +
                      (2 * (kMaxRestart + 1) + 8) * sizeof(double) + 16 * 256;
  if (!scratch.reserve(need)) return fail(ctx, LSMPS_CUDA_ERROR, "scratch allocation failed");
  Solver s{};
  s.ctx = ctx;
  s.n = n;
  s.nb = nb;
  s.A = &A;
  s.ldv = ldv;
  s.V = scratch.take<double>(static_cast<size_t>(m + 1) * ldv);
  s.w = scratch.take<double>(ldv);
  double* dinv = scratch.take<double>(ldv);
  s.partial = scratch.take<double>(static_cast<size_t>(kMaxRestart + 1) * nb);
  s.dev_h = scratch.take<double>(2 * (kMaxRestart + 1) + 8);
  if (!s.V || !s.w || !dinv || !s.partial || !s.dev_h) return fail(ctx, LSMPS_CUDA_ERROR, "scratch exhausted");
  static thread_local double* pinned = nullptr;
  if (!pinned && cudaMallocHost(&pinned, (2 * (kMaxRestart + 1) + 8) * sizeof(double)) != cudaSuccess) {
    pinned = nullptr;
    return fail(ctx, LSMPS_CUDA_ERROR, "pinned allocation failed");
  }
  s.host = pinned;
  const bool jacobi = opt.preconditioner == LSMPS_PRECONDITIONER_JACOBI;
  if (jacobi) {
    launch(ctx, jacobi_kernel, dim3(div_up(n, kSolveThreads)), dim3(kSolveThreads), 0, n,
           static_cast<const index_t*>(A.row_offsets), static_cast<const index_t*>(A.col_indices),
           static_cast<const double*>(A.values), dinv);
    s.dinv = dinv;
  }
  if (!opt.use_initial_guess) launch(ctx, zero_kernel, dim3(div_up(n, kSolveThreads)), dim3(kSolveThreads), 0, n, x);

  // r0 = b - A x0 in V[0]
  double beta2 = 0.0;
  if (!s.residual(b, x, s.V, beta2)) return check_launch(ctx, "PPE solve");
  const double beta0 = std::sqrt(beta2);
  const double target = opt.convergence == LSMPS_CONVERGENCE_RELATIVE_INITIAL ? opt.tolerance * beta0 : opt.tolerance;
  double beta = beta0;
  int iters = 0;
  bool converged = beta <= target;
  std::vector<double> H(static_cast<size_t>(m + 1) * m), cs(m), sn(m), g(m + 1), y(m + 1);
  while (!converged && iters < opt.max_iters) {
    // V[0] = r / beta
    launch(ctx, scale_kernel, s.grid1(), dim3(kSolveThreads), 0, n, static_cast<const double*>(s.V), 1.0 / beta, s.V);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j = 0;
    for (; j < m && iters < opt.max_iters; ++j) {
      double* vj = s.V + static_cast<size_t>(j) * ldv;
      s.spmv(vj, s.w, jacobi);
      const int kc = j + 1;
      // CGS2: two passes of h = V^T w, w -= V h; the second pass also gives |w|^2.
      for (int pass = 0; pass < 2; ++pass) {
        double* hp = s.dev_h + pass * (kMaxRestart + 1);
        launch(ctx, dots_kernel, dim3(nb, kc), dim3(kSolveThreads), 0, n, static_cast<const double*>(s.V), ldv,
               static_cast<const double*>(s.w), s.partial);
        launch(ctx, reduce_kernel, dim3(kc), dim3(kSolveThreads), 0, static_cast<const double*>(s.partial), nb, hp, 0);
        launch(ctx, update_kernel, s.grid1(), dim3(kSolveThreads), 0, n, static_cast<const double*>(s.V), ldv, kc,
               static_cast<const double*>(hp), s.w, s.partial);
      }
      launch(ctx, reduce_kernel, dim3(1), dim3(kSolveThreads), 0, static_cast<const double*>(s.partial), nb,
             s.dev_h + 2 * (kMaxRestart + 1), 0);
      if (cudaMemcpyAsync(s.host, s.dev_h, (2 * (kMaxRestart + 1) + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                          ctx->stream) != cudaSuccess ||
          cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return check_launch(ctx, "PPE solve");
      ++iters;
      double* col = &H[static_cast<size_t>(j) * (m + 1)];
      for (int k = 0; k <= j; ++k) col[k] = s.host[k] + s.host[kMaxRestart + 1 + k];
      const double hnext = std::sqrt(s.host[2 * (kMaxRestart + 1)]);
      col[j + 1] = hnext;
      // previous rotations, then the one that zeroes col[j + 1]
      for (int k = 0; k < j; ++k) {
        const double t = cs[k] * col[k] + sn[k] * col[k + 1];
        col[k + 1] = -sn[k] * col[k] + cs[k] * col[k + 1];
        col[k] = t;
      }
      const double den = std::hypot(col[j], col[j + 1]);
      cs[j] = den > 0.0 ? col[j] / den : 1.0;
      sn[j] = den > 0.0 ? col[j + 1] / den : 0.0;
      col[j] = den;
      col[j + 1] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      const double estimate = std::fabs(g[j + 1]);
      // hnext == 0: the Krylov space is invariant (the update below solves
      // the system on it); stop the cycle there.
      if (estimate <= target || hnext == 0.0) {
        ++j;
        break;
      }
      if (j + 1 < m && iters < opt.max_iters)
        launch(ctx, scale_kernel, s.grid1(), dim3(kSolveThreads), 0, n, static_cast<const double*>(s.w),
               1.0 / hnext, s.V + static_cast<size_t>(j + 1) * ldv);
    }
    // y = R^-1 g (back substitution on the rotated Hessenberg), x += M^-1 V y
    for (int k = j - 1; k >= 0; --k) {
      double t = g[k];
      for (int c = k + 1; c < j; ++c) t -= H[static_cast<size_t>(c) * (m + 1) + k] * y[c];
      const double d = H[static_cast<size_t>(k) * (m + 1) + k];
      y[k] = d != 0.0 ? t / d : 0.0;
    }
    for (int k = 0; k < j; ++k) s.host[k] = y[k];
    if (cudaMemcpyAsync(s.dev_h, s.host, j * sizeof(double), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
      return check_launch(ctx, "PPE solve");
    launch(ctx, correct_kernel, s.grid1(), dim3(kSolveThreads), 0, n, static_cast<const double*>(s.V), ldv, j,
           static_cast<const double*>(s.dev_h), static_cast<const double*>(s.dinv), x);
    // true residual for the next cycle (and the report)
    if (!s.residual(b, x, s.V, beta2)) return check_launch(ctx, "PPE solve");
    beta = std::sqrt(beta2);
    converged = beta <= target;
  }
  if (opt.clamp_negative) launch(ctx, clamp_kernel, dim3(div_up(n, kSolveThreads)), dim3(kSolveThreads), 0, n, x);
  if (report) *report = lsmps_solver_report{iters, converged ? 1 : 0, beta0, beta};
  return check_launch(ctx, "PPE solve");
}

}  // namespace lsmps

using namespace lsmps;

extern "C" void lsmps_solver_options_default(lsmps_solver_options* options) {
  if (options) solver_options_default(options);
}

extern "C" lsmps_status lsmps_solve_ppe(lsmps_ctx* ctx, const lsmps_csr_matrix* matrix, const double* rhs,
                                        double* pressure, const lsmps_solver_options* options,
                                        lsmps_solver_report* report) {
  if (!ctx || !matrix) return LSMPS_INVALID_ARGUMENT;
  lsmps_solver_options opt;
  solver_options_default(&opt);
  if (options) opt = *options;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  st = solve_ppe_impl(ctx, *matrix, rhs, pressure, opt, report);
  return end_call(ctx, st);
}
