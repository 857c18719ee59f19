// adjoint.cuh - pieces shared by the two differentiable operator pairs
// (adjoint.cu: fluid-only operators; step_adjoint.cu: the step's operators
// with their wall terms).
#pragma once

#include "common.cuh"

namespace lsmps {

constexpr int kAdjThreads = 128;

// s = d / r_e and the Type-A basis of s (moment_matrix.cu:152-175).
__device__ __forceinline__ void basis_div(double dx, double dy, double dz, double inv_re, double b[9], double s[3]) {
  s[0] = dx * inv_re;
  s[1] = dy * inv_re;
  s[2] = dz * inv_re;
  b[0] = s[0];
  b[1] = s[1];
  b[2] = s[2];
  b[3] = s[0] * s[0];
  b[4] = s[1] * s[1];
  b[5] = s[2] * s[2];
  b[6] = s[0] * s[1];
  b[7] = s[1] * s[2];
  b[8] = s[2] * s[0];
}

__device__ __forceinline__ double dot9(const double* a, const double* b) {
  double v = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) v = fma(a[k], b[k], v);
  return v;
}

// y = X r for the column-major symmetric 9x9 X.
__device__ __forceinline__ void apply(const double* __restrict__ x, const double r[9], double y[9]) {
#pragma unroll
  for (int a = 0; a < 9; ++a) y[a] = 0.0;
#pragma unroll
  for (int c = 0; c < 9; ++c) {
#pragma unroll
    for (int a = 0; a < 9; ++a) y[a] = fma(x[a + c * 9], r[c], y[a]);
  }
}

// J_b(s)^T beta: the derivative of b . beta with respect to s.
__device__ __forceinline__ void basis_jt(const double s[3], const double beta[9], double out[3]) {
  out[0] = beta[0] + 2.0 * s[0] * beta[3] + s[1] * beta[6] + s[2] * beta[8];
  out[1] = beta[1] + 2.0 * s[1] * beta[4] + s[0] * beta[6] + s[2] * beta[7];
  out[2] = beta[2] + 2.0 * s[2] * beta[5] + s[1] * beta[7] + s[0] * beta[8];
}

// The transpose of a CSR table (entries sorted stably by neighbour): the
// entries that list particle j are tsrc[tb[j] .. te[j]) (entry offsets, in
// ascending order; tb[j] = -1 when none), owner[o] the row of entry o.
struct CsrTranspose {
  index_t total;
  index_t* tb;
  index_t* te;
  const index_t* tsrc;
  index_t* owner;
};

// Queues the transpose of fn (its first n rows) on the context's stream, in
// scratch taken from `scratch`; reads the entry count back first.
lsmps_status build_csr_transpose(lsmps_ctx* ctx, Scratch& scratch, const lsmps_csr& fn, index_t n,
                                 CsrTranspose* out);

}  // namespace lsmps
