// adjoint.cu - the LSMPS field operators and the fluid-only PPE rows as a
// forward/backward pair (no counterpart in the reference, which has no
// derivatives).
//
// Per fluid particle i over its fluid CSR row N(i), with s_ij = (x_j - x_i)/r_e,
// w_ij = 1 - |s_ij|, b_ij the Type-A basis (moment_matrix.cu:152-175) and the
// fluid-only Type-A moment matrix M_i = sum_j w_ij b_ij b_ij^T + reg_i I
// (moment_matrix.cu:254-309 with no wall term; reg_i = lambda tr/9):
//   R_i(phi) = sum_j w_ij b_ij (phi_j - phi_i),  y_i(phi) = M_i^-1 R_i(phi)
//   gradient    g_i   = y_i(f)[0..2] / r_e                (pressure_correction.cu:226-266)
//   Laplacian   lap_i = 2 / r_e^2 sum_{r=3..5} y_i(f)[r]    (explicit_update.cu:164-176)
//   divergence  div_i = sum_c y_i(v_c)[c] / r_e             (ppe_matrix.cu:355-361)
//   PPE row i   a_ij = 2 w_ij (l_i . b_ij) / (r_e^2 rho), l_i = sum_{r=3..5} M_i^-1[r, :],
//               diagonal -sum_j a_ij first, rhs_i = div_i / dt (ppe_matrix.cu:243-370
//               without the wall terms)
//
// Backward, for a loss L with cotangents of every output:
//   ybar_i(phi) is the cotangent of y_i(phi), Rbar_i(phi) = M_i^-1 ybar_i(phi)
//   (M symmetric), and for the PPE rows h_i = c sum_j abar_ij w_ij b_ij,
//   hhat_i = M_i^-1 h_i (abar_ij = the off-diagonal cotangent minus the
//   diagonal's).  Field cotangents: phibar_j += w_ij b_ij . Rbar_i(phi),
//   phibar_i -= the same.  Position cotangents: with d = x_j - x_i,
//   dL = alpha_ij dw_ij + beta_ij . db_ij, where
//     alpha = sum_phi (Rbar.b)(dphi - b.y) + c abar (l.b) - (hhat.b)(b.l)
//             - rho (lambda/9) |b|^2
//     beta  = w sum_phi [Rbar (dphi - b.y) - (Rbar.b) y] + c abar w l
//             - w [(b.l) hhat + (hhat.b) l] - rho (lambda/9) 2 w b
//   (rho = sum_phi Rbar.y + hhat.l; the lambda terms only when tr > 0), and
//   dL/dd = (-alpha d/|d| + J_b(s)^T beta) / r_e is added to xbar_j and
//   subtracted from xbar_i.
//
// The backward recomputes M_i^-1 from the positions (no stored inverse is
// needed) unless the caller passes the inverse the forward wrote.
//
// Each CSR entry (i, j) contributes to the cotangents of both its owner i and
// its neighbour j.  The default backward is deterministic: after the
// per-particle stash pass it builds the transpose of the CSR (entries sorted
// stably by neighbour, so each particle's incoming entries are in ascending
// entry order) and every particle gathers its own row's terms and its
// incoming entries' terms in a fixed order, with no atomics: repeated runs
// give the same bits.  lsmps_ctx_set_adjoint_atomic(ctx, 1) selects the
// scatter form instead (FP64 atomics into the neighbours; no transpose, but
// the result depends on the atomics' order at the rounding level).
#include <algorithm>

#include "adjoint.cuh"
#include "cells.cuh"
#include "impl.cuh"
#include "packed.cuh"

namespace lsmps {
namespace {

constexpr int kThreads = 128;
constexpr int kStash = 92;  // Rbar(4x9) y(4x9) hhat(9) l(9) rho flag

struct OpsArgs {
  index_t n;
  const double4* fp;
  const index_t* fo;
  const index_t* fi;
  const double* f;
  const double* vx;
  const double* vy;
  const double* vz;
  const double* inv;  // [n][81] column-major
  double re;
  double inv_re;
  double ppe_scale;  // 2 / (r_e^2 rho)
  double inv_dt;
  double lambda;
  lsmps_operator_out out;
  lsmps_operator_out bar;  // backward: cotangents
  double* stash;
  double* fbar;
  double* vbar[3];
  double* xbar[3];
};

__device__ __forceinline__ double opt(const double* p, index_t i) { return p ? p[i] : 0.0; }

__global__ void __launch_bounds__(kThreads) ops_forward_kernel(OpsArgs a) {
  const index_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double4 pi = ld4(a.fp, i);
  const double* __restrict__ x = a.inv + static_cast<size_t>(i) * 81;
  const double fi_ = a.f[i], vxi = a.vx[i], vyi = a.vy[i], vzi = a.vz[i];
  const bool ppe = a.out.ppe_values != nullptr;
  double l[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) l[c] = x[3 + c * 9] + x[4 + c * 9] + x[5 + c * 9];
  double rf[9], rx[9], ry[9], rz[9], b[9], s[3];
#pragma unroll
  for (int k = 0; k < 9; ++k) rf[k] = rx[k] = ry[k] = rz[k] = 0.0;
  const index_t nb = a.fo[i], ne = a.fo[i + 1];
  const index_t row = i + nb;
  double diag = 0.0;
  for (index_t o = nb; o < ne; ++o) {
    const index_t j = a.fi[o];
    const double4 q = ld4(a.fp, j);
    const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
    const double w = lin_weight(sqrt(dx * dx + dy * dy + dz * dz), a.re);
    double coef = 0.0;
    if (w > 0.0) {
      basis_div(dx, dy, dz, a.inv_re, b, s);
      const double df = a.f[j] - fi_, dvx = a.vx[j] - vxi, dvy = a.vy[j] - vyi, dvz = a.vz[j] - vzi;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const double wb = w * b[k];
        rf[k] = fma(wb, df, rf[k]);
        rx[k] = fma(wb, dvx, rx[k]);
        ry[k] = fma(wb, dvy, ry[k]);
        rz[k] = fma(wb, dvz, rz[k]);
      }
      if (ppe) {
        coef = a.ppe_scale * w * dot9(l, b);
        diag -= coef;
      }
    }
    if (ppe) {
      a.out.ppe_col_indices[row + 1 + o - nb] = j;
      a.out.ppe_values[row + 1 + o - nb] = coef;
    }
  }
  double y[9];
  apply(x, rf, y);
  if (a.out.grad_x) {
    a.out.grad_x[i] = y[0] * a.inv_re;
    a.out.grad_y[i] = y[1] * a.inv_re;
    a.out.grad_z[i] = y[2] * a.inv_re;
  }
  if (a.out.laplacian) a.out.laplacian[i] = 2.0 * (y[3] + y[4] + y[5]) * a.inv_re * a.inv_re;
  double div = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    div = fma(x[0 + k * 9], rx[k], div);
    div = fma(x[1 + k * 9], ry[k], div);
    div = fma(x[2 + k * 9], rz[k], div);
  }
  div *= a.inv_re;
  if (a.out.divergence) a.out.divergence[i] = div;
  if (ppe) {
    a.out.ppe_row_offsets[i] = row;
    if (i + 1 == a.n) a.out.ppe_row_offsets[a.n] = a.n + ne;
    a.out.ppe_col_indices[row] = i;
    a.out.ppe_values[row] = diag;
    if (a.out.ppe_rhs) a.out.ppe_rhs[i] = div * a.inv_dt;
  }
}

// Per-particle backward quantities (the stash): Rbar and y of the four
// fields, hhat and l of the PPE rows, rho and whether tr > 0.
__global__ void __launch_bounds__(kThreads) ops_adjoint_rows_kernel(OpsArgs a) {
  const index_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double4 pi = ld4(a.fp, i);
  const double* __restrict__ x = a.inv + static_cast<size_t>(i) * 81;
  const double fi_ = a.f[i], vxi = a.vx[i], vyi = a.vy[i], vzi = a.vz[i];
  double* st = a.stash + static_cast<size_t>(i) * kStash;
  const bool ppe = a.bar.ppe_values != nullptr;
  const index_t nb = a.fo[i], ne = a.fo[i + 1];
  const index_t row = i + nb;
  const double diag_bar = ppe ? a.bar.ppe_values[row] : 0.0;
  double rf[9], rx[9], ry[9], rz[9], h[9], b[9], s[3];
#pragma unroll
  for (int k = 0; k < 9; ++k) rf[k] = rx[k] = ry[k] = rz[k] = h[k] = 0.0;
  double trace = 0.0;  // of the fluid sum, before regularisation
  for (index_t o = nb; o < ne; ++o) {
    const index_t j = a.fi[o];
    const double4 q = ld4(a.fp, j);
    const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
    const double w = lin_weight(sqrt(dx * dx + dy * dy + dz * dz), a.re);
    if (w <= 0.0) continue;
    basis_div(dx, dy, dz, a.inv_re, b, s);
    trace = fma(w, dot9(b, b), trace);
    const double df = a.f[j] - fi_, dvx = a.vx[j] - vxi, dvy = a.vy[j] - vyi, dvz = a.vz[j] - vzi;
    const double ab = ppe ? a.ppe_scale * (a.bar.ppe_values[row + 1 + o - nb] - diag_bar) : 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const double wb = w * b[k];
      rf[k] = fma(wb, df, rf[k]);
      rx[k] = fma(wb, dvx, rx[k]);
      ry[k] = fma(wb, dvy, ry[k]);
      rz[k] = fma(wb, dvz, rz[k]);
      h[k] = fma(wb, ab, h[k]);
    }
  }
  double t[9], u[9];
  // y of the four fields, stored at 36..71
  apply(x, rf, u);
#pragma unroll
  for (int k = 0; k < 9; ++k) st[36 + k] = u[k];
  double rho = 0.0;
  // cotangent of y(f): gradient rows 0..2, Laplacian rows 3..5
  const double lapb = 2.0 * opt(a.bar.laplacian, i) * a.inv_re * a.inv_re;
  t[0] = opt(a.bar.grad_x, i) * a.inv_re;
  t[1] = opt(a.bar.grad_y, i) * a.inv_re;
  t[2] = opt(a.bar.grad_z, i) * a.inv_re;
  t[3] = t[4] = t[5] = lapb;
  t[6] = t[7] = t[8] = 0.0;
  double rb[9];
  apply(x, t, rb);
#pragma unroll
  for (int k = 0; k < 9; ++k) st[k] = rb[k];
  rho += dot9(rb, u);
  // divergence (and PPE rhs = div / dt): cotangent (dbar / r_e) e_c of y(v_c)
  const double dbar = (opt(a.bar.divergence, i) + opt(a.bar.ppe_rhs, i) * a.inv_dt) * a.inv_re;
  const double* rv[3] = {rx, ry, rz};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    apply(x, rv[c], u);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      rb[k] = dbar * x[k + c * 9];  // Rbar = M^-1 (dbar e_c) = dbar * column c
      st[9 * (c + 1) + k] = rb[k];
      st[36 + 9 * (c + 1) + k] = u[k];
    }
    rho += dot9(rb, u);
  }
  // PPE rows: hhat = M^-1 h, l = sum of rows 3..5
  apply(x, h, u);
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double lk = x[3 + k * 9] + x[4 + k * 9] + x[5 + k * 9];
    st[72 + k] = u[k];
    st[81 + k] = lk;
    rho = fma(u[k], lk, rho);
  }
  st[90] = rho;
  st[91] = trace > 0.0 ? 1.0 : 0.0;
}

// Terms of one CSR entry of owner i (stash st, position pi, field values
// phii) with neighbour j: tphi[p] is added to phibar_p[j] and taken from
// phibar_p[i], g is added to xbar[j] and taken from xbar[i].  ab is the
// entry's PPE cotangent (c (abar_ij - abar_ii)), rho_reg the owner's
// regularisation factor.  False for an entry with zero weight or distance.
__device__ __forceinline__ bool pair_terms(const OpsArgs& a, const double* __restrict__ st, const double4& pi,
                                           const double phii[4], index_t j, double ab, double rho_reg,
                                           double tphi[4], double g[3]) {
  const double4 q = ld4(a.fp, j);
  const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
  const double dist = sqrt(dx * dx + dy * dy + dz * dz);
  const double w = lin_weight(dist, a.re);
  if (w <= 0.0 || dist <= 0.0) return false;
  double b[9], s[3], beta[9];
  basis_div(dx, dy, dz, a.inv_re, b, s);
  double alpha = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) beta[k] = 0.0;
  const double* phi[4] = {a.f, a.vx, a.vy, a.vz};
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const double* rb = st + 9 * p;
    const double* y = st + 36 + 9 * p;
    const double rbb = dot9(rb, b);
    const double e = (phi[p][j] - phii[p]) - dot9(b, y);
    alpha = fma(rbb, e, alpha);
#pragma unroll
    for (int k = 0; k < 9; ++k) beta[k] = fma(w, rb[k] * e - rbb * y[k], beta[k]);
    tphi[p] = w * rbb;
  }
  if (a.bar.ppe_values != nullptr) {
    const double* hh = st + 72;
    const double* l = st + 81;
    const double lb = dot9(l, b), hb = dot9(hh, b);
    alpha += ab * lb - hb * lb;
#pragma unroll
    for (int k = 0; k < 9; ++k) beta[k] += ab * w * l[k] - w * (lb * hh[k] + hb * l[k]);
  }
  if (rho_reg != 0.0) {
    alpha -= rho_reg * dot9(b, b);
#pragma unroll
    for (int k = 0; k < 9; ++k) beta[k] -= rho_reg * 2.0 * w * b[k];
  }
  // dL/dd = (-alpha d/|d| + J_b(s)^T beta) / r_e
  const double inv_d = 1.0 / dist;
  g[0] = (-alpha * dx * inv_d + beta[0] + 2.0 * s[0] * beta[3] + s[1] * beta[6] + s[2] * beta[8]) * a.inv_re;
  g[1] = (-alpha * dy * inv_d + beta[1] + 2.0 * s[1] * beta[4] + s[0] * beta[6] + s[2] * beta[7]) * a.inv_re;
  g[2] = (-alpha * dz * inv_d + beta[2] + 2.0 * s[2] * beta[5] + s[1] * beta[7] + s[0] * beta[8]) * a.inv_re;
  return true;
}

// The owner-side quantities of particle i that pair_terms needs.
struct OwnerTerms {
  double4 pi;
  const double* st;
  double phii[4];
  index_t nb;
  index_t row;
  double diag_bar;
  double rho_reg;
};

__device__ __forceinline__ OwnerTerms owner_terms(const OpsArgs& a, index_t i) {
  OwnerTerms t;
  t.pi = ld4(a.fp, i);
  t.st = a.stash + static_cast<size_t>(i) * kStash;
  t.phii[0] = a.f[i];
  t.phii[1] = a.vx[i];
  t.phii[2] = a.vy[i];
  t.phii[3] = a.vz[i];
  t.nb = a.fo[i];
  t.row = i + t.nb;
  t.diag_bar = a.bar.ppe_values != nullptr ? a.bar.ppe_values[t.row] : 0.0;
  t.rho_reg = t.st[91] != 0.0 ? t.st[90] * a.lambda / 9.0 : 0.0;
  return t;
}

// PPE cotangent of entry o of the owner's row.
__device__ __forceinline__ double entry_ab(const OpsArgs& a, const OwnerTerms& t, index_t o) {
  return a.bar.ppe_values != nullptr ? a.ppe_scale * (a.bar.ppe_values[t.row + 1 + o - t.nb] - t.diag_bar) : 0.0;
}

// Scatter form (lsmps_ctx_set_adjoint_atomic): each owner adds its entries'
// terms into its neighbours with FP64 atomics.
__global__ void __launch_bounds__(kThreads) ops_adjoint_scatter_kernel(OpsArgs a) {
  const index_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const OwnerTerms t = owner_terms(a, i);
  double* phibar[4] = {a.fbar, a.vbar[0], a.vbar[1], a.vbar[2]};
  const index_t ne = a.fo[i + 1];
  double own_x = 0.0, own_y = 0.0, own_z = 0.0;
  double own_phi[4] = {0.0, 0.0, 0.0, 0.0};
  for (index_t o = t.nb; o < ne; ++o) {
    const index_t j = a.fi[o];
    double tphi[4], g[3];
    if (!pair_terms(a, t.st, t.pi, t.phii, j, entry_ab(a, t, o), t.rho_reg, tphi, g)) continue;
#pragma unroll
    for (int p = 0; p < 4; ++p)
      if (phibar[p]) {
        atomicAdd(&phibar[p][j], tphi[p]);
        own_phi[p] -= tphi[p];
      }
    if (a.xbar[0]) {
      atomicAdd(&a.xbar[0][j], g[0]);
      atomicAdd(&a.xbar[1][j], g[1]);
      atomicAdd(&a.xbar[2][j], g[2]);
    }
    own_x -= g[0];
    own_y -= g[1];
    own_z -= g[2];
  }
  if (a.xbar[0]) {
    atomicAdd(&a.xbar[0][i], own_x);
    atomicAdd(&a.xbar[1][i], own_y);
    atomicAdd(&a.xbar[2][i], own_z);
  }
#pragma unroll
  for (int p = 0; p < 4; ++p)
    if (phibar[p]) atomicAdd(&phibar[p][i], own_phi[p]);
}

// Deterministic form: particle j sums, in a fixed order, the terms of its
// incoming entries (the transpose row [tb[j], te[j]) of entry offsets,
// ascending) and then subtracts those of its own row, and writes its
// cotangents (no atomics, no accumulation into the outputs).
__global__ void __launch_bounds__(kThreads) ops_adjoint_gather_kernel(OpsArgs a, const index_t* __restrict__ tb,
                                                                      const index_t* __restrict__ te,
                                                                      const index_t* __restrict__ tsrc,
                                                                      const index_t* __restrict__ owner) {
  const index_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  double acc_phi[4] = {0.0, 0.0, 0.0, 0.0};
  double acc_x = 0.0, acc_y = 0.0, acc_z = 0.0;
  const index_t b0 = tb[j], e0 = te[j];
  if (b0 >= 0) {
    for (index_t k = b0; k < e0; ++k) {
      const index_t o = tsrc[k];
      const OwnerTerms t = owner_terms(a, owner[o]);
      double tphi[4], g[3];
      if (!pair_terms(a, t.st, t.pi, t.phii, j, entry_ab(a, t, o), t.rho_reg, tphi, g)) continue;
#pragma unroll
      for (int p = 0; p < 4; ++p) acc_phi[p] += tphi[p];
      acc_x += g[0];
      acc_y += g[1];
      acc_z += g[2];
    }
  }
  const OwnerTerms t = owner_terms(a, j);
  const index_t ne = a.fo[j + 1];
  for (index_t o = t.nb; o < ne; ++o) {
    double tphi[4], g[3];
    if (!pair_terms(a, t.st, t.pi, t.phii, a.fi[o], entry_ab(a, t, o), t.rho_reg, tphi, g)) continue;
#pragma unroll
    for (int p = 0; p < 4; ++p) acc_phi[p] -= tphi[p];
    acc_x -= g[0];
    acc_y -= g[1];
    acc_z -= g[2];
  }
  double* phibar[4] = {a.fbar, a.vbar[0], a.vbar[1], a.vbar[2]};
#pragma unroll
  for (int p = 0; p < 4; ++p)
    if (phibar[p]) phibar[p][j] = acc_phi[p];
  if (a.xbar[0]) {
    a.xbar[0][j] = acc_x;
    a.xbar[1][j] = acc_y;
    a.xbar[2][j] = acc_z;
  }
}

}  // namespace

// Transpose of the CSR, step 1: for every entry o of row i, key = its
// neighbour (indices outside [0, n) become the sentinel n), value = o, and
// owner[o] = i.  Eight lanes per row.
__global__ void __launch_bounds__(kAdjThreads) transpose_keys_kernel(const index_t* __restrict__ fo,
                                                                  const index_t* __restrict__ fi, index_t n,
                                                                  index_t* __restrict__ keys,
                                                                  index_t* __restrict__ vals,
                                                                  index_t* __restrict__ owner) {
  const index_t i = static_cast<index_t>((static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) / 8);
  const int lane = threadIdx.x & 7;
  if (i >= n) return;
  const index_t ne = fo[i + 1];
  for (index_t o = fo[i] + lane; o < ne; o += 8) {
    const index_t j = fi[o];
    keys[o] = (j >= 0 && j < n) ? j : n;
    vals[o] = o;
    owner[o] = i;
  }
}

lsmps_status build_csr_transpose(lsmps_ctx* ctx, Scratch& scratch, const lsmps_csr& fn, index_t n,
                                 CsrTranspose* out) {
  index_t total = 0;
  if (cudaMemcpyAsync(&total, fn.offsets + n, sizeof(index_t), cudaMemcpyDeviceToHost, ctx->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    return fail(ctx, LSMPS_CUDA_ERROR, "reading the neighbour count failed");
  if (total < 0 || static_cast<size_t>(total) > fn.neighbor_count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "neighbour table offsets exceed its capacity");
  const size_t k = static_cast<size_t>(total);
  const int tiles = total ? div_up(total, kSortTile) : 0;
  const size_t hist_entries = static_cast<size_t>(tiles) * kRadixBins;
  const size_t bytes = 5 * (k * sizeof(index_t) + 256) + 2 * ((n + 1) * sizeof(index_t) + 256) +
                       hist_entries * sizeof(index_t) + 256 + 4 * scan_scratch_bytes(hist_entries + 1) + 4096;
  if (!scratch.reserve(bytes)) return fail(ctx, LSMPS_CUDA_ERROR, "CSR transpose scratch allocation failed");
  index_t* keys = scratch.take<index_t>(k + 1);
  index_t* vals = scratch.take<index_t>(k + 1);
  index_t* alt_keys = scratch.take<index_t>(k + 1);
  index_t* alt_vals = scratch.take<index_t>(k + 1);
  index_t* owner = scratch.take<index_t>(k + 1);
  index_t* tb = scratch.take<index_t>(static_cast<size_t>(n) + 1);
  index_t* te = scratch.take<index_t>(static_cast<size_t>(n) + 1);
  index_t* hist = scratch.take<index_t>(hist_entries + 1);
  if (!keys || !vals || !alt_keys || !alt_vals || !owner || !tb || !te || !hist)
    return fail(ctx, LSMPS_CUDA_ERROR, "CSR transpose scratch exhausted");
  cudaMemsetAsync(tb, 0xff, (static_cast<size_t>(n) + 1) * sizeof(index_t), ctx->stream);
  cudaMemsetAsync(te, 0xff, (static_cast<size_t>(n) + 1) * sizeof(index_t), ctx->stream);
  out->total = total;
  out->tb = tb;
  out->te = te;
  out->tsrc = vals;
  out->owner = owner;
  if (total == 0) return check_launch(ctx, "CSR transpose");
  launch(ctx, transpose_keys_kernel, dim3(div_up(static_cast<long long>(n) * 8, kAdjThreads)), dim3(kAdjThreads),
         0, fn.offsets, fn.indices, n, keys, vals, owner);
  const int passes = (key_bits(static_cast<long long>(n) + 1) + kRadixBits - 1) / kRadixBits;
  index_t *k0 = keys, *v0 = vals, *k1 = alt_keys, *v1 = alt_vals;
  for (int p = 0; p < passes; ++p) {
    const int shift = p * kRadixBits;
    launch(ctx, radix_hist_kernel, dim3(tiles), dim3(kSortThreads), 0, static_cast<const index_t*>(k0), total,
           shift, hist, tiles);
    lsmps_status st = exclusive_scan_i32(ctx, scratch, hist, hist, hist_entries, nullptr, nullptr);
    if (st) return st;
    launch(ctx, radix_scatter_kernel, dim3(tiles), dim3(kSortThreads), 0, static_cast<const index_t*>(k0),
           static_cast<const index_t*>(v0), k1, v1, total, shift, static_cast<const index_t*>(hist), tiles);
    std::swap(k0, k1);
    std::swap(v0, v1);
  }
  const int range_blocks = static_cast<int>(std::min<long long>(div_up(total, 256), ctx->sm_count * 8LL));
  launch(ctx, ranges_kernel, dim3(range_blocks), dim3(256), 0, static_cast<const index_t*>(k0), total, tb, te);
  out->tsrc = v0;
  return check_launch(ctx, "CSR transpose");
}

// Context scratch of the operator pair: the fluid-only inverse, its trace /
// regularisation / info, and the backward stash.
bool ensure_adjoint(lsmps_ctx* ctx, size_t n) {
  if (n <= ctx->adj_cap) return true;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(ctx->stream, &cap);
  if (cap != cudaStreamCaptureStatusNone) return false;
  cudaStreamSynchronize(ctx->stream);
  free_adjoint(ctx);
  bool ok = cudaMalloc(&ctx->adj_inverse, n * 81 * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ctx->adj_trace, n * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ctx->adj_reg, n * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ctx->adj_info, n * sizeof(int32_t)) == cudaSuccess &&
            cudaMalloc(&ctx->adj_count, sizeof(int32_t)) == cudaSuccess &&
            cudaMalloc(&ctx->adj_stash, n * kStash * sizeof(double)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    free_adjoint(ctx);
    return false;
  }
  ctx->adj_cap = n;
  return true;
}

void free_adjoint(lsmps_ctx* ctx) {
  void* ps[] = {ctx->adj_inverse, ctx->adj_trace, ctx->adj_reg, ctx->adj_info, ctx->adj_count, ctx->adj_stash};
  for (void* p : ps)
    if (p) cudaFree(p);
  ctx->adj_inverse = nullptr;
  ctx->adj_trace = nullptr;
  ctx->adj_reg = nullptr;
  ctx->adj_info = nullptr;
  ctx->adj_count = nullptr;
  ctx->adj_stash = nullptr;
  ctx->adj_cap = 0;
}

namespace {

lsmps_status check_inputs(lsmps_ctx* ctx, const lsmps_fluid& fl, const lsmps_csr& fn, const lsmps_params& p,
                          const double* f, const lsmps_vector& v) {
  if (!(p.support_radius > 0.0)) return fail(ctx, LSMPS_INVALID_ARGUMENT, "support radius must be positive");
  if (fn.particle_count < fl.count) return fail(ctx, LSMPS_INVALID_ARGUMENT, "neighbour table smaller than fluid");
  if (v.count < fl.count) return fail(ctx, LSMPS_INVALID_ARGUMENT, "vector field smaller than fluid");
  if (fl.count && (!fl.x || !fl.y || !fl.z || !f || !v.x || !v.y || !v.z || !fn.offsets || !fn.indices))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "operator inputs missing");
  return check_neighbor_tables(ctx, fl.count, 0, fn, nullptr);
}

// Fluid-only Type-A moments into the context's inverse (or `inverse`).
lsmps_status moments(lsmps_ctx* ctx, const lsmps_fluid& fl, const lsmps_csr& fn, const lsmps_params& p,
                     double* inverse) {
  lsmps_moment m{};
  m.particle_count = fl.count;
  m.matrix_size = 9;
  m.kind = LSMPS_MOMENT_FLUID_ONLY_A;
  m.support_radius = p.support_radius;
  m.wall_weight_scale = p.lsmps_wall_weight_scale;
  m.inverse_matrices = inverse;
  m.moment_trace = ctx->adj_trace;
  m.regularization_added = ctx->adj_reg;
  m.info = ctx->adj_info;
  m.inversion_count = ctx->adj_count;
  lsmps_walls none{};
  lsmps_csr wn{fl.count, 0, fn.offsets, fn.indices};  // unused by the fluid-only kind
  const int prec = ctx->precision;
  ctx->precision = LSMPS_PRECISION_PLAIN;
  const lsmps_status st = prepare_moments_impl(ctx, fl, none, fn, wn, p, &m, 1);
  ctx->precision = prec;
  return st;
}

// The deterministic backward after the stash pass: the CSR's transpose,
// then the gather.
lsmps_status transpose_and_gather(lsmps_ctx* ctx, const lsmps_csr& fn, const OpsArgs& a) {
  Scratch scratch(ctx);
  CsrTranspose tr{};
  lsmps_status st = build_csr_transpose(ctx, scratch, fn, a.n, &tr);
  if (st) return st;
  launch(ctx, ops_adjoint_gather_kernel, dim3(div_up(a.n, kThreads)), dim3(kThreads), 0, a,
         static_cast<const index_t*>(tr.tb), static_cast<const index_t*>(tr.te), tr.tsrc,
         static_cast<const index_t*>(tr.owner));
  return check_launch(ctx, "operators backward (transpose and gather)");
}

OpsArgs make_args(lsmps_ctx* ctx, const lsmps_fluid& fl, const lsmps_csr& fn, const lsmps_params& p, const double* f,
                  const lsmps_vector& v, const double* inverse) {
  OpsArgs a{};
  a.n = static_cast<index_t>(fl.count);
  a.fp = ctx->pack_fluid[0];
  a.fo = fn.offsets;
  a.fi = fn.indices;
  a.f = f;
  a.vx = v.x;
  a.vy = v.y;
  a.vz = v.z;
  a.inv = inverse;
  a.re = p.support_radius;
  a.inv_re = 1.0 / p.support_radius;
  a.ppe_scale = 2.0 / (p.support_radius * p.support_radius * p.density);
  a.inv_dt = p.time_step > 0.0 ? 1.0 / p.time_step : 0.0;
  a.lambda = p.lsmps_regularization;
  a.stash = ctx->adj_stash;
  return a;
}

}  // namespace
}  // namespace lsmps

using namespace lsmps;

extern "C" lsmps_status lsmps_operators_forward(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_csr* fn,
                                                const lsmps_params* params, const double* f, const lsmps_vector* v,
                                                const lsmps_operator_out* out, double* inverse_out) {
  if (!ctx || !fluid || !fn || !params || !v || !out) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  st = check_inputs(ctx, *fluid, *fn, *params, f, *v);
  if (!st && out->count < fluid->count) st = fail(ctx, LSMPS_INVALID_ARGUMENT, "operator outputs too small");
  if (!st && fluid->count == 0) return end_call(ctx, LSMPS_OK);
  if (!st && (!ensure_adjoint(ctx, fluid->count) || !ensure_packs(ctx, fluid->count, 0)))
    st = fail(ctx, LSMPS_CUDA_ERROR, "operator scratch allocation failed");
  if (st) return end_call(ctx, st);
  double* inverse = inverse_out ? inverse_out : ctx->adj_inverse;
  st = moments(ctx, *fluid, *fn, *params, inverse);
  if (st) return end_call(ctx, st);
  pack4(ctx, fluid->x, fluid->y, fluid->z, nullptr, fluid->count, ctx->pack_fluid[0]);
  OpsArgs a = make_args(ctx, *fluid, *fn, *params, f, *v, inverse);
  a.out = *out;
  launch(ctx, ops_forward_kernel, dim3(div_up(a.n, kThreads)), dim3(kThreads), 0, a);
  return end_call(ctx, check_launch(ctx, "operators forward"));
}

extern "C" lsmps_status lsmps_operators_backward(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_csr* fn,
                                                 const lsmps_params* params, const double* f, const lsmps_vector* v,
                                                 const lsmps_operator_out* cotangent, const double* inverse,
                                                 double* f_bar, const lsmps_vector* v_bar,
                                                 const lsmps_vector* x_bar) {
  if (!ctx || !fluid || !fn || !params || !v || !cotangent) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  st = check_inputs(ctx, *fluid, *fn, *params, f, *v);
  if (!st && cotangent->count < fluid->count) st = fail(ctx, LSMPS_INVALID_ARGUMENT, "cotangents too small");
  if (!st && ((v_bar && v_bar->count < fluid->count) || (x_bar && x_bar->count < fluid->count)))
    st = fail(ctx, LSMPS_INVALID_ARGUMENT, "gradient outputs too small");
  if (!st && fluid->count == 0) return end_call(ctx, LSMPS_OK);
  if (!st && (!ensure_adjoint(ctx, fluid->count) || !ensure_packs(ctx, fluid->count, 0)))
    st = fail(ctx, LSMPS_CUDA_ERROR, "operator scratch allocation failed");
  if (st) return end_call(ctx, st);
  const size_t n = fluid->count;
  const bool atomic = ctx->adjoint_atomic;
  if (atomic) {
    // The scatter form accumulates into the gradients: start from zero.
    if (f_bar) cudaMemsetAsync(f_bar, 0, n * sizeof(double), ctx->stream);
    const lsmps_vector* outs[2] = {v_bar, x_bar};
    for (const lsmps_vector* o : outs)
      if (o) {
        cudaMemsetAsync(o->x, 0, n * sizeof(double), ctx->stream);
        cudaMemsetAsync(o->y, 0, n * sizeof(double), ctx->stream);
        cudaMemsetAsync(o->z, 0, n * sizeof(double), ctx->stream);
      }
  }
  // The inverse is recomputed from the positions unless the caller kept the
  // forward's.
  if (!inverse) {
    st = moments(ctx, *fluid, *fn, *params, ctx->adj_inverse);
    if (st) return end_call(ctx, st);
  }
  pack4(ctx, fluid->x, fluid->y, fluid->z, nullptr, n, ctx->pack_fluid[0]);
  OpsArgs a = make_args(ctx, *fluid, *fn, *params, f, *v, inverse ? inverse : ctx->adj_inverse);
  a.bar = *cotangent;
  a.fbar = f_bar;
  a.vbar[0] = v_bar ? v_bar->x : nullptr;
  a.vbar[1] = v_bar ? v_bar->y : nullptr;
  a.vbar[2] = v_bar ? v_bar->z : nullptr;
  a.xbar[0] = x_bar ? x_bar->x : nullptr;
  a.xbar[1] = x_bar ? x_bar->y : nullptr;
  a.xbar[2] = x_bar ? x_bar->z : nullptr;
  launch(ctx, ops_adjoint_rows_kernel, dim3(div_up(a.n, kThreads)), dim3(kThreads), 0, a);
  if (atomic) {
    launch(ctx, ops_adjoint_scatter_kernel, dim3(div_up(a.n, kThreads)), dim3(kThreads), 0, a);
  } else {
    st = transpose_and_gather(ctx, *fn, a);
    if (st) return end_call(ctx, st);
  }
  return end_call(ctx, check_launch(ctx, "operators backward"));
}

extern "C" lsmps_status lsmps_ctx_set_adjoint_atomic(lsmps_ctx* ctx, int on) {
  if (!ctx || (on != 0 && on != 1)) return LSMPS_INVALID_ARGUMENT;
  ctx->adjoint_atomic = on != 0;
  return LSMPS_OK;
}
