// step_adjoint.cu - the step's LSMPS operators with their wall terms as a
// forward/backward pair (no counterpart in the reference, which has no
// derivatives).
//
// Per fluid particle i, over its fluid row N(i) and wall row W(i), with
// s = d / r_e, w = 1 - |s| (moment_matrix.cu:145-150), b the Type-A basis,
// q the wall Neumann vector of the wall's normal n (moment_matrix.cu:177-201),
// lambda_w the wall weight scale and reg = lambda tr(S) / 9 (tr > 0) or lambda:
//   velocity kind   S_v = sum_N w b b^T + sum_W lambda_w w b b^T,
//                   R_c = sum_N w b (u_j,c - u_i,c) + sum_W lambda_w w b (u_w,c - u_i,c),
//                   y_c = (S_v + reg I)^-1 R_c
//                   lap_c = 2 / r_e^2 (y_c[3] + y_c[4] + y_c[5])   (explicit_update.cu:178-248)
//                   div   = sum_c y_c[c] / r_e                     (ppe_matrix.cu:355-361)
//   pressure kind   S_p = sum_N w b b^T + sum_W lambda_w w q q^T,
//                   R_p = sum_N w b (p_j - p_i) + sum_W lambda_w w q (r_e rho g.n),
//                   y_p = (S_p + reg I)^-1 R_p,  grad = y_p[0..2] / r_e  (pressure_correction.cu:200-276)
//                   L = rows 3 + 4 + 5 of (S_p + reg I)^-1; PPE row: a_ij = c w (L . b),
//                   c = 2 / (r_e^2 rho), diagonal -sum a_ij; wall_rhs = sum_W 2 lambda_w w (g.n) (L . q) / r_e;
//                   rhs = div / dt - wall_rhs                       (ppe_matrix.cu:243-370)
// Surface and Splash rows are Dirichlet rows (diagonal 1, neighbour slots 0,
// rhs = div = wall_rhs = 0); the gradient of a Splash particle is 0.
//
// Backward (labels, walls and both CSR tables fixed).  With the cotangents
// ybar of the y's, Rbar = M^-1 ybar for each field (M symmetric); the PPE
// rows' cotangent on L, h = sum_N c abar_ij w b + sum_W 2 lambda_w w (g.n)
// wrb q / r_e (abar_ij = the slot's cotangent minus the diagonal's,
// wrb = wall_rhs_bar - rhs_bar), gives hhat = M_p^-1 h.  The matrices'
// cotangents are -sum Rbar y^T (and -hhat L^T for M_p), plus, through the
// regularisation, lambda/9 times their trace on the diagonal (rho = sum
// Rbar . y (+ hhat . L) per kind).  A fluid entry (i, j) then contributes
// dL = alpha dw + beta . db with
//   alpha = sum_fields (Rbar . b)(dphi - b . y) - (hhat . b)(L . b) + c abar (L . b)
//           - (lambda/9)(rho_v + rho_p) |b|^2
//   beta  = w sum_fields [Rbar (dphi - b . y) - (Rbar . b) y] - w [(L . b) hhat + (hhat . b) L]
//           + c abar w L - 2 w (lambda/9)(rho_v + rho_p) b
// (fields: u_x, u_y, u_z on the velocity kind, p on the pressure kind), and
// its field cotangents w (Rbar . b) go to phibar_j and are taken from
// phibar_i.  A wall entry changes only its owner: with omega = lambda_w w,
// dL/domega = sum_c (Rbar_c . b)(du_c - b . y_c) - (lambda/9) rho_v |b|^2
//           + (Rbar_p . q)(r_e rho g.n - q . y_p) - (hhat . q)(L . q) - (lambda/9) rho_p |q|^2
//           + 2 (g.n)(L . q) wrb / r_e,
// and the cotangents of b and q follow the same pattern.  Positions: with
// d = x_j - x_i, dL/dd = (-(dL/dw) d / |d| + J_b^T dL/db + J_q^T dL/dq) / r_e,
// added to xbar_j (fluid neighbours) and taken from xbar_i.
//
// The inverses of both kinds are recomputed from the positions in the
// backward.  Deterministic form (default): every particle sums its own
// row's and wall row's terms and, through the CSR's transpose, the terms of
// the rows that list it, in a fixed order; atomic form
// (lsmps_ctx_set_adjoint_atomic): FP64 atomics into the neighbours.
#include <algorithm>

#include "adjoint.cuh"
#include "cells.cuh"
#include "impl.cuh"
#include "packed.cuh"

namespace lsmps {
namespace {

constexpr int kThreads = kAdjThreads;
// Stash per particle: Rbar of u_x, u_y, u_z (27), their y (27), Rbar_p (9),
// y_p (9), hhat (9), L (9), the regularisation factors of both kinds, the
// Dirichlet flag and wrb.
constexpr int kRbV = 0, kYV = 27, kRbP = 54, kYP = 63, kHh = 72, kL = 81, kRegV = 90, kRegP = 91, kDir = 92,
              kWrb = 93, kStashStep = 96;

struct StepOpsArgs {
  index_t n;
  const double4* fp;  // fluid {x, y, z, p}
  const double4* fv;  // fluid {u_x, u_y, u_z, -}
  const double4* wp;  // walls {x, y, z, -}
  const double4* wv;  // walls {u_x, u_y, u_z, -}
  const double4* wn;  // walls {n_x, n_y, n_z, -}
  const index_t* fo;
  const index_t* fi;
  const index_t* wo;
  const index_t* wi;
  const int32_t* label;
  const double* inv_v;  // [n][81] column-major
  const double* inv_p;
  const double* tr_v;
  const double* tr_p;
  double re;
  double inv_re;
  double lam_w;
  double lambda;
  double rho;
  double inv_dt;
  double c_ppe;  // 2 / (r_e^2 rho)
  double gx, gy, gz;
  lsmps_step_operator_out out;
  lsmps_step_operator_out bar;
  double* stash;
  double* ubar[3];
  double* pbar;
  double* xbar[3];
};

__device__ __forceinline__ double opt(const double* p, index_t i) { return p ? p[i] : 0.0; }

__device__ __forceinline__ bool dirichlet_row(const int32_t* label, index_t i) {
  if (!label) return false;
  const int t = label[i];
  return t == LSMPS_SURFACE_SURFACE || t == LSMPS_SURFACE_SPLASH;
}

__device__ __forceinline__ bool splash(const int32_t* label, index_t i) {
  return label && label[i] == LSMPS_SURFACE_SPLASH;
}

__device__ __forceinline__ void lap_row(const double* __restrict__ x, double l[9]) {
#pragma unroll
  for (int c = 0; c < 9; ++c) l[c] = x[3 + c * 9] + x[4 + c * 9] + x[5 + c * 9];
}

// Forward: the right-hand sides of both kinds over both rows, the PPE row,
// then the inverses applied.
__global__ void __launch_bounds__(kThreads) step_ops_forward_kernel(StepOpsArgs a) {
  const index_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double4 pi = ld4(a.fp, i), ui = ld4(a.fv, i);
  const double* __restrict__ xv = a.inv_v + static_cast<size_t>(i) * 81;
  const double* __restrict__ xp = a.inv_p + static_cast<size_t>(i) * 81;
  const bool dir = dirichlet_row(a.label, i);
  const bool ppe = a.out.ppe_values != nullptr;
  double l[9];
  lap_row(xp, l);
  double rx[9], ry[9], rz[9], rp[9], b[9], s[3];
#pragma unroll
  for (int k = 0; k < 9; ++k) rx[k] = ry[k] = rz[k] = rp[k] = 0.0;
  const index_t nb = a.fo[i], ne = a.fo[i + 1];
  const index_t row = i + nb;
  double diag = 0.0;
  for (index_t o = nb; o < ne; ++o) {
    const index_t j = a.fi[o];
    const double4 q = ld4(a.fp, j), v = ld4(a.fv, j);
    const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
    const double w = lin_weight(sqrt(dx * dx + dy * dy + dz * dz), a.re);
    double coef = 0.0;
    if (w > 0.0) {
      basis_div(dx, dy, dz, a.inv_re, b, s);
      const double dux = v.x - ui.x, duy = v.y - ui.y, duz = v.z - ui.z, dp = q.w - pi.w;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const double wb = w * b[k];
        rx[k] = fma(wb, dux, rx[k]);
        ry[k] = fma(wb, duy, ry[k]);
        rz[k] = fma(wb, duz, rz[k]);
        rp[k] = fma(wb, dp, rp[k]);
      }
      if (!dir) {
        coef = a.c_ppe * w * dot9(l, b);
        diag -= coef;
      }
    }
    if (ppe) {
      a.out.ppe_col_indices[row + 1 + o - nb] = j;
      a.out.ppe_values[row + 1 + o - nb] = coef;
    }
  }
  double wall_rhs = 0.0;
  const index_t we = a.wo[i + 1];
  for (index_t o = a.wo[i]; o < we; ++o) {
    const index_t j = a.wi[o];
    const double4 q = ld4(a.wp, j), v = ld4(a.wv, j), nrm = ld4(a.wn, j);
    const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
    const double w = lin_weight(sqrt(dx * dx + dy * dy + dz * dz), a.re);
    if (w <= 0.0) continue;
    const double om = a.lam_w * w;
    basis_div(dx, dy, dz, a.inv_re, b, s);
    const double dux = v.x - ui.x, duy = v.y - ui.y, duz = v.z - ui.z;
    double q9[9];
    neumann_a(dx, dy, dz, nrm.x, nrm.y, nrm.z, a.inv_re, q9);
    const double gn = a.gx * nrm.x + a.gy * nrm.y + a.gz * nrm.z;
    const double src = a.re * a.rho * gn;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const double ob = om * b[k];
      rx[k] = fma(ob, dux, rx[k]);
      ry[k] = fma(ob, duy, ry[k]);
      rz[k] = fma(ob, duz, rz[k]);
      rp[k] = fma(om * q9[k], src, rp[k]);
    }
    if (!dir) wall_rhs += 2.0 * om * gn * dot9(l, q9) * a.inv_re;
  }
  double y[9];
  double div = 0.0;
  const double* rv[3] = {rx, ry, rz};
  double* lap[3] = {a.out.lap_x, a.out.lap_y, a.out.lap_z};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    apply(xv, rv[c], y);
    if (lap[c]) lap[c][i] = 2.0 * (y[3] + y[4] + y[5]) * a.inv_re * a.inv_re;
    div += y[c];
  }
  div *= a.inv_re;
  apply(xp, rp, y);
  const bool spl = splash(a.label, i);
  if (a.out.grad_x) {
    a.out.grad_x[i] = spl ? 0.0 : y[0] * a.inv_re;
    a.out.grad_y[i] = spl ? 0.0 : y[1] * a.inv_re;
    a.out.grad_z[i] = spl ? 0.0 : y[2] * a.inv_re;
  }
  if (dir) {
    div = 0.0;
    wall_rhs = 0.0;
  }
  if (a.out.divergence) a.out.divergence[i] = div;
  if (a.out.wall_rhs) a.out.wall_rhs[i] = wall_rhs;
  if (a.out.ppe_rhs) a.out.ppe_rhs[i] = dir ? 0.0 : div * a.inv_dt - wall_rhs;
  if (ppe) {
    a.out.ppe_row_offsets[i] = row;
    if (i + 1 == a.n) a.out.ppe_row_offsets[a.n] = a.n + ne;
    a.out.ppe_col_indices[row] = i;
    a.out.ppe_values[row] = dir ? 1.0 : diag;
  }
}

// Backward, pass 1: the stash of every particle (Rbar, y of the four
// fields, hhat, L, the regularisation factors, the Dirichlet flag, wrb).
__global__ void __launch_bounds__(kThreads) step_ops_rows_kernel(StepOpsArgs a) {
  const index_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double4 pi = ld4(a.fp, i), ui = ld4(a.fv, i);
  const double* __restrict__ xv = a.inv_v + static_cast<size_t>(i) * 81;
  const double* __restrict__ xp = a.inv_p + static_cast<size_t>(i) * 81;
  double* st = a.stash + static_cast<size_t>(i) * kStashStep;
  const bool dir = dirichlet_row(a.label, i);
  const bool ppe = a.bar.ppe_values != nullptr && !dir;
  const index_t nb = a.fo[i], ne = a.fo[i + 1];
  const index_t row = i + nb;
  const double diag_bar = ppe ? a.bar.ppe_values[row] : 0.0;
  const double wrb = dir ? 0.0 : opt(a.bar.wall_rhs, i) - opt(a.bar.ppe_rhs, i);
  double rx[9], ry[9], rz[9], rp[9], h[9], b[9], s[3];
#pragma unroll
  for (int k = 0; k < 9; ++k) rx[k] = ry[k] = rz[k] = rp[k] = h[k] = 0.0;
  for (index_t o = nb; o < ne; ++o) {
    const index_t j = a.fi[o];
    const double4 q = ld4(a.fp, j), v = ld4(a.fv, j);
    const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
    const double w = lin_weight(sqrt(dx * dx + dy * dy + dz * dz), a.re);
    if (w <= 0.0) continue;
    basis_div(dx, dy, dz, a.inv_re, b, s);
    const double dux = v.x - ui.x, duy = v.y - ui.y, duz = v.z - ui.z, dp = q.w - pi.w;
    const double ab = ppe ? a.c_ppe * (a.bar.ppe_values[row + 1 + o - nb] - diag_bar) : 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const double wb = w * b[k];
      rx[k] = fma(wb, dux, rx[k]);
      ry[k] = fma(wb, duy, ry[k]);
      rz[k] = fma(wb, duz, rz[k]);
      rp[k] = fma(wb, dp, rp[k]);
      h[k] = fma(wb, ab, h[k]);
    }
  }
  const index_t we = a.wo[i + 1];
  for (index_t o = a.wo[i]; o < we; ++o) {
    const index_t j = a.wi[o];
    const double4 q = ld4(a.wp, j), v = ld4(a.wv, j), nrm = ld4(a.wn, j);
    const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
    const double w = lin_weight(sqrt(dx * dx + dy * dy + dz * dz), a.re);
    if (w <= 0.0) continue;
    const double om = a.lam_w * w;
    basis_div(dx, dy, dz, a.inv_re, b, s);
    const double dux = v.x - ui.x, duy = v.y - ui.y, duz = v.z - ui.z;
    double q9[9];
    neumann_a(dx, dy, dz, nrm.x, nrm.y, nrm.z, a.inv_re, q9);
    const double gn = a.gx * nrm.x + a.gy * nrm.y + a.gz * nrm.z;
    const double src = a.re * a.rho * gn;
    const double hw = 2.0 * om * gn * a.inv_re * wrb;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const double ob = om * b[k];
      rx[k] = fma(ob, dux, rx[k]);
      ry[k] = fma(ob, duy, ry[k]);
      rz[k] = fma(ob, duz, rz[k]);
      rp[k] = fma(om * q9[k], src, rp[k]);
      h[k] = fma(hw, q9[k], h[k]);
    }
  }
  // velocity kind: cotangents of y_c from lap_c (rows 3..5) and, on the
  // PPE rows, from div (and rhs = div / dt - wall_rhs)
  const double dbar = dir ? 0.0 : (opt(a.bar.divergence, i) + opt(a.bar.ppe_rhs, i) * a.inv_dt) * a.inv_re;
  const double* lapb[3] = {a.bar.lap_x, a.bar.lap_y, a.bar.lap_z};
  const double* rv[3] = {rx, ry, rz};
  double rho_v = 0.0, t[9], u[9], rb[9];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    apply(xv, rv[c], u);
    const double lb = 2.0 * opt(lapb[c], i) * a.inv_re * a.inv_re;
#pragma unroll
    for (int k = 0; k < 9; ++k) t[k] = (k >= 3 && k <= 5 ? lb : 0.0) + (k == c ? dbar : 0.0);
    apply(xv, t, rb);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      st[kRbV + 9 * c + k] = rb[k];
      st[kYV + 9 * c + k] = u[k];
    }
    rho_v += dot9(rb, u);
  }
  // pressure kind: gradient rows 0..2 (not for Splash), the PPE rows' L
  apply(xp, rp, u);
  const bool spl = splash(a.label, i);
#pragma unroll
  for (int k = 0; k < 9; ++k) t[k] = 0.0;
  if (!spl) {
    t[0] = opt(a.bar.grad_x, i) * a.inv_re;
    t[1] = opt(a.bar.grad_y, i) * a.inv_re;
    t[2] = opt(a.bar.grad_z, i) * a.inv_re;
  }
  apply(xp, t, rb);
  double rho_p = dot9(rb, u);
  double l[9], hh[9];
  lap_row(xp, l);
  apply(xp, h, hh);
  rho_p += dot9(hh, l);
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    st[kRbP + k] = rb[k];
    st[kYP + k] = u[k];
    st[kHh + k] = hh[k];
    st[kL + k] = l[k];
  }
  st[kRegV] = a.tr_v[i] > 0.0 ? rho_v * a.lambda / 9.0 : 0.0;
  st[kRegP] = a.tr_p[i] > 0.0 ? rho_p * a.lambda / 9.0 : 0.0;
  st[kDir] = dir ? 1.0 : 0.0;
  st[kWrb] = wrb;
}

// The owner-side values pair_terms needs.
struct StepOwner {
  double4 pi;
  double4 ui;
  const double* st;
  index_t nb;
  index_t row;
  double diag_bar;
  bool ppe;
};

__device__ __forceinline__ StepOwner step_owner(const StepOpsArgs& a, index_t i) {
  StepOwner t;
  t.pi = ld4(a.fp, i);
  t.ui = ld4(a.fv, i);
  t.st = a.stash + static_cast<size_t>(i) * kStashStep;
  t.nb = a.fo[i];
  t.row = i + t.nb;
  t.ppe = a.bar.ppe_values != nullptr && t.st[kDir] == 0.0;
  t.diag_bar = t.ppe ? a.bar.ppe_values[t.row] : 0.0;
  return t;
}

// Terms of fluid entry o of owner t with neighbour j: tu[c] and tp go to
// the neighbour's field cotangents and are taken from the owner's; g goes to
// xbar_j and is taken from xbar_i.  False for an entry with zero weight or
// zero distance.
__device__ __forceinline__ bool step_pair_terms(const StepOpsArgs& a, const StepOwner& t, index_t o, index_t j,
                                                double tu[3], double& tp, double g[3]) {
  const double4 q = ld4(a.fp, j), v = ld4(a.fv, j);
  const double dx = q.x - t.pi.x, dy = q.y - t.pi.y, dz = q.z - t.pi.z;
  const double dist = sqrt(dx * dx + dy * dy + dz * dz);
  const double w = lin_weight(dist, a.re);
  if (w <= 0.0 || dist <= 0.0) return false;
  const double* st = t.st;
  double b[9], s[3], beta[9];
  basis_div(dx, dy, dz, a.inv_re, b, s);
  double alpha = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) beta[k] = 0.0;
  const double dphi[4] = {v.x - t.ui.x, v.y - t.ui.y, v.z - t.ui.z, q.w - t.pi.w};
  const int rb_at[4] = {kRbV, kRbV + 9, kRbV + 18, kRbP};
  const int y_at[4] = {kYV, kYV + 9, kYV + 18, kYP};
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const double* rb = st + rb_at[f];
    const double* y = st + y_at[f];
    const double rbb = dot9(rb, b);
    const double e = dphi[f] - dot9(b, y);
    alpha = fma(rbb, e, alpha);
#pragma unroll
    for (int k = 0; k < 9; ++k) beta[k] = fma(w, rb[k] * e - rbb * y[k], beta[k]);
    if (f < 3)
      tu[f] = w * rbb;
    else
      tp = w * rbb;
  }
  const double* hh = st + kHh;
  const double* l = st + kL;
  const double lb = dot9(l, b), hb = dot9(hh, b);
  alpha -= hb * lb;
#pragma unroll
  for (int k = 0; k < 9; ++k) beta[k] -= w * (lb * hh[k] + hb * l[k]);
  if (t.ppe) {
    const double ab = a.c_ppe * (a.bar.ppe_values[t.row + 1 + o - t.nb] - t.diag_bar);
    alpha += ab * lb;
#pragma unroll
    for (int k = 0; k < 9; ++k) beta[k] += ab * w * l[k];
  }
  const double reg = st[kRegV] + st[kRegP];
  if (reg != 0.0) {
    alpha -= reg * dot9(b, b);
#pragma unroll
    for (int k = 0; k < 9; ++k) beta[k] -= reg * 2.0 * w * b[k];
  }
  double jt[3];
  basis_jt(s, beta, jt);
  const double inv_d = 1.0 / dist;
  g[0] = (-alpha * dx * inv_d + jt[0]) * a.inv_re;
  g[1] = (-alpha * dy * inv_d + jt[1]) * a.inv_re;
  g[2] = (-alpha * dz * inv_d + jt[2]) * a.inv_re;
  return true;
}

// Terms of the owner's wall row (walls are held fixed: only the owner's
// cotangents change): adds to tu (taken from u_i's cotangent) and g (taken
// from x_i's).
__device__ __forceinline__ void step_wall_terms(const StepOpsArgs& a, const StepOwner& t, index_t i, double tu[3],
                                                double g[3]) {
  const double* st = t.st;
  const double* hh = st + kHh;
  const double* l = st + kL;
  const index_t we = a.wo[i + 1];
  for (index_t o = a.wo[i]; o < we; ++o) {
    const index_t j = a.wi[o];
    const double4 q = ld4(a.wp, j), v = ld4(a.wv, j), nrm = ld4(a.wn, j);
    const double dx = q.x - t.pi.x, dy = q.y - t.pi.y, dz = q.z - t.pi.z;
    const double dist = sqrt(dx * dx + dy * dy + dz * dz);
    const double w = lin_weight(dist, a.re);
    if (w <= 0.0 || dist <= 0.0) continue;
    const double om = a.lam_w * w;
    double b[9], s[3], beta[9], gam[9], q9[9];
    basis_div(dx, dy, dz, a.inv_re, b, s);
    neumann_a(dx, dy, dz, nrm.x, nrm.y, nrm.z, a.inv_re, q9);
    const double gn = a.gx * nrm.x + a.gy * nrm.y + a.gz * nrm.z;
    const double src = a.re * a.rho * gn;
    double alpha = 0.0;  // dL / domega
#pragma unroll
    for (int k = 0; k < 9; ++k) beta[k] = gam[k] = 0.0;
    // velocity kind, Dirichlet samples
    const double du[3] = {v.x - t.ui.x, v.y - t.ui.y, v.z - t.ui.z};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double* rb = st + kRbV + 9 * c;
      const double* y = st + kYV + 9 * c;
      const double rbb = dot9(rb, b);
      const double e = du[c] - dot9(b, y);
      alpha = fma(rbb, e, alpha);
#pragma unroll
      for (int k = 0; k < 9; ++k) beta[k] = fma(om, rb[k] * e - rbb * y[k], beta[k]);
      tu[c] += om * rbb;
    }
    if (st[kRegV] != 0.0) {
      alpha -= st[kRegV] * dot9(b, b);
#pragma unroll
      for (int k = 0; k < 9; ++k) beta[k] -= st[kRegV] * 2.0 * om * b[k];
    }
    // pressure kind, Neumann terms and the PPE wall source
    {
      const double* rb = st + kRbP;
      const double* y = st + kYP;
      const double rqq = dot9(rb, q9);
      const double e = src - dot9(q9, y);
      alpha = fma(rqq, e, alpha);
#pragma unroll
      for (int k = 0; k < 9; ++k) gam[k] = fma(om, rb[k] * e - rqq * y[k], gam[k]);
      const double lq = dot9(l, q9), hq = dot9(hh, q9);
      alpha -= hq * lq;
#pragma unroll
      for (int k = 0; k < 9; ++k) gam[k] -= om * (lq * hh[k] + hq * l[k]);
      if (st[kRegP] != 0.0) {
        alpha -= st[kRegP] * dot9(q9, q9);
#pragma unroll
        for (int k = 0; k < 9; ++k) gam[k] -= st[kRegP] * 2.0 * om * q9[k];
      }
      const double wrb = st[kWrb];
      if (wrb != 0.0) {
        const double f = 2.0 * gn * a.inv_re * wrb;
        alpha += f * lq;
#pragma unroll
        for (int k = 0; k < 9; ++k) gam[k] += f * om * l[k];
      }
    }
    // dL/ds = J_b^T beta + J_q^T gamma; J_q from q3..q8 (linear in s)
    double jt[3];
    basis_jt(s, beta, jt);
    jt[0] += 2.0 * nrm.x * gam[3] + nrm.y * gam[6] + nrm.z * gam[8];
    jt[1] += 2.0 * nrm.y * gam[4] + nrm.x * gam[6] + nrm.z * gam[7];
    jt[2] += 2.0 * nrm.z * gam[5] + nrm.y * gam[7] + nrm.x * gam[8];
    const double dw = a.lam_w * alpha;  // dL / dw
    const double inv_d = 1.0 / dist;
    g[0] += (-dw * dx * inv_d + jt[0]) * a.inv_re;
    g[1] += (-dw * dy * inv_d + jt[1]) * a.inv_re;
    g[2] += (-dw * dz * inv_d + jt[2]) * a.inv_re;
  }
}

// Atomic form: each owner scatters its fluid entries' terms into the
// neighbours and keeps its own (fluid and wall) terms.
__global__ void __launch_bounds__(kThreads) step_ops_scatter_kernel(StepOpsArgs a) {
  const index_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const StepOwner t = step_owner(a, i);
  double own_u[3] = {0.0, 0.0, 0.0}, own_g[3] = {0.0, 0.0, 0.0}, own_p = 0.0;
  const index_t ne = a.fo[i + 1];
  for (index_t o = t.nb; o < ne; ++o) {
    const index_t j = a.fi[o];
    double tu[3], tp, g[3];
    if (!step_pair_terms(a, t, o, j, tu, tp, g)) continue;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (a.ubar[c]) atomicAdd(&a.ubar[c][j], tu[c]);
      own_u[c] -= tu[c];
      if (a.xbar[c]) atomicAdd(&a.xbar[c][j], g[c]);
      own_g[c] -= g[c];
    }
    if (a.pbar) atomicAdd(&a.pbar[j], tp);
    own_p -= tp;
  }
  double wu[3] = {0.0, 0.0, 0.0}, wg[3] = {0.0, 0.0, 0.0};
  step_wall_terms(a, t, i, wu, wg);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (a.ubar[c]) atomicAdd(&a.ubar[c][i], own_u[c] - wu[c]);
    if (a.xbar[c]) atomicAdd(&a.xbar[c][i], own_g[c] - wg[c]);
  }
  if (a.pbar) atomicAdd(&a.pbar[i], own_p);
}

// Deterministic form: particle j gathers its incoming fluid entries' terms
// (the transpose row, ascending entry order), then its own fluid row's and
// wall row's, and writes its cotangents.
__global__ void __launch_bounds__(kThreads) step_ops_gather_kernel(StepOpsArgs a, const index_t* __restrict__ tb,
                                                                   const index_t* __restrict__ te,
                                                                   const index_t* __restrict__ tsrc,
                                                                   const index_t* __restrict__ owner) {
  const index_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  double acc_u[3] = {0.0, 0.0, 0.0}, acc_g[3] = {0.0, 0.0, 0.0}, acc_p = 0.0;
  const index_t b0 = tb[j], e0 = te[j];
  if (b0 >= 0) {
    for (index_t k = b0; k < e0; ++k) {
      const index_t o = tsrc[k];
      const StepOwner t = step_owner(a, owner[o]);
      double tu[3], tp, g[3];
      if (!step_pair_terms(a, t, o, j, tu, tp, g)) continue;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        acc_u[c] += tu[c];
        acc_g[c] += g[c];
      }
      acc_p += tp;
    }
  }
  const StepOwner t = step_owner(a, j);
  const index_t ne = a.fo[j + 1];
  for (index_t o = t.nb; o < ne; ++o) {
    double tu[3], tp, g[3];
    if (!step_pair_terms(a, t, o, a.fi[o], tu, tp, g)) continue;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      acc_u[c] -= tu[c];
      acc_g[c] -= g[c];
    }
    acc_p -= tp;
  }
  double wu[3] = {0.0, 0.0, 0.0}, wg[3] = {0.0, 0.0, 0.0};
  step_wall_terms(a, t, j, wu, wg);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (a.ubar[c]) a.ubar[c][j] = acc_u[c] - wu[c];
    if (a.xbar[c]) a.xbar[c][j] = acc_g[c] - wg[c];
  }
  if (a.pbar) a.pbar[j] = acc_p;
}

lsmps_status check_step_inputs(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w, const lsmps_csr& fn,
                               const lsmps_csr& wn, const lsmps_params& p) {
  if (!(p.support_radius > 0.0)) return fail(ctx, LSMPS_INVALID_ARGUMENT, "support radius must be positive");
  if (!(p.density > 0.0)) return fail(ctx, LSMPS_INVALID_ARGUMENT, "density must be positive");
  if (fn.particle_count < f.count || wn.particle_count < f.count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "neighbour tables smaller than fluid");
  if (f.count && (!f.x || !f.y || !f.z || !f.vx || !f.vy || !f.vz || !f.pressure || !fn.offsets || !fn.indices ||
                  !wn.offsets || (wn.neighbor_count && !wn.indices)))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "step operator inputs missing");
  if (w.count && (!w.x || !w.y || !w.z || !w.vx || !w.vy || !w.vz || !w.normal_x || !w.normal_y || !w.normal_z))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "wall positions, velocities and normals are required");
  return check_neighbor_tables(ctx, f.count, w.count, fn, &wn);
}

// Both kinds' inverses (plain FP64) into the context's step-operator scratch,
// and the neighbour records.
lsmps_status prepare_step_ops(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w, const lsmps_csr& fn,
                              const lsmps_csr& wn, const lsmps_params& p, StepOpsArgs& a) {
  const size_t n = f.count;
  if (!ensure_step_ops(ctx, n) || !ensure_packs(ctx, n, w.count))
    return fail(ctx, LSMPS_CUDA_ERROR, "step operator scratch allocation failed");
  lsmps_moment m[2]{};
  const int kinds[2] = {LSMPS_MOMENT_VELOCITY_WALL_DIRICHLET_A, LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_A};
  for (int k = 0; k < 2; ++k) {
    m[k].particle_count = n;
    m[k].matrix_size = 9;
    m[k].kind = kinds[k];
    m[k].support_radius = p.support_radius;
    m[k].wall_weight_scale = p.lsmps_wall_weight_scale;
    m[k].inverse_matrices = ctx->sop_inverse[k];
    m[k].moment_trace = ctx->sop_trace[k];
    m[k].regularization_added = ctx->sop_reg[k];
    m[k].info = ctx->sop_info[k];
    m[k].inversion_count = ctx->sop_count + k;
  }
  const int prec = ctx->precision;
  const int32_t* order = ctx->order;
  ctx->precision = LSMPS_PRECISION_PLAIN;
  ctx->order = nullptr;
  const lsmps_status st = prepare_moments_impl(ctx, f, w, fn, wn, p, m, 2);
  ctx->precision = prec;
  ctx->order = order;
  if (st) return st;
  pack4(ctx, f.x, f.y, f.z, f.pressure, n, ctx->pack_fluid[0]);
  pack4(ctx, f.vx, f.vy, f.vz, nullptr, n, ctx->pack_fluid[1]);
  pack4(ctx, w.x, w.y, w.z, nullptr, w.count, ctx->pack_wall[0]);
  pack4(ctx, w.vx, w.vy, w.vz, nullptr, w.count, ctx->pack_wall[1]);
  pack4(ctx, w.normal_x, w.normal_y, w.normal_z, nullptr, w.count, ctx->pack_wall[2]);
  a = StepOpsArgs{};
  a.n = static_cast<index_t>(n);
  a.fp = ctx->pack_fluid[0];
  a.fv = ctx->pack_fluid[1];
  a.wp = ctx->pack_wall[0];
  a.wv = ctx->pack_wall[1];
  a.wn = ctx->pack_wall[2];
  a.fo = fn.offsets;
  a.fi = fn.indices;
  a.wo = wn.offsets;
  a.wi = wn.indices;
  a.label = f.surface_type;
  a.inv_v = ctx->sop_inverse[0];
  a.inv_p = ctx->sop_inverse[1];
  a.tr_v = ctx->sop_trace[0];
  a.tr_p = ctx->sop_trace[1];
  a.re = p.support_radius;
  a.inv_re = 1.0 / p.support_radius;
  a.lam_w = p.lsmps_wall_weight_scale;
  a.lambda = p.lsmps_regularization;
  a.rho = p.density;
  a.inv_dt = p.time_step > 0.0 ? 1.0 / p.time_step : 0.0;
  a.c_ppe = 2.0 / (p.support_radius * p.support_radius * p.density);
  a.gx = p.gravity[0];
  a.gy = p.gravity[1];
  a.gz = p.gravity[2];
  a.stash = ctx->sop_stash;
  return LSMPS_OK;
}

}  // namespace

// Context scratch of the step operator pair.
bool ensure_step_ops(lsmps_ctx* ctx, size_t n) {
  if (n <= ctx->sop_cap) return true;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(ctx->stream, &cap);
  if (cap != cudaStreamCaptureStatusNone) return false;
  cudaStreamSynchronize(ctx->stream);
  free_step_ops(ctx);
  bool ok = cudaMalloc(&ctx->sop_count, 2 * sizeof(int32_t)) == cudaSuccess &&
            cudaMalloc(&ctx->sop_stash, n * kStashStep * sizeof(double)) == cudaSuccess;
  for (int k = 0; k < 2 && ok; ++k)
    ok = cudaMalloc(&ctx->sop_inverse[k], n * 81 * sizeof(double)) == cudaSuccess &&
         cudaMalloc(&ctx->sop_trace[k], n * sizeof(double)) == cudaSuccess &&
         cudaMalloc(&ctx->sop_reg[k], n * sizeof(double)) == cudaSuccess &&
         cudaMalloc(&ctx->sop_info[k], n * sizeof(int32_t)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    free_step_ops(ctx);
    return false;
  }
  ctx->sop_cap = n;
  return true;
}

void free_step_ops(lsmps_ctx* ctx) {
  for (int k = 0; k < 2; ++k) {
    void* ps[] = {ctx->sop_inverse[k], ctx->sop_trace[k], ctx->sop_reg[k], ctx->sop_info[k]};
    for (void* p : ps)
      if (p) cudaFree(p);
    ctx->sop_inverse[k] = nullptr;
    ctx->sop_trace[k] = nullptr;
    ctx->sop_reg[k] = nullptr;
    ctx->sop_info[k] = nullptr;
  }
  if (ctx->sop_count) cudaFree(ctx->sop_count);
  if (ctx->sop_stash) cudaFree(ctx->sop_stash);
  ctx->sop_count = nullptr;
  ctx->sop_stash = nullptr;
  ctx->sop_cap = 0;
}

}  // namespace lsmps

using namespace lsmps;

extern "C" lsmps_status lsmps_step_operators_forward(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                                     const lsmps_walls* walls, const lsmps_csr* fn,
                                                     const lsmps_csr* wn, const lsmps_params* params,
                                                     const lsmps_step_operator_out* out) {
  if (!ctx || !fluid || !walls || !fn || !wn || !params || !out) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  st = check_step_inputs(ctx, *fluid, *walls, *fn, *wn, *params);
  if (!st && out->count < fluid->count) st = fail(ctx, LSMPS_INVALID_ARGUMENT, "operator outputs too small");
  if (!st && fluid->count == 0) return end_call(ctx, LSMPS_OK);
  if (st) return end_call(ctx, st);
  StepOpsArgs a;
  st = prepare_step_ops(ctx, *fluid, *walls, *fn, *wn, *params, a);
  if (st) return end_call(ctx, st);
  a.out = *out;
  launch(ctx, step_ops_forward_kernel, dim3(div_up(a.n, kThreads)), dim3(kThreads), 0, a);
  return end_call(ctx, check_launch(ctx, "step operators forward"));
}

extern "C" lsmps_status lsmps_step_operators_backward(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                                      const lsmps_walls* walls, const lsmps_csr* fn,
                                                      const lsmps_csr* wn, const lsmps_params* params,
                                                      const lsmps_step_operator_out* cotangent,
                                                      const lsmps_vector* u_bar, double* p_bar,
                                                      const lsmps_vector* x_bar) {
  if (!ctx || !fluid || !walls || !fn || !wn || !params || !cotangent) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  st = check_step_inputs(ctx, *fluid, *walls, *fn, *wn, *params);
  if (!st && cotangent->count < fluid->count) st = fail(ctx, LSMPS_INVALID_ARGUMENT, "cotangents too small");
  if (!st && ((u_bar && u_bar->count < fluid->count) || (x_bar && x_bar->count < fluid->count)))
    st = fail(ctx, LSMPS_INVALID_ARGUMENT, "gradient outputs too small");
  if (!st && fluid->count == 0) return end_call(ctx, LSMPS_OK);
  if (st) return end_call(ctx, st);
  StepOpsArgs a;
  st = prepare_step_ops(ctx, *fluid, *walls, *fn, *wn, *params, a);
  if (st) return end_call(ctx, st);
  a.bar = *cotangent;
  a.ubar[0] = u_bar ? u_bar->x : nullptr;
  a.ubar[1] = u_bar ? u_bar->y : nullptr;
  a.ubar[2] = u_bar ? u_bar->z : nullptr;
  a.pbar = p_bar;
  a.xbar[0] = x_bar ? x_bar->x : nullptr;
  a.xbar[1] = x_bar ? x_bar->y : nullptr;
  a.xbar[2] = x_bar ? x_bar->z : nullptr;
  const size_t n = fluid->count;
  launch(ctx, step_ops_rows_kernel, dim3(div_up(a.n, kThreads)), dim3(kThreads), 0, a);
  if (ctx->adjoint_atomic) {
    // the scatter form accumulates: start from zero
    double* outs[7] = {a.ubar[0], a.ubar[1], a.ubar[2], a.pbar, a.xbar[0], a.xbar[1], a.xbar[2]};
    for (double* o : outs)
      if (o) cudaMemsetAsync(o, 0, n * sizeof(double), ctx->stream);
    launch(ctx, step_ops_scatter_kernel, dim3(div_up(a.n, kThreads)), dim3(kThreads), 0, a);
  } else {
    Scratch scratch(ctx);
    CsrTranspose tr{};
    st = build_csr_transpose(ctx, scratch, *fn, a.n, &tr);
    if (st) return end_call(ctx, st);
    launch(ctx, step_ops_gather_kernel, dim3(div_up(a.n, kThreads)), dim3(kThreads), 0, a,
           static_cast<const index_t*>(tr.tb), static_cast<const index_t*>(tr.te), tr.tsrc,
           static_cast<const index_t*>(tr.owner));
  }
  return end_call(ctx, check_launch(ctx, "step operators backward"));
}
