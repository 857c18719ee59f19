// ppe.cu - PPE CSR rows and right-hand side.
// Replaces assemble_ppe_matrix_and_rhs (src/ppe/ppe_matrix.cu:517-551):
// build_ppe_row_offsets_kernel (:133-146) is folded into the row kernel, which
// restates assemble_ppe_system_kernel (:243-370).  Row i starts at
// i + fluid_offsets[i]; slot 0 is the diagonal, then one slot per fluid
// neighbour in CSR order (columns unsorted).  Surface and Splash rows are
// Dirichlet rows: diagonal 1, neighbour slots 0, rhs 0 (:124-131, :262-276).
#include "impl.cuh"
#include "mixed.cuh"
#include "packed.cuh"

namespace lsmps {
namespace {

constexpr int kThreads = 128;

struct PpeArgs {
  lsmps_fluid fluid;
  lsmps_walls walls;
  const index_t* fo;
  const index_t* fi;
  const index_t* wo;
  const index_t* wi;
  const double* tvx;
  const double* tvy;
  const double* tvz;
  const double* twx;
  const double* twy;
  const double* twz;
  const double* vinv;
  const double* pinv;
  double re;
  double inv_re;
  double vwall_scale;
  double pwall_scale;
  double density;
  double dt;
  const double* dt_dev;  // device time step (overrides dt when set)
  double gx, gy, gz;
  index_t* row_offsets;
  index_t* col;
  double* val;
  double* rhs;
  double* divergence;
  double* wall_rhs_out;  // pressure_laplacian (holds the wall Neumann term, :367-369)
  // Mixed form: operator rows [Laplacian row, rows 0..2] per particle of the
  // velocity and pressure inverses, in place of vinv / pinv.
  MixedRows vrows;
  MixedRows prows;
  // 32-byte neighbour records (packed.cuh) for the lane kernels: fluid
  // {x, y, z, -} and {u*x, u*y, u*z, -}; walls {x, y, z, -},
  // {u*x, u*y, u*z, -} and {nx, ny, nz, -}.
  const double4* fp;
  const double4* fu;
  const double4* wp;
  const double4* wu;
  const double4* wn;
  const int32_t* order;  // visiting order of the lane kernel (lsmps_ctx::order) or NULL
  // The lane kernels' neighbour rows for the records: fi, or the table's
  // cell-sorted rows with fp / fu packed in that order (sorted = 1; a
  // column written is then order[sorted position], the neighbour's index:
  // the entries of nearby rows fall in a few lines of the cell list, where
  // fi[o] would be one more line per row).
  const index_t* fs;
  int sorted;
  // Merged batch (lsmps_ctx::box_ppe): each row written into its box's own
  // matrix, columns in the box's numbering; NULL: into col / val.
  const PpeBoxOut* box_out;
  const BoxGrid* boxes;
  int nbox;
  DeviceStatus* status;
};

// Where row i's slots go: the matrix given (r0 = the row's first slot), or,
// in a merged batch, its box's own matrix, with the box's first fluid index
// subtracted from every column (the box's rows start at merged slot
// fb + fo[fb]).  False (and the capacity flag raised with the slots the box
// needs so far) when the row does not fit its box's matrix: nothing of the
// row is written.
struct PpeDest {
  index_t* col;
  double* val;
  index_t r0;
  index_t shift;
};

__device__ __forceinline__ bool ppe_dest(const PpeArgs& a, index_t i, index_t row, index_t entries, PpeDest& d) {
  if (!a.box_out) {
    d = PpeDest{a.col, a.val, row, 0};
    return true;
  }
  const int bx = box_of(a.boxes, a.nbox, i, 1);
  const index_t fb = a.boxes[bx].fluid_base;
  const PpeBoxOut o = a.box_out[bx];
  d = PpeDest{o.col, o.val, row - (fb + a.fo[fb]), fb};
  const unsigned long long need = static_cast<unsigned long long>(d.r0) + 1ull + static_cast<unsigned long long>(entries);
  if (need > o.cap) {
    record_required(a.status, need);
    return false;
  }
  return true;
}

__device__ __forceinline__ double dot9(const double a[9], const double b[9]) {
  double v = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) v = fma(a[k], b[k], v);
  return v;
}

__device__ __forceinline__ void acc_rhs(const double b[9], double w, double ux, double uy, double uz, double rx[9],
                                        double ry[9], double rz[9]) {
#pragma unroll
  for (int r = 0; r < 9; ++r) {
    const double wb = w * b[r];
    rx[r] = fma(wb, ux, rx[r]);
    ry[r] = fma(wb, uy, ry[r]);
    rz[r] = fma(wb, uz, rz[r]);
  }
}

// (Gx . b) ux + (Gy . b) uy + (Gz . b) uz for one neighbour.
__device__ __forceinline__ double div_term(const double gx[9], const double gy[9], const double gz[9],
                                           const double b[9], double ux, double uy, double uz) {
  double cx = 0.0, cy = 0.0, cz = 0.0;
#pragma unroll
  for (int r = 0; r < 9; ++r) {
    cx = fma(gx[r], b[r], cx);
    cy = fma(gy[r], b[r], cy);
    cz = fma(gz[r], b[r], cz);
  }
  return fma(cx, ux, fma(cy, uy, cz * uz));
}

__device__ __forceinline__ double coeff_row(const double* __restrict__ inv, const double rhs[9], int row) {
  double c = 0.0;
#pragma unroll
  for (int col = 0; col < 9; ++col) c = fma(inv[row + col * 9], rhs[col], c);
  return c;
}

__global__ void __launch_bounds__(kThreads) ppe_kernel(PpeArgs a) {
  const index_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const index_t n = static_cast<index_t>(a.fluid.count);
  if (i >= n) return;
  const index_t nb = a.fo[i], ne = a.fo[i + 1];
  const index_t row = i + nb;
  a.row_offsets[i] = row;
  if (i + 1 == n) a.row_offsets[n] = n + ne;
  PpeDest d;
  if (!ppe_dest(a, i, row, ne - nb, d)) return;
  const int type = a.fluid.surface_type ? a.fluid.surface_type[i] : LSMPS_SURFACE_INNER;
  if (type == LSMPS_SURFACE_SURFACE || type == LSMPS_SURFACE_SPLASH) {
    d.col[d.r0] = i - d.shift;
    d.val[d.r0] = 1.0;
    for (index_t o = nb; o < ne; ++o) {
      d.col[d.r0 + 1 + o - nb] = a.fi[o] - d.shift;
      d.val[d.r0 + 1 + o - nb] = 0.0;
    }
    a.rhs[i] = 0.0;
    a.divergence[i] = 0.0;
    if (a.wall_rhs_out) a.wall_rhs_out[i] = 0.0;
    return;
  }
  const double* __restrict__ fx = a.fluid.x;
  const double* __restrict__ fy = a.fluid.y;
  const double* __restrict__ fz = a.fluid.z;
  const double xi = fx[i], yi = fy[i], zi = fz[i];
  // compute_pressure_laplacian_row, ppe_matrix.cu:203-215
  const double* __restrict__ pinv = a.pinv + static_cast<size_t>(i) * 81;
  double L[9];
#pragma unroll
  for (int col = 0; col < 9; ++col) L[col] = pinv[3 + col * 9] + pinv[4 + col * 9] + pinv[5 + col * 9];
  const double uxi = a.tvx[i], uyi = a.tvy[i], uzi = a.tvz[i];
  const double scale = 2.0 / (a.re * a.re * a.density);
  double rx[9], ry[9], rz[9], b[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) rx[r] = ry[r] = rz[r] = 0.0;
  double diag = 0.0;
  for (index_t o = nb; o < ne; ++o) {
    const index_t j = a.fi[o];
    const double dx = fx[j] - xi, dy = fy[j] - yi, dz = fz[j] - zi;
    const double w = lin_weight_mul(sqrt(dx * dx + dy * dy + dz * dz), a.inv_re);
    double off = 0.0;
    if (w > 0.0) {
      basis_a_mul(dx, dy, dz, a.inv_re, b);
      off = w * dot9(L, b) * scale;
      diag -= off;
      acc_rhs(b, w, a.tvx[j] - uxi, a.tvy[j] - uyi, a.tvz[j] - uzi, rx, ry, rz);
    }
    d.col[d.r0 + 1 + o - nb] = j - d.shift;
    d.val[d.r0 + 1 + o - nb] = off;
  }
  double wall_rhs = 0.0;
  const index_t we = a.wo[i + 1];
  for (index_t o = a.wo[i]; o < we; ++o) {
    const index_t j = a.wi[o];
    const double dx = a.walls.x[j] - xi, dy = a.walls.y[j] - yi, dz = a.walls.z[j] - zi;
    const double bw = lin_weight_mul(sqrt(dx * dx + dy * dy + dz * dz), a.inv_re);
    if (bw <= 0.0) continue;
    basis_a_mul(dx, dy, dz, a.inv_re, b);
    acc_rhs(b, a.vwall_scale * bw, a.twx[j] - uxi, a.twy[j] - uyi, a.twz[j] - uzi, rx, ry, rz);
    const double nx = a.walls.normal_x[j], ny = a.walls.normal_y[j], nz = a.walls.normal_z[j];
    const double ng = a.gx * nx + a.gy * ny + a.gz * nz;
    double q[9];
    neumann_a(dx, dy, dz, nx, ny, nz, a.inv_re, q);
    wall_rhs += 2.0 * a.pwall_scale * bw * ng * dot9(L, q) * a.inv_re;
  }
  const double* __restrict__ vinv = a.vinv + static_cast<size_t>(i) * 81;
  const double div = (coeff_row(vinv, rx, 0) + coeff_row(vinv, ry, 1) + coeff_row(vinv, rz, 2)) * a.inv_re;
  d.col[d.r0] = i - d.shift;
  d.val[d.r0] = diag;
  a.divergence[i] = div;
  a.rhs[i] = div / (a.dt_dev ? *a.dt_dev : a.dt) - wall_rhs;
  if (a.wall_rhs_out) a.wall_rhs_out[i] = wall_rhs;
}

// The same row with G lanes per particle: lane l takes the neighbours
// nb + l, nb + l + G, ..., so the G lanes write G consecutive (col, val)
// slots per round and issue G independent gathers.  The partial sums (the
// diagonal, the 27 divergence moments and the wall Neumann term) are added
// across the group with shuffles; lane 0 finishes the row.  The sums are
// associated differently from the one-lane kernel (rounding-level change).
//
// Mixed (the mixed form): the pressure Laplacian row L comes from the
// pressure operator rows and the divergence rows from the velocity operator
// rows (FP32, or FP64 for FP64-route particles); geometry, coefficients, the
// diagonal (minus the sum of the off-diagonal values) and the RHS sums stay
// FP64.
template <int G, bool Mixed>
__device__ __forceinline__ void ppe_row(const PpeArgs& a, index_t i, index_t vt, int l, bool write_offsets) {
  const index_t self = self_of(a.sorted, vt, i);
  const index_t n = static_cast<index_t>(a.fluid.count);
  const index_t nb = a.fo[i], ne = a.fo[i + 1];
  const index_t row = i + nb;
  if (l == 0 && write_offsets) {
    a.row_offsets[i] = row;
    if (i + 1 == n) a.row_offsets[n] = n + ne;
  }
  PpeDest d;
  if (!ppe_dest(a, i, row, ne - nb, d)) return;  // uniform over the lane group
  const int type = a.fluid.surface_type ? a.fluid.surface_type[i] : LSMPS_SURFACE_INNER;
  if (type == LSMPS_SURFACE_SURFACE || type == LSMPS_SURFACE_SPLASH) {
    for (index_t o = nb + l; o < ne; o += G) {
      d.col[d.r0 + 1 + o - nb] = a.fi[o] - d.shift;
      d.val[d.r0 + 1 + o - nb] = 0.0;
    }
    if (l == 0) {
      d.col[d.r0] = i - d.shift;
      d.val[d.r0] = 1.0;
      a.rhs[i] = 0.0;
      a.divergence[i] = 0.0;
      if (a.wall_rhs_out) a.wall_rhs_out[i] = 0.0;
    }
    return;
  }
  const double4 pi = ld4(a.fp, self);
  const double xi = pi.x, yi = pi.y, zi = pi.z;
  // The pressure Laplacian row, once per group in shared memory: read by
  // broadcast in every neighbour's dot product, it holds no registers.
  __shared__ double s_L[kThreads / G][9];
  double* L = s_L[threadIdx.x / G];
  if (l == 0) {
    double Lr[9];
    if (Mixed) {
      load_row9(a.prows, vt, 0, Lr);
    } else {
      const double* __restrict__ pinv = a.pinv + static_cast<size_t>(i) * 81;
#pragma unroll
      for (int col = 0; col < 9; ++col) Lr[col] = pinv[3 + col * 9] + pinv[4 + col * 9] + pinv[5 + col * 9];
    }
#pragma unroll
    for (int col = 0; col < 9; ++col) L[col] = Lr[col];
  }
  __syncwarp(group_mask<G>());
  const double uxi = a.tvx[i], uyi = a.tvy[i], uzi = a.tvz[i];
  const double scale = 2.0 / (a.re * a.re * a.density);
  // The velocity gradient rows (rows 0..2 of the velocity inverse, or the
  // mixed-form rows 1..3) are applied to each neighbour's basis vector:
  // sum_j w_j sum_c (G_c . b_j) du_c,j equals sum_c G_c . sum_j w_j b_j du_c,j
  // up to rounding, with one accumulator instead of 27.
  double gx[9], gy[9], gz[9], b[9];
  if (Mixed) {
    load_row9(a.vrows, vt, 1, gx);
    load_row9(a.vrows, vt, 2, gy);
    load_row9(a.vrows, vt, 3, gz);
  } else {
    const double* __restrict__ vinv = a.vinv + static_cast<size_t>(i) * 81;
#pragma unroll
    for (int col = 0; col < 9; ++col) {
      gx[col] = vinv[0 + col * 9];
      gy[col] = vinv[1 + col * 9];
      gz[col] = vinv[2 + col * 9];
    }
  }
  double dsum = 0.0;
  double diag = 0.0;
  // Each lane loads its next neighbour's records, and the index after that,
  // while it works on this one.
  index_t o = nb + l;
  index_t jn = o < ne ? a.fs[o] : i;
  index_t jnn = o + G < ne ? a.fs[o + G] : i;
  double4 qn = ld4(a.fp, jn), un = ld4(a.fu, jn);
  index_t cn = a.sorted ? a.order[jn] : jn;
  for (; o < ne; o += G) {
    const index_t j = cn;  // the column
    const double4 q = qn, u = un;
    if (o + G < ne) {
      jn = jnn;
      qn = ld4(a.fp, jn);
      un = ld4(a.fu, jn);
      cn = a.sorted ? a.order[jn] : jn;
      if (o + 2 * G < ne) jnn = a.fs[o + 2 * G];
    }
    const double dx = q.x - xi, dy = q.y - yi, dz = q.z - zi;
    const double w = lin_weight_mul(sqrt(dx * dx + dy * dy + dz * dz), a.inv_re);
    double off = 0.0;
    if (w > 0.0) {
      basis_a_mul(dx, dy, dz, a.inv_re, b);
      off = w * dot9(L, b) * scale;
      diag -= off;
      dsum = fma(w, div_term(gx, gy, gz, b, u.x - uxi, u.y - uyi, u.z - uzi), dsum);
    }
    d.col[d.r0 + 1 + o - nb] = j - d.shift;
    d.val[d.r0 + 1 + o - nb] = off;
  }
  double wall_rhs = 0.0;
  const index_t we = a.wo[i + 1];
  for (index_t o = a.wo[i] + l; o < we; o += G) {
    const index_t j = a.wi[o];
    const double4 q = ld4(a.wp, j), u = ld4(a.wu, j), nrm = ld4(a.wn, j);
    const double dx = q.x - xi, dy = q.y - yi, dz = q.z - zi;
    const double bw = lin_weight_mul(sqrt(dx * dx + dy * dy + dz * dz), a.inv_re);
    if (bw <= 0.0) continue;
    basis_a_mul(dx, dy, dz, a.inv_re, b);
    dsum = fma(a.vwall_scale * bw, div_term(gx, gy, gz, b, u.x - uxi, u.y - uyi, u.z - uzi), dsum);
    const double nx = nrm.x, ny = nrm.y, nz = nrm.z;
    const double ng = a.gx * nx + a.gy * ny + a.gz * nz;
    double qn9[9];
    neumann_a(dx, dy, dz, nx, ny, nz, a.inv_re, qn9);
    wall_rhs += 2.0 * a.pwall_scale * bw * ng * dot9(L, qn9) * a.inv_re;
  }
  const unsigned mask = group_mask<G>();
  diag = group_sum<G>(diag, mask);
  wall_rhs = group_sum<G>(wall_rhs, mask);
  dsum = group_sum<G>(dsum, mask);
  if (l != 0) return;
  const double div = dsum * a.inv_re;
  d.col[d.r0] = i - d.shift;
  d.val[d.r0] = diag;
  a.divergence[i] = div;
  a.rhs[i] = div / (a.dt_dev ? *a.dt_dev : a.dt) - wall_rhs;
  if (a.wall_rhs_out) a.wall_rhs_out[i] = wall_rhs;
}

template <int G, bool Mixed>
__global__ void __launch_bounds__(kThreads, 4) ppe_lanes_kernel(PpeArgs a) {
  const index_t t = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int l = threadIdx.x & (G - 1);
  // Whole groups leave together, so the shuffles see full groups.
  if (t >= static_cast<index_t>(a.fluid.count)) return;
  const index_t i = visit(a.order, t);
  ppe_row<G, Mixed>(a, i, t, l, true);
}

// The mixed form with FP32 arithmetic; the particles whose rows took the
// FP64 route get their row offsets here and their rows from ppe_list_kernel.
//
// FP32 arithmetic: each neighbour's offset is formed in FP64 and rounded
// once to FP32 (r_e-scaled); distance, weight, basis, the coefficient
// a_ij = 2 w (L . b) / (r_e^2 rho) and the divergence term are FP32, with the
// FP32 operator rows; the diagonal (minus the sum of the stored off-diagonal
// values), the divergence sum and the wall Neumann sum accumulate in FP64.
template <int G>
__device__ __forceinline__ void ppe_row32(const PpeArgs& a, index_t i, index_t vt, int l) {
  const index_t self = self_of(a.sorted, vt, i);
  const index_t n = static_cast<index_t>(a.fluid.count);
  const index_t nb = a.fo[i], ne = a.fo[i + 1];
  const index_t row = i + nb;
  if (l == 0) {
    a.row_offsets[i] = row;
    if (i + 1 == n) a.row_offsets[n] = n + ne;
  }
  if (a.vrows.flag[vt] | a.prows.flag[vt]) return;  // FP64 rows: ppe_list_kernel
  PpeDest d;
  if (!ppe_dest(a, i, row, ne - nb, d)) return;  // uniform over the lane group
  const int type = a.fluid.surface_type ? a.fluid.surface_type[i] : LSMPS_SURFACE_INNER;
  if (type == LSMPS_SURFACE_SURFACE || type == LSMPS_SURFACE_SPLASH) {
    for (index_t o = nb + l; o < ne; o += G) {
      d.col[d.r0 + 1 + o - nb] = a.fi[o] - d.shift;
      d.val[d.r0 + 1 + o - nb] = 0.0;
    }
    if (l == 0) {
      d.col[d.r0] = i - d.shift;
      d.val[d.r0] = 1.0;
      a.rhs[i] = 0.0;
      a.divergence[i] = 0.0;
      if (a.wall_rhs_out) a.wall_rhs_out[i] = 0.0;
    }
    return;
  }
  const double4 pi = ld4(a.fp, self);
  // The group's four operator rows in shared memory (read by broadcast in
  // every neighbour's dot products; they hold no registers): the pressure
  // Laplacian row L, then the velocity gradient rows 0, 1, 2, each padded to
  // 12 floats so that every row starts on 16 bytes and is read as two float4
  // and one float.  Within a quarter warp the groups' rows sit 48 floats
  // apart: different banks.
  __shared__ __align__(16) float s_rows[kThreads / G][48];
  float* L = s_rows[threadIdx.x / G];
  const float* gx = L + 12;
  const float* gy = L + 24;
  const float* gz = L + 36;
  for (int c = l; c < 36; c += G)
    L[(c / 9) * 12 + c % 9] =
        c < 9 ? a.prows.f32[static_cast<size_t>(vt) * 36 + c] : a.vrows.f32[static_cast<size_t>(vt) * 36 + c];
  __syncwarp(group_mask<G>());
  float b[9];
  const double uxi = a.tvx[i], uyi = a.tvy[i], uzi = a.tvz[i];
  const float scale = static_cast<float>(2.0 / (a.re * a.re * a.density));
  double dsum = 0.0, diag = 0.0;
  index_t o = nb + l;
  index_t jn = o < ne ? a.fs[o] : i;
  index_t jnn = o + G < ne ? a.fs[o + G] : i;
  double4 qn = ld4(a.fp, jn), un = ld4(a.fu, jn);
  index_t cn = a.sorted ? a.order[jn] : jn;
  for (; o < ne; o += G) {
    const index_t j = cn;  // the column
    const double4 q = qn, u = un;
    if (o + G < ne) {
      jn = jnn;
      qn = ld4(a.fp, jn);
      un = ld4(a.fu, jn);
      cn = a.sorted ? a.order[jn] : jn;
      if (o + 2 * G < ne) jnn = a.fs[o + 2 * G];
    }
    const float w = basis_f32(q.x - pi.x, q.y - pi.y, q.z - pi.z, a.inv_re, b);
    float off = 0.0f;
    if (w > 0.0f) {
      off = w * dot9f_a16(L, b) * scale;
      diag -= static_cast<double>(off);
      const float dux = static_cast<float>(u.x - uxi), duy = static_cast<float>(u.y - uyi),
                  duz = static_cast<float>(u.z - uzi);
      const float cx = dot9f_a16(gx, b), cy = dot9f_a16(gy, b), cz = dot9f_a16(gz, b);
      dsum += static_cast<double>(w * fmaf(cx, dux, fmaf(cy, duy, cz * duz)));
    }
    d.col[d.r0 + 1 + o - nb] = j - d.shift;
    d.val[d.r0 + 1 + o - nb] = static_cast<double>(off);
  }
  double wall_rhs = 0.0;
  const index_t we = a.wo[i + 1];
  const float vws = static_cast<float>(a.vwall_scale);
  const float pws = static_cast<float>(2.0 * a.pwall_scale);
  {  // the next wall's records are loaded while this one is used
    index_t o = a.wo[i] + l;
    index_t jn = o < we ? a.wi[o] : 0;
    double4 qn = make_double4(0.0, 0.0, 0.0, 0.0), un = qn, nrmn = qn;
    if (o < we) {
      qn = ld4(a.wp, jn);
      un = ld4(a.wu, jn);
      nrmn = ld4(a.wn, jn);
    }
    for (; o < we; o += G) {
      const double4 q = qn, u = un, nrm = nrmn;
      if (o + G < we) {
        jn = a.wi[o + G];
        qn = ld4(a.wp, jn);
        un = ld4(a.wu, jn);
        nrmn = ld4(a.wn, jn);
      }
      const float w = basis_f32(q.x - pi.x, q.y - pi.y, q.z - pi.z, a.inv_re, b);
      if (w <= 0.0f) continue;
      const float dux = static_cast<float>(u.x - uxi), duy = static_cast<float>(u.y - uyi),
                  duz = static_cast<float>(u.z - uzi);
      const float cx = dot9f_a16(gx, b), cy = dot9f_a16(gy, b), cz = dot9f_a16(gz, b);
      dsum += static_cast<double>(vws * w * fmaf(cx, dux, fmaf(cy, duy, cz * duz)));
      const float nx = static_cast<float>(nrm.x), ny = static_cast<float>(nrm.y), nz = static_cast<float>(nrm.z);
      // wall Neumann vector (moment_matrix.cu:177-201) of the scaled offset
      const float q9[9] = {nx, ny, nz, 2.0f * b[0] * nx, 2.0f * b[1] * ny, 2.0f * b[2] * nz,
                           fmaf(b[1], nx, b[0] * ny), fmaf(b[2], ny, b[1] * nz), fmaf(b[0], nz, b[2] * nx)};
      const double ng = a.gx * nrm.x + a.gy * nrm.y + a.gz * nrm.z;
      wall_rhs += static_cast<double>(pws * w * dot9f_a16(L, q9)) * ng * a.inv_re;
  }
  }
  const unsigned mask = group_mask<G>();
  diag = group_sum<G>(diag, mask);
  wall_rhs = group_sum<G>(wall_rhs, mask);
  dsum = group_sum<G>(dsum, mask);
  if (l != 0) return;
  const double div = dsum * a.inv_re;
  d.col[d.r0] = i - d.shift;
  d.val[d.r0] = diag;
  a.divergence[i] = div;
  a.rhs[i] = div / (a.dt_dev ? *a.dt_dev : a.dt) - wall_rhs;
  if (a.wall_rhs_out) a.wall_rhs_out[i] = wall_rhs;
}

template <int G>
__global__ void __launch_bounds__(kThreads, 7) ppe32_kernel(PpeArgs a) {
  const index_t t = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int l = threadIdx.x & (G - 1);
  if (t >= static_cast<index_t>(a.fluid.count)) return;
  const index_t i = visit(a.order, t);
  ppe_row32<G>(a, i, t, l);
}

// The rows of the FP64-route particles (FP64 arithmetic, ppe_row<G, true>):
// first every particle of the velocity kind's list, then those of the
// pressure kind's list that are not on the velocity kind's.  Lane groups
// stride over the lists.
template <int G>
__global__ void __launch_bounds__(kThreads, 4) ppe_list_kernel(PpeArgs a) {
  const index_t groups = static_cast<index_t>(gridDim.x * blockDim.x / G);
  const index_t g0 = static_cast<index_t>((blockIdx.x * blockDim.x + threadIdx.x) / G);
  const int l = threadIdx.x & (G - 1);
  const index_t nv = static_cast<index_t>(*a.vrows.count), np = static_cast<index_t>(*a.prows.count);
  for (index_t t = g0; t < nv + np; t += groups) {
    const index_t vt = t < nv ? a.vrows.list[t] : a.prows.list[t - nv];  // a visiting position
    const index_t i = visit(a.order, vt);
    if (t >= nv && a.vrows.flag[vt]) continue;
    ppe_row<G, true>(a, i, vt, l, false);
  }
}

// Neighbour records of the lane kernels: positions and u* of the fluid,
// positions, u* and normals of the walls.
bool pack_ppe(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w, const lsmps_fluid& tv,
              const lsmps_walls& tw, const lsmps_csr& fn, PpeArgs& a) {
  if (!ensure_packs(ctx, f.count, w.count)) return false;
  const index_t* srows = sorted_rows_of(ctx, fn, f.count);
  a.fs = srows ? srows : a.fi;
  a.sorted = srows ? 1 : 0;
  pack_fluid_positions(ctx, f, srows ? ctx->order : nullptr);
  pack4(ctx, tv.vx, tv.vy, tv.vz, nullptr, f.count, ctx->pack_fluid[1], srows ? ctx->order : nullptr);
  pack_wall_positions(ctx, w);
  pack4(ctx, tw.vx, tw.vy, tw.vz, nullptr, w.count, ctx->pack_wall[1]);
  pack_wall_normals(ctx, w);
  a.fp = ctx->pack_fluid[0];
  a.fu = ctx->pack_fluid[1];
  a.wp = ctx->pack_wall[0];
  a.wu = ctx->pack_wall[1];
  a.wn = ctx->pack_wall[2];
  return true;
}

}  // namespace

lsmps_status assemble_ppe_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w, const lsmps_params& p,
                               const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_fluid& tv,
                               const lsmps_walls& tw, const lsmps_moment& vm, const lsmps_moment& pm,
                               const lsmps_ppe& ws) {
  // validate_matrix_workspace, ppe_matrix.cu:62-84 (nnz checked against the
  // CSR capacity, as the reference does).
  if (ws.matrix.rows < f.count || ws.matrix.cols < f.count || ws.matrix.nnz < f.count + fn.neighbor_count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "PPE matrix workspace is smaller than the requested fluid system");
  if (vm.kind != LSMPS_MOMENT_VELOCITY_WALL_DIRICHLET_A || vm.matrix_size != 9 || vm.particle_count < f.count)
    return fail(ctx, LSMPS_NOT_PREPARED, "PPE requires a prepared velocity Type-A moment matrix");
  if (pm.kind != LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_A || pm.matrix_size != 9 || pm.particle_count < f.count)
    return fail(ctx, LSMPS_NOT_PREPARED, "PPE requires a prepared pressure Type-A moment matrix");
  if (f.count == 0) return LSMPS_OK;
  if (const lsmps_status cs = check_neighbor_tables(ctx, f.count, w.count, fn, &wn)) return cs;
  if (!ws.matrix.row_offsets || !ws.matrix.col_indices || !ws.matrix.values || !ws.rhs || !ws.divergence ||
      !tv.vx || !tv.vy || !tv.vz || !vm.inverse_matrices || !pm.inverse_matrices)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "PPE workspace requires matrix, rhs, divergence and velocity buffers");
  if (tw.count > 0 && (!tw.vx || !tw.vy || !tw.vz))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "PPE RHS assembly requires temporary wall velocity buffers");
  PpeArgs a{};
  a.fluid = f;
  a.walls = w;
  a.fo = fn.offsets;
  a.fi = fn.indices;
  a.wo = wn.offsets;
  a.wi = wn.indices;
  a.tvx = tv.vx;
  a.tvy = tv.vy;
  a.tvz = tv.vz;
  a.twx = tw.vx;
  a.twy = tw.vy;
  a.twz = tw.vz;
  a.vinv = vm.inverse_matrices;
  a.pinv = pm.inverse_matrices;
  a.re = pm.support_radius;
  a.inv_re = 1.0 / pm.support_radius;
  a.vwall_scale = vm.wall_weight_scale;
  a.pwall_scale = pm.wall_weight_scale;
  a.density = p.density;
  a.dt = p.time_step;
  a.dt_dev = ctx->device_dt;
  a.gx = p.gravity[0];
  a.gy = p.gravity[1];
  a.gz = p.gravity[2];
  a.row_offsets = ws.matrix.row_offsets;
  a.order = ctx->order;
  a.col = ws.matrix.col_indices;
  a.val = ws.matrix.values;
  a.box_out = ctx->box_ppe;
  a.boxes = ctx->boxes;
  a.nbox = ctx->nbox;
  a.status = ctx->d_status;
  a.rhs = ws.rhs;
  a.divergence = ws.divergence;
  a.wall_rhs_out = ws.pressure_laplacian;
  a.fs = a.fi;
  if (ctx->knob[LSMPS_KNOB_PPE_LANES] != 0 && !pack_ppe(ctx, f, w, tv, tw, fn, a))
    return fail(ctx, LSMPS_CUDA_ERROR, "pack allocation failed");
  const long long rows = static_cast<long long>(f.count);
  switch (ctx->knob[LSMPS_KNOB_PPE_LANES]) {
    case 1: launch_named(ctx, "ppe_lanes_kernel<4, false>", ppe_lanes_kernel<4, false>, dim3(div_up(rows * 4, kThreads)), dim3(kThreads), 0, a); break;
    case 2: launch_named(ctx, "ppe_lanes_kernel<8, false>", ppe_lanes_kernel<8, false>, dim3(div_up(rows * 8, kThreads)), dim3(kThreads), 0, a); break;
    case 3: launch_named(ctx, "ppe_lanes_kernel<16, false>", ppe_lanes_kernel<16, false>, dim3(div_up(rows * 16, kThreads)), dim3(kThreads), 0, a); break;
    default: launch(ctx, ppe_kernel, dim3(div_up(rows, kThreads)), dim3(kThreads), 0, a); break;
  }
  return check_launch(ctx, "PPE assembly");
}

lsmps_status assemble_ppe_mixed_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w,
                                     const lsmps_params& p, const lsmps_csr& fn, const lsmps_csr& wn,
                                     const lsmps_fluid& tv, const lsmps_walls& tw, const lsmps_moment& vm,
                                     const lsmps_moment& pm, const lsmps_ppe& ws) {
  if (ws.matrix.rows < f.count || ws.matrix.cols < f.count || ws.matrix.nnz < f.count + fn.neighbor_count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "PPE matrix workspace is smaller than the requested fluid system");
  if (f.count == 0) return LSMPS_OK;
  if (const lsmps_status cs = check_neighbor_tables(ctx, f.count, w.count, fn, &wn)) return cs;
  if (!ws.matrix.row_offsets || !ws.matrix.col_indices || !ws.matrix.values || !ws.rhs || !ws.divergence ||
      !tv.vx || !tv.vy || !tv.vz)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "PPE workspace requires matrix, rhs, divergence and velocity buffers");
  if (tw.count > 0 && (!tw.vx || !tw.vy || !tw.vz))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "PPE RHS assembly requires temporary wall velocity buffers");
  if (!ctx->mixed_rows[0] || !ctx->mixed_rows[1] || !ctx->mixed_count || ctx->mixed_cap < f.count)
    return fail(ctx, LSMPS_NOT_PREPARED, "mixed operator rows were not prepared");
  PpeArgs a{};
  a.fluid = f;
  a.walls = w;
  a.fo = fn.offsets;
  a.fi = fn.indices;
  a.wo = wn.offsets;
  a.wi = wn.indices;
  a.tvx = tv.vx;
  a.tvy = tv.vy;
  a.tvz = tv.vz;
  a.twx = tw.vx;
  a.twy = tw.vy;
  a.twz = tw.vz;
  a.vrows = mixed_rows_of(ctx, 0);
  a.prows = mixed_rows_of(ctx, 1);
  a.re = pm.support_radius;
  a.inv_re = 1.0 / pm.support_radius;
  a.vwall_scale = vm.wall_weight_scale;
  a.pwall_scale = pm.wall_weight_scale;
  a.density = p.density;
  a.dt = p.time_step;
  a.dt_dev = ctx->device_dt;
  a.gx = p.gravity[0];
  a.gy = p.gravity[1];
  a.gz = p.gravity[2];
  a.row_offsets = ws.matrix.row_offsets;
  a.order = ctx->order;
  a.col = ws.matrix.col_indices;
  a.val = ws.matrix.values;
  a.box_out = ctx->box_ppe;
  a.boxes = ctx->boxes;
  a.nbox = ctx->nbox;
  a.status = ctx->d_status;
  a.rhs = ws.rhs;
  a.divergence = ws.divergence;
  a.wall_rhs_out = ws.pressure_laplacian;
  if (!pack_ppe(ctx, f, w, tv, tw, fn, a)) return fail(ctx, LSMPS_CUDA_ERROR, "pack allocation failed");
  const long long rows = static_cast<long long>(f.count);
  const dim3 list_grid(static_cast<unsigned>(ctx->sm_count * 2));
  switch (ctx->knob[LSMPS_KNOB_PPE_LANES]) {
    case 0:
    case 1:
      launch_named(ctx, "ppe32_kernel<4>", ppe32_kernel<4>, dim3(div_up(rows * 4, kThreads)), dim3(kThreads), 0, a);
      launch_named(ctx, "ppe_list_kernel<4>", ppe_list_kernel<4>, list_grid, dim3(kThreads), 0, a);
      break;
    case 3:
      launch_named(ctx, "ppe32_kernel<16>", ppe32_kernel<16>, dim3(div_up(rows * 16, kThreads)), dim3(kThreads), 0, a);
      launch_named(ctx, "ppe_list_kernel<16>", ppe_list_kernel<16>, list_grid, dim3(kThreads), 0, a);
      break;
    default:
      launch_named(ctx, "ppe32_kernel<8>", ppe32_kernel<8>, dim3(div_up(rows * 8, kThreads)), dim3(kThreads), 0, a);
      launch_named(ctx, "ppe_list_kernel<8>", ppe_list_kernel<8>, list_grid, dim3(kThreads), 0, a);
      break;
  }
  return check_launch(ctx, "PPE assembly (mixed)");
}

}  // namespace lsmps

using namespace lsmps;

extern "C" lsmps_status lsmps_assemble_ppe(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_walls* walls,
                                           const lsmps_params* params, const lsmps_csr* fn, const lsmps_csr* wn,
                                           const lsmps_fluid* tv, const lsmps_walls* tw, const lsmps_moment* vm,
                                           const lsmps_moment* pm, const lsmps_ppe* ws) {
  if (!ctx || !fluid || !walls || !params || !fn || !wn || !tv || !tw || !vm || !pm || !ws)
    return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  return end_call(ctx, assemble_ppe_impl(ctx, *fluid, *walls, *params, *fn, *wn, *tv, *tw, *vm, *pm, *ws));
}
