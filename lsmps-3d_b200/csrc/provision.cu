// provision.cu - explicit viscous/gravity update u* (the PPE's velocity input).
// Replaces DeviceProvisionExplicitUpdate::compute_temporary_velocity of
// src/provision/explicit_update.cu:366-399: compute_velocity_laplacian_kernel
// (:178-248), combine_explicit_velocity_kernel (:250-270) and
// combine_explicit_wall_velocity_kernel (:272-284).  The reference sums the
// moment right-hand sides sum_j w_j b_j (u_j - u_i) (accumulate_velocity_rhs,
// :148-162) and then applies rows 3..5 of the inverse
// (laplacian_from_inverse_rhs, :164-176); laplacian_kernel applies the summed
// row to each neighbour's basis vector instead (the same value up to
// rounding, fewer operations and registers).
#include "impl.cuh"
#include "mixed.cuh"
#include "packed.cuh"

namespace lsmps {
namespace {

constexpr int kThreads = 128;

// Neighbour records: fp = {x, y, z, 0}, fv = {vx, vy, vz, 0} per fluid
// particle, wp / wv the same for walls (packed.cuh).
struct LaplacianArgs {
  index_t n;
  const double4* fp;
  const double4* fv;
  const double4* wp;
  const double4* wv;
  const index_t* fo;
  const index_t* fi;
  const index_t* wo;
  const index_t* wi;
  const double* inverse;
  double re;
  double inv_re;
  double wall_scale;
  double* lx;
  double* ly;
  double* lz;
  const int32_t* order;  // visiting order (lsmps_ctx::order) or NULL
  int sorted;            // fi and the fluid packs in cell-sorted positions (sorted_rows_of)
};

// Mixed (the mixed form): the row comes from the mixed-form operator rows
// (FP32, or FP64 for the FP64-route particles); the sums are the same FP64
// sums.
//
// G lanes per particle (G = 1, 2, 4; LSMPS_KNOB_GATHER_LANES): lane l sums the
// entries l, l + G, ... of both rows and the groups' partial sums are added
// with shuffles (a rounding-level reassociation for G > 1).
template <bool Mixed, int G>
__device__ __forceinline__ void laplacian_of(const LaplacianArgs& a, const MixedRows& rows, index_t i, index_t vt,
                                             int l) {
  const index_t self = self_of(a.sorted, vt, i);
  const double4 pi = ld4(a.fp, self);
  const double4 ui = ld4(a.fv, self);
  // The particle's Laplacian row L (the sum of the inverse's rows 3..5, or
  // the mixed-form row) is applied to every neighbour's basis vector:
  // sum_j w_j (L . b_j) (u_j - u_i) equals L . sum_j w_j b_j (u_j - u_i) up
  // to rounding, with 13 FP64 operations per neighbour instead of 36 and
  // three accumulators instead of 27.
  double L[9];
  if (Mixed) {
    load_row9(rows, vt, 0, L);
  } else {
    const double* __restrict__ inv = a.inverse + static_cast<size_t>(i) * 81;
#pragma unroll
    for (int col = 0; col < 9; ++col) L[col] = inv[3 + col * 9] + inv[4 + col * 9] + inv[5 + col * 9];
  }
  double b[9], cx = 0.0, cy = 0.0, cz = 0.0;
  const index_t fe = a.fo[i + 1];
  index_t o = a.fo[i] + l;
  index_t jn = o < fe ? a.fi[o] : i;
  index_t jnn = o + G < fe ? a.fi[o + G] : i;
  double4 qn = ld4(a.fp, jn), un = ld4(a.fv, jn);
  for (; o < fe; o += G) {
    // the next neighbour's records, and the index after that, are loaded
    // while this one is summed
    const double4 q = qn, u = un;
    if (o + G < fe) {
      jn = jnn;
      qn = ld4(a.fp, jn);
      un = ld4(a.fv, jn);
      if (o + 2 * G < fe) jnn = a.fi[o + 2 * G];
    }
    const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
    const double w = lin_weight_mul(sqrt(dx * dx + dy * dy + dz * dz), a.inv_re);
    if (w <= 0.0) continue;
    basis_a_mul(dx, dy, dz, a.inv_re, b);
    double lb = 0.0;
#pragma unroll
    for (int r = 0; r < 9; ++r) lb = fma(L[r], b[r], lb);
    const double s = w * lb;
    cx = fma(s, u.x - ui.x, cx);
    cy = fma(s, u.y - ui.y, cy);
    cz = fma(s, u.z - ui.z, cz);
  }
  const index_t we = a.wo[i + 1];
  {  // the next wall's records are loaded while this one is used
    index_t o = a.wo[i] + l;
    index_t jn = o < we ? a.wi[o] : 0;
    double4 qn = make_double4(0.0, 0.0, 0.0, 0.0), un = qn;
    if (o < we) {
      qn = ld4(a.wp, jn);
      un = ld4(a.wv, jn);
    }
    for (; o < we; o += G) {
      const double4 q = qn, u = un;
      if (o + G < we) {
        jn = a.wi[o + G];
        qn = ld4(a.wp, jn);
        un = ld4(a.wv, jn);
      }
      const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
      const double w = a.wall_scale * lin_weight_mul(sqrt(dx * dx + dy * dy + dz * dz), a.inv_re);
      if (w <= 0.0) continue;
      basis_a_mul(dx, dy, dz, a.inv_re, b);
      double lb = 0.0;
#pragma unroll
      for (int r = 0; r < 9; ++r) lb = fma(L[r], b[r], lb);
      const double s = w * lb;
      cx = fma(s, u.x - ui.x, cx);
      cy = fma(s, u.y - ui.y, cy);
      cz = fma(s, u.z - ui.z, cz);
  }
  }
  if (G > 1) {
    const unsigned mask = group_mask<G>();
    cx = group_sum<G>(cx, mask);
    cy = group_sum<G>(cy, mask);
    cz = group_sum<G>(cz, mask);
    if (l != 0) return;
  }
  const double scale = 2.0 / (a.re * a.re);
  a.lx[i] = scale * cx;
  a.ly[i] = scale * cy;
  a.lz[i] = scale * cz;
}

template <bool Mixed, int G>
__global__ void __launch_bounds__(kThreads, 5) laplacian_kernel(LaplacianArgs a, MixedRows rows) {
  const index_t t = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int l = threadIdx.x & (G - 1);
  if (t >= a.n) return;  // the whole group
  const index_t i = visit(a.order, t);
  laplacian_of<Mixed, G>(a, rows, i, t, l);
}

// Mixed form with FP32 arithmetic: each neighbour's offset is formed in FP64
// and rounded once to FP32 (r_e-scaled); distance, weight, basis and the
// coefficient w (L . b) with the FP32 Laplacian row are FP32; the coefficient
// times the FP64 velocity difference accumulates in FP64.  Particles whose
// velocity rows took the FP64 route are left to laplacian_list_kernel.
template <int G>
__global__ void __launch_bounds__(kThreads, 7) laplacian32_kernel(LaplacianArgs a, MixedRows rows) {
  const index_t t = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int l = threadIdx.x & (G - 1);
  if (t >= a.n) return;  // the whole group
  const index_t i = visit(a.order, t);
  if (rows.flag[t]) return;
  const index_t self = self_of(a.sorted, t, i);
  const double4 pi = ld4(a.fp, self);
  const double4 ui = ld4(a.fv, self);
  // the Laplacian row in registers (9 floats)
  float L[9];
  load_row9f(rows, t, 0, L);
  float b[9];
  double cx = 0.0, cy = 0.0, cz = 0.0;
  const index_t fe = a.fo[i + 1];
  index_t o = a.fo[i] + l;
  index_t jn = o < fe ? a.fi[o] : i;
  index_t jnn = o + G < fe ? a.fi[o + G] : i;
  double4 qn = ld4(a.fp, jn), un = ld4(a.fv, jn);
  for (; o < fe; o += G) {
    const double4 q = qn, u = un;
    if (o + G < fe) {
      jn = jnn;
      qn = ld4(a.fp, jn);
      un = ld4(a.fv, jn);
      if (o + 2 * G < fe) jnn = a.fi[o + 2 * G];
    }
    const float w = basis_f32(q.x - pi.x, q.y - pi.y, q.z - pi.z, a.inv_re, b);
    if (w <= 0.0f) continue;
    const double s = static_cast<double>(w * dot9f(L, b));
    cx = fma(s, u.x - ui.x, cx);
    cy = fma(s, u.y - ui.y, cy);
    cz = fma(s, u.z - ui.z, cz);
  }
  const float wall_scale = static_cast<float>(a.wall_scale);
  const index_t we = a.wo[i + 1];
  {  // the next wall's records are loaded while this one is used
    index_t o = a.wo[i] + l;
    index_t jn = o < we ? a.wi[o] : 0;
    double4 qn = make_double4(0.0, 0.0, 0.0, 0.0), un = qn;
    if (o < we) {
      qn = ld4(a.wp, jn);
      un = ld4(a.wv, jn);
    }
    for (; o < we; o += G) {
      const double4 q = qn, u = un;
      if (o + G < we) {
        jn = a.wi[o + G];
        qn = ld4(a.wp, jn);
        un = ld4(a.wv, jn);
      }
      const float w = wall_scale * basis_f32(q.x - pi.x, q.y - pi.y, q.z - pi.z, a.inv_re, b);
      if (w <= 0.0f) continue;
      const double s = static_cast<double>(w * dot9f(L, b));
      cx = fma(s, u.x - ui.x, cx);
      cy = fma(s, u.y - ui.y, cy);
      cz = fma(s, u.z - ui.z, cz);
  }
  }
  if (G > 1) {
    const unsigned mask = group_mask<G>();
    cx = group_sum<G>(cx, mask);
    cy = group_sum<G>(cy, mask);
    cz = group_sum<G>(cz, mask);
    if (l != 0) return;
  }
  const double scale = 2.0 / (a.re * a.re);
  a.lx[i] = scale * cx;
  a.ly[i] = scale * cy;
  a.lz[i] = scale * cz;
}

// The FP64-route particles of the velocity kind (FP64 arithmetic,
// laplacian_of<true, G>); lane groups stride over the list.
template <int G>
__global__ void __launch_bounds__(kThreads, 5) laplacian_list_kernel(LaplacianArgs a, MixedRows rows) {
  const index_t groups = static_cast<index_t>(gridDim.x * blockDim.x / G);
  const int l = threadIdx.x & (G - 1);
  const index_t count = static_cast<index_t>(*rows.count);
  for (index_t t = static_cast<index_t>((blockIdx.x * blockDim.x + threadIdx.x) / G); t < count; t += groups) {
    const index_t vt = rows.list[t];  // a visiting position
    const index_t i = visit(a.order, vt);
    laplacian_of<true, G>(a, rows, i, vt, l);
  }
}

// combine_explicit_velocity_kernel, explicit_update.cu:250-270
__global__ void combine_kernel(lsmps_fluid f, lsmps_params p, const double* __restrict__ lx,
                               const double* __restrict__ ly, const double* __restrict__ lz, double* tx, double* ty,
                               double* tz, const double* __restrict__ dtp) {
  const double dt = dtp ? *dtp : p.time_step;
  for (index_t i = blockIdx.x * blockDim.x + threadIdx.x; i < static_cast<index_t>(f.count);
       i += gridDim.x * blockDim.x) {
    const bool splash = f.surface_type != nullptr && f.surface_type[i] == LSMPS_SURFACE_SPLASH;
    const double nu = splash ? 0.0 : p.kinematic_viscosity;
    tx[i] = f.vx[i] + dt * (nu * lx[i] + p.gravity[0]);
    ty[i] = f.vy[i] + dt * (nu * ly[i] + p.gravity[1]);
    tz[i] = f.vz[i] + dt * (nu * lz[i] + p.gravity[2]);
  }
}

// combine_explicit_wall_velocity_kernel, explicit_update.cu:272-284
__global__ void wall_combine_kernel(lsmps_walls w, lsmps_params p, double* tx, double* ty, double* tz,
                                    const double* __restrict__ dtp) {
  const double dt = dtp ? *dtp : p.time_step;
  for (index_t i = blockIdx.x * blockDim.x + threadIdx.x; i < static_cast<index_t>(w.count);
       i += gridDim.x * blockDim.x) {
    tx[i] = w.vx[i] + dt * p.gravity[0];
    ty[i] = w.vy[i] + dt * p.gravity[1];
    tz[i] = w.vz[i] + dt * p.gravity[2];
  }
}

template <bool Mixed>
void launch_laplacian(lsmps_ctx* ctx, const LaplacianArgs& a, const MixedRows& rows) {
  const long long n = a.n;
  switch (ctx->knob[LSMPS_KNOB_GATHER_LANES]) {
    case 1:
      launch_named(ctx, Mixed ? "laplacian_kernel<true, 2>" : "laplacian_kernel<false, 2>", laplacian_kernel<Mixed, 2>,
                   dim3(div_up(2 * n, kThreads)), dim3(kThreads), 0, a, rows);
      break;
    case 2:
      launch_named(ctx, Mixed ? "laplacian_kernel<true, 4>" : "laplacian_kernel<false, 4>", laplacian_kernel<Mixed, 4>,
                   dim3(div_up(4 * n, kThreads)), dim3(kThreads), 0, a, rows);
      break;
    default:
      launch_named(ctx, Mixed ? "laplacian_kernel<true, 1>" : "laplacian_kernel<false, 1>", laplacian_kernel<Mixed, 1>,
                   dim3(div_up(n, kThreads)), dim3(kThreads), 0, a, rows);
      break;
  }
}

int pointwise_blocks(lsmps_ctx* ctx, size_t n) {
  const long long b = div_up(static_cast<long long>(n), 256);
  const long long cap = static_cast<long long>(ctx->sm_count) * 8;
  return static_cast<int>(b < cap ? b : cap);
}

}  // namespace

lsmps_status velocity_laplacian_mixed_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w,
                                           const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_moment& vm,
                                           const lsmps_vector& lap) {
  if (lap.count < f.count) return fail(ctx, LSMPS_INVALID_ARGUMENT, "Provision laplacian workspace is too small");
  if (f.count == 0) return LSMPS_OK;
  if (const lsmps_status cs = check_neighbor_tables(ctx, f.count, w.count, fn, &wn)) return cs;
  if (!lap.x || !lap.y || !lap.z || !f.vx || !f.vy || !f.vz)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Provision buffers missing");
  if (w.count > 0 && (!w.vx || !w.vy || !w.vz)) return fail(ctx, LSMPS_INVALID_ARGUMENT, "wall velocity missing");
  if (!ctx->mixed_rows[0] || !ctx->mixed_count || ctx->mixed_cap < f.count)
    return fail(ctx, LSMPS_NOT_PREPARED, "mixed velocity operator rows were not prepared");
  if (!ensure_packs(ctx, f.count, w.count)) return fail(ctx, LSMPS_CUDA_ERROR, "pack allocation failed");
  const index_t* srows = sorted_rows_of(ctx, fn, f.count);
  pack4(ctx, f.vx, f.vy, f.vz, nullptr, f.count, ctx->pack_fluid[1], srows ? ctx->order : nullptr);
  pack4(ctx, w.vx, w.vy, w.vz, nullptr, w.count, ctx->pack_wall[1]);
  // fluid and wall positions are still packed from the moment stage (in the
  // same order: the rows' form is the same within a step)
  LaplacianArgs a{static_cast<index_t>(f.count), ctx->pack_fluid[0], ctx->pack_fluid[1], ctx->pack_wall[0],
                  ctx->pack_wall[1], fn.offsets, srows ? srows : fn.indices, wn.offsets, wn.indices, nullptr,
                  vm.support_radius, 1.0 / vm.support_radius, vm.wall_weight_scale, lap.x, lap.y, lap.z,
                  ctx->order, srows ? 1 : 0};
  const MixedRows rows = mixed_rows_of(ctx, 0);
  const long long n = a.n;
  const dim3 list_grid(static_cast<unsigned>(ctx->sm_count * 2));
  switch (ctx->knob[LSMPS_KNOB_GATHER_LANES]) {
    case 1:
      launch_named(ctx, "laplacian32_kernel<2>", laplacian32_kernel<2>, dim3(div_up(2 * n, kThreads)), dim3(kThreads),
                   0, a, rows);
      launch_named(ctx, "laplacian_list_kernel<2>", laplacian_list_kernel<2>, list_grid, dim3(kThreads), 0, a, rows);
      break;
    case 2:
      launch_named(ctx, "laplacian32_kernel<4>", laplacian32_kernel<4>, dim3(div_up(4 * n, kThreads)), dim3(kThreads),
                   0, a, rows);
      launch_named(ctx, "laplacian_list_kernel<4>", laplacian_list_kernel<4>, list_grid, dim3(kThreads), 0, a, rows);
      break;
    default:
      launch_named(ctx, "laplacian32_kernel<1>", laplacian32_kernel<1>, dim3(div_up(n, kThreads)), dim3(kThreads), 0,
                   a, rows);
      launch_named(ctx, "laplacian_list_kernel<1>", laplacian_list_kernel<1>, list_grid, dim3(kThreads), 0, a, rows);
      break;
  }
  return check_launch(ctx, "velocity laplacian (mixed)");
}

lsmps_status velocity_laplacian_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w,
                                     const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_moment& vm,
                                     const lsmps_vector& lap) {
  if (vm.kind != LSMPS_MOMENT_VELOCITY_WALL_DIRICHLET_A || vm.matrix_size != 9 || vm.particle_count < f.count)
    return fail(ctx, LSMPS_NOT_PREPARED, "Provision requires a prepared velocity Type-A moment matrix");
  if (lap.count < f.count) return fail(ctx, LSMPS_INVALID_ARGUMENT, "Provision laplacian workspace is too small");
  if (f.count == 0) return LSMPS_OK;
  if (const lsmps_status cs = check_neighbor_tables(ctx, f.count, w.count, fn, &wn)) return cs;
  if (!vm.inverse_matrices || !lap.x || !lap.y || !lap.z || !f.vx || !f.vy || !f.vz)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Provision buffers missing");
  if (w.count > 0 && (!w.vx || !w.vy || !w.vz)) return fail(ctx, LSMPS_INVALID_ARGUMENT, "wall velocity missing");
  if (!ensure_packs(ctx, f.count, w.count)) return fail(ctx, LSMPS_CUDA_ERROR, "pack allocation failed");
  const index_t* srows = sorted_rows_of(ctx, fn, f.count);
  const index_t* pord = srows ? ctx->order : nullptr;
  pack_fluid_positions(ctx, f, pord);
  pack4(ctx, f.vx, f.vy, f.vz, nullptr, f.count, ctx->pack_fluid[1], pord);
  pack_wall_positions(ctx, w);
  pack4(ctx, w.vx, w.vy, w.vz, nullptr, w.count, ctx->pack_wall[1]);
  LaplacianArgs a{static_cast<index_t>(f.count), ctx->pack_fluid[0], ctx->pack_fluid[1], ctx->pack_wall[0],
                  ctx->pack_wall[1], fn.offsets, srows ? srows : fn.indices, wn.offsets, wn.indices,
                  vm.inverse_matrices, vm.support_radius, 1.0 / vm.support_radius, vm.wall_weight_scale, lap.x,
                  lap.y, lap.z, ctx->order, srows ? 1 : 0};
  launch_laplacian<false>(ctx, a, MixedRows{});
  return check_launch(ctx, "velocity laplacian");
}

lsmps_status temporary_velocity_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_params& p,
                                     const lsmps_vector& lap, const lsmps_fluid& t) {
  if (t.count < f.count || lap.count < f.count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Provision temporary velocity target is smaller than fluid particle count");
  if (f.count == 0) return LSMPS_OK;
  if (!t.vx || !t.vy || !t.vz) return fail(ctx, LSMPS_INVALID_ARGUMENT, "temporary velocity requires vx/vy/vz");
  launch(ctx, combine_kernel, dim3(pointwise_blocks(ctx, f.count)), dim3(256), 0, f, p,
         static_cast<const double*>(lap.x), static_cast<const double*>(lap.y), static_cast<const double*>(lap.z),
         t.vx, t.vy, t.vz, ctx->device_dt);
  return check_launch(ctx, "temporary velocity");
}

lsmps_status temporary_wall_velocity_impl(lsmps_ctx* ctx, const lsmps_walls& w, const lsmps_params& p,
                                          const lsmps_walls& t) {
  if (t.count < w.count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Provision temporary wall velocity target is smaller than wall particle count");
  if (w.count == 0) return LSMPS_OK;
  if (!t.vx || !t.vy || !t.vz) return fail(ctx, LSMPS_INVALID_ARGUMENT, "temporary wall velocity requires vx/vy/vz");
  launch(ctx, wall_combine_kernel, dim3(pointwise_blocks(ctx, w.count)), dim3(256), 0, w, p, t.vx, t.vy, t.vz,
         ctx->device_dt);
  return check_launch(ctx, "temporary wall velocity");
}

}  // namespace lsmps

using namespace lsmps;

extern "C" {

lsmps_status lsmps_velocity_laplacian(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_walls* walls,
                                      const lsmps_csr* fn, const lsmps_csr* wn, const lsmps_moment* vm,
                                      const lsmps_vector* lap) {
  if (!ctx || !fluid || !walls || !fn || !wn || !vm || !lap) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  return end_call(ctx, velocity_laplacian_impl(ctx, *fluid, *walls, *fn, *wn, *vm, *lap));
}

lsmps_status lsmps_temporary_velocity(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_params* params,
                                      const lsmps_vector* lap, const lsmps_fluid* t) {
  if (!ctx || !fluid || !params || !lap || !t) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  return end_call(ctx, temporary_velocity_impl(ctx, *fluid, *params, *lap, *t));
}

lsmps_status lsmps_temporary_wall_velocity(lsmps_ctx* ctx, const lsmps_walls* walls, const lsmps_params* params,
                                           const lsmps_walls* t) {
  if (!ctx || !walls || !params || !t) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  return end_call(ctx, temporary_wall_velocity_impl(ctx, *walls, *params, *t));
}

}  // extern "C"
