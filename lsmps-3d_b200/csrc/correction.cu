// correction.cu - pressure-gradient correction of velocity and position.
// Replaces DevicePressureCorrection::apply and its free functions
// (src/correction/pressure_correction.cu:188-515, 598-734): pressure clamp,
// LSMPS pressure gradient, particle shifting, velocity/position update,
// wall anti-penetration and velocity smoothing.
#include "impl.cuh"
#include "mixed.cuh"
#include "packed.cuh"

namespace lsmps {
namespace {

constexpr int kThreads = 128;

__device__ __forceinline__ bool is_splash(const int32_t* type, index_t i) {
  return type != nullptr && type[i] == LSMPS_SURFACE_SPLASH;
}

__device__ __forceinline__ bool is_surface(const int32_t* type, index_t i) {
  if (type == nullptr) return false;
  const int t = type[i];
  return t == LSMPS_SURFACE_SURFACE || t == LSMPS_SURFACE_SPLASH;
}

// clamp_fluid_pressure_kernel, pressure_correction.cu:188-198
__global__ void clamp_kernel(index_t n, double* pressure, double* fluid_pressure) {
  for (index_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double p = pressure[i];
    const double c = p < 0.0 ? 0.0 : p;
    pressure[i] = c;
    if (fluid_pressure != nullptr && fluid_pressure != pressure) fluid_pressure[i] = c;
  }
}

struct GatherArgs {
  lsmps_fluid fluid;
  lsmps_walls walls;
  const index_t* fo;
  const index_t* fi;
  const index_t* wo;
  const index_t* wi;
  lsmps_params p;
  // 32-byte records of the fused gradient/shifting kernel: fluid
  // {x, y, z, pressure}, walls {x, y, z, -} and {nx, ny, nz, -}.
  const double4* fpp = nullptr;
  const double4* wp = nullptr;
  const double4* wn = nullptr;
  const int32_t* order = nullptr;  // visiting order of the fused kernel (lsmps_ctx::order) or NULL
  int sorted = 0;  // fused kernels: fi and fpp in cell-sorted positions (sorted_rows_of)
};

// compute_pressure_gradient_kernel, pressure_correction.cu:200-276
__global__ void __launch_bounds__(kThreads) gradient_kernel(GatherArgs a, const double* __restrict__ pressure,
                                                            const double* __restrict__ pinv, double re,
                                                            double wall_scale, double* gx, double* gy,
                                                            double* gz) {
  const index_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= static_cast<index_t>(a.fluid.count)) return;
  if (is_splash(a.fluid.surface_type, i)) {
    gx[i] = gy[i] = gz[i] = 0.0;
    return;
  }
  const double* __restrict__ fx = a.fluid.x;
  const double* __restrict__ fy = a.fluid.y;
  const double* __restrict__ fz = a.fluid.z;
  const double xi = fx[i], yi = fy[i], zi = fz[i];
  const double inv_re = 1.0 / re;
  const double pi = pressure[i];
  double rhs[9], b[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) rhs[r] = 0.0;
  const index_t fe = a.fo[i + 1];
  for (index_t o = a.fo[i]; o < fe; ++o) {
    const index_t j = a.fi[o];
    const double dx = fx[j] - xi, dy = fy[j] - yi, dz = fz[j] - zi;
    const double w = correction_weight_mul(sqrt(dx * dx + dy * dy + dz * dz), inv_re);
    if (w <= 0.0) continue;
    basis_a_mul(dx, dy, dz, inv_re, b);
    const double dp = pressure[j] - pi;
#pragma unroll
    for (int r = 0; r < 9; ++r) rhs[r] = fma(w * b[r], dp, rhs[r]);
  }
  const index_t we = a.wo[i + 1];
  for (index_t o = a.wo[i]; o < we; ++o) {
    const index_t j = a.wi[o];
    const double dx = a.walls.x[j] - xi, dy = a.walls.y[j] - yi, dz = a.walls.z[j] - zi;
    const double w = wall_scale * correction_weight_mul(sqrt(dx * dx + dy * dy + dz * dz), inv_re);
    if (w <= 0.0) continue;
    const double nx = a.walls.normal_x[j], ny = a.walls.normal_y[j], nz = a.walls.normal_z[j];
    double q[9];
    neumann_a(dx, dy, dz, nx, ny, nz, inv_re, q);
    const double ng = a.p.gravity[0] * nx + a.p.gravity[1] * ny + a.p.gravity[2] * nz;
    const double wr = re * a.p.density * ng;
#pragma unroll
    for (int r = 0; r < 9; ++r) rhs[r] = fma(w * q[r], wr, rhs[r]);
  }
  const double* __restrict__ inv = pinv + static_cast<size_t>(i) * 81;
  double c0 = 0.0, c1 = 0.0, c2 = 0.0;
#pragma unroll
  for (int col = 0; col < 9; ++col) {
    c0 = fma(inv[0 + col * 9], rhs[col], c0);
    c1 = fma(inv[1 + col * 9], rhs[col], c1);
    c2 = fma(inv[2 + col * 9], rhs[col], c2);
  }
  gx[i] = c0 * inv_re;
  gy[i] = c1 * inv_re;
  gz[i] = c2 * inv_re;
}

// compute_particle_shifting_kernel, pressure_correction.cu:278-367
__global__ void __launch_bounds__(kThreads) shifting_kernel(GatherArgs a, double* sx_out, double* sy_out,
                                                            double* sz_out) {
  const index_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= static_cast<index_t>(a.fluid.count)) return;
  if (a.p.ps_displacement_scale <= 0.0 || is_splash(a.fluid.surface_type, i)) {
    sx_out[i] = sy_out[i] = sz_out[i] = 0.0;
    return;
  }
  const double* __restrict__ fx = a.fluid.x;
  const double* __restrict__ fy = a.fluid.y;
  const double* __restrict__ fz = a.fluid.z;
  const double xi = fx[i], yi = fy[i], zi = fz[i];
  const double dmin = a.p.ps_min_distance_ratio * a.p.particle_spacing;
  const double smax = a.p.ps_max_displacement_ratio * a.p.particle_spacing;
  const double scale = a.p.ps_displacement_scale;
  double shx = 0.0, shy = 0.0, shz = 0.0, nx = 0.0, ny = 0.0, nz = 0.0;
  const index_t fe = a.fo[i + 1];
  for (index_t o = a.fo[i]; o < fe; ++o) {
    const index_t j = a.fi[o];
    const double dx = xi - fx[j], dy = yi - fy[j], dz = zi - fz[j];
    const double d = sqrt(dx * dx + dy * dy + dz * dz);
    if (d <= 0.0 || d >= dmin) continue;
    // The reference's exact expressions (pressure_correction.cu:318-324): for
    // stacked particles the summed unit vectors nearly cancel, so the
    // projection below amplifies any change of operation order.
    const double push = scale * (dmin - d) / d;
    shx += push * dx;
    shy += push * dy;
    shz += push * dz;
    nx += dx / d;
    ny += dy / d;
    nz += dz / d;
  }
  const index_t we = a.wo[i + 1];
  for (index_t o = a.wo[i]; o < we; ++o) {
    const index_t j = a.wi[o];
    const double dx = xi - a.walls.x[j], dy = yi - a.walls.y[j], dz = zi - a.walls.z[j];
    const double d = sqrt(dx * dx + dy * dy + dz * dz);
    if (d <= 0.0 || d >= dmin) continue;
    const double push = scale * (dmin - d);
    shx = fma(push, a.walls.normal_x[j], shx);
    shy = fma(push, a.walls.normal_y[j], shy);
    shz = fma(push, a.walls.normal_z[j], shz);
  }
  if (is_surface(a.fluid.surface_type, i)) {
    const double nn = sqrt(nx * nx + ny * ny + nz * nz);
    if (nn > 0.0) {
      nx /= nn;
      ny /= nn;
      nz /= nn;
      const double nc = shx * nx + shy * ny + shz * nz;
      shx -= nc * nx;
      shy -= nc * ny;
      shz -= nc * nz;
    }
  }
  const double sn = sqrt(shx * shx + shy * shy + shz * shz);
  if (sn > smax && sn > 0.0) {
    const double sc = smax / sn;
    shx *= sc;
    shy *= sc;
    shz *= sc;
  }
  sx_out[i] = shx;
  sy_out[i] = shy;
  sz_out[i] = shz;
}

// update_velocity_position_kernel, pressure_correction.cu:369-402
__global__ void update_kernel(lsmps_fluid f, const double* __restrict__ tx, const double* __restrict__ ty,
                              const double* __restrict__ tz, double dt_host, const double* __restrict__ dtp,
                              double density,
                              const double* __restrict__ gx, const double* __restrict__ gy,
                              const double* __restrict__ gz, const double* __restrict__ sx,
                              const double* __restrict__ sy, const double* __restrict__ sz) {
  const double dt = dtp ? *dtp : dt_host;
  for (index_t i = blockIdx.x * blockDim.x + threadIdx.x; i < static_cast<index_t>(f.count);
       i += gridDim.x * blockDim.x) {
    const bool splash = is_splash(f.surface_type, i);
    const double ox = f.vx[i], oy = f.vy[i], oz = f.vz[i];
    double nx = tx[i], ny = ty[i], nz = tz[i];
    if (!splash) {
      const double ps = dt / density;
      nx -= ps * gx[i];
      ny -= ps * gy[i];
      nz -= ps * gz[i];
    }
    f.x[i] += 0.5 * dt * (ox + nx) + sx[i];
    f.y[i] += 0.5 * dt * (oy + ny) + sy[i];
    f.z[i] += 0.5 * dt * (oz + nz) + sz[i];
    f.vx[i] = nx;
    f.vy[i] = ny;
    f.vz[i] = nz;
  }
}

// anti_penetration_kernel, pressure_correction.cu:404-444: sequential over the
// wall row in CSR order, one thread per particle.
__global__ void __launch_bounds__(kThreads) anti_penetration_kernel(lsmps_fluid f, lsmps_walls w,
                                                                    const index_t* __restrict__ wo,
                                                                    const index_t* __restrict__ wi,
                                                                    double clearance) {
  const index_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= static_cast<index_t>(f.count)) return;
  const index_t we = wo[i + 1];
  index_t o = wo[i];
  if (o >= we) return;
  double x = f.x[i], y = f.y[i], z = f.z[i];
  double vx = f.vx[i], vy = f.vy[i], vz = f.vz[i];
  bool moved = false;
  for (; o < we; ++o) {
    const index_t j = wi[o];
    const double nx = w.normal_x[j], ny = w.normal_y[j], nz = w.normal_z[j];
    const double sd = (x - w.x[j]) * nx + (y - w.y[j]) * ny + (z - w.z[j]) * nz;
    if (sd >= clearance) continue;
    const double c = clearance - sd;
    x += c * nx;
    y += c * ny;
    z += c * nz;
    const double nv = vx * nx + vy * ny + vz * nz;
    if (nv < 0.0) {
      vx -= nv * nx;
      vy -= nv * ny;
      vz -= nv * nz;
    }
    moved = true;
  }
  if (moved) {
    f.x[i] = x;
    f.y[i] = y;
    f.z[i] = z;
    f.vx[i] = vx;
    f.vy[i] = vy;
    f.vz[i] = vz;
  }
}

// smooth_velocity_kernel, pressure_correction.cu:446-504, on neighbour records
// fp = {x, y, z, 0} and fv = {vx, vy, vz, label} (packed.cuh).
template <int G>
__global__ void __launch_bounds__(kThreads) smooth_kernel(index_t n, const double4* __restrict__ fp,
                                                          const double4* __restrict__ fv,
                                                          const index_t* __restrict__ fo,
                                                          const index_t* __restrict__ fi, double re, double strength,
                                                          double* ox, double* oy, double* oz,
                                                          const int32_t* __restrict__ order, int sorted) {
  // G lanes per particle (lane l takes entries l, l + G, ...); the group
  // leaves or continues as a whole.
  const index_t t = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int l = threadIdx.x & (G - 1);
  if (t >= n) return;
  const index_t i = visit(order, t);
  const index_t self = self_of(sorted, t, i);
  const double inv_re = 1.0 / re;
  constexpr double kSplash = static_cast<double>(LSMPS_SURFACE_SPLASH);
  const double4 ui = ld4(fv, self);
  if (strength <= 0.0 || ui.w == kSplash) {
    if (l == 0) {
      ox[i] = ui.x;
      oy[i] = ui.y;
      oz[i] = ui.z;
    }
    return;
  }
  const double4 pi = ld4(fp, self);
  double ws = 0.0, ax = 0.0, ay = 0.0, az = 0.0;
  const index_t fe = fo[i + 1];
  index_t o = fo[i] + l;
  index_t jn = o < fe ? fi[o] : i;
  double4 un = ld4(fv, jn), qn = ld4(fp, jn);
  for (; o < fe; o += G) {
    // the next neighbour's records are loaded while this one is summed
    const double4 u = un, q = qn;
    if (o + G < fe) {
      jn = fi[o + G];
      un = ld4(fv, jn);
      qn = ld4(fp, jn);
    }
    if (u.w == kSplash) continue;
    const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
    const double w = correction_weight_mul(sqrt(dx * dx + dy * dy + dz * dz), inv_re);
    if (w <= 0.0) continue;
    ws += w;
    ax = fma(w, u.x, ax);
    ay = fma(w, u.y, ay);
    az = fma(w, u.z, az);
  }
  if (G > 1) {
    const unsigned mask = group_mask<G>();
    ws = group_sum<G>(ws, mask);
    ax = group_sum<G>(ax, mask);
    ay = group_sum<G>(ay, mask);
    az = group_sum<G>(az, mask);
    if (l != 0) return;
  }
  if (ws <= 0.0) {
    ox[i] = ui.x;
    oy[i] = ui.y;
    oz[i] = ui.z;
    return;
  }
  const double alpha = strength < 0.0 ? 0.0 : (strength > 1.0 ? 1.0 : strength);
  ox[i] = (1.0 - alpha) * ui.x + alpha * ax / ws;
  oy[i] = (1.0 - alpha) * ui.y + alpha * ay / ws;
  oz[i] = (1.0 - alpha) * ui.z + alpha * az / ws;
}

// copy_smoothed_velocity_kernel, pressure_correction.cu:506-515
__global__ void copy_kernel(index_t n, const double* __restrict__ sx, const double* __restrict__ sy,
                            const double* __restrict__ sz, double* vx, double* vy, double* vz) {
  for (index_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    vx[i] = sx[i];
    vy[i] = sy[i];
    vz[i] = sz[i];
  }
}

int pointwise_blocks(lsmps_ctx* ctx, size_t n) {
  const long long b = div_up(static_cast<long long>(n), 256);
  const long long cap = static_cast<long long>(ctx->sm_count) * 8;
  return static_cast<int>(b < cap ? b : cap);
}

lsmps_status check_fluid(lsmps_ctx* ctx, const lsmps_fluid& f) {
  if (f.count > 0 && (!f.x || !f.y || !f.z || !f.vx || !f.vy || !f.vz))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Pressure correction requires fluid position and velocity arrays");
  return LSMPS_OK;
}

lsmps_status check_vector(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_vector& v, const char* what) {
  if (v.count < f.count || (f.count > 0 && (!v.x || !v.y || !v.z))) return fail(ctx, LSMPS_INVALID_ARGUMENT, what);
  return LSMPS_OK;
}

}  // namespace

lsmps_status clamp_pressure_impl(lsmps_ctx* ctx, const lsmps_fluid& f, double* pressure) {
  if (f.count > 0 && !pressure) return fail(ctx, LSMPS_INVALID_ARGUMENT, "Pressure correction requires a pressure array");
  if (f.count == 0) return LSMPS_OK;
  launch(ctx, clamp_kernel, dim3(pointwise_blocks(ctx, f.count)), dim3(256), 0, static_cast<index_t>(f.count),
         pressure, f.pressure);
  return check_launch(ctx, "pressure clamp");
}

lsmps_status pressure_gradient_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w, const lsmps_csr& fn,
                                    const lsmps_csr& wn, const double* pressure, const lsmps_params& p,
                                    const lsmps_moment& pm, const lsmps_vector& g) {
  lsmps_status st = check_fluid(ctx, f);
  if (st) return st;
  if ((st = check_vector(ctx, f, g, "Pressure gradient workspace is too small"))) return st;
  if (pm.kind != LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_A || pm.matrix_size != 9 || pm.particle_count < f.count)
    return fail(ctx, LSMPS_NOT_PREPARED, "Pressure correction requires a prepared pressure Type-A moment matrix");
  if (f.count > 0 && (!pressure || !pm.inverse_matrices))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Pressure gradient requires pressure and inverse buffers");
  if (f.count == 0) return LSMPS_OK;
  if (const lsmps_status cs = check_neighbor_tables(ctx, f.count, w.count, fn, &wn)) return cs;
  GatherArgs a{f, w, fn.offsets, fn.indices, wn.offsets, wn.indices, p};
  launch(ctx, gradient_kernel, dim3(div_up(static_cast<long long>(f.count), kThreads)), dim3(kThreads), 0, a,
         pressure, static_cast<const double*>(pm.inverse_matrices), pm.support_radius, pm.wall_weight_scale, g.x, g.y,
         g.z);
  return check_launch(ctx, "pressure gradient");
}

lsmps_status particle_shifting_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w, const lsmps_csr& fn,
                                    const lsmps_csr& wn, const lsmps_params& p, const lsmps_vector& s) {
  lsmps_status st = check_fluid(ctx, f);
  if (st) return st;
  if ((st = check_vector(ctx, f, s, "PS displacement workspace is too small"))) return st;
  if (f.count == 0) return LSMPS_OK;
  if (const lsmps_status cs = check_neighbor_tables(ctx, f.count, w.count, fn, &wn)) return cs;
  GatherArgs a{f, w, fn.offsets, fn.indices, wn.offsets, wn.indices, p};
  launch(ctx, shifting_kernel, dim3(div_up(static_cast<long long>(f.count), kThreads)), dim3(kThreads), 0, a, s.x, s.y,
         s.z);
  return check_launch(ctx, "particle shifting");
}

lsmps_status update_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_fluid& t, const lsmps_params& p,
                         const lsmps_vector& g, const lsmps_vector& s) {
  lsmps_status st = check_fluid(ctx, f);
  if (st) return st;
  if (t.count < f.count || (f.count && (!t.vx || !t.vy || !t.vz)))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Pressure correction temporary velocity target is too small");
  if ((st = check_vector(ctx, f, g, "Pressure gradient workspace is too small"))) return st;
  if ((st = check_vector(ctx, f, s, "PS displacement workspace is too small"))) return st;
  if (f.count == 0) return LSMPS_OK;
  launch(ctx, update_kernel, dim3(pointwise_blocks(ctx, f.count)), dim3(256), 0, f,
         static_cast<const double*>(t.vx), static_cast<const double*>(t.vy), static_cast<const double*>(t.vz),
         p.time_step, ctx->device_dt, p.density, static_cast<const double*>(g.x), static_cast<const double*>(g.y),
         static_cast<const double*>(g.z), static_cast<const double*>(s.x), static_cast<const double*>(s.y),
         static_cast<const double*>(s.z));
  return check_launch(ctx, "velocity/position update");
}

lsmps_status anti_penetration_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w, const lsmps_csr& wn,
                                   const lsmps_params& p) {
  const double clearance = p.wall_clearance_ratio * p.particle_spacing;
  if (f.count == 0 || clearance <= 0.0) return LSMPS_OK;
  if (const lsmps_status cs = check_table(ctx, wn.offsets, wn.indices, f.count, wn.neighbor_count, w.count,
                                          "wall neighbour table: offset or index out of range"))
    return cs;
  launch(ctx, anti_penetration_kernel, dim3(div_up(static_cast<long long>(f.count), kThreads)), dim3(kThreads), 0, f,
         w, static_cast<const index_t*>(wn.offsets), static_cast<const index_t*>(wn.indices), clearance);
  return check_launch(ctx, "anti-penetration");
}

lsmps_status smooth_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_csr& fn, const lsmps_params& p,
                         const lsmps_vector& sm, bool copy_back) {
  lsmps_status st = check_fluid(ctx, f);
  if (st) return st;
  if ((st = check_vector(ctx, f, sm, "Velocity smoothing workspace is too small"))) return st;
  if (f.count == 0) return LSMPS_OK;
  if (const lsmps_status cs = check_neighbor_tables(ctx, f.count, 0, fn, nullptr)) return cs;
  if (!ensure_packs(ctx, f.count, 0)) return fail(ctx, LSMPS_CUDA_ERROR, "pack allocation failed");
  const index_t* srows = sorted_rows_of(ctx, fn, f.count);
  const index_t* pord = srows ? ctx->order : nullptr;
  const index_t* fi = srows ? srows : static_cast<const index_t*>(fn.indices);
  const int sorted = srows ? 1 : 0;
  pack4(ctx, f.x, f.y, f.z, nullptr, f.count, ctx->pack_fluid[0], pord);
  pack4_label(ctx, f.vx, f.vy, f.vz, f.surface_type, f.count, ctx->pack_fluid[1], pord);
  const long long n = static_cast<long long>(f.count);
  const double4* fp = ctx->pack_fluid[0];
  const double4* fv = ctx->pack_fluid[1];
  switch (ctx->knob[LSMPS_KNOB_GATHER_LANES]) {
    case 1:
      launch(ctx, smooth_kernel<2>, dim3(div_up(2 * n, kThreads)), dim3(kThreads), 0, static_cast<index_t>(n), fp, fv,
             static_cast<const index_t*>(fn.offsets), fi, p.support_radius, p.velocity_smoothing_strength, sm.x,
             sm.y, sm.z, ctx->order, sorted);
      break;
    case 2:
      launch(ctx, smooth_kernel<4>, dim3(div_up(4 * n, kThreads)), dim3(kThreads), 0, static_cast<index_t>(n), fp, fv,
             static_cast<const index_t*>(fn.offsets), fi, p.support_radius, p.velocity_smoothing_strength, sm.x,
             sm.y, sm.z, ctx->order, sorted);
      break;
    default:
      launch(ctx, smooth_kernel<1>, dim3(div_up(n, kThreads)), dim3(kThreads), 0, static_cast<index_t>(n), fp, fv,
             static_cast<const index_t*>(fn.offsets), fi, p.support_radius, p.velocity_smoothing_strength, sm.x,
             sm.y, sm.z, ctx->order, sorted);
      break;
  }
  if (copy_back)
    launch(ctx, copy_kernel, dim3(pointwise_blocks(ctx, f.count)), dim3(256), 0, static_cast<index_t>(f.count),
           static_cast<const double*>(sm.x), static_cast<const double*>(sm.y), static_cast<const double*>(sm.z), f.vx,
           f.vy, f.vz);
  return check_launch(ctx, "velocity smoothing");
}

namespace {

// Outputs of the gradient/shifting pass.
struct GradShiftOut {
  double* pressure;
  double* fluid_pressure;
  const double* pinv;
  MixedRows prows;
  double re;
  double wall_scale;
  double* gx;
  double* gy;
  double* gz;
  double* sx;
  double* sy;
  double* sz;
};

// clamp_fluid_pressure_kernel + compute_pressure_gradient_kernel +
// compute_particle_shifting_kernel in one pass over the rows.  All three read
// the pre-update neighbourhood only.  The clamp is applied to every pressure
// read (a neighbour's slot may or may not be clamped yet when it is read; both
// give the same clamped value), and each thread writes its own clamped value.
// The shifting offsets x_i - x_j are the exact negations of x_j - x_i, so the
// outputs are bitwise those of the separate kernels.
//
// Mixed (the mixed form): the FP64 gradient sums are contracted with rows
// 0..2 of the pressure operator rows (FP32, or FP64 for FP64-route
// particles) instead of the full inverse.
//
// G lanes share a particle (G = 1, 2, 4: LSMPS_KNOB_GATHER_LANES): lane l
// takes row entries l, l + G, ...; the 15 partial sums are combined with
// shuffles and lane 0 finishes the particle.
template <bool Mixed, int G>
__device__ __forceinline__ void gradient_shifting_of(const GatherArgs& a, const GradShiftOut& out, index_t i,
                                                     index_t vt, int l) {
  const index_t self = self_of(a.sorted, vt, i);
  double* pressure = out.pressure;
  double* fluid_pressure = out.fluid_pressure;
  const double* __restrict__ pinv = out.pinv;
  const MixedRows& prows = out.prows;
  const double re = out.re, wall_scale = out.wall_scale;
  double *gx = out.gx, *gy = out.gy, *gz = out.gz, *sx_out = out.sx, *sy_out = out.sy, *sz_out = out.sz;
  const double praw = pressure[i];
  const double pi = praw < 0.0 ? 0.0 : praw;
  if (l == 0) {
    pressure[i] = pi;
    if (fluid_pressure != nullptr && fluid_pressure != pressure) fluid_pressure[i] = pi;
  }
  const bool splash = is_splash(a.fluid.surface_type, i);
  const bool do_grad = !splash;
  const bool do_shift = !(a.p.ps_displacement_scale <= 0.0 || splash);
  if (!do_grad && !do_shift) {
    if (l == 0) {
      gx[i] = gy[i] = gz[i] = 0.0;
      sx_out[i] = sy_out[i] = sz_out[i] = 0.0;
    }
    return;
  }
  const double4 own = ld4(a.fpp, self);
  const double xi = own.x, yi = own.y, zi = own.z;
  const double inv_re = 1.0 / re;
  const double dmin = a.p.ps_min_distance_ratio * a.p.particle_spacing;
  const double scale = a.p.ps_displacement_scale;
  double rhs[9], b[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) rhs[r] = 0.0;
  double shx = 0.0, shy = 0.0, shz = 0.0, nx = 0.0, ny = 0.0, nz = 0.0;
  // {x, y, z, raw pressure} of the neighbours, packed before the launch (the
  // clamp is applied on read, as for every pressure this kernel reads); the
  // next record is loaded while this one is used.
  const index_t fe = a.fo[i + 1];
  index_t o = a.fo[i] + l;
  double4 qn = ld4(a.fpp, o < fe ? a.fi[o] : i);
  index_t jnn = o + G < fe ? a.fi[o + G] : i;  // the index after the next
  for (; o < fe; o += G) {
    const double4 q = qn;
    if (o + G < fe) {
      qn = ld4(a.fpp, jnn);
      if (o + 2 * G < fe) jnn = a.fi[o + 2 * G];
    }
    const double dx = q.x - xi, dy = q.y - yi, dz = q.z - zi;
    const double d = sqrt(dx * dx + dy * dy + dz * dz);
    if (do_grad) {
      const double w = correction_weight_mul(d, inv_re);
      if (w > 0.0) {
        basis_a_mul(dx, dy, dz, inv_re, b);
        const double pj = q.w;
        const double dp = (pj < 0.0 ? 0.0 : pj) - pi;
#pragma unroll
        for (int r = 0; r < 9; ++r) rhs[r] = fma(w * b[r], dp, rhs[r]);
      }
    }
    if (do_shift && d > 0.0 && d < dmin) {
      const double ex = -dx, ey = -dy, ez = -dz;
      const double push = scale * (dmin - d) / d;
      shx += push * ex;
      shy += push * ey;
      shz += push * ez;
      nx += ex / d;
      ny += ey / d;
      nz += ez / d;
    }
  }
  const index_t we = a.wo[i + 1];
  {  // the next wall's records are loaded while this one is used
    index_t o = a.wo[i] + l;
    index_t jn = o < we ? a.wi[o] : 0;
    double4 qn = make_double4(0.0, 0.0, 0.0, 0.0), nrmn = qn;
    if (o < we) {
      qn = ld4(a.wp, jn);
      nrmn = ld4(a.wn, jn);
    }
    for (; o < we; o += G) {
      const double4 q = qn, nrm = nrmn;
      if (o + G < we) {
        jn = a.wi[o + G];
        qn = ld4(a.wp, jn);
        nrmn = ld4(a.wn, jn);
      }
      const double dx = q.x - xi, dy = q.y - yi, dz = q.z - zi;
      const double d = sqrt(dx * dx + dy * dy + dz * dz);
      const double wnx = nrm.x, wny = nrm.y, wnz = nrm.z;
      if (do_grad) {
        const double w = wall_scale * correction_weight_mul(d, inv_re);
        if (w > 0.0) {
          double q[9];
          neumann_a(dx, dy, dz, wnx, wny, wnz, inv_re, q);
          const double ng = a.p.gravity[0] * wnx + a.p.gravity[1] * wny + a.p.gravity[2] * wnz;
          const double wr = re * a.p.density * ng;
#pragma unroll
          for (int r = 0; r < 9; ++r) rhs[r] = fma(w * q[r], wr, rhs[r]);
        }
      }
      if (do_shift && d > 0.0 && d < dmin) {
        const double push = scale * (dmin - d);
        shx = fma(push, wnx, shx);
        shy = fma(push, wny, shy);
        shz = fma(push, wnz, shz);
      }
  }
  }
  if (G > 1) {
    const unsigned gm = group_mask<G>();
#pragma unroll
    for (int r = 0; r < 9; ++r) rhs[r] = group_sum<G>(rhs[r], gm);
    shx = group_sum<G>(shx, gm);
    shy = group_sum<G>(shy, gm);
    shz = group_sum<G>(shz, gm);
    nx = group_sum<G>(nx, gm);
    ny = group_sum<G>(ny, gm);
    nz = group_sum<G>(nz, gm);
    if (l != 0) return;
  }
  if (do_grad && Mixed) {
    double g[9], c0 = 0.0, c1 = 0.0, c2 = 0.0;
    load_row9(prows, vt, 1, g);
#pragma unroll
    for (int col = 0; col < 9; ++col) c0 = fma(g[col], rhs[col], c0);
    load_row9(prows, vt, 2, g);
#pragma unroll
    for (int col = 0; col < 9; ++col) c1 = fma(g[col], rhs[col], c1);
    load_row9(prows, vt, 3, g);
#pragma unroll
    for (int col = 0; col < 9; ++col) c2 = fma(g[col], rhs[col], c2);
    gx[i] = c0 * inv_re;
    gy[i] = c1 * inv_re;
    gz[i] = c2 * inv_re;
  } else if (do_grad) {
    const double* __restrict__ inv = pinv + static_cast<size_t>(i) * 81;
    double c0 = 0.0, c1 = 0.0, c2 = 0.0;
#pragma unroll
    for (int col = 0; col < 9; ++col) {
      c0 = fma(inv[0 + col * 9], rhs[col], c0);
      c1 = fma(inv[1 + col * 9], rhs[col], c1);
      c2 = fma(inv[2 + col * 9], rhs[col], c2);
    }
    gx[i] = c0 * inv_re;
    gy[i] = c1 * inv_re;
    gz[i] = c2 * inv_re;
  } else {
    gx[i] = gy[i] = gz[i] = 0.0;
  }
  if (do_shift) {
    if (is_surface(a.fluid.surface_type, i)) {
      const double nn = sqrt(nx * nx + ny * ny + nz * nz);
      if (nn > 0.0) {
        nx /= nn;
        ny /= nn;
        nz /= nn;
        const double nc = shx * nx + shy * ny + shz * nz;
        shx -= nc * nx;
        shy -= nc * ny;
        shz -= nc * nz;
      }
    }
    const double smax = a.p.ps_max_displacement_ratio * a.p.particle_spacing;
    const double sn = sqrt(shx * shx + shy * shy + shz * shz);
    if (sn > smax && sn > 0.0) {
      const double sc = smax / sn;
      shx *= sc;
      shy *= sc;
      shz *= sc;
    }
    sx_out[i] = shx;
    sy_out[i] = shy;
    sz_out[i] = shz;
  } else {
    sx_out[i] = sy_out[i] = sz_out[i] = 0.0;
  }
}

template <bool Mixed, int G>
__global__ void __launch_bounds__(kThreads, 6) gradient_shifting_kernel(GatherArgs a, GradShiftOut out) {
  const long long tt = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const index_t t = static_cast<index_t>(tt / G);
  const int l = static_cast<int>(tt % G);
  if (t >= static_cast<index_t>(a.fluid.count)) return;  // the whole group
  const index_t i = visit(a.order, t);
  gradient_shifting_of<Mixed, G>(a, out, i, t, l);
}

// The FP64-route particles of the pressure kind (gradient_shifting_of<true,
// G>, FP64 arithmetic); lane groups stride over the list.
template <int G>
__global__ void __launch_bounds__(kThreads, 6) gradient_shifting_list_kernel(GatherArgs a, GradShiftOut out) {
  const index_t groups = static_cast<index_t>(gridDim.x * blockDim.x / G);
  const int l = threadIdx.x & (G - 1);
  const index_t count = static_cast<index_t>(*out.prows.count);
  for (index_t t = static_cast<index_t>((blockIdx.x * blockDim.x + threadIdx.x) / G); t < count; t += groups) {
    const index_t vt = out.prows.list[t];  // a visiting position
    const index_t i = visit(a.order, vt);
    gradient_shifting_of<true, G>(a, out, i, vt, l);
  }
}

// Mixed form with FP32 arithmetic for the gradient: each neighbour's offset
// is formed in FP64 and rounded once to FP32 (r_e-scaled); weight, basis and
// the nine moment right-hand-side sums w b (p_j - p_i) are FP32 (each lane's
// partial sums, added across the lane group in FP64), and the FP32 gradient
// rows are applied in FP64.  Particle shifting keeps the reference's FP64
// expressions: a pair is tested in FP32 first (|s|^2 against (d_min / r_e)^2
// with a relative margin of 1e-5, far above the FP32 rounding of |s|^2) and
// only pairs that pass are evaluated, and decided, in FP64.  Particles whose
// pressure rows took the FP64 route are left to gradient_shifting_list_kernel.
template <int G>
__global__ void __launch_bounds__(kThreads, 6) gradient32_kernel(GatherArgs a, GradShiftOut out) {
  const long long tt = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const index_t t = static_cast<index_t>(tt / G);
  const int l = static_cast<int>(tt % G);
  if (t >= static_cast<index_t>(a.fluid.count)) return;  // the whole group
  const index_t i = visit(a.order, t);
  if (out.prows.flag[t]) return;
  const double praw = out.pressure[i];
  const double pi = praw < 0.0 ? 0.0 : praw;
  if (l == 0) {
    out.pressure[i] = pi;
    if (out.fluid_pressure != nullptr && out.fluid_pressure != out.pressure) out.fluid_pressure[i] = pi;
  }
  const bool splash = is_splash(a.fluid.surface_type, i);
  const bool do_shift = !(a.p.ps_displacement_scale <= 0.0 || splash);
  if (splash) {
    if (l == 0) {
      out.gx[i] = out.gy[i] = out.gz[i] = 0.0;
      out.sx[i] = out.sy[i] = out.sz[i] = 0.0;
    }
    return;
  }
  const double4 own = ld4(a.fpp, self_of(a.sorted, t, i));
  const double inv_re = 1.0 / out.re;
  const double dmin = a.p.ps_min_distance_ratio * a.p.particle_spacing;
  const float dmin_s2 = static_cast<float>(dmin * inv_re * dmin * inv_re) * (1.0f + 1e-5f);
  const double scale = a.p.ps_displacement_scale;
  float rhs[9], b[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) rhs[r] = 0.0f;
  double shx = 0.0, shy = 0.0, shz = 0.0, nx = 0.0, ny = 0.0, nz = 0.0;
  const index_t fe = a.fo[i + 1];
  index_t o = a.fo[i] + l;
  double4 qn = ld4(a.fpp, o < fe ? a.fi[o] : i);
  index_t jnn = o + G < fe ? a.fi[o + G] : i;
  for (; o < fe; o += G) {
    const double4 q = qn;
    if (o + G < fe) {
      qn = ld4(a.fpp, jnn);
      if (o + 2 * G < fe) jnn = a.fi[o + 2 * G];
    }
    const double dx = q.x - own.x, dy = q.y - own.y, dz = q.z - own.z;
    const float w = basis_f32(dx, dy, dz, inv_re, b);
    const float s2 = b[3] + b[4] + b[5];
    if (w > 0.0f && s2 > 0.0f) {
      const double pj = q.w;
      const float wdp = w * static_cast<float>((pj < 0.0 ? 0.0 : pj) - pi);
#pragma unroll
      for (int r = 0; r < 9; ++r) rhs[r] = fmaf(wdp, b[r], rhs[r]);
    }
    if (do_shift && s2 < dmin_s2) {
      const double d = sqrt(dx * dx + dy * dy + dz * dz);
      if (d > 0.0 && d < dmin) {
        const double ex = -dx, ey = -dy, ez = -dz;
        const double push = scale * (dmin - d) / d;
        shx += push * ex;
        shy += push * ey;
        shz += push * ez;
        nx += ex / d;
        ny += ey / d;
        nz += ez / d;
      }
    }
  }
  const float wscale = static_cast<float>(out.wall_scale);
  const float wr = static_cast<float>(out.re * a.p.density);
  const index_t we = a.wo[i + 1];
  {  // the next wall's records are loaded while this one is used
    index_t o = a.wo[i] + l;
    index_t jn = o < we ? a.wi[o] : 0;
    double4 qn = make_double4(0.0, 0.0, 0.0, 0.0), nrmn = qn;
    if (o < we) {
      qn = ld4(a.wp, jn);
      nrmn = ld4(a.wn, jn);
    }
    for (; o < we; o += G) {
      const double4 q = qn, nrm = nrmn;
      if (o + G < we) {
        jn = a.wi[o + G];
        qn = ld4(a.wp, jn);
        nrmn = ld4(a.wn, jn);
      }
      const double dx = q.x - own.x, dy = q.y - own.y, dz = q.z - own.z;
      const float w = wscale * basis_f32(dx, dy, dz, inv_re, b);
      const float s2 = b[3] + b[4] + b[5];
      const float nxf = static_cast<float>(nrm.x), nyf = static_cast<float>(nrm.y), nzf = static_cast<float>(nrm.z);
      if (w > 0.0f && s2 > 0.0f) {
        // wall Neumann vector (moment_matrix.cu:177-201) of the scaled offset
        const float q9[9] = {nxf, nyf, nzf, 2.0f * b[0] * nxf, 2.0f * b[1] * nyf, 2.0f * b[2] * nzf,
                             fmaf(b[1], nxf, b[0] * nyf), fmaf(b[2], nyf, b[1] * nzf), fmaf(b[0], nzf, b[2] * nxf)};
        const float ng = static_cast<float>(a.p.gravity[0] * nrm.x + a.p.gravity[1] * nrm.y + a.p.gravity[2] * nrm.z);
        const float wq = w * wr * ng;
#pragma unroll
        for (int r = 0; r < 9; ++r) rhs[r] = fmaf(wq, q9[r], rhs[r]);
      }
      if (do_shift && s2 < dmin_s2) {
        const double d = sqrt(dx * dx + dy * dy + dz * dz);
        if (d > 0.0 && d < dmin) {
          const double push = scale * (dmin - d);
          shx = fma(push, nrm.x, shx);
          shy = fma(push, nrm.y, shy);
          shz = fma(push, nrm.z, shz);
        }
      }
  }
  }
  double rd[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) rd[r] = static_cast<double>(rhs[r]);
  if (G > 1) {
    const unsigned gm = group_mask<G>();
#pragma unroll
    for (int r = 0; r < 9; ++r) rd[r] = group_sum<G>(rd[r], gm);
    shx = group_sum<G>(shx, gm);
    shy = group_sum<G>(shy, gm);
    shz = group_sum<G>(shz, gm);
    nx = group_sum<G>(nx, gm);
    ny = group_sum<G>(ny, gm);
    nz = group_sum<G>(nz, gm);
    if (l != 0) return;
  }
  {
    float g[27];
    load_rows123f(out.prows, t, g);
    double c0 = 0.0, c1 = 0.0, c2 = 0.0;
#pragma unroll
    for (int col = 0; col < 9; ++col) {
      c0 = fma(static_cast<double>(g[col]), rd[col], c0);
      c1 = fma(static_cast<double>(g[9 + col]), rd[col], c1);
      c2 = fma(static_cast<double>(g[18 + col]), rd[col], c2);
    }
    out.gx[i] = c0 * inv_re;
    out.gy[i] = c1 * inv_re;
    out.gz[i] = c2 * inv_re;
  }
  if (do_shift) {
    if (is_surface(a.fluid.surface_type, i)) {
      const double nn = sqrt(nx * nx + ny * ny + nz * nz);
      if (nn > 0.0) {
        nx /= nn;
        ny /= nn;
        nz /= nn;
        const double nc = shx * nx + shy * ny + shz * nz;
        shx -= nc * nx;
        shy -= nc * ny;
        shz -= nc * nz;
      }
    }
    const double smax = a.p.ps_max_displacement_ratio * a.p.particle_spacing;
    const double sn = sqrt(shx * shx + shy * shy + shz * shz);
    if (sn > smax && sn > 0.0) {
      const double sc = smax / sn;
      shx *= sc;
      shy *= sc;
      shz *= sc;
    }
    out.sx[i] = shx;
    out.sy[i] = shy;
    out.sz[i] = shz;
  } else {
    out.sx[i] = out.sy[i] = out.sz[i] = 0.0;
  }
}

// update_velocity_position_kernel followed by anti_penetration_kernel for the
// same particle: the anti-penetration pass reads only the particle's own
// updated state and the walls, so running it right after the update in the
// same thread gives the same result as the two reference kernels.
__global__ void __launch_bounds__(kThreads) update_anti_penetration_kernel(
    lsmps_fluid f, const index_t* __restrict__ wo, const index_t* __restrict__ wi,
    const double* __restrict__ tx, const double* __restrict__ ty, const double* __restrict__ tz, double dt_host,
    const double* __restrict__ dtp, double density, const double* __restrict__ gx, const double* __restrict__ gy, const double* __restrict__ gz,
    const double* __restrict__ sx, const double* __restrict__ sy, const double* __restrict__ sz, double clearance,
    const double4* __restrict__ wp, const double4* __restrict__ wn) {
  const index_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= static_cast<index_t>(f.count)) return;
  const double dt = dtp ? *dtp : dt_host;
  const bool splash = is_splash(f.surface_type, i);
  const double ox = f.vx[i], oy = f.vy[i], oz = f.vz[i];
  double vx = tx[i], vy = ty[i], vz = tz[i];
  if (!splash) {
    const double ps = dt / density;
    vx -= ps * gx[i];
    vy -= ps * gy[i];
    vz -= ps * gz[i];
  }
  double x = f.x[i], y = f.y[i], z = f.z[i];
  x += 0.5 * dt * (ox + vx) + sx[i];
  y += 0.5 * dt * (oy + vy) + sy[i];
  z += 0.5 * dt * (oz + vz) + sz[i];
  if (clearance > 0.0 && wo[i] < wo[i + 1]) {
    // the wall records {x, y, z, -} and {nx, ny, nz, -}, the next wall's
    // loaded while this one is applied (in row order)
    const index_t wb = wo[i], we = wo[i + 1];
    index_t jn = wi[wb];
    double4 qn = ld4(wp, jn), nn = ld4(wn, jn);
    for (index_t o = wb; o < we; ++o) {
      const double4 q = qn, nrm = nn;
      if (o + 1 < we) {
        jn = wi[o + 1];
        qn = ld4(wp, jn);
        nn = ld4(wn, jn);
      }
      const double nx = nrm.x, ny = nrm.y, nz = nrm.z;
      const double sd = (x - q.x) * nx + (y - q.y) * ny + (z - q.z) * nz;
      if (sd >= clearance) continue;
      const double c = clearance - sd;
      x += c * nx;
      y += c * ny;
      z += c * nz;
      const double nv = vx * nx + vy * ny + vz * nz;
      if (nv < 0.0) {
        vx -= nv * nx;
        vy -= nv * ny;
        vz -= nv * nz;
      }
    }
  }
  f.x[i] = x;
  f.y[i] = y;
  f.z[i] = z;
  f.vx[i] = vx;
  f.vy[i] = vy;
  f.vz[i] = vz;
}

// gradient_shifting_kernel with the context's lane count (LSMPS_KNOB_GATHER_LANES).
template <bool Mixed>
void launch_gradient_shifting(lsmps_ctx* ctx, size_t count, const GatherArgs& a, const GradShiftOut& out) {
  const long long n = static_cast<long long>(count);
  switch (ctx->knob[LSMPS_KNOB_GATHER_LANES]) {
    case 1:
      launch_named(ctx, Mixed ? "gradient_shifting_kernel<true, 2>" : "gradient_shifting_kernel<false, 2>",
                   gradient_shifting_kernel<Mixed, 2>, dim3(div_up(2 * n, kThreads)), dim3(kThreads), 0, a, out);
      break;
    case 2:
      launch_named(ctx, Mixed ? "gradient_shifting_kernel<true, 4>" : "gradient_shifting_kernel<false, 4>",
                   gradient_shifting_kernel<Mixed, 4>, dim3(div_up(4 * n, kThreads)), dim3(kThreads), 0, a, out);
      break;
    default:
      launch_named(ctx, Mixed ? "gradient_shifting_kernel<true, 1>" : "gradient_shifting_kernel<false, 1>",
                   gradient_shifting_kernel<Mixed, 1>, dim3(div_up(n, kThreads)), dim3(kThreads), 0, a, out);
  }
}

// The mixed form: FP32 kernel, then the FP64-route particles.
void launch_gradient32(lsmps_ctx* ctx, size_t count, const GatherArgs& a, const GradShiftOut& out) {
  const long long n = static_cast<long long>(count);
  const dim3 list_grid(static_cast<unsigned>(ctx->sm_count * 2));
  switch (ctx->knob[LSMPS_KNOB_GATHER_LANES]) {
    case 1:
      launch_named(ctx, "gradient32_kernel<2>", gradient32_kernel<2>, dim3(div_up(2 * n, kThreads)), dim3(kThreads), 0,
                   a, out);
      launch_named(ctx, "gradient_shifting_list_kernel<2>", gradient_shifting_list_kernel<2>, list_grid,
                   dim3(kThreads), 0, a, out);
      break;
    case 2:
      launch_named(ctx, "gradient32_kernel<4>", gradient32_kernel<4>, dim3(div_up(4 * n, kThreads)), dim3(kThreads), 0,
                   a, out);
      launch_named(ctx, "gradient_shifting_list_kernel<4>", gradient_shifting_list_kernel<4>, list_grid,
                   dim3(kThreads), 0, a, out);
      break;
    default:
      launch_named(ctx, "gradient32_kernel<1>", gradient32_kernel<1>, dim3(div_up(n, kThreads)), dim3(kThreads), 0, a,
                   out);
      launch_named(ctx, "gradient_shifting_list_kernel<1>", gradient_shifting_list_kernel<1>, list_grid,
                   dim3(kThreads), 0, a, out);
  }
}

}  // namespace

// Pressure clamp, LSMPS pressure gradient and particle shifting in one pass
// (the first half of the fused correction; also run alone by the autotuner:
// it writes only the gradient and shift vectors and the clamped pressure,
// which the step clamps anyway).
lsmps_status gradient_shifting_stage(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w,
                                     const lsmps_csr& fn, const lsmps_csr& wn, double* pressure,
                                     const lsmps_params& p, const lsmps_moment& pm, const lsmps_vector& g,
                                     const lsmps_vector& s, bool mixed) {
  if (f.count == 0) return LSMPS_OK;
  if (const lsmps_status cs = check_neighbor_tables(ctx, f.count, w.count, fn, &wn)) return cs;
  const index_t* srows = sorted_rows_of(ctx, fn, f.count);
  GatherArgs a{f, w, fn.offsets, srows ? srows : fn.indices, wn.offsets, wn.indices, p};
  a.sorted = srows ? 1 : 0;
  if (!ensure_packs(ctx, f.count, w.count)) return fail(ctx, LSMPS_CUDA_ERROR, "pack allocation failed");
  pack4(ctx, f.x, f.y, f.z, pressure, f.count, ctx->pack_fluid[0], srows ? ctx->order : nullptr);
  pack_wall_positions(ctx, w);
  pack_wall_normals(ctx, w);
  a.fpp = ctx->pack_fluid[0];
  a.wp = ctx->pack_wall[0];
  a.wn = ctx->pack_wall[2];
  a.order = ctx->order;
  GradShiftOut out{pressure, f.pressure, nullptr, MixedRows{}, pm.support_radius, pm.wall_weight_scale,
                   g.x, g.y, g.z, s.x, s.y, s.z};
  if (mixed) {
    if (!ctx->mixed_rows[1] || !ctx->mixed_count || ctx->mixed_cap < f.count)
      return fail(ctx, LSMPS_NOT_PREPARED, "mixed pressure operator rows were not prepared");
    out.prows = mixed_rows_of(ctx, 1);
    launch_gradient32(ctx, f.count, a, out);
  } else {
    if (!pm.inverse_matrices) return fail(ctx, LSMPS_INVALID_ARGUMENT, "pressure inverse buffer missing");
    out.pinv = pm.inverse_matrices;
    launch_gradient_shifting<false>(ctx, f.count, a, out);
  }
  return check_launch(ctx, "gradient/shifting");
}

lsmps_status pressure_correction_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w,
                                      const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_fluid& t,
                                      double* pressure, const lsmps_params& p, const lsmps_moment& pm,
                                      const lsmps_vector& g, const lsmps_vector& s, const lsmps_vector& sm,
                                      bool mixed) {
  lsmps_status st = check_fluid(ctx, f);
  if (st) return st;
  if (f.count > 0 && !pressure) return fail(ctx, LSMPS_INVALID_ARGUMENT, "Pressure correction requires a pressure array");
  if ((st = check_vector(ctx, f, g, "Pressure gradient workspace is too small"))) return st;
  if ((st = check_vector(ctx, f, s, "PS displacement workspace is too small"))) return st;
  if (t.count < f.count || (f.count && (!t.vx || !t.vy || !t.vz)))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Pressure correction temporary velocity target is too small");
  if (pm.kind != LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_A || pm.matrix_size != 9 || pm.particle_count < f.count)
    return fail(ctx, LSMPS_NOT_PREPARED, "Pressure correction requires a prepared pressure Type-A moment matrix");
  if (f.count == 0) return LSMPS_OK;
  st = gradient_shifting_stage(ctx, f, w, fn, wn, pressure, p, pm, g, s, mixed);
  if (st) return st;
  const int blocks = div_up(static_cast<long long>(f.count), kThreads);
  launch(ctx, update_anti_penetration_kernel, dim3(blocks), dim3(kThreads), 0, f,
         static_cast<const index_t*>(wn.offsets), static_cast<const index_t*>(wn.indices),
         static_cast<const double*>(t.vx), static_cast<const double*>(t.vy), static_cast<const double*>(t.vz),
         p.time_step, ctx->device_dt, p.density, static_cast<const double*>(g.x), static_cast<const double*>(g.y),
         static_cast<const double*>(g.z), static_cast<const double*>(s.x), static_cast<const double*>(s.y),
         static_cast<const double*>(s.z), p.wall_clearance_ratio * p.particle_spacing,
         static_cast<const double4*>(ctx->pack_wall[0]), static_cast<const double4*>(ctx->pack_wall[2]));
  st = check_launch(ctx, "gradient/shifting, update/anti-penetration");
  if (!st) st = smooth_impl(ctx, f, fn, p, sm, true);
  return st;
}

}  // namespace lsmps

using namespace lsmps;

#define LSMPS_API_BODY(expr)                  \
  do {                                        \
    lsmps_status st_ = begin_call(ctx);       \
    if (st_) return st_;                      \
    return end_call(ctx, (expr));             \
  } while (0)

extern "C" {

lsmps_status lsmps_clamp_particle_pressure(lsmps_ctx* ctx, const lsmps_fluid* fluid, double* pressure) {
  if (!ctx || !fluid) return LSMPS_INVALID_ARGUMENT;
  LSMPS_API_BODY(clamp_pressure_impl(ctx, *fluid, pressure));
}

lsmps_status lsmps_pressure_gradient(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_walls* walls,
                                     const lsmps_csr* fn, const lsmps_csr* wn, const double* pressure,
                                     const lsmps_params* params, const lsmps_moment* pm, const lsmps_vector* g) {
  if (!ctx || !fluid || !walls || !fn || !wn || !params || !pm || !g) return LSMPS_INVALID_ARGUMENT;
  LSMPS_API_BODY(pressure_gradient_impl(ctx, *fluid, *walls, *fn, *wn, pressure, *params, *pm, *g));
}

lsmps_status lsmps_particle_shifting(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_walls* walls,
                                     const lsmps_csr* fn, const lsmps_csr* wn, const lsmps_params* params,
                                     const lsmps_vector* s) {
  if (!ctx || !fluid || !walls || !fn || !wn || !params || !s) return LSMPS_INVALID_ARGUMENT;
  LSMPS_API_BODY(particle_shifting_impl(ctx, *fluid, *walls, *fn, *wn, *params, *s));
}

lsmps_status lsmps_update_velocity_position(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_fluid* t,
                                            const lsmps_params* params, const lsmps_vector* g,
                                            const lsmps_vector* s) {
  if (!ctx || !fluid || !t || !params || !g || !s) return LSMPS_INVALID_ARGUMENT;
  LSMPS_API_BODY(update_impl(ctx, *fluid, *t, *params, *g, *s));
}

lsmps_status lsmps_anti_penetration(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_walls* walls,
                                    const lsmps_csr* wn, const lsmps_params* params) {
  if (!ctx || !fluid || !walls || !wn || !params) return LSMPS_INVALID_ARGUMENT;
  LSMPS_API_BODY(anti_penetration_impl(ctx, *fluid, *walls, *wn, *params));
}

lsmps_status lsmps_smooth_particle_velocity(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_csr* fn,
                                            const lsmps_params* params, const lsmps_vector* sm) {
  if (!ctx || !fluid || !fn || !params || !sm) return LSMPS_INVALID_ARGUMENT;
  LSMPS_API_BODY(smooth_impl(ctx, *fluid, *fn, *params, *sm, true));
}

lsmps_status lsmps_pressure_correction(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_walls* walls,
                                       const lsmps_csr* fn, const lsmps_csr* wn, const lsmps_fluid* t,
                                       double* pressure, const lsmps_params* params, const lsmps_moment* pm,
                                       const lsmps_vector* g, const lsmps_vector* s, const lsmps_vector* sm) {
  if (!ctx || !fluid || !walls || !fn || !wn || !t || !params || !pm || !g || !s || !sm)
    return LSMPS_INVALID_ARGUMENT;
  LSMPS_API_BODY(pressure_correction_impl(ctx, *fluid, *walls, *fn, *wn, *t, pressure, *params, *pm, *g, *s, *sm));
}

}  // extern "C"
