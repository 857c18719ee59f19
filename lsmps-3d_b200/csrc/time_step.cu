// time_step.cu - the driver's time-step control on the device.
//
// The reference takes the step's time step on the host: max_velocity
// (src/app/simulation_driver.cu:110-143) computes |u| per fluid particle on
// the device, copies all N magnitudes to the host and takes the largest
// finite one there; SimulationTimeManager::advance (src/core/time_step.cpp:
// 104-150) then forms dt = clamp(min(dt_prev * growth, cfl * l0 / |u|max),
// min, max), cut to the remaining time.  Here both run on the device into a
// device-resident lsmps_time_state, and the kernels that use dt can read it
// from there (lsmps_ctx_set_device_time_step), so a time loop needs no host
// round trip and can be captured in one CUDA graph.
//
// The magnitudes use the reference's expression sqrt(vx*vx + vy*vy + vz*vz);
// the maximum of finite values does not depend on the reduction order, and
// the dt formula is the same sequence of IEEE operations: the state matches
// the reference's host computation bit for bit.
#include <algorithm>
#include <cmath>

#include "impl.cuh"

namespace lsmps {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double warp_max(double v) {
  for (int d = 16; d > 0; d >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, d));
  return v;
}

// partial[bx] = the largest finite |u| in this block's slice (0 if none).
__global__ void __launch_bounds__(kThreads) max_speed_kernel(lsmps_fluid f, double* __restrict__ partial) {
  double m = 0.0;
  for (index_t i = blockIdx.x * kThreads + threadIdx.x; i < static_cast<index_t>(f.count);
       i += gridDim.x * kThreads) {
    const double vx = f.vx[i], vy = f.vy[i], vz = f.vz[i];
    const double s = sqrt(vx * vx + vy * vy + vz * vz);
    if (isfinite(s) && s > m) m = s;
  }
  __shared__ double red[kThreads / kWarp];
  m = warp_max(m);
  if ((threadIdx.x & (kWarp - 1)) == 0) red[threadIdx.x / kWarp] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kThreads / kWarp; ++w) m = fmax(m, red[w]);
    partial[blockIdx.x] = m;
  }
}

// The maximum over the partials, then SimulationTimeManager::advance.
__global__ void __launch_bounds__(kThreads)
    advance_kernel(const double* __restrict__ partial, int nb, lsmps_time_limits lim, lsmps_time_state* st) {
  double m = 0.0;
  for (int b = threadIdx.x; b < nb; b += kThreads) m = fmax(m, partial[b]);
  __shared__ double red[kThreads / kWarp];
  m = warp_max(m);
  if ((threadIdx.x & (kWarp - 1)) == 0) red[threadIdx.x / kWarp] = m;
  __syncthreads();
  if (threadIdx.x != 0) return;
  for (int w = 1; w < kThreads / kWarp; ++w) m = fmax(m, red[w]);
  const double umax = m;
  // cfl_limited_time_step, time_step.cpp:104-111
  const double cfl_dt = (!(umax > 0.0) || !isfinite(umax)) ? lim.max_time_step : lim.cfl * lim.particle_spacing / umax;
  // next_time_step, time_step.cpp:113-122 (std::min, std::clamp)
  const double growth_limited = st->time_step * lim.growth_factor;
  double dt = cfl_dt < growth_limited ? cfl_dt : growth_limited;
  dt = dt < lim.min_time_step ? lim.min_time_step : (lim.max_time_step < dt ? lim.max_time_step : dt);
  const double remaining = lim.final_time - st->current_time;
  if (remaining > 0.0 && dt > remaining) dt = remaining;
  // advance, time_step.cpp:124-132
  st->current_time += dt;
  st->time_step = dt;
  st->cfl_time_step = cfl_dt;
  st->max_velocity = umax;
  st->step_index += 1;
}

bool positive_finite(double v) { return std::isfinite(v) && v > 0.0; }

}  // namespace

lsmps_status validate_time_limits(lsmps_ctx* ctx, const lsmps_time_limits& l) {
  // validate_time_step_limits, time_step.cpp:61-78
  if (!positive_finite(l.min_time_step) || !positive_finite(l.max_time_step) || !positive_finite(l.growth_factor) ||
      !positive_finite(l.cfl) || !positive_finite(l.particle_spacing) || !std::isfinite(l.final_time) ||
      l.final_time < 0.0)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "TimeStepLimits fields must be positive and finite");
  if (l.growth_factor < 1.0) return fail(ctx, LSMPS_INVALID_ARGUMENT, "TimeStepLimits field 'growth_factor' must be >= 1");
  if (l.min_time_step > l.max_time_step)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "TimeStepLimits requires min_time_step <= max_time_step");
  return LSMPS_OK;
}

lsmps_status advance_time_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_time_limits& lim,
                               lsmps_time_state* st) {
  lsmps_status s = validate_time_limits(ctx, lim);
  if (s) return s;
  if (!st) return fail(ctx, LSMPS_INVALID_ARGUMENT, "time state missing");
  if (f.count > 0 && (!f.vx || !f.vy || !f.vz)) return fail(ctx, LSMPS_INVALID_ARGUMENT, "fluid velocity missing");
  const int nb = static_cast<int>(std::min<long long>(div_up(static_cast<long long>(f.count), kThreads),
                                                      2LL * ctx->sm_count));
  Scratch scratch(ctx);
  if (!scratch.reserve(static_cast<size_t>(nb + 1) * sizeof(double) + 512))
    return fail(ctx, LSMPS_CUDA_ERROR, "scratch allocation failed");
  double* partial = scratch.take<double>(nb + 1);
  if (!partial) return fail(ctx, LSMPS_CUDA_ERROR, "scratch exhausted");
  if (nb > 0) launch(ctx, max_speed_kernel, dim3(nb), dim3(kThreads), 0, f, partial);
  launch(ctx, advance_kernel, dim3(1), dim3(kThreads), 0, static_cast<const double*>(partial), nb, lim, st);
  return check_launch(ctx, "time-step control");
}

}  // namespace lsmps

using namespace lsmps;

extern "C" void lsmps_time_state_init(const lsmps_time_limits* limits, double time_step, lsmps_time_state* out) {
  if (!limits || !out) return;
  // SimulationTimeManager::reset, time_step.cpp:85-94
  const double lo = limits->min_time_step, hi = limits->max_time_step;
  out->current_time = 0.0;
  out->time_step = time_step < lo ? lo : (hi < time_step ? hi : time_step);
  out->cfl_time_step = 0.0;
  out->max_velocity = 0.0;
  out->step_index = 0;
}

extern "C" lsmps_status lsmps_advance_time(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_time_limits* limits,
                                           lsmps_time_state* device_state) {
  if (!ctx || !fluid || !limits) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  st = advance_time_impl(ctx, *fluid, *limits, device_state);
  return end_call(ctx, st);
}

extern "C" lsmps_status lsmps_ctx_set_device_time_step(lsmps_ctx* ctx, const double* device_time_step) {
  if (!ctx) return LSMPS_INVALID_ARGUMENT;
  ctx->device_dt = device_time_step;
  return LSMPS_OK;
}

extern "C" lsmps_status lsmps_ctx_set_cell_order(lsmps_ctx* ctx, int on) {
  if (!ctx) return LSMPS_INVALID_ARGUMENT;
  ctx->cell_order = on != 0;
  return LSMPS_OK;
}

extern "C" lsmps_status lsmps_ctx_copy_sorted_rows(lsmps_ctx* ctx, int32_t* dst, size_t count) {
  if (!ctx || (count > 0 && !dst)) return LSMPS_INVALID_ARGUMENT;
  if (!ctx->spos_table || count > ctx->fluid_spos_cap)
    return lsmps::fail(ctx, LSMPS_NOT_PREPARED, "no cell-sorted rows of that length are held");
  if (count && cudaMemcpyAsync(dst, ctx->fluid_spos, count * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                               ctx->stream) != cudaSuccess)
    return lsmps::check_launch(ctx, "sorted rows copy");
  return ctx->synchronous ? lsmps_ctx_synchronize(ctx) : LSMPS_OK;
}

extern "C" lsmps_status lsmps_ctx_set_sorted_rows(lsmps_ctx* ctx, int on) {
  if (!ctx) return LSMPS_INVALID_ARGUMENT;
  ctx->sorted_rows = on != 0;
  if (!ctx->sorted_rows) ctx->spos_table = nullptr;
  return LSMPS_OK;
}
