// autotune.cu - lsmps_autotune: picks each launch-shape knob (lsmps_knob) by
// timing its variants on the caller's own state.
//
// Only stages that are pure functions of the step state are timed, so tuning
// never advances the simulation: the moment stage (its outputs are rebuilt
// from the positions) for LSMPS_KNOB_MOMENT_OCCUPANCY and the PPE assembly
// (rebuilt from u*, the moments and the CSR) for LSMPS_KNOB_PPE_LANES, the
// velocity Laplacian, gradient/shifting and smoothing gathers (their outputs are
// rebuilt from the state; the smoothing result is not copied back) for
// LSMPS_KNOB_GATHER_LANES.  The
// state's temporary velocity must hold u* of the current positions (it does
// after any lsmps_step or the provision entry points); its values only feed
// the timed kernels' arithmetic, not their control flow.
//
// Each variant is launched once untimed, then `repeats` times between two
// CUDA events on the context's stream; the variant with the smallest mean
// time wins and stays set on the context.
#include <cfloat>

#include "impl.cuh"

using namespace lsmps;

namespace {

template <typename F>
lsmps_status time_variants(lsmps_ctx* ctx, int knob, int repeats, F&& run, double* best_ms_out) {
  const int variants = lsmps_knob_variants(knob);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return fail(ctx, LSMPS_CUDA_ERROR, "autotune event creation failed");
  }
  int best = ctx->knob[knob];
  double best_ms = DBL_MAX;
  lsmps_status st = LSMPS_OK;
  for (int v = 0; v < variants && !st; ++v) {
    ctx->knob[knob] = v;
    st = run();  // warm-up (and first-touch of any lazily grown buffer)
    if (st) break;
    cudaEventRecord(e0, ctx->stream);
    for (int r = 0; r < repeats && !st; ++r) st = run();
    cudaEventRecord(e1, ctx->stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      st = check_launch(ctx, "autotune timing");
      break;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double mean = static_cast<double>(ms) / repeats;
    if (mean < best_ms) {
      best_ms = mean;
      best = v;
    }
  }
  ctx->knob[knob] = best;
  if (best_ms_out) *best_ms_out = best_ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

}  // namespace

extern "C" lsmps_status lsmps_autotune(lsmps_ctx* ctx, const lsmps_params* params, const lsmps_step_state* s,
                                       int repeats, double* best_ms) {
  if (!ctx || !params || !s || repeats <= 0) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  const bool mixed = ctx->precision == LSMPS_PRECISION_MIXED;
  // time the kernels in the order lsmps_step will visit the fluid
  if (ctx->cell_order && s->fluid.count > 0 && s->fluid_cells.sorted_indices == ctx->built_order &&
      ctx->built_order_count == s->fluid.count)
    ctx->order = s->fluid_cells.sorted_indices;
  auto moments = [&]() -> lsmps_status {
    if (mixed)
      return mixed_step_moments_impl(ctx, s->fluid, s->walls, s->fluid_neighbors, s->wall_neighbors, *params,
                                     s->velocity_moment, s->pressure_moment);
    const lsmps_moment kinds[2] = {s->velocity_moment, s->pressure_moment};
    return prepare_moments_impl(ctx, s->fluid, s->walls, s->fluid_neighbors, s->wall_neighbors, *params, kinds, 2);
  };
  auto ppe = [&]() -> lsmps_status {
    if (mixed)
      return assemble_ppe_mixed_impl(ctx, s->fluid, s->walls, *params, s->fluid_neighbors, s->wall_neighbors,
                                     s->temporary_velocity, s->temporary_wall_velocity, s->velocity_moment,
                                     s->pressure_moment, s->ppe);
    return assemble_ppe_impl(ctx, s->fluid, s->walls, *params, s->fluid_neighbors, s->wall_neighbors,
                             s->temporary_velocity, s->temporary_wall_velocity, s->velocity_moment,
                             s->pressure_moment, s->ppe);
  };
  double ms[LSMPS_KNOB_COUNT] = {0.0, 0.0, 0.0};
  st = time_variants(ctx, LSMPS_KNOB_MOMENT_OCCUPANCY, repeats, moments, &ms[0]);
  // the PPE reads the moment outputs of the chosen variant
  if (!st) st = moments();
  if (!st) st = time_variants(ctx, LSMPS_KNOB_PPE_LANES, repeats, ppe, &ms[1]);
  // The three passes this knob shapes: the velocity Laplacian, the pressure
  // gradient + shifting pass (on a copy of the pressure, which it clamps in
  // place) and the smoothing pass without its copy back into the velocities.
  double* pressure_copy = nullptr;
  if (!st && s->pressure && s->fluid.count) {
    if (cudaMalloc(&pressure_copy, s->fluid.count * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      pressure_copy = nullptr;
      st = fail(ctx, LSMPS_CUDA_ERROR, "autotune pressure copy allocation failed");
    } else {
      cudaMemcpyAsync(pressure_copy, s->pressure, s->fluid.count * sizeof(double), cudaMemcpyDeviceToDevice,
                      ctx->stream);
    }
  }
  lsmps_fluid fluid_copy = s->fluid;
  fluid_copy.pressure = pressure_copy;
  auto gathers = [&]() -> lsmps_status {
    lsmps_status r = mixed ? velocity_laplacian_mixed_impl(ctx, s->fluid, s->walls, s->fluid_neighbors,
                                                           s->wall_neighbors, s->velocity_moment, s->velocity_laplacian)
                           : velocity_laplacian_impl(ctx, s->fluid, s->walls, s->fluid_neighbors, s->wall_neighbors,
                                                     s->velocity_moment, s->velocity_laplacian);
    if (!r && pressure_copy)
      r = gradient_shifting_stage(ctx, fluid_copy, s->walls, s->fluid_neighbors, s->wall_neighbors, pressure_copy,
                                  *params, s->pressure_moment, s->pressure_gradient, s->ps_displacement, mixed);
    if (!r) r = smooth_impl(ctx, s->fluid, s->fluid_neighbors, *params, s->smoothed_velocity, false);
    return r;
  };
  if (!st) st = time_variants(ctx, LSMPS_KNOB_GATHER_LANES, repeats, gathers, &ms[2]);
  if (pressure_copy) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(pressure_copy);
  }
  ctx->order = nullptr;
  if (best_ms)
    for (int k = 0; k < LSMPS_KNOB_COUNT; ++k) best_ms[k] = ms[k];
  return end_call(ctx, st);
}
