// step.cu - one LSMPS time step on caller-owned buffers, in the reference
// driver's order (src/app/simulation_driver.cu:346-383 without the PPE solve
// and the I/O): moments -> provision -> PPE assembly -> pressure correction ->
// neighbour rebuild -> surface labels.  All work is queued on the context's
// stream with no host synchronisation inside, so a step can be captured in a
// CUDA graph once the context's scratch is reserved.
#include "impl.cuh"

using namespace lsmps;

namespace {

void wait_for_inputs(lsmps_ctx* ctx, bool overlap) {
  if (overlap && ctx->step_input_event)
    cudaStreamWaitEvent(ctx->stream, static_cast<cudaEvent_t>(ctx->step_input_event), 0);
}

}  // namespace

extern "C" lsmps_status lsmps_step(lsmps_ctx* ctx, const lsmps_params* params, const lsmps_step_state* s) {
  if (!ctx || !params || !s) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  StageRange step_range("lsmps_step");
  Scratch scratch(ctx);
  if (!scratch.reserve(neighbor_scratch_bytes(s->fluid.count, s->walls.count, s->fluid_cells.cell_count)))
    return fail(ctx, LSMPS_CUDA_ERROR, "scratch allocation failed (reserve before graph capture)");
  // The gather kernels visit the fluid in cell order: the fluid cell list of
  // the state, when this context built it last (every step ends by
  // rebuilding it; the caller builds it before the first step), so it is
  // known to be a permutation of the fluid.  The labels after the rebuild use
  // the rebuilt list.  The visiting order changes no result.
  if (ctx->cell_order && s->fluid.count > 0 && s->fluid_cells.sorted_indices == ctx->built_order &&
      ctx->built_order_count == s->fluid.count)
    ctx->order = s->fluid_cells.sorted_indices;
  // The driver prepares the moment caches once per geometry generation; the
  // geometry changes every step, so every step builds them once.  Each stage
  // is an NVTX range.
  const bool mixed = ctx->precision == LSMPS_PRECISION_MIXED;
  // Record packs made by one stage are reused by the next where their
  // contents are the same (packed.cuh).
  ctx->step_packs = true;
  ctx->packs_ready = 0;
  // The caller's copy/compute overlap events (lsmps_ctx_set_step_events),
  // outside stream capture only.
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(ctx->stream, &capture);
  const bool overlap = capture == cudaStreamCaptureStatusNone;
  {
    StageRange range("lsmps moments + velocity Laplacian");
    if (mixed) {
      // FP32 assembly and factorisation with FP64 refinement; the consumers
      // read the compact FP32 operator rows instead of the full inverses.
      // (the walls are first read after the fluid sums: the moment stage
      // waits for the caller's wall event there)
      ctx->walls_wait_event = overlap ? ctx->step_wall_event : nullptr;
      st = mixed_step_moments_impl(ctx, s->fluid, s->walls, s->fluid_neighbors, s->wall_neighbors, *params,
                                   s->velocity_moment, s->pressure_moment);
      ctx->walls_wait_event = nullptr;
      if (!st) wait_for_inputs(ctx, overlap);
      if (!st)
        st = velocity_laplacian_mixed_impl(ctx, s->fluid, s->walls, s->fluid_neighbors, s->wall_neighbors,
                                           s->velocity_moment, s->velocity_laplacian);
    } else {
      const lsmps_moment kinds[2] = {s->velocity_moment, s->pressure_moment};
      if (overlap && ctx->step_wall_event)
        cudaStreamWaitEvent(ctx->stream, static_cast<cudaEvent_t>(ctx->step_wall_event), 0);
      st = prepare_moments_impl(ctx, s->fluid, s->walls, s->fluid_neighbors, s->wall_neighbors, *params, kinds, 2);
      if (!st) wait_for_inputs(ctx, overlap);
      if (!st)
        st = velocity_laplacian_impl(ctx, s->fluid, s->walls, s->fluid_neighbors, s->wall_neighbors,
                                     s->velocity_moment, s->velocity_laplacian);
    }
  }
  {
    StageRange range("lsmps provision + PPE rows");
    if (!st) st = temporary_velocity_impl(ctx, s->fluid, *params, s->velocity_laplacian, s->temporary_velocity);
    if (!st) st = temporary_wall_velocity_impl(ctx, s->walls, *params, s->temporary_wall_velocity);
    if (!st && mixed)
      st = assemble_ppe_mixed_impl(ctx, s->fluid, s->walls, *params, s->fluid_neighbors, s->wall_neighbors,
                                   s->temporary_velocity, s->temporary_wall_velocity, s->velocity_moment,
                                   s->pressure_moment, s->ppe);
    else if (!st)
      st = assemble_ppe_impl(ctx, s->fluid, s->walls, *params, s->fluid_neighbors, s->wall_neighbors,
                             s->temporary_velocity, s->temporary_wall_velocity, s->velocity_moment,
                             s->pressure_moment, s->ppe);
  }
  {
    StageRange range("lsmps pressure correction");
    if (!st)
      st = pressure_correction_impl(ctx, s->fluid, s->walls, s->fluid_neighbors, s->wall_neighbors,
                                    s->temporary_velocity, s->pressure, *params, s->pressure_moment,
                                    s->pressure_gradient, s->ps_displacement, s->smoothed_velocity, mixed);
    if (!st && overlap && ctx->step_output_event &&
        cudaEventRecord(static_cast<cudaEvent_t>(ctx->step_output_event), ctx->stream) != cudaSuccess)
      st = check_launch(ctx, "step output event");
  }
  {
    StageRange range("lsmps neighbour rebuild + labels");
    if (!st)
      st = build_neighbor_lists_impl(ctx, scratch, s->fluid, s->walls, *params, s->fluid_cells, s->wall_cells,
                                     s->fluid_neighbors, s->wall_neighbors);
    if (!st)
      st = classify_surface_impl(ctx, s->fluid, s->walls, s->fluid_neighbors, s->wall_neighbors, *params, nullptr);
  }
  ctx->order = nullptr;
  ctx->step_packs = false;
  ctx->packs_ready = 0;
  return end_call(ctx, st);
}
