// impl.cuh - stream-ordered implementations behind the C ABI entry points.
// Each queues its kernels on ctx->stream and returns host-side validation
// failures; device-side status is folded by end_call / lsmps_ctx_synchronize.
#pragma once

#include "common.cuh"

namespace lsmps {

// The cell-sorted rows of fluid table fn (n particles) when the gathers may
// read them: this context's last build of that table wrote them for the cell
// list the fluid is being visited by (lsmps_ctx::order, set inside
// lsmps_step).  The gathers then read these rows and fluid records packed in
// that order (pack4's `order`), and a particle finds its own record at its
// visiting position (self_of).  NULL: CSR indices and records by index.
inline const index_t* sorted_rows_of(const lsmps_ctx* ctx, const lsmps_csr& fn, size_t n) {
  return (ctx->sorted_rows && ctx->order && ctx->spos_table == fn.offsets && ctx->spos_order == ctx->order &&
          ctx->spos_count == n && n > 0)
             ? ctx->fluid_spos
             : nullptr;
}

double reference_number_density(double l0, double re);
lsmps_status classify_surface_impl(lsmps_ctx* ctx, const lsmps_fluid& fluid, const lsmps_walls& walls,
                                   const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_params& p,
                                   const lsmps_surface_diagnostics* diag);
lsmps_status virtual_light_impl(lsmps_ctx* ctx, const lsmps_fluid& fluid, const lsmps_walls& walls,
                                const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_params& p,
                                int32_t* open_count, double* open_fraction);
lsmps_status prepare_moments_impl(lsmps_ctx* ctx, const lsmps_fluid& fluid, const lsmps_walls& walls,
                                  const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_params& p,
                                  const lsmps_moment* kinds, int count);
// Mixed form of the step's moment stage: compact FP32 operator rows of the
// velocity and pressure Type-A inverses in ctx->mixed_rows (the views get
// trace, regularisation, info and inversion_count; their inverse_matrices
// are not written).
lsmps_status mixed_step_moments_impl(lsmps_ctx* ctx, const lsmps_fluid& fluid, const lsmps_walls& walls,
                                     const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_params& p,
                                     const lsmps_moment& vm, const lsmps_moment& pm);
lsmps_status velocity_laplacian_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w,
                                     const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_moment& vm,
                                     const lsmps_vector& lap);
// Mixed form (after mixed_step_moments_impl in the same step: reads the
// position packs it left and ctx->mixed_rows).
lsmps_status velocity_laplacian_mixed_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w,
                                           const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_moment& vm,
                                           const lsmps_vector& lap);
lsmps_status temporary_velocity_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_params& p,
                                     const lsmps_vector& lap, const lsmps_fluid& t);
lsmps_status temporary_wall_velocity_impl(lsmps_ctx* ctx, const lsmps_walls& w, const lsmps_params& p,
                                          const lsmps_walls& t);
lsmps_status assemble_ppe_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w, const lsmps_params& p,
                               const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_fluid& tv,
                               const lsmps_walls& tw, const lsmps_moment& vm, const lsmps_moment& pm,
                               const lsmps_ppe& ws);
lsmps_status assemble_ppe_mixed_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w,
                                     const lsmps_params& p, const lsmps_csr& fn, const lsmps_csr& wn,
                                     const lsmps_fluid& tv, const lsmps_walls& tw, const lsmps_moment& vm,
                                     const lsmps_moment& pm, const lsmps_ppe& ws);
// Pressure clamp + gradient + particle shifting (the first half of the fused
// correction), and the velocity smoothing pass (copy_back = false leaves the
// smoothed velocity in `sm` only).
lsmps_status gradient_shifting_stage(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w,
                                     const lsmps_csr& fn, const lsmps_csr& wn, double* pressure,
                                     const lsmps_params& p, const lsmps_moment& pm, const lsmps_vector& g,
                                     const lsmps_vector& s, bool mixed);
lsmps_status smooth_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_csr& fn, const lsmps_params& p,
                         const lsmps_vector& sm, bool copy_back);
lsmps_status pressure_correction_impl(lsmps_ctx* ctx, const lsmps_fluid& f, const lsmps_walls& w,
                                      const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_fluid& t,
                                      double* pressure, const lsmps_params& p, const lsmps_moment& pm,
                                      const lsmps_vector& g, const lsmps_vector& s, const lsmps_vector& sm,
                                      bool mixed = false);
lsmps_status build_neighbor_lists_impl(lsmps_ctx* ctx, Scratch& scratch, const lsmps_fluid& fluid,
                                       const lsmps_walls& walls, const lsmps_params& p,
                                       const lsmps_cells& fc, const lsmps_cells& wc, const lsmps_csr& fn,
                                       const lsmps_csr& wn);
size_t neighbor_scratch_bytes(size_t n_fluid, size_t n_wall, size_t ncell);

}  // namespace lsmps
