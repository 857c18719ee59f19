// packed.cu - streaming pack kernels for 32-byte neighbour records.
#include "packed.cuh"

namespace lsmps {

__global__ void pack4_kernel(const double* __restrict__ a, const double* __restrict__ b,
                             const double* __restrict__ c, const double* __restrict__ d, index_t n,
                             double4* __restrict__ out, const index_t* __restrict__ order) {
  for (index_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const index_t j = order ? order[i] : i;
    out[i] = make_double4(a[j], b[j], c[j], d ? d[j] : 0.0);
  }
}

__global__ void pack4_label_kernel(const double* __restrict__ a, const double* __restrict__ b,
                                   const double* __restrict__ c, const int32_t* __restrict__ label, index_t n,
                                   double4* __restrict__ out, const index_t* __restrict__ order) {
  for (index_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const index_t j = order ? order[i] : i;
    out[i] = make_double4(a[j], b[j], c[j], label ? static_cast<double>(label[j]) : 0.0);
  }
}

int stream_blocks(lsmps_ctx* ctx, size_t n) {
  const long long b = div_up(static_cast<long long>(n), 256);
  const long long cap = static_cast<long long>(ctx->sm_count) * 8;
  return static_cast<int>(b < 1 ? 1 : (b < cap ? b : cap));
}

namespace {

constexpr unsigned kWallPositions = 1u, kWallNormals = 2u, kFluidPositions = 4u;

// A pack into one of the reusable buffers replaces what it held.
void forget(lsmps_ctx* ctx, const double4* out) {
  if (out == ctx->pack_wall[0]) ctx->packs_ready &= ~kWallPositions;
  if (out == ctx->pack_wall[2]) ctx->packs_ready &= ~kWallNormals;
  if (out == ctx->pack_fluid[0]) ctx->packs_ready &= ~kFluidPositions;
}

}  // namespace

void pack4(lsmps_ctx* ctx, const double* a, const double* b, const double* c, const double* d, size_t n,
           double4* out, const index_t* order) {
  forget(ctx, out);
  if (n == 0) return;
  launch(ctx, pack4_kernel, dim3(stream_blocks(ctx, n)), dim3(256), 0, a, b, c, d, static_cast<index_t>(n), out,
         order);
}

void pack4_label(lsmps_ctx* ctx, const double* a, const double* b, const double* c, const int32_t* label, size_t n,
                 double4* out, const index_t* order) {
  forget(ctx, out);
  if (n == 0) return;
  launch(ctx, pack4_label_kernel, dim3(stream_blocks(ctx, n)), dim3(256), 0, a, b, c, label,
         static_cast<index_t>(n), out, order);
}

void pack_wall_positions(lsmps_ctx* ctx, const lsmps_walls& w) {
  if (ctx->step_packs && (ctx->packs_ready & kWallPositions)) return;
  pack4(ctx, w.x, w.y, w.z, nullptr, w.count, ctx->pack_wall[0]);
  if (ctx->step_packs) ctx->packs_ready |= kWallPositions;
}

void pack_wall_normals(lsmps_ctx* ctx, const lsmps_walls& w) {
  if (ctx->step_packs && (ctx->packs_ready & kWallNormals)) return;
  pack4(ctx, w.normal_x, w.normal_y, w.normal_z, nullptr, w.count, ctx->pack_wall[2]);
  if (ctx->step_packs) ctx->packs_ready |= kWallNormals;
}

void pack_fluid_positions(lsmps_ctx* ctx, const lsmps_fluid& f, const index_t* order) {
  if (ctx->step_packs && (ctx->packs_ready & kFluidPositions) && ctx->packs_fluid_order == order) return;
  pack4(ctx, f.x, f.y, f.z, nullptr, f.count, ctx->pack_fluid[0], order);
  if (ctx->step_packs) {
    ctx->packs_ready |= kFluidPositions;
    ctx->packs_fluid_order = order;
  }
}

}  // namespace lsmps
