// context.cu - the opaque context of the C ABI: stream, scratch, device status.
#include <cstring>
#include <new>

#include "impl.cuh"

namespace lsmps {

bool Scratch::reserve(size_t bytes) {
  if (bytes <= ctx_->scratch_bytes) return true;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(ctx_->stream, &cap);
  if (cap != cudaStreamCaptureStatusNone) return false;  // sizes must be reserved before capture
  if (ctx_->scratch) {
    cudaStreamSynchronize(ctx_->stream);
    cudaFree(ctx_->scratch);
    ctx_->scratch = nullptr;
    ctx_->scratch_bytes = 0;
  }
  const size_t grown = bytes + bytes / 4;
  if (cudaMalloc(&ctx_->scratch, grown) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  ctx_->scratch_bytes = grown;
  return true;
}

void free_mixed(lsmps_ctx* ctx) {
  if (ctx->mixed_sums) cudaFree(ctx->mixed_sums);
  ctx->mixed_sums = nullptr;
  if (ctx->mixed_count) cudaFree(ctx->mixed_count);
  ctx->mixed_count = nullptr;
  for (int k = 0; k < 2; ++k) {
    if (ctx->mixed_rows[k]) cudaFree(ctx->mixed_rows[k]);
    if (ctx->mixed_rows64[k]) cudaFree(ctx->mixed_rows64[k]);
    if (ctx->mixed_flag[k]) cudaFree(ctx->mixed_flag[k]);
    if (ctx->mixed_list[k]) cudaFree(ctx->mixed_list[k]);
    ctx->mixed_list[k] = nullptr;
    ctx->mixed_rows[k] = nullptr;
    ctx->mixed_rows64[k] = nullptr;
    ctx->mixed_flag[k] = nullptr;
  }
  ctx->mixed_cap = 0;
}

bool ensure_mixed(lsmps_ctx* ctx, size_t nf) {
  if (nf <= ctx->mixed_cap) return true;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(ctx->stream, &cap);
  if (cap != cudaStreamCaptureStatusNone) return false;
  cudaStreamSynchronize(ctx->stream);
  free_mixed(ctx);
  bool ok = cudaMalloc(&ctx->mixed_sums, nf * 31 * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ctx->mixed_count, 4 * sizeof(unsigned int)) == cudaSuccess;
  for (int k = 0; k < 2 && ok; ++k) {
    ok = cudaMalloc(&ctx->mixed_rows[k], nf * 36 * sizeof(float)) == cudaSuccess &&
         cudaMalloc(&ctx->mixed_rows64[k], nf * 36 * sizeof(double)) == cudaSuccess &&
         cudaMalloc(&ctx->mixed_flag[k], nf) == cudaSuccess &&
         cudaMalloc(&ctx->mixed_list[k], nf * sizeof(int32_t)) == cudaSuccess;
  }
  if (ok) ok = cudaMemsetAsync(ctx->mixed_count, 0, 4 * sizeof(unsigned int), ctx->stream) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    free_mixed(ctx);
    return false;
  }
  ctx->mixed_cap = nf;
  return true;
}

bool ensure_packs(lsmps_ctx* ctx, size_t nf, size_t nw) {
  if (nf <= ctx->pack_fluid_cap && nw <= ctx->pack_wall_cap) return true;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(ctx->stream, &cap);
  if (cap != cudaStreamCaptureStatusNone) return false;
  cudaStreamSynchronize(ctx->stream);
  ctx->packs_ready = 0;  // new buffers hold nothing a stage could reuse
  if (nf > ctx->pack_fluid_cap) {
    for (auto& p : ctx->pack_fluid) {
      if (p) cudaFree(p);
      p = nullptr;
    }
    ctx->pack_fluid_cap = 0;
    for (auto& p : ctx->pack_fluid)
      if (cudaMalloc(&p, nf * sizeof(double4)) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
    ctx->pack_fluid_cap = nf;
  }
  if (nw > ctx->pack_wall_cap) {
    for (auto& p : ctx->pack_wall) {
      if (p) cudaFree(p);
      p = nullptr;
    }
    ctx->pack_wall_cap = 0;
    for (auto& p : ctx->pack_wall)
      if (cudaMalloc(&p, nw * sizeof(double4)) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
    ctx->pack_wall_cap = nw;
  }
  return true;
}

bool ensure_sorted_rows(lsmps_ctx* ctx, size_t entries, size_t nf) {
  if (entries <= ctx->fluid_spos_cap && nf <= ctx->sorted_labels_cap) return true;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(ctx->stream, &cap);
  if (cap != cudaStreamCaptureStatusNone) return false;
  cudaStreamSynchronize(ctx->stream);
  ctx->spos_table = nullptr;
  if (entries > ctx->fluid_spos_cap) {
    if (ctx->fluid_spos) cudaFree(ctx->fluid_spos);
    ctx->fluid_spos = nullptr;
    ctx->fluid_spos_cap = 0;
    if (cudaMalloc(&ctx->fluid_spos, entries * sizeof(int32_t)) != cudaSuccess) {
      cudaGetLastError();
      ctx->fluid_spos = nullptr;
      return false;
    }
    ctx->fluid_spos_cap = entries;
  }
  if (nf > ctx->sorted_labels_cap) {
    if (ctx->sorted_labels) cudaFree(ctx->sorted_labels);
    ctx->sorted_labels = nullptr;
    ctx->sorted_labels_cap = 0;
    if (cudaMalloc(&ctx->sorted_labels, nf * sizeof(int32_t)) != cudaSuccess) {
      cudaGetLastError();
      ctx->sorted_labels = nullptr;
      return false;
    }
    ctx->sorted_labels_cap = nf;
  }
  return true;
}

lsmps_status fail(lsmps_ctx* ctx, lsmps_status st, const char* what) {
  if (ctx) ctx->last_error = what;
  return st;
}

lsmps_status check_launch(lsmps_ctx* ctx, const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return LSMPS_OK;
  ctx->last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return LSMPS_CUDA_ERROR;
}

lsmps_status begin_call(lsmps_ctx* ctx) {
  if (ctx->synchronous) {
    if (cudaMemsetAsync(ctx->d_status, 0, sizeof(DeviceStatus), ctx->stream) != cudaSuccess)
      return check_launch(ctx, "status reset");
  }
  return LSMPS_OK;
}

lsmps_status fold_status(lsmps_ctx* ctx) {
  if (cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(DeviceStatus), cudaMemcpyDeviceToHost,
                      ctx->stream) != cudaSuccess)
    return check_launch(ctx, "status readback");
  const cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    ctx->last_error = std::string("stream synchronize: ") + cudaGetErrorString(e);
    return LSMPS_CUDA_ERROR;
  }
  const DeviceStatus s = *ctx->h_status;
  cudaMemsetAsync(ctx->d_status, 0, sizeof(DeviceStatus), ctx->stream);
  ctx->fallbacks += s.fallbacks;
  if (s.flags & kFlagBadIndex) {
    ctx->last_error = "neighbour table offset or index out of range";
    return LSMPS_INVALID_ARGUMENT;
  }
  if (s.flags & kFlagNonFinite) {
    ctx->last_error = "non-finite particle coordinate";
    return LSMPS_NON_FINITE;
  }
  if (s.flags & kFlagIndexOverflow) {
    ctx->last_error = "count exceeds the 32-bit index range";
    return LSMPS_INDEX_OVERFLOW;
  }
  if (s.flags & kFlagCapacity) {
    ctx->required = s.required;
    ctx->last_error = "neighbour list capacity exceeded: required " + std::to_string(s.required);
    return LSMPS_CAPACITY_EXCEEDED;
  }
  return LSMPS_OK;
}

lsmps_ctx::ProfileRecord* profile_slot(lsmps_ctx* ctx, const char* name) {
  if (ctx->profile_used == ctx->profile.size()) {
    lsmps_ctx::ProfileRecord r{name, nullptr, nullptr};
    if (cudaEventCreate(&r.start) != cudaSuccess || cudaEventCreate(&r.stop) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    ctx->profile.push_back(r);
  }
  lsmps_ctx::ProfileRecord* r = &ctx->profile[ctx->profile_used++];
  r->name = name;
  return r;
}

lsmps_status end_call(lsmps_ctx* ctx, lsmps_status st) {
  if (st != LSMPS_OK) return st;
  const lsmps_status ls = check_launch(ctx, "kernel launch");
  if (ls != LSMPS_OK) return ls;
  if (!ctx->synchronous) return LSMPS_OK;
  return fold_status(ctx);
}

}  // namespace lsmps

using namespace lsmps;

extern "C" {

lsmps_status lsmps_ctx_create(int device, lsmps_ctx** out) {
  if (!out) return LSMPS_INVALID_ARGUMENT;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return LSMPS_CUDA_ERROR;
  }
  lsmps_ctx* ctx = new (std::nothrow) lsmps_ctx();
  if (!ctx) return LSMPS_CUDA_ERROR;
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&ctx->d_status, sizeof(DeviceStatus)) != cudaSuccess ||
      cudaMallocHost(&ctx->h_status, sizeof(DeviceStatus)) != cudaSuccess) {
    cudaGetLastError();
    lsmps_ctx_destroy(ctx);
    return LSMPS_CUDA_ERROR;
  }
  ctx->stream = ctx->own_stream;
  cudaMemsetAsync(ctx->d_status, 0, sizeof(DeviceStatus), ctx->stream);
  std::memset(ctx->h_status, 0, sizeof(DeviceStatus));
  cudaStreamSynchronize(ctx->stream);
  *out = ctx;
  return LSMPS_OK;
}

void lsmps_ctx_destroy(lsmps_ctx* ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& r : ctx->profile) {
    cudaEventDestroy(r.start);
    cudaEventDestroy(r.stop);
  }
  if (ctx->scratch) cudaFree(ctx->scratch);
  for (auto p : ctx->pack_fluid)
    if (p) cudaFree(p);
  for (auto p : ctx->pack_wall)
    if (p) cudaFree(p);
  if (ctx->fluid_spos) cudaFree(ctx->fluid_spos);
  if (ctx->sorted_labels) cudaFree(ctx->sorted_labels);
  free_mixed(ctx);
  free_adjoint(ctx);
  free_step_ops(ctx);
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->h_status) cudaFreeHost(ctx->h_status);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

lsmps_status lsmps_ctx_set_stream(lsmps_ctx* ctx, void* stream) {
  if (!ctx) return LSMPS_INVALID_ARGUMENT;
  // NULL selects the legacy default stream, so work orders with other users
  // of that stream (for example a framework's default stream).
  ctx->stream = static_cast<cudaStream_t>(stream);
  return LSMPS_OK;
}

void* lsmps_ctx_stream(lsmps_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

lsmps_status lsmps_ctx_set_precision(lsmps_ctx* ctx, int precision) {
  if (!ctx || (precision != LSMPS_PRECISION_PLAIN && precision != LSMPS_PRECISION_MIXED))
    return LSMPS_INVALID_ARGUMENT;
  ctx->precision = precision;
  return LSMPS_OK;
}

lsmps_status lsmps_ctx_set_synchronous(lsmps_ctx* ctx, int synchronous) {
  if (!ctx) return LSMPS_INVALID_ARGUMENT;
  ctx->synchronous = synchronous != 0;
  return LSMPS_OK;
}

lsmps_status lsmps_ctx_reserve(lsmps_ctx* ctx, size_t fluid_capacity, size_t wall_capacity, size_t cell_capacity) {
  if (!ctx) return LSMPS_INVALID_ARGUMENT;
  const size_t n = fluid_capacity > wall_capacity ? fluid_capacity : wall_capacity;
  size_t need = cell_list_scratch_bytes(n, cell_capacity);
  const size_t s2 = scan_scratch_bytes(fluid_capacity + 1) + 4096;
  if (s2 > need) need = s2;
  // what lsmps_step's neighbour rebuild takes, so that a step can be captured
  const size_t s3 = neighbor_scratch_bytes(fluid_capacity, wall_capacity, cell_capacity);
  if (s3 > need) need = s3;
  Scratch s(ctx);
  if (!s.reserve(need)) return fail(ctx, LSMPS_CUDA_ERROR, "scratch allocation failed");
  if (!ensure_packs(ctx, fluid_capacity, wall_capacity)) return fail(ctx, LSMPS_CUDA_ERROR, "pack allocation failed");
  if (ctx->precision == LSMPS_PRECISION_MIXED && !ensure_mixed(ctx, fluid_capacity))
    return fail(ctx, LSMPS_CUDA_ERROR, "mixed-form allocation failed");
  return LSMPS_OK;
}

lsmps_status lsmps_ctx_synchronize(lsmps_ctx* ctx) {
  if (!ctx) return LSMPS_INVALID_ARGUMENT;
  const lsmps_status ls = check_launch(ctx, "kernel launch");
  if (ls != LSMPS_OK) return ls;
  return fold_status(ctx);
}

uint64_t lsmps_ctx_required(lsmps_ctx* ctx) { return ctx ? ctx->required : 0; }

uint64_t lsmps_ctx_fp64_fallbacks(lsmps_ctx* ctx) { return ctx ? ctx->fallbacks : 0; }

lsmps_status lsmps_ctx_set_condition_threshold(lsmps_ctx* ctx, double threshold) {
  if (!ctx || !(threshold >= 1.0)) return LSMPS_INVALID_ARGUMENT;
  ctx->kappa_threshold = threshold;
  return LSMPS_OK;
}

int lsmps_knob_variants(int knob) {
  switch (knob) {
    case LSMPS_KNOB_MOMENT_OCCUPANCY: return 3;
    case LSMPS_KNOB_PPE_LANES: return 4;
    case LSMPS_KNOB_GATHER_LANES: return 3;
    default: return 0;
  }
}

lsmps_status lsmps_ctx_set_knob(lsmps_ctx* ctx, int knob, int value) {
  if (!ctx || knob < 0 || knob >= LSMPS_KNOB_COUNT || value < 0 || value >= lsmps_knob_variants(knob))
    return LSMPS_INVALID_ARGUMENT;
  ctx->knob[knob] = value;
  return LSMPS_OK;
}

int lsmps_ctx_knob(lsmps_ctx* ctx, int knob) {
  if (!ctx || knob < 0 || knob >= LSMPS_KNOB_COUNT) return -1;
  return ctx->knob[knob];
}

lsmps_status lsmps_ctx_set_step_events(lsmps_ctx* ctx, void* wall_event, void* input_event, void* output_event) {
  if (!ctx) return LSMPS_INVALID_ARGUMENT;
  ctx->step_wall_event = wall_event;
  ctx->step_input_event = input_event;
  ctx->step_output_event = output_event;
  return LSMPS_OK;
}

lsmps_status lsmps_ctx_set_profiling(lsmps_ctx* ctx, int on) {
  if (!ctx) return LSMPS_INVALID_ARGUMENT;
  ctx->profiling = on != 0;
  ctx->profile_used = 0;
  return LSMPS_OK;
}

int lsmps_ctx_profile_report(lsmps_ctx* ctx, char* names, size_t names_len, double* total_ms, uint64_t* launches,
                             int max_entries) {
  if (!ctx || max_entries < 0) return -1;
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  std::vector<std::string> keys;
  std::vector<double> ms;
  std::vector<uint64_t> cnt;
  for (size_t k = 0; k < ctx->profile_used; ++k) {
    const auto& r = ctx->profile[k];
    float t = 0.0f;
    if (cudaEventElapsedTime(&t, r.start, r.stop) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    size_t e = 0;
    while (e < keys.size() && keys[e] != r.name) ++e;
    if (e == keys.size()) {
      keys.emplace_back(r.name);
      ms.push_back(0.0);
      cnt.push_back(0);
    }
    ms[e] += t;
    ++cnt[e];
  }
  ctx->profile_used = 0;
  const int n = static_cast<int>(keys.size() < static_cast<size_t>(max_entries) ? keys.size() : max_entries);
  std::string joined;
  for (int e = 0; e < n; ++e) {
    if (total_ms) total_ms[e] = ms[e];
    if (launches) launches[e] = cnt[e];
    joined += keys[e];
    joined += '\n';
  }
  if (names && names_len) {
    const size_t m = joined.size() < names_len - 1 ? joined.size() : names_len - 1;
    std::memcpy(names, joined.data(), m);
    names[m] = '\0';
  }
  return n;
}

uint64_t lsmps_ctx_launch_count(lsmps_ctx* ctx) { return ctx ? ctx->launches : 0; }

const char* lsmps_ctx_last_error(lsmps_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

const char* lsmps_status_string(int status) {
  switch (status) {
    case LSMPS_OK: return "OK";
    case LSMPS_CAPACITY_EXCEEDED: return "CAPACITY_EXCEEDED";
    case LSMPS_INVALID_ARGUMENT: return "INVALID_ARGUMENT";
    case LSMPS_NOT_PREPARED: return "NOT_PREPARED";
    case LSMPS_NON_SPD: return "NON_SPD";
    case LSMPS_CUDA_ERROR: return "CUDA_ERROR";
    case LSMPS_INDEX_OVERFLOW: return "INDEX_OVERFLOW";
    case LSMPS_NON_FINITE: return "NON_FINITE";
    default: return "UNKNOWN";
  }
}

void lsmps_params_default(lsmps_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->particle_spacing = 0.01;
  p->support_radius = 0.031;
  p->near_surface_radius = 0.015;
  p->grid.cell_size = 0.031;
  p->grid.dims[0] = p->grid.dims[1] = p->grid.dims[2] = 1;
  p->time_step = 1.0e-4;
  p->density = 1000.0;
  p->kinematic_viscosity = 1.0e-6;
  p->gravity[2] = -9.81;
  p->splash_neighbor_threshold = 4;
  p->include_wall_neighbors = 1;
  p->number_density_ratio_threshold = 0.85;
  p->air_open_ratio_threshold = 0.33;
  p->air_anisotropy_threshold = 0.033;
  p->wall_normal_independence_threshold = 0.25;
  p->virtual_light_cone_cosine = 0.8660254037844386;
  p->lsmps_regularization = 1.0e-8;
  p->lsmps_wall_weight_scale = 1.0;
  p->ps_displacement_scale = 0.05;
  p->ps_min_distance_ratio = 0.85;
  p->ps_max_displacement_ratio = 0.2;
  p->wall_clearance_ratio = 0.25;
  p->velocity_smoothing_strength = 0.1;
}

}  // extern "C"
