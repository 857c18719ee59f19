// mixed.cuh - operator rows of the mixed form (LSMPS_PRECISION_MIXED).
//
// Per fluid particle and moment kind the step's consumers need four rows of
// the inverse moment matrix: t = 0 the Laplacian row (rows 3 + 4 + 5), t = 1..3
// rows 0, 1, 2 (the gradient / divergence rows).  A particle whose matrix was
// factorised in FP32 and refined in FP64 keeps them as 36 floats; a particle
// whose matrix took the FP64 route (failed FP32 factor or condition estimate
// above the threshold) keeps them as 36 doubles, marked by flag = 1, so the
// consumers' FP64 arithmetic never sees an ill-conditioned row rounded to
// FP32.
#pragma once

#include "common.cuh"

namespace lsmps {

struct MixedRows {
  const float* f32;      // [n][36]
  const double* f64;     // [n][36], valid where flag[i] != 0
  const uint8_t* flag;   // [n]
};

inline MixedRows mixed_rows_of(const lsmps_ctx* ctx, int kind) {
  return MixedRows{ctx->mixed_rows[kind], ctx->mixed_rows64[kind], ctx->mixed_flag[kind]};
}

// Row t (0..3) of particle i as doubles.
__device__ __forceinline__ void load_row9(const MixedRows& r, index_t i, int t, double out[9]) {
  const size_t base = static_cast<size_t>(i) * 36 + t * 9;
  if (r.flag[i]) {
#pragma unroll
    for (int c = 0; c < 9; ++c) out[c] = r.f64[base + c];
  } else {
#pragma unroll
    for (int c = 0; c < 9; ++c) out[c] = static_cast<double>(r.f32[base + c]);
  }
}

}  // namespace lsmps
