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

// The rows of particle number t in the visiting order (lsmps_ctx::order;
// the particle's index where there is none).
struct MixedRows {
  const float* f32;           // [n][36]
  const double* f64;          // [n][36], valid where flag[t] != 0
  const uint8_t* flag;        // [n]
  const int32_t* list;        // the flagged visiting positions, *count of them
  const unsigned int* count;
};

inline MixedRows mixed_rows_of(const lsmps_ctx* ctx, int kind) {
  return MixedRows{ctx->mixed_rows[kind], ctx->mixed_rows64[kind], ctx->mixed_flag[kind], ctx->mixed_list[kind],
                   ctx->mixed_count ? ctx->mixed_count + kind : nullptr};
}

// Row t (0..3) at visiting position i as floats (positions without the flag).  A
// particle's 36 floats start on 16 bytes: row 0 is read as two float4 and
// one float.
__device__ __forceinline__ void load_row9f(const MixedRows& r, index_t i, int t, float out[9]) {
  const float* p = r.f32 + static_cast<size_t>(i) * 36 + t * 9;
  if (t == 0) {
    const float4 a = reinterpret_cast<const float4*>(p)[0];
    const float4 b = reinterpret_cast<const float4*>(p)[1];
    out[0] = a.x, out[1] = a.y, out[2] = a.z, out[3] = a.w;
    out[4] = b.x, out[5] = b.y, out[6] = b.z, out[7] = b.w;
    out[8] = p[8];
    return;
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) out[c] = p[c];
}

// Rows 1, 2, 3 at visiting position i (floats 9..35) as g[0..26]: read as seven
// float4 over floats 8..35 (16-byte aligned), the first value dropped.
__device__ __forceinline__ void load_rows123f(const MixedRows& r, index_t i, float g[27]) {
  const float4* p = reinterpret_cast<const float4*>(r.f32 + static_cast<size_t>(i) * 36 + 8);
  float v[28];
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    const float4 q = p[k];
    v[4 * k] = q.x, v[4 * k + 1] = q.y, v[4 * k + 2] = q.z, v[4 * k + 3] = q.w;
  }
#pragma unroll
  for (int c = 0; c < 27; ++c) g[c] = v[c + 1];
}

// FP32 geometry of one neighbour from the FP64 coordinate difference d:
// s = d / r_e rounded to FP32, the Type-A basis of s, and the weight
// w = 1 - |s| (0 outside the support).  The weight is formed as
// (1 - |s|^2) / (1 + |s|) with |s|^2 and 1 - |s|^2 in FP64: for a neighbour
// near the edge of the support 1 - |s| cancels, and from FP32 components it
// would carry an absolute error of ~1e-7, a large relative error of a small
// weight (and of the PPE coefficient proportional to it); this form keeps the
// weight's relative error near FP32 rounding.  Returns w.
__device__ __forceinline__ float basis_f32(double dx, double dy, double dz, double inv_re, float b[9]) {
  const float inv_re_f = static_cast<float>(inv_re);
  const float sx = static_cast<float>(dx) * inv_re_f;
  const float sy = static_cast<float>(dy) * inv_re_f;
  const float sz = static_cast<float>(dz) * inv_re_f;
  const double s2 = fma(dx, dx, fma(dy, dy, dz * dz)) * (inv_re * inv_re);
  const float w = s2 < 1.0 ? __fdividef(static_cast<float>(1.0 - s2), 1.0f + sqrtf(static_cast<float>(s2))) : 0.0f;
  b[0] = sx;
  b[1] = sy;
  b[2] = sz;
  b[3] = sx * sx;
  b[4] = sy * sy;
  b[5] = sz * sz;
  b[6] = sx * sy;
  b[7] = sy * sz;
  b[8] = sz * sx;
  return w;
}

// a . b for a row of 9 floats at a 16-byte aligned address (shared memory):
// read as two float4 and one float, three loads instead of nine.
__device__ __forceinline__ float dot9f_a16(const float* __restrict__ a, const float b[9]) {
  const float4 p = *reinterpret_cast<const float4*>(a);
  const float4 q = *reinterpret_cast<const float4*>(a + 4);
  float v = p.x * b[0];
  v = fmaf(p.y, b[1], v);
  v = fmaf(p.z, b[2], v);
  v = fmaf(p.w, b[3], v);
  v = fmaf(q.x, b[4], v);
  v = fmaf(q.y, b[5], v);
  v = fmaf(q.z, b[6], v);
  v = fmaf(q.w, b[7], v);
  return fmaf(a[8], b[8], v);
}

__device__ __forceinline__ float dot9f(const float a[9], const float b[9]) {
  float v = a[0] * b[0];
#pragma unroll
  for (int k = 1; k < 9; ++k) v = fmaf(a[k], b[k], v);
  return v;
}

// Row t (0..3) of the particle at visiting position i as doubles.
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
