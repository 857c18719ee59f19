// packed.cuh - 32-byte neighbour records.
//
// Gather kernels read, for every CSR entry, several FP64 fields of the
// neighbour (x, y, z and one more: pressure, a velocity component, a label).
// Read from the SoA arrays each field is a separate 8-byte access in a
// different cache sector; packed as one double4 {x, y, z, aux} the record is
// one aligned 32-byte sector.  The packs are built by small streaming kernels
// from the caller's SoA arrays into context scratch before a gather kernel
// runs; the SoA arrays stay the interface.
#pragma once

#include "common.cuh"

namespace lsmps {

// out[k] = {a[j], b[j], c[j], d ? d[j] : 0} with j = order ? order[k] : k
// (order: a cell list's sorted indices, for records in cell-sorted order)
__global__ void pack4_kernel(const double* __restrict__ a, const double* __restrict__ b,
                             const double* __restrict__ c, const double* __restrict__ d, index_t n,
                             double4* __restrict__ out, const index_t* __restrict__ order);

// out[k] = {a[j], b[j], c[j], (double)label[j]} (label may be null -> 0), j as above
__global__ void pack4_label_kernel(const double* __restrict__ a, const double* __restrict__ b,
                                   const double* __restrict__ c, const int32_t* __restrict__ label, index_t n,
                                   double4* __restrict__ out, const index_t* __restrict__ order);

int stream_blocks(lsmps_ctx* ctx, size_t n);

// Queue a pack of three (or four) SoA arrays into out[n], in index order or,
// with `order`, in that order.
void pack4(lsmps_ctx* ctx, const double* a, const double* b, const double* c, const double* d, size_t n,
           double4* out, const index_t* order = nullptr);
void pack4_label(lsmps_ctx* ctx, const double* a, const double* b, const double* c, const int32_t* label, size_t n,
                 double4* out, const index_t* order = nullptr);

// The wall positions {x, y, z, 0} into pack_wall[0], the wall normals into
// pack_wall[2], the fluid positions into pack_fluid[0] (in `order`, as
// pack4).  Inside lsmps_step a repeated request finds the pack made earlier
// in the step (lsmps_ctx::packs_ready) and queues nothing.
void pack_wall_positions(lsmps_ctx* ctx, const lsmps_walls& w);
void pack_wall_normals(lsmps_ctx* ctx, const lsmps_walls& w);
void pack_fluid_positions(lsmps_ctx* ctx, const lsmps_fluid& f, const index_t* order);

// One record through the read-only path as one 32-byte vector load (sm_100:
// a single load instruction per record and lane, where two 16-byte loads
// cost two passes of the L1 data pipe for the same sector).  The records
// are 32-byte aligned (cudaMalloc'ed arrays of 32-byte records).
__device__ __forceinline__ double4 ld4(const double4* __restrict__ p, index_t j) {
  double4 r;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w)
      : "l"(p + j));
  return r;
}

}  // namespace lsmps
