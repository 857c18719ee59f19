// dropin.hpp - plumbing shared by the C++17 drop-in of lsmps3D's hot-path
// modules.
//
// The drop-in defines the reference's own module API (namespace lsmps3d, as
// declared by its headers include/lsmps3d/{neighbor,surface,moment_matrix,
// provision,ppe,correction}/*.cuh) on top of the C ABI of lsmps_b200.h.  Each
// .cpp file of this directory stands in for one source file of the reference:
//
//   neighbor_search.cpp      src/neighbor/neighbor_search.cu
//   surface_detection.cpp    src/surface/surface_detection.cu
//   moment_matrix.cpp        src/moment_matrix/moment_matrix.cu
//   explicit_update.cpp      src/provision/explicit_update.cu
//   ppe_matrix.cpp           src/ppe/ppe_matrix.cu
//   pressure_correction.cpp  src/correction/pressure_correction.cu
//
// so a build of lsmps3D links these (and liblsmps_b200.so) instead of those
// six files and keeps the rest of its tree (core/runtime.cu with the particle
// and neighbour-list owners, the driver, I/O) unchanged.
//
// Semantics kept from the reference:
// - every call runs on the legacy default stream and has finished when it
//   returns (the reference synchronises after each kernel);
// - a failed check prints one line to stderr and ends the process with
//   EXIT_FAILURE, as the reference's checks do.  With the environment
//   variable LSMPS_DROPIN_THROW=1 the drop-in throws std::runtime_error with
//   the same message instead, for hosts that must not exit.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "lsmps3d/core/config.hpp"
#include "lsmps3d/moment_matrix/moment_matrix.cuh"
#include "lsmps3d/neighbor/cell_list.cuh"
#include "lsmps3d/particle/neighbor_list.cuh"
#include "lsmps3d/particle/particle_data.cuh"
#include "lsmps_b200.h"

namespace lsmps3d::dropin {

static_assert(sizeof(real) == sizeof(double),
              "the drop-in implements the reference's LSMPS3D_USE_DOUBLE build (real = double)");
static_assert(sizeof(index_t) == sizeof(int32_t), "index_t is a 32-bit integer");

// The C ABI context of the calling thread's current device: created on first
// use, bound to the legacy default stream, synchronous.
lsmps_ctx* context();

// Reports a failed check the reference's way (see the file comment).
[[noreturn]] void fail(const std::string& message);

// A non-OK status of a C ABI call becomes fail(<the context's message>).
void check(lsmps_status status);

lsmps_params params_of(const SimulationConfig& config);
lsmps_grid grid_of(const CellGrid& grid);
lsmps_fluid view_of(const FluidParticleSoA& fluid);
lsmps_walls view_of(const WallParticleSoA& walls);
lsmps_csr view_of(const NeighborListView& neighbors);
lsmps_cells view_of(const CellListView& cells);
lsmps_moment view_of(const MomentMatrixView& moment);

// cudaMalloc / cudaFree of `count` elements, reporting failures as fail().
template <typename T>
void device_alloc(T*& ptr, size_type count) {
  ptr = nullptr;
  if (count == 0) return;
  if (cudaMalloc(reinterpret_cast<void**>(&ptr), count * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    fail("CUDA allocation failed");
  }
}

template <typename T>
void device_free(T*& ptr) noexcept {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
}

}  // namespace lsmps3d::dropin
