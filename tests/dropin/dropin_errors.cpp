// dropin_errors.cpp - error behaviour of the C++17 drop-in (lsmps-3d_b200/dropin)
// against the reference's convention: a failed check prints one line to
// stderr and exits with EXIT_FAILURE; with LSMPS_DROPIN_THROW=1 the same
// message is thrown as std::runtime_error.  Run by tests/test_gpu_dropin.py:
//
//   dropin_errors capacity    neighbour table one entry short
//   dropin_errors unprepared  a moment view read before prepare_matrices
//   dropin_errors grid        a cell grid with a zero dimension
//
// Each case prints "caught: <message>" and returns 0 if the message was
// thrown; otherwise the drop-in has already ended the process.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "lsmps3d/moment_matrix/moment_matrix.cuh"
#include "lsmps3d/neighbor/neighbor_search.cuh"

namespace {

template <typename T>
T* device_array(const std::vector<T>& host) {
  T* p = nullptr;
  if (cudaMalloc(&p, (host.empty() ? 1 : host.size()) * sizeof(T)) != cudaSuccess) std::abort();
  if (!host.empty()) cudaMemcpy(p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice);
  return p;
}

int run(const char* which) {
  using namespace lsmps3d;
  // Four fluid particles in a row 0.5 apart, radius 0.75: six directed
  // fluid-fluid pairs; no walls.
  const std::vector<real> x{0.25, 0.75, 1.25, 1.75}, y(4, 0.25), z(4, 0.25);
  FluidParticleSoA fluid{};
  fluid.count = 4;
  fluid.x = device_array(x);
  fluid.y = device_array(y);
  fluid.z = device_array(z);
  WallParticleSoA walls{};
  SimulationConfig config;
  config.cell_origin = Vec3{0, 0, 0};
  config.cell_size = 1.0;
  config.cell_dims = Int3{2, 1, 1};
  config.support_radius = 0.75;
  const size_type cells = 2;
  CellListView fluid_cells{4, cells, device_array(std::vector<index_t>(4)), device_array(std::vector<index_t>(4)),
                           device_array(std::vector<index_t>(cells)), device_array(std::vector<index_t>(cells))};
  CellListView wall_cells{0, cells, nullptr, nullptr, device_array(std::vector<index_t>(cells)),
                          device_array(std::vector<index_t>(cells))};
  NeighborListView fluid_neighbors{4, 5, device_array(std::vector<index_t>(5)),
                                   device_array(std::vector<index_t>(5))};
  NeighborListView wall_neighbors{4, 0, device_array(std::vector<index_t>(5)), nullptr};
  if (std::strcmp(which, "capacity") == 0) {
    build_neighbor_lists(fluid, walls, config, fluid_cells, wall_cells, fluid_neighbors, wall_neighbors);
  } else if (std::strcmp(which, "unprepared") == 0) {
    DeviceMomentMatrix moments(4, config);
    (void)moments.velocity_type_a();
  } else if (std::strcmp(which, "grid") == 0) {
    build_cell_list(fluid, CellGrid{Vec3{0, 0, 0}, 1.0, Int3{2, 0, 1}}, fluid_cells);
  } else {
    std::fprintf(stderr, "unknown case %s\n", which);
    return 2;
  }
  std::printf("no error reported\n");
  return 3;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  try {
    return run(argv[1]);
  } catch (const std::runtime_error& e) {
    std::printf("caught: %s\n", e.what());
    return 0;
  }
}
