// neighbor_search.cpp - the reference's neighbour-search module
// (include/lsmps3d/neighbor/neighbor_search.cuh:10-24, replacing
// src/neighbor/neighbor_search.cu) on the C ABI: cell lists with the
// library's stable radix sort and CSR tables in the reference's row order.
#include "lsmps3d/neighbor/neighbor_search.cuh"

#include <string>

#include "dropin.hpp"

namespace lsmps3d {

// build_cell_list(FluidParticleSoA, ...), neighbor_search.cu:337-339.
void build_cell_list(const FluidParticleSoA& particles, const CellGrid& grid, CellListView cells) {
  const lsmps_grid g = dropin::grid_of(grid);
  const lsmps_cells c = dropin::view_of(cells);
  dropin::check(lsmps_build_cell_list(dropin::context(), particles.x, particles.y, particles.z, particles.count,
                                      &g, &c));
}

// build_cell_list(WallParticleSoA, ...), neighbor_search.cu:341-343.
void build_cell_list(const WallParticleSoA& particles, const CellGrid& grid, CellListView cells) {
  const lsmps_grid g = dropin::grid_of(grid);
  const lsmps_cells c = dropin::view_of(cells);
  dropin::check(lsmps_build_cell_list(dropin::context(), particles.x, particles.y, particles.z, particles.count,
                                      &g, &c));
}

// build_neighbor_lists(...), neighbor_search.cu:345-367: both cell lists, then
// the fluid-fluid (self excluded) and fluid-wall tables.  A table whose
// capacity is too small fails with the required entry count.
void build_neighbor_lists(const FluidParticleSoA& fluid, const WallParticleSoA& walls,
                          const SimulationConfig& config, CellListView fluid_cells, CellListView wall_cells,
                          NeighborListView fluid_neighbors, NeighborListView wall_neighbors) {
  const lsmps_params p = dropin::params_of(config);
  const lsmps_fluid f = dropin::view_of(fluid);
  const lsmps_walls w = dropin::view_of(walls);
  const lsmps_cells fc = dropin::view_of(fluid_cells);
  const lsmps_cells wc = dropin::view_of(wall_cells);
  const lsmps_csr fn = dropin::view_of(fluid_neighbors);
  const lsmps_csr wn = dropin::view_of(wall_neighbors);
  lsmps_ctx* ctx = dropin::context();
  const lsmps_status st = lsmps_build_neighbor_lists(ctx, &f, &w, &p, &fc, &wc, &fn, &wn);
  if (st == LSMPS_CAPACITY_EXCEEDED) {
    // require_neighbor_capacity's report, neighbor_search.cu:22-30
    const uint64_t required = lsmps_ctx_required(ctx);
    const size_type capacity =
        required > fluid_neighbors.neighbor_count ? fluid_neighbors.neighbor_count : wall_neighbors.neighbor_count;
    dropin::fail("Neighbor list capacity exceeded: required " + std::to_string(required) + ", capacity " +
                 std::to_string(capacity));
  }
  dropin::check(st);
}

}  // namespace lsmps3d
