// surface_detection.cpp - the reference's surface module
// (include/lsmps3d/surface/surface_detection.cuh:10-43, replacing
// src/surface/surface_detection.cu) on the C ABI.
#include "lsmps3d/surface/surface_detection.cuh"

#include "dropin.hpp"

namespace lsmps3d {

// compute_uniform_reference_number_density, surface_detection.cu:494-520.
real compute_uniform_reference_number_density(real particle_spacing, real support_radius) {
  const double n0 = lsmps_reference_number_density(particle_spacing, support_radius);
  if (n0 < 0.0) dropin::fail("Reference number density requires positive spacing and support radius");
  return n0;
}

// classify_surface_particles, surface_detection.cu:522-553: primary labels
// and the NearSurface expansion; diagnostics pointers may be null.
void classify_surface_particles(const FluidParticleSoA& fluid, const WallParticleSoA& walls,
                                const NeighborListView& fluid_neighbors, const NeighborListView& wall_neighbors,
                                const SimulationConfig& config, SurfaceDetectionDiagnosticsView diagnostics) {
  const lsmps_params p = dropin::params_of(config);
  const lsmps_fluid f = dropin::view_of(fluid);
  const lsmps_walls w = dropin::view_of(walls);
  const lsmps_csr fn = dropin::view_of(fluid_neighbors);
  const lsmps_csr wn = dropin::view_of(wall_neighbors);
  const lsmps_surface_diagnostics d{diagnostics.fluid_neighbor_count, diagnostics.wall_neighbor_count,
                                    diagnostics.number_density,       diagnostics.number_density_ratio,
                                    diagnostics.anisotropy,           diagnostics.air_open_ratio,
                                    diagnostics.air_anisotropy,       diagnostics.surface_normal_x,
                                    diagnostics.surface_normal_y,     diagnostics.surface_normal_z};
  dropin::check(lsmps_classify_surface(dropin::context(), &f, &w, &fn, &wn, &p, &d));
}

// compute_virtual_light_diagnostics, surface_detection.cu:555-578.
void compute_virtual_light_diagnostics(const FluidParticleSoA& fluid, const WallParticleSoA& walls,
                                       const NeighborListView& fluid_neighbors,
                                       const NeighborListView& wall_neighbors, const SimulationConfig& config,
                                       VirtualLightDiagnosticsView diagnostics) {
  const lsmps_params p = dropin::params_of(config);
  const lsmps_fluid f = dropin::view_of(fluid);
  const lsmps_walls w = dropin::view_of(walls);
  const lsmps_csr fn = dropin::view_of(fluid_neighbors);
  const lsmps_csr wn = dropin::view_of(wall_neighbors);
  dropin::check(lsmps_virtual_light(dropin::context(), &f, &w, &fn, &wn, &p, diagnostics.open_direction_count,
                                    diagnostics.open_fraction));
}

}  // namespace lsmps3d
