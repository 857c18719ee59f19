// pressure_correction.cpp - the reference's correction module
// (include/lsmps3d/correction/pressure_correction.cuh:11-118, replacing
// src/correction/pressure_correction.cu) on the C ABI: pressure clamp, LSMPS
// pressure gradient, particle shifting, velocity/position update,
// anti-penetration and velocity smoothing.
#include "lsmps3d/correction/pressure_correction.cuh"

#include <utility>

#include "dropin.hpp"

namespace lsmps3d {
namespace {

void swap_vector_views(CorrectionVectorView& a, CorrectionVectorView& b) noexcept {
  std::swap(a.count, b.count);
  std::swap(a.x, b.x);
  std::swap(a.y, b.y);
  std::swap(a.z, b.z);
}

lsmps_vector vector_of(const CorrectionVectorView& v) { return lsmps_vector{v.count, v.x, v.y, v.z}; }

// validate_pressure_moment_matrix, pressure_correction.cu:96-111
void require_prepared_pressure_moment(const FluidParticleSoA& fluid, const MomentMatrixView& m) {
  if (!m.is_ready || m.kind != MomentMatrixKind::PressureWallNeumannTypeA ||
      m.basis_kind != MomentBasisKind::TypeA || m.matrix_size != kMomentTypeABasis3DSize ||
      m.particle_count < fluid.count)
    dropin::fail("Pressure correction requires a prepared pressure Type-A moment matrix");
  if (fluid.count > 0 && m.inverse_matrices == nullptr)
    dropin::fail("Pressure correction pressure moment inverse buffer is missing");
}

}  // namespace

DeviceCorrectionWorkspace::DeviceCorrectionWorkspace(size_type fluid_capacity) { resize(fluid_capacity); }

DeviceCorrectionWorkspace::~DeviceCorrectionWorkspace() { release(); }

DeviceCorrectionWorkspace::DeviceCorrectionWorkspace(DeviceCorrectionWorkspace&& other) noexcept {
  swap_vector_views(pressure_gradient_, other.pressure_gradient_);
  swap_vector_views(ps_displacement_, other.ps_displacement_);
  swap_vector_views(smoothed_velocity_, other.smoothed_velocity_);
}

DeviceCorrectionWorkspace& DeviceCorrectionWorkspace::operator=(DeviceCorrectionWorkspace&& other) noexcept {
  if (this != &other) {
    release();
    swap_vector_views(pressure_gradient_, other.pressure_gradient_);
    swap_vector_views(ps_displacement_, other.ps_displacement_);
    swap_vector_views(smoothed_velocity_, other.smoothed_velocity_);
  }
  return *this;
}

void DeviceCorrectionWorkspace::resize(size_type fluid_capacity) {
  if (fluid_capacity == pressure_gradient_.count) return;
  release();
  for (CorrectionVectorView* v : {&pressure_gradient_, &ps_displacement_, &smoothed_velocity_}) {
    v->count = fluid_capacity;
    dropin::device_alloc(v->x, fluid_capacity);
    dropin::device_alloc(v->y, fluid_capacity);
    dropin::device_alloc(v->z, fluid_capacity);
  }
}

void DeviceCorrectionWorkspace::release() noexcept {
  for (CorrectionVectorView* v : {&pressure_gradient_, &ps_displacement_, &smoothed_velocity_}) {
    dropin::device_free(v->x);
    dropin::device_free(v->y);
    dropin::device_free(v->z);
    v->count = 0;
  }
}

// Three 3-vectors per particle (pressure_correction.cu:579-581).
size_type DeviceCorrectionWorkspace::bytes() const noexcept { return pressure_gradient_.count * 9 * sizeof(real); }

DevicePressureCorrection::DevicePressureCorrection(size_type fluid_capacity, SimulationConfig config)
    : config_(std::move(config)), workspace_(fluid_capacity) {}

void DevicePressureCorrection::resize(size_type fluid_capacity) { workspace_.resize(fluid_capacity); }

void DevicePressureCorrection::set_config(SimulationConfig config) { config_ = std::move(config); }

size_type DevicePressureCorrection::bytes() const noexcept { return workspace_.bytes(); }

// DevicePressureCorrection::apply, pressure_correction.cu:598-645: clamp ->
// gradient -> shifting -> update -> anti-penetration -> smoothing, one C ABI
// call after the moment caches are current.
void DevicePressureCorrection::apply(const FluidParticleSoA& fluid, const WallParticleSoA& walls,
                                     const NeighborListView& fluid_neighbors, const NeighborListView& wall_neighbors,
                                     const FluidParticleSoA& temporary_velocity, const real* pressure,
                                     DeviceMomentMatrix& moment_matrices, unsigned long long geometry_generation) {
  if (workspace_.capacity() < fluid.count) workspace_.resize(fluid.count);
  moment_matrices.set_config(config_);
  moment_matrices.resize(fluid.count);
  moment_matrices.prepare_matrices(fluid, walls, fluid_neighbors, wall_neighbors, geometry_generation);
  const MomentMatrixView pressure_moment = moment_matrices.pressure_type_a();
  require_prepared_pressure_moment(fluid, pressure_moment);
  const lsmps_params p = dropin::params_of(config_);
  const lsmps_fluid f = dropin::view_of(fluid);
  const lsmps_walls w = dropin::view_of(walls);
  const lsmps_csr fn = dropin::view_of(fluid_neighbors);
  const lsmps_csr wn = dropin::view_of(wall_neighbors);
  const lsmps_fluid tv = dropin::view_of(temporary_velocity);
  const lsmps_moment pm = dropin::view_of(pressure_moment);
  const lsmps_vector g = vector_of(workspace_.pressure_gradient());
  const lsmps_vector s = vector_of(workspace_.ps_displacement());
  const lsmps_vector sm = vector_of(workspace_.smoothed_velocity());
  dropin::check(lsmps_pressure_correction(dropin::context(), &f, &w, &fn, &wn, &tv, const_cast<real*>(pressure), &p,
                                          &pm, &g, &s, &sm));
}

// clamp_particle_pressure, pressure_correction.cu:647-655 (the reference also
// writes through its const pointer).
void clamp_particle_pressure(const FluidParticleSoA& fluid, const real* pressure) {
  const lsmps_fluid f = dropin::view_of(fluid);
  dropin::check(lsmps_clamp_particle_pressure(dropin::context(), &f, const_cast<real*>(pressure)));
}

// compute_pressure_gradient, pressure_correction.cu:657-682.
void compute_pressure_gradient(const FluidParticleSoA& fluid, const WallParticleSoA& walls,
                               const NeighborListView& fluid_neighbors, const NeighborListView& wall_neighbors,
                               const real* pressure, const SimulationConfig& config,
                               const MomentMatrixView& pressure_moment, CorrectionVectorView pressure_gradient) {
  require_prepared_pressure_moment(fluid, pressure_moment);
  const lsmps_params p = dropin::params_of(config);
  const lsmps_fluid f = dropin::view_of(fluid);
  const lsmps_walls w = dropin::view_of(walls);
  const lsmps_csr fn = dropin::view_of(fluid_neighbors);
  const lsmps_csr wn = dropin::view_of(wall_neighbors);
  const lsmps_moment pm = dropin::view_of(pressure_moment);
  const lsmps_vector g = vector_of(pressure_gradient);
  dropin::check(lsmps_pressure_gradient(dropin::context(), &f, &w, &fn, &wn, pressure, &p, &pm, &g));
}

// compute_particle_shifting_displacement, pressure_correction.cu:684-699.
void compute_particle_shifting_displacement(const FluidParticleSoA& fluid, const WallParticleSoA& walls,
                                            const NeighborListView& fluid_neighbors,
                                            const NeighborListView& wall_neighbors, const SimulationConfig& config,
                                            CorrectionVectorView ps_displacement) {
  const lsmps_params p = dropin::params_of(config);
  const lsmps_fluid f = dropin::view_of(fluid);
  const lsmps_walls w = dropin::view_of(walls);
  const lsmps_csr fn = dropin::view_of(fluid_neighbors);
  const lsmps_csr wn = dropin::view_of(wall_neighbors);
  const lsmps_vector s = vector_of(ps_displacement);
  dropin::check(lsmps_particle_shifting(dropin::context(), &f, &w, &fn, &wn, &p, &s));
}

// update_velocity_and_position, pressure_correction.cu:701-716.
void update_velocity_and_position(const FluidParticleSoA& fluid, const FluidParticleSoA& temporary_velocity,
                                  const SimulationConfig& config, CorrectionVectorView pressure_gradient,
                                  CorrectionVectorView ps_displacement) {
  const lsmps_params p = dropin::params_of(config);
  const lsmps_fluid f = dropin::view_of(fluid);
  const lsmps_fluid tv = dropin::view_of(temporary_velocity);
  const lsmps_vector g = vector_of(pressure_gradient);
  const lsmps_vector s = vector_of(ps_displacement);
  dropin::check(lsmps_update_velocity_position(dropin::context(), &f, &tv, &p, &g, &s));
}

// smooth_particle_velocity, pressure_correction.cu:718-734.
void smooth_particle_velocity(const FluidParticleSoA& fluid, const NeighborListView& fluid_neighbors,
                              const SimulationConfig& config, CorrectionVectorView smoothed_velocity) {
  const lsmps_params p = dropin::params_of(config);
  const lsmps_fluid f = dropin::view_of(fluid);
  const lsmps_csr fn = dropin::view_of(fluid_neighbors);
  const lsmps_vector sm = vector_of(smoothed_velocity);
  dropin::check(lsmps_smooth_particle_velocity(dropin::context(), &f, &fn, &p, &sm));
}

}  // namespace lsmps3d
