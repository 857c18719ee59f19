// explicit_update.cpp - the reference's provision module
// (include/lsmps3d/provision/explicit_update.cuh:11-91, replacing
// src/provision/explicit_update.cu) on the C ABI: the LSMPS velocity
// Laplacian and u* = u + dt (nu lap u + g) for fluid (Splash rows without the
// viscous term) and wall particles.
#include "lsmps3d/provision/explicit_update.cuh"

#include <utility>

#include "dropin.hpp"

namespace lsmps3d {
namespace {

void swap_views(ProvisionVelocityView& a, ProvisionVelocityView& b) noexcept {
  std::swap(a.count, b.count);
  std::swap(a.vx, b.vx);
  std::swap(a.vy, b.vy);
  std::swap(a.vz, b.vz);
}

void require_prepared_velocity_moment(const FluidParticleSoA& fluid, const MomentMatrixView& m) {
  // validate_velocity_moment_matrix, explicit_update.cu:105-119
  if (!m.is_ready || m.kind != MomentMatrixKind::VelocityWallDirichletTypeA ||
      m.basis_kind != MomentBasisKind::TypeA || m.matrix_size != kMomentTypeABasis3DSize ||
      m.particle_count < fluid.count)
    dropin::fail("Provision requires a prepared velocity Type-A moment matrix");
  if (fluid.count > 0 && m.inverse_matrices == nullptr)
    dropin::fail("Provision velocity moment matrix inverse buffer is missing");
}

lsmps_vector vector_of(const ProvisionVelocityView& v) { return lsmps_vector{v.count, v.vx, v.vy, v.vz}; }

}  // namespace

DeviceProvisionWorkspace::DeviceProvisionWorkspace(size_type fluid_capacity) { resize(fluid_capacity); }

DeviceProvisionWorkspace::DeviceProvisionWorkspace(size_type fluid_capacity, size_type wall_capacity) {
  resize(fluid_capacity, wall_capacity);
}

DeviceProvisionWorkspace::~DeviceProvisionWorkspace() { release(); }

DeviceProvisionWorkspace::DeviceProvisionWorkspace(DeviceProvisionWorkspace&& other) noexcept {
  swap_views(fluid_view_, other.fluid_view_);
  swap_views(wall_view_, other.wall_view_);
}

DeviceProvisionWorkspace& DeviceProvisionWorkspace::operator=(DeviceProvisionWorkspace&& other) noexcept {
  if (this != &other) {
    release();
    swap_views(fluid_view_, other.fluid_view_);
    swap_views(wall_view_, other.wall_view_);
  }
  return *this;
}

void DeviceProvisionWorkspace::resize(size_type fluid_capacity) { resize(fluid_capacity, wall_view_.count); }

void DeviceProvisionWorkspace::resize(size_type fluid_capacity, size_type wall_capacity) {
  if (fluid_capacity == fluid_view_.count && wall_capacity == wall_view_.count) return;
  release();
  fluid_view_.count = fluid_capacity;
  dropin::device_alloc(fluid_view_.vx, fluid_capacity);
  dropin::device_alloc(fluid_view_.vy, fluid_capacity);
  dropin::device_alloc(fluid_view_.vz, fluid_capacity);
  wall_view_.count = wall_capacity;
  dropin::device_alloc(wall_view_.vx, wall_capacity);
  dropin::device_alloc(wall_view_.vy, wall_capacity);
  dropin::device_alloc(wall_view_.vz, wall_capacity);
}

void DeviceProvisionWorkspace::release() noexcept {
  dropin::device_free(fluid_view_.vx);
  dropin::device_free(fluid_view_.vy);
  dropin::device_free(fluid_view_.vz);
  fluid_view_.count = 0;
  dropin::device_free(wall_view_.vx);
  dropin::device_free(wall_view_.vy);
  dropin::device_free(wall_view_.vz);
  wall_view_.count = 0;
}

size_type DeviceProvisionWorkspace::bytes() const noexcept {
  return (fluid_view_.count + wall_view_.count) * 3 * sizeof(real);
}

DeviceProvisionExplicitUpdate::DeviceProvisionExplicitUpdate(size_type fluid_capacity, SimulationConfig config)
    : config_(std::move(config)), workspace_(fluid_capacity) {}

void DeviceProvisionExplicitUpdate::resize(size_type fluid_capacity) {
  workspace_.resize(fluid_capacity, workspace_.wall_capacity());
}

void DeviceProvisionExplicitUpdate::set_config(SimulationConfig config) { config_ = std::move(config); }

size_type DeviceProvisionExplicitUpdate::bytes() const noexcept { return workspace_.bytes(); }

// compute_temporary_velocity, explicit_update.cu:366-399.
void DeviceProvisionExplicitUpdate::compute_temporary_velocity(
    const FluidParticleSoA& fluid, const WallParticleSoA& walls, const NeighborListView& fluid_neighbors,
    const NeighborListView& wall_neighbors, DeviceMomentMatrix& moment_matrices,
    unsigned long long geometry_generation, FluidParticleSoA temporary_velocity,
    WallParticleSoA temporary_wall_velocity) {
  if (workspace_.capacity() < fluid.count || workspace_.wall_capacity() < walls.count)
    workspace_.resize(fluid.count, walls.count);
  moment_matrices.set_config(config_);
  moment_matrices.resize(fluid.count);
  moment_matrices.prepare_matrices(fluid, walls, fluid_neighbors, wall_neighbors, geometry_generation);
  const MomentMatrixView velocity_moment = moment_matrices.velocity_type_a();
  require_prepared_velocity_moment(fluid, velocity_moment);
  const lsmps_fluid f = dropin::view_of(fluid);
  const lsmps_walls w = dropin::view_of(walls);
  const lsmps_csr fn = dropin::view_of(fluid_neighbors);
  const lsmps_csr wn = dropin::view_of(wall_neighbors);
  const lsmps_moment vm = dropin::view_of(velocity_moment);
  const lsmps_vector lap = vector_of(workspace_.view());
  lsmps_ctx* ctx = dropin::context();
  if (fluid.count > 0) dropin::check(lsmps_velocity_laplacian(ctx, &f, &w, &fn, &wn, &vm, &lap));
  compute_provision_temporary_velocity(fluid, config_, workspace_.view(), temporary_velocity);
  compute_provision_temporary_wall_velocity(walls, config_, temporary_wall_velocity);
}

// compute_provision_temporary_velocity, explicit_update.cu:401-415.
void compute_provision_temporary_velocity(const FluidParticleSoA& fluid, const SimulationConfig& config,
                                          const ProvisionVelocityView& velocity_laplacian,
                                          FluidParticleSoA temporary_velocity) {
  const lsmps_params p = dropin::params_of(config);
  const lsmps_fluid f = dropin::view_of(fluid);
  const lsmps_vector lap = vector_of(velocity_laplacian);
  const lsmps_fluid t = dropin::view_of(temporary_velocity);
  dropin::check(lsmps_temporary_velocity(dropin::context(), &f, &p, &lap, &t));
}

// compute_provision_temporary_wall_velocity, explicit_update.cu:417-430.
void compute_provision_temporary_wall_velocity(const WallParticleSoA& walls, const SimulationConfig& config,
                                               WallParticleSoA temporary_wall_velocity) {
  const lsmps_params p = dropin::params_of(config);
  const lsmps_walls w = dropin::view_of(walls);
  const lsmps_walls t = dropin::view_of(temporary_wall_velocity);
  dropin::check(lsmps_temporary_wall_velocity(dropin::context(), &w, &p, &t));
}

}  // namespace lsmps3d
