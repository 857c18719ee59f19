// dropin.cpp - context, error reporting and view conversions of the drop-in.
#include "dropin.hpp"

#include <cstdlib>
#include <cstring>
#include <iostream>
#include <mutex>
#include <stdexcept>

namespace lsmps3d::dropin {
namespace {

constexpr int kMaxDevices = 64;

std::mutex& context_lock() {
  static std::mutex m;
  return m;
}

lsmps_ctx*& context_slot(int device) {
  // Contexts live for the whole process: their scratch is released with the
  // CUDA context at exit, so no destructor runs after the runtime shut down.
  static lsmps_ctx* contexts[kMaxDevices] = {};
  return contexts[device];
}

bool throw_mode() {
  static const bool on = [] {
    const char* v = std::getenv("LSMPS_DROPIN_THROW");
    return v != nullptr && std::strcmp(v, "1") == 0;
  }();
  return on;
}

}  // namespace

lsmps_ctx* context() {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) {
    cudaGetLastError();
    fail("CUDA device query failed");
  }
  std::lock_guard<std::mutex> guard(context_lock());
  lsmps_ctx*& ctx = context_slot(device);
  if (ctx == nullptr) {
    lsmps_ctx* created = nullptr;
    if (lsmps_ctx_create(device, &created) != LSMPS_OK) fail("CUDA context set-up failed");
    lsmps_ctx_set_stream(created, nullptr);  // the legacy default stream, as the reference
    lsmps_ctx_set_synchronous(created, 1);
    ctx = created;
  }
  return ctx;
}

void fail(const std::string& message) {
  if (throw_mode()) throw std::runtime_error(message);
  std::cerr << message << std::endl;
  std::exit(EXIT_FAILURE);
}

void check(lsmps_status status) {
  if (status == LSMPS_OK) return;
  const char* message = lsmps_ctx_last_error(context());
  fail(message != nullptr && message[0] != '\0' ? std::string(message)
                                                 : std::string(lsmps_status_string(status)));
}

lsmps_params params_of(const SimulationConfig& c) {
  lsmps_params p;
  lsmps_params_default(&p);
  p.particle_spacing = c.particle_spacing;
  p.support_radius = c.support_radius;
  p.near_surface_radius = c.near_surface_radius;
  p.grid = grid_of(c.cell_grid());
  p.time_step = c.time_step;
  p.density = c.density;
  p.kinematic_viscosity = c.kinematic_viscosity;
  p.gravity[0] = c.gravity.x;
  p.gravity[1] = c.gravity.y;
  p.gravity[2] = c.gravity.z;
  p.splash_neighbor_threshold = c.splash_neighbor_threshold;
  p.include_wall_neighbors = c.include_wall_neighbors ? 1 : 0;
  p.number_density_ratio_threshold = c.number_density_ratio_threshold;
  p.air_open_ratio_threshold = c.air_open_ratio_threshold;
  p.air_anisotropy_threshold = c.air_anisotropy_threshold;
  p.wall_normal_independence_threshold = c.wall_normal_independence_threshold;
  p.virtual_light_cone_cosine = c.virtual_light_cone_cosine;
  p.lsmps_regularization = c.lsmps_regularization;
  p.lsmps_wall_weight_scale = c.lsmps_wall_weight_scale;
  p.ps_displacement_scale = c.ps_displacement_scale;
  p.ps_min_distance_ratio = c.ps_min_distance_ratio;
  p.ps_max_displacement_ratio = c.ps_max_displacement_ratio;
  p.wall_clearance_ratio = c.wall_clearance_ratio;
  p.velocity_smoothing_strength = c.velocity_smoothing_strength;
  return p;
}

lsmps_grid grid_of(const CellGrid& g) {
  lsmps_grid out;
  out.origin[0] = g.origin.x;
  out.origin[1] = g.origin.y;
  out.origin[2] = g.origin.z;
  out.cell_size = g.cell_size;
  out.dims[0] = g.dims.x;
  out.dims[1] = g.dims.y;
  out.dims[2] = g.dims.z;
  return out;
}

lsmps_fluid view_of(const FluidParticleSoA& f) {
  return lsmps_fluid{f.count, f.x, f.y, f.z, f.vx, f.vy, f.vz, f.pressure, f.surface_type};
}

lsmps_walls view_of(const WallParticleSoA& w) {
  return lsmps_walls{w.count, w.x, w.y, w.z, w.vx, w.vy, w.vz, w.normal_x, w.normal_y, w.normal_z};
}

lsmps_csr view_of(const NeighborListView& n) {
  return lsmps_csr{n.particle_count, n.neighbor_count, n.offsets, n.indices};
}

lsmps_cells view_of(const CellListView& c) {
  return lsmps_cells{c.particle_count, c.cell_count, c.cell_ids, c.sorted_indices, c.cell_begin, c.cell_end};
}

lsmps_moment view_of(const MomentMatrixView& m) {
  lsmps_moment out;
  out.particle_count = m.particle_count;
  out.matrix_size = m.matrix_size;
  out.kind = static_cast<int32_t>(m.kind);
  out.support_radius = m.support_radius;
  out.wall_weight_scale = m.wall_weight_scale;
  // The C ABI names its outputs non-const; consumers only read them.
  out.inverse_matrices = const_cast<double*>(m.inverse_matrices);
  out.moment_trace = const_cast<double*>(m.moment_trace);
  out.regularization_added = const_cast<double*>(m.regularization_added);
  out.info = const_cast<int32_t*>(m.info);
  out.inversion_count = const_cast<int32_t*>(m.inversion_count);
  return out;
}

}  // namespace lsmps3d::dropin
