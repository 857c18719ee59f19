// ref_harness.cu -- TEST INFRASTRUCTURE, not part of the product.
//
// Drives the reference lsmps3D CUDA path (its own sources, compiled by
// oracle/Makefile into oracle/_ref/) through the reference's public C++ module
// API, stage by stage or as whole benchmark steps, and copies every output
// back to caller-provided host arrays.  Used on the GPU machine to pin the
// oracle and the sm_100a path against the reference's own CUDA results, and as
// the reference timing arm of bench.py.
//
// The step follows src/app/simulation_driver.cu:346-383 with the PPE solve
// replaced by the pressure input (fluid.pressure, clamped in place by the
// correction) and without time-step control and output.
#include <cuda_runtime.h>

#include <cstdio>
#include <memory>
#include <vector>

#include "lsmps3d/core/config.hpp"
#include "lsmps3d/core/cuda_check.cuh"
#include "lsmps3d/core/workspace.cuh"
#include "lsmps3d/correction/pressure_correction.cuh"
#include "lsmps3d/moment_matrix/moment_matrix.cuh"
#include "lsmps3d/neighbor/neighbor_search.cuh"
#include "lsmps3d/ppe/ppe_matrix.cuh"
#include "lsmps3d/provision/explicit_update.cuh"
#include "lsmps3d/surface/surface_detection.cuh"
#include "lsmps_b200.h"

namespace {

using namespace lsmps3d;

struct Harness {
  SimulationConfig config;
  WorkspaceSpec spec;
  std::unique_ptr<SimulationWorkspace> workspace;
  std::unique_ptr<DeviceFluidParticles> temporary_velocity;
  std::unique_ptr<DeviceWallParticles> temporary_wall_velocity;
  std::unique_ptr<DeviceMomentMatrix> moments;
  std::unique_ptr<DeviceProvisionExplicitUpdate> provision;
  std::unique_ptr<DevicePpeMatrixAssembler> ppe;
  std::unique_ptr<DevicePressureCorrection> correction;
  unsigned long long generation = 0;
  cudaEvent_t e0{}, e1{};
};

SimulationConfig config_from(const lsmps_params* p) {
  SimulationConfig c;
  c.particle_spacing = p->particle_spacing;
  c.support_radius = p->support_radius;
  c.near_surface_radius = p->near_surface_radius;
  c.cell_origin = Vec3{p->grid.origin[0], p->grid.origin[1], p->grid.origin[2]};
  c.cell_size = p->grid.cell_size;
  c.cell_dims = Int3{p->grid.dims[0], p->grid.dims[1], p->grid.dims[2]};
  c.time_step = p->time_step;
  c.density = p->density;
  c.kinematic_viscosity = p->kinematic_viscosity;
  c.gravity = Vec3{p->gravity[0], p->gravity[1], p->gravity[2]};
  c.splash_neighbor_threshold = p->splash_neighbor_threshold;
  c.number_density_ratio_threshold = p->number_density_ratio_threshold;
  c.air_open_ratio_threshold = p->air_open_ratio_threshold;
  c.air_anisotropy_threshold = p->air_anisotropy_threshold;
  c.include_wall_neighbors = p->include_wall_neighbors != 0;
  c.wall_normal_independence_threshold = p->wall_normal_independence_threshold;
  c.virtual_light_cone_cosine = p->virtual_light_cone_cosine;
  c.lsmps_regularization = p->lsmps_regularization;
  c.lsmps_wall_weight_scale = p->lsmps_wall_weight_scale;
  c.ps_displacement_scale = p->ps_displacement_scale;
  c.ps_min_distance_ratio = p->ps_min_distance_ratio;
  c.ps_max_displacement_ratio = p->ps_max_displacement_ratio;
  c.wall_clearance_ratio = p->wall_clearance_ratio;
  c.velocity_smoothing_strength = p->velocity_smoothing_strength;
  return c;
}

template <typename T>
void up(T* dst, const T* src, size_t n) {
  if (n) LSMPS3D_CUDA_CHECK(cudaMemcpy(dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
}

template <typename T>
void down(T* dst, const T* src, size_t n) {
  if (n && dst) LSMPS3D_CUDA_CHECK(cudaMemcpy(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost));
}

void provision_stage(Harness& h) {
  auto v = h.workspace->view();
  h.provision->compute_temporary_velocity(v.fluid, v.walls, v.fluid_neighbors, v.wall_neighbors, *h.moments,
                                          h.generation, h.temporary_velocity->view(),
                                          h.temporary_wall_velocity->view());
}

void ppe_stage(Harness& h) {
  auto v = h.workspace->view();
  h.ppe->assemble(v.fluid, v.walls, v.fluid_neighbors, v.wall_neighbors, h.temporary_velocity->view(),
                  h.temporary_wall_velocity->view(), *h.moments, h.generation);
}

void correction_stage(Harness& h) {
  auto v = h.workspace->view();
  h.correction->apply(v.fluid, v.walls, v.fluid_neighbors, v.wall_neighbors, h.temporary_velocity->view(),
                      v.fluid.pressure, *h.moments, h.generation);
}

// rebuild_geometry, simulation_driver.cu:252-264
void rebuild_stage(Harness& h) {
  auto v = h.workspace->view();
  build_neighbor_lists(v.fluid, v.walls, h.config, v.fluid_cells, v.wall_cells, v.fluid_neighbors, v.wall_neighbors);
  ++h.generation;
  classify_surface_particles(v.fluid, v.walls, v.fluid_neighbors, v.wall_neighbors, h.config);
}

}  // namespace

extern "C" {

void* ref_create(const lsmps_params* p, size_t n_fluid, size_t n_wall, size_t max_fluid_neighbors,
                 size_t max_wall_neighbors) {
  auto* h = new Harness();
  h->config = config_from(p);
  h->spec = WorkspaceSpec{n_fluid, n_wall, max_fluid_neighbors, max_wall_neighbors, h->config.cell_capacity()};
  h->workspace = std::make_unique<SimulationWorkspace>(h->spec);
  h->temporary_velocity = std::make_unique<DeviceFluidParticles>(n_fluid);
  h->temporary_wall_velocity = std::make_unique<DeviceWallParticles>(n_wall);
  h->moments = std::make_unique<DeviceMomentMatrix>(n_fluid, h->config);
  h->provision = std::make_unique<DeviceProvisionExplicitUpdate>(n_fluid, h->config);
  h->ppe = std::make_unique<DevicePpeMatrixAssembler>(n_fluid, n_fluid + h->spec.fluid_neighbor_capacity(),
                                                      h->config);
  h->correction = std::make_unique<DevicePressureCorrection>(n_fluid, h->config);
  cudaEventCreate(&h->e0);
  cudaEventCreate(&h->e1);
  return h;
}

void ref_destroy(void* handle) {
  auto* h = static_cast<Harness*>(handle);
  if (!h) return;
  cudaEventDestroy(h->e0);
  cudaEventDestroy(h->e1);
  delete h;
}

size_t ref_workspace_bytes(void* handle) {
  auto* h = static_cast<Harness*>(handle);
  return h->workspace->bytes() + h->moments->bytes() + h->ppe->bytes() + h->correction->bytes() +
         h->provision->bytes();
}

int ref_upload(void* handle, const lsmps_fluid* f, const lsmps_walls* w) {
  auto* h = static_cast<Harness*>(handle);
  auto v = h->workspace->view();
  const size_t n = v.fluid.count, m = v.walls.count;
  up(v.fluid.x, f->x, n);
  up(v.fluid.y, f->y, n);
  up(v.fluid.z, f->z, n);
  up(v.fluid.vx, f->vx, n);
  up(v.fluid.vy, f->vy, n);
  up(v.fluid.vz, f->vz, n);
  up(v.fluid.pressure, f->pressure, n);
  up(v.fluid.surface_type, f->surface_type, n);
  up(v.walls.x, w->x, m);
  up(v.walls.y, w->y, m);
  up(v.walls.z, w->z, m);
  up(v.walls.vx, w->vx, m);
  up(v.walls.vy, w->vy, m);
  up(v.walls.vz, w->vz, m);
  up(v.walls.normal_x, w->normal_x, m);
  up(v.walls.normal_y, w->normal_y, m);
  up(v.walls.normal_z, w->normal_z, m);
  return 0;
}

int ref_rebuild(void* handle) {
  rebuild_stage(*static_cast<Harness*>(handle));
  return 0;
}

int ref_provision(void* handle) {
  provision_stage(*static_cast<Harness*>(handle));
  return 0;
}

int ref_assemble_ppe(void* handle) {
  ppe_stage(*static_cast<Harness*>(handle));
  return 0;
}

int ref_correction(void* handle) {
  correction_stage(*static_cast<Harness*>(handle));
  return 0;
}

// `steps` benchmark steps; per-step device times (ms, CUDA events around the
// whole step on the legacy default stream the reference uses) into ms[].
int ref_steps(void* handle, int steps, float* ms) {
  auto* h = static_cast<Harness*>(handle);
  for (int s = 0; s < steps; ++s) {
    cudaEventRecord(h->e0, 0);
    provision_stage(*h);
    ppe_stage(*h);
    correction_stage(*h);
    LSMPS3D_CUDA_CHECK(cudaDeviceSynchronize());
    rebuild_stage(*h);
    cudaEventRecord(h->e1, 0);
    cudaEventSynchronize(h->e1);
    if (ms) cudaEventElapsedTime(&ms[s], h->e0, h->e1);
  }
  return 0;
}

int ref_download_fluid(void* handle, const lsmps_fluid* out) {
  auto v = static_cast<Harness*>(handle)->workspace->view();
  const size_t n = v.fluid.count;
  down(out->x, v.fluid.x, n);
  down(out->y, v.fluid.y, n);
  down(out->z, v.fluid.z, n);
  down(out->vx, v.fluid.vx, n);
  down(out->vy, v.fluid.vy, n);
  down(out->vz, v.fluid.vz, n);
  down(out->pressure, v.fluid.pressure, n);
  down(out->surface_type, v.fluid.surface_type, n);
  return 0;
}

// which: 0 fluid, 1 wall.  Host arrays sized like the caller's view.
int ref_download_cells(void* handle, int which, const lsmps_cells* out) {
  auto v = static_cast<Harness*>(handle)->workspace->view();
  const CellListView c = which == 0 ? v.fluid_cells : v.wall_cells;
  const size_t n = which == 0 ? v.fluid.count : v.walls.count;
  down(out->cell_ids, c.cell_ids, n);
  down(out->sorted_indices, c.sorted_indices, n);
  down(out->cell_begin, c.cell_begin, c.cell_count);
  down(out->cell_end, c.cell_end, c.cell_count);
  return 0;
}

// Returns the number of CSR entries (offsets[N]); indices copied up to
// min(entries, out->neighbor_count).
long long ref_download_csr(void* handle, int which, const lsmps_csr* out) {
  auto v = static_cast<Harness*>(handle)->workspace->view();
  const NeighborListView c = which == 0 ? v.fluid_neighbors : v.wall_neighbors;
  const size_t n = v.fluid.count;
  std::vector<index_t> off(n + 1);
  down(off.data(), c.offsets, n + 1);
  if (out->offsets) std::copy(off.begin(), off.end(), out->offsets);
  const size_t total = static_cast<size_t>(off[n]);
  down(out->indices, c.indices, total < out->neighbor_count ? total : out->neighbor_count);
  return static_cast<long long>(total);
}

// kind: 0 velocity Dirichlet-A, 1 pressure Neumann-A, 2 pressure Neumann-B, 3 fluid-only A.
int ref_download_moment(void* handle, int kind, const lsmps_moment* out) {
  auto* h = static_cast<Harness*>(handle);
  const MomentMatrixView m = kind == 0   ? h->moments->velocity_type_a()
                             : kind == 1 ? h->moments->pressure_type_a()
                             : kind == 2 ? h->moments->pressure_type_b()
                                         : h->moments->fluid_only_type_a();
  const size_t n = h->workspace->view().fluid.count;
  const size_t nn = static_cast<size_t>(m.matrix_size) * m.matrix_size;
  down(out->inverse_matrices, m.inverse_matrices, n * nn);
  down(out->moment_trace, m.moment_trace, n);
  down(out->regularization_added, m.regularization_added, n);
  down(out->info, m.info, n);
  down(out->inversion_count, m.inversion_count, 1);
  return 0;
}

int ref_download_temporary(void* handle, const lsmps_fluid* fluid, const lsmps_walls* walls) {
  auto* h = static_cast<Harness*>(handle);
  const auto t = h->temporary_velocity->view();
  const auto tw = h->temporary_wall_velocity->view();
  down(fluid->vx, t.vx, t.count);
  down(fluid->vy, t.vy, t.count);
  down(fluid->vz, t.vz, t.count);
  down(walls->vx, tw.vx, tw.count);
  down(walls->vy, tw.vy, tw.count);
  down(walls->vz, tw.vz, tw.count);
  return 0;
}

// Returns the assembler's active nnz; values/cols copied for the written
// N + K_f slots (the rest of the active range is never written, ppe_matrix.cu:494-499).
long long ref_download_ppe(void* handle, const lsmps_ppe* out, size_t written) {
  auto* h = static_cast<Harness*>(handle);
  const PpeWorkspaceView w = h->ppe->workspace();
  const size_t n = h->workspace->view().fluid.count;
  down(out->matrix.row_offsets, w.matrix.row_offsets, n + 1);
  down(out->matrix.col_indices, w.matrix.col_indices, written);
  down(out->matrix.values, w.matrix.values, written);
  down(out->rhs, w.rhs, n);
  down(out->divergence, w.divergence, n);
  down(out->pressure_laplacian, w.pressure_laplacian, n);
  return static_cast<long long>(w.matrix.nnz);
}

int ref_download_correction(void* handle, const lsmps_vector* gradient, const lsmps_vector* shift) {
  auto* h = static_cast<Harness*>(handle);
  const auto g = h->correction->pressure_gradient();
  const auto s = h->correction->ps_displacement();
  const size_t n = h->workspace->view().fluid.count;
  down(gradient->x, g.x, n);
  down(gradient->y, g.y, n);
  down(gradient->z, g.z, n);
  down(shift->x, s.x, n);
  down(shift->y, s.y, n);
  down(shift->z, s.z, n);
  return 0;
}

// compute_virtual_light_diagnostics on the current geometry (after
// ref_rebuild); the open-direction counts and fractions into host arrays.
int ref_virtual_light(void* handle, int32_t* open_count, double* open_fraction) {
  auto* h = static_cast<Harness*>(handle);
  auto v = h->workspace->view();
  const size_t n = v.fluid.count;
  int* d_count = nullptr;
  real* d_fraction = nullptr;
  LSMPS3D_CUDA_CHECK(cudaMalloc(&d_count, (n ? n : 1) * sizeof(int)));
  LSMPS3D_CUDA_CHECK(cudaMalloc(&d_fraction, (n ? n : 1) * sizeof(real)));
  compute_virtual_light_diagnostics(v.fluid, v.walls, v.fluid_neighbors, v.wall_neighbors, h->config,
                                    VirtualLightDiagnosticsView{d_count, d_fraction});
  down(open_count, d_count, n);
  down(open_fraction, d_fraction, n);
  cudaFree(d_count);
  cudaFree(d_fraction);
  return 0;
}

// `steps` timed calls of compute_virtual_light_diagnostics on the current
// geometry; per-call device times (ms, CUDA events on the legacy default
// stream) into ms[].
int ref_virtual_light_steps(void* handle, int steps, float* ms) {
  auto* h = static_cast<Harness*>(handle);
  auto v = h->workspace->view();
  const size_t n = v.fluid.count;
  int* d_count = nullptr;
  real* d_fraction = nullptr;
  LSMPS3D_CUDA_CHECK(cudaMalloc(&d_count, (n ? n : 1) * sizeof(int)));
  LSMPS3D_CUDA_CHECK(cudaMalloc(&d_fraction, (n ? n : 1) * sizeof(real)));
  for (int s = 0; s < steps; ++s) {
    cudaEventRecord(h->e0, 0);
    compute_virtual_light_diagnostics(v.fluid, v.walls, v.fluid_neighbors, v.wall_neighbors, h->config,
                                      VirtualLightDiagnosticsView{d_count, d_fraction});
    cudaEventRecord(h->e1, 0);
    cudaEventSynchronize(h->e1);
    if (ms) cudaEventElapsedTime(&ms[s], h->e0, h->e1);
  }
  cudaFree(d_count);
  cudaFree(d_fraction);
  return 0;
}

}  // extern "C"
