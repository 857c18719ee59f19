// moment_matrix.cpp - the reference's DeviceMomentMatrix
// (include/lsmps3d/moment_matrix/moment_matrix.cuh:36-68, replacing
// src/moment_matrix/moment_matrix.cu) on the C ABI.
//
// The four kinds the reference keeps (velocity Dirichlet Type-A, pressure
// Neumann Type-A and Type-B, fluid-only Type-A) are cached per kind under the
// reference's request key (kind, support radius, regularisation, wall weight
// scale, geometry generation; moment_matrix.cu:117-123).  prepare_matrices
// rebuilds only the stale kinds and hands them to ONE lsmps_prepare_moments
// call, which assembles kinds that share the Type-A fluid sum in one pass
// over the rows and inverts each matrix in registers (no cuSOLVER, no
// per-column solves, no factor copies or pointer arrays).  Each cache holds
// only what the public view exposes: the column-major inverses, trace,
// regularisation, Cholesky info and the build counter.
#include "lsmps3d/moment_matrix/moment_matrix.cuh"

#include <utility>

#include "dropin.hpp"

namespace lsmps3d {
namespace {

struct Request {
  MomentMatrixKind kind{MomentMatrixKind::VelocityWallDirichletTypeA};
  real support_radius{};
  real regularization{};
  real wall_weight_scale{};
  unsigned long long geometry_generation{};

  bool operator==(const Request& o) const {
    return kind == o.kind && support_radius == o.support_radius && regularization == o.regularization &&
           wall_weight_scale == o.wall_weight_scale && geometry_generation == o.geometry_generation;
  }
};

MomentBasisKind basis_of(MomentMatrixKind kind) {
  return kind == MomentMatrixKind::PressureWallNeumannTypeB ? MomentBasisKind::TypeB : MomentBasisKind::TypeA;
}

struct Cache {
  MomentMatrixKind kind{};
  size_type particle_count{};
  int matrix_size{kMomentTypeABasis3DSize};
  Request request{};
  bool has_request{false};
  bool is_ready{false};
  real* inverse_matrices{};
  real* moment_trace{};
  real* regularization_added{};
  int* info{};
  int* inversion_count{};

  explicit Cache(MomentMatrixKind k) : kind(k), matrix_size(moment_basis_size(basis_of(k))) {}
  ~Cache() { release(); }
  Cache(const Cache&) = delete;
  Cache& operator=(const Cache&) = delete;

  // MatrixCache::resize, moment_matrix.cu:353-374: reallocates only when the
  // particle count changes, and a reallocated cache is not ready.
  void resize(size_type n) {
    if (n == particle_count && inversion_count != nullptr) return;
    release();
    particle_count = n;
    const size_type nn = static_cast<size_type>(matrix_size) * matrix_size;
    dropin::device_alloc(inverse_matrices, n * nn);
    dropin::device_alloc(moment_trace, n);
    dropin::device_alloc(regularization_added, n);
    dropin::device_alloc(info, n);
    dropin::device_alloc(inversion_count, 1);
    if (cudaMemset(inversion_count, 0, sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      dropin::fail("CUDA memset failed");
    }
  }

  void release() noexcept {
    dropin::device_free(inverse_matrices);
    dropin::device_free(moment_trace);
    dropin::device_free(regularization_added);
    dropin::device_free(info);
    dropin::device_free(inversion_count);
    particle_count = 0;
    has_request = false;
    is_ready = false;
  }

  size_type bytes() const noexcept {
    const size_type nn = static_cast<size_type>(matrix_size) * matrix_size;
    return particle_count * (nn * sizeof(real) + 2 * sizeof(real) + sizeof(int)) +
           (inversion_count ? sizeof(int) : 0);
  }

  // make_public_view, moment_matrix.cu:478-492.
  MomentMatrixView view() const {
    MomentMatrixView v;
    v.particle_count = particle_count;
    v.matrix_size = matrix_size;
    v.basis_kind = basis_of(kind);
    v.kind = kind;
    v.support_radius = has_request ? request.support_radius : real{};
    v.wall_weight_scale = has_request ? request.wall_weight_scale : real{};
    v.geometry_generation = has_request ? request.geometry_generation : 0ull;
    v.is_ready = is_ready;
    v.inverse_matrices = inverse_matrices;
    v.moment_trace = moment_trace;
    v.regularization_added = regularization_added;
    v.info = info;
    v.inversion_count = inversion_count;
    return v;
  }
};

}  // namespace

struct DeviceMomentMatrix::Impl {
  explicit Impl(SimulationConfig c) : config(std::move(c)) {}

  SimulationConfig config{};
  unsigned long long geometry_generation{};
  bool has_prepared_generation{false};
  Cache caches[4] = {Cache(MomentMatrixKind::VelocityWallDirichletTypeA),
                     Cache(MomentMatrixKind::PressureWallNeumannTypeA),
                     Cache(MomentMatrixKind::PressureWallNeumannTypeB), Cache(MomentMatrixKind::FluidOnlyTypeA)};

  const Cache& cache(MomentMatrixKind kind) const {
    require_prepared();
    return caches[static_cast<int>(kind)];
  }

  void require_prepared() const {
    if (!has_prepared_generation)
      dropin::fail("Moment operators must prepare matrices before computing operators");
  }
};

DeviceMomentMatrix::DeviceMomentMatrix() : impl_(std::make_unique<Impl>(SimulationConfig{})) {}

DeviceMomentMatrix::DeviceMomentMatrix(size_type fluid_capacity, SimulationConfig config)
    : impl_(std::make_unique<Impl>(std::move(config))) {
  resize(fluid_capacity);
}

DeviceMomentMatrix::~DeviceMomentMatrix() = default;
DeviceMomentMatrix::DeviceMomentMatrix(DeviceMomentMatrix&& other) noexcept = default;
DeviceMomentMatrix& DeviceMomentMatrix::operator=(DeviceMomentMatrix&& other) noexcept = default;

void DeviceMomentMatrix::resize(size_type fluid_capacity) {
  for (Cache& c : impl_->caches) c.resize(fluid_capacity);
  impl_->has_prepared_generation = false;
}

void DeviceMomentMatrix::release() noexcept {
  for (Cache& c : impl_->caches) c.release();
  impl_->has_prepared_generation = false;
}

void DeviceMomentMatrix::set_config(SimulationConfig config) {
  impl_->config = std::move(config);
  impl_->has_prepared_generation = false;
}

const SimulationConfig& DeviceMomentMatrix::config() const noexcept { return impl_->config; }

size_type DeviceMomentMatrix::bytes() const noexcept {
  size_type total = 0;
  for (const Cache& c : impl_->caches) total += c.bytes();
  return total;
}

// prepare_matrices, moment_matrix.cu:615-654 (with ensure_matrix_internal,
// :398-476, per kind): a kind whose request matches its ready cache is kept.
void DeviceMomentMatrix::prepare_matrices(const FluidParticleSoA& fluid, const WallParticleSoA& walls,
                                          const NeighborListView& fluid_neighbors,
                                          const NeighborListView& wall_neighbors,
                                          unsigned long long geometry_generation) {
  Impl& im = *impl_;
  im.geometry_generation = geometry_generation;
  const SimulationConfig& c = im.config;
  if (c.support_radius <= real{0}) dropin::fail("Moment support radius must be positive");
  if (c.lsmps_regularization < real{0}) dropin::fail("Moment regularization must be non-negative");
  if (c.lsmps_wall_weight_scale < real{0}) dropin::fail("Moment wall weight scale must be non-negative");
  lsmps_moment stale[4];
  Cache* stale_caches[4];
  int count = 0;
  for (Cache& cache : im.caches) {
    if (cache.particle_count < fluid.count) dropin::fail("Invalid Moment matrix cache");
    if (fluid.count > fluid_neighbors.particle_count || fluid.count > wall_neighbors.particle_count)
      dropin::fail("Moment matrix neighbor lists are smaller than fluid particle count");
    const Request request{cache.kind, c.support_radius, c.lsmps_regularization, c.lsmps_wall_weight_scale,
                          geometry_generation};
    if (cache.has_request && cache.request == request && cache.is_ready) continue;
    cache.request = request;
    cache.has_request = true;
    cache.is_ready = false;
    if (fluid.count == 0) {
      cache.is_ready = true;
      continue;
    }
    MomentMatrixView v = cache.view();
    stale[count] = dropin::view_of(v);
    stale_caches[count] = &cache;
    ++count;
  }
  if (count > 0) {
    const lsmps_params p = dropin::params_of(c);
    const lsmps_fluid f = dropin::view_of(fluid);
    const lsmps_walls w = dropin::view_of(walls);
    const lsmps_csr fn = dropin::view_of(fluid_neighbors);
    const lsmps_csr wn = dropin::view_of(wall_neighbors);
    const lsmps_status st = lsmps_prepare_moments(dropin::context(), &f, &w, &fn, &wn, &p, stale, count);
    // A matrix that is not SPD is reported per particle through info, as
    // cuSOLVER's potrfBatched does in the reference; the build itself succeeded.
    if (st != LSMPS_NON_SPD) dropin::check(st);
    for (int k = 0; k < count; ++k) stale_caches[k]->is_ready = true;
  }
  im.has_prepared_generation = true;
}

MomentMatrixView DeviceMomentMatrix::velocity_type_a() const {
  return impl_->cache(MomentMatrixKind::VelocityWallDirichletTypeA).view();
}

MomentMatrixView DeviceMomentMatrix::pressure_type_a() const {
  return impl_->cache(MomentMatrixKind::PressureWallNeumannTypeA).view();
}

MomentMatrixView DeviceMomentMatrix::pressure_type_b() const {
  return impl_->cache(MomentMatrixKind::PressureWallNeumannTypeB).view();
}

MomentMatrixView DeviceMomentMatrix::fluid_only_type_a() const {
  return impl_->cache(MomentMatrixKind::FluidOnlyTypeA).view();
}

}  // namespace lsmps3d
