// ppe_matrix.cpp - the reference's PPE module
// (include/lsmps3d/ppe/ppe_matrix.cuh:15-129, replacing src/ppe/ppe_matrix.cu)
// on the C ABI: the PPE workspace owner, the assembler, the free assembly
// function, and the AmgxPpeSolver front end.
#include "lsmps3d/ppe/ppe_matrix.cuh"

#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <utility>

#include "dropin.hpp"

namespace lsmps3d {
namespace {

void swap_ppe_views(PpeWorkspaceView& a, PpeWorkspaceView& b) noexcept {
  std::swap(a.matrix, b.matrix);
  std::swap(a.rhs, b.rhs);
  std::swap(a.pressure, b.pressure);
  std::swap(a.divergence, b.divergence);
  std::swap(a.pressure_laplacian, b.pressure_laplacian);
}

// validate_ppe_moment_matrix, ppe_matrix.cu:108-122
void require_prepared_moment(const FluidParticleSoA& fluid, const MomentMatrixView& m, MomentMatrixKind kind,
                             const char* label) {
  if (!m.is_ready || m.kind != kind || m.basis_kind != MomentBasisKind::TypeA ||
      m.matrix_size != kMomentTypeABasis3DSize || m.particle_count < fluid.count)
    dropin::fail(std::string("PPE requires a prepared ") + label + " Type-A moment matrix");
  if (fluid.count > 0 && m.inverse_matrices == nullptr)
    dropin::fail(std::string("PPE moment matrix inverse buffer is missing for ") + label);
}

}  // namespace

DevicePpeWorkspace::DevicePpeWorkspace(size_type fluid_capacity, size_type matrix_nnz_capacity) {
  resize(fluid_capacity, matrix_nnz_capacity);
}

DevicePpeWorkspace::~DevicePpeWorkspace() { release(); }

DevicePpeWorkspace::DevicePpeWorkspace(DevicePpeWorkspace&& other) noexcept {
  swap_ppe_views(view_, other.view_);
  std::swap(matrix_nnz_capacity_, other.matrix_nnz_capacity_);
}

DevicePpeWorkspace& DevicePpeWorkspace::operator=(DevicePpeWorkspace&& other) noexcept {
  if (this != &other) {
    release();
    swap_ppe_views(view_, other.view_);
    std::swap(matrix_nnz_capacity_, other.matrix_nnz_capacity_);
  }
  return *this;
}

// DevicePpeWorkspace::resize, ppe_matrix.cu:425-442: reallocates only on a
// change of either capacity.
void DevicePpeWorkspace::resize(size_type fluid_capacity, size_type matrix_nnz_capacity) {
  if (fluid_capacity == view_.matrix.rows && matrix_nnz_capacity == matrix_nnz_capacity_) return;
  release();
  view_.matrix.rows = fluid_capacity;
  view_.matrix.cols = fluid_capacity;
  view_.matrix.nnz = matrix_nnz_capacity;
  matrix_nnz_capacity_ = matrix_nnz_capacity;
  dropin::device_alloc(view_.matrix.row_offsets, fluid_capacity + 1);
  dropin::device_alloc(view_.matrix.col_indices, matrix_nnz_capacity);
  dropin::device_alloc(view_.matrix.values, matrix_nnz_capacity);
  dropin::device_alloc(view_.rhs, fluid_capacity);
  dropin::device_alloc(view_.pressure, fluid_capacity);
  dropin::device_alloc(view_.divergence, fluid_capacity);
  dropin::device_alloc(view_.pressure_laplacian, fluid_capacity);
}

void DevicePpeWorkspace::set_active_matrix_nnz(size_type matrix_nnz) {
  if (matrix_nnz > matrix_nnz_capacity_) dropin::fail("PPE active matrix nnz exceeds allocated matrix capacity");
  view_.matrix.nnz = matrix_nnz;
}

void DevicePpeWorkspace::release() noexcept {
  dropin::device_free(view_.matrix.row_offsets);
  dropin::device_free(view_.matrix.col_indices);
  dropin::device_free(view_.matrix.values);
  dropin::device_free(view_.rhs);
  dropin::device_free(view_.pressure);
  dropin::device_free(view_.divergence);
  dropin::device_free(view_.pressure_laplacian);
  view_ = {};
  matrix_nnz_capacity_ = 0;
}

// The reference's accounting (ppe_matrix.cu:464-467): offsets, the CSR slots,
// and four per-row vectors.
size_type DevicePpeWorkspace::bytes() const noexcept {
  return (view_.matrix.rows + 1) * sizeof(index_t) + matrix_nnz_capacity_ * (sizeof(index_t) + sizeof(real)) +
         view_.matrix.rows * 4 * sizeof(real);
}

DevicePpeMatrixAssembler::DevicePpeMatrixAssembler(size_type fluid_capacity, size_type matrix_nnz_capacity,
                                                   SimulationConfig config)
    : config_(std::move(config)), workspace_(fluid_capacity, matrix_nnz_capacity) {}

void DevicePpeMatrixAssembler::resize(size_type fluid_capacity, size_type matrix_nnz_capacity) {
  workspace_.resize(fluid_capacity, matrix_nnz_capacity);
}

void DevicePpeMatrixAssembler::set_config(SimulationConfig config) { config_ = std::move(config); }

size_type DevicePpeMatrixAssembler::bytes() const noexcept { return workspace_.bytes(); }

// DevicePpeMatrixAssembler::assemble, ppe_matrix.cu:486-515: the active nnz
// is N + the fluid CSR capacity (the rows use N + the CSR entries).
void DevicePpeMatrixAssembler::assemble(const FluidParticleSoA& fluid, const WallParticleSoA& walls,
                                        const NeighborListView& fluid_neighbors,
                                        const NeighborListView& wall_neighbors,
                                        const FluidParticleSoA& temporary_velocity,
                                        const WallParticleSoA& temporary_wall_velocity,
                                        DeviceMomentMatrix& moment_matrices, unsigned long long geometry_generation) {
  const size_type required_nnz = fluid.count + fluid_neighbors.neighbor_count;
  if (workspace_.fluid_capacity() < fluid.count || workspace_.matrix_nnz_capacity() < required_nnz)
    resize(fluid.count, required_nnz);
  workspace_.set_active_matrix_nnz(required_nnz);
  const PpeWorkspaceView workspace_view = workspace_.view();
  moment_matrices.set_config(config_);
  moment_matrices.resize(fluid.count);
  moment_matrices.prepare_matrices(fluid, walls, fluid_neighbors, wall_neighbors, geometry_generation);
  assemble_ppe_matrix_and_rhs(fluid, walls, config_, fluid_neighbors, wall_neighbors, temporary_velocity,
                              temporary_wall_velocity, moment_matrices.velocity_type_a(),
                              moment_matrices.pressure_type_a(), workspace_view);
}

// assemble_ppe_matrix_and_rhs, ppe_matrix.cu:517-551.
void assemble_ppe_matrix_and_rhs(const FluidParticleSoA& fluid, const WallParticleSoA& walls,
                                 const SimulationConfig& config, const NeighborListView& fluid_neighbors,
                                 const NeighborListView& wall_neighbors, const FluidParticleSoA& temporary_velocity,
                                 const WallParticleSoA& temporary_wall_velocity,
                                 const MomentMatrixView& velocity_moment, const MomentMatrixView& pressure_moment,
                                 const PpeWorkspaceView& workspace) {
  require_prepared_moment(fluid, velocity_moment, MomentMatrixKind::VelocityWallDirichletTypeA, "velocity");
  require_prepared_moment(fluid, pressure_moment, MomentMatrixKind::PressureWallNeumannTypeA, "pressure");
  const lsmps_params p = dropin::params_of(config);
  const lsmps_fluid f = dropin::view_of(fluid);
  const lsmps_walls w = dropin::view_of(walls);
  const lsmps_csr fn = dropin::view_of(fluid_neighbors);
  const lsmps_csr wn = dropin::view_of(wall_neighbors);
  const lsmps_fluid tv = dropin::view_of(temporary_velocity);
  const lsmps_walls tw = dropin::view_of(temporary_wall_velocity);
  const lsmps_moment vm = dropin::view_of(velocity_moment);
  const lsmps_moment pm = dropin::view_of(pressure_moment);
  const lsmps_ppe ws{lsmps_csr_matrix{workspace.matrix.rows, workspace.matrix.cols, workspace.matrix.nnz,
                                      workspace.matrix.row_offsets, workspace.matrix.col_indices,
                                      workspace.matrix.values},
                     workspace.rhs, workspace.pressure, workspace.divergence, workspace.pressure_laplacian};
  dropin::check(lsmps_assemble_ppe(dropin::context(), &f, &w, &p, &fn, &wn, &tv, &tw, &vm, &pm, &ws));
}

// AmgxPpeSolver (ppe_matrix.cu:553-679).  The reference hands the system to
// AMGX; here lsmps_solve_ppe runs the same method on the device (restarted
// GMRES from a zero initial guess, then the clamp of negative pressures)
// without the host round trip of the CSR.  The configuration file, when one
// is given and exists, is read in AMGX's JSON form for the settings that
// method has: the outer solver must be GMRES; max_iters, tolerance,
// gmres_n_restart, convergence (RELATIVE_INI or ABSOLUTE) and the
// preconditioner's solver (NOSOLVER, or BLOCK_JACOBI / JACOBI_L1 for
// diagonal scaling) are honoured.  Without a file the settings are the
// reference's built-in configuration (:604-610).
namespace {

std::string read_text(const std::filesystem::path& path) {
  std::ifstream in(path);
  std::ostringstream text;
  text << in.rdbuf();
  return text.str();
}

// Position just after `"key"` and the following ':' (npos if absent).
size_t value_of(const std::string& text, const std::string& key, size_t from = 0) {
  const size_t k = text.find("\"" + key + "\"", from);
  if (k == std::string::npos) return std::string::npos;
  const size_t colon = text.find(':', k + key.size() + 2);
  return colon == std::string::npos ? std::string::npos : colon + 1;
}

bool number_of(const std::string& text, const std::string& key, double& out) {
  const size_t v = value_of(text, key);
  if (v == std::string::npos) return false;
  char* end = nullptr;
  const double d = std::strtod(text.c_str() + v, &end);
  if (end == text.c_str() + v) return false;
  out = d;
  return true;
}

// The string value that starts at v (after blanks); empty for other values.
std::string string_at(const std::string& text, size_t v) {
  if (v == std::string::npos) return {};
  const size_t a = text.find_first_not_of(" \t\r\n", v);
  if (a == std::string::npos || text[a] != '"') return {};
  const size_t b = a == std::string::npos ? a : text.find('"', a + 1);
  return b == std::string::npos ? std::string() : text.substr(a + 1, b - a - 1);
}

lsmps_solver_options options_from(const std::filesystem::path& path) {
  lsmps_solver_options o;
  lsmps_solver_options_default(&o);
  std::error_code ec;
  if (path.empty() || !std::filesystem::exists(path, ec)) return o;
  const std::string text = read_text(path);
  // The outer solver: the "solver" value that is not the preconditioner's.
  const size_t pre = value_of(text, "preconditioner");
  std::string outer;
  for (size_t at = 0;;) {
    const size_t v = value_of(text, "solver", at);
    if (v == std::string::npos) break;
    const std::string name = string_at(text, v);
    const bool in_preconditioner = pre != std::string::npos && v > pre && text.find('}', pre) > v;
    if (!name.empty() && !in_preconditioner) outer = name;
    at = v;
  }
  if (outer != "GMRES") dropin::fail("PPE solver configuration " + path.string() + " must use GMRES");
  double d = 0.0;
  if (number_of(text, "max_iters", d)) o.max_iters = static_cast<int32_t>(d);
  if (number_of(text, "tolerance", d)) o.tolerance = d;
  if (number_of(text, "gmres_n_restart", d)) o.restart = static_cast<int32_t>(d);
  const std::string convergence = string_at(text, value_of(text, "convergence"));
  if (convergence == "ABSOLUTE") {
    o.convergence = LSMPS_CONVERGENCE_ABSOLUTE;
  } else if (!convergence.empty() && convergence != "RELATIVE_INI" && convergence != "RELATIVE_INI_CORE") {
    dropin::fail("unsupported PPE solver convergence " + convergence);
  }
  if (pre != std::string::npos) {
    const std::string name = string_at(text, value_of(text, "solver", pre));
    if (name == "BLOCK_JACOBI" || name == "JACOBI_L1") {
      o.preconditioner = LSMPS_PRECONDITIONER_JACOBI;
    } else if (!name.empty() && name != "NOSOLVER") {
      dropin::fail("unsupported PPE preconditioner " + name);
    }
  }
  return o;
}

}  // namespace

struct AmgxPpeSolver::Impl {
  Impl(std::filesystem::path path, bool stats) : config_path(std::move(path)), print_solve_stats(stats) {}
  std::filesystem::path config_path;
  bool print_solve_stats{false};
};

AmgxPpeSolver::AmgxPpeSolver(std::filesystem::path config_path, bool print_solve_stats)
    : impl_(std::make_unique<Impl>(std::move(config_path), print_solve_stats)) {}

AmgxPpeSolver::~AmgxPpeSolver() = default;
AmgxPpeSolver::AmgxPpeSolver(AmgxPpeSolver&&) noexcept = default;
AmgxPpeSolver& AmgxPpeSolver::operator=(AmgxPpeSolver&&) noexcept = default;

// LSMPS_DROPIN_SOLVER=off reproduces the reference's build without AMGX (no
// solve available), e.g. to compare its diagnostic programs output for output.
bool AmgxPpeSolver::is_available() noexcept {
  const char* v = std::getenv("LSMPS_DROPIN_SOLVER");
  return v == nullptr || std::string(v) != "off";
}

const std::filesystem::path& AmgxPpeSolver::config_path() const noexcept { return impl_->config_path; }

void AmgxPpeSolver::solve(const CsrMatrixView& matrix, const real* rhs, real* pressure) {
  if (matrix.rows == 0) return;
  if (matrix.rows != matrix.cols || matrix.row_offsets == nullptr || matrix.col_indices == nullptr ||
      matrix.values == nullptr || rhs == nullptr || pressure == nullptr)
    dropin::fail("AMGX PPE solve requires a square CSR matrix, rhs, and solution buffer");
  if (!is_available())
    dropin::fail(
        "AMGX support is not enabled in this build. Configure with AMGX headers and library available to use "
        "AmgxPpeSolver.");
  const lsmps_solver_options options = options_from(impl_->config_path);
  const lsmps_csr_matrix a{matrix.rows, matrix.cols, matrix.nnz, matrix.row_offsets, matrix.col_indices,
                           matrix.values};
  lsmps_solver_report report{};
  dropin::check(lsmps_solve_ppe(dropin::context(), &a, rhs, pressure, &options, &report));
  if (impl_->print_solve_stats)
    std::cout << "PPE GMRES(" << options.restart << "): " << report.iterations << " iterations, residual "
              << report.initial_residual << " -> " << report.final_residual
              << (report.converged ? " (converged)" : " (not converged)") << std::endl;
}

}  // namespace lsmps3d
