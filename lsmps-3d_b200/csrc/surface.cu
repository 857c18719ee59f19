// surface.cu - Inner / NearSurface / Surface / Splash labels.
// Replaces classify_surface_particles (src/surface/surface_detection.cu:522-553):
// classify_primary_surface_kernel (:199-320) and expand_near_surface_kernel
// (:322-348), plus the host-side reference number density (:494-520).
//
// The labels compare floating sums with thresholds, so each particle's sums
// are accumulated by one thread in CSR row order with the reference's own
// expressions: the FP64 values, and hence the labels, are the reference's.
#include <cmath>

#include "impl.cuh"
#include "packed.cuh"

namespace lsmps {
namespace {

constexpr int kSurfaceThreads = 128;

__device__ __forceinline__ double safe_rsqrt(double v) { return rsqrt(v > 1.0e-20 ? v : 1.0e-20); }

// accumulate_neighbor_moments, surface_detection.cu:33-59
__device__ __forceinline__ void accumulate(double dx, double dy, double dz, double re, double& nd, double& sx,
                                           double& sy, double& sz, int& weighted) {
  const double d2 = dx * dx + dy * dy + dz * dz;
  if (d2 <= 0.0) return;
  const double d = sqrt(d2);
  const double w = lin_weight(d, re);
  if (w <= 0.0) return;
  const double inv_d = 1.0 / d;
  nd += w;
  sx += w * dx * inv_d;
  sy += w * dy * inv_d;
  sz += w * dz * inv_d;
  ++weighted;
}

struct Basis3 {
  int count;
  double x[3], y[3], z[3];
};

// add_wall_basis_direction, surface_detection.cu:123-149
__device__ __forceinline__ void add_direction(Basis3& b, double x, double y, double z, double thr) {
  double rx = x, ry = y, rz = z;
  for (int k = 0; k < b.count; ++k) {
    const double proj = rx * b.x[k] + ry * b.y[k] + rz * b.z[k];
    rx -= proj * b.x[k];
    ry -= proj * b.y[k];
    rz -= proj * b.z[k];
  }
  const double len2 = rx * rx + ry * ry + rz * rz;
  if (len2 <= thr * thr || b.count >= 3) return;
  const double inv = safe_rsqrt(len2);
  b.x[b.count] = rx * inv;
  b.y[b.count] = ry * inv;
  b.z[b.count] = rz * inv;
  ++b.count;
}

struct SurfaceArgs {
  lsmps_fluid fluid;
  lsmps_walls walls;
  const index_t* fo;
  const index_t* fi;
  const index_t* wo;
  const index_t* wi;
  lsmps_params p;
  double n0;
  lsmps_surface_diagnostics diag;
  // 32-byte records (packed.cuh): fluid {x, y, z, -}, walls {x, y, z, -} and
  // {nx, ny, nz, -}.
  const double4* fp;
  const double4* wp;
  const double4* wn;
  const int32_t* order;  // visiting order (lsmps_ctx::order) or NULL
  // fi and fp in cell-sorted positions (sorted_rows_of): the labels are also
  // written by visiting position into sorted_labels, for the expansion
  int sorted;
  int32_t* sorted_labels;
};

__global__ void __launch_bounds__(kSurfaceThreads) classify_kernel(SurfaceArgs a) {
  const index_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= static_cast<index_t>(a.fluid.count)) return;
  const index_t i = visit(a.order, t);
  const index_t fb = a.fo[i], fe = a.fo[i + 1];
  const index_t wb = a.wo[i], we = a.wo[i + 1];
  const index_t fcount = fe - fb, wcount = we - wb;
  const index_t cls = a.p.include_wall_neighbors ? fcount + wcount : fcount;
  const double re = a.p.support_radius;
  const double4 own = ld4(a.fp, self_of(a.sorted, t, i));
  const double px = own.x, py = own.y, pz = own.z;
  double nd = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
  int weighted = 0;
  // the next neighbour's record is loaded while this one is accumulated
  double4 qn = ld4(a.fp, fb < fe ? a.fi[fb] : i);
  index_t jnn = fb + 1 < fe ? a.fi[fb + 1] : i;  // the index after the next
  for (index_t o = fb; o < fe; ++o) {
    const double4 q = qn;
    if (o + 1 < fe) {
      qn = ld4(a.fp, jnn);
      if (o + 2 < fe) jnn = a.fi[o + 2];
    }
    accumulate(q.x - px, q.y - py, q.z - pz, re, nd, sx, sy, sz, weighted);
  }
  if (a.p.include_wall_neighbors) {
    for (index_t o = wb; o < we; ++o) {
      const double4 q = ld4(a.wp, a.wi[o]);
      accumulate(q.x - px, q.y - py, q.z - pz, re, nd, sx, sy, sz, weighted);
    }
  }
  double aniso = 0.0;
  if (weighted > 0) aniso = sqrt(sx * sx + sy * sy + sz * sz) / static_cast<double>(weighted);
  const double ratio = nd / a.n0;
  const double mx = -sx, my = -sy, mz = -sz;
  const double ml2 = mx * mx + my * my + mz * mz;
  double ax = mx, ay = my, az = mz;
  if (ml2 > 0.0 && a.p.include_wall_neighbors) {
    // build_wall_basis, surface_detection.cu:151-197
    Basis3 basis;
    basis.count = 0;
    for (index_t o = wb; o < we; ++o) {
      const index_t j = a.wi[o];
      const double4 q = ld4(a.wp, j);
      const double dx = q.x - px, dy = q.y - py, dz = q.z - pz;
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 <= 0.0) continue;
      const double d = sqrt(d2);
      if (lin_weight(d, re) <= 0.0) continue;
      const double4 nrm = ld4(a.wn, j);
      const double nx = nrm.x, ny = nrm.y, nz = nrm.z;
      const double nl2 = nx * nx + ny * ny + nz * nz;
      if (nl2 <= 0.0) continue;
      const double inv = safe_rsqrt(nl2);
      add_direction(basis, -nx * inv, -ny * inv, -nz * inv, a.p.wall_normal_independence_threshold);
    }
    for (int k = 0; k < basis.count; ++k) {
      const double proj = ax * basis.x[k] + ay * basis.y[k] + az * basis.z[k];
      if (proj > 0.0) {
        ax -= proj * basis.x[k];
        ay -= proj * basis.y[k];
        az -= proj * basis.z[k];
      }
    }
  }
  const double al2 = ax * ax + ay * ay + az * az;
  const double al = sqrt(al2);
  const double ml = sqrt(ml2);
  const double open = ml > 0.0 ? al / ml : 0.0;
  const double aaniso = weighted > 0 ? al / static_cast<double>(weighted) : 0.0;
  int type = LSMPS_SURFACE_INNER;
  if (cls < a.p.splash_neighbor_threshold) {
    type = LSMPS_SURFACE_SPLASH;
  } else if (ratio < a.p.number_density_ratio_threshold && open > a.p.air_open_ratio_threshold &&
             aaniso > a.p.air_anisotropy_threshold) {
    type = LSMPS_SURFACE_SURFACE;
  }
  a.fluid.surface_type[i] = type;
  if (a.sorted) a.sorted_labels[t] = type;
  const lsmps_surface_diagnostics& d = a.diag;
  if (d.fluid_neighbor_count) d.fluid_neighbor_count[i] = fcount;
  if (d.wall_neighbor_count) d.wall_neighbor_count[i] = wcount;
  if (d.number_density) d.number_density[i] = nd;
  if (d.number_density_ratio) d.number_density_ratio[i] = ratio;
  if (d.anisotropy) d.anisotropy[i] = aniso;
  if (d.air_open_ratio) d.air_open_ratio[i] = open;
  if (d.air_anisotropy) d.air_anisotropy[i] = aaniso;
  if (d.surface_normal_x || d.surface_normal_y || d.surface_normal_z) {
    double snx = 0.0, sny = 0.0, snz = 0.0;
    if (al2 > 0.0) {
      const double inv = safe_rsqrt(al2);
      snx = ax * inv;
      sny = ay * inv;
      snz = az * inv;
    }
    if (d.surface_normal_x) d.surface_normal_x[i] = snx;
    if (d.surface_normal_y) d.surface_normal_y[i] = sny;
    if (d.surface_normal_z) d.surface_normal_z[i] = snz;
  }
}

// expand_near_surface_kernel, surface_detection.cu:322-348.  Only Inner rows
// are written and only Surface labels are read, so the pass is race-free.
// Reads the 4-byte label of each neighbour first; positions are read only
// for the (few) Surface neighbours.  kExpandLanes lanes share a row (lane l
// takes entries l, l + kExpandLanes, ...); the answer is whether any lane
// found a Surface neighbour within r_ns, which does not depend on the order.
constexpr int kExpandLanes = 4;

// With cell-sorted rows (sorted_labels non-NULL), fi and fp are in sorted
// positions and the neighbours' labels are read from sorted_labels.
__global__ void __launch_bounds__(kSurfaceThreads) expand_kernel(const double4* __restrict__ fp, int32_t* type,
                                                                 index_t n, const index_t* __restrict__ fo,
                                                                 const index_t* __restrict__ fi, double r2,
                                                                 const int32_t* __restrict__ order,
                                                                 const int32_t* __restrict__ sorted_labels) {
  const index_t t = (blockIdx.x * blockDim.x + threadIdx.x) / kExpandLanes;
  const int l = threadIdx.x & (kExpandLanes - 1);
  if (t >= n) return;  // the whole group
  const index_t i = visit(order, t);
  // (the particle's own label from classify: sorted_labels[t] equals type[i]
  // until this thread writes it)
  if ((sorted_labels ? sorted_labels[t] : type[i]) != LSMPS_SURFACE_INNER) return;
  const int32_t* __restrict__ nlab = sorted_labels ? sorted_labels : type;
  const double4 own = ld4(fp, sorted_labels ? t : i);
  bool near = false;
  const index_t fe = fo[i + 1];
  // kExpandBatch entries per lane and round: their indices, then their
  // labels, are loaded together, so a round costs two dependent load
  // latencies instead of two per entry.
  constexpr int kExpandBatch = 4;
  for (index_t o = fo[i] + l; o < fe && !near; o += kExpandLanes * kExpandBatch) {
    index_t j[kExpandBatch];
    int32_t lab[kExpandBatch];
#pragma unroll
    for (int k = 0; k < kExpandBatch; ++k) {
      const index_t e = o + k * kExpandLanes;
      j[k] = e < fe ? fi[e] : -1;
    }
#pragma unroll
    for (int k = 0; k < kExpandBatch; ++k) lab[k] = j[k] >= 0 ? nlab[j[k]] : LSMPS_SURFACE_INNER;
#pragma unroll
    for (int k = 0; k < kExpandBatch; ++k) {
      if (lab[k] != LSMPS_SURFACE_SURFACE) continue;
      const double4 q = ld4(fp, j[k]);
      const double dx = q.x - own.x, dy = q.y - own.y, dz = q.z - own.z;
      near = near || dx * dx + dy * dy + dz * dz <= r2;
    }
  }
  // Only Inner rows are written and only Surface labels are read, so the
  // in-place update is race-free.
  const unsigned hit = __ballot_sync(group_mask<kExpandLanes>(), near);
  if (l == 0 && hit != 0u) type[i] = LSMPS_SURFACE_NEAR_SURFACE;
}

// Virtual-light openness, virtual_light_kernel (surface_detection.cu:445-475).
// The 14 light directions of virtual_light_direction (:350-382): the six axes,
// then (±1, ±1, 0)/√2 in the order ++, +-, -+, --, then (1, 0, ±1)/√2 and
// (0, 1, ±1)/√2.  A direction is blocked when some neighbour within the
// support radius has (d · dir)/|d| >= cone cosine.
//
// The reference walks the neighbour rows once per direction (14 passes); here
// each neighbour is read once and tested against all 14 directions, and the
// blocked directions are kept as a 14-bit mask.  Whether a direction is
// blocked does not depend on the order in which neighbours are tested, so
// kLightLanes lanes share a row and OR their masks.  The projection is the
// reference's expression, (dx·ux + dy·uy + dz·uz)·rsqrt(d²), term for term.
constexpr int kLightDirections = 14;
constexpr int kLightLanes = 4;

// The projections of virtual_light_direction's 14 unit vectors, each the
// reference's (dx ux + dy uy + dz uz) * rsqrt(d2) with the terms whose
// component is 0 left out: x*1 = x, x*(-1) = -x and adding x*0 = ±0 are
// exact, so for finite offsets the values are bit-identical to the full
// expression, while the FP64 pipe (this kernel's bound) does about half the
// work.  The two-term sums keep the reference's operand order, so the
// compiler contracts them into the same FMA as the three-term form.
__device__ __forceinline__ unsigned blocked_directions(double dx, double dy, double dz, double re2, double cone) {
  const double d2 = dx * dx + dy * dy + dz * dz;
  if (d2 <= 0.0 || d2 > re2) return 0u;
  const double inv = safe_rsqrt(d2);
  constexpr double s = 0.7071067811865475;
  const double px = dx * inv, py = dy * inv, pz = dz * inv;
  unsigned mask = 0u;
  mask |= (px >= cone) ? 1u << 0 : 0u;
  mask |= (-px >= cone) ? 1u << 1 : 0u;
  mask |= (py >= cone) ? 1u << 2 : 0u;
  mask |= (-py >= cone) ? 1u << 3 : 0u;
  mask |= (pz >= cone) ? 1u << 4 : 0u;
  mask |= (-pz >= cone) ? 1u << 5 : 0u;
  mask |= ((dx * s + dy * s) * inv >= cone) ? 1u << 6 : 0u;
  mask |= ((dx * s + dy * -s) * inv >= cone) ? 1u << 7 : 0u;
  mask |= ((dx * -s + dy * s) * inv >= cone) ? 1u << 8 : 0u;
  mask |= ((dx * -s + dy * -s) * inv >= cone) ? 1u << 9 : 0u;
  mask |= ((dx * s + dz * s) * inv >= cone) ? 1u << 10 : 0u;
  mask |= ((dx * s + dz * -s) * inv >= cone) ? 1u << 11 : 0u;
  mask |= ((dy * s + dz * s) * inv >= cone) ? 1u << 12 : 0u;
  mask |= ((dy * s + dz * -s) * inv >= cone) ? 1u << 13 : 0u;
  return mask;
}

__global__ void __launch_bounds__(kSurfaceThreads)
    virtual_light_kernel(const double4* __restrict__ fp, const double4* __restrict__ wp, index_t n,
                         const index_t* __restrict__ fo, const index_t* __restrict__ fi,
                         const index_t* __restrict__ wo, const index_t* __restrict__ wi, int include_walls,
                         double re2, double cone, int32_t* open_count, double* open_fraction) {
  const index_t i = (blockIdx.x * blockDim.x + threadIdx.x) / kLightLanes;
  const int l = threadIdx.x & (kLightLanes - 1);
  if (i >= n) return;  // the whole group
  const double4 own = ld4(fp, i);
  constexpr unsigned kAll = (1u << kLightDirections) - 1u;
  const unsigned gm = group_mask<kLightLanes>();
  unsigned blocked = 0u;
  // The group walks the row kLightLanes entries at a time and merges its
  // masks after each round, so it stops as soon as all 14 directions are
  // blocked (every lane runs the same rounds).
  const index_t fe = fo[i + 1];
  for (index_t base = fo[i]; base < fe && blocked != kAll; base += kLightLanes) {
    const index_t o = base + l;
    if (o < fe) {
      const double4 q = ld4(fp, fi[o]);
      blocked |= blocked_directions(q.x - own.x, q.y - own.y, q.z - own.z, re2, cone);
    }
    blocked = __reduce_or_sync(gm, blocked);
  }
  if (include_walls) {
    const index_t we = wo[i + 1];
    for (index_t base = wo[i]; base < we && blocked != kAll; base += kLightLanes) {
      const index_t o = base + l;
      if (o < we) {
        const double4 q = ld4(wp, wi[o]);
        blocked |= blocked_directions(q.x - own.x, q.y - own.y, q.z - own.z, re2, cone);
      }
      blocked = __reduce_or_sync(gm, blocked);
    }
  }
  if (l != 0) return;
  const int open = kLightDirections - __popc(blocked);
  if (open_count) open_count[i] = open;
  if (open_fraction) open_fraction[i] = static_cast<double>(open) / static_cast<double>(kLightDirections);
}

}  // namespace

lsmps_status virtual_light_impl(lsmps_ctx* ctx, const lsmps_fluid& fluid, const lsmps_walls& walls,
                                const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_params& p,
                                int32_t* open_count, double* open_fraction) {
  // validate_surface_inputs and the checks of compute_virtual_light_diagnostics,
  // surface_detection.cu:477-492, 555-578.
  if (!(p.support_radius > 0.0))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Surface detection support radius must be positive");
  if (fluid.count > fn.particle_count || fluid.count > wn.particle_count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Surface detection neighbor lists are smaller than fluid particle count");
  if (!(p.virtual_light_cone_cosine >= -1.0 && p.virtual_light_cone_cosine <= 1.0))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Virtual light cone cosine must be in [-1, 1]");
  if (!open_count && !open_fraction)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Virtual light diagnostics require at least one output buffer");
  if (fluid.count == 0) return LSMPS_OK;
  if (const lsmps_status cs = check_neighbor_tables(ctx, fluid.count, walls.count, fn, &wn)) return cs;
  if (!ensure_packs(ctx, fluid.count, walls.count)) return fail(ctx, LSMPS_CUDA_ERROR, "pack allocation failed");
  pack4(ctx, fluid.x, fluid.y, fluid.z, nullptr, fluid.count, ctx->pack_fluid[0]);
  pack4(ctx, walls.x, walls.y, walls.z, nullptr, walls.count, ctx->pack_wall[0]);
  const index_t n = static_cast<index_t>(fluid.count);
  launch(ctx, virtual_light_kernel, dim3(div_up(static_cast<long long>(n) * kLightLanes, kSurfaceThreads)),
         dim3(kSurfaceThreads), 0, static_cast<const double4*>(ctx->pack_fluid[0]),
         static_cast<const double4*>(ctx->pack_wall[0]), n, static_cast<const index_t*>(fn.offsets),
         static_cast<const index_t*>(fn.indices), static_cast<const index_t*>(wn.offsets),
         static_cast<const index_t*>(wn.indices), p.include_wall_neighbors ? 1 : 0,
         p.support_radius * p.support_radius, p.virtual_light_cone_cosine, open_count, open_fraction);
  return check_launch(ctx, "virtual light diagnostics");
}

// compute_uniform_reference_number_density, surface_detection.cu:494-520.
double reference_number_density(double l0, double re) {
  if (!(l0 > 0.0) || !(re > 0.0)) return -1.0;
  const int extent = static_cast<int>(std::ceil(re / l0));
  double n0 = 0.0;
  for (int iz = -extent; iz <= extent; ++iz)
    for (int iy = -extent; iy <= extent; ++iy)
      for (int ix = -extent; ix <= extent; ++ix) {
        if (ix == 0 && iy == 0 && iz == 0) continue;
        const double dx = ix * l0, dy = iy * l0, dz = iz * l0;
        const double d = std::sqrt(dx * dx + dy * dy + dz * dz);
        n0 += d >= re ? 0.0 : 1.0 - d / re;
      }
  return n0;
}

lsmps_status classify_surface_impl(lsmps_ctx* ctx, const lsmps_fluid& fluid, const lsmps_walls& walls,
                                   const lsmps_csr& fn, const lsmps_csr& wn, const lsmps_params& p,
                                   const lsmps_surface_diagnostics* diag) {
  if (!(p.support_radius > 0.0))
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Surface detection support radius must be positive");
  if (fluid.count > fn.particle_count || fluid.count > wn.particle_count)
    return fail(ctx, LSMPS_INVALID_ARGUMENT, "Surface detection neighbor lists are smaller than fluid particle count");
  if (p.near_surface_radius < 0.0) return fail(ctx, LSMPS_INVALID_ARGUMENT, "Near-surface radius must be non-negative");
  const double n0 = reference_number_density(p.particle_spacing, p.support_radius);
  if (!(n0 > 0.0)) return fail(ctx, LSMPS_INVALID_ARGUMENT, "Reference number density must be positive");
  if (fluid.count == 0) return LSMPS_OK;
  if (const lsmps_status cs = check_neighbor_tables(ctx, fluid.count, walls.count, fn, &wn)) return cs;
  if (!fluid.surface_type) return fail(ctx, LSMPS_INVALID_ARGUMENT, "surface_type buffer missing");
  const index_t* srows = sorted_rows_of(ctx, fn, fluid.count);
  SurfaceArgs a{};
  a.fluid = fluid;
  a.walls = walls;
  a.fo = fn.offsets;
  a.fi = srows ? srows : fn.indices;
  a.sorted = srows ? 1 : 0;
  a.sorted_labels = srows ? ctx->sorted_labels : nullptr;
  a.wo = wn.offsets;
  a.wi = wn.indices;
  a.p = p;
  a.n0 = n0;
  if (diag) a.diag = *diag;
  if (!ensure_packs(ctx, fluid.count, walls.count)) return fail(ctx, LSMPS_CUDA_ERROR, "pack allocation failed");
  pack4(ctx, fluid.x, fluid.y, fluid.z, nullptr, fluid.count, ctx->pack_fluid[0], srows ? ctx->order : nullptr);
  pack_wall_positions(ctx, walls);
  pack_wall_normals(ctx, walls);
  a.fp = ctx->pack_fluid[0];
  a.wp = ctx->pack_wall[0];
  a.wn = ctx->pack_wall[2];
  a.order = ctx->order;
  const index_t n = static_cast<index_t>(fluid.count);
  launch(ctx, classify_kernel, dim3(div_up(n, kSurfaceThreads)), dim3(kSurfaceThreads), 0, a);
  if (p.near_surface_radius > 0.0) {
    launch(ctx, expand_kernel, dim3(div_up(static_cast<long long>(n) * kExpandLanes, kSurfaceThreads)),
           dim3(kSurfaceThreads), 0,
           static_cast<const double4*>(ctx->pack_fluid[0]), fluid.surface_type, n,
           static_cast<const index_t*>(fn.offsets), a.fi, p.near_surface_radius * p.near_surface_radius,
           static_cast<const int32_t*>(ctx->order), static_cast<const int32_t*>(a.sorted_labels));
  }
  return check_launch(ctx, "surface classification");
}

}  // namespace lsmps

using namespace lsmps;

extern "C" double lsmps_reference_number_density(double particle_spacing, double support_radius) {
  return reference_number_density(particle_spacing, support_radius);
}

extern "C" lsmps_status lsmps_classify_surface(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_walls* walls,
                                               const lsmps_csr* fluid_neighbors, const lsmps_csr* wall_neighbors,
                                               const lsmps_params* params,
                                               const lsmps_surface_diagnostics* diagnostics) {
  if (!ctx || !fluid || !walls || !fluid_neighbors || !wall_neighbors || !params) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  st = classify_surface_impl(ctx, *fluid, *walls, *fluid_neighbors, *wall_neighbors, *params, diagnostics);
  return end_call(ctx, st);
}

extern "C" lsmps_status lsmps_virtual_light(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_walls* walls,
                                            const lsmps_csr* fluid_neighbors, const lsmps_csr* wall_neighbors,
                                            const lsmps_params* params, int32_t* open_direction_count,
                                            double* open_fraction) {
  if (!ctx || !fluid || !walls || !fluid_neighbors || !wall_neighbors || !params) return LSMPS_INVALID_ARGUMENT;
  lsmps_status st = begin_call(ctx);
  if (st) return st;
  st = virtual_light_impl(ctx, *fluid, *walls, *fluid_neighbors, *wall_neighbors, *params, open_direction_count,
                          open_fraction);
  return end_call(ctx, st);
}
