"""Builds StepBuffers (host or device) from the reference known-answer
fixtures in golden/reference_kats.json."""

import numpy as np


def params_from(pkg, kat, grid=None):
    p = pkg.abi.default_params()
    for k, v in kat.get("params", {}).items():
        if k == "gravity":
            p.gravity[:] = v
        else:
            setattr(p, k, v)
    if "support_radius" in kat:
        p.support_radius = kat["support_radius"]
    g = grid or kat.get("grid")
    if g is not None:
        p.grid.origin[:] = g["origin"]
        p.grid.cell_size = g["cell_size"]
        p.grid.dims[:] = g["dims"]
    else:
        p.grid.cell_size = p.support_radius
    return p


def buffers_from(pkg, alloc, kat):
    fl = kat["fluid"]
    wl = kat.get("walls", {"x": []})
    nf, nw = len(fl["x"]), len(wl["x"])
    g = kat.get("grid")
    nc = int(np.prod(g["dims"])) if g else 1
    if "fluid_offsets" in kat:
        cap_f = len(kat["fluid_indices"])
        cap_w = 0
        b = pkg.buffers.StepBuffers(alloc, nf, nw, nc, fluid_capacity=cap_f, wall_capacity=cap_w)
        alloc.copy_(b.fluid_neighbors["offsets"], np.asarray(kat["fluid_offsets"], np.int32))
        alloc.copy_(b.fluid_neighbors["indices"], np.asarray(kat["fluid_indices"], np.int32))
        alloc.copy_(b.wall_neighbors["offsets"], np.zeros(nf + 1, np.int32))
    else:
        b = pkg.buffers.StepBuffers(alloc, nf, nw, nc, kat.get("max_fluid_neighbors", 256),
                                    kat.get("max_wall_neighbors", 256))
    for k, v in fl.items():
        alloc.copy_(b.fluid[k], np.asarray(v, np.float64))
    if "surface_type" in kat:
        alloc.copy_(b.fluid["surface_type"], np.asarray(kat["surface_type"], np.int32))
    for k, v in wl.items():
        alloc.copy_(b.walls[k], np.asarray(v, np.float64))
    return b


def rows(off, idx, n):
    return [sorted(int(v) for v in idx[off[i]:off[i + 1]]) for i in range(n)]


def rel_err(g, o, floor_frac=1e-3, scale=None):
    """max(normwise, elementwise) relative error of g against o.
    normwise = max|g-o| / scale, scale = max|o| unless given (pass the
    magnitude of the whole vector field for one of its components);
    elementwise = max |g-o|/|o| over entries with |o| >= floor_frac * scale
    (entries that cancel to near zero are covered by the normwise term)."""
    g = np.asarray(g, dtype=np.float64)
    o = np.asarray(o, dtype=np.float64)
    if o.size == 0:
        return 0.0
    s = float(np.max(np.abs(o))) if scale is None else float(scale)
    if s == 0.0:
        return float(np.max(np.abs(g)))
    d = np.abs(g - o)
    big = np.abs(o) >= floor_frac * s
    elem = float(np.max(d[big] / np.abs(o[big]))) if big.any() else 0.0
    return max(float(np.max(d)) / s, elem)


def vec_err(g: dict, o: dict, comps, extra_scale: dict | None = None):
    """rel_err of each component against the scale of the whole vector (and
    of `extra_scale`'s same-named arrays, e.g. the operands of a cancellation)."""
    arrays = [np.asarray(o[c]) for c in comps]
    if extra_scale is not None:
        arrays += [np.asarray(extra_scale[c]) for c in comps if c in extra_scale]
    scale = max(float(np.max(np.abs(a))) if a.size else 0.0 for a in arrays)
    return {c: rel_err(g[c], o[c], scale=scale if scale > 0 else None) for c in comps}


EPS64 = 2.0 ** -52


def inverse_err_over_kappa(got, ref, trace, reg):
    """Per-particle error of 9 x 9 moment inverses (rows of 81 entries)
    against a reference, max |dX| / max |X|, divided by 2^-52 kappa_est with
    kappa_est = (trace + 9 reg) ||X||_F, an upper bound of the 2-norm
    condition number within a factor of 27 (trace = the moment trace before
    regularisation, reg = the regularisation added to each diagonal entry).
    Rounding-level agreement reads O(1) whatever the conditioning."""
    g = np.asarray(got, dtype=np.float64).reshape(-1, 81)
    r = np.asarray(ref, dtype=np.float64).reshape(-1, 81)
    if r.shape[0] == 0:
        return 0.0
    per = np.max(np.abs(g - r), axis=1) / np.max(np.abs(r), axis=1)
    kappa = (np.asarray(trace) + 9.0 * np.asarray(reg)) * np.sqrt(np.einsum("ij,ij->i", r, r))
    return float(np.max(per / (EPS64 * kappa)))


def coef_rel_err(values, ref_values, floor_frac=1e-4):
    """Per-coefficient relative error of a matrix's values against a
    reference: max |a - r| / max(|r|, floor), floor = floor_frac times the
    largest |r| (coefficients below the floor are measured against it)."""
    v = np.asarray(values, dtype=np.float64)
    r = np.asarray(ref_values, dtype=np.float64)
    if r.size == 0:
        return 0.0
    floor = floor_frac * float(np.max(np.abs(r)))
    if floor == 0.0:
        return float(np.max(np.abs(v)))
    return float(np.max(np.abs(v - r) / np.maximum(np.abs(r), floor)))


def row_rel_err(values, ref_values, row_offsets):
    """Row-normwise relative error of a CSR matrix against a reference with
    the same pattern: max over rows of max_j |a_ij - r_ij| / max_j |r_ij|
    (rows whose reference is all zero are compared absolutely).  This is the
    "max relative error in PPE coefficients" the mixed form is held to: each
    coefficient's error measured against the size of its own row."""
    v = np.asarray(values, dtype=np.float64)
    r = np.asarray(ref_values, dtype=np.float64)
    off = np.asarray(row_offsets, dtype=np.int64)
    n = off.size - 1
    if n <= 0:
        return 0.0
    d = np.abs(v[: off[-1]] - r[: off[-1]])
    a = np.abs(r[: off[-1]])
    lengths = np.diff(off)
    nz = lengths > 0
    starts = off[:-1][nz]
    dmax = np.maximum.reduceat(d, starts)
    amax = np.maximum.reduceat(a, starts)
    per_row = np.where(amax > 0, dmax / np.where(amax > 0, amax, 1.0), dmax)
    return float(per_row.max()) if per_row.size else 0.0


LIGHT_DIRECTIONS = np.array(
    [[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]]
    + [[a * 0.7071067811865475, b * 0.7071067811865475, 0] for a, b in ((1, 1), (1, -1), (-1, 1), (-1, -1))]
    + [[0.7071067811865475, 0, 0.7071067811865475], [0.7071067811865475, 0, -0.7071067811865475],
       [0, 0.7071067811865475, 0.7071067811865475], [0, 0.7071067811865475, -0.7071067811865475]])


def light_ties(b, params, eps=1e-12):
    """Per fluid particle, how many of the 14 virtual-light directions have a
    neighbour whose projection lies within eps of the cone cosine.  Such a
    direction's open/blocked answer depends on the last bits of the
    projection (FMA contraction, the device rsqrt), so the CPU oracle and the
    device may differ there by up to that many directions."""
    n = b.n_fluid
    ties = np.zeros((n, 14), dtype=bool)
    re2 = params.support_radius ** 2
    rows = [("fluid", b.fluid)]
    if params.include_wall_neighbors:
        rows.append(("wall", b.walls))
    for which, src in rows:
        off, idx = b.csr_rows(which)
        owner = np.repeat(np.arange(n), np.diff(off[: n + 1]))
        idx = idx[: len(owner)]
        d = np.stack([src[c][idx] - b.fluid[c][owner] for c in ("x", "y", "z")], 1)
        d2 = (d * d).sum(1)
        ok = (d2 > 0) & (d2 <= re2)
        proj = (d[ok] @ LIGHT_DIRECTIONS.T) / np.sqrt(d2[ok])[:, None]
        near = np.abs(proj - params.virtual_light_cone_cosine) <= eps
        np.logical_or.at(ties, owner[ok], near)
    return ties.sum(1)
