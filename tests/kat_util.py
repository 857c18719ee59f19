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
