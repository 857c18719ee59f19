"""lsmps_build_cell_list_noalloc (fixed static scratch, no context, no
allocation) against lsmps_build_cell_list (context scratch).

Integer outputs, so the tolerance is zero: cell ids, sorted indices and cell
ranges must be bit-identical.  Each case calls the allocation-free entry
point twice in a row on the same output buffers (with the buffers poisoned
in between) so that state left in the static scratch by the first call cannot
hide in the second.  The file is named to be collected last and also passes
alone in a fresh process; test_noalloc_first_in_a_fresh_process makes the
allocation-free entry point the first library call of a new process and
checks that, once its first call has done the per-device set-up, later calls
leave the device's free memory unchanged.
"""

import ctypes
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _grid(pkg, origin, cell_size, dims):
    g = pkg.abi.Grid()
    g.origin[:] = origin
    g.cell_size = cell_size
    g.dims[:] = dims
    return g


def _cells(pkg, torch, n, ncell):
    out = {k: torch.full((n if k in ("cell_ids", "sorted_indices") else ncell,), -7, dtype=torch.int32,
                         device="cuda") for k in ("cell_ids", "sorted_indices", "cell_begin", "cell_end")}
    view = pkg.abi.Cells()
    view.particle_count, view.cell_count = n, ncell
    for k, v in out.items():
        setattr(view, k, v.data_ptr())
    return out, view


def _compare(pkg, device_api, xyz, grid):
    import torch

    lib = device_api._lib
    n = xyz[0].shape[0]
    ncell = int(np.prod(list(grid.dims)))
    t = [torch.from_numpy(np.ascontiguousarray(c)).cuda() for c in xyz]
    ptrs = [c.data_ptr() for c in t]
    ctx = device_api.Context(0)
    try:
        want, want_view = _cells(pkg, torch, n, ncell)
        ctx.build_cell_list(*ptrs, n, grid, want_view)
    finally:
        ctx.close()
    stream = torch.cuda.Stream()
    got, got_view = _cells(pkg, torch, n, ncell)
    for call in range(2):
        for v in got.values():
            v.fill_(-7)
        torch.cuda.synchronize()
        st = lib.lsmps_build_cell_list_noalloc(ctypes.c_void_p(stream.cuda_stream), *ptrs, n, ctypes.byref(grid),
                                               ctypes.byref(got_view))
        assert st == pkg.abi.OK, (call, pkg.abi.STATUS_NAMES.get(st, st))
        for k in want:
            assert torch.equal(got[k], want[k]), (call, k)


def test_noalloc_cell_list_dam_break(pkg, device_api):
    """Fluid and wall particles of a 30 x 15 x 30 dam break (3,360 cells:
    12-bit ids, two radix passes)."""
    case = pkg.cases.dam_break(30, 15, 30)
    f, w = case.fluid, case.walls
    grid = case.params.grid
    _compare(pkg, device_api, (f["x"], f["y"], f["z"]), grid)
    _compare(pkg, device_api, (w["x"], w["y"], w["z"]), grid)


def test_noalloc_cell_list_at_its_limit(pkg, device_api):
    """Exactly LSMPS_NOALLOC_MAX_PARTICLES random particles on a grid of
    4.32M cells (23-bit ids, three radix passes), duplicates included."""
    rng = np.random.default_rng(11)
    n = pkg.abi.NOALLOC_MAX_PARTICLES
    dims = (180, 160, 150)
    xyz = [rng.random(n) * d * 0.01 for d in dims]
    xyz[0][: n // 8] = xyz[0][n // 8: n // 4]  # shared cells, so stability matters
    _compare(pkg, device_api, xyz, _grid(pkg, (0.0, 0.0, 0.0), 0.01, dims))


def test_noalloc_cell_list_rejects_sizes_beyond_its_limit(pkg, device_api):
    import torch

    lib = device_api._lib
    n = pkg.abi.NOALLOC_MAX_PARTICLES + 1
    grid = _grid(pkg, (0.0, 0.0, 0.0), 0.01, (4, 4, 4))
    _, view = _cells(pkg, torch, n, 64)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    st = lib.lsmps_build_cell_list_noalloc(None, x.data_ptr(), x.data_ptr(), x.data_ptr(), n, ctypes.byref(grid),
                                           ctypes.byref(view))
    assert st == pkg.abi.CAPACITY_EXCEEDED


def test_noalloc_cell_list_empty_and_non_finite(pkg, device_api):
    import torch

    lib = device_api._lib
    grid = _grid(pkg, (0.0, 0.0, 0.0), 0.1, (5, 5, 5))
    out, view = _cells(pkg, torch, 0, 125)
    assert lib.lsmps_build_cell_list_noalloc(None, None, None, None, 0, ctypes.byref(grid),
                                             ctypes.byref(view)) == pkg.abi.OK
    torch.cuda.synchronize()
    assert bool((out["cell_begin"] == -1).all()) and bool((out["cell_end"] == -1).all())
    x = torch.tensor([0.05, float("nan"), 0.25], dtype=torch.float64, device="cuda")
    out, view = _cells(pkg, torch, 3, 125)
    st = lib.lsmps_build_cell_list_noalloc(None, x.data_ptr(), x.data_ptr(), x.data_ptr(), 3, ctypes.byref(grid),
                                           ctypes.byref(view))
    assert st == pkg.abi.NON_FINITE


_FRESH_PROCESS = textwrap.dedent("""
    import ctypes, sys
    import numpy as np
    import torch
    sys.path.insert(0, sys.argv[1])
    import __graft_entry__ as e
    pkg = e.load_package()
    abi = pkg.abi
    lib = abi.load_library()
    case = pkg.cases.dam_break(30, 15, 30)
    f = case.fluid
    n = case.n_fluid
    grid = case.params.grid
    ncell = case.n_cells
    xyz = [torch.from_numpy(np.ascontiguousarray(f[c])).cuda() for c in "xyz"]
    out = {k: torch.full((n if k in ("cell_ids", "sorted_indices") else ncell,), -7, dtype=torch.int32,
                         device="cuda") for k in ("cell_ids", "sorted_indices", "cell_begin", "cell_end")}
    view = abi.Cells()
    view.particle_count, view.cell_count = n, ncell
    for k, v in out.items():
        setattr(view, k, v.data_ptr())
    empty = abi.Cells()
    empty.particle_count, empty.cell_count = 0, ncell
    empty.cell_begin, empty.cell_end = out["cell_begin"].data_ptr(), out["cell_end"].data_ptr()
    torch.cuda.synchronize()
    # first library call of the process: count = 0 (set-up only), then n
    st = lib.lsmps_build_cell_list_noalloc(None, None, None, None, 0, ctypes.byref(grid), ctypes.byref(empty))
    assert st == abi.OK, st
    # result copies allocated before the measurement, so that torch's
    # allocator takes no new device memory between the two readings
    results = [{k: torch.empty_like(v) for k, v in out.items()} for _ in range(3)]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for r in results:
        st = lib.lsmps_build_cell_list_noalloc(None, *[t.data_ptr() for t in xyz], n, ctypes.byref(grid),
                                               ctypes.byref(view))
        assert st == abi.OK, st
        for k, v in out.items():
            r[k].copy_(v)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, ("device memory changed across calls", free0, free1)
    sorted_ids = results[0]["cell_ids"].cpu().numpy()
    assert np.all(np.diff(sorted_ids) >= 0)
    for r in results[1:]:
        for k in r:
            assert torch.equal(r[k], results[0][k]), k
    # the same sort through the context entry point, after the fact
    from importlib import import_module
    api = import_module("lsmps3d_b200.api")
    ctx = api.Context(0)
    want = {k: torch.full_like(v, -7) for k, v in out.items()}
    wv = abi.Cells()
    wv.particle_count, wv.cell_count = n, ncell
    for k, v in want.items():
        setattr(wv, k, v.data_ptr())
    ctx.build_cell_list(*[t.data_ptr() for t in xyz], n, grid, wv)
    ctx.close()
    for k in want:
        assert torch.equal(want[k], results[0][k]), k
    print("FRESH_PROCESS_OK", free0 - free1)
""")


def test_noalloc_first_in_a_fresh_process(pkg, device_api):
    """The allocation-free entry point as the first library call of a new
    process (count = 0, then a real sort), with nothing loaded beforehand by
    a context call; the device's free memory is the same before and after
    three more calls, and the result equals the context entry point's."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FRESH_PROCESS, root], capture_output=True, text=True, timeout=600,
                       cwd=root)
    assert r.returncode == 0 and "FRESH_PROCESS_OK" in r.stdout, r.stdout[-2000:] + r.stderr[-4000:]
