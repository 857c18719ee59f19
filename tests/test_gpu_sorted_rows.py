"""Cell-sorted rows (lsmps_ctx_set_sorted_rows): lsmps_step's gathers reading
the table's sorted-position rows and records packed in cell order give the
same states, bit for bit, as the gathers reading the CSR indices and records
in index order, in both precision forms, over several steps (each step
rebuilds the tables and the sorted rows), on lattice-numbered and randomly
numbered fluid, including the FP64-route particles of the scattered splash
case.  The sorted rows themselves are checked against the table: entry e of
particle i's row is the sorted position of the neighbour fi[e].  Tolerance
zero for every output."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "pressure", "surface_type")
CASES = [
    ("dam_break", dict(nx=24, ny=12, nz=24, l0=0.005)),
    ("dam_break_shuffled", dict(nx=24, ny=12, nz=24, l0=0.005)),
    ("splash_scattered", dict(nx=40, ny=10, nz=40, l0=0.005)),
]


def run(pkg, api, case, precision, sorted_rows, steps):
    import torch

    p = case.params
    dev = api.device_buffers(case)
    ctx = api.Context(0, precision=precision)
    ctx.set_sorted_rows(sorted_rows)
    ctx.build_neighbor_lists(dev, p)
    ctx.classify_surface(dev, p)
    state = dev.step_state(p)
    for _ in range(steps):
        ctx.step(dev, p, state)
    ctx.synchronize()
    torch.cuda.synchronize()
    out = dev.numpy("fluid")
    rows = dev.csr_rows("fluid")
    extra = {}
    if precision == pkg.abi.PRECISION_MIXED:
        extra["fallbacks"] = ctx.fp64_fallbacks
    ctx.close()
    return out, rows, extra


@pytest.mark.parametrize("name,kw", CASES)
@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_sorted_rows_change_no_result(pkg, device_api, name, kw, form):
    prec = pkg.abi.PRECISION_PLAIN if form == "plain" else pkg.abi.PRECISION_MIXED
    case = pkg.cases.CASES[name](**kw)
    a, rows_a, ea = run(pkg, device_api, case, prec, True, steps=3)
    b, rows_b, eb = run(pkg, device_api, case, prec, False, steps=3)
    for k in FIELDS:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(rows_a[0], rows_b[0]) and np.array_equal(rows_a[1], rows_b[1])
    assert ea == eb
    if name == "splash_scattered" and form == "mixed":
        assert ea["fallbacks"] > 0  # the FP64-route lists were exercised


def test_sorted_rows_are_the_tables_sorted_positions(pkg, device_api):
    import torch

    case = pkg.cases.CASES["dam_break_shuffled"](nx=20, ny=10, nz=20, l0=0.005)
    p = case.params
    dev = device_api.device_buffers(case)
    ctx = device_api.Context(0)
    ctx.build_neighbor_lists(dev, p)
    torch.cuda.synchronize()
    offsets, indices = dev.csr_rows("fluid")
    sorted_idx = dev.numpy("fluid_cells")["sorted_indices"][: case.n_fluid]
    rank = np.empty(case.n_fluid, dtype=np.int64)
    rank[sorted_idx] = np.arange(case.n_fluid)
    spos = ctx.sorted_rows(int(offsets[-1]))
    assert np.array_equal(spos, rank[indices[: offsets[-1]]])
    ctx.close()
