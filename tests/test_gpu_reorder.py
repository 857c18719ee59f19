"""lsmps_reorder_fluid: renumbering the fluid in cell order leaves the step's
results unchanged up to the renumbering, bit for bit (the rebuilt rows list
the same neighbours in the same order), and validates its arguments."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "pressure", "surface_type")


def test_reordered_step_equals_renumbered_step(pkg, device_api):
    import torch

    case = pkg.cases.CASES["dam_break_shuffled"](nx=24, ny=12, nz=24, l0=0.005)
    p = case.params
    ctx = device_api.Context(0)
    # A: the step on the shuffled numbering
    a = device_api.device_buffers(case)
    ctx.build_neighbor_lists(a, p)
    ctx.classify_surface(a, p)
    before = a.numpy("fluid")
    ao, ai = a.csr_rows("fluid")  # the rows the step starts from
    ctx.step(a, p)
    fa = a.numpy("fluid")
    # B: renumber in cell order, rebuild the rows, step
    b = device_api.device_buffers(case)
    ctx.build_neighbor_lists(b, p)
    ctx.classify_surface(b, p)
    perm_t = torch.empty(case.n_fluid, dtype=torch.int32, device="cuda")
    ctx.reorder_fluid(b, perm_t.data_ptr())
    perm = perm_t.cpu().numpy()
    assert np.array_equal(np.sort(perm), np.arange(case.n_fluid))
    renumbered = b.numpy("fluid")
    for k in FIELDS:
        assert np.array_equal(renumbered[k], before[k][perm]), k
    # the new numbering follows the cells: sorted cell ids are ascending
    ctx.build_neighbor_lists(b, p)
    cells = b.numpy("fluid_cells")
    assert np.array_equal(cells["sorted_indices"], np.arange(case.n_fluid))
    bo, bi = b.csr_rows("fluid")
    inv = np.empty_like(perm)
    inv[perm] = np.arange(case.n_fluid)
    # row k of B is row perm[k] of A under the new numbers, in the same order
    for k in range(0, case.n_fluid, 97):
        row_a = ai[ao[perm[k]]:ao[perm[k] + 1]]
        assert np.array_equal(bi[bo[k]:bo[k + 1]], inv[row_a]), k
    ctx.step(b, p)
    fb = b.numpy("fluid")
    for k in FIELDS:
        assert np.array_equal(fb[k], fa[k][perm]), k
    with pytest.raises(device_api.LsmpsError):
        bad = b.cells_view("fluid")
        bad.particle_count = case.n_fluid - 1
        st = device_api._lib.lsmps_reorder_fluid(ctx.h, __import__("ctypes").byref(b.fluid_view()),
                                                 __import__("ctypes").byref(bad), None)
        ctx.check(st)
    ctx.close()
