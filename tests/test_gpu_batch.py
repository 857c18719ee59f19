"""Batched boxes in one captured CUDA graph (lsmps_batch_*): every box after
one graph launch equals the same box stepped alone by lsmps_step (same
kernels on the same inputs, so bit-identical), in both precision forms."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1], ids=["plain", "mixed"])
def test_graph_batch_matches_sequential_steps(pkg, device_api, precision):
    boxes = pkg.cases.batched_boxes(count=6, seed=11, n_min=2_000, n_max=20_000)
    bufs, refs = [], []
    for case in boxes:
        p = case.params
        b = device_api.device_buffers(case)
        r = device_api.device_buffers(case)
        c = device_api.Context(0)
        try:
            for x in (b, r):
                c.build_neighbor_lists(x, p)
                c.classify_surface(x, p)
            c.set_precision(precision)
            c.step(r, p)  # the reference: this box stepped alone
        finally:
            c.close()
        bufs.append((b, p))
        refs.append(r)
    batch = device_api.Batch(0, streams=3)
    try:
        for b, p in bufs:
            batch.add(b, p)
        # default launch shapes, as in the solo steps (the autotuner may pick
        # lane counts that reassociate sums at the rounding level)
        batch.capture(precision=precision, autotune_repeats=0)
        batch.launch()
        batch.synchronize()
    finally:
        batch.close()
    for (b, _), r, case in zip(bufs, refs, boxes):
        got, want = b.numpy("fluid"), r.numpy("fluid")
        for k in want:
            assert np.array_equal(got[k], want[k]), (case.name, k)
        for which in ("fluid", "wall"):
            go, gi = b.csr_rows(which)
            ro, ri = r.csr_rows(which)
            assert np.array_equal(go, ro) and np.array_equal(gi, ri), (case.name, which)


@pytest.mark.parametrize("precision", [0, 1], ids=["plain", "mixed"])
def test_graph_batch_64_boxes_matches_solo_steps(pkg, device_api, precision):
    """The batched workload itself: 64 boxes with fluid counts log-uniform in
    [8k, 200k] (seed 7), hydrostatic or dam-break layout by seeded coin flip,
    3 wall layers, stepped by one graph over 8 worker streams; every box
    equals the same box stepped alone by lsmps_step, bit for bit."""
    boxes = pkg.cases.batched_boxes()
    assert len(boxes) == 64
    bufs, refs = [], []
    c = device_api.Context(0)
    try:
        c.set_precision(precision)
        for case in boxes:
            p = case.params
            b = device_api.device_buffers(case)
            r = device_api.device_buffers(case)
            for x in (b, r):
                c.build_neighbor_lists(x, p)
                c.classify_surface(x, p)
            c.step(r, p)
            bufs.append((b, p))
            refs.append(r)
    finally:
        c.close()
    batch = device_api.Batch(0, streams=8)
    try:
        for b, p in bufs:
            batch.add(b, p)
        batch.capture(precision=precision, autotune_repeats=0)
        batch.launch()
        batch.synchronize()
    finally:
        batch.close()
    for (b, _), r, case in zip(bufs, refs, boxes):
        got, want = b.numpy("fluid"), r.numpy("fluid")
        for k in want:
            assert np.array_equal(got[k], want[k]), (case.name, k)
        for which in ("fluid", "wall"):
            go, gi = b.csr_rows(which)
            ro, ri = r.csr_rows(which)
            assert np.array_equal(go, ro) and np.array_equal(gi, ri), (case.name, which)
        gp, rp = b.numpy("ppe"), r.numpy("ppe")
        nnz = int(rp["row_offsets"][-1])
        for k in ("row_offsets", "rhs", "divergence"):
            assert np.array_equal(gp[k], rp[k]), (case.name, k)
        assert np.array_equal(gp["values"][:nnz], rp["values"][:nnz]), case.name
        assert np.array_equal(gp["col_indices"][:nnz], rp["col_indices"][:nnz]), case.name


def test_merged_batch_reports_a_box_over_its_own_capacity(pkg, device_api):
    """A box whose own neighbour tables and PPE matrix are too small for its
    rows (the merged set's tables, the sum of the boxes', are large enough):
    the launch reports LSMPS_CAPACITY_EXCEEDED, writes nothing past that box's
    capacities (guard entries beyond them keep their fill), and the other
    boxes still equal their solo steps."""
    import torch

    boxes = pkg.cases.batched_boxes(count=3, seed=5, n_min=2_000, n_max=6_000)
    small = 1
    bufs, refs = [], {}
    c = device_api.Context(0)
    try:
        c.set_precision(1)
        for k, case in enumerate(boxes):
            p = case.params
            b = device_api.device_buffers(case)
            if k == small:
                # views 16 entries per particle wide over the full-size arrays;
                # everything past them is a guard
                b.cap_f = 16 * case.n_fluid
                b.nnz_cap = case.n_fluid + b.cap_f
                b.fluid_neighbors["indices"][b.cap_f:] = -7
                b.ppe["col_indices"][b.nnz_cap:] = -7
            else:
                c.build_neighbor_lists(b, p)
                c.classify_surface(b, p)
                r = device_api.device_buffers(case)
                c.build_neighbor_lists(r, p)
                c.classify_surface(r, p)
                c.step(r, p)
                refs[k] = r
            bufs.append((b, p))
    finally:
        c.close()
    torch.cuda.synchronize()
    batch = device_api.Batch(0, streams=3)
    try:
        for b, p in bufs:
            batch.add(b, p)
        batch.capture(precision=1, autotune_repeats=0)
        assert batch.merged
        batch.launch()
        with pytest.raises(device_api.LsmpsError) as err:
            batch.synchronize()
        assert err.value.status == pkg.abi.CAPACITY_EXCEEDED, err.value
    finally:
        batch.close()
    b = bufs[small][0]
    assert torch.all(b.fluid_neighbors["indices"][b.cap_f:] == -7)
    assert torch.all(b.ppe["col_indices"][b.nnz_cap:] == -7)
    for k, r in refs.items():
        got, want = bufs[k][0].numpy("fluid"), r.numpy("fluid")
        for name in want:
            assert np.array_equal(got[name], want[name]), (k, name)
