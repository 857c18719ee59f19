"""Parity of the sm_100a path (through the C ABI) with the CPU oracle.

Integer outputs (sorted cell ids, sorted indices, cell ranges, CSR offsets
and rows in their native order, surface labels) must be bit-exact.  Floating
outputs are compared with the metric of rel_err below; the plain (FP64) form must stay within
PLAIN_RTOL.  The two sides differ only in operation order (FMA
contraction, multiply-by-reciprocal) and, for the moment inverse, in the
factorisation route (L^-T L^-1 versus substitution against identity columns),
so the bound is set by rounding times the moment matrices' conditioning.
"""

import os
import sys

import numpy as np
import pytest

from kat_util import buffers_from, inverse_err_over_kappa, light_ties, params_from, rel_err, rows, vec_err

pytestmark = pytest.mark.gpu

# Plain form against the FP64 oracle: every floating output within 1e-10
# (normwise against the field's scale, elementwise above 1e-3 of it); the
# largest measured is 6e-12 (PPE values of the splash case).  Moment
# inverses: within INVERSE_KAPPA_FACTOR * 2^-52 * kappa_est per particle
# (measured at most 0.4; ill-conditioned Surface matrices of the splash case
# differ by 3e-8 relative at kappa ~ 1e8).
PLAIN_RTOL = 1e-10
INVERSE_KAPPA_FACTOR = 8.0


def both(pkg, device_api, case_or_kat, kat=False, **kw):
    """Device and host StepBuffers loaded with the same input."""
    if kat:
        dev = buffers_from(pkg, pkg.buffers.TorchAlloc("cuda"), case_or_kat)
        host = buffers_from(pkg, pkg.buffers.NumpyAlloc(), case_or_kat)
    else:
        c = case_or_kat
        dev = pkg.buffers.StepBuffers(pkg.buffers.TorchAlloc("cuda"), c.n_fluid, c.n_wall, c.n_cells, **kw)
        host = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), c.n_fluid, c.n_wall, c.n_cells, **kw)
        dev.load_case(c)
        host.load_case(c)
    return dev, host


@pytest.fixture(scope="module")
def ctx(device_api):
    return device_api.Context(0)


# --- reference known-answer tests on the device -----------------------------

def test_neighbor_search_kat_gpu(pkg, device_api, ctx, oracle, kats):
    k = kats["neighbor_search"]
    dev, host = both(pkg, device_api, k, kat=True)
    p = params_from(pkg, k)
    ctx.build_neighbor_lists(dev, p)
    off, idx = dev.csr_rows("fluid")
    assert off.tolist() == k["expected_fluid_offsets"]
    assert rows(off, idx, 5) == [sorted(x) for x in k["expected_fluid_rows"]]
    off, idx = dev.csr_rows("wall")
    assert off.tolist() == k["expected_wall_offsets"]
    assert rows(off, idx, 5) == [sorted(x) for x in k["expected_wall_rows"]]
    oracle.build_neighbor_lists(host, p)
    for which in ("fluid", "wall"):
        go, gi = dev.csr_rows(which)
        ho, hi = host.csr_rows(which)
        assert np.array_equal(go, ho) and np.array_equal(gi, hi)


def test_neighbor_capacity_exceeded_gpu(pkg, device_api, ctx, kats):
    k = kats["neighbor_search"]
    dev = buffers_from(pkg, pkg.buffers.TorchAlloc("cuda"), k)
    dev.cap_f = 5
    p = params_from(pkg, k)
    with pytest.raises(device_api.LsmpsError) as e:
        ctx.build_neighbor_lists(dev, p)
    assert e.value.status == pkg.abi.CAPACITY_EXCEEDED and ctx.required == 6


def test_surface_detection_kat_gpu(pkg, device_api, ctx, kats):
    k = kats["surface_detection"]
    dev = buffers_from(pkg, pkg.buffers.TorchAlloc("cuda"), k)
    p = params_from(pkg, k)
    ctx.build_neighbor_lists(dev, p)
    ctx.classify_surface(dev, p)
    lab = dev.numpy("fluid")["surface_type"]
    for i, v in k["expected_labels_at"].items():
        assert lab[int(i)] == v


@pytest.mark.parametrize("name", ["provision", "ppe", "pressure_correction"])
def test_operator_kats_gpu(pkg, device_api, ctx, oracle, kats, name):
    k = kats[name]
    dev, host = both(pkg, device_api, k, kat=True)
    p = params_from(pkg, k)
    if name != "provision":
        for comp in ("vx", "vy", "vz"):
            dev.alloc.copy_(dev.temporary_velocity[comp], np.asarray(k["fluid"][comp]))
            host.temporary_velocity[comp][:] = np.asarray(k["fluid"][comp])
    ctx.prepare_moments(dev, p, [0, 1])
    oracle.prepare_moment(host, p, 0)
    oracle.prepare_moment(host, p, 1)
    c, tol = k["center"], k["tolerance"]
    if name == "provision":
        ctx.provision(dev, p)
        oracle.provision(host, p)
        lap = dev.numpy("velocity_laplacian")
        assert abs(lap["x"][c] - k["expected_laplacian_x_center"]) <= tol
        for comp in ("vx", "vy", "vz"):
            assert rel_err(dev.numpy("temporary_velocity")[comp], host.temporary_velocity[comp]) < PLAIN_RTOL
    elif name == "ppe":
        ctx.assemble_ppe(dev, p)
        oracle.assemble_ppe(host, p)
        ppe = dev.numpy("ppe")
        assert abs(ppe["divergence"][c] - k["expected_divergence_center"]) <= tol
        assert abs(ppe["rhs"][c] - k["expected_rhs_center"]) <= tol
        assert np.array_equal(ppe["row_offsets"], host.ppe["row_offsets"])
        assert np.array_equal(ppe["col_indices"], host.ppe["col_indices"])
        assert rel_err(ppe["values"], host.ppe["values"]) < PLAIN_RTOL
    else:
        ctx.pressure_correction(dev, p)
        oracle.pressure_correction(host, p)
        g = dev.numpy("pressure_gradient")
        assert np.allclose([g[a][c] for a in "xyz"], k["expected_gradient_center"], atol=tol)
        f = dev.numpy("fluid")
        for comps in (("x", "y", "z"), ("vx", "vy", "vz")):
            for comp, e in vec_err(f, host.fluid, comps).items():
                assert e < PLAIN_RTOL, (comp, e)


# --- full pipeline on seeded synthetic cases ---------------------------------

CASES = [
    ("hydrostatic", dict(n=20, l0=0.01)),
    ("dam_break", dict(nx=24, ny=12, nz=24, l0=0.005)),
    ("splash", dict(nx=40, ny=10, nz=40, l0=0.0025)),
    # the same dam break with the fluid numbered in random order
    ("dam_break_shuffled", dict(nx=24, ny=12, nz=24, l0=0.005)),
]


@pytest.fixture(scope="module", params=CASES, ids=[c[0] for c in CASES])
def pipeline(request, pkg, device_api, ctx, oracle):
    """Run each stage on both sides from the same inputs; return both buffer
    sets after every stage has been compared."""
    name, kw = request.param
    case = pkg.cases.CASES[name](**kw)
    p = case.params
    dev, host = both(pkg, device_api, case)
    ctx.build_neighbor_lists(dev, p)
    st, req = oracle.build_neighbor_lists(host, p)
    assert st == 0
    return case, dev, host


def test_cells_bit_exact(pipeline):
    case, dev, host = pipeline
    for which in ("fluid_cells", "wall_cells"):
        g, h = dev.numpy(which), host.numpy(which)
        for k in ("cell_ids", "sorted_indices", "cell_begin", "cell_end"):
            assert np.array_equal(g[k], h[k]), (which, k)


def test_csr_bit_exact_native_order(pipeline):
    case, dev, host = pipeline
    for which in ("fluid", "wall"):
        go, gi = dev.csr_rows(which)
        ho, hi = host.csr_rows(which)
        assert np.array_equal(go, ho), which
        assert np.array_equal(gi, hi), which


@pytest.mark.parametrize("walls", [1, 0], ids=["with_walls", "fluid_only"])
def test_virtual_light_matches_oracle(pkg, device_api, pipeline, ctx, oracle, walls):
    # Open-direction counts are integers: bit-exact, except where a
    # neighbour's projection lies within 1e-12 of the cone cosine (lattice
    # vectors at exactly 30 degrees to a light direction): there the answer
    # depends on the projection's last bits, which the oracle (no FMA
    # contraction, 1/sqrt) need not share with the device (the reference's own
    # expression and rsqrt; bit-exact against the reference in
    # test_gpu_reference.py).  Such particles may differ by at most their
    # number of tied directions.
    import torch

    case, dev, host = pipeline
    p = type(case.params).from_buffer_copy(case.params)
    p.include_wall_neighbors = walls
    n = case.n_fluid
    count = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    frac = torch.full((n,), -1.0, dtype=torch.float64, device="cuda")
    ctx.virtual_light(dev, p, count.data_ptr(), frac.data_ptr())
    hc = np.zeros(n, np.int32)
    hf = np.zeros(n, np.float64)
    assert oracle.virtual_light(host, p, hc, hf) == 0
    gc = count.cpu().numpy()
    ties = light_ties(host, p)
    clear = ties == 0
    assert np.array_equal(gc[clear], hc[clear]), np.flatnonzero(clear & (gc != hc))[:10]
    assert np.all(np.abs(gc - hc) <= ties)
    print(f"{case.name} walls={walls}: {int((~clear).sum())} particles with a tied direction, "
          f"{int((gc != hc).sum())} differ from the oracle")
    assert np.array_equal(frac.cpu().numpy(), gc / 14.0)
    print(f"{case.name} walls={walls}: open directions histogram {np.bincount(gc, minlength=15).tolist()}")
    # count only
    c2 = torch.zeros((n,), dtype=torch.int32, device="cuda")
    ctx.virtual_light(dev, p, c2.data_ptr(), None)
    assert torch.equal(c2, count)
    with pytest.raises(device_api.LsmpsError):
        ctx.virtual_light(dev, p, None, None)


def test_pipeline_stages_match_oracle(pkg, pipeline, ctx, oracle):
    case, dev, host = pipeline
    p = case.params
    # labels
    ctx.classify_surface(dev, p)
    assert oracle.classify_surface(host, p) == 0
    assert np.array_equal(dev.numpy("fluid")["surface_type"], host.fluid["surface_type"])
    # moments (velocity Dirichlet-A and pressure Neumann-A, fused on the device)
    ctx.prepare_moments(dev, p, [0, 1])
    for kind in (0, 1):
        assert oracle.prepare_moment(host, p, kind) == 0
        gm = {k: dev.alloc.to_numpy(v) for k, v in dev.moments[kind].items()}
        hm = host.moments[kind]
        assert np.array_equal(gm["info"], hm["info"])
        assert gm["inversion_count"][0] >= 1
        assert rel_err(gm["moment_trace"], hm["moment_trace"]) < 1e-12
        ok = hm["info"] == 0
        gi = gm["inverse_matrices"].reshape(-1, 81)[ok]
        hi = hm["inverse_matrices"].reshape(-1, 81)[ok]
        per = np.max(np.abs(gi - hi), axis=1) / np.max(np.abs(hi), axis=1)
        ek = inverse_err_over_kappa(gi, hi, hm["moment_trace"][ok], hm["regularization_added"][ok])
        print(f"{case.name} kind {kind}: inverse max rel err {per.max():.3e} median {np.median(per):.3e}; "
              f"max over eps kappa {ek:.3f}")
        assert ek < INVERSE_KAPPA_FACTOR
    # provision
    ctx.provision(dev, p)
    oracle.provision(host, p)
    for comp in ("vx", "vy", "vz"):
        e = rel_err(dev.numpy("temporary_velocity")[comp], host.temporary_velocity[comp])
        assert e < PLAIN_RTOL, (comp, e)
    # PPE
    ctx.assemble_ppe(dev, p)
    oracle.assemble_ppe(host, p)
    g = dev.numpy("ppe")
    nnz = int(host.ppe["row_offsets"][-1])
    assert np.array_equal(g["row_offsets"], host.ppe["row_offsets"])
    assert np.array_equal(g["col_indices"][:nnz], host.ppe["col_indices"][:nnz])
    for k in ("values", "rhs", "divergence", "pressure_laplacian"):
        a, b = (g[k][:nnz], host.ppe[k][:nnz]) if k == "values" else (g[k], host.ppe[k])
        e = rel_err(a, b)
        print(f"{case.name} ppe {k}: max rel err {e:.3e}")
        assert e < PLAIN_RTOL, (k, e)
    # correction (pressure = clamped fluid.pressure, in place)
    ctx.pressure_correction(dev, p)
    oracle.pressure_correction(host, p)
    f = dev.numpy("fluid")
    # The corrected velocity is u* - dt/rho grad p, which cancels almost
    # exactly in hydrostatic balance: its error scale is |u*|.
    errs = {**vec_err(f, host.fluid, ("x", "y", "z")),
            **vec_err(f, host.fluid, ("vx", "vy", "vz"), extra_scale=host.temporary_velocity),
            "pressure": rel_err(f["pressure"], host.fluid["pressure"])}
    for comp, e in errs.items():
        print(f"{case.name} corrected {comp}: max rel err {e:.3e}")
        assert e < PLAIN_RTOL, (comp, e)


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_full_step_matches_oracle(pkg, device_api, ctx, oracle, name, kw):
    """lsmps_step == the oracle's step on the same state (geometry rebuilt
    first on both sides so both start from identical CSR and labels)."""
    case = pkg.cases.CASES[name](**kw)
    p = case.params
    dev, host = both(pkg, device_api, case)
    ctx.build_neighbor_lists(dev, p)
    ctx.classify_surface(dev, p)
    oracle.build_neighbor_lists(host, p)
    oracle.classify_surface(host, p)
    ctx.step(dev, p)
    st, _ = oracle.step(host, p)
    assert st == 0
    assert np.array_equal(dev.numpy("fluid")["surface_type"], host.fluid["surface_type"])
    for which in ("fluid", "wall"):
        go, gi = dev.csr_rows(which)
        ho, hi = host.csr_rows(which)
        assert np.array_equal(go, ho) and np.array_equal(gi, hi)
    f = dev.numpy("fluid")
    for comps in (("x", "y", "z"), ("vx", "vy", "vz")):
        for comp, e in vec_err(f, host.fluid, comps, extra_scale=host.temporary_velocity).items():
            print(f"{name} step {comp}: max rel err {e:.3e}")
            assert e < PLAIN_RTOL, (comp, e)


KNOB_VARIANTS = [(0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 2), (1, 3), (2, 0), (2, 1), (2, 2)]


@pytest.mark.parametrize("knob,value", KNOB_VARIANTS, ids=[f"knob{k}={v}" for k, v in KNOB_VARIANTS])
def test_launch_variants_match_oracle(pkg, device_api, oracle, knob, value):
    """Every launch-shape variant (lsmps_knob) computes the oracle's moments
    and PPE system: splash case, so Dirichlet rows and Splash particles are
    in it."""
    case = pkg.cases.CASES["splash"](nx=40, ny=10, nz=40, l0=0.0025)
    p = case.params
    dev, host = both(pkg, device_api, case)
    c = device_api.Context(0)
    try:
        c.set_knob(knob, value)
        assert c.knob(knob) == value
        c.build_neighbor_lists(dev, p)
        c.classify_surface(dev, p)
        c.prepare_moments(dev, p, [0, 1])
        c.provision(dev, p)
        c.assemble_ppe(dev, p)
    finally:
        c.close()
    assert oracle.build_neighbor_lists(host, p)[0] == 0
    assert oracle.classify_surface(host, p) == 0
    assert np.array_equal(dev.numpy("fluid")["surface_type"], host.fluid["surface_type"])
    for kind in (0, 1):
        assert oracle.prepare_moment(host, p, kind) == 0
        gm = {k: dev.alloc.to_numpy(v) for k, v in dev.moments[kind].items()}
        hm = host.moments[kind]
        assert np.array_equal(gm["info"], hm["info"])
        ok = hm["info"] == 0
        gi = gm["inverse_matrices"].reshape(-1, 81)[ok]
        hi = hm["inverse_matrices"].reshape(-1, 81)[ok]
        assert inverse_err_over_kappa(gi, hi, hm["moment_trace"][ok], hm["regularization_added"][ok]) < \
            INVERSE_KAPPA_FACTOR
    oracle.provision(host, p)
    oracle.assemble_ppe(host, p)
    g = dev.numpy("ppe")
    nnz = int(host.ppe["row_offsets"][-1])
    assert np.array_equal(g["row_offsets"], host.ppe["row_offsets"])
    assert np.array_equal(g["col_indices"][:nnz], host.ppe["col_indices"][:nnz])
    for k in ("values", "rhs", "divergence", "pressure_laplacian"):
        a, b = (g[k][:nnz], host.ppe[k][:nnz]) if k == "values" else (g[k], host.ppe[k])
        e = rel_err(a, b)
        print(f"knob {knob}={value} ppe {k}: max rel err {e:.3e}")
        assert e < PLAIN_RTOL, k


def test_autotune_leaves_state_and_picks_valid_variants(pkg, device_api):
    case = pkg.cases.dam_break(nx=24, ny=12, nz=24, l0=0.005)
    p = case.params
    dev = device_api.device_buffers(case)
    c = device_api.Context(0)
    try:
        c.build_neighbor_lists(dev, p)
        c.classify_surface(dev, p)
        c.step(dev, p)
        before = {k: v.copy() for k, v in dev.numpy("fluid").items()}
        rows_before = dev.csr_rows("fluid")
        for prec in (pkg.abi.PRECISION_PLAIN, pkg.abi.PRECISION_MIXED):
            c.set_precision(prec)
            tuned = c.autotune(dev, p, repeats=2)
            lib = device_api._lib
            for k, (v, ms) in tuned.items():
                assert 0 <= v < lib.lsmps_knob_variants(k) and ms > 0.0
        after = dev.numpy("fluid")
        for k in before:
            assert np.array_equal(before[k], after[k]), k
        ro, ri = dev.csr_rows("fluid")
        assert np.array_equal(ro, rows_before[0]) and np.array_equal(ri, rows_before[1])
    finally:
        c.close()


@pytest.mark.parametrize("lanes", [1, 2], ids=["gather2", "gather4"])
def test_gather_lanes_step_matches_oracle(pkg, device_api, oracle, lanes):
    """The lane-parallel velocity-Laplacian and smoothing passes against the
    oracle's step, on a moving fluid (so both passes do real work)."""
    case = pkg.cases.CASES["dam_break"](nx=24, ny=12, nz=24, l0=0.005)
    f = case.fluid
    f["vx"] = 0.1 * np.sin(f["x"] / 0.12)
    f["vy"] = 0.1 * np.cos(f["y"] / 0.12)
    f["vz"] = 0.1 * f["z"] / 0.12
    p = case.params
    dev, host = both(pkg, device_api, case)
    c = device_api.Context(0)
    try:
        c.set_knob(pkg.abi.KNOB_GATHER_LANES, lanes)
        c.build_neighbor_lists(dev, p)
        c.classify_surface(dev, p)
        c.step(dev, p)
    finally:
        c.close()
    oracle.build_neighbor_lists(host, p)
    oracle.classify_surface(host, p)
    assert oracle.step(host, p)[0] == 0
    lap = vec_err(dev.numpy("velocity_laplacian"), host.numpy("velocity_laplacian"), ("x", "y", "z"))
    g = dev.numpy("fluid")
    state = {**vec_err(g, host.fluid, ("x", "y", "z")), **vec_err(g, host.fluid, ("vx", "vy", "vz"))}
    for k, e in {**lap, **state}.items():
        assert e < PLAIN_RTOL, (k, e)


@pytest.mark.parametrize("precision", [0, 1], ids=["plain", "mixed"])
def test_cell_visiting_order_changes_no_result(pkg, device_api, precision):
    # lsmps_step visits the fluid in cell order when the context built the
    # state's cell list; every output must equal the index-order step's, bit
    # for bit (on the randomly numbered dam break, where the two orders differ most).
    case = pkg.cases.CASES["dam_break_shuffled"](nx=24, ny=12, nz=24, l0=0.005)
    p = case.params
    out = []
    for cell_order in (False, True):
        c = device_api.Context(0)
        c.set_precision(precision)
        c.set_cell_order(cell_order)
        dev = device_api.device_buffers(case)
        c.build_neighbor_lists(dev, p)
        c.classify_surface(dev, p)
        for _ in range(2):
            c.step(dev, p)
        snap = {f"fluid.{k}": v for k, v in dev.numpy("fluid").items()}
        snap.update({f"ppe.{k}": v for k, v in dev.numpy("ppe").items()})
        for name in ("pressure_gradient", "ps_displacement", "velocity_laplacian"):
            snap.update({f"{name}.{k}": v for k, v in dev.numpy(name).items()})
        out.append(snap)
        c.close()
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k


def test_knob_arguments_checked(device_api):
    c = device_api.Context(0)
    try:
        with pytest.raises(device_api.LsmpsError):
            c.set_knob(2, 3)
        with pytest.raises(device_api.LsmpsError):
            c.set_knob(7, 0)
        assert c.knob(0) == 1 and c.knob(1) == 1 and c.knob(2) == 2
    finally:
        c.close()


def test_deterministic_repeat(pkg, device_api, ctx):
    case = pkg.cases.dam_break(nx=16, ny=8, nz=16, l0=0.005)
    outs = []
    for _ in range(2):
        dev = device_api.device_buffers(case)
        ctx.build_neighbor_lists(dev, case.params)
        ctx.classify_surface(dev, case.params)
        ctx.step(dev, case.params)
        outs.append((dev.csr_rows("fluid"), dev.numpy("fluid")))
    (o0, f0), (o1, f1) = outs
    assert np.array_equal(o0[0], o1[0]) and np.array_equal(o0[1], o1[1])
    for k in f0:
        assert np.array_equal(f0[k], f1[k]), k


# --- edge cases ---------------------------------------------------------------

def test_empty_fluid(pkg, device_api, ctx):
    case = pkg.cases.hydrostatic_box(n=4)
    p = case.params
    b = pkg.buffers.StepBuffers(pkg.buffers.TorchAlloc("cuda"), 0, case.n_wall, case.n_cells)
    b.load_case(type(case)(case.name, case.l0, {k: v[:0] for k, v in case.fluid.items()}, case.walls, p))
    ctx.build_neighbor_lists(b, p)
    assert b.csr_rows("fluid")[0].tolist() == [0]
    ctx.classify_surface(b, p)
    ctx.step(b, p)


def test_non_finite_coordinate_reported(pkg, device_api, ctx):
    case = pkg.cases.hydrostatic_box(n=6)
    case.fluid["x"][3] = np.nan
    dev = device_api.device_buffers(case)
    with pytest.raises(device_api.LsmpsError) as e:
        ctx.build_neighbor_lists(dev, case.params)
    assert e.value.status == pkg.abi.NON_FINITE


def test_overloaded_and_out_of_grid_cells(pkg, device_api, ctx, oracle):
    """Particles outside the grid are clamped into edge cells
    (neighbor_search.cu:36-46); an edge cell holding more candidates than the
    shared-memory stage takes the exact global-memory path.  Rows must still
    match the oracle bit for bit."""
    rng = np.random.default_rng(11)
    case = pkg.cases.hydrostatic_box(n=10, l0=0.01)
    n = case.n_fluid
    # pile 1500 particles just outside the low x face (clamped into cells at ix = 0)
    k = 1500
    extra = {c: np.asarray(v) for c, v in case.fluid.items()}
    ox = case.params.grid.origin[0]
    add = {"x": ox - 0.004 - rng.random(k) * 0.002, "y": 0.02 + rng.random(k) * 0.004,
           "z": 0.02 + rng.random(k) * 0.004}
    fluid = {}
    for c, v in extra.items():
        if c in add:
            fluid[c] = np.concatenate([v, add[c]])
        else:
            fluid[c] = np.concatenate([v, np.zeros(k, dtype=v.dtype)])
    big = type(case)(case.name, case.l0, fluid, case.walls, case.params)
    dev, host = both(pkg, device_api, big, max_fluid_neighbors=2048, max_wall_neighbors=256)
    ctx.build_neighbor_lists(dev, big.params)
    oracle.build_neighbor_lists(host, big.params)
    for which in ("fluid", "wall"):
        go, gi = dev.csr_rows(which)
        ho, hi = host.csr_rows(which)
        assert np.array_equal(go, ho) and np.array_equal(gi, hi)
    assert n + k == big.n_fluid


@pytest.mark.parametrize("radius_l0", [2.0, 3.0, 6.0 ** 0.5])
def test_csr_pairs_at_the_radius(pkg, device_api, ctx, oracle, radius_l0):
    """An unjittered lattice with the support radius equal to a lattice
    distance (2 l0, 3 l0 = |(2,2,1)| l0, sqrt(6) l0 = |(2,1,1)| l0): many
    pairs lie within rounding of r, where the FP32 screen must hand over to
    the reference's FP64 test.  Rows must match the oracle, and the
    reference's own CUDA path where it is built, bit for bit."""
    case = pkg.cases.hydrostatic_box(n=12, l0=0.01)
    p = case.params
    p.support_radius = radius_l0 * case.l0
    p.grid.cell_size = p.support_radius
    pkg.cases.derive_grid(p, [case.fluid["x"], case.walls["x"]], [case.fluid["y"], case.walls["y"]],
                          [case.fluid["z"], case.walls["z"]])
    dev, host = both(pkg, device_api, case, max_fluid_neighbors=256, max_wall_neighbors=256)
    ctx.build_neighbor_lists(dev, p)
    oracle.build_neighbor_lists(host, p)
    for which in ("fluid", "wall"):
        go, gi = dev.csr_rows(which)
        ho, hi = host.csr_rows(which)
        assert np.array_equal(go, ho) and np.array_equal(gi, hi), which
    # the reference's own CUDA path decides the ties the same way (its device
    # distance test contracts into fused multiply-adds, as the oracle states)
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import reference as ref_mod

    if ref_mod.available():
        rb = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), case.n_fluid, case.n_wall, case.n_cells,
                                     max_fluid_neighbors=256, max_wall_neighbors=256)
        rb.load_case(case)
        ref = ref_mod.ReferencePath(pkg.abi, case, rb, 256, 256)
        ref.rebuild()
        ref.fetch_geometry()
        for which in ("fluid", "wall"):
            go, gi = dev.csr_rows(which)
            ro, ri = rb.csr_rows(which)
            assert np.array_equal(go, ro) and np.array_equal(gi, ri), ("reference", which)


def test_cell_list_random_keys_stable(pkg, device_api, ctx, oracle):
    """Radix passes over many digits: random positions on a large grid."""
    rng = np.random.default_rng(5)
    n = 300_000
    grid = pkg.abi.Grid()
    grid.origin[:] = (0.0, 0.0, 0.0)
    grid.cell_size = 0.01
    grid.dims[:] = (180, 160, 150)  # 4.32M cells: 23-bit keys, 3 radix passes
    x, y, z = (rng.random(n) * d * 0.01 for d in (180, 160, 150))
    import torch

    t = {c: torch.from_numpy(v).cuda() for c, v in zip("xyz", (x, y, z))}
    ncell = 180 * 160 * 150
    out = {k: torch.zeros(n if k in ("cell_ids", "sorted_indices") else ncell, dtype=torch.int32, device="cuda")
           for k in ("cell_ids", "sorted_indices", "cell_begin", "cell_end")}
    cv = pkg.abi.Cells()
    cv.particle_count, cv.cell_count = n, ncell
    for k, v in out.items():
        setattr(cv, k, v.data_ptr())
    ctx.build_cell_list(t["x"].data_ptr(), t["y"].data_ptr(), t["z"].data_ptr(), n, grid, cv)
    host = {k: np.zeros(v.numel(), np.int32) for k, v in out.items()}
    hv = pkg.abi.Cells()
    hv.particle_count, hv.cell_count = n, ncell
    for k, v in host.items():
        setattr(hv, k, v.ctypes.data)
    assert oracle.build_cell_list(x, y, z, grid, hv) == 0
    for k in out:
        assert np.array_equal(out[k].cpu().numpy(), host[k]), k
