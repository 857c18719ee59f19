"""The CPU oracle pinned against the reference's own known answers
(tests/unit/*.cu of lsmps-3D, restated in golden/reference_kats.json) and
against analytic properties the reference's diagnostics print."""

import numpy as np
import pytest

from kat_util import buffers_from, params_from, rows


def test_reference_number_density_lattice(oracle):
    # 122 lattice neighbours inside r_e = 3.1 l0 sum to n0 = 29.993
    # (compute_uniform_reference_number_density, surface_detection.cu:494-520).
    n0 = oracle.reference_number_density(0.01, 0.031)
    assert abs(n0 - 29.993) < 5e-4
    assert oracle.reference_number_density(0.0, 1.0) < 0


def test_neighbor_search_kat(pkg, oracle, kats):
    k = kats["neighbor_search"]
    b = buffers_from(pkg, pkg.buffers.NumpyAlloc(), k)
    p = params_from(pkg, k)
    st, req = oracle.build_neighbor_lists(b, p)
    assert st == 0
    off, idx = b.csr_rows("fluid")
    assert off.tolist() == k["expected_fluid_offsets"]
    assert rows(off, idx, 5) == [sorted(r) for r in k["expected_fluid_rows"]]
    off, idx = b.csr_rows("wall")
    assert off.tolist() == k["expected_wall_offsets"]
    assert rows(off, idx, 5) == [sorted(r) for r in k["expected_wall_rows"]]
    assert req == (6, 5)


def test_neighbor_search_capacity_exceeded(pkg, oracle, kats):
    k = dict(kats["neighbor_search"])
    b = buffers_from(pkg, pkg.buffers.NumpyAlloc(), k)
    b.cap_f = 5  # one short of the 6 fluid entries
    p = params_from(pkg, k)
    st, req = oracle.build_neighbor_lists(b, p)
    assert st == pkg.abi.CAPACITY_EXCEEDED and req[0] == 6


def test_surface_detection_kat(pkg, oracle, kats):
    k = kats["surface_detection"]
    b = buffers_from(pkg, pkg.buffers.NumpyAlloc(), k)
    p = params_from(pkg, k)
    st, _ = oracle.build_neighbor_lists(b, p)
    assert st == 0
    a = pkg.buffers.NumpyAlloc()
    diag_arrays = {n: a.zeros(8, "f64") for n in ("number_density", "number_density_ratio", "anisotropy",
                                                   "air_open_ratio", "air_anisotropy")}
    d = pkg.abi.SurfaceDiagnostics()
    for n, arr in diag_arrays.items():
        setattr(d, n, a.ptr(arr))
    assert oracle.classify_surface(b, p, d) == 0
    labels = b.fluid["surface_type"]
    for i, lab in k["expected_labels_at"].items():
        assert labels[int(i)] == lab, (i, labels.tolist())
    # smoke_surface_detection.cu:228-236
    n0 = oracle.reference_number_density(p.particle_spacing, p.support_radius)
    nd, ratio, an = diag_arrays["number_density"], diag_arrays["number_density_ratio"], diag_arrays["anisotropy"]
    assert abs(ratio[1] - nd[1] / n0) < 1e-5
    assert ratio[0] > ratio[1] and an[1] > an[0]
    assert diag_arrays["air_open_ratio"][1] > 0 and diag_arrays["air_anisotropy"][1] > 0


def test_virtual_light_kat(pkg, oracle, kats):
    # smoke_surface_detection.cu:238-264: the particle at the edge of the
    # cluster sees more open directions than the centre one, and the isolated
    # particle 6 sees (almost) all of them.
    k = kats["surface_detection"]
    b = buffers_from(pkg, pkg.buffers.NumpyAlloc(), k)
    p = params_from(pkg, k)
    assert oracle.build_neighbor_lists(b, p)[0] == 0
    count = np.zeros(8, np.int32)
    frac = np.zeros(8, np.float64)
    assert oracle.virtual_light(b, p, count, frac) == 0
    hi, lo = k["expected_open_count_greater"]
    assert count[hi] > count[lo], count.tolist()
    for i, above in k["expected_open_fraction_above"].items():
        assert frac[int(i)] > above
    assert np.array_equal(frac, count / 14.0)
    # either output alone, and neither (an argument error, surface_detection.cu:567-570)
    c2 = np.full(8, -1, np.int32)
    assert oracle.virtual_light(b, p, c2, None) == 0 and np.array_equal(c2, count)
    assert oracle.virtual_light(b, p, None, None) == pkg.abi.INVALID_ARGUMENT
    p.virtual_light_cone_cosine = 1.5
    assert oracle.virtual_light(b, p, count, None) == pkg.abi.INVALID_ARGUMENT


def test_virtual_light_lattice(pkg, oracle):
    # On a cubic lattice with r_e > sqrt(2) l0 every one of the 14 directions
    # has a neighbour exactly on it (projection 1), so an interior particle is
    # closed; an isolated particle is open in all 14.  Walls only close
    # directions when include_wall_neighbors is set.
    l0 = 1.0
    pts = [(ix, iy, iz) for iz in range(5) for iy in range(5) for ix in range(5)]
    pts.append((20.0, 20.0, 20.0))
    k = {"fluid": {"x": [q[0] * l0 for q in pts], "y": [q[1] * l0 for q in pts], "z": [q[2] * l0 for q in pts]},
         "walls": {"x": [2.0], "y": [2.0], "z": [-1.0]},
         "grid": {"origin": [-2.0, -2.0, -2.0], "cell_size": 1.5, "dims": [16, 16, 16]},
         "params": {"support_radius": 1.5, "particle_spacing": l0, "virtual_light_cone_cosine": 0.8660254,
                    "include_wall_neighbors": 1},
         "max_fluid_neighbors": 32, "max_wall_neighbors": 4}
    b = buffers_from(pkg, pkg.buffers.NumpyAlloc(), k)
    p = params_from(pkg, k)
    assert oracle.build_neighbor_lists(b, p)[0] == 0
    n = len(pts)
    count = np.zeros(n, np.int32)
    assert oracle.virtual_light(b, p, count, None) == 0
    centre = pts.index((2, 2, 2))
    bottom = pts.index((2, 2, 0))
    assert count[centre] == 0
    assert count[n - 1] == 14
    with_wall = int(count[bottom])
    p.include_wall_neighbors = 0
    assert oracle.virtual_light(b, p, count, None) == 0
    # the wall below closes -z (direction 5) and nothing else near it
    assert int(count[bottom]) == with_wall + 1


def _moment_case(pkg, k):
    b = buffers_from(pkg, pkg.buffers.NumpyAlloc(), k)
    p = params_from(pkg, k)
    return b, p


def test_moment_matrix_kat(pkg, oracle, kats):
    k = kats["moment_matrix"]
    b, p = _moment_case(pkg, k)
    for kind in range(4):
        assert oracle.prepare_moment(b, p, kind) == 0
        m = pkg.abi.MOMENT_SIZE[kind]
        inv = b.moments[kind]["inverse_matrices"].reshape(-1, m, m)
        assert np.isfinite(inv[k["center"]]).all()
        assert (b.moments[kind]["info"] == 0).all()
        assert b.moments[kind]["inversion_count"][0] == 1
        # the explicit inverse is symmetric and inverts the assembled matrix
        c = inv[k["center"]]
        assert np.allclose(c, c.T, rtol=1e-10, atol=1e-8)


def test_moment_inverse_matches_dense_inverse(pkg, oracle, kats):
    """Cross-check the restated Cholesky+substitution against numpy on the
    matrices rebuilt in Python from the same formula (moment_matrix.cu:145-309)."""
    k = kats["moment_matrix"]
    b, p = _moment_case(pkg, k)
    assert oracle.prepare_moment(b, p, 0) == 0
    x, y, z = (np.asarray(k["fluid"][c]) for c in "xyz")
    re = p.support_radius
    for i in (0, 13, 26):
        M = np.zeros((9, 9))
        for j in range(27):
            if j == i:
                continue
            d = np.array([x[j] - x[i], y[j] - y[i], z[j] - z[i]])
            dist = np.sqrt(d @ d)
            w = 1 - dist / re
            s = d / re
            bv = np.array([s[0], s[1], s[2], s[0] ** 2, s[1] ** 2, s[2] ** 2, s[0] * s[1], s[1] * s[2], s[2] * s[0]])
            M += w * np.outer(bv, bv)
        tr = np.trace(M)
        M += np.eye(9) * p.lsmps_regularization * tr / 9
        ref = np.linalg.inv(M)
        got = b.moments[0]["inverse_matrices"].reshape(-1, 9, 9)[i].T  # column-major
        assert np.allclose(got, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())
        assert abs(b.moments[0]["moment_trace"][i] - tr) < 1e-12 * tr


def test_provision_kat(pkg, oracle, kats):
    k = kats["provision"]
    b, p = _moment_case(pkg, k)
    assert oracle.prepare_moment(b, p, 0) == 0
    assert oracle.provision(b, p) == 0
    c = k["center"]
    tol = k["tolerance"]
    assert abs(b.velocity_laplacian["x"][c] - k["expected_laplacian_x_center"]) <= tol
    vx = np.asarray(k["fluid"]["vx"])
    g = k["params"]["gravity"]
    dt = k["params"]["time_step"]
    nu = k["params"]["kinematic_viscosity"]
    assert abs(b.temporary_velocity["vx"][c] - (vx[c] + dt * (nu * 4.0 + g[0]))) <= tol
    assert abs(b.temporary_velocity["vy"][c] - (-2.0 + dt * g[1])) <= tol
    assert abs(b.temporary_velocity["vx"][0] - (vx[0] + dt * g[0])) <= tol  # Splash: no viscosity
    wv = k["walls"]
    for comp, gi in (("vx", 0), ("vy", 1), ("vz", 2)):
        assert abs(b.temporary_wall_velocity[comp][0] - (wv[comp][0] + dt * g[gi])) <= tol


def test_ppe_kat(pkg, oracle, kats):
    k = kats["ppe"]
    b, p = _moment_case(pkg, k)
    for comp in ("vx", "vy", "vz"):
        b.temporary_velocity[comp][:] = np.asarray(k["fluid"][comp])
    assert oracle.prepare_moment(b, p, 0) == 0
    assert oracle.prepare_moment(b, p, 1) == 0
    assert oracle.assemble_ppe(b, p) == 0
    ro = b.ppe["row_offsets"]
    assert ro[0] == 0 and ro[-1] == k["expected_nnz"] == b.nnz_cap
    col, val = b.ppe["col_indices"], b.ppe["values"]
    assert col[ro[0]] == 0 and val[ro[0]] == 1.0 and b.ppe["rhs"][0] == 0.0
    c = k["center"]
    tol = k["tolerance"]
    assert abs(b.ppe["divergence"][c] - k["expected_divergence_center"]) <= tol
    assert abs(b.ppe["rhs"][c] - k["expected_rhs_center"]) <= tol
    row = slice(ro[c], ro[c + 1])
    assert col[ro[c]] == c and np.isfinite(val[row]).all() and abs(val[ro[c]]) > 0
    # diagonal = -sum of off-diagonals (ppe_matrix.cu:300-302)
    assert abs(val[ro[c]] + val[ro[c] + 1:ro[c + 1]].sum()) < 1e-9 * abs(val[ro[c]])


def test_pressure_correction_kat(pkg, oracle, kats):
    k = kats["pressure_correction"]
    b, p = _moment_case(pkg, k)
    for comp in ("vx", "vy", "vz"):
        b.temporary_velocity[comp][:] = np.asarray(k["fluid"][comp])
    assert oracle.prepare_moment(b, p, 1) == 0
    x0 = b.fluid["x"].copy()
    assert oracle.pressure_correction(b, p) == 0
    c = k["center"]
    tol = k["tolerance"]
    grad = [b.pressure_gradient[a][c] for a in "xyz"]
    assert np.allclose(grad, k["expected_gradient_center"], atol=tol)
    assert b.pressure_gradient["x"][0] == 0.0  # Splash
    sc = p.time_step / p.density
    ev = [0.5 - sc * 2.0, -0.25 + sc * 3.0, 0.75 - sc * 4.0]
    assert np.allclose([b.fluid[v][c] for v in ("vx", "vy", "vz")], ev, atol=tol)
    assert abs(b.fluid["x"][c] - (x0[c] + 0.5 * p.time_step * (0.5 + ev[0]))) <= tol


def test_hydrostatic_case_step_properties(pkg, oracle):
    """Config-1-sized hydrostatic box: the rebuilt geometry is stable, interior
    particles are Inner, the free surface layer is Surface, and the LSMPS
    pressure gradient of the hydrostatic field is (0, 0, -rho g) inside
    (hydrostatic_surface_diagnostics.cu:687-702 prints this)."""
    case = pkg.cases.hydrostatic_box(n=12, l0=0.01)
    a = pkg.buffers.NumpyAlloc()
    b = pkg.buffers.StepBuffers(a, case.n_fluid, case.n_wall, case.n_cells)
    b.load_case(case)
    p = case.params
    st, req = oracle.build_neighbor_lists(b, p)
    assert st == 0
    off, _ = b.csr_rows("fluid")
    counts = np.diff(off)
    assert counts.max() == 122  # interior lattice neighbourhood at r_e = 3.1 l0
    assert oracle.classify_surface(b, p) == 0
    lab = b.fluid["surface_type"].reshape(12, 12, 12)
    # the top layer away from the walls (the wall-normal basis removes the
    # opening next to the side walls, surface_detection.cu:251-262)
    assert (lab[-1, 2:-2, 2:-2] == pkg.abi.SURFACE).all()
    assert (lab[2:-3, 3:-3, 3:-3] == pkg.abi.INNER).all()
    assert oracle.prepare_moment(b, p, 1) == 0
    pr = b.fluid["pressure"].copy()
    g = pkg.abi.Vector()
    st = oracle.L.oracle_pressure_gradient(
        oracle_ref(b.fluid_view()), oracle_ref(b.walls_view()), oracle_ref(b.csr_view("fluid")),
        oracle_ref(b.csr_view("wall")), pr.ctypes.data, oracle_ref(p),
        oracle_ref(b.moment_view(1)), oracle_ref(b.vector_view(b.pressure_gradient)))
    assert st == 0
    gz = b.pressure_gradient["z"].reshape(12, 12, 12)
    assert np.allclose(gz[3:-4, 4:-4, 4:-4], -1000 * 9.81, rtol=1e-6)


def oracle_ref(x):
    import ctypes

    return ctypes.byref(x)


def test_tank_walls_vectorised_matches_loop(pkg):
    slow = pkg.cases.tank_walls(5, 4, 7, 0.1)
    fast = pkg.cases._tank_walls_fast(5, 4, 7, 0.1)
    for s, f in zip(slow, fast):
        assert np.array_equal(s, f)


def test_splitmix64_known_values(pkg):
    # splitmix64 reference outputs for seed 0 (first three values of the stream)
    z = pkg.cases.splitmix64(0, 3)
    assert [int(v) for v in z] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]
    u = pkg.cases.uniform01(7, 1000)
    assert (u >= 0).all() and (u < 1).all()


@pytest.mark.parametrize("name", ["hydrostatic", "dam_break", "splash"])
def test_case_generators_shapes(pkg, name):
    small = {"hydrostatic": dict(n=6), "dam_break": dict(nx=8, ny=4, nz=8), "splash": dict(nx=8, ny=4, nz=8)}
    c = pkg.cases.CASES[name](**small[name])
    assert c.n_fluid > 0 and c.n_wall > 0
    assert c.params.support_radius <= c.params.grid.cell_size
    for arr in c.fluid.values():
        assert arr.shape[0] == c.n_fluid
