"""The oracle's PPE solve (restarted GMRES, the algorithm the reference runs
through AMGX) pinned against the reference's AMGX known answers and against
dense direct solves and residual properties (no GPU)."""

import numpy as np
import pytest

from kat_util import buffers_from, params_from  # noqa: F401  (fixture helpers)


def options(pkg, **kw):
    o = pkg.abi.default_solver_options()
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def csr_of(dense):
    rows, cols = np.nonzero(dense)
    off = np.zeros(dense.shape[0] + 1, np.int32)
    np.add.at(off, rows + 1, 1)
    return np.cumsum(off).astype(np.int32), cols.astype(np.int32), dense[rows, cols].astype(np.float64)


def random_system(n, seed, density=0.02, dominance=2.0, scale_rows=False):
    rng = np.random.default_rng(seed)
    a = np.where(rng.random((n, n)) < density, rng.standard_normal((n, n)), 0.0)
    np.fill_diagonal(a, 0.0)
    d = np.abs(a).sum(1) * dominance + 1.0
    a += np.diag(d)
    if scale_rows:
        a *= np.exp(rng.uniform(-4, 4, n))[:, None]
    return a, rng.standard_normal(n)


def test_amgx_smoke_kat(pkg, oracle, kats):
    # smoke_ppe_matrix.cu:52-117: [[4, -1], [-1, 4]] p = (3, 3) -> p = (1, 1);
    # p = -(1, 1) for the negated right-hand side is clamped to 0.
    k = kats["ppe_solve"]
    ro = np.asarray(k["row_offsets"], np.int32)
    ci = np.asarray(k["col_indices"], np.int32)
    va = np.asarray(k["values"], np.float64)
    x = np.full(2, 7.0)
    st, rep = oracle.solve_ppe(ro, ci, va, np.asarray(k["rhs"]), x, options(pkg))
    assert st == 0 and rep.converged == 1 and rep.iterations <= 2
    assert np.allclose(x, k["expected"], atol=k["tolerance"], rtol=0)
    st, rep = oracle.solve_ppe(ro, ci, va, np.asarray(k["negated_rhs"]), x, options(pkg))
    assert st == 0
    assert np.allclose(x, k["expected_negated_clamped"], atol=k["tolerance"], rtol=0)


@pytest.mark.parametrize("precond", [0, 1], ids=["none", "jacobi"])
def test_converges_to_direct_solve(pkg, oracle, precond):
    a, b = random_system(300, 1, scale_rows=bool(precond))
    ro, ci, va = csr_of(a)
    x = np.zeros(300)
    st, rep = oracle.solve_ppe(ro, ci, va, b, x, options(pkg, tolerance=1e-12, max_iters=400, clamp_negative=0,
                                                        preconditioner=precond))
    assert st == 0 and rep.converged == 1
    ref = np.linalg.solve(a, b)
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-9
    r = np.linalg.norm(b - a @ x)
    assert abs(r - rep.final_residual) <= 1e-12 * np.linalg.norm(b)
    assert rep.final_residual <= 1e-12 * rep.initial_residual


def test_jacobi_helps_badly_scaled_rows(pkg, oracle):
    a, b = random_system(300, 2, scale_rows=True)
    ro, ci, va = csr_of(a)
    its = []
    for precond in (0, 1):
        x = np.zeros(300)
        st, rep = oracle.solve_ppe(ro, ci, va, b, x, options(pkg, tolerance=1e-8, max_iters=300, clamp_negative=0,
                                                            preconditioner=precond))
        assert st == 0
        its.append((rep.iterations, rep.converged))
    assert its[1][1] == 1 and its[1][0] < its[0][0]


def test_iteration_limit_and_report(pkg, oracle):
    a, b = random_system(200, 3, dominance=0.3)
    ro, ci, va = csr_of(a)
    x = np.zeros(200)
    st, rep = oracle.solve_ppe(ro, ci, va, b, x, options(pkg, max_iters=7, restart=3, clamp_negative=0))
    assert st == 0 and rep.iterations == 7
    assert rep.initial_residual == pytest.approx(np.linalg.norm(b), rel=1e-14)
    assert rep.final_residual == pytest.approx(np.linalg.norm(b - a @ x), rel=1e-10)
    assert rep.final_residual < rep.initial_residual
    # max_iters = 0: x stays at the zero initial guess
    x[:] = 5.0
    st, rep = oracle.solve_ppe(ro, ci, va, b, x, options(pkg, max_iters=0))
    assert st == 0 and rep.iterations == 0 and not x.any()
    # invalid restart
    st, _ = oracle.solve_ppe(ro, ci, va, b, x, options(pkg, restart=0))
    assert st == pkg.abi.INVALID_ARGUMENT


def test_ppe_system_of_hydrostatic_case(pkg, oracle):
    # The oracle's own assembled PPE rows (Dirichlet rows for the free surface):
    # 100 GMRES(20) steps lower the residual, and the reported residual is the
    # true one.
    case = pkg.cases.CASES["hydrostatic"](n=10, l0=0.01)
    p = case.params
    b = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), case.n_fluid, case.n_wall, case.n_cells)
    b.load_case(case)
    assert oracle.build_neighbor_lists(b, p)[0] == 0
    assert oracle.classify_surface(b, p) == 0
    for kind in (0, 1):
        assert oracle.prepare_moment(b, p, kind) == 0
    assert oracle.provision(b, p) == 0
    assert oracle.assemble_ppe(b, p) == 0
    ro = b.ppe["row_offsets"]
    nnz = int(ro[-1])
    ci, va, rhs = b.ppe["col_indices"][:nnz], b.ppe["values"][:nnz], b.ppe["rhs"]
    x = np.zeros(case.n_fluid)
    st, rep = oracle.solve_ppe(ro, ci, va, rhs, x, options(pkg, clamp_negative=0))
    assert st == 0 and rep.iterations >= 1
    dense = np.zeros((case.n_fluid, case.n_fluid))
    for i in range(case.n_fluid):
        np.add.at(dense[i], ci[ro[i]:ro[i + 1]], va[ro[i]:ro[i + 1]])
    assert rep.final_residual == pytest.approx(np.linalg.norm(rhs - dense @ x), rel=1e-9, abs=1e-300)
    assert rep.final_residual <= rep.initial_residual
