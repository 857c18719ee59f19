"""The device PPE solve (lsmps_solve_ppe: restarted GMRES, the method the
reference runs through AMGX in AmgxPpeSolver::solve, src/ppe/ppe_matrix.cu:
586-679) against the oracle's restatement and against direct solves.

The device and the oracle run the same algorithm (CGS2 Arnoldi, Givens
rotations, the same restart and stopping rules) with different summation
orders, so their iterates agree to rounding amplified by the Krylov process:
bounds below are written per comparison.  Converged solves are also checked
against numpy's dense solve, and every reported residual against
||b - A x|| recomputed on the host.
"""

import numpy as np
import pytest

from kat_util import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(device_api):
    return device_api.Context(0)


def options(pkg, **kw):
    o = pkg.abi.default_solver_options()
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def device_csr(pkg, ro, ci, va):
    import torch

    t = [torch.as_tensor(np.ascontiguousarray(a)).cuda() for a in (ro, ci, va)]
    m = pkg.abi.CsrMatrix(len(ro) - 1, len(ro) - 1, len(va), t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr())
    return m, t


def dev_solve(pkg, ctx, ro, ci, va, rhs, opt):
    import torch

    m, keep = device_csr(pkg, ro, ci, va)
    b = torch.as_tensor(np.asarray(rhs, np.float64)).cuda()
    x = torch.full((len(ro) - 1,), 3.0, dtype=torch.float64, device="cuda")
    rep = ctx.solve_csr(m, b.data_ptr(), x.data_ptr(), opt)
    return x.cpu().numpy(), rep


def csr_of(dense):
    rows, cols = np.nonzero(dense)
    off = np.zeros(dense.shape[0] + 1, np.int32)
    np.add.at(off, rows + 1, 1)
    return np.cumsum(off).astype(np.int32), cols.astype(np.int32), dense[rows, cols].astype(np.float64)


def csr_matvec(ro, ci, va, x):
    rows = np.repeat(np.arange(len(ro) - 1), np.diff(ro))
    return np.bincount(rows, weights=va * x[ci], minlength=len(ro) - 1)


def test_amgx_smoke_kat_on_device(pkg, ctx, kats):
    # smoke_ppe_matrix.cu:52-117
    k = kats["ppe_solve"]
    ro, ci, va = (np.asarray(k[n], t) for n, t in (("row_offsets", np.int32), ("col_indices", np.int32),
                                                    ("values", np.float64)))
    x, rep = dev_solve(pkg, ctx, ro, ci, va, k["rhs"], options(pkg))
    assert rep.converged == 1 and rep.iterations <= 2
    assert np.allclose(x, k["expected"], atol=k["tolerance"], rtol=0)
    x, rep = dev_solve(pkg, ctx, ro, ci, va, k["negated_rhs"], options(pkg))
    assert np.allclose(x, k["expected_negated_clamped"], atol=k["tolerance"], rtol=0)


@pytest.mark.parametrize("precond", [0, 1], ids=["none", "jacobi"])
def test_converged_solve_matches_direct(pkg, ctx, oracle, precond):
    rng = np.random.default_rng(7)
    n = 2000
    a = np.where(rng.random((n, n)) < 0.005, rng.standard_normal((n, n)), 0.0)
    np.fill_diagonal(a, 0.0)
    a += np.diag(2.0 * np.abs(a).sum(1) + 1.0)
    if precond:
        a *= np.exp(rng.uniform(-3, 3, n))[:, None]
    b = rng.standard_normal(n)
    ro, ci, va = csr_of(a)
    opt = options(pkg, tolerance=1e-12, max_iters=500, clamp_negative=0, preconditioner=precond, restart=30)
    x, rep = dev_solve(pkg, ctx, ro, ci, va, b, opt)
    assert rep.converged == 1
    ref = np.linalg.solve(a, b)
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-9
    assert abs(np.linalg.norm(b - a @ x) - rep.final_residual) <= 1e-12 * np.linalg.norm(b)
    xo = np.zeros(n)
    st, repo = oracle.solve_ppe(ro, ci, va, b, xo, opt)
    assert st == 0 and abs(repo.iterations - rep.iterations) <= 1
    print(f"precond={precond}: device {rep.iterations} its, oracle {repo.iterations} its")


CASES = [
    ("hydrostatic", dict(n=20, l0=0.01)),
    ("dam_break", dict(nx=24, ny=12, nz=24, l0=0.005)),
    ("splash", dict(nx=40, ny=10, nz=40, l0=0.0025)),
]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_ppe_system_matches_oracle(pkg, device_api, ctx, oracle, name, kw):
    # The device-assembled PPE rows of each case, solved with the reference's
    # configuration (GMRES(20), 100 iterations, 1e-6 relative) on the device
    # and by the oracle on the same rows.
    case = pkg.cases.CASES[name](**kw)
    p = case.params
    dev = pkg.buffers.StepBuffers(pkg.buffers.TorchAlloc("cuda"), case.n_fluid, case.n_wall, case.n_cells)
    dev.load_case(case)
    ctx.build_neighbor_lists(dev, p)
    ctx.classify_surface(dev, p)
    ctx.prepare_moments(dev, p, [0, 1])
    ctx.provision(dev, p)
    ctx.assemble_ppe(dev, p)
    g = dev.numpy("ppe")
    ro = g["row_offsets"]
    nnz = int(ro[-1])
    ci, va, rhs = g["col_indices"][:nnz].copy(), g["values"][:nnz].copy(), g["rhs"].copy()
    for opt in (options(pkg, clamp_negative=0), options(pkg)):
        rep = ctx.solve_ppe(dev, opt)
        x = dev.numpy("ppe")["pressure"]
        xo = np.zeros(case.n_fluid)
        st, repo = oracle.solve_ppe(ro, ci, va, rhs, xo, opt)
        assert st == 0
        assert rep.iterations == repo.iterations
        assert rep.initial_residual == pytest.approx(repo.initial_residual, rel=1e-12)
        e_res = abs(rep.final_residual - repo.final_residual) / rep.initial_residual
        e_x = rel_err(x, xo)
        print(f"{case.name} clamp={opt.clamp_negative}: {rep.iterations} its, residual "
              f"{rep.final_residual / rep.initial_residual:.3e} of initial (oracle "
              f"{repo.final_residual / repo.initial_residual:.3e}); |dres|/r0 {e_res:.2e}, x rel err {e_x:.2e}")
        assert e_res < 1e-8
        assert e_x < 1e-6
        if not opt.clamp_negative:
            r = np.linalg.norm(rhs - csr_matvec(ro, ci, va, x))
            assert r == pytest.approx(rep.final_residual, rel=1e-8)
        else:
            assert (x >= 0).all()


def test_solve_is_deterministic_and_checks_arguments(pkg, device_api, ctx):
    import torch

    rng = np.random.default_rng(3)
    n = 5000
    a = np.where(rng.random((n, n)) < 0.002, rng.standard_normal((n, n)), 0.0)
    a += np.diag(np.abs(a).sum(1) + 0.5)
    ro, ci, va = csr_of(a)
    b = rng.standard_normal(n)
    x1, r1 = dev_solve(pkg, ctx, ro, ci, va, b, options(pkg, clamp_negative=0))
    x2, r2 = dev_solve(pkg, ctx, ro, ci, va, b, options(pkg, clamp_negative=0))
    assert np.array_equal(x1, x2) and r1.final_residual == r2.final_residual
    m, keep = device_csr(pkg, ro, ci, va)
    bt = torch.as_tensor(b).cuda()
    xt = torch.zeros(n, dtype=torch.float64, device="cuda")
    for bad in (dict(restart=0), dict(restart=65), dict(max_iters=-1), dict(preconditioner=7)):
        with pytest.raises(device_api.LsmpsError):
            ctx.solve_csr(m, bt.data_ptr(), xt.data_ptr(), options(pkg, **bad))
    # max_iters = 0: the zero initial guess is returned
    xt.fill_(9.0)
    rep = ctx.solve_csr(m, bt.data_ptr(), xt.data_ptr(), options(pkg, max_iters=0))
    assert rep.iterations == 0 and not xt.any()
