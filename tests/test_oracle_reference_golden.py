"""The CPU oracle pinned against outputs of the reference's own CUDA path
(golden/reference_<case>.npz, written on a B200 by
golden/make_reference_golden.py from the reference sources built in oracle/_ref).

Integer outputs (cell lists, CSR rows in native order, labels, PPE columns)
must be bit-exact.  Floating outputs must agree to FP64 rounding times the
moment-matrix conditioning; the reference inverts with cuSOLVER's batched
potrf/potrs and the oracle with its own Cholesky and substitutions.
"""

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_reference_golden as gold  # noqa: E402

from kat_util import rel_err, vec_err  # noqa: E402


def load(name):
    path = os.path.join(HERE, "golden", f"reference_{name}.npz")
    if not os.path.exists(path):
        pytest.fail(f"golden fixture {path} missing: run tests/golden/make_reference_golden.py on a GPU machine")
    return dict(np.load(path))


@pytest.mark.parametrize("name", list(gold.GOLDEN_CASES))
def test_oracle_matches_reference_cuda(pkg, oracle, name):
    g = load(name)
    kind, kw = gold.GOLDEN_CASES[name]
    case = pkg.cases.CASES[kind](**kw)
    assert str(g["input_sha256"]) == gold.input_digest(case), "seeded inputs drifted from the fixture"
    p = case.params
    b = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), case.n_fluid, case.n_wall, case.n_cells)
    b.load_case(case)
    # geometry
    st, _ = oracle.build_neighbor_lists(b, p)
    assert st == 0
    assert oracle.classify_surface(b, p) == 0
    for which, d in (("fluid", b.fluid_cells), ("wall", b.wall_cells)):
        for k, v in d.items():
            assert np.array_equal(v, g[f"geometry/{which}_cells/{k}"]), (which, k)
    for which in ("fluid", "wall"):
        off, idx = b.csr_rows(which)
        assert np.array_equal(off, g[f"geometry/{which}_offsets"])
        assert np.array_equal(idx, g[f"geometry/{which}_indices"])
    assert np.array_equal(b.fluid["surface_type"], g["geometry/surface_type"])
    # moments and provision
    for k in (0, 1):
        assert oracle.prepare_moment(b, p, k) == 0
        m = b.moments[k]
        assert np.array_equal(m["info"], g[f"provision/moment{k}/info"])
        assert rel_err(m["moment_trace"], g[f"provision/moment{k}/moment_trace"]) < 1e-12
        assert rel_err(m["regularization_added"], g[f"provision/moment{k}/regularization_added"]) < 1e-12
        rows = g["provision/inverse_rows"]
        inv = m["inverse_matrices"].reshape(-1, 81)[rows]
        ref = g[f"provision/moment{k}/inverse"]
        per = np.max(np.abs(inv - ref), axis=1) / np.max(np.abs(ref), axis=1)
        assert per.max() < 1e-6, per.max()
    assert oracle.provision(b, p) == 0
    for k in ("vx", "vy", "vz"):
        assert rel_err(b.temporary_velocity[k], g[f"provision/temporary_{k}"]) < 1e-9
        assert np.array_equal(b.temporary_wall_velocity[k], g[f"provision/temporary_wall_{k}"])
    # PPE
    assert oracle.assemble_ppe(b, p) == 0
    written = g["ppe/values"].shape[0]
    assert int(g["ppe/active_nnz"]) == case.n_fluid + b.cap_f
    assert np.array_equal(b.ppe["row_offsets"], g["ppe/row_offsets"])
    assert np.array_equal(b.ppe["col_indices"][:written], g["ppe/col_indices"])
    assert rel_err(b.ppe["values"][:written], g["ppe/values"]) < 1e-6
    for k in ("rhs", "divergence", "pressure_laplacian"):
        assert rel_err(b.ppe[k], g[f"ppe/{k}"]) < 1e-6, k
    # correction
    assert oracle.pressure_correction(b, p) == 0
    ref_fluid = {k: g[f"correction/{k}"] for k in ("x", "y", "z", "vx", "vy", "vz", "pressure")}
    errs = {**vec_err(b.fluid, ref_fluid, ("x", "y", "z")),
            **vec_err(b.fluid, ref_fluid, ("vx", "vy", "vz"), extra_scale=b.temporary_velocity),
            "pressure": rel_err(b.fluid["pressure"], ref_fluid["pressure"])}
    for k, e in errs.items():
        assert e < 1e-6, (k, e)
    for vec, key in ((b.pressure_gradient, "gradient"), (b.ps_displacement, "shift")):
        ref_vec = {k: g[f"correction/{key}_{k}"] for k in ("x", "y", "z")}
        for k, e in vec_err(vec, ref_vec, ("x", "y", "z")).items():
            assert e < 1e-6, (key, k, e)
    # rebuild on the moved particles
    st, _ = oracle.build_neighbor_lists(b, p)
    assert st == 0
    assert oracle.classify_surface(b, p) == 0
    assert np.array_equal(b.fluid["surface_type"], g["rebuilt/surface_type"])
    for which in ("fluid", "wall"):
        off, idx = b.csr_rows(which)
        assert np.array_equal(off, g[f"rebuilt/{which}_offsets"])
        assert np.array_equal(idx, g[f"rebuilt/{which}_indices"])
