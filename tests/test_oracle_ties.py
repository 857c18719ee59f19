"""The oracle's neighbour test at exact ties, on the CPU.

The reference decides `dx*dx + dy*dy + dz*dz <= r^2` on the device, where
nvcc contracts the sum into fused multiply-adds.  On an unjittered lattice
whose spacing divides r, thousands of pairs lie within rounding of r and the
contracted and twice-rounded sums decide some of them differently.  The
oracle states the contracted order fma(dz, dz, fma(dx, dx, dy*dy)), the one
that reproduces the reference's CUDA path pair for pair (checked on a GPU by
tests/test_gpu_parity.py::test_csr_pairs_at_the_radius).  Here the oracle's
rows are checked against a brute-force restatement of that order, with each
fused multiply-add evaluated exactly in rational arithmetic and rounded once.
"""

from fractions import Fraction

import numpy as np
import pytest


def _fma(a: float, b: float, c: float) -> float:
    # one rounding of the exact a*b + c (Fraction -> float rounds to nearest)
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _fused_within(dx: float, dy: float, dz: float, r2: float) -> bool:
    return _fma(dz, dz, _fma(dx, dx, dy * dy)) <= r2


@pytest.mark.parametrize("radius_l0,flips", [(3.0, True), (6.0 ** 0.5, False)])
def test_oracle_ties_follow_the_contracted_sum(pkg, oracle, radius_l0, flips):
    case = pkg.cases.hydrostatic_box(n=12, l0=0.01)
    p = case.params
    p.support_radius = radius_l0 * case.l0
    p.grid.cell_size = p.support_radius
    pkg.cases.derive_grid(p, [case.fluid["x"], case.walls["x"]], [case.fluid["y"], case.walls["y"]],
                          [case.fluid["z"], case.walls["z"]])
    b = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), case.n_fluid, case.n_wall, case.n_cells,
                                max_fluid_neighbors=256, max_wall_neighbors=256)
    b.load_case(case)
    st, _ = oracle.build_neighbor_lists(b, p)
    assert st == 0
    off, idx = b.csr_rows("fluid")

    x, y, z = (np.asarray(case.fluid[c]) for c in "xyz")
    r2 = p.support_radius * p.support_radius
    dx = x[:, None] - x[None, :]
    dy = y[:, None] - y[None, :]
    dz = z[:, None] - z[None, :]
    twice = dx * dx + dy * dy + dz * dz
    expect = twice <= r2
    near = np.argwhere(np.abs(twice - r2) <= 8 * np.spacing(r2))
    flipped = 0
    for i, j in near:
        fused = _fused_within(float(dx[i, j]), float(dy[i, j]), float(dz[i, j]), r2)
        flipped += int(fused != expect[i, j])
        expect[i, j] = fused
    np.fill_diagonal(expect, False)
    # at r = 3 l0 the lattice holds ties that the two sums decide differently
    # (208 of them); at sqrt(6) l0 they agree
    assert (flipped > 0) == flips
    for i in range(case.n_fluid):
        got = set(idx[off[i]:off[i + 1]].tolist())
        want = set(np.flatnonzero(expect[i]).tolist())
        assert got == want, i
