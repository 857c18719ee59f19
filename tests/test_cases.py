"""Seeded synthetic workloads (no GPU): the batched-box generator is
deterministic and draws sizes log-uniform within its bounds."""


def test_batched_boxes_deterministic(pkg):
    a = pkg.cases.batched_boxes(count=8, seed=7, n_min=1_000, n_max=30_000)
    b = pkg.cases.batched_boxes(count=8, seed=7, n_min=1_000, n_max=30_000)
    assert [c.name for c in a] == [c.name for c in b]
    for c, d in zip(a, b):
        assert c.n_fluid == d.n_fluid and c.n_wall == d.n_wall
        assert (c.fluid["x"] == d.fluid["x"]).all()
    kinds = {c.name.split("_", 1)[1].split("_")[0] for c in a}
    assert kinds <= {"hydrostatic", "dam"}
    # the rounding of the lattice sides keeps each box within ~35% of its draw
    assert all(300 <= c.n_fluid <= 45_000 for c in a)
