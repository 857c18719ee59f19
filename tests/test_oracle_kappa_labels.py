"""Why the mixed form routes matrices to FP64 by their condition estimate and
not by label.

The FP64 oracle's Type-A moment inverses of the splash dam break with the
lifted particles scattered off the lattice (40 x 10 x 40, the case of
tests/test_gpu_mixed.py) give, per surface label, the estimate
kappa_est = (trace M + 9 reg) ||M^-1||_F that the library's threshold is
compared with (an upper bound of kappa_2 within a factor 27).  Ill-conditioned
matrices are not confined to the Surface and Splash labels: a few Inner and
NearSurface particles of the sparse lifted layer reach kappa ~ 1e9, while
most Surface particles stay below 1e4.  A label route would factorise the
former in FP32 (one refinement then leaves a relative error of order
(kappa 2^-24)^2, far above the tolerance) and spend FP64 on the latter; the
condition estimate routes exactly the matrices that need it, nearly every
Splash matrix among them.  CPU only.
"""

import numpy as np

NAMES = {0: "inner", 1: "near_surface", 2: "surface", 3: "splash"}


def test_ill_conditioned_matrices_by_label(pkg, oracle):
    case = pkg.cases.splash_scattered(nx=40, ny=10, nz=40, l0=0.0025)
    p = case.params
    h = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), case.n_fluid, case.n_wall, case.n_cells)
    h.load_case(case)
    oracle.build_neighbor_lists(h, p)
    assert oracle.classify_surface(h, p) == 0
    labels = h.fluid["surface_type"].copy()
    for kind in (0, 1):
        assert oracle.prepare_moment(h, p, kind) == 0
        m = h.moments[kind]
        x = m["inverse_matrices"].reshape(-1, 81)
        kappa = (m["moment_trace"] + 9.0 * m["regularization_added"]) * np.sqrt((x * x).sum(axis=1))
        above = {}
        for t, name in NAMES.items():
            k = kappa[labels == t]
            above[name] = int((k > 1e4).sum())
            print(f"kind {kind} {name}: {k.size} particles, median kappa_est {np.median(k):.3g}, "
                  f"max {k.max():.3g}, above 1e4: {above[name]}, above 1e6: {int((k > 1e6).sum())}")
        # nearly every Splash matrix is ill-conditioned (a Splash particle
        # with no neighbour at all has M = reg I, perfectly conditioned) ...
        splash = kappa[labels == 3]
        assert splash.size > 0 and (splash > 1e4).mean() >= 0.9
        # ... but so are some Inner / NearSurface ones, and most Surface ones are not
        assert above["inner"] + above["near_surface"] > 0
        assert above["surface"] < 0.5 * int((labels == 2).sum())
