"""Parity at the full sizes of the benchmark workloads, through the C ABI:

* the 500k dam break (fluid block 100 x 50 x 100, l0 = 0.005, seeded jitter
  of +-0.05 l0, 3 wall layers);
* the 2M splash-heavy dam break (fluid block 200 x 50 x 200, l0 = 0.0025,
  5 % of the fluid lifted into the 10 l0 band above the free surface,
  3 wall layers).

Each workload is checked as stated (fluid at rest, hydrostatic pressure) and
again from a moving state (a smooth swirl velocity), so that the velocity
Laplacian, the PPE divergence and the viscous part of u* are not zero.

1. Integer outputs against the reference's own CUDA path (oracle/_ref, built
   from the reference sources) and against the CPU oracle, bit for bit: both
   cell lists, both CSR tables in their native row order, the labels, the
   PPE row offsets and column indices, and the rebuild after the step.
2. Floating outputs of the plain (FP64) form against the FP64 oracle, each
   stage from the same inputs on both sides, with the bounds below.  The two
   sides differ only in operation order (FMA contraction, reciprocal
   multiplies, the order of the inverse's substitutions), so each bound is
   rounding (2^-52) times a stated factor.  Moment inverses: per particle,
   max |dM^-1| / max |M^-1| <= INVERSE_EPS_FACTOR * 2^-52 * kappa_est, with
   kappa_est = (trace M) * ||M^-1||_F from the oracle's own matrix, an
   upper bound of the 2-norm condition number within a factor of 27.
   Fields: the normwise/elementwise metric of kat_util.rel_err.
3. Floating outputs against the reference CUDA path, with the same bounds
   (its inverses come from cuSOLVER's batched potrf/potrs).

Set LSMPS_PARITY_REPORT to a file path to have the measured maxima written
there as JSON.
"""

import json
import os
import sys
import time

import numpy as np
import pytest

from kat_util import inverse_err_over_kappa, rel_err, vec_err

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import reference as ref_mod  # noqa: E402

EPS = 2.0 ** -52
# Measured at both sizes: inverses at most 0.40 of 2^-52 kappa_est; fields at
# most 6e-12 (PPE values), against the oracle and against the reference's
# CUDA path.  The bounds sit 20x above.
INVERSE_EPS_FACTOR = 8.0
# Plain-form field bounds against the FP64 oracle (normwise against the
# field's scale, elementwise on entries above 1e-3 of it).
FIELD_RTOL = 1e-10
PPE_RTOL = 1e-10
STATE_RTOL = 1e-10
REFERENCE_RTOL = 1e-10

CASES = [
    ("dam_break_500k", "dam_break", dict(nx=100, ny=50, nz=100, l0=0.005)),
    ("splash_2M", "splash", dict(nx=200, ny=50, nz=200, l0=0.0025)),
]

_report: dict = {}


def _swirl(fluid):
    span = max(float(np.ptp(fluid[k])) for k in ("x", "y", "z")) or 1.0
    return {"vx": 0.1 * np.sin(fluid["x"] / span), "vy": 0.1 * np.cos(fluid["y"] / span),
            "vz": 0.1 * fluid["z"] / span}


def _dev_ppe(dev, nnz):
    """Device PPE arrays, the matrix arrays cut to the written entries."""
    out = {}
    for k, v in dev.ppe.items():
        out[k] = (v[:nnz] if k in ("values", "col_indices") else v).cpu().numpy()
    return out


def _dev_moment(dev, kind):
    return {k: v.cpu().numpy() for k, v in dev.moments[kind].items()}


def _kappa_est(hm):
    inv = hm["inverse_matrices"].reshape(-1, 81)
    reg = hm["regularization_added"]
    return (hm["moment_trace"] + 9.0 * reg) * np.sqrt(np.einsum("ij,ij->i", inv, inv))


def _compare_geometry(dev, other, label, rep):
    for which in ("fluid_cells", "wall_cells"):
        g = dev.numpy(which)
        h = other.numpy(which)
        for k in ("cell_ids", "sorted_indices", "cell_begin", "cell_end"):
            assert np.array_equal(g[k], h[k]), (label, which, k)
    for which in ("fluid", "wall"):
        go, gi = dev.csr_rows(which)
        ho, hi = other.csr_rows(which)
        assert np.array_equal(go, ho), (label, which, "offsets")
        assert np.array_equal(gi, hi), (label, which, "indices")
        rep[f"K_{which}"] = int(go[-1])
    lab_d = dev.fluid["surface_type"].cpu().numpy()
    assert np.array_equal(lab_d, other.fluid["surface_type"]), (label, "labels")
    rep["labels"] = np.bincount(lab_d, minlength=4).tolist()


def _float_stages(pkg, ctx, oracle, dev, host, p, rep, tag):
    """Moments, provision, PPE rows and correction on both sides from the
    same state; errors of the device against the oracle into rep[tag]."""
    r = rep.setdefault(tag, {})
    ctx.prepare_moments(dev, p, [0, 1])
    for kind in (0, 1):
        assert oracle.prepare_moment(host, p, kind) == 0
        gm = _dev_moment(dev, kind)
        hm = host.moments[kind]
        assert np.array_equal(gm["info"], hm["info"])
        r[f"trace_{kind}"] = rel_err(gm["moment_trace"], hm["moment_trace"])
        assert r[f"trace_{kind}"] < 1e-12
        ok = hm["info"] == 0
        gi = gm["inverse_matrices"].reshape(-1, 81)
        hi = hm["inverse_matrices"].reshape(-1, 81)
        per = np.max(np.abs(gi - hi), axis=1) / np.max(np.abs(hi), axis=1)
        kap = _kappa_est(hm)
        ratio = per / (EPS * kap)
        r[f"inverse_{kind}_max_rel"] = float(per[ok].max())
        r[f"inverse_{kind}_max_over_eps_kappa"] = float(ratio[ok].max())
        r[f"inverse_{kind}_kappa_est_max"] = float(kap[ok].max())
        assert ratio[ok].max() <= INVERSE_EPS_FACTOR, (kind, float(ratio[ok].max()))
    ctx.provision(dev, p)
    assert oracle.provision(host, p) == 0
    lap = vec_err(dev.numpy("velocity_laplacian"), host.numpy("velocity_laplacian"), ("x", "y", "z"))
    ustar = vec_err(dev.numpy("temporary_velocity"), host.temporary_velocity, ("vx", "vy", "vz"))
    for k, e in lap.items():
        r[f"laplacian_{k}"] = e
        assert e < FIELD_RTOL, ("laplacian", k, e)
    for k, e in ustar.items():
        r[f"u_star_{k}"] = e
        assert e < FIELD_RTOL, ("u*", k, e)
    wu = dev.numpy("temporary_wall_velocity")
    for k in ("vx", "vy", "vz"):
        assert np.array_equal(wu[k], host.temporary_wall_velocity[k]), ("wall u*", k)

    ctx.assemble_ppe(dev, p)
    assert oracle.assemble_ppe(host, p) == 0
    nnz = int(host.ppe["row_offsets"][-1])
    g = _dev_ppe(dev, nnz)
    assert np.array_equal(g["row_offsets"], host.ppe["row_offsets"])
    assert np.array_equal(g["col_indices"], host.ppe["col_indices"][:nnz])
    for k in ("values", "rhs", "divergence", "pressure_laplacian"):
        b = host.ppe[k][:nnz] if k == "values" else host.ppe[k]
        e = rel_err(g[k], b)
        r[f"ppe_{k}"] = e
        assert e < PPE_RTOL, ("ppe", k, e)

    ctx.pressure_correction(dev, p)
    assert oracle.pressure_correction(host, p) == 0
    grad = vec_err(dev.numpy("pressure_gradient"), host.numpy("pressure_gradient"), ("x", "y", "z"))
    f = dev.numpy("fluid")
    state = {**vec_err(f, host.fluid, ("x", "y", "z")),
             **vec_err(f, host.fluid, ("vx", "vy", "vz"), extra_scale=host.temporary_velocity),
             "pressure": rel_err(f["pressure"], host.fluid["pressure"])}
    for k, e in grad.items():
        r[f"grad_p_{k}"] = e
        assert e < FIELD_RTOL, ("grad p", k, e)
    for k, e in state.items():
        r[f"corrected_{k}"] = e
        assert e < STATE_RTOL, ("corrected", k, e)
    return f


@pytest.mark.parametrize("label,name,kw", CASES, ids=[c[0] for c in CASES])
def test_full_size_parity(pkg, device_api, oracle, label, name, kw):
    t0 = time.perf_counter()
    case = pkg.cases.CASES[name](**kw)
    p = case.params
    rep = _report.setdefault(label, {"n_fluid": case.n_fluid, "n_wall": case.n_wall, "cells": case.n_cells,
                                     "oracle_threads": oracle.max_threads()})
    ctx = device_api.Context(0)
    dev = device_api.device_buffers(case)
    try:
        ctx.build_neighbor_lists(dev, p)
        ctx.classify_surface(dev, p)

        # 1. the reference's own CUDA path: integers bit for bit
        if ref_mod.available():
            rb = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), case.n_fluid, case.n_wall, case.n_cells)
            rb.load_case(case)
            ref = ref_mod.ReferencePath(pkg.abi, case, rb)
            try:
                ref.rebuild()
                ref.fetch_geometry()
                _compare_geometry(dev, rb, "reference", rep.setdefault("reference", {}))
                ref.provision()
                ref.fetch_moments(p)
                ref.fetch_provision()
                ref.assemble_ppe()
                nnz = case.n_fluid + int(rb.csr_rows("fluid")[0][-1])
                ref.fetch_ppe(nnz)
                ctx.prepare_moments(dev, p, [0, 1])
                ctx.provision(dev, p)
                ctx.assemble_ppe(dev, p)
                g = _dev_ppe(dev, nnz)
                assert np.array_equal(g["row_offsets"], rb.ppe["row_offsets"])
                assert np.array_equal(g["col_indices"], rb.ppe["col_indices"][:nnz])
                rr = rep["reference"]
                for kind in (0, 1):
                    gm = _dev_moment(dev, kind)
                    hm = rb.moments[kind]
                    ok = hm["info"] == 0
                    gi = gm["inverse_matrices"].reshape(-1, 81)[ok]
                    hi = hm["inverse_matrices"].reshape(-1, 81)[ok]
                    rr[f"inverse_{kind}_max_rel"] = float(
                        (np.max(np.abs(gi - hi), axis=1) / np.max(np.abs(hi), axis=1)).max())
                    rr[f"inverse_{kind}_max_over_eps_kappa"] = inverse_err_over_kappa(
                        gi, hi, hm["moment_trace"][ok], hm["regularization_added"][ok])
                    assert rr[f"inverse_{kind}_max_over_eps_kappa"] <= INVERSE_EPS_FACTOR
                for k in ("values", "rhs", "divergence", "pressure_laplacian"):
                    b = rb.ppe[k][:nnz] if k == "values" else rb.ppe[k]
                    rr[f"ppe_{k}"] = rel_err(g[k], b)
                    assert rr[f"ppe_{k}"] < REFERENCE_RTOL, ("reference ppe", k)
                ref.correction()
                ref.fetch_correction()
                ctx.pressure_correction(dev, p)
                f = dev.numpy("fluid")
                for k, e in {**vec_err(f, rb.fluid, ("x", "y", "z")),
                             **vec_err(f, rb.fluid, ("vx", "vy", "vz"), extra_scale=rb.temporary_velocity)}.items():
                    rr[f"corrected_{k}"] = e
                    assert e < REFERENCE_RTOL, ("reference corrected", k, e)
                # the rebuild on the moved particles
                ref.rebuild()
                ref.fetch_geometry()
                ctx.build_neighbor_lists(dev, p)
                ctx.classify_surface(dev, p)
                _compare_geometry(dev, rb, "reference rebuild", rep.setdefault("reference_rebuild", {}))
            finally:
                ref.close()
            del ref, rb
            # back to the stated input for the oracle comparison
            dev.load_case(case)
            ctx.build_neighbor_lists(dev, p)
            ctx.classify_surface(dev, p)
        else:
            rep["reference"] = "oracle/_ref not built: reference comparison skipped"

        # 2. the oracle: integers bit for bit, floats stage by stage
        host = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), case.n_fluid, case.n_wall, case.n_cells)
        host.load_case(case)
        assert oracle.build_neighbor_lists(host, p)[0] == 0
        assert oracle.classify_surface(host, p) == 0
        _compare_geometry(dev, host, "oracle", rep.setdefault("oracle_geometry", {}))
        _float_stages(pkg, ctx, oracle, dev, host, p, rep, "at_rest")

        # the rebuild after the step, on the device's moved particles
        f = dev.numpy("fluid")
        for k in ("x", "y", "z"):
            host.fluid[k][:] = f[k]
        ctx.build_neighbor_lists(dev, p)
        ctx.classify_surface(dev, p)
        assert oracle.build_neighbor_lists(host, p)[0] == 0
        assert oracle.classify_surface(host, p) == 0
        _compare_geometry(dev, host, "oracle rebuild", rep.setdefault("oracle_rebuild", {}))

        # 3. the same geometry from a moving state
        host.load_case(case)
        dev.load_case(case)
        sw = _swirl(case.fluid)
        for k, v in sw.items():
            host.fluid[k][:] = v
            dev.alloc.copy_(dev.fluid[k], v)
        ctx.build_neighbor_lists(dev, p)
        ctx.classify_surface(dev, p)
        assert oracle.build_neighbor_lists(host, p)[0] == 0
        assert oracle.classify_surface(host, p) == 0
        _float_stages(pkg, ctx, oracle, dev, host, p, rep, "moving")
    finally:
        ctx.close()
    rep["seconds"] = round(time.perf_counter() - t0, 1)
    print(f"\n{label}: " + json.dumps(rep, indent=1, default=float))
    out = os.environ.get("LSMPS_PARITY_REPORT")
    if out:
        with open(out, "w") as fh:
            json.dump(_report, fh, indent=1, default=float)
