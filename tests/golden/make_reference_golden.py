"""Writes tests/golden/reference_<case>.npz: outputs of the reference's own
CUDA path (oracle/_ref/libref_lsmps.so, built from the reference sources) on
small seeded cases, stage by stage:

  geometry   rebuild_geometry (cell lists, CSR tables, labels)
  provision  moments of the step's generation and u*
  ppe        PPE CSR rows, rhs, divergence, wall term
  correction corrected positions/velocities, pressure gradient, shifting
  rebuilt    labels and CSR after the step's neighbour rebuild

Inputs are not stored: they are regenerated bit-for-bit by the seeded case
generator (lsmps3d_b200.cases), and a SHA-256 of the input arrays is stored
to catch any drift.  Inverse matrices are stored for a seeded sample of rows.

Run on a machine with a GPU and the built reference library:
    python tests/golden/make_reference_golden.py [outdir]
"""

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import __graft_entry__ as ge  # noqa: E402

GOLDEN_CASES = {
    "hydrostatic_10": ("hydrostatic", dict(n=10, l0=0.01)),
    "dam_break_12x6x12": ("dam_break", dict(nx=12, ny=6, nz=12, l0=0.005)),
    "splash_20x6x20": ("splash", dict(nx=20, ny=6, nz=20, l0=0.0025)),
}
INVERSE_SAMPLE = 48


def input_digest(case) -> str:
    h = hashlib.sha256()
    for group in (case.fluid, case.walls):
        for k in sorted(group):
            h.update(k.encode())
            h.update(np.ascontiguousarray(group[k]).tobytes())
    for name, _ in type(case.params)._fields_:
        v = getattr(case.params, name)
        h.update(repr(list(v) if hasattr(v, "__len__") else (v if not hasattr(v, "_fields_") else
                 (list(v.origin), v.cell_size, list(v.dims)))).encode())
    return h.hexdigest()


def sample_rows(n: int) -> np.ndarray:
    rng = np.random.default_rng(2024)
    return np.sort(rng.choice(n, size=min(n, INVERSE_SAMPLE), replace=False))


def run_case(pkg, ref_mod, name):
    kind, kw = GOLDEN_CASES[name]
    case = pkg.cases.CASES[kind](**kw)
    p = case.params
    b = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), case.n_fluid, case.n_wall, case.n_cells)
    b.load_case(case)
    ref = ref_mod.ReferencePath(pkg.abi, case, b)
    out = {"input_sha256": np.array(input_digest(case))}
    ref.rebuild()
    tf, tw = ref.fetch_geometry()
    for which, d in (("fluid", b.fluid_cells), ("wall", b.wall_cells)):
        for k, v in d.items():
            out[f"geometry/{which}_cells/{k}"] = v.copy()
    for which in ("fluid", "wall"):
        off, idx = b.csr_rows(which)
        out[f"geometry/{which}_offsets"] = off
        out[f"geometry/{which}_indices"] = idx
    out["geometry/surface_type"] = b.fluid["surface_type"].copy()
    ref.provision()
    ref.fetch_moments(p)
    ref.fetch_provision()
    rows = sample_rows(case.n_fluid)
    out["provision/inverse_rows"] = rows
    for kind in (0, 1):
        m = b.moments[kind]
        out[f"provision/moment{kind}/inverse"] = m["inverse_matrices"].reshape(-1, 81)[rows].copy()
        for k in ("moment_trace", "regularization_added", "info", "inversion_count"):
            out[f"provision/moment{kind}/{k}"] = m[k].copy()
    for k, v in b.temporary_velocity.items():
        out[f"provision/temporary_{k}"] = v.copy()
    for k, v in b.temporary_wall_velocity.items():
        out[f"provision/temporary_wall_{k}"] = v.copy()
    ref.assemble_ppe()
    written = case.n_fluid + tf
    nnz = ref.fetch_ppe(written)
    out["ppe/active_nnz"] = np.array(nnz)
    out["ppe/row_offsets"] = b.ppe["row_offsets"].copy()
    out["ppe/col_indices"] = b.ppe["col_indices"][:written].copy()
    out["ppe/values"] = b.ppe["values"][:written].copy()
    for k in ("rhs", "divergence", "pressure_laplacian"):
        out[f"ppe/{k}"] = b.ppe[k].copy()
    ref.correction()
    ref.fetch_correction()
    for k in ("x", "y", "z", "vx", "vy", "vz", "pressure"):
        out[f"correction/{k}"] = b.fluid[k].copy()
    for k in ("x", "y", "z"):
        out[f"correction/gradient_{k}"] = b.pressure_gradient[k].copy()
        out[f"correction/shift_{k}"] = b.ps_displacement[k].copy()
    ref.rebuild()
    ref.fetch_geometry()
    out["rebuilt/surface_type"] = b.fluid["surface_type"].copy()
    for which in ("fluid", "wall"):
        off, idx = b.csr_rows(which)
        out[f"rebuilt/{which}_offsets"] = off
        out[f"rebuilt/{which}_indices"] = idx
    ref.close()
    return out


def main():
    outdir = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))
    pkg = ge.load_package()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reference as ref_mod

    for name in GOLDEN_CASES:
        data = run_case(pkg, ref_mod, name)
        path = os.path.join(outdir, f"reference_{name}.npz")
        np.savez_compressed(path, **data)
        print(f"wrote {path} ({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
