"""The C++17 drop-in (lsmps-3d_b200/dropin) under the reference's own unit tests.

`make -C oracle unit` builds each of the reference's unit-test programs
(tests/unit/smoke_*.cu of lsmps-3D, from its sources) twice: linked with the
reference's six module sources (oracle/_ref/unit/reference/) and linked with
the drop-in library, which replaces those six sources and keeps the
reference's core/runtime.cu (oracle/_ref/unit/dropin/).  Each program checks
its own known answers (labels, CSR rows, moment views, Laplacian, PPE row,
divergence, RHS, gradient, corrected velocity and position, workspace byte
accounting) and exits 0 when they hold.

smoke_ppe_matrix.cu also requires configs/amgx_ppe.json, relative to the
working directory, to name a GMRES solver (the lsmps-3D repository carries
that file; the snapshot these programs were built from does not), so the
programs run in a directory holding a configuration of that form.
"""

import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
UNIT = os.path.join(ROOT, "oracle", "_ref", "unit")
CHECKS = os.path.join(ROOT, "lsmps-3d_b200", "dropin", "_build", "dropin_errors")
TESTS = ["smoke_neighbor_search", "smoke_surface_detection", "smoke_moment_matrix",
         "smoke_provision_explicit_update", "smoke_ppe_matrix", "smoke_pressure_correction",
         "smoke_particle_copy"]

if not os.path.exists(os.path.join(UNIT, "dropin", TESTS[0])):
    pytest.skip("oracle/_ref/unit not built (the reference sources are needed to build it)",
                allow_module_level=True)

# The solver settings of the reference's built-in AMGX configuration
# (ppe_matrix.cu:604-610) in AMGX's JSON form.
AMGX_CONFIG = {
    "config_version": 2,
    "solver": {"solver": "GMRES", "preconditioner": {"solver": "NOSOLVER"}, "max_iters": 100,
               "tolerance": 1e-06, "convergence": "RELATIVE_INI", "norm": "L2", "use_scalar_norm": 1},
}


@pytest.fixture(scope="module")
def workdir(tmp_path_factory):
    d = tmp_path_factory.mktemp("unit")
    os.makedirs(d / "configs")
    with open(d / "configs" / "amgx_ppe.json", "w") as f:
        json.dump(AMGX_CONFIG, f, indent=2)
        f.write("\n")
    text = (d / "configs" / "amgx_ppe.json").read_text()
    assert '"solver": "GMRES"' in text
    return d


def run(path, cwd, *args, env=None):
    return subprocess.run([path, *args], cwd=cwd, capture_output=True, text=True, timeout=300, env=env)


@pytest.mark.parametrize("name", TESTS)
def test_reference_unit_test_on_dropin(name, workdir):
    ref = run(os.path.join(UNIT, "reference", name), workdir)
    print(f"{name} on the reference modules: exit {ref.returncode} {ref.stderr.strip()[:300]}")
    got = run(os.path.join(UNIT, "dropin", name), workdir)
    print(f"{name} on the drop-in: exit {got.returncode} {got.stderr.strip()[:300]}")
    assert got.returncode == 0, got.stdout + got.stderr


@pytest.mark.parametrize("case,message", [
    ("capacity", "Neighbor list capacity exceeded: required 6, capacity 5"),
    ("unprepared", "Moment operators must prepare matrices before computing operators"),
    ("grid", "Invalid cell grid configuration"),
])
def test_dropin_error_convention(case, message, workdir):
    # The reference's convention: one line on stderr, exit status EXIT_FAILURE.
    r = run(CHECKS, workdir, case)
    assert r.returncode == 1, r.stdout + r.stderr
    assert r.stderr.strip() == message
    # LSMPS_DROPIN_THROW=1: the same message as std::runtime_error.
    env = dict(os.environ, LSMPS_DROPIN_THROW="1")
    r = run(CHECKS, workdir, case, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == f"caught: {message}"


# --- the reference's diagnostic programs -------------------------------------

def parse_vtk(path):
    """Point fields of a legacy ASCII VTK file written by the reference's
    LegacyVtkWriter: {name: array} (vectors as (n, 3)), plus "POINTS"."""
    import numpy as np

    tok = open(path).read().split()
    fields, i = {}, 0
    n = None
    while i < len(tok):
        t = tok[i]
        if t == "POINTS":
            n = int(tok[i + 1])
            fields["POINTS"] = np.array(tok[i + 3:i + 3 + 3 * n], dtype=float).reshape(n, 3)
            i += 3 + 3 * n
        elif t == "SCALARS":
            name = tok[i + 1]
            start = i + 6  # SCALARS name type 1 LOOKUP_TABLE default
            fields[name] = np.array(tok[start:start + n], dtype=float)
            i = start + n
        elif t == "VECTORS":
            name = tok[i + 1]
            fields[name] = np.array(tok[i + 3:i + 3 + 3 * n], dtype=float).reshape(n, 3)
            i += 3 + 3 * n
        else:
            i += 1
    return fields


def parse_csv(path):
    import csv

    with open(path) as f:
        rows = list(csv.reader(f))
    return rows[0], rows[1:]


def compare_outputs(ref_dir, our_dir, skip_fields=(), rtol=1e-6, scale_with=None):
    """Every CSV and VTK file the reference build wrote, field by field:
    integer-valued columns exactly, real ones within rtol of the field's scale
    (the files carry 9 significant digits).  scale_with maps a field that is a
    cancellation (a residual) to the fields whose magnitude sets its rounding
    error."""
    scale_with = scale_with or {}
    import numpy as np

    worst = {}
    files = sorted(p.relative_to(ref_dir) for p in ref_dir.rglob("*") if p.suffix in (".csv", ".vtk"))
    assert files, "the reference build wrote no output"
    for rel in files:
        a, b = ref_dir / rel, our_dir / rel
        assert b.exists(), rel
        if rel.suffix == ".csv":
            ha, ra = parse_csv(a)
            hb, rb = parse_csv(b)
            assert ha == hb and len(ra) == len(rb), rel
            for c, name in enumerate(ha):
                col_a = [r[c] for r in ra]
                col_b = [r[c] for r in rb]
                try:
                    va, vb = np.array(col_a, float), np.array(col_b, float)
                except ValueError:  # names (surface_type_name, expected_surface)
                    assert col_a == col_b, (rel, name)
                    continue
                if np.all(va == np.round(va)) and "count" in name or name in ("particle_id", "surface_type"):
                    assert np.array_equal(va, vb), (rel, name)
                scale = max(np.max(np.abs(va)), 1e-300)
                worst[f"{rel}:{name}"] = float(np.max(np.abs(va - vb)) / scale)
        else:
            fa, fb = parse_vtk(a), parse_vtk(b)
            assert sorted(fa) == sorted(fb), rel
            for name in fa:
                if name in skip_fields:
                    continue
                va, vb = fa[name], fb[name]
                if name in ("surface_type", "fluid_neighbor_count", "wall_neighbor_count", "ppe_matrix_row_nnz"):
                    assert np.array_equal(va, vb), (rel, name)
                scale = max([np.max(np.abs(va)), 1e-300] + [np.max(np.abs(fa[o])) for o in scale_with.get(name, ())])
                worst[f"{rel}:{name}"] = float(np.max(np.abs(va - vb)) / scale)
    bad = {k: v for k, v in worst.items() if v > rtol}
    return worst, bad


def test_complex_surface_diagnostics_program(workdir):
    # Five surface-detection cases (inclined plane, sine wave, droplet,
    # cylinder, stepped box): labels, counts, densities, anisotropies and
    # normals written by the reference's own program, through the drop-in.
    ref_out, our_out = workdir / "complex_ref", workdir / "complex_dropin"
    r = run(os.path.join(UNIT, "reference", "complex_surface_diagnostics"), workdir, "all", str(ref_out))
    assert r.returncode == 0, r.stderr
    g = run(os.path.join(UNIT, "dropin", "complex_surface_diagnostics"), workdir, "all", str(our_out))
    assert g.returncode == 0, g.stderr
    assert g.stdout.replace(str(our_out), "@") == r.stdout.replace(str(ref_out), "@")
    worst, bad = compare_outputs(ref_out, our_out, rtol=1e-7)
    print(f"complex surface diagnostics: {len(worst)} fields, worst relative difference "
          f"{max(worst.values()):.2e}")
    assert not bad, bad


def test_hydrostatic_surface_diagnostics_program(workdir):
    # Neighbours, labels, moments, provision, PPE rows and the pressure
    # operators of a half-full hydrostatic box.  The reference here has no
    # AMGX, so its program skips the solve: the drop-in runs with its solver
    # switched off (LSMPS_DROPIN_SOLVER=off) to take the same branch.
    ref_out, our_out = workdir / "hydro_ref", workdir / "hydro_dropin"
    r = run(os.path.join(UNIT, "reference", "hydrostatic_surface_diagnostics"), workdir, str(ref_out))
    assert r.returncode == 0, r.stderr
    env = dict(os.environ, LSMPS_DROPIN_SOLVER="off")
    g = run(os.path.join(UNIT, "dropin", "hydrostatic_surface_diagnostics"), workdir, str(our_out), env=env)
    assert g.returncode == 0, g.stderr
    # A p_true - b cancels to ~1e-6 of its operands: its error is measured
    # against the right-hand side and the residual with the wall term.
    worst, bad = compare_outputs(ref_out, our_out, rtol=1e-6, scale_with={
        "ppe_hydrostatic_residual": ("ppe_rhs", "ppe_hydrostatic_residual_plus_wall_rhs")})
    print(f"hydrostatic diagnostics: {len(worst)} fields, worst relative difference {max(worst.values()):.2e}")
    for k in sorted(worst, key=worst.get)[-5:]:
        print(f"  {k}: {worst[k]:.2e}")
    assert not bad, bad
    # and with the device solve (the drop-in's AmgxPpeSolver)
    g = run(os.path.join(UNIT, "dropin", "hydrostatic_surface_diagnostics"), workdir, str(workdir / "hydro_solve"))
    assert g.returncode == 0, g.stderr
    print("\n".join(line for line in g.stdout.splitlines() if "PPE" in line))


# --- the reference's simulation driver ---------------------------------------

def _write_driver_inputs(pkg, d, out_dir, final_time=2.0e-3):
    """A small jittered dam break (24 x 12 x 24 fluid, 3 wall layers) as the
    driver's CSV inputs and INI configuration (docs/implementation_notes.md:
    100-122 format; every double written in full precision)."""
    import numpy as np

    case = pkg.cases.CASES["dam_break"](nx=24, ny=12, nz=24, l0=0.005)
    p = case.params
    f, w = case.fluid, case.walls
    with open(d / "fluid.csv", "w") as fh:
        fh.write("x,y,z,vx,vy,vz\n")
        for row in zip(*(np.asarray(f[k], float) for k in ("x", "y", "z", "vx", "vy", "vz"))):
            fh.write(",".join(repr(float(v)) for v in row) + "\n")
    with open(d / "walls.csv", "w") as fh:
        fh.write("x,y,z,vx,vy,vz,normal_x,normal_y,normal_z\n")
        for row in zip(*(np.asarray(w[k], float) for k in ("x", "y", "z", "vx", "vy", "vz", "normal_x",
                                                               "normal_y", "normal_z"))):
            fh.write(",".join(repr(float(v)) for v in row) + "\n")
    r = repr
    ini = f"""[geometry]
particle_spacing={r(p.particle_spacing)}
support_radius={r(p.support_radius)}
near_surface_radius={r(p.near_surface_radius)}
cell_size={r(p.support_radius)}

[simulation]
time_step=1e-4
min_time_step=1e-6
max_time_step=2e-4
time_step_growth_factor=1.05
final_time={r(final_time)}
output_interval=1e-3
density={r(p.density)}
kinematic_viscosity={r(p.kinematic_viscosity)}
gravity_x={r(p.gravity[0])}
gravity_y={r(p.gravity[1])}
gravity_z={r(p.gravity[2])}

[surface]
splash_neighbor_threshold={p.splash_neighbor_threshold}
number_density_ratio_threshold={r(p.number_density_ratio_threshold)}
air_open_ratio_threshold={r(p.air_open_ratio_threshold)}
air_anisotropy_threshold={r(p.air_anisotropy_threshold)}
include_wall_neighbors={'true' if p.include_wall_neighbors else 'false'}
wall_normal_independence_threshold={r(p.wall_normal_independence_threshold)}

[lsmps]
regularization={r(p.lsmps_regularization)}
wall_weight_scale={r(p.lsmps_wall_weight_scale)}

[correction]
ps_displacement_scale={r(p.ps_displacement_scale)}
ps_min_distance_ratio={r(p.ps_min_distance_ratio)}
ps_max_displacement_ratio={r(p.ps_max_displacement_ratio)}
wall_clearance_ratio={r(p.wall_clearance_ratio)}
velocity_smoothing_strength={r(p.velocity_smoothing_strength)}

[files]
fluid_particle_file={d / 'fluid.csv'}
wall_particle_file={d / 'walls.csv'}
output_directory={out_dir}
vtk_file_prefix=dam_break
amgx_config_path={d / 'configs' / 'amgx_ppe.json'}
"""
    path = out_dir.parent / (out_dir.name + ".ini")
    path.write_text(ini)
    return path, case


def test_reference_driver_program(pkg, workdir):
    # The reference's whole time loop (src/app/simulation_driver.cu: CFL time
    # step, provision, PPE assembly, [solve], correction, rebuild, labels, VTK
    # output) built against the drop-in, against the same program built from
    # the reference's modules.  With the solve off on both sides (the
    # reference here has no AMGX), every VTK file the two write must agree:
    # labels exactly, the real fields to 1e-9 of their scale (14 steps; the
    # outputs are written with 9 significant digits).
    ref_ini, _ = _write_driver_inputs(pkg, workdir, workdir / "drv_ref")
    our_ini, _ = _write_driver_inputs(pkg, workdir, workdir / "drv_dropin")
    r = run(os.path.join(UNIT, "reference", "lsmps3d_driver"), workdir, str(ref_ini))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    env = dict(os.environ, LSMPS_DROPIN_SOLVER="off")
    g = run(os.path.join(UNIT, "dropin", "lsmps3d_driver"), workdir, str(our_ini), env=env)
    assert g.returncode == 0, g.stdout[-2000:] + g.stderr[-2000:]
    worst, bad = compare_outputs(workdir / "drv_ref", workdir / "drv_dropin", rtol=1e-9)
    print(f"driver outputs: {len(worst)} fields, worst relative difference {max(worst.values()):.2e}")
    for k in sorted(worst, key=worst.get)[-4:]:
        print(f"  {k}: {worst[k]:.2e}")
    assert not bad, bad
    # The same loop with the device PPE solve (the drop-in's AmgxPpeSolver).
    sol_ini, _ = _write_driver_inputs(pkg, workdir, workdir / "drv_solve")
    g = run(os.path.join(UNIT, "dropin", "lsmps3d_driver"), workdir, str(sol_ini))
    assert g.returncode == 0, g.stdout[-2000:] + g.stderr[-2000:]
    import numpy as np

    last = sorted((workdir / "drv_solve").rglob("*.vtk"))
    fields = parse_vtk([p for p in last if "wall" not in p.name][-1])
    assert np.all(np.isfinite(fields["pressure"])) and fields["pressure"].max() > 0.0
    print(f"with the device solve: final pressure max {fields['pressure'].max():.3e}")
