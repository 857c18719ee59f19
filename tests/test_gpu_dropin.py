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
