"""The C ABI without a GPU: every function include/lsmps_b200.h declares is
exported by the library and bound in abi.py, and the ctypes structs have the
C layout (checked against offsetof/sizeof from a compiled C program)."""

import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lsmps_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lsmps_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib(pkg):
    import importlib

    importlib.import_module("lsmps3d_b200.build").build_all()
    return pkg.abi.load_library()


def test_header_and_bindings_agree(pkg):
    assert declared_functions() == sorted(pkg.abi.exported_names())


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib._name], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (lsmps_[a-z0-9_]+)$", out, flags=re.M))
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing


def test_host_only_entry_points(lib, pkg):
    # No device work: the reference number density (surface_detection.cu:494-520)
    # and the status strings.
    assert abs(lib.lsmps_reference_number_density(0.01, 0.031) - 29.993) < 5e-4
    assert lib.lsmps_reference_number_density(-1.0, 0.031) < 0
    assert lib.lsmps_status_string(1) == b"CAPACITY_EXCEEDED"
    p = pkg.abi.Params()
    lib.lsmps_params_default(ctypes.byref(p))
    d = pkg.abi.default_params()
    for name, _ in pkg.abi.Params._fields_:
        a, b = getattr(p, name), getattr(d, name)
        if name == "grid":
            assert a.cell_size == b.cell_size and list(a.dims) == list(b.dims)
        elif name == "gravity":
            assert list(a) == list(b)
        else:
            assert a == b, name


def test_context_options_reject_a_missing_context(lib, pkg):
    # Host-side argument checks of the context switches (no device touched).
    inv = pkg.abi.INVALID_ARGUMENT
    assert lib.lsmps_ctx_set_sorted_rows(None, 1) == inv
    assert lib.lsmps_ctx_copy_sorted_rows(None, None, 0) == inv
    assert lib.lsmps_ctx_set_cell_order(None, 1) == inv
    assert lib.lsmps_ctx_set_step_events(None, None, None, None) == inv


def test_solver_options_default(lib, pkg):
    o = pkg.abi.SolverOptions()
    lib.lsmps_solver_options_default(ctypes.byref(o))
    d = pkg.abi.default_solver_options()
    for name, _ in pkg.abi.SolverOptions._fields_:
        assert getattr(o, name) == getattr(d, name), name


def test_time_state_init(lib, pkg):
    lim = pkg.abi.TimeLimits(min_time_step=1e-6, max_time_step=1e-3, growth_factor=1.05, cfl=0.2,
                             particle_spacing=0.01, final_time=1.0)
    st = pkg.abi.TimeState()
    for dt, want in ((1e-4, 1e-4), (1.0, 1e-3), (1e-9, 1e-6)):
        lib.lsmps_time_state_init(ctypes.byref(lim), dt, ctypes.byref(st))
        assert st.time_step == want and st.current_time == 0.0 and st.step_index == 0


STRUCTS = ["lsmps_fluid", "lsmps_walls", "lsmps_grid", "lsmps_cells", "lsmps_csr", "lsmps_vector",
           "lsmps_surface_diagnostics", "lsmps_moment", "lsmps_csr_matrix", "lsmps_ppe", "lsmps_params",
           "lsmps_step_state", "lsmps_operator_out", "lsmps_step_operator_out", "lsmps_solver_options",
           "lsmps_solver_report", "lsmps_time_limits", "lsmps_time_state"]
PY = {"lsmps_fluid": "Fluid", "lsmps_walls": "Walls", "lsmps_grid": "Grid", "lsmps_cells": "Cells",
      "lsmps_csr": "Csr", "lsmps_vector": "Vector", "lsmps_surface_diagnostics": "SurfaceDiagnostics",
      "lsmps_moment": "Moment", "lsmps_csr_matrix": "CsrMatrix", "lsmps_ppe": "Ppe", "lsmps_params": "Params",
      "lsmps_step_state": "StepState", "lsmps_operator_out": "OperatorOut",
      "lsmps_step_operator_out": "StepOperatorOut",
      "lsmps_solver_options": "SolverOptions", "lsmps_solver_report": "SolverReport",
      "lsmps_time_limits": "TimeLimits", "lsmps_time_state": "TimeState"}


def test_struct_layout_matches_header(pkg, tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "lsmps_b200.h"', 'int main(void) {']
    for s in STRUCTS:
        lines.append(f'  printf("{s} size %zu\\n", sizeof({s}));')
        for name, _ in getattr(pkg.abi, PY[s])._fields_:
            lines.append(f'  printf("{s} {name} %zu\\n", offsetof({s}, {name}));')
    lines.append("  return 0; }")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    for line in filter(None, out):
        s, field, val = line.split()
        cls = getattr(pkg.abi, PY[s])
        got = ctypes.sizeof(cls) if field == "size" else getattr(cls, field).offset
        assert got == int(val), (s, field, got, val)


def test_reference_view_layout_identical(pkg):
    """The ABI views mirror the reference's views with real = double:
    FluidParticleSoA is size_t + 7 real* + int* (particle_data.cuh:7-17),
    CellGrid is Vec3 + real + Int3 (cell_list.cuh:7-15)."""
    assert ctypes.sizeof(pkg.abi.Fluid) == 8 + 8 * 8
    assert ctypes.sizeof(pkg.abi.Walls) == 8 + 9 * 8
    assert ctypes.sizeof(pkg.abi.Grid) == 48
    assert ctypes.sizeof(pkg.abi.Cells) == 16 + 4 * 8
    assert ctypes.sizeof(pkg.abi.Csr) == 16 + 2 * 8
