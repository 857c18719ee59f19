"""The C++17 drop-in exports the reference's module API (no GPU needed).

Every external symbol in namespace lsmps3d that the reference's six hot-path
module objects define (built from its sources into oracle/_ref/obj/) must be
defined by liblsmps3d_dropin.so, so a program linked against those modules
links against the drop-in instead; and every C ABI symbol the drop-in uses
must be exported by liblsmps_b200.so.
"""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "lsmps-3d_b200", "dropin", "_build", "liblsmps3d_dropin.so")
LIB = os.path.join(ROOT, "lsmps-3d_b200", "liblsmps_b200.so")
REF_OBJ = os.path.join(ROOT, "oracle", "_ref", "obj")
MODULES = ["neighbor_search", "surface_detection", "moment_matrix", "explicit_update", "ppe_matrix",
           "pressure_correction"]

if shutil.which("nm") is None or not os.path.exists(DROPIN):
    pytest.skip("drop-in not built (it compiles against the reference's headers)", allow_module_level=True)


def nm(path, *flags):
    out = subprocess.run(["nm", *flags, path], capture_output=True, text=True, check=True).stdout
    syms = set()
    for line in out.splitlines():
        parts = line.split(maxsplit=2)
        if len(parts) == 3 and parts[1] in ("T", "W", "U", "V", "B", "D", "R"):
            syms.add((parts[1], parts[2]))
        elif len(parts) == 2 and parts[0] == "U":
            syms.add(("U", parts[1]))
    return syms


def defined(syms):
    return {s for kind, s in syms if kind != "U"}


def test_dropin_defines_reference_module_api():
    if not all(os.path.exists(os.path.join(REF_OBJ, m + ".o")) for m in MODULES):
        pytest.skip("reference module objects not built")
    ours = defined(nm(DROPIN, "-D", "--defined-only"))
    missing = []
    for m in MODULES:
        for kind, s in nm(os.path.join(REF_OBJ, m + ".o"), "--defined-only", "--extern-only"):
            if kind not in ("T", "W"):
                continue
            demangled = subprocess.run(["c++filt", s], capture_output=True, text=True).stdout.strip()
            # namespace-scope API of lsmps3d: skip the anonymous namespace, CUDA
            # kernel stubs, library template instances and the reference's
            # unexported helpers (not declared in any of its headers)
            if not demangled.startswith(("lsmps3d::", "void lsmps3d::")) and "lsmps3d::" not in demangled.split("(")[0]:
                continue
            if any(t in demangled for t in ("(anonymous namespace)", "__device_stub", "thrust::", "cub::",
                                            "make_matrix_request", "SimulationConfig::SimulationConfig",
                                            "std::unique_ptr")):
                continue
            if s not in ours:
                missing.append(demangled)
    assert not missing, missing


def test_dropin_c_abi_imports_resolve():
    imports = {s for kind, s in nm(DROPIN, "-D") if kind == "U" and s.startswith("lsmps_")}
    assert imports, "the drop-in forwards to the C ABI"
    exported = defined(nm(LIB, "-D", "--defined-only"))
    assert imports <= exported, sorted(imports - exported)
