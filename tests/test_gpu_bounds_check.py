"""The bounds-checked build (liblsmps_b200_checked.so, -DLSMPS_BOUNDS_CHECK).

1. On a valid dam break it computes the same step as the normal build, bit
   for bit (the checks read the tables and change nothing).
2. Neighbour tables and PPE matrices with one bad entry (an index past the
   particle set, an offset past the table's capacity, offsets that go
   backwards) are refused with LSMPS_INVALID_ARGUMENT by every entry point
   that reads them, before any kernel reads the table; after the table is
   repaired the same context runs the call successfully.

Only the checked library is ever given a bad table (in a child process, so
that the normal library of the test session is not replaced).
"""

import json
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent(r"""
    import json, sys
    import numpy as np
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    pkg = ge.load_package()
    import importlib
    api = importlib.import_module("lsmps3d_b200.api")
    abi = pkg.abi
    assert api._lib._name.endswith("liblsmps_b200_checked.so"), api._lib._name
    import torch

    case = pkg.cases.dam_break(20, 10, 20)
    p = case.params
    ctx = api.Context(0)
    dev = api.device_buffers(case)
    ctx.build_neighbor_lists(dev, p)
    ctx.classify_surface(dev, p)
    ctx.step(dev, p)
    f = dev.numpy("fluid")
    np.savez(OUT, **{k: f[k] for k in ("x", "y", "z", "vx", "vy", "vz", "pressure", "surface_type")})

    results = {}

    def expect_invalid(name, call):
        try:
            call()
        except api.LsmpsError as e:
            results[name] = abi.STATUS_NAMES.get(e.status, e.status)
            return
        results[name] = "OK"

    def corrupt(t, k, v):
        old = int(t[k].item())
        t[k] = v
        torch.cuda.synchronize()
        return old

    dev = api.device_buffers(case)
    ctx.build_neighbor_lists(dev, p)
    ctx.classify_surface(dev, p)
    nf, nw = case.n_fluid, case.n_wall
    fo, fi = dev.fluid_neighbors["offsets"], dev.fluid_neighbors["indices"]
    wo, wi = dev.wall_neighbors["offsets"], dev.wall_neighbors["indices"]
    k = int(fo[nf // 2].item())
    kw = int(wo[int(np.argmax(np.diff(wo.cpu().numpy())))].item())
    bad = {
        "fluid index past the fluid": (fi, k, nf + 3),
        "negative fluid index": (fi, k, -1),
        "wall index past the walls": (wi, kw, nw),
        "fluid offset past the capacity": (fo, nf // 3, dev.cap_f + 100),
        "fluid offsets backwards": (fo, nf // 3 + 1, 0),
        "wall offset past the capacity": (wo, nf, dev.cap_w + 1),
    }
    for what, (t, at, v) in bad.items():
        old = corrupt(t, at, v)
        expect_invalid(what + ": classify_surface", lambda: ctx.classify_surface(dev, p))
        expect_invalid(what + ": prepare_moments", lambda: ctx.prepare_moments(dev, p, [0, 1]))
        expect_invalid(what + ": provision", lambda: ctx.provision(dev, p))
        expect_invalid(what + ": step", lambda: ctx.step(dev, p))
        corrupt(t, at, old)
    # valid tables again: the same context runs every stage
    ctx.classify_surface(dev, p)
    ctx.prepare_moments(dev, p, [0, 1])
    ctx.provision(dev, p)
    ctx.assemble_ppe(dev, p)
    ppe_cols, ppe_rows = dev.ppe["col_indices"], dev.ppe["row_offsets"]
    kp = int(ppe_rows[nf // 2].item()) + 1
    for what, (t, at, v) in {"PPE column past the rows": (ppe_cols, kp, nf),
                             "PPE row offset past the capacity": (ppe_rows, nf // 2, dev.nnz_cap + 1)}.items():
        old = corrupt(t, at, v)
        expect_invalid(what + ": solve_ppe", lambda: ctx.solve_ppe(dev))
        corrupt(t, at, old)
    old = corrupt(fi, k, nf + 3)
    expect_invalid("fluid index past the fluid: assemble_ppe", lambda: ctx.assemble_ppe(dev, p))
    expect_invalid("fluid index past the fluid: pressure_correction", lambda: ctx.pressure_correction(dev, p))
    corrupt(fi, k, old)
    ctx.assemble_ppe(dev, p)
    ctx.solve_ppe(dev)
    ctx.pressure_correction(dev, p)
    results["repaired"] = "OK"
    ctx.close()
    print(json.dumps(results))
""")


def test_checked_build_same_step_and_refuses_bad_tables(pkg, device_api, tmp_path):
    checked = os.path.join(ROOT, "lsmps-3d_b200", pkg.abi.CHECKED_LIB_NAME)
    importlib = __import__("importlib")
    importlib.import_module("lsmps3d_b200.build").build_all(bounds_check=True)
    out = str(tmp_path / "checked_step.npz")
    env = dict(os.environ, LSMPS_B200_LIBRARY=checked)
    src = f"ROOT = {ROOT!r}\nOUT = {out!r}\n" + CHILD
    proc = subprocess.run([sys.executable, "-c", src], env=env, capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stdout[-2000:] + proc.stderr[-4000:]
    results = json.loads(proc.stdout.strip().splitlines()[-1])
    for name, status in results.items():
        print(f"{name}: {status}")
    assert results.pop("repaired") == "OK"
    assert results and all(s == "INVALID_ARGUMENT" for s in results.values()), results

    # the normal build on the same case, same calls
    case = pkg.cases.dam_break(20, 10, 20)
    p = case.params
    ctx = device_api.Context(0)
    try:
        dev = device_api.device_buffers(case)
        ctx.build_neighbor_lists(dev, p)
        ctx.classify_surface(dev, p)
        ctx.step(dev, p)
        f = dev.numpy("fluid")
    finally:
        ctx.close()
    got = np.load(out)
    for k in got.files:
        assert np.array_equal(got[k], f[k]), k
