"""One small LSMPS step on cuda:0 through the C ABI, checked against the
CPU oracle (used by __graft_entry__.smoke())."""

from __future__ import annotations

import numpy as np

from . import cases
from .buffers import NumpyAlloc, StepBuffers, TorchAlloc


def run(oracle_module) -> None:
    from . import abi, api

    case = cases.dam_break(nx=12, ny=6, nz=12, l0=0.005)
    p = case.params
    dev = StepBuffers(TorchAlloc("cuda:0"), case.n_fluid, case.n_wall, case.n_cells)
    host = StepBuffers(NumpyAlloc(), case.n_fluid, case.n_wall, case.n_cells)
    dev.load_case(case)
    host.load_case(case)
    ctx = api.Context(0)
    orc = oracle_module.Oracle(abi)
    ctx.build_neighbor_lists(dev, p)
    ctx.classify_surface(dev, p)
    orc.build_neighbor_lists(host, p)
    orc.classify_surface(host, p)
    launches0 = ctx.launch_count
    ctx.step(dev, p)
    st, _ = orc.step(host, p)
    if st != 0:
        raise RuntimeError(f"oracle step failed: {st}")
    go, gi = dev.csr_rows("fluid")
    ho, hi = host.csr_rows("fluid")
    if not (np.array_equal(go, ho) and np.array_equal(gi, hi)):
        raise AssertionError("fluid CSR differs from the oracle")
    if not np.array_equal(dev.numpy("fluid")["surface_type"], host.fluid["surface_type"]):
        raise AssertionError("surface labels differ from the oracle")
    f = dev.numpy("fluid")
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        o = host.fluid[k]
        err = np.max(np.abs(f[k] - o)) / max(float(np.max(np.abs(o))), 1e-300)
        if err > 1e-7:
            raise AssertionError(f"{k}: relative error {err:.3e} against the oracle")
    print(f"smoke ok: {case.n_fluid} fluid / {case.n_wall} wall particles, "
          f"{ctx.launch_count - launches0} kernel launches in one step")
    ctx.close()
