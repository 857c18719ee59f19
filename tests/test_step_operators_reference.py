"""CPU check of the torch FP64 restatement of the step's operators with
their wall terms (the autograd reference of tests/test_gpu_step_adjoint.py)
against the oracle's stages on the same state: velocity Laplacian
(provision), PPE rows, divergence, wall Neumann term and right-hand side,
pressure gradient.  This pins the differentiated operators to the
reference's algorithm before any GPU comparison."""

import ctypes

import numpy as np

from test_gpu_step_adjoint import fields, torch_step_operators


def test_torch_step_operators_equal_the_oracle_stages(pkg, oracle):
    import torch

    case = pkg.cases.lattice_box(n=6, l0=0.01)
    p = case.params
    b = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), case.n_fluid, case.n_wall, case.n_cells)
    b.load_case(case)
    assert oracle.build_neighbor_lists(b, p)[0] == 0
    assert oracle.classify_surface(b, p) == 0
    off, idx = b.csr_rows("fluid")
    woff, widx = b.csr_rows("wall")
    lab = b.fluid["surface_type"].copy()
    assert (lab == 2).any() and woff[-1] > 0
    u, pr, uw = fields(case)
    f, w = case.fluid, case.walls
    ref = torch_step_operators(torch.from_numpy(np.stack([f[k] for k in "xyz"], 1).copy()), torch.from_numpy(u),
                               torch.from_numpy(pr), torch.from_numpy(np.stack([w[k] for k in "xyz"], 1).copy()),
                               torch.from_numpy(np.stack([w[k] for k in ("normal_x", "normal_y", "normal_z")], 1).copy()),
                               torch.from_numpy(uw), off, idx, woff, widx, lab, p)
    ref = {k: v.numpy() for k, v in ref.items()}
    for c, k in enumerate(("vx", "vy", "vz")):
        b.fluid[k][:] = u[:, c]
        b.walls[k][:] = uw[:, c]
        b.temporary_velocity[k][:] = u[:, c]
        b.temporary_wall_velocity[k][:] = uw[:, c]
    b.fluid["pressure"][:] = pr
    assert oracle.prepare_moment(b, p, 0) == 0 and oracle.prepare_moment(b, p, 1) == 0
    assert oracle.provision(b, p) == 0
    lap = b.numpy("velocity_laplacian")
    # provision overwrote u* (fluid and walls) with u + dt (nu lap + g); the PPE takes u* = u here
    for c, k in enumerate(("vx", "vy", "vz")):
        b.temporary_velocity[k][:] = u[:, c]
        b.temporary_wall_velocity[k][:] = uw[:, c]
    assert oracle.assemble_ppe(b, p) == 0
    gv = b.vector_view(b.pressure_gradient)
    assert oracle.L.oracle_pressure_gradient(
        ctypes.byref(b.fluid_view()), ctypes.byref(b.walls_view()), ctypes.byref(b.csr_view("fluid")),
        ctypes.byref(b.csr_view("wall")), b.fluid["pressure"].ctypes.data, ctypes.byref(p),
        ctypes.byref(b.moment_view(1)), ctypes.byref(gv)) == 0
    grad = b.numpy("pressure_gradient")
    nnz = int(b.ppe["row_offsets"][-1])
    pairs = [("lap_" + c, lap[c], ref["lap_" + c]) for c in "xyz"] + \
            [("grad_" + c, grad[c], ref["grad_" + c]) for c in "xyz"] + \
            [("ppe_values", b.ppe["values"][:nnz], ref["ppe_values"]), ("ppe_rhs", b.ppe["rhs"], ref["ppe_rhs"]),
             ("divergence", b.ppe["divergence"], ref["divergence"]),
             ("wall_rhs", b.ppe["pressure_laplacian"], ref["wall_rhs"])]
    for name, o, r in pairs:
        err = np.max(np.abs(o - r)) / max(np.max(np.abs(o)), 1e-300)
        assert err < 1e-12, (name, err)
