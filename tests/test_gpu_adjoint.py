"""The differentiable operator pair through the C ABI
(lsmps_operators_forward / lsmps_operators_backward).

Two checks of the hand-written adjoint:

* against an FP64 reference gradient: the same operators written directly in
  torch (float64, CPU) and differentiated by autograd, on a 12^3 jittered
  lattice, for the gradients with respect to the scalar field f, the vector
  field v and the positions;
* against FP64 central finite differences on the 64^3 = 262,144-particle
  jittered lattice: eps = 1e-6 l0 on 64 seeded particles, neighbour topology
  frozen (the CSR is an input), samples with a pair within 10 eps of r_e
  (where the weight's derivative jumps) skipped.

Inputs: f = sin(2 pi x/L) cos(2 pi y/L) + 0.1 z/L + N(0, 1e-3) (seed 4), the
cotangent of every output N(0, 1) (seed 5), samples seed 6.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FORWARD_RTOL = 1e-10
ADJOINT_RTOL = 1e-9
FD_RTOL = 1e-5


class Operators:
    """The operator pair on one particle set with a frozen CSR."""

    def __init__(self, pkg, device_api, case):
        import torch

        self.torch, self.pkg, self.api = torch, pkg, device_api
        self.p = case.params
        self.dev = device_api.device_buffers(case)
        self.ctx = device_api.Context(0)
        self.ctx.build_neighbor_lists(self.dev, self.p)
        self.n = case.n_fluid
        off, idx = self.dev.csr_rows("fluid")
        self.off, self.idx = off, idx
        self.k = int(off[-1])
        self.lib = device_api._lib

    def _fluid(self, x):
        v = self.pkg.abi.Fluid()
        v.count = self.n
        v.x, v.y, v.z = (t.data_ptr() for t in x)
        return v

    def _vec(self, ts):
        v = self.pkg.abi.Vector()
        v.count = self.n
        v.x, v.y, v.z = (t.data_ptr() for t in ts)
        return v

    def _out(self, d):
        o = self.pkg.abi.OperatorOut()
        o.count = self.n
        for k, t in d.items():
            setattr(o, k, t.data_ptr())
        return o

    def alloc_out(self):
        t = self.torch
        z = lambda m, dt=t.float64: t.zeros(m, dtype=dt, device="cuda")  # noqa: E731
        return {"grad_x": z(self.n), "grad_y": z(self.n), "grad_z": z(self.n), "laplacian": z(self.n),
                "divergence": z(self.n), "ppe_row_offsets": z(self.n + 1, t.int32),
                "ppe_col_indices": z(self.n + self.k, t.int32), "ppe_values": z(self.n + self.k),
                "ppe_rhs": z(self.n)}

    def forward(self, x, f, v):
        out = self.alloc_out()
        st = self.lib.lsmps_operators_forward(self.ctx.h, ctypes.byref(self._fluid(x)),
                                              ctypes.byref(self.dev.csr_view("fluid")), ctypes.byref(self.p),
                                              ctypes.c_void_p(f.data_ptr()), ctypes.byref(self._vec(v)),
                                              ctypes.byref(self._out(out)), None)
        self.ctx.check(st)
        return out

    def backward(self, x, f, v, cot):
        t = self.torch
        fbar = t.zeros(self.n, dtype=t.float64, device="cuda")
        vbar = [t.zeros(self.n, dtype=t.float64, device="cuda") for _ in range(3)]
        xbar = [t.zeros(self.n, dtype=t.float64, device="cuda") for _ in range(3)]
        st = self.lib.lsmps_operators_backward(self.ctx.h, ctypes.byref(self._fluid(x)),
                                               ctypes.byref(self.dev.csr_view("fluid")), ctypes.byref(self.p),
                                               ctypes.c_void_p(f.data_ptr()), ctypes.byref(self._vec(v)),
                                               ctypes.byref(self._out(cot)), None,
                                               ctypes.c_void_p(fbar.data_ptr()), ctypes.byref(self._vec(vbar)),
                                               ctypes.byref(self._vec(xbar)))
        self.ctx.check(st)
        return fbar, vbar, xbar


def fields(pkg, case):
    f_ = case.fluid
    L = 64 * case.l0
    f = (np.sin(2 * np.pi * f_["x"] / L) * np.cos(2 * np.pi * f_["y"] / L) + 0.1 * f_["z"] / L
         + 1e-3 * pkg.cases.normal(4, case.n_fluid))
    v = [np.cos(2 * np.pi * f_["y"] / L), np.sin(2 * np.pi * f_["z"] / L), f_["x"] / L]
    return f, v


def cotangents(pkg, ops):
    t = ops.torch
    g = pkg.cases.normal(5, 5 * ops.n + 2 * (ops.n + ops.k))
    names = ["grad_x", "grad_y", "grad_z", "laplacian", "divergence", "ppe_rhs"]
    cot, pos = {}, 0
    for name in names:
        cot[name] = t.from_numpy(g[pos:pos + ops.n].copy()).cuda()
        pos += ops.n
    cot["ppe_values"] = t.from_numpy(g[pos:pos + ops.n + ops.k].copy()).cuda()
    return cot


def torch_operators(x, f, v, off, idx, p):
    """The operators in plain torch float64 (the FP64 reference).  Matrix
    products are written as elementwise products and sums and torch runs on
    one thread here, so that the reference's own rounding does not depend on
    the BLAS kernel or the thread count of the process."""
    import torch

    threads = torch.get_num_threads()
    torch.set_num_threads(1)
    try:
        return _torch_operators(x, f, v, off, idx, p)
    finally:
        torch.set_num_threads(threads)


def _torch_operators(x, f, v, off, idx, p):
    import torch

    n = x.shape[0]
    re, lam = p.support_radius, p.lsmps_regularization
    off_t = torch.from_numpy(off.astype(np.int64))
    rows = torch.repeat_interleave(torch.arange(n), off_t[1:] - off_t[:-1])
    cols = torch.from_numpy(idx.astype(np.int64))
    d = x[cols] - x[rows]
    dist = torch.sqrt((d * d).sum(1))
    w = torch.clamp(1.0 - dist / re, min=0.0)
    s = d / re
    b = torch.stack([s[:, 0], s[:, 1], s[:, 2], s[:, 0] ** 2, s[:, 1] ** 2, s[:, 2] ** 2, s[:, 0] * s[:, 1],
                     s[:, 1] * s[:, 2], s[:, 2] * s[:, 0]], 1)
    S = torch.zeros(n, 9, 9, dtype=x.dtype).index_add(0, rows, w[:, None, None] * b[:, :, None] * b[:, None, :])
    tr = torch.diagonal(S, dim1=1, dim2=2).sum(1)
    reg = lam * torch.where(tr > 0, tr / 9.0, torch.ones_like(tr))
    M = S + reg[:, None, None] * torch.eye(9, dtype=x.dtype)
    X = torch.linalg.inv(M)

    def R(phi):
        return torch.zeros(n, 9, dtype=x.dtype).index_add(0, rows, (w * (phi[cols] - phi[rows]))[:, None] * b)

    yf = (X * R(f)[:, None, :]).sum(2)
    out = {"grad_x": yf[:, 0] / re, "grad_y": yf[:, 1] / re, "grad_z": yf[:, 2] / re,
           "laplacian": 2.0 * (yf[:, 3] + yf[:, 4] + yf[:, 5]) / re ** 2}
    div = sum((X[:, c, :] * R(v[c])).sum(1) for c in range(3)) / re
    out["divergence"] = div
    ell = X[:, 3, :] + X[:, 4, :] + X[:, 5, :]
    a = 2.0 * w * (ell[rows] * b).sum(1) / (re * re * p.density)
    diag = -torch.zeros(n, dtype=x.dtype).index_add(0, rows, a)
    row_start = torch.arange(n) + off_t[:-1]
    pos = torch.arange(len(idx)) - off_t[rows] + row_start[rows] + 1
    vals = torch.zeros(n + len(idx), dtype=x.dtype).index_put((row_start,), diag).index_put((pos,), a)
    out["ppe_values"] = vals
    out["ppe_rhs"] = div / p.time_step
    return out


def test_forward_and_adjoint_match_fp64_autograd(pkg, device_api):
    import torch

    case = pkg.cases.lattice_box(n=12, l0=0.01)
    ops = Operators(pkg, device_api, case)
    f_np, v_np = fields(pkg, case)
    x = [torch.from_numpy(case.fluid[k].copy()).cuda() for k in ("x", "y", "z")]
    f = torch.from_numpy(f_np).cuda()
    v = [torch.from_numpy(a.copy()).cuda() for a in v_np]
    out = ops.forward(x, f, v)
    cot = cotangents(pkg, ops)
    fbar, vbar, xbar = ops.backward(x, f, v, cot)
    # torch reference on the CPU
    xr = torch.from_numpy(np.stack([case.fluid[k] for k in ("x", "y", "z")], 1).copy()).requires_grad_(True)
    fr = torch.from_numpy(f_np.copy()).requires_grad_(True)
    vr = [torch.from_numpy(a.copy()).requires_grad_(True) for a in v_np]
    ref = torch_operators(xr, fr, vr, ops.off, ops.idx, ops.p)
    assert np.array_equal(out["ppe_row_offsets"].cpu().numpy()[:-1], (np.arange(ops.n) + ops.off[:-1]))
    # Every output against its own maximum (v is divergence-free, so the
    # divergence and the PPE rhs are discretization noise of about 1e-3 of the
    # velocity-gradient scale: their own maximum is the strict measure).
    for k, r in ref.items():
        g = out[k].cpu().numpy()
        rn = r.detach().numpy()
        err = np.max(np.abs(g - rn)) / max(np.max(np.abs(rn)), 1e-300)
        print(f"\nforward {k}: {err:.2e}")
        assert err < FORWARD_RTOL, (k, err)
    loss = sum((cot[k].cpu() * r).sum() for k, r in ref.items())
    loss.backward()
    pairs = [("f", fbar, fr.grad), ("vx", vbar[0], vr[0].grad), ("vy", vbar[1], vr[1].grad),
             ("vz", vbar[2], vr[2].grad)] + [(f"x{c}", xbar[c], xr.grad[:, c]) for c in range(3)]
    for name, got, want in pairs:
        g, w_ = got.cpu().numpy(), want.numpy()
        err = np.max(np.abs(g - w_)) / max(np.max(np.abs(w_)), 1e-300)
        print(f"adjoint d/d{name}: {err:.2e}")
        assert err < ADJOINT_RTOL, (name, err)


def test_adjoint_against_finite_differences_64cubed(pkg, device_api):
    import torch

    case = pkg.cases.lattice_box(n=64, l0=0.01)
    ops = Operators(pkg, device_api, case)
    f_np, v_np = fields(pkg, case)
    x = [torch.from_numpy(case.fluid[k].copy()).cuda() for k in ("x", "y", "z")]
    f = torch.from_numpy(f_np).cuda()
    v = [torch.from_numpy(a.copy()).cuda() for a in v_np]
    cot = cotangents(pkg, ops)
    fbar, vbar, xbar = ops.backward(x, f, v, cot)
    keys = list(cot)

    def loss_delta(plus, minus):
        return sum(float((cot[k] * (plus[k] - minus[k])).sum()) for k in keys)

    eps = 1e-6 * case.l0
    re = ops.p.support_radius
    pos = np.stack([case.fluid[k] for k in ("x", "y", "z")], 1)
    samples = (pkg.cases.uniform01(6, 64) * ops.n).astype(np.int64)
    scale = float(max(t.abs().max() for t in xbar))
    checked, worst = 0, 0.0
    for k in samples:
        nbrs = ops.idx[ops.off[k]:ops.off[k + 1]]
        dist = np.linalg.norm(pos[nbrs] - pos[k], axis=1)
        if np.any(np.abs(dist - re) < 10 * eps):
            continue
        for c in range(3):
            x[c][k] += eps
            plus = ops.forward(x, f, v)
            x[c][k] -= 2 * eps
            minus = ops.forward(x, f, v)
            x[c][k] += eps
            fd = loss_delta(plus, minus) / (2 * eps)
            ad = float(xbar[c][k])
            err = abs(fd - ad) / max(abs(ad), 1e-3 * scale)
            worst = max(worst, err)
            assert err < FD_RTOL, (int(k), c, fd, ad)
        checked += 1
    # field cotangents: the outputs are linear in f and v, so a difference
    # quotient is exact up to rounding
    for k in samples[:16]:
        for name, arr, bar in (("f", f, fbar), ("vx", v[0], vbar[0])):
            h = 1e-6
            arr[k] += h
            plus = ops.forward(x, f, v)
            arr[k] -= 2 * h
            minus = ops.forward(x, f, v)
            arr[k] += h
            fd = loss_delta(plus, minus) / (2 * h)
            ad = float(bar[k])
            assert abs(fd - ad) <= FD_RTOL * max(abs(ad), 1e-3 * float(bar.abs().max())), (name, int(k), fd, ad)
    print(f"\nfinite differences: {checked} particles x 3 coordinates, worst relative error {worst:.2e}")
    assert checked >= 48


def test_forward_is_bitwise_reproducible(pkg, device_api):
    """The forward (and the fluid-only inverse it builds) has no atomics and
    no reduction across threads: repeated calls on the same inputs must give
    the same bits.  The torch FP64 restatement on the CPU is run twice as
    well and its repeatability reported."""
    import torch

    case = pkg.cases.lattice_box(n=12, l0=0.01)
    ops = Operators(pkg, device_api, case)
    f_np, v_np = fields(pkg, case)
    x = [torch.from_numpy(case.fluid[k].copy()).cuda() for k in ("x", "y", "z")]
    f = torch.from_numpy(f_np).cuda()
    v = [torch.from_numpy(a.copy()).cuda() for a in v_np]
    runs = []
    for _ in range(5):
        out = ops.alloc_out()
        inv = torch.full((ops.n * 81,), float("nan"), dtype=torch.float64, device="cuda")
        st = ops.lib.lsmps_operators_forward(ops.ctx.h, ctypes.byref(ops._fluid(x)),
                                             ctypes.byref(ops.dev.csr_view("fluid")), ctypes.byref(ops.p),
                                             ctypes.c_void_p(f.data_ptr()), ctypes.byref(ops._vec(v)),
                                             ctypes.byref(ops._out(out)), ctypes.c_void_p(inv.data_ptr()))
        ops.ctx.check(st)
        out["inverse"] = inv
        runs.append({k: t.cpu().numpy() for k, t in out.items()})
    for r in runs[1:]:
        for k in r:
            assert np.array_equal(r[k], runs[0][k]), k
    xr = torch.from_numpy(np.stack([case.fluid[k] for k in ("x", "y", "z")], 1).copy())
    fr = torch.from_numpy(f_np.copy())
    vr = [torch.from_numpy(a.copy()) for a in v_np]
    refs = [torch_operators(xr, fr, vr, ops.off, ops.idx, ops.p) for _ in range(3)]
    moved = [k for k in refs[0] if any(not torch.equal(r[k], refs[0][k]) for r in refs[1:])]
    print(f"\ntorch FP64 restatement: outputs that differ between identical runs: {moved}")


def test_backward_deterministic_and_atomic_forms(pkg, device_api):
    """The default backward (CSR transpose + gather, no atomics) gives the
    same bits on repeated calls, and agrees with the scatter form (FP64
    atomics) to rounding."""
    import torch

    case = pkg.cases.lattice_box(n=12, l0=0.01)
    ops = Operators(pkg, device_api, case)
    f_np, v_np = fields(pkg, case)
    x = [torch.from_numpy(case.fluid[k].copy()).cuda() for k in ("x", "y", "z")]
    f = torch.from_numpy(f_np).cuda()
    v = [torch.from_numpy(a.copy()).cuda() for a in v_np]
    cot = cotangents(pkg, ops)

    def flat(res):
        fbar, vbar, xbar = res
        return [t.cpu().numpy() for t in [fbar, *vbar, *xbar]]

    det = [flat(ops.backward(x, f, v, cot)) for _ in range(3)]
    for r in det[1:]:
        for a_, b_ in zip(r, det[0]):
            assert np.array_equal(a_, b_)
    ops.ctx.set_adjoint_atomic(True)
    try:
        atom = flat(ops.backward(x, f, v, cot))
    finally:
        ops.ctx.set_adjoint_atomic(False)
    for name, a_, b_ in zip(["f", "vx", "vy", "vz", "xx", "xy", "xz"], atom, det[0]):
        err = np.max(np.abs(a_ - b_)) / max(np.max(np.abs(b_)), 1e-300)
        print(f"\natomic vs deterministic d/d{name}: {err:.2e}")
        assert err < 1e-12, (name, err)
