"""The step's operators with their wall terms as a differentiable pair
(lsmps_step_operators_forward / lsmps_step_operators_backward): the velocity
Laplacian and divergence with the velocity Dirichlet-A moments (wall
samples), the pressure gradient and the PPE rows with the pressure
Neumann-A moments (wall Neumann terms and the wall source of the PPE
right-hand side), Dirichlet rows for Surface and Splash particles.

Checks:

* forward and backward against the same operators written directly in
  torch (float64, CPU) and differentiated by autograd, on a 12^3 jittered
  lattice in a tank with 3 wall layers (wall velocities and the fluid's
  velocity and pressure fields non-trivial, labels from the device's
  classification, so that Surface rows are Dirichlet rows);
* repeatability of the deterministic backward and agreement of the atomic
  form;
* FP64 central finite differences on the 64^3 = 262,144-particle jittered
  lattice with its 3 wall layers: eps = 1e-6 l0 on 64 seeded particles, half
  of them drawn from the particles whose rows have walls, topology and labels
  frozen, samples with a pair (fluid or wall) within 10 eps of r_e skipped.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FORWARD_RTOL = 1e-10
ADJOINT_RTOL = 1e-9
FD_RTOL = 1e-5
OUTPUTS = ("lap_x", "lap_y", "lap_z", "divergence", "grad_x", "grad_y", "grad_z", "ppe_values", "ppe_rhs", "wall_rhs")


def fields(case):
    """Velocity, pressure and wall velocity fields of a lattice case."""
    f, w = case.fluid, case.walls
    L = float(np.ptp(f["x"])) or 1.0
    u = np.stack([np.sin(2 * np.pi * f["y"] / L), np.cos(2 * np.pi * f["z"] / L) * 0.5,
                  0.3 * np.sin(2 * np.pi * f["x"] / L) + 0.1 * f["z"] / L], 1)
    p = 1000.0 * 9.81 * (f["z"].max() + case.l0 - f["z"]) + 5.0 * np.sin(2 * np.pi * f["x"] / L)
    uw = np.stack([0.2 * np.cos(2 * np.pi * w["y"] / L), 0.1 * np.ones_like(w["x"]), 0.05 * w["x"] / L], 1)
    return u, p, uw


class StepOps:
    def __init__(self, pkg, device_api, case):
        import torch

        self.torch, self.pkg = torch, pkg
        self.p = case.params
        self.case = case
        self.dev = device_api.device_buffers(case)
        u, pr, uw = fields(case)
        for c, k in enumerate(("vx", "vy", "vz")):
            self.dev.alloc.copy_(self.dev.fluid[k], u[:, c])
            self.dev.alloc.copy_(self.dev.walls[k], uw[:, c])
        self.dev.alloc.copy_(self.dev.fluid["pressure"], pr)
        self.ctx = device_api.Context(0)
        self.ctx.build_neighbor_lists(self.dev, self.p)
        self.ctx.classify_surface(self.dev, self.p)
        self.n = case.n_fluid
        self.off, self.idx = self.dev.csr_rows("fluid")
        self.woff, self.widx = self.dev.csr_rows("wall")
        self.k = int(self.off[-1])
        self.labels = self.dev.fluid["surface_type"].cpu().numpy().copy()
        self.lib = device_api._lib

    def alloc_out(self):
        t = self.torch
        z = lambda m, dt=t.float64: t.zeros(m, dtype=dt, device="cuda")  # noqa: E731
        out = {k: z(self.n) for k in OUTPUTS if k != "ppe_values"}
        out["ppe_values"] = z(self.n + self.k)
        out["ppe_row_offsets"] = z(self.n + 1, t.int32)
        out["ppe_col_indices"] = z(self.n + self.k, t.int32)
        return out

    def _out(self, d):
        o = self.pkg.abi.StepOperatorOut()
        o.count = self.n
        for k, v in d.items():
            setattr(o, k, v.data_ptr())
        return o

    def fluid_view(self, x=None):
        v = self.dev.fluid_view()
        if x is not None:
            v.x, v.y, v.z = (t.data_ptr() for t in x)
        return v

    def forward(self, x=None):
        out = self.alloc_out()
        st = self.lib.lsmps_step_operators_forward(
            self.ctx.h, ctypes.byref(self.fluid_view(x)), ctypes.byref(self.dev.walls_view()),
            ctypes.byref(self.dev.csr_view("fluid")), ctypes.byref(self.dev.csr_view("wall")),
            ctypes.byref(self.p), ctypes.byref(self._out(out)))
        self.ctx.check(st)
        return out

    def backward(self, cot, x=None):
        t = self.torch
        ub = [t.zeros(self.n, dtype=t.float64, device="cuda") for _ in range(3)]
        pb = t.zeros(self.n, dtype=t.float64, device="cuda")
        xb = [t.zeros(self.n, dtype=t.float64, device="cuda") for _ in range(3)]

        def vec(ts):
            v = self.pkg.abi.Vector()
            v.count = self.n
            v.x, v.y, v.z = (a.data_ptr() for a in ts)
            return v

        st = self.lib.lsmps_step_operators_backward(
            self.ctx.h, ctypes.byref(self.fluid_view(x)), ctypes.byref(self.dev.walls_view()),
            ctypes.byref(self.dev.csr_view("fluid")), ctypes.byref(self.dev.csr_view("wall")),
            ctypes.byref(self.p), ctypes.byref(self._out(cot)), ctypes.byref(vec(ub)),
            ctypes.c_void_p(pb.data_ptr()), ctypes.byref(vec(xb)))
        self.ctx.check(st)
        return ub, pb, xb

    def cotangents(self, seed=5):
        t = self.torch
        g = self.pkg.cases.normal(seed, 9 * self.n + self.n + self.k)
        cot, pos = {}, 0
        for k in OUTPUTS:
            m = self.n + self.k if k == "ppe_values" else self.n
            cot[k] = t.from_numpy(g[pos:pos + m].copy()).cuda()
            pos += m
        return cot


def basis(s):
    import torch

    return torch.stack([s[:, 0], s[:, 1], s[:, 2], s[:, 0] ** 2, s[:, 1] ** 2, s[:, 2] ** 2, s[:, 0] * s[:, 1],
                        s[:, 1] * s[:, 2], s[:, 2] * s[:, 0]], 1)


def torch_step_operators(x, u, p, xw, nw, uw, off, idx, woff, widx, labels, prm):
    """The step's operators in plain torch float64 (the FP64 reference), on
    one thread and with matrix products written as elementwise sums, so that
    its rounding does not depend on the BLAS kernel or the thread count."""
    import torch

    threads = torch.get_num_threads()
    torch.set_num_threads(1)
    try:
        return _torch_step_operators(x, u, p, xw, nw, uw, off, idx, woff, widx, labels, prm)
    finally:
        torch.set_num_threads(threads)


def _torch_step_operators(x, u, p, xw, nw, uw, off, idx, woff, widx, labels, prm):
    import torch

    n = x.shape[0]
    re, lam, lw = prm.support_radius, prm.lsmps_regularization, prm.lsmps_wall_weight_scale
    rho, dt = prm.density, prm.time_step
    g = torch.tensor(list(prm.gravity), dtype=x.dtype)
    off_t = torch.from_numpy(off.astype(np.int64))
    woff_t = torch.from_numpy(woff.astype(np.int64))
    rows = torch.repeat_interleave(torch.arange(n), off_t[1:] - off_t[:-1])
    cols = torch.from_numpy(idx.astype(np.int64))
    wrows = torch.repeat_interleave(torch.arange(n), woff_t[1:] - woff_t[:-1])
    wcols = torch.from_numpy(widx.astype(np.int64))
    lab = torch.from_numpy(labels.astype(np.int64))
    dirm = (lab == 2) | (lab == 3)
    spl = lab == 3
    d = x[cols] - x[rows]
    w = torch.clamp(1.0 - torch.sqrt((d * d).sum(1)) / re, min=0.0)
    b = basis(d / re)
    dw = xw[wcols] - x[wrows]
    ww = lw * torch.clamp(1.0 - torch.sqrt((dw * dw).sum(1)) / re, min=0.0)
    sw = dw / re
    bw = basis(sw)
    nn = nw[wcols]
    q = torch.stack([nn[:, 0], nn[:, 1], nn[:, 2], 2 * sw[:, 0] * nn[:, 0], 2 * sw[:, 1] * nn[:, 1],
                     2 * sw[:, 2] * nn[:, 2], sw[:, 1] * nn[:, 0] + sw[:, 0] * nn[:, 1],
                     sw[:, 2] * nn[:, 1] + sw[:, 1] * nn[:, 2], sw[:, 0] * nn[:, 2] + sw[:, 2] * nn[:, 0]], 1)
    z9 = torch.zeros(n, 9, 9, dtype=x.dtype)
    S = z9.index_add(0, rows, w[:, None, None] * b[:, :, None] * b[:, None, :])
    SV = S.index_add(0, wrows, ww[:, None, None] * bw[:, :, None] * bw[:, None, :])
    SP = S.index_add(0, wrows, ww[:, None, None] * q[:, :, None] * q[:, None, :])

    def reg_inv(M):
        tr = torch.diagonal(M, dim1=1, dim2=2).sum(1)
        reg = lam * torch.where(tr > 0, tr / 9.0, torch.ones_like(tr))
        return torch.linalg.inv(M + reg[:, None, None] * torch.eye(9, dtype=x.dtype))

    XV, XP = reg_inv(SV), reg_inv(SP)
    z = torch.zeros(n, 9, dtype=x.dtype)
    RV = torch.stack([z.index_add(0, rows, (w * (u[cols, c] - u[rows, c]))[:, None] * b)
                      .index_add(0, wrows, (ww * (uw[wcols, c] - u[wrows, c]))[:, None] * bw) for c in range(3)], 2)
    yV = (XV[:, :, :, None] * RV[:, None, :, :]).sum(2)
    out = {}
    lap = 2.0 * (yV[:, 3, :] + yV[:, 4, :] + yV[:, 5, :]) / re ** 2
    out["lap_x"], out["lap_y"], out["lap_z"] = lap[:, 0], lap[:, 1], lap[:, 2]
    keep = (~dirm).to(x.dtype)
    div = (yV[:, 0, 0] + yV[:, 1, 1] + yV[:, 2, 2]) / re * keep
    gn = (nn * g).sum(1)
    RP = z.index_add(0, rows, (w * (p[cols] - p[rows]))[:, None] * b).index_add(0, wrows, (ww * re * rho * gn)[:, None] * q)
    yP = (XP * RP[:, None, :]).sum(2)
    gmask = (~spl).to(x.dtype)
    out["grad_x"], out["grad_y"], out["grad_z"] = (yP[:, c] / re * gmask for c in range(3))
    L = XP[:, 3, :] + XP[:, 4, :] + XP[:, 5, :]
    a = 2.0 / (re * re * rho) * w * (L[rows] * b).sum(1) * keep[rows]
    diag = -torch.zeros(n, dtype=x.dtype).index_add(0, rows, a)
    wall_rhs = torch.zeros(n, dtype=x.dtype).index_add(0, wrows, 2.0 * ww * gn * (L[wrows] * q).sum(1) / re) * keep
    out["divergence"] = div
    out["wall_rhs"] = wall_rhs
    out["ppe_rhs"] = (div / dt - wall_rhs) * keep
    row_start = torch.arange(n) + off_t[:-1]
    pos = torch.arange(len(idx)) - off_t[rows] + row_start[rows] + 1
    diag_v = torch.where(dirm, torch.ones_like(diag), diag)
    out["ppe_values"] = torch.zeros(n + len(idx), dtype=x.dtype).index_put((row_start,), diag_v).index_put((pos,), a)
    return out


def test_step_operators_match_fp64_autograd(pkg, device_api):
    import torch

    case = pkg.cases.lattice_box(n=12, l0=0.01)
    ops = StepOps(pkg, device_api, case)
    assert (ops.labels == 2).any(), "the case should hold Surface (Dirichlet) rows"
    assert int(ops.woff[-1]) > 0
    out = ops.forward()
    cot = ops.cotangents()
    ub, pb, xb = ops.backward(cot)
    u, p, uw = fields(case)
    f, w = case.fluid, case.walls
    xr = torch.from_numpy(np.stack([f[k] for k in ("x", "y", "z")], 1).copy()).requires_grad_(True)
    ur = torch.from_numpy(u.copy()).requires_grad_(True)
    pr = torch.from_numpy(p.copy()).requires_grad_(True)
    xw = torch.from_numpy(np.stack([w[k] for k in ("x", "y", "z")], 1).copy())
    nw = torch.from_numpy(np.stack([w[k] for k in ("normal_x", "normal_y", "normal_z")], 1).copy())
    ref = torch_step_operators(xr, ur, pr, xw, nw, torch.from_numpy(uw), ops.off, ops.idx, ops.woff, ops.widx,
                               ops.labels, ops.p)
    assert np.array_equal(out["ppe_row_offsets"].cpu().numpy()[:-1], np.arange(ops.n) + ops.off[:-1])
    for k, r in ref.items():
        g = out[k].cpu().numpy()
        rn = r.detach().numpy()
        err = np.max(np.abs(g - rn)) / max(np.max(np.abs(rn)), 1e-300)
        print(f"\nforward {k}: {err:.2e} (scale {np.max(np.abs(rn)):.3e})")
        assert err < FORWARD_RTOL, (k, err)
    loss = sum((cot[k].cpu() * r).sum() for k, r in ref.items())
    loss.backward()
    pairs = [(f"u{c}", ub[c], ur.grad[:, c]) for c in range(3)] + [("p", pb, pr.grad)] + \
            [(f"x{c}", xb[c], xr.grad[:, c]) for c in range(3)]
    for name, got, want in pairs:
        g, w_ = got.cpu().numpy(), want.numpy()
        err = np.max(np.abs(g - w_)) / max(np.max(np.abs(w_)), 1e-300)
        print(f"adjoint d/d{name}: {err:.2e}")
        assert err < ADJOINT_RTOL, (name, err)


def test_step_operators_backward_repeatable_and_atomic_form(pkg, device_api):
    case = pkg.cases.lattice_box(n=12, l0=0.01)
    ops = StepOps(pkg, device_api, case)
    cot = ops.cotangents()

    def flat(res):
        ub, pb, xb = res
        return [t.cpu().numpy() for t in [*ub, pb, *xb]]

    det = [flat(ops.backward(cot)) for _ in range(3)]
    for r in det[1:]:
        for a_, b_ in zip(r, det[0]):
            assert np.array_equal(a_, b_)
    ops.ctx.set_adjoint_atomic(True)
    try:
        atom = flat(ops.backward(cot))
    finally:
        ops.ctx.set_adjoint_atomic(False)
    for a_, b_ in zip(atom, det[0]):
        assert np.max(np.abs(a_ - b_)) <= 1e-12 * max(np.max(np.abs(b_)), 1e-300)


def test_step_adjoint_against_finite_differences_64cubed(pkg, device_api):
    case = pkg.cases.lattice_box(n=64, l0=0.01)
    ops = StepOps(pkg, device_api, case)
    t = ops.torch
    cot = ops.cotangents()
    x = [t.from_numpy(case.fluid[k].copy()).cuda() for k in ("x", "y", "z")]
    ub, pb, xb = ops.backward(cot, x)
    keys = list(cot)

    def loss_delta(plus, minus):
        return sum(float((cot[k] * (plus[k] - minus[k])).sum()) for k in keys)

    eps = 1e-6 * case.l0
    re = ops.p.support_radius
    pos = np.stack([case.fluid[k] for k in ("x", "y", "z")], 1)
    wpos = np.stack([case.walls[k] for k in ("x", "y", "z")], 1)
    has_wall = np.flatnonzero(np.diff(ops.woff) > 0)
    pick_all = (pkg.cases.uniform01(6, 32) * ops.n).astype(np.int64)
    pick_wall = has_wall[(pkg.cases.uniform01(7, 32) * has_wall.size).astype(np.int64)]
    samples = np.concatenate([pick_wall, pick_all])
    scale = float(max(v.abs().max() for v in xb))
    checked, with_walls, worst = 0, 0, 0.0
    for k in samples:
        nbrs = ops.idx[ops.off[k]:ops.off[k + 1]]
        wn = ops.widx[ops.woff[k]:ops.woff[k + 1]]
        dist = np.concatenate([np.linalg.norm(pos[nbrs] - pos[k], axis=1), np.linalg.norm(wpos[wn] - pos[k], axis=1)])
        if np.any(np.abs(dist - re) < 10 * eps):
            continue
        for c in range(3):
            x[c][k] += eps
            plus = ops.forward(x)
            x[c][k] -= 2 * eps
            minus = ops.forward(x)
            x[c][k] += eps
            fd = loss_delta(plus, minus) / (2 * eps)
            ad = float(xb[c][k])
            err = abs(fd - ad) / max(abs(ad), 1e-3 * scale)
            worst = max(worst, err)
            assert err < FD_RTOL, (int(k), c, fd, ad)
        checked += 1
        with_walls += int(wn.size > 0)
    print(f"\nfinite differences: {checked} particles ({with_walls} with wall rows) x 3 coordinates, worst relative "
          f"error {worst:.2e}")
    assert checked >= 48 and with_walls >= 24
