"""Algorithmic (compulsory) bytes of one LSMPS step and of each kernel.

Every array a stage must read or write is counted once per stage, from the
run's actual N_f (fluid), N_w (wall), K_f / K_w (CSR entries) and C (cells);
S is the size of the floating type (8 for FP64 storage).  Neighbour gathers
(positions of j) are counted once per array, i.e. perfect cache reuse: the
model is the floor a kernel can reach, and achieved/peak compares a kernel
with that floor.
"""

from __future__ import annotations


def step_terms(nf: int, nw: int, kf: int, kw: int, c: int, s: int = 8) -> dict[str, int]:
    """Per-stage compulsory bytes of one benchmark step (provision -> PPE ->
    correction -> neighbour rebuild -> surface labels, moments built once)."""
    k = kf + kw
    pos = 3 * s * (nf + nw)
    t = {}
    # cell lists: positions, (id, index) write, one sort read+write of keys and
    # values, cell begin/end
    t["cells"] = sum(3 * s * n + 8 * n + 16 * n + 8 * c for n in (nf, nw))
    # CSR count + write: positions, cell data, offsets, rows
    t["csr"] = pos + 4 * (nf + nw) + 16 * c + 8 * (nf + 1) + 4 * k
    t["surface"] = 8 * nf + 4 * k + pos + 3 * s * nw + 4 * nf + (4 * nf + 4 * nf + 4 * kf + 3 * s * nf)
    moment_kind = 8 * nf + 4 * k + pos + 3 * s * nw + 81 * s * nf + 2 * s * nf
    t["moment"] = 2 * moment_kind
    t["provision"] = 8 * nf + 4 * k + pos + pos + 81 * s * nf + 6 * s * nf + 3 * s * nw
    t["ppe"] = (4 * (nf + 1) + 8 * nf + 4 * k + pos + pos + 4 * nf + 2 * 81 * s * nf + 3 * s * nw
                + (4 + s) * (nf + kf) + 3 * s * nf)
    t["gradient"] = 8 * nf + 4 * k + pos + s * nf + 3 * s * nw + 81 * s * nf + 3 * s * nf
    t["shifting"] = 8 * nf + 4 * k + pos + 3 * s * nw + 4 * nf + 3 * s * nf
    t["update"] = nf * (2 * 3 * s + 2 * 3 * s + 3 * 3 * s + 4)
    t["anti_penetration"] = 8 * nf + 4 * kw + 6 * s * nw + 2 * 6 * s * nf
    t["smoothing"] = 8 * nf + 4 * kf + 3 * s * nf + 3 * s * nf + 4 * nf + 3 * s * nf + 6 * s * nf
    return t


def step_bytes(nf: int, nw: int, kf: int, kw: int, c: int, s: int = 8) -> int:
    return sum(step_terms(nf, nw, kf, kw, c, s).values())


def kernel_bytes(nf: int, nw: int, kf: int, kw: int, c: int, s: int = 8) -> dict[str, int]:
    """Algorithmic bytes per launch of the step's kernels (names as the
    library's profiler reports them): every array the kernel must read or
    write counted once, neighbour gathers included once per array.  The two
    CSR kernels run once per table (fluid, wall); their figure is the mean of
    the two launches."""
    k = kf + kw
    pos_f = 3 * s * nf
    pos_w = 3 * s * nw
    rows = 8 * (nf + 1) + 4 * k  # fluid and wall CSR offsets + indices
    out = {}
    moment_kind_out = (81 * s + 2 * s + 4) * nf  # inverse, trace, regularisation, info
    moment_in = rows + pos_f + 2 * pos_w  # wall positions + normals
    out["moment_a_kernel<V,P>"] = out["moment_a_split_kernel"] = moment_in + 2 * moment_kind_out
    out["moment_a_kernel<V>"] = out["moment_a_kernel<P>"] = moment_in + moment_kind_out
    lap = rows + 2 * pos_f + 2 * pos_w + 3 * s * nf
    # the two mixed stages in one kernel (row halves on two warps)
    out["moment_mixed_split_kernel<false>"] = (4 * (nf + 1) + 4 * kf + pos_f + 2 * (4 * (nf + 1) + 4 * kw + 2 * pos_w)
                                               + 2 * (36 * 4 + 2 * s + 4) * nf)
    out["laplacian_kernel<false>"] = lap + 81 * s * nf
    out["laplacian_kernel<true>"] = lap + 9 * 4 * nf  # the FP32 Laplacian row
    ppe_common = rows + 2 * pos_f + 4 * nf + 3 * pos_w + 4 * (nf + 1) + (4 + s) * (nf + kf) + 3 * s * nf
    out["ppe_kernel"] = ppe_common + 2 * 81 * s * nf
    for g in (4, 8, 16):
        out[f"ppe_lanes_kernel<{g}, false>"] = ppe_common + 2 * 81 * s * nf
        # mixed form: the pressure Laplacian row and the three velocity rows, FP32
        out[f"ppe_lanes_kernel<{g}, true>"] = ppe_common + 36 * 4 * nf
    grad_common = rows + 4 * nf + pos_f + 3 * s * nf + 2 * pos_w + 6 * s * nf
    out["gradient_shifting_kernel<false>"] = grad_common + 81 * s * nf
    out["gradient_shifting_kernel<true>"] = grad_common + 27 * 4 * nf
    # mixed-form moment stages: FP32 assembly into FP64 monomial totals, then
    # per kind the FP32 factorisation, refinement and the 36-float rows
    out["moment_sums_kernel"] = 4 * (nf + 1) + 4 * kf + pos_f + 31 * 8 * nf
    out["moment_rows_kernel<false>"] = (2 * 31 * 8 * nf + 2 * (4 * (nf + 1) + 4 * kw + pos_f + 2 * pos_w)
                                        + 2 * (36 * 4 + 2 * s + 4) * nf)
    out["update_anti_penetration_kernel"] = (4 * (nf + 1) + 4 * kw + 4 * nf + 2 * pos_f + 3 * pos_f
                                             + 2 * pos_w + 2 * pos_f)
    out["smooth_kernel"] = 4 * (nf + 1) + 4 * kf + 2 * pos_f + 4 * nf + pos_f
    out["copy_kernel"] = 2 * pos_f
    # lane-parallel variants (LSMPS_KNOB_GATHER_LANES) move the same bytes
    for g in (1, 2, 4):
        for m in ("false", "true"):
            out[f"laplacian_kernel<{m}, {g}>"] = out[f"laplacian_kernel<{m}>"]
            out[f"gradient_shifting_kernel<{m}, {g}>"] = out[f"gradient_shifting_kernel<{m}>"]
        out[f"smooth_kernel<{g}>"] = out["smooth_kernel"]
    # the mixed form's FP32-arithmetic kernels read and write what the mixed
    # lane kernels do (their FP64 list passes touch only the few FP64-route
    # particles)
    for g in (1, 2, 4):
        out[f"laplacian32_kernel<{g}>"] = out["laplacian_kernel<true>"]
        out[f"gradient32_kernel<{g}>"] = out["gradient_shifting_kernel<true>"]
    for g in (4, 8, 16):
        out[f"ppe32_kernel<{g}>"] = out[f"ppe_lanes_kernel<{g}, true>"]
    out["classify_kernel"] = rows + pos_f + 2 * pos_w + 4 * nf
    out["expand_kernel"] = 4 * (nf + 1) + 4 * kf + 8 * nf
    count_fluid = 2 * pos_f + 8 * c + 4 * nf + 4 * nf
    count_wall = pos_f + pos_w + 8 * c + 4 * nw + 4 * nf
    out["csr_count_kernel"] = (count_fluid + count_wall) // 2
    out["csr_write_kernel"] = (count_fluid + count_wall + 8 * nf + 4 * k) // 2
    # virtual-light diagnostic (not in the step): rows, positions, count + fraction
    out["virtual_light_kernel"] = rows + pos_f + pos_w + (4 + s) * nf
    return out


def solve_kernel_bytes(rows: int, nnz: int, restart: int = 20, s: int = 8) -> dict[str, int]:
    """Algorithmic bytes per launch of the PPE solve's kernels (csrc/solve.cu)
    on a system of `rows` rows and `nnz` stored entries: the SpMV reads the
    row offsets, the (column, value) pairs, the input vector once and writes
    the output; the Gram-Schmidt passes stream the basis vectors they use (on
    average half the restart length plus one per pass)."""
    vec = s * rows
    avg_basis = (restart + 1) / 2.0
    return {
        "spmv_kernel<kSpmvLanes>": 4 * (rows + 1) + (4 + s) * nnz + 2 * vec,
        "dots_kernel": int(vec * (avg_basis + 1)),
        "update_kernel": int(vec * (avg_basis + 2)),
        "scale_kernel": 2 * vec,
        "correct_kernel": int(vec * (restart + 2)),
        "residual_kernel": 2 * vec,
    }
