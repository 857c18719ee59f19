"""lsmps_ctx_set_step_events and host_loop.HostResidentLoop: a time loop over
particle state kept in pinned host memory, whose copies overlap the steps
(the next step's positions arriving in a second device buffer while the
current step's rebuild runs; the wall geometry during the fluid moment sums;
velocities, pressure, labels and wall velocities while the moments are built;
positions, velocities and pressure leaving while the rebuild and the labels
run), gives the same states, bit for bit, as the same loop with every copy
serialised around the step, in both precision forms.  Integer and floating
outputs: tolerance zero."""

import pytest

pytestmark = pytest.mark.gpu

FLUID_IN = ("x", "y", "z", "vx", "vy", "vz", "pressure", "surface_type")
WALLS_IN = ("x", "y", "z", "normal_x", "normal_y", "normal_z", "vx", "vy", "vz")
FLUID_OUT = ("x", "y", "z", "vx", "vy", "vz", "pressure", "surface_type")


def serial_loop(api, case, precision, steps):
    """Copy in, step, copy out, one after another on one stream."""
    import torch

    p = case.params
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        dev = api.device_buffers(case)
        ctx = api.Context(0, precision=precision)
        ctx.build_neighbor_lists(dev, p)
        ctx.classify_surface(dev, p)
        state = dev.step_state(p)
        hf = {k: dev.fluid[k].detach().to("cpu").pin_memory() for k in FLUID_IN}
        hw = {k: dev.walls[k].detach().to("cpu").pin_memory() for k in WALLS_IN}
        ctx.set_synchronous(False)
        for _ in range(steps):
            for k in FLUID_IN:
                dev.fluid[k].copy_(hf[k], non_blocking=True)
            for k in WALLS_IN:
                dev.walls[k].copy_(hw[k], non_blocking=True)
            ctx.step(dev, p, state)
            for k in FLUID_OUT:
                hf[k].copy_(dev.fluid[k], non_blocking=True)
        ctx.synchronize()
        torch.cuda.synchronize()
        rows = {k: v.cpu().clone() for k, v in dev.fluid_neighbors.items()}
        ctx.close()
    return {k: hf[k].clone() for k in FLUID_OUT}, rows


def overlapped_loop(pkg, api, case, precision, steps):
    import importlib

    import torch

    host_loop = importlib.import_module("lsmps3d_b200.host_loop")
    p = case.params
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        dev = api.device_buffers(case)
        ctx = api.Context(0, precision=precision)
        ctx.build_neighbor_lists(dev, p)
        ctx.classify_surface(dev, p)
        ctx.set_synchronous(False)
        loop = host_loop.HostResidentLoop(ctx, dev, p)
        for _ in range(steps):
            loop.step()
        loop.sync()
        ctx.synchronize()
        torch.cuda.synchronize()
        loop.close()
        rows = {k: v.cpu().clone() for k, v in dev.fluid_neighbors.items()}
        ctx.close()
    return {k: loop.host_fluid[k].clone() for k in FLUID_OUT}, rows


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_overlapped_host_loop_matches_serial(pkg, device_api, precision):
    import torch

    prec = pkg.abi.PRECISION_PLAIN if precision == "plain" else pkg.abi.PRECISION_MIXED
    case = pkg.cases.dam_break(30, 15, 30)
    # five steps: the two position buffers in turn
    serial, rows_s = serial_loop(device_api, case, prec, steps=5)
    overlapped, rows_o = overlapped_loop(pkg, device_api, case, prec, steps=5)
    for f in serial:
        assert torch.equal(serial[f], overlapped[f]), f
    for k in rows_s:
        assert torch.equal(rows_s[k], rows_o[k]), k
