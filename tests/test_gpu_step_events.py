"""lsmps_ctx_set_step_events: a host-resident step loop whose copies overlap
the step (the wall geometry arriving during the fluid moment sums; velocities,
pressure, labels and wall velocities while the moments are built; positions,
velocities and pressure leaving while the neighbour rebuild and the labels
run) gives the same states, bit for bit, as
the same loop with every copy serialised around the step, in both precision
forms.  Integer and floating outputs: tolerance zero."""

import pytest

pytestmark = pytest.mark.gpu

FIRST = [("fluid", k) for k in ("x", "y", "z")]
GEOMETRY = [("walls", k) for k in ("x", "y", "z", "normal_x", "normal_y", "normal_z")]
SECOND = [("fluid", k) for k in ("vx", "vy", "vz", "pressure", "surface_type")] + [("walls", k)
                                                                                   for k in ("vx", "vy", "vz")]
OUT_EARLY = [("fluid", k) for k in ("x", "y", "z", "vx", "vy", "vz", "pressure")]
OUT_LATE = [("fluid", "surface_type")]


def host_loop(pkg, api, case, precision, overlap, steps=3):
    import torch

    p = case.params
    stream = torch.cuda.Stream()
    copy_stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        dev = api.device_buffers(case)
        ctx = api.Context(0, precision=precision)
        ctx.build_neighbor_lists(dev, p)
        ctx.classify_surface(dev, p)
        state = dev.step_state(p)
        host = {f: getattr(dev, f[0])[f[1]].detach().to("cpu").pin_memory() for f in FIRST + GEOMETRY + SECOND}
        ctx.set_synchronous(False)

        def d(f):
            return getattr(dev, f[0])[f[1]]

        ev_wall, ev_in, ev_out = torch.cuda.Event(), torch.cuda.Event(), torch.cuda.Event()
        ev_wall.record(copy_stream)
        ev_in.record(copy_stream)
        ev_out.record(stream)
        if overlap:
            ctx.set_step_events(ev_wall.cuda_event, ev_in.cuda_event, ev_out.cuda_event)
        for _ in range(steps):
            if overlap:
                stream.wait_stream(copy_stream)
                copy_stream.wait_stream(stream)
                for f in FIRST:
                    d(f).copy_(host[f], non_blocking=True)
                with torch.cuda.stream(copy_stream):
                    for f in GEOMETRY:
                        d(f).copy_(host[f], non_blocking=True)
                    ev_wall.record(copy_stream)
                    for f in SECOND:
                        d(f).copy_(host[f], non_blocking=True)
                    ev_in.record(copy_stream)
                ctx.step(dev, p, state)
                copy_stream.wait_event(ev_out)
                with torch.cuda.stream(copy_stream):
                    for f in OUT_EARLY:
                        host[f].copy_(d(f), non_blocking=True)
                for f in OUT_LATE:
                    host[f].copy_(d(f), non_blocking=True)
            else:
                for f in FIRST + GEOMETRY + SECOND:
                    d(f).copy_(host[f], non_blocking=True)
                ctx.step(dev, p, state)
                for f in OUT_EARLY + OUT_LATE:
                    host[f].copy_(d(f), non_blocking=True)
        stream.wait_stream(copy_stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        ctx.set_step_events(None, None, None)
        rows = {k: v.cpu().clone() for k, v in dev.fluid_neighbors.items()}
        ctx.close()
    return {f: host[f].clone() for f in OUT_EARLY + OUT_LATE}, rows


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_overlapped_host_loop_matches_serial(pkg, device_api, precision):
    import torch

    prec = pkg.abi.PRECISION_PLAIN if precision == "plain" else pkg.abi.PRECISION_MIXED
    case = pkg.cases.dam_break(30, 15, 30)
    serial, rows_s = host_loop(pkg, device_api, case, prec, overlap=False)
    overlapped, rows_o = host_loop(pkg, device_api, case, prec, overlap=True)
    for f in serial:
        assert torch.equal(serial[f], overlapped[f]), f
    for k in rows_s:
        assert torch.equal(rows_s[k], rows_o[k]), k
