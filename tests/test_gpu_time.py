"""Device time-step control (lsmps_advance_time, lsmps_ctx_set_device_time_step):
the reference driver's max_velocity + SimulationTimeManager::advance on the
device, bit-exact against the oracle; a step taking dt from device memory
equals the step taking it from the params; and a captured CUDA graph of the
time loop (advance, step) replays the eager loop bit for bit."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def limits(pkg, **kw):
    lim = pkg.abi.TimeLimits(min_time_step=1e-7, max_time_step=1e-3, growth_factor=1.05, cfl=0.2,
                             particle_spacing=0.0025, final_time=1.0)
    for k, v in kw.items():
        setattr(lim, k, v)
    return lim


def state_tensor(torch, pkg, lim, dt0):
    host = pkg.abi.TimeState()
    pkg.abi.load_library().lsmps_time_state_init(__import__("ctypes").byref(lim), dt0, __import__("ctypes").byref(host))
    raw = np.frombuffer(bytes(host), dtype=np.uint8).copy()
    return torch.as_tensor(raw).cuda()


def read_state(pkg, t):
    return pkg.abi.TimeState.from_buffer_copy(t.cpu().numpy().tobytes())


def test_advance_time_matches_oracle(pkg, device_api, oracle):
    import torch

    ctx = device_api.Context(0)
    rng = np.random.default_rng(5)
    n = 100_000
    dev = pkg.buffers.StepBuffers(pkg.buffers.TorchAlloc("cuda"), n, 0, 1)
    host = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), n, 0, 1)
    lim = limits(pkg, final_time=3e-4)
    st_dev = state_tensor(torch, pkg, lim, 1e-4)
    st_host = read_state(pkg, st_dev)
    for rnd in range(6):
        v = rng.standard_normal((3, n)) * (10.0 ** (rnd - 2))
        if rnd == 3:
            v[0, 17] = np.nan
            v[1, 99] = np.inf
        if rnd == 4:
            v[:] = 0.0
        for c, k in enumerate(("vx", "vy", "vz")):
            host.fluid[k][:] = v[c]
            dev.alloc.copy_(dev.fluid[k], v[c])
        ctx.advance_time(dev, lim, st_dev.data_ptr())
        assert oracle.advance_time(host, lim, st_host) == 0
        got = read_state(pkg, st_dev)
        for name, _ in pkg.abi.TimeState._fields_:
            assert getattr(got, name) == getattr(st_host, name), (rnd, name, getattr(got, name),
                                                                 getattr(st_host, name))
    # (the driver stops once current_time >= final_time; advancing past it
    # takes clamped steps again, as the reference's manager does)
    assert got.step_index == 6
    with pytest.raises(device_api.LsmpsError):
        ctx.advance_time(dev, limits(pkg, growth_factor=0.5), st_dev.data_ptr())
    ctx.close()


def _snapshot(dev):
    f = dev.numpy("fluid")
    return {k: f[k].copy() for k in ("x", "y", "z", "vx", "vy", "vz", "pressure", "surface_type")} | \
           {"rhs": dev.numpy("ppe")["rhs"].copy()}


def test_device_time_step_equals_params_time_step(pkg, device_api):
    import torch

    case = pkg.cases.CASES["dam_break"](nx=24, ny=12, nz=24, l0=0.005)
    out = []
    for use_device in (False, True):
        ctx = device_api.Context(0)
        dev = device_api.device_buffers(case)
        p = type(case.params).from_buffer_copy(case.params)
        ctx.build_neighbor_lists(dev, p)
        ctx.classify_surface(dev, p)
        dt = torch.tensor([2.5e-4], dtype=torch.float64, device="cuda")
        if use_device:
            p.time_step = 123.0  # must not be read
            ctx.set_device_time_step(dt.data_ptr())
        else:
            p.time_step = 2.5e-4
        for _ in range(2):
            ctx.step(dev, p)
        out.append(_snapshot(dev))
        ctx.close()
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k


def test_captured_time_loop_replays_eager_loop(pkg, device_api):
    import torch

    case = pkg.cases.CASES["dam_break"](nx=24, ny=12, nz=24, l0=0.005)
    lim = limits(pkg, particle_spacing=case.params.particle_spacing)
    results = []
    for captured in (False, True):
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            ctx = device_api.Context(0)
            dev = device_api.device_buffers(case)
            p = case.params
            ctx.reserve(case.n_fluid, case.n_wall, case.n_cells)
            ctx.build_neighbor_lists(dev, p)
            ctx.classify_surface(dev, p)
            state = dev.step_state(p)
            st = state_tensor(torch, pkg, lim, 1e-4)
            ctx.set_device_time_step(st.data_ptr() + 8)  # &state->time_step
            ctx.set_stream(stream.cuda_stream)
            ctx.set_synchronous(False)
            # one eager step first (sizes scratch and packs outside capture)
            ctx.advance_time(dev, lim, st.data_ptr())
            ctx.step(dev, p, state)
            ctx.synchronize()
            if captured:
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=stream):
                    for _ in range(3):
                        ctx.advance_time(dev, lim, st.data_ptr())
                        ctx.step(dev, p, state)
                g.replay()
                stream.synchronize()
                ctx.synchronize()
                del g
            else:
                for _ in range(3):
                    ctx.advance_time(dev, lim, st.data_ptr())
                    ctx.step(dev, p, state)
                ctx.synchronize()
            torch.cuda.synchronize()
            results.append((_snapshot(dev), read_state(pkg, st)))
            ctx.close()
    (a, sa), (b, sb) = results
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    for name, _ in pkg.abi.TimeState._fields_:
        assert getattr(sa, name) == getattr(sb, name), name
    assert sa.step_index == 4 and sa.time_step > 0
    print(f"after 4 steps: t = {sa.current_time:.6e}, dt = {sa.time_step:.3e}, |u|max = {sa.max_velocity:.3e}")
