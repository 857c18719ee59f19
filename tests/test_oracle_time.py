"""The oracle's time-step control (max_velocity + SimulationTimeManager::
advance of the reference driver) against hand-computed answers (no GPU)."""

import numpy as np
import pytest


def limits(pkg, **kw):
    lim = pkg.abi.TimeLimits(min_time_step=1e-6, max_time_step=1e-3, growth_factor=1.05, cfl=0.2,
                             particle_spacing=0.01, final_time=1.0)
    for k, v in kw.items():
        setattr(lim, k, v)
    return lim


def fluid(pkg, v):
    b = pkg.buffers.StepBuffers(pkg.buffers.NumpyAlloc(), len(v), 0, 1)
    for c, k in enumerate(("vx", "vy", "vz")):
        b.fluid[k][:] = [row[c] for row in v]
    return b


def test_cfl_growth_clamp_and_final_time(pkg, oracle):
    st = pkg.abi.TimeState(current_time=0.0, time_step=1e-4)
    b = fluid(pkg, [(2.0, 0.0, 0.0), (0.0, 1.0, 0.0)])
    assert oracle.advance_time(b, limits(pkg), st) == 0
    # cfl dt = 0.2 * 0.01 / 2 = 1e-3; growth limit 1.05e-4 wins
    assert st.max_velocity == 2.0 and st.cfl_time_step == 0.2 * 0.01 / 2.0
    assert st.time_step == 1e-4 * 1.05 and st.current_time == 1e-4 * 1.05 and st.step_index == 1
    # fast fluid: the CFL limit wins, clamped below by min_time_step
    b = fluid(pkg, [(1e6, 0.0, 0.0)])
    oracle.advance_time(b, limits(pkg), st)
    assert st.time_step == 1e-6
    # at rest: cfl dt = max_time_step; growth from 1e-6
    b = fluid(pkg, [(0.0, 0.0, 0.0)])
    oracle.advance_time(b, limits(pkg), st)
    assert st.cfl_time_step == 1e-3 and st.time_step == 1e-6 * 1.05
    # cut to the remaining time
    st2 = pkg.abi.TimeState(current_time=1.0 - 1e-5, time_step=1e-3)
    oracle.advance_time(b, limits(pkg), st2)
    assert st2.time_step == pytest.approx(1e-5, rel=1e-9) and st2.current_time == pytest.approx(1.0)


def test_non_finite_speeds_are_ignored(pkg, oracle):
    st = pkg.abi.TimeState(current_time=0.0, time_step=1e-4)
    b = fluid(pkg, [(np.nan, 0.0, 0.0), (np.inf, 1.0, 0.0), (0.0, 0.5, 0.0)])
    oracle.advance_time(b, limits(pkg), st)
    assert st.max_velocity == 0.5
