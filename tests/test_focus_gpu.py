"""Focal tracker and PID focus control on the GPU.

The tracker reads the temperature increment of every step (debug.T or
transducer.pid), so these runs also exercise the temperature branch.  Without
the controller the tracked depths match the oracle's.  With it the source's
focus moves every step and the focused source's hard aperture edge (a boundary
cell is active while its distance to the focus is at most the focal distance)
turns rounding-level differences into a different source, so the controlled
run is checked against the controller's own arithmetic instead: every control
depth follows from the tracked depths by focal_PID and the clamp.
"""
import math

import numpy as np
import pytest

import _bind as B
import crp
from test_parity_gpu import TOL_FP64

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_tracked_depths_match_oracle():
    cfg = B.small_config()
    steps = 200
    cpu = B.OracleSim(cfg)
    cpu.step(steps)
    with crp.Sim(cfg) as gpu:
        gpu.step(steps)
        a, b = gpu.focus_history("actual"), cpu.focus_history("actual")
        assert a.shape == b.shape == (steps + 1,)
        assert _rel(a, b) < 1e-9, _rel(a, b)
        assert b[-1] > 0.0
        assert np.array_equal(gpu.focus_history("control"), cpu.focus_history("control"))
        for k in ("T", "p0"):
            assert _rel(gpu.field(k), cpu.field(k)) < TOL_FP64, k


def test_control_depths_follow_the_pid():
    start = 20
    cfg = B.small_config(tr_pid=1, tr_pid_start_step=start)
    steps = 150
    with crp.Sim(cfg) as gpu:
        gpu.step(steps)
        a, c = gpu.focus_history("actual"), gpu.focus_history("control")
    assert len(a) == steps + 1 and len(c) == 1 + steps - start
    ty = cfg.tr_focal_dist * 0.5 * math.sqrt(3.0)
    K, Pc = 0.2 * 0.60, 1000.0
    D, I = K * 0.125 * Pc, K / (0.5 * Pc)
    cum = 0.0
    expect = [c[0]]
    for n in range(start + 1, steps + 1):  # control from step pid_start_step + 1 on
        e = ty - a[n]
        cum += e
        y = ty + (K * e + D * (a[n - 1] - a[n]) + I * cum)
        expect.append(min(max(y, ty), cfg.grid_ly))
    assert abs(c[0] - ty) < 1e-15
    np.testing.assert_allclose(c, expect, rtol=1e-13, atol=0.0)
    assert c[-1] != c[0]


def test_focus_state_carries_to_the_next_pass():
    """transducer.pid_iterate: the second pass starts from the first one's
    control point, PID sums and filter state (pid_init of solve_bubbles)."""
    cfg = B.small_config(tr_pid=1, tr_pid_start_step=5)
    with crp.Sim(cfg) as first:
        first.step(40)
        st = first.focus_state()
        last = first.focus_history("control")[-1]
    assert st.control_y == last
    with crp.Sim(cfg) as second:
        second.set_focus_state(st)
        assert second.focus_history("control")[0] == last
        second.step(10)
        st2 = second.focus_state()
        assert st2.err_total_y != st.err_total_y
