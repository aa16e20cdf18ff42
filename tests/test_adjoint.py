"""Source elements of the pressure source on the CPU oracle (the reference for
the CUDA path's phased source and its adjoint, tests/test_adjoint_gpu.py).

Elements have no counterpart in the reference; with their defaults (amplitude 1,
phase 0) the source, and so every field, must be exactly the reference's.
"""
import numpy as np

import _bind as B

STEPS = 150


def _cfg(**over):
    base = dict(bub_enable=0, ext_elements=4)
    base.update(over)
    return B.small_config(**base)


def test_default_elements_leave_the_fields_unchanged():
    with_el, without = B.OracleSim(_cfg()), B.OracleSim(_cfg(ext_elements=0))
    try:
        with_el.step(STEPS)
        without.step(STEPS)
        for name in ("p0", "vx", "vy"):
            assert np.array_equal(with_el.field(name), without.field(name)), name
    finally:
        with_el.close()
        without.close()


def test_objective_is_quadratic_in_the_amplitudes():
    """Without bubbles the step is linear in the source, so J(2a) = 4 J(a)."""
    cfg = _cfg()
    rng = np.random.default_rng(11)
    amp, phase = rng.uniform(0.5, 1.5, 4), rng.uniform(-1.0, 1.0, 4)
    J1 = B.oracle_focal_objective(cfg, amp, phase, STEPS, 2.5e-3)
    J2 = B.oracle_focal_objective(cfg, 2.0 * amp, phase, STEPS, 2.5e-3)
    assert J1 > 0
    assert abs(J2 - 4.0 * J1) <= 1e-12 * J2


def test_elements_need_a_pressure_source():
    import crp
    import pytest

    with pytest.raises(crp.CrpError):
        B.OracleSim(_cfg(tr_focused_p=0, tr_focused_v=1))
