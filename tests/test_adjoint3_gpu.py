"""crp_adjoint on the 3-D grid (ext.grid_z > 0, bubbles off): the gradient of
the focal objective J = sum over the steps of dt sum w p0^2 (w = dx dy dz over
the cells within the focal radius of the bowl's focus) with respect to the
hemispherical array's element amplitudes and phases, from the hand-written
adjoint of the 3-D FDTD/PML step, against

- J from the 3-D oracle's p0 after every step (1e-9);
- central finite differences of J on the CUDA path (amplitudes: J is
  quadratic in them; phases: h = 1e-4 rad);
- central finite differences on the FP64 oracle (the accuracy bar: 1e-3).
"""
import numpy as np
import pytest

import _bind as B
import crp
from test_cart3d import cart3d_small

pytestmark = pytest.mark.gpu

STEPS = 110
RADIUS = 0.7e-3
ELEMS = 8
H = 2e-4


def _cfg(**over):
    return cart3d_small(N=40, elems=ELEMS, **over)


def _params():
    rng = np.random.default_rng(3)
    return rng.uniform(0.6, 1.4, ELEMS), None


def gpu_objective(cfg, amp=None, phase=None, grads=False):
    with crp.Sim(cfg) as sim:
        if amp is not None:
            sim.set_source_elements(amp, phase)
        J, ga, gp = sim.adjoint(STEPS, RADIUS, ELEMS if grads else 0)
        dt = sim.dims3.dt
    return (J, ga, gp, dt) if grads else J


def default_phases(cfg):
    """The bowl's focusing phases (omega |x_e - focus| / c mod 2 pi), as crp_create sets them."""
    n, Ra = cfg.ext_array_elements, cfg.ext_array_radius
    N = cfg.grid_x
    c = 0.5 * N * H
    golden = np.pi * (3.0 - np.sqrt(5.0))
    e = np.arange(n)
    ct = -(e + 0.5) / n
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    x, y, z = c + Ra * st * np.cos(golden * e), c + Ra * st * np.sin(golden * e), c + Ra * ct
    d = np.sqrt((x - c - cfg.ext_array_focus_dx) ** 2 + (y - c) ** 2 + (z - c) ** 2)
    return np.fmod(2 * np.pi * cfg.tr_freq * d / cfg.ext_c_inf, 2 * np.pi)


def oracle_objective(cfg, amp, phase, dt):
    sim = B.OracleSim3(cfg)
    try:
        sim.set_source_elements(amp, phase)
        N = cfg.grid_x
        idx = np.arange(N + 2)
        cc = (idx - 0.5) * H - 0.5 * N * H
        zz, yy, xx = np.meshgrid(cc, cc, cc - cfg.ext_array_focus_dx, indexing="ij")
        inside = (xx ** 2 + yy ** 2 + zz ** 2 <= RADIUS ** 2)
        inside[0, :, :] = inside[-1, :, :] = inside[:, 0, :] = inside[:, -1, :] = False
        inside[:, :, 0] = inside[:, :, -1] = False
        w = np.where(inside, H ** 3, 0.0)
        J = 0.0
        for _ in range(STEPS):
            sim.step(1)
            p0 = sim.field("p0")
            J += dt * float(np.sum(w * p0 * p0))
        return J
    finally:
        sim.close()


def test_objective_matches_the_oracle():
    cfg = _cfg()
    amp = _params()[0]
    phase = default_phases(cfg)
    J, ga, gp, dt = gpu_objective(cfg, amp, phase, grads=True)
    Jo = oracle_objective(cfg, amp, phase, dt)
    assert Jo > 0
    assert abs(J - Jo) <= 1e-9 * Jo, (J, Jo)


def test_gradient_matches_finite_differences():
    cfg = _cfg()
    amp = _params()[0]
    phase = default_phases(cfg)
    J, ga, gp, _ = gpu_objective(cfg, amp, phase, grads=True)
    scale = max(np.abs(ga).max(), np.abs(gp).max())
    assert scale > 0
    for e in range(ELEMS):
        h = 1e-4 * amp[e]
        a1, a2 = amp.copy(), amp.copy()
        a1[e] += h
        a2[e] -= h
        fd = (gpu_objective(cfg, a1, phase) - gpu_objective(cfg, a2, phase)) / (2 * h)
        assert abs(fd - ga[e]) <= 1e-6 * scale, ("amp", e, fd, ga[e])
        h = 1e-4
        p1, p2 = phase.copy(), phase.copy()
        p1[e] += h
        p2[e] -= h
        fd = (gpu_objective(cfg, amp, p1) - gpu_objective(cfg, amp, p2)) / (2 * h)
        assert abs(fd - gp[e]) <= 1e-5 * scale, ("phase", e, fd, gp[e])


def test_gradient_matches_the_oracle():
    cfg = _cfg()
    amp = _params()[0]
    phase = default_phases(cfg)
    J, ga, gp, dt = gpu_objective(cfg, amp, phase, grads=True)
    scale = max(np.abs(ga).max(), np.abs(gp).max())
    for e in (0, ELEMS - 1):
        h = 1e-4 * amp[e]
        a1, a2 = amp.copy(), amp.copy()
        a1[e] += h
        a2[e] -= h
        fd = (oracle_objective(cfg, a1, phase, dt) - oracle_objective(cfg, a2, phase, dt)) / (2 * h)
        assert abs(fd - ga[e]) <= 1e-3 * scale, ("amp", e, fd, ga[e])
        h = 1e-4
        p1, p2 = phase.copy(), phase.copy()
        p1[e] += h
        p2[e] -= h
        fd = (oracle_objective(cfg, amp, p1, dt) - oracle_objective(cfg, amp, p2, dt)) / (2 * h)
        assert abs(fd - gp[e]) <= 1e-3 * scale, ("phase", e, fd, gp[e])


def test_bubbles_are_unsupported():
    cfg = _cfg(bubbles=50)
    with crp.Sim(cfg, crp.seed_bubbles3(cfg)) as sim:
        with pytest.raises(crp.CrpError) as e:
            sim.adjoint(10, RADIUS, ELEMS)
        assert e.value.status == 2  # CRP_ERR_UNSUPPORTED


def test_repeated_calls_reuse_the_workspace():
    # As on the 2-D grid: the kept workspace, grown and then reused, gives
    # each call exactly what a fresh handle stepped to the same state gives.
    cfg = _cfg()
    amp, _ = _params()
    with crp.Sim(cfg) as a:
        a.set_source_elements(amp, default_phases(cfg))
        got = [a.adjoint(steps, RADIUS, ELEMS) for steps in (30, 60, 20)]
    before = 0
    for steps, (J, ga, gp) in zip((30, 60, 20), got):
        with crp.Sim(cfg) as b:
            b.set_source_elements(amp, default_phases(cfg))
            if before:
                b.step(before)
            Jb, gab, gpb = b.adjoint(steps, RADIUS, ELEMS)
        assert J == Jb and np.array_equal(ga, gab) and np.array_equal(gp, gpb), steps
        before += steps
