"""crp_adjoint (C ABI): the gradient of the focal objective with respect to the
source elements' amplitudes and phases, from the hand-written discrete adjoint
of the FDTD/PML step, against

- central finite differences of J on the CUDA path itself (amplitudes: J is
  quadratic in them, so the difference quotient is exact up to rounding;
  phases: h = 1e-4 rad, truncation O(h^2));
- an FP64 reference gradient: central finite differences of J on the CPU
  oracle (the accuracy bar: within 1e-3 relative);
- torch.autograd.gradcheck through a thin torch.autograd.Function whose
  backward is crp_adjoint (only here, for the gradient tests).

Three configurations cover the source placements and boundaries the adjoint
handles: the reference's source on the y = 0 ghost row (no y0 PML, axis at x0,
cylindrical), an [ext] source row above a y0 PML with a burst ramp, and a
planar plane source with a PML at x0.
"""
import numpy as np
import pytest

import _bind as B
import crp

pytestmark = pytest.mark.gpu

STEPS = 300
RADIUS = 2.5e-3
CASES = {
    "ghost_row_focused": dict(),
    "source_row_ramp": dict(pml_y0=1, ext_source_row=9, ext_ramp_cycles=0.5),
    "planar_plane_pml_x0": dict(tr_cylindrical=0, tr_focused_p=0, tr_plane_p=1, pml_x0=1, ext_elements=3),
}


def _cfg(name, **over):
    base = dict(bub_enable=0, ext_elements=4)
    base.update(CASES[name])
    base.update(over)
    return B.small_config(**base)


def _params(n, seed=5):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.5, 1.5, n), rng.uniform(-1.0, 1.0, n)


def gpu_objective(cfg, amp, phase, steps=STEPS, grads=False):
    n = cfg.ext_elements
    with crp.Sim(cfg) as sim:
        sim.set_source_elements(amp, phase)
        J, ga, gp = sim.adjoint(steps, RADIUS, n if grads else 0)
    return (J, ga, gp) if grads else J


@pytest.mark.parametrize("name", list(CASES))
def test_objective_matches_the_oracle(name):
    cfg = _cfg(name)
    amp, phase = _params(cfg.ext_elements)
    J = gpu_objective(cfg, amp, phase)
    Jo = B.oracle_focal_objective(cfg, amp, phase, STEPS, RADIUS)
    assert Jo > 0
    assert abs(J - Jo) <= 1e-9 * Jo, (J, Jo)


@pytest.mark.parametrize("name", list(CASES))
def test_gradient_matches_finite_differences(name):
    cfg = _cfg(name)
    n = cfg.ext_elements
    amp, phase = _params(n)
    J, ga, gp = gpu_objective(cfg, amp, phase, grads=True)
    scale = max(np.abs(ga).max(), np.abs(gp).max())
    for e in range(n):
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


@pytest.mark.parametrize("name", list(CASES))
def test_gradient_matches_the_fp64_reference_gradient(name):
    cfg = _cfg(name)
    n = cfg.ext_elements
    amp, phase = _params(n, seed=9)
    _, ga, gp = gpu_objective(cfg, amp, phase, grads=True)
    ref_a, ref_p = np.zeros(n), np.zeros(n)
    for e in range(n):
        h = 1e-4 * amp[e]
        a1, a2 = amp.copy(), amp.copy()
        a1[e] += h
        a2[e] -= h
        ref_a[e] = (B.oracle_focal_objective(cfg, a1, phase, STEPS, RADIUS)
                    - B.oracle_focal_objective(cfg, a2, phase, STEPS, RADIUS)) / (2 * h)
        h = 1e-4
        p1, p2 = phase.copy(), phase.copy()
        p1[e] += h
        p2[e] -= h
        ref_p[e] = (B.oracle_focal_objective(cfg, amp, p1, STEPS, RADIUS)
                    - B.oracle_focal_objective(cfg, amp, p2, STEPS, RADIUS)) / (2 * h)
    scale = max(np.abs(ref_a).max(), np.abs(ref_p).max())
    assert np.abs(ga - ref_a).max() <= 1e-3 * scale, (ga, ref_a)
    assert np.abs(gp - ref_p).max() <= 1e-3 * scale, (gp, ref_p)
    print(name, "max |adjoint - oracle FD| / scale:", np.abs(ga - ref_a).max() / scale, np.abs(gp - ref_p).max() / scale)


def test_gradient_through_torch_autograd():
    import torch

    cfg = _cfg("ghost_row_focused", grid_x=32, grid_y=64, grid_lx=3.2e-3, grid_ly=6.4e-3, tr_focal_dist=5.0e-3,
               ext_elements=3)
    steps = 200

    class FocalObjective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, amp, phase):
            J, ga, gp = gpu_objective(cfg, amp.detach().numpy(), phase.detach().numpy(), steps, grads=True)
            ctx.save_for_backward(torch.from_numpy(ga), torch.from_numpy(gp))
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, g):
            ga, gp = ctx.saved_tensors
            return g * ga, g * gp

    amp = torch.tensor([0.9, 1.2, 0.7], dtype=torch.float64, requires_grad=True)
    phase = torch.tensor([0.3, -0.5, 0.1], dtype=torch.float64, requires_grad=True)
    J = FocalObjective.apply(amp, phase)
    assert J.item() > 0
    assert torch.autograd.gradcheck(FocalObjective.apply, (amp, phase), eps=1e-5, atol=1e-8 * J.item(), rtol=1e-5)


def test_default_elements_leave_the_fields_unchanged():
    for over in (dict(), dict(bub_enable=1)):
        a_cfg, b_cfg = _cfg("ghost_row_focused", **over), _cfg("ghost_row_focused", ext_elements=0, **over)
        with crp.Sim(a_cfg) as a, crp.Sim(b_cfg) as b:
            a.step(150)
            b.step(150)
            for name in ("p0", "vx", "vy"):
                assert np.array_equal(a.field(name), b.field(name)), (over, name)


def test_unsupported_and_invalid():
    with crp.Sim(_cfg("ghost_row_focused", bub_enable=1)) as sim:
        with pytest.raises(crp.CrpError) as e:
            sim.adjoint(10, RADIUS, 4)
        assert e.value.status == 2  # CRP_ERR_UNSUPPORTED
    with crp.Sim(_cfg("ghost_row_focused", ext_elements=0)) as sim:
        J, ga, gp = sim.adjoint(10, RADIUS, 0)  # J alone needs no elements
        assert ga is None and J >= 0
    with crp.Sim(_cfg("ghost_row_focused")) as sim:
        with pytest.raises(crp.CrpError):
            sim.set_source_elements(np.ones(3), np.zeros(3))  # n must equal ext.elements


def test_mixed_path_forward_gives_the_same_gradient():
    """The reverse sweep is FP64 in both paths; with the mixed path's forward
    (FP32 value + compensation fields) J and the gradient move only by that
    storage's rounding."""
    cfg64 = _cfg("source_row_ramp")
    cfgmx = _cfg("source_row_ramp", ext_precision=1)
    amp, phase = _params(cfg64.ext_elements)
    J64, ga64, gp64 = gpu_objective(cfg64, amp, phase, grads=True)
    Jmx, gamx, gpmx = gpu_objective(cfgmx, amp, phase, grads=True)
    scale = max(np.abs(ga64).max(), np.abs(gp64).max())
    assert abs(Jmx - J64) <= 1e-6 * J64
    assert np.abs(gamx - ga64).max() <= 1e-6 * scale
    assert np.abs(gpmx - gp64).max() <= 1e-6 * scale


def test_repeated_calls_reuse_the_workspace():
    # crp_adjoint keeps its device workspace with the handle.  Calls of 60,
    # 120 and 40 steps (the workspace grows, then is reused larger than
    # needed) each continue from the state the previous call left, and give
    # exactly what a fresh handle advanced to that state by crp_step gives.
    cfg = _cfg("ghost_row_focused")
    amp, phase = _params(cfg.ext_elements)
    n = cfg.ext_elements
    with crp.Sim(cfg) as a:
        a.set_source_elements(amp, phase)
        got = [a.adjoint(steps, RADIUS, n) for steps in (60, 120, 40)]
    before = 0
    for steps, (J, ga, gp) in zip((60, 120, 40), got):
        with crp.Sim(cfg) as b:
            b.set_source_elements(amp, phase)
            if before:
                b.step(before)
            Jb, gab, gpb = b.adjoint(steps, RADIUS, n)
        assert J == Jb and np.array_equal(ga, gab) and np.array_equal(gp, gpb), steps
        before += steps
