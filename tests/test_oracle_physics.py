"""Known-answer tests of the physics the oracle restates (no golden vectors exist
in the reference; these pin behaviour the equations imply)."""
import ctypes

import numpy as np
import pytest

import _bind as B
import crp

vp = ctypes.c_void_p


def _p(a):
    return a.ctypes.data_as(vp)


def bubble_params(R0=5e-6, dt0=1e-9):
    PL0, sig = 0.1e6, 0.0725
    return np.array([R0, PL0 + 2 * sig / R0, PL0, 293.15, 1.4, sig, 1.0e-3, 998.0, 26.2e-3, dt0])


def history(bp, R_init, dt_mix, n, dpl=0.0):
    lib = B.oracle_lib()
    lib.crpo_bubble_history.restype = ctypes.c_int64
    lib.crpo_bubble_history.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int32, vp, vp]
    R, PG = np.zeros(n), np.zeros(n)
    total = lib.crpo_bubble_history(_p(bp), R_init, dt_mix, dpl, n, _p(R), _p(PG))
    assert total > 0
    return R, PG, total


def test_equilibrium_bubble_stays_put():
    """PG0 = PL0 + 2 sigma / R0 balances the liquid: R stays at R0."""
    bp = bubble_params()
    R, PG, total = history(bp, bp[0], 1e-8, 400)
    assert np.abs(R / bp[0] - 1).max() < 1e-9
    assert total >= 400 * 10  # at least dt_mix / dt0 sub-steps per mixture step


def test_free_oscillation_frequency_and_damping():
    """A slightly displaced bubble rings between its isothermal and adiabatic
    natural frequencies (surface tension included), near the thermal model's
    omega_N (solveOmegaN), and decays (thermal + viscous damping)."""
    R0 = 5e-6
    bp = bubble_params(R0, dt0=2e-10)
    dt_mix = 2e-9
    n = 6000
    R, _, _ = history(bp, 1.005 * R0, dt_mix, n)
    x = R / R0 - 1
    # zero crossings of the detrended signal give the period
    xc = x - x[n // 2:].mean()
    s = np.signbit(xc)
    idx = np.nonzero(s[1:] != s[:-1])[0]
    assert len(idx) > 6
    period = 2 * np.median(np.diff(idx[:12])) * dt_mix
    omega_meas = 2 * np.pi / period
    alpha = np.zeros(2)
    omega_n = B.oracle_lib().crpo_omega_n(_p(bp.copy()), bp[1], R0, _p(alpha))
    assert abs(omega_meas / omega_n - 1) < 0.15, (omega_meas, omega_n)
    # omega^2 = (3 kappa PG0 - 2 sigma / R0) / (rho R0^2), kappa between 1 and gamma
    rho, PG0, sig = bp[7], bp[1], bp[5]
    w_iso = np.sqrt((3 * 1.0 * PG0 - 2 * sig / R0) / (rho * R0 ** 2))
    w_ad = np.sqrt((3 * 1.4 * PG0 - 2 * sig / R0) / (rho * R0 ** 2))
    assert w_iso < omega_meas < w_ad, (w_iso, omega_meas, w_ad)
    first = np.abs(x[: n // 6]).max()
    last = np.abs(x[-n // 6:] - x[-n // 6:].mean()).max()
    assert last < 0.5 * first


def test_void_fraction_conservation_planar():
    """Partition of unity of the smooth delta: sum f_g dx dy = sum (4/3) pi n_B R^3."""
    cfg = B.small_config(tr_cylindrical=0, tr_box_size=1.6e-3)
    o = B.OracleSim(cfg)
    fg = o.field("f_g")
    R, nb = o.bubbles("R_t"), o.bubbles("n_B")
    lhs = fg.sum() * o.dims.dx * o.dims.dy
    rhs = (4.0 / 3.0 * np.pi * nb * R ** 3).sum()
    assert abs(lhs - rhs) <= 1e-12 * rhs


def plane_wave_cfg(**over):
    base = dict(grid_x=8, grid_y=400, grid_lx=0.8e-3, grid_ly=40e-3, pml_x0=0, pml_x1=0, pml_y0=0, pml_y1=1,
                pml_grid_number=40, pml_sigma=0.001, tr_cylindrical=0, tr_focused_p=0, tr_plane_p=1,
                tr_on_wave=1, tr_off_wave=1000, tr_amp=0.01, sim_cfl=0.5, bub_enable=0)
    base.update(over)
    return B.small_config(**base)


def test_plane_wave_speed():
    """A one-cycle plane pulse travels at c_inf (rigid side walls, no bubbles)."""
    cfg = plane_wave_cfg()
    o = B.OracleSim(cfg)
    j1, j2 = 60, 260
    tr1, tr2 = [], []
    for _ in range(1000):
        o.step(1)
        p = o.field("p0")
        tr1.append(p[j1, 4])
        tr2.append(p[j2, 4])
    tr1, tr2 = np.array(tr1), np.array(tr2)
    # arrival of the pulse peak
    dt = o.dims.dt
    t1 = np.argmax(tr1) * dt
    t2 = np.argmax(tr2) * dt
    c = (j2 - j1) * o.dims.dy / (t2 - t1)
    assert abs(c / 1500.0 - 1) < 0.01, c


def test_pml_absorbs():
    """The y1 PML reflects little of a pulse: compare with a rigid y1 wall."""
    def reflected(pml):
        cfg = plane_wave_cfg(pml_y1=pml, grid_y=300, grid_ly=30e-3)
        o = B.OracleSim(cfg)
        j = 100
        tr = []
        for _ in range(1100):
            o.step(1)
            tr.append(o.field("p0")[j, 4])
        tr = np.array(tr)
        dt, dy = o.dims.dt, o.dims.dy
        # incident pulse passes row j by ~ (j*dy + 1 wavelength)/c; the echo comes later
        t_echo = int(((2 * 300 - j) * dy - 40 * dy * (pml == 1)) / 1500.0 / dt * 0.9)
        inc = np.abs(tr[: int(t_echo * 0.7)]).max()
        ref = np.abs(tr[t_echo:]).max()
        return ref / inc

    r_pml = reflected(1)
    r_wall = reflected(0)
    assert r_wall > 0.5
    assert r_pml < 0.05 * r_wall, (r_pml, r_wall)


def test_focus_tracker_and_pid_histories():
    """Focal tracker and PID (src/bubble_CUDA.cu:123-153, 310-352) in the oracle:
    one tracked depth per step after the initial 0; one control depth per step
    after transducer.pid_start_step, each clamped to [focus depth, LY]; the
    source's focus follows the last control depth."""
    import math

    cfg = B.small_config(tr_pid=1, tr_pid_start_step=10)
    o = B.OracleSim(cfg)
    o.step(40)
    a, c = o.focus_history("actual"), o.focus_history("control")
    fpy = cfg.tr_focal_dist * math.sqrt(3.0) / 2
    assert len(a) == 41 and a[0] == 0.0
    assert len(c) == 1 + 30
    assert abs(c[0] - fpy) < 1e-15
    assert np.all(c >= fpy - 1e-15) and np.all(c <= cfg.grid_ly)
    assert c[-1] != c[0]
    # Without the controller the focus stays where the source aims it.
    o2 = B.OracleSim(B.small_config())
    o2.step(20)
    assert len(o2.focus_history("actual")) == 21 and len(o2.focus_history("control")) == 1


def test_butterworth_filter_settles_to_its_dc_gain():
    """filter_loop's coefficients (inc/bubble_CUDA_kernel.cuh:117-129): a
    constant input settles to 16 / gain / (1 - sum of the feedback
    coefficients) = 0.99723 of itself (the coefficients are rounded) within a
    few thousand steps."""
    xv, yv = [0.0] * 5, [0.0] * 5
    gain = 6.522112693e+08
    out = 0.0
    for _ in range(20000):
        xv = xv[1:] + [1.0 / gain]
        yv = yv[1:] + [0.0]
        yv[4] = ((xv[0] + xv[4]) + 4 * (xv[1] + xv[3]) + 6 * xv[2] + (-0.9676955438 * yv[0]) + (3.9025587848 * yv[1])
                 + (-5.9020258615 * yv[2]) + (3.9671625959 * yv[3]))
        out = yv[4]
    dc = 16.0 / gain / (1.0 - (-0.9676955438 + 3.9025587848 - 5.9020258615 + 3.9671625959))
    assert abs(dc - 0.99723) < 1e-5
    assert abs(out - dc) < 1e-8
