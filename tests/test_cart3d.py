"""The 3-D Cartesian extension (ext.grid_z > 0) on CPU: the oracle's bowl
focuses where its phases aim, the 3-D void fraction is conserved, and the
product's 3-D seeding equals the oracle's bit for bit."""
import ctypes
import os

import numpy as np
import pytest

import _bind as B
import crp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def cart3d_small(N=40, h=2e-4, elems=32, bubbles=0, **over):
    """A small 3-D case: N^3 cells of h, a PML of 6 cells on every face, a bowl
    of `elems` elements 7 cells inside the PML, 1 MHz, 0.2 MPa."""
    c = crp.Config()
    B.oracle_lib().crpo_config_defaults(ctypes.byref(c))
    c.grid_x = c.grid_y = c.ext_grid_z = N
    c.grid_lx = c.grid_ly = c.ext_grid_lz = N * h
    c.pml_x0 = c.pml_x1 = c.pml_y0 = c.pml_y1 = c.ext_pml_z0 = c.ext_pml_z1 = 1
    c.pml_grid_number, c.pml_sigma, c.pml_order = 6, 0.01, 2
    c.sim_cfl, c.sim_order, c.sim_smooth_delta_band = 0.4, 2, 2
    c.tr_amp, c.tr_freq, c.tr_on_wave, c.tr_off_wave = 0.2e6 / (998 * 1482), 1e6, 20, 1000
    c.ext_rho_inf, c.ext_c_inf, c.ext_p_inf, c.ext_ramp_cycles = 998.0, 1482.0, 101325.0, 1.0
    c.ext_array_elements, c.ext_array_radius = elems, (N / 2 - 7) * h
    c.bub_enable = 1 if bubbles else 0
    c.bub_R0, c.bub_P0, c.bub_T0, c.bub_gamma = 3e-6, 101325.0, 293.15, 1.4
    c.bub_sigma, c.bub_mu, c.bub_rho, c.bub_K0 = 0.0725, 1e-3, 998.0, 26.2e-3
    c.ext_bubble_count, c.ext_bubble_seed, c.ext_cloud_shape, c.ext_cloud_r = bubbles, 5, 1, 1e-3
    c.ext_r0_sigma_ln, c.ext_n_b = 0.3, 1.0
    for k, v in over.items():
        setattr(c, k, v)
    return c


@pytest.mark.parametrize("dx_focus", [0.0, 1.0e-3])
def test_bowl_focuses_at_its_focus(dx_focus):
    c = cart3d_small(ext_array_focus_dx=dx_focus)
    o = B.OracleSim3(c)
    assert o.dims3.source_cells > 100
    peak = np.zeros(o.field("p0").shape)
    for _ in range(12):
        o.step(10)
        peak = np.maximum(peak, np.abs(o.field("p0")))
    k, j, i = np.unravel_index(np.argmax(peak[8:-8, 8:-8, 8:-8]), peak[8:-8, 8:-8, 8:-8].shape)
    k, j, i = k + 8, j + 8, i + 8
    h = 2e-4
    xf = 20 * h + dx_focus
    assert abs((i - 0.5) * h - xf) <= 2.5 * h, (i, j, k)
    assert abs((j - 0.5) * h - 20 * h) <= 2.5 * h and abs((k - 0.5) * h - 20 * h) <= 2.5 * h
    assert peak.max() > 5 * 0.2e6  # focal gain of the bowl


def test_void_fraction_conservation_3d():
    c = cart3d_small(bubbles=300)
    o = B.OracleSim3(c, B.oracle_seed_bubbles3(c))
    fg = o.field("f_g")
    R, nb = o.bubbles("R_t"), o.bubbles("n_B")
    lhs = fg.sum() * (2e-4) ** 3
    rhs = (4.0 / 3.0 * np.pi * nb * R ** 3).sum()
    assert abs(lhs - rhs) <= 1e-12 * rhs


@pytest.mark.parametrize("shape", [0, 1, 2])
def test_seeding3_matches(shape):
    c = cart3d_small(bubbles=2049, ext_cloud_shape=shape, ext_cloud_h=2e-3, ext_array_focus_dx=5e-4)
    a, b = crp.seed_bubbles3(c), B.oracle_seed_bubbles3(c)
    for u, v in zip((a.x, a.y, a.z, a.r0, a.n_b), (b.x, b.y, b.z, b.r0, b.n_b)):
        assert np.array_equal(u.view(np.uint64), v.view(np.uint64))


def test_3d_bubbles_at_rest_stay():
    c = cart3d_small(bubbles=100, tr_amp=0.0)
    o = B.OracleSim3(c, B.oracle_seed_bubbles3(c))
    o.step(30)
    R, R0 = o.bubbles("R_t"), o.bubbles("R0")
    assert np.abs(R / R0 - 1).max() < 1e-10
