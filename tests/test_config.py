"""Configuration keys, defaults and grammar of the reference's Boost config files
(src/bubbles.cpp:61-195)."""
import os

import pytest

import crp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _reference_root():
    """Root of the reference tree recorded by oracle/build_ref.sh, if it ran here."""
    p = os.path.join(ROOT, "oracle", "_ref", "reference_root")
    return open(p).read().strip() if os.path.exists(p) else ""


REF_SAMPLE = os.path.join(_reference_root(), "confs", "Sample.txt") if _reference_root() else ""


def test_defaults_are_the_reference_defaults():
    c = crp.defaults()
    assert (c.tr_pid, c.tr_pid_start_step, c.tr_init_control, c.tr_pid_iterate) == (0, 1, 0.0, 1)
    assert c.bub_enable == 0 and c.dbg_display == 4
    assert (c.dbg_fg, c.dbg_T, c.dbg_p, c.dbg_v, c.dbg_bubbles) == (1, 1, 0, 0, 1)
    assert (c.ext_rho_inf, c.ext_c_inf, c.ext_p_inf) == (1000.0, 1500.0, 1e5)


def test_small_conf_values():
    c = crp.parse_file(os.path.join(ROOT, "tests", "golden", "small.conf"))
    assert (c.grid_x, c.grid_y, c.grid_lx, c.grid_ly) == (48, 96, 4.8e-3, 9.6e-3)
    assert (c.pml_x0, c.pml_x1, c.pml_y0, c.pml_y1, c.pml_grid_number) == (0, 1, 0, 1, 8)
    assert c.tr_focused_p == 1 and c.tr_cylindrical == 1 and c.bub_enable == 1
    assert c.bub_K0 == 26.2e-3 and c.bub_sigma == 7.2e-2


GRAMMAR = """
sph = 1
# comment line
[grid]
x	=	300   # trailing comment
lx = 30e-3
[pml]
x1 = true
y1 = yes
x0 = off
[transducer]
plane_wave_p = 1
transducer_p = 1
[ext]
precision = mixed
cloud_shape = gaussian
bubble_seed = 0xC0DA0001
"""


def test_grammar():
    c = crp.parse_string(GRAMMAR)
    assert c.opt_sph == 1 and c.grid_x == 300 and c.grid_lx == 30e-3
    assert (c.pml_x1, c.pml_y1, c.pml_x0) == (1, 1, 0)
    assert c.tr_plane_p == 1  # transducer.transducer_p; plane_wave_p is not a registered key
    assert c.ext_precision == 1 and c.ext_cloud_shape == 2 and c.ext_bubble_seed == 0xC0DA0001


@pytest.mark.parametrize("text", ["[grid]\nx = 3.5\n", "[grid]\nx = 3\nx = 4\n", "[pml]\nx0 = maybe\n",
                                  "[grid\nx=1\n", "[grid]\nx\n"])
def test_grammar_errors(text):
    with pytest.raises(crp.CrpError) as e:
        crp.parse_string(text)
    assert e.value.status == 9


def test_unknown_keys_ignored():
    c = crp.parse_string("[grid]\nx = 5\nnot_a_key = 7\n[nosection]\nfoo = bar\n")
    assert c.grid_x == 5


@pytest.mark.skipif(not os.path.exists(REF_SAMPLE), reason="reference tree not present")
def test_reference_sample_parses():
    """confs/Sample.txt gives the values Boost would store (unregistered keys dropped)."""
    c = crp.parse_file(REF_SAMPLE)
    assert (c.grid_x, c.grid_y, c.grid_lx, c.grid_ly) == (300, 600, 30e-3, 60e-3)
    assert (c.pml_x0, c.pml_x1, c.pml_y0, c.pml_y1, c.pml_grid_number, c.pml_sigma, c.pml_order) == \
        (0, 1, 0, 1, 10, 0.10, 2)
    assert (c.sim_cfl, c.sim_dt0, c.sim_n_step_max, c.sim_t_step_max, c.sim_save_interval, c.sim_order,
            c.sim_smooth_delta_band) == (0.10, 0.10, 20000, 0.0, 100, 2, 2)
    assert (c.tr_amp, c.tr_freq, c.tr_focal_dist, c.tr_pid, c.tr_pid_start_step, c.tr_pid_iterate) == \
        (1.5e-2, 1.0e6, 40e-3, 1, 5000, 2)
    assert (c.tr_box_size, c.tr_cylindrical, c.tr_on_wave, c.tr_off_wave) == (30e-3, 1, 2, 0)
    # plane_wave_v / plane_wave_p are not registered keys (transducer_v/p are).
    assert (c.tr_plane_v, c.tr_plane_p, c.tr_focused_v, c.tr_focused_p) == (0, 0, 0, 1)
    assert (c.bub_enable, c.bub_fg0, c.bub_R0, c.bub_P0, c.bub_T0, c.bub_gamma) == (1, 1e-7, 6.5e-7, 0.1e6, 293.15, 1.4)
    assert (c.bub_sigma, c.bub_mu, c.bub_rho, c.bub_K0) == (7.2e-2, 891e-6, 1e3, 26.2e-3)
    assert (c.dbg_display, c.dbg_fg, c.dbg_T, c.dbg_p, c.dbg_v, c.dbg_bubbles) == (7, 1, 1, 1, 0, 0)
    assert c.opt_sph == 1


def test_seeding_is_reproducible_and_in_cloud():
    c = crp.parse_file(os.path.join(ROOT, "cuda-rp_b200", "configs", "axisym_256x512.conf"))
    a, b = crp.seed_bubbles(c), crp.seed_bubbles(c)
    for u, v in zip((a.x, a.y, a.r0, a.n_b), (b.x, b.y, b.r0, b.n_b)):
        assert (u == v).all()
    import numpy as np

    fy = c.tr_focal_dist * 0.5 * np.sqrt(3.0)
    assert len(a.x) == 4096 and (a.x >= 0).all() and (a.x <= c.ext_cloud_r).all()
    assert (np.abs(a.y - fy) <= c.ext_cloud_h / 2).all()
    med = np.median(a.r0)
    assert abs(med / c.bub_R0 - 1) < 0.05
    assert abs(np.std(np.log(a.r0)) - c.ext_r0_sigma_ln) < 0.02
    # area-uniform in r: E[r^2] = R^2 / 2
    assert abs(np.mean(a.x ** 2) / c.ext_cloud_r ** 2 - 0.5) < 0.03
