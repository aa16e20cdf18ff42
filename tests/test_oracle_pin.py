"""The oracle against the reference's own code.

Two pins: golden vectors produced by the reference's functions compiled on the
host (tests/golden/ref_host.npz, made by tests/golden/make_ref_golden.py host),
and — where oracle/_ref is built — the same functions called live on fresh
inputs.  Host arithmetic is compared bit for bit.
"""
import ctypes
import os

import numpy as np
import pytest

import _bind as B
import crp

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_host.npz")
vp = ctypes.c_void_p


def _p(a):
    return a.ctypes.data_as(vp)


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


HOST_CASES = {
    "small": {},
    "planar_pml_all": dict(pml_x0=1, pml_y0=1, tr_cylindrical=0, pml_order=3, pml_sigma=0.01, pml_grid_number=5),
    "sample_like": dict(grid_x=300, grid_y=600, grid_lx=30e-3, grid_ly=60e-3, pml_grid_number=10, sim_cfl=0.1,
                        tr_amp=1.5e-2, tr_focal_dist=40e-3, tr_box_size=30e-3, bub_fg0=1e-7, bub_R0=6.5e-7,
                        bub_mu=891e-6, tr_pid=1, tr_pid_start_step=5000),
}


@pytest.mark.parametrize("name", list(HOST_CASES))
def test_scalars_sigma_bubbles_match_reference(gold, name):
    cfg = B.small_config(**HOST_CASES[name])
    o = B.oracle_lib()
    sc = np.zeros(21)
    o.crpo_host_scalars(ctypes.byref(cfg), _p(sc))
    assert np.array_equal(sc, gold[f"{name}/scalars"])
    X, Y = cfg.grid_x, cfg.grid_y
    arrs = [np.zeros(n) for n in (X + 2, Y + 2, X + 3, Y + 3, X + 3, X + 2)]
    o.crpo_host_sigma(ctypes.byref(cfg), *[_p(a) for a in arrs])
    for k, a in zip(["mx", "my", "nx", "ny", "xu", "rxp"], arrs):
        assert np.array_equal(a, gold[f"{name}/{k}"]), k
    # Lattice bubbles: positions, weights, radius, gas pressure of bubble_input.
    if cfg.bub_enable:
        sim = B.OracleSim(cfg)
        n = sim.dims.num_bubbles
        assert n == int(gold[f"{name}/bubble_count"])
        g = gold[f"{name}/bubbles"]
        step = max(1, n // 500)
        assert np.array_equal(sim.bubbles("x")[::step], g[:, 0])
        assert np.array_equal(sim.bubbles("y")[::step], g[:, 1])
        assert np.array_equal(sim.bubbles("n_B")[::step], g[:, 2])
        assert np.array_equal(sim.bubbles("R_t")[::step], g[:, 3])
        assert np.array_equal(sim.bubbles("PG_p")[::step], g[:, 4])
        assert np.array_equal(sim.bubbles("dt")[::step], g[:, 5])


def test_bubble_physics_matches_reference(gold):
    o = B.oracle_lib()
    bp = gold["phys/bp"]
    rp_in, rp_out = gold["phys/rp_in"], gold["phys/rp_out"]
    PG, PL, R = gold["phys/PG"], gold["phys/PL"], gold["phys/R"]
    m = len(R)
    for k in range(m):
        st = rp_in[k].copy()
        o.crpo_rp_step(_p(bp[k].copy()), _p(st), PG[k], PL[k])
        assert np.array_equal(st, rp_out[k]), k
        a = np.zeros(2)
        w = o.crpo_omega_n(_p(bp[k].copy()), PG[k], R[k], _p(a))
        assert w == gold["phys/omega"][k] and np.array_equal(a, gold["phys/alpha"][k]), k
    ul = gold["phys/ups_lp"]
    for k in range(len(ul)):
        out = np.zeros(4)
        o.crpo_upsilon_lp(gold["phys/a_re"][k], gold["phys/a_im"][k], 1.4, R[k % m], _p(out))
        assert np.array_equal(out, ul[k]), k
    lp = ul[:m, 2:4]
    for k in range(m):
        v = o.crpo_solve_pg(_p(bp[k].copy()), PG[k], rp_in[k, 1], R[k], gold["phys/omega"][k] + 1.0,
                            rp_in[k, 4], lp[k, 0], lp[k, 1])
        assert v == gold["phys/pg"][k], k


@pytest.mark.skipif(not B.ref_available(), reason="oracle/_ref not built")
def test_live_reference_on_fresh_inputs():
    """Fresh random inputs through both implementations (not only the fixture)."""
    r, o = B.ref_lib(), B.oracle_lib()
    rng = np.random.default_rng(12345)
    for _ in range(300):
        R0 = 10 ** rng.uniform(-6.8, -4.8)
        PL0 = rng.uniform(5e4, 2e5)
        bp = np.array([R0, PL0 + 2 * 0.0725 / R0, PL0, 293.15, rng.uniform(1.1, 1.67), 0.0725,
                       rng.uniform(5e-4, 2e-3), 998.0, 0.026, 10 ** rng.uniform(-10.5, -8.5)])
        st0 = np.array([R0 * rng.uniform(0.1, 5), R0 * rng.uniform(0.1, 5), R0, rng.normal(0, 20), bp[9] * 0.9,
                        bp[9] * rng.uniform(0.1, 20)])
        pg, pl = bp[1] * rng.uniform(0.01, 100), rng.uniform(-1e6, 5e6)
        a, b = st0.copy(), st0.copy()
        r.crp_ref_rp_step(_p(bp.copy()), _p(a), pg, pl)
        o.crpo_rp_step(_p(bp.copy()), _p(b), pg, pl)
        assert np.array_equal(a, b)
        al_r, al_o = np.zeros(2), np.zeros(2)
        wr = r.crp_ref_omega_n(_p(bp.copy()), pg, st0[0], _p(al_r))
        wo = o.crpo_omega_n(_p(bp.copy()), pg, st0[0], _p(al_o))
        assert wr == wo and np.array_equal(al_r, al_o)


@pytest.mark.skipif(not B.ref_available(), reason="oracle/_ref not built")
def test_live_reference_array_index():
    """init_array's 28 index bounds for several grid sizes and FDTD orders."""
    r = B.ref_lib()
    for X, Y, order in [(48, 96, 2), (7, 3, 2), (300, 600, 2), (20, 30, 4)]:
        cfg = B.small_config(grid_x=X, grid_y=Y, sim_order=order)
        ai = np.zeros(28, np.int32)
        r.crp_ref_host_array_index(ctypes.byref(B.ref_params(cfg)), _p(ai))
        ms, me, ns, ne = ai[:4]
        assert (ms, me, ns, ne) == (-order // 2 + 1, order // 2, -order // 2, order // 2 - 1)
        if order == 2:
            sim = B.OracleSim(cfg)
            d = sim.dims
            # i1m = iend1m - ista1m + 1 etc. (src/bubble_CUDA.cu:1242-1249)
            assert d.i1m == ai[9] - ai[8] + 1 and d.i2m == ai[13] - ai[12] + 1 and d.i2n == ai[15] - ai[14] + 1
            assert d.j1m == ai[21] - ai[20] + 1 and d.j2m == ai[25] - ai[24] + 1 and d.j2n == ai[27] - ai[26] + 1
