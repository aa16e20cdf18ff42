"""ext.rp_reuse: from a step's second Picard iteration on, the radius solve
keeps the results of every bubble whose gathered liquid pressure is bitwise
unchanged since the last solve.  Every input of such a bubble's solve is then
unchanged, so the run must equal the one that re-solves every bubble (the
reference's loop, src/bubble_CUDA.cu:239-276) bit for bit: fields, bubbles,
Picard counts and sub-step counts, in both precisions, both radius schemes,
host-driven and graph steps, 2-D and 3-D."""
import numpy as np
import pytest

import _bind as B
import crp
from test_cart3d import cart3d_small
from test_parity_gpu import CASES

pytestmark = pytest.mark.gpu

BUB = ("x", "y", "R_t", "R_p", "R_n", "d1_R_p", "PG_p", "PL_p", "PL_n", "dt", "Q_B", "v_x", "v_y")


def _run(cfg, steps, bub=None):
    with crp.Sim(cfg, bub) as s:
        for chunk in (steps // 2, steps - steps // 2):
            s.step(chunk)
        st = s.stats()
        fields = ("p0", "vx", "vy", "f_g", "f_gn") + (("vz",) if cfg.ext_grid_z else ())
        out = {k: s.field(k) for k in fields}
        for k in BUB + (("z", "v_z") if cfg.ext_grid_z else ()):
            out["bub_" + k] = s.bubbles(k)
        counts = (st.steps, st.picard_total, st.picard_max, st.picard_stalls, st.rp_substeps_max, st.time)
        return out, counts, st.rp_reused


def _same(a, b):
    (fa, ca, ra), (fb, cb, rb) = a, b
    assert ca == cb, (ca, cb)
    for k in fa:
        assert np.array_equal(fa[k].view(np.uint64), fb[k].view(np.uint64)), k
    return ra, rb


@pytest.mark.parametrize("graphs", [0, 1])
@pytest.mark.parametrize("scheme", [0, 1])
@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("name", ["focus_p", "strong_drive", "focus_v_wall_burst"])
def test_reuse_is_bit_exact_2d(name, prec, scheme, graphs):
    over, steps = CASES[name]
    res = []
    for reuse in (0, 1):
        cfg = B.small_config(**over, ext_precision=prec, ext_rp_scheme=scheme, ext_graphs=graphs,
                             ext_rp_reuse=reuse)
        res.append(_run(cfg, steps))
    r_off, r_on = _same(*res)
    print(name, prec, scheme, graphs, "picard", res[1][1][1], "kept", r_on)
    assert r_off == 0
    if name == "focus_p":
        # The focused wave reaches the cloud's bubbles one after another: the
        # ones it has not reached keep their solves while the others iterate.
        assert r_on > 0


@pytest.mark.parametrize("scheme", [0, 1])
@pytest.mark.parametrize("prec", [0, 1])
def test_reuse_is_bit_exact_3d(prec, scheme):
    res = []
    for reuse in (0, 1):
        cfg = cart3d_small(bubbles=300, tr_amp=0.6e6 / (998 * 1482), ext_precision=prec, ext_rp_scheme=scheme,
                   ext_rp_reuse=reuse)
        res.append(_run(cfg, 70, crp.seed_bubbles3(cfg)))
    r_off, r_on = _same(*res)
    print(prec, scheme, "picard", res[1][1][1], "kept", r_on)
    assert r_off == 0 and r_on > 0
