"""crp_save_state / crp_load_state: a simulation put back to a snapshot
continues bit for bit as it did after the save (2-D in both precisions, host
and graph steps, the temperature branch with its focal history; 3-D), also in
a second handle made from the same configuration; snapshots of another shape
are refused."""
import numpy as np
import pytest

import _bind as B
import crp
from test_cart3d import cart3d_small
from test_parity_gpu import CASES

pytestmark = pytest.mark.gpu


def _state(sim, three=False):
    fields = ("p0", "vx", "vy", "f_g", "f_gn", "f_gm") + (("vz",) if three else ())
    out = {k: sim.field(k) for k in fields}
    if sim.dims.num_bubbles:
        for k in ("R_t", "PG_p", "PL_p", "x", "y", "d1_R_p"):
            out["bub_" + k] = sim.bubbles(k)
    st = sim.stats()
    out["stats"] = np.array([st.steps, st.picard_total, st.picard_max, st.rp_substeps_max, st.rp_reused])
    out["time"] = np.array([st.time])
    return out


def _same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("graphs", [0, 1])
@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("name", ["focus_p", "strong_drive"])
def test_load_continues_bit_for_bit(name, prec, graphs):
    over, _ = CASES[name]
    cfg = B.small_config(**over, ext_precision=prec, ext_graphs=graphs)
    with crp.Sim(cfg) as sim:
        sim.step(50)
        snap = sim.save_state()
        sim.step(40)
        a = _state(sim)
        sim.load_state(snap)
        sim.step(40)
        b = _state(sim)
        _same(a, b)
        # A snapshot object is overwritten by the next save of the same simulation.
        sim.save_state(snap)
        sim.step(10)
        sim.load_state(snap)
        _same(_state(sim), b)
        with crp.Sim(cfg) as other:
            other.load_state(snap)
            other.step(10)
            sim.step(10)
            _same(_state(other), _state(sim))
        snap.free()


def test_temperature_branch_and_focus_history():
    cfg = B.small_config(dbg_T=1)
    with crp.Sim(cfg) as sim:
        sim.step(60)
        snap = sim.save_state()
        sim.step(30)
        a, ha, ta = _state(sim), sim.focus_history("actual"), sim.field("T")
        assert len(ha) == 91
        sim.load_state(snap)
        assert len(sim.focus_history("actual")) == 61
        sim.step(30)
        _same(a, _state(sim))
        assert np.array_equal(ha, sim.focus_history("actual"))
        assert np.array_equal(ta, sim.field("T"))


@pytest.mark.parametrize("prec", [0, 1])
def test_3d_load_continues_bit_for_bit(prec):
    cfg = cart3d_small(bubbles=300, tr_amp=0.6e6 / (998 * 1482), ext_precision=prec)
    bub = crp.seed_bubbles3(cfg)
    with crp.Sim(cfg, bub) as sim:
        sim.step(30)
        snap = sim.save_state()
        sim.step(30)
        a = _state(sim, True)
        sim.load_state(snap)
        sim.step(30)
        _same(a, _state(sim, True))


def test_snapshot_of_another_shape_is_refused():
    a, b = B.small_config(), B.small_config(grid_x=32, grid_y=64, grid_lx=3.2e-3, grid_ly=6.4e-3)
    with crp.Sim(a) as sa, crp.Sim(b) as sb:
        snap = sa.save_state()
        with pytest.raises(crp.CrpError) as e:
            sb.load_state(snap)
        assert e.value.status == 1  # CRP_ERR_INVALID
        with pytest.raises(crp.CrpError):
            sb.save_state(snap)
