"""Batched sweep (crp_batch): concurrent simulations give the results of the
same simulations run one by one, bit for bit."""
import numpy as np
import pytest

import _bind as B
import crp

pytestmark = pytest.mark.gpu


def _configs():
    a = B.small_config()
    b = B.small_config(grid_x=32, grid_y=64, grid_lx=3.2e-3, grid_ly=6.4e-3, tr_box_size=1.0e-3, tr_amp=0.3)
    c = B.small_config(tr_cylindrical=0, tr_freq=2.0e6, ext_bubble_count=200, ext_bubble_seed=11,
                       ext_cloud_r=1.0e-3, ext_cloud_h=2.0e-3, ext_r0_sigma_ln=0.3)
    d = B.small_config(grid_x=64, grid_y=128, grid_lx=6.4e-3, grid_ly=12.8e-3, tr_focal_dist=10e-3, bub_enable=0)
    return [a, b, c, d]


def _state(sim):
    out = [sim.field(k) for k in ("p0", "vx", "vy", "f_g")]
    if sim.dims.num_bubbles:
        out.append(sim.bubbles("R_t"))
    return out


def test_batch_matches_individual_runs():
    cfgs = _configs()
    steps = [60, 45, 30, 80]
    with crp.Batch(cfgs) as batch:
        assert len(batch.sims) == 4
        per = batch.run(steps, threads=4)
        assert per == [0, 0, 0, 0]
        got = [_state(s) for s in batch.sims]
        st = [s.stats().steps for s in batch.sims]
    assert st == steps
    for k, cfg in enumerate(cfgs):
        with crp.Sim(cfg) as one:
            one.step(steps[k])
            ref = _state(one)
        for a, b in zip(got[k], ref):
            assert np.array_equal(a, b), k


def test_batch_reports_per_simulation_status():
    """A simulation that hits its Picard cap fails alone; the others finish."""
    cfgs = _configs()[:2]
    cfgs[0].ext_picard_cap = 0  # any step with bubbles needs >= 1 Picard iteration
    with crp.Batch(cfgs) as batch:
        with pytest.raises(crp.CrpError) as e:
            batch.run([10, 10])
        assert e.value.status == 6  # CRP_ERR_PICARD
        assert batch.sims[1].stats().steps == 10


def test_handles_run_from_other_host_threads():
    """A simulation and a batch created on one host thread and advanced from
    others (whose current device the library sets from the handle) give the
    same results as on the creating thread."""
    import threading

    cfgs = _configs()[:2]
    with crp.Sim(cfgs[0]) as here:
        here.step(40)
        ref = _state(here)
    errors = []
    with crp.Sim(cfgs[0]) as sim, crp.Batch(cfgs) as batch:
        def work():
            try:
                sim.step(40)
                batch.run([40, 40], threads=2)
            except Exception as e:  # noqa: BLE001 - reported below
                errors.append(e)

        t = threading.Thread(target=work)
        t.start()
        t.join()
        assert not errors, errors
        for a, b in zip(_state(sim), ref):
            assert np.array_equal(a, b)
        for a, b in zip(_state(batch.sims[0]), ref):
            assert np.array_equal(a, b)
