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


def _batch_state(batch):
    return [(_state(s), s.stats().steps, s.stats().picard_total) for s in batch.sims]


def _equal(u, v):
    for (fa, sa, pa), (fb, sb, pb) in zip(u, v):
        assert (sa, pa) == (sb, pb)
        for a, b in zip(fa, fb):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("setting", [dict(mode=crp.BATCH_GRAPHS), dict(fdtd_rows=4), dict(fdtd_rows=16),
                                     dict(rp_bubbles_per_lane=16), dict(blocking=1, threads=8),
                                     dict(mode=crp.BATCH_GRAPHS, fdtd_rows=16, rp_bubbles_per_lane=4)])
def test_batch_settings_give_the_same_results(setting):
    """Graph-queued steps (device-side Picard control, one host thread) and
    other launch shapes give the thread-pool run's results bit for bit,
    including a simulation without bubbles (host steps beside the graphs)."""
    cfgs = _configs()
    steps = [60, 45, 30, 80]
    runs = []
    for s in (None, setting):
        with crp.Batch(cfgs) as batch:
            if s is not None:
                t = batch.tuning
                for k, v in s.items():
                    setattr(t, k, v)
                batch.tuning = t
            batch.run(steps[:2] + [10, 10])
            batch.run([a - b for a, b in zip(steps, steps[:2] + [10, 10])])
            runs.append(_batch_state(batch))
    _equal(*runs)


def test_batch_tune_restores_and_applies():
    """crp_batch_tune times its candidate settings on the batch itself and
    leaves every simulation where it was; the tuned run equals an untuned one."""
    cfgs = _configs()
    with crp.Batch(cfgs) as ref:
        ref.run([20] * 4)
        ref.run([30] * 4)
        want = _batch_state(ref)
    with crp.Batch(cfgs) as batch:
        batch.run([20] * 4)
        before = _batch_state(batch)
        best, tried = batch.tune(trial_steps=5)
        print(best.as_dict(), [t.as_dict() for t in tried])
        assert len(tried) == 8  # default, graphs, 16 threads, blocking waits, rows 4 and 16, lanes 4 and 16
        assert all(t.ms_per_step > 0 for t in tried)
        assert best.ms_per_step == min(t.ms_per_step for t in tried)
        _equal(_batch_state(batch), before)
        assert batch.tuning.as_dict() == best.as_dict()
        batch.run([30] * 4)
        _equal(_batch_state(batch), want)


def test_batch_with_a_3d_simulation():
    """A 3-D simulation in a batch runs its host-driven steps beside the 2-D
    simulations' graph-queued ones, with the same results as in thread mode."""
    from test_cart3d import cart3d_small

    c3 = cart3d_small(bubbles=100, tr_amp=0.3e6 / (998 * 1482))
    cfgs = [_configs()[0], c3]
    bubs = [None, crp.seed_bubbles3(c3)]
    runs = []
    for mode in (crp.BATCH_THREADS, crp.BATCH_GRAPHS):
        with crp.Batch(cfgs, bubs) as batch:
            t = batch.tuning
            t.mode = mode
            batch.tuning = t
            batch.run([40, 40])
            runs.append([batch.sims[0].field("p0"), batch.sims[1].field("p0"), batch.sims[1].bubbles("R_t"),
                         batch.sims[1].stats().steps])
    for a, b in zip(*runs):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    assert runs[0][3] == 40
