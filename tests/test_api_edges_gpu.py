"""Edge cases of the snapshot, tuning and batch entry points: invalid values
are refused with CRP_ERR_INVALID and change nothing; a radius-kernel width
above the occupancy limit is clamped; an empty bubble population runs; a
non-finite pressure is reported whether the steps run one per call or queued."""
import numpy as np
import pytest

import _bind as B
import crp

pytestmark = pytest.mark.gpu

INVALID = 1
NONFINITE = 7


def test_tuning_values():
    with crp.Sim(B.small_config()) as sim:
        t0 = sim.tuning
        assert t0.fdtd_rows == 8 and t0.rp_blocks == 0 and t0.rp_blocks_max >= 1
        for rows, blocks in ((7, 0), (8, -1), (0, 0)):
            t = crp.Tuning(rows, blocks, 0)
            with pytest.raises(crp.CrpError) as e:
                sim.tuning = t
            assert e.value.status == INVALID
        assert sim.tuning.fdtd_rows == 8
        sim.tuning = crp.Tuning(16, 10 ** 6, 0)  # clamped to the occupancy limit
        assert sim.tuning.fdtd_rows == 16 and sim.tuning.rp_blocks == 10 ** 6
        sim.step(20)
        assert sim.stats().steps == 20


def test_batch_tuning_values():
    with crp.Batch([B.small_config()]) as batch:
        for field, value in (("mode", 2), ("fdtd_rows", 5), ("rp_bubbles_per_lane", 0), ("blocking", 2),
                             ("threads", -1)):
            t = batch.tuning
            setattr(t, field, value)
            with pytest.raises(crp.CrpError) as e:
                batch.tuning = t
            assert e.value.status == INVALID
        assert batch.tuning.as_dict()["mode"] == "threads"
        lib = batch.lib
        assert lib.crp_batch_tune(batch.h, 0, None, None, 0, None) == INVALID


def test_state_arguments():
    lib = crp.load()
    with crp.Sim(B.small_config()) as sim:
        assert lib.crp_save_state(sim.h, None) == INVALID
        assert lib.crp_load_state(sim.h, None) == INVALID
        assert lib.crp_state_bytes(None) == 0
        assert lib.crp_state_bytes(sim.h) > 0
        lib.crp_state_free(None)


def test_empty_bubble_population():
    """Bubbles on, but the lattice's box holds no cell centre: no bubbles."""
    cfg = B.small_config(bub_enable=1, tr_box_size=1e-9)
    with crp.Sim(cfg) as sim:
        assert sim.dims.num_bubbles == 0
        sim.step(30)
        snap = sim.save_state()
        sim.step(10)
        p = sim.field("p0")
        sim.load_state(snap)
        sim.step(10)
        assert np.array_equal(p, sim.field("p0"))


@pytest.mark.parametrize("per_call", [1, 40])
def test_non_finite_pressure_is_reported(per_call):
    # Bubbles off, so no memory index depends on a field value.  After a first
    # finite step the element amplitudes overflow the source (1e308 x the
    # surface pressure): the source row becomes infinite, its neighbours
    # inf - inf = NaN.  Steps without bubbles run queued when more than one is
    # asked for, and their scalars are read once at the end.
    cfg = B.small_config(bub_enable=0, ext_elements=4)
    with crp.Sim(cfg) as sim:
        sim.step(1)
        sim.set_source_elements(np.full(4, 1e308), np.zeros(4))
        with pytest.raises(crp.CrpError) as e:
            for _ in range(120 // per_call):
                sim.step(per_call)
        assert e.value.status == NONFINITE
        assert not np.isfinite(sim.field("p0")).all()
