"""The rk45 radius scheme (ext.rp_scheme = rk45) on the CUDA path against the
oracle's restatement of the same scheme, through the C ABI.

FP64: every field and bubble quantity within the FP64 parity tolerance
(test_parity_gpu.TOL_FP64), the step counts equal.  Mixed precision (thermal
model in FP32 outside the stiff phase R < 0.3 R0 or |R'| > 0.1 c_inf): within
the mixed path's tolerances against the FP64 oracle (test_mixed_gpu)."""
import numpy as np
import pytest

import _bind as B
import crp
from test_mixed_gpu import TOL_BUBBLE, TOL_FIELD, rel_l2
from test_parity_gpu import CASES, TOL_FP64, _compare

pytestmark = pytest.mark.gpu

RK_CASES = ["focus_p", "plane_p_all_cells", "strong_drive", "ext_source_row_ramp", "focus_v_wall_burst"]


@pytest.mark.parametrize("name", RK_CASES)
def test_rk45_fp64_matches_oracle(name):
    over, steps = CASES[name]
    cfg = B.small_config(ext_rp_scheme=1, **over)
    cpu = B.OracleSim(cfg)
    with crp.Sim(cfg) as gpu:
        for chunk in (steps // 2, steps - steps // 2):
            gpu.step(chunk)
            cpu.step(chunk)
        gs, cs = gpu.stats(), cpu.stats()
        print(name, "picard", gs.picard_total, cs.picard_total, "steps max", gs.rp_substeps_max, cs.rp_substeps_max)
        assert abs(gs.picard_total - cs.picard_total) <= max(2, cs.picard_total // 50)
        # The next trial step size comes from the error estimate, a difference of
        # stage combinations that cancels to ~1e-7 of the stages: its rounding
        # moves the proposed step by up to a few 1e-4 (measured 2e-4) while the
        # state it produces agrees to 1e-10.  It is a controller quantity,
        # compared more loosely than the state.
        _compare(gpu, cpu, TOL_FP64, loose={"bub_dt": 1e-2})
        if gpu.dims.num_bubbles:
            assert np.all(gpu.bubbles("re") == 0.0)
            assert abs(gs.rp_substeps_max - cs.rp_substeps_max) <= max(2, cs.rp_substeps_max // 20)


@pytest.mark.parametrize("name", ["focus_p", "strong_drive"])
def test_rk45_mixed_matches_oracle(name):
    over, steps = CASES[name]
    cfg = B.small_config(ext_rp_scheme=1, **over)
    cpu = B.OracleSim(cfg)
    cpu.step(steps)
    cfg.ext_precision = 1
    with crp.Sim(cfg) as gpu:
        gpu.step(steps)
        errs = {k: rel_l2(gpu.field(k), cpu.field(k)) for k in ("p0", "vx", "vy", "f_g")}
        errs["R_t"] = rel_l2(gpu.bubbles("R_t"), cpu.bubbles("R_t"))
        errs["PG_p"] = rel_l2(gpu.bubbles("PG_p"), cpu.bubbles("PG_p"))
        print(name, {k: f"{v:.2e}" for k, v in errs.items()})
        assert errs["p0"] < TOL_FIELD and errs["vx"] < TOL_FIELD and errs["vy"] < TOL_FIELD, errs
        assert errs["f_g"] < TOL_BUBBLE and errs["R_t"] < TOL_BUBBLE and errs["PG_p"] < TOL_BUBBLE, errs


def test_rk45_tolerance_sets_accuracy():
    """Tighter rtol moves the result towards the tightest (a converged solution)."""
    over, steps = CASES["strong_drive"]
    runs = {}
    for tol in (1e-4, 1e-6, 1e-9):
        cfg = B.small_config(ext_rp_scheme=1, ext_rp_tol=tol, **over)
        with crp.Sim(cfg) as gpu:
            gpu.step(steps)
            runs[tol] = gpu.bubbles("R_t")
    e4 = rel_l2(runs[1e-4], runs[1e-9])
    e6 = rel_l2(runs[1e-6], runs[1e-9])
    print("rk45 R_t vs rtol 1e-9:", e4, e6)
    assert e6 < e4 and e6 < 1e-4
