"""Mixed-precision path (ext.precision = mixed) against the FP64 oracle.

The mixed path stores velocity and pressure as FP32 values with an FP32
compensation term (about 48 significant bits), stores the void-fraction
history in FP32 (sums in FP64), and evaluates the bubble thermal model
(omega_N, alpha_N, Lp_N) in FP32; the Rayleigh-Plesset radius update, its
step-size control and the gas-pressure update stay FP64.

Tolerances (relative L2 over the field, against the FP64 oracle after N steps):
pressure and velocity 1e-4 (the accuracy target for the focal pressure), void
fraction and bubble radii 1e-3.
"""
import numpy as np
import pytest

import _bind as B
import crp
from test_parity_gpu import CASES

pytestmark = pytest.mark.gpu

TOL_FIELD = 1e-4
TOL_BUBBLE = 1e-3


def rel_l2(a, b):
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / n) if n > 0 else float(np.linalg.norm(a))


@pytest.mark.parametrize("name", ["focus_p", "plane_p_all_cells", "strong_drive", "ext_source_row_ramp"])
def test_mixed_matches_oracle(name):
    over, steps = CASES[name]
    cfg = B.small_config(**over)
    cpu = B.OracleSim(cfg)
    cpu.step(steps)
    cfg.ext_precision = 1
    with crp.Sim(cfg) as gpu:
        gpu.step(steps)
        errs = {k: rel_l2(gpu.field(k), cpu.field(k)) for k in ("p0", "vx", "vy", "f_g")}
        if gpu.dims.num_bubbles:
            errs["R_t"] = rel_l2(gpu.bubbles("R_t"), cpu.bubbles("R_t"))
            errs["PG_p"] = rel_l2(gpu.bubbles("PG_p"), cpu.bubbles("PG_p"))
        print(name, {k: f"{v:.2e}" for k, v in errs.items()}, "picard", gpu.stats().picard_total,
              cpu.stats().picard_total)
        assert errs["p0"] < TOL_FIELD and errs["vx"] < TOL_FIELD and errs["vy"] < TOL_FIELD, errs
        assert errs["f_g"] < TOL_BUBBLE, errs
        if "R_t" in errs:
            assert errs["R_t"] < TOL_BUBBLE and errs["PG_p"] < TOL_BUBBLE, errs


def test_mixed_is_deterministic():
    over, steps = CASES["plane_p_all_cells"]
    cfg = B.small_config(ext_precision=1, **over)
    out = []
    for _ in range(2):
        with crp.Sim(cfg) as gpu:
            gpu.step(steps)
            out.append([gpu.field("p0"), gpu.field("f_g"), gpu.bubbles("R_t")])
    for a, b in zip(*out):
        assert np.array_equal(a, b)
