"""The TMA-staged FDTD tile kernel (fdtd_tile, selected by the environment
variable CRP_FDTD_TILE when a simulation is created) against the oracle on the
parity cases, FP64 and mixed: the same arithmetic as the strip kernel in
another organisation, kept for the roofline comparison."""
import os

import numpy as np
import pytest

import _bind as B
import crp
from test_parity_gpu import CASES, TOL_FP64, _compare

pytestmark = pytest.mark.gpu


@pytest.fixture
def tile_kernel():
    os.environ["CRP_FDTD_TILE"] = "1"
    yield
    del os.environ["CRP_FDTD_TILE"]


@pytest.mark.parametrize("name", ["focus_p", "plane_p_all_cells", "focus_v_wall_burst", "ext_source_row_ramp",
                                  "rigid_y1_mirror", "wide_planar"])
def test_tile_kernel_matches_oracle(name, tile_kernel):
    over, steps = CASES[name]
    cfg = B.small_config(**over)
    cpu = B.OracleSim(cfg)
    with crp.Sim(cfg) as gpu:
        gpu.step(steps)
        cpu.step(steps)
        _compare(gpu, cpu, TOL_FP64)


def test_tile_kernel_mixed_and_strip_agree(tile_kernel):
    over, steps = CASES["strong_drive"]
    out = []
    for tile in (True, False):
        if not tile:
            del os.environ["CRP_FDTD_TILE"]
        cfg = B.small_config(**over, ext_precision=1)
        with crp.Sim(cfg) as gpu:
            gpu.step(steps)
            out.append(gpu.field("p0"))
        os.environ["CRP_FDTD_TILE"] = "1"
    a, b = out
    assert float(np.abs(a - b).max() / np.abs(b).max()) < 1e-9
