"""The paths on which picard_gate keeps the queued first radius solve closed,
against the oracle: steps whose prediction already meets the Picard tolerance
(the loop does not run), and bubbles that cross into another cell (the bins are
rebuilt before the loop runs)."""
import numpy as np
import pytest

import _bind as B
import crp
from test_parity_gpu import CASES, TOL_FP64, _compare

pytestmark = pytest.mark.gpu


def test_loop_skipped_matches_oracle():
    over, steps = CASES["focus_p"]
    cfg = B.small_config(ext_picard_tol=1.0e30, **over)
    cpu = B.OracleSim(cfg)
    with crp.Sim(cfg) as gpu:
        gpu.step(steps)
        cpu.step(steps)
        assert gpu.stats().picard_total == cpu.stats().picard_total == 0
        _compare(gpu, cpu, TOL_FP64)


def boundary_bubbles(cfg):
    """Bubbles 1e-13 m on either side of the cell boundaries y = (k - 1/2) dy
    (where the cell index floor(y / dy + 1/2) changes) of rows 20 and 28, so that
    the wave's first velocities move some of them into the next cell."""
    dx, dy = cfg.grid_lx / cfg.grid_x, cfg.grid_ly / cfg.grid_y
    xs, ys = [], []
    for k in (20, 28):
        for side in (-1.0, 1.0):
            for ix in range(4, 20):
                xs.append((ix + 0.25) * dx)
                ys.append((k - 0.5) * dy + side * 1.0e-13)
    n = len(xs)
    return crp.Bubbles(np.array(xs), np.array(ys), np.full(n, 3.0e-6), np.full(n, 50.0))


def test_bubbles_crossing_cells_match_oracle():
    over, steps = CASES["strong_drive"]
    cfg = B.small_config(**over)
    bub = boundary_bubbles(cfg)
    cpu = B.OracleSim(cfg, bub)
    with crp.Sim(cfg, bub) as gpu:
        iny0 = gpu.bubbles("ibn_y").copy()
        gpu.step(steps)
        cpu.step(steps)
        crossed = int((gpu.bubbles("ibn_y") != iny0).sum())
        print("bubbles that changed cell:", crossed, "picard", gpu.stats().picard_total, cpu.stats().picard_total)
        assert crossed > 0
        _compare(gpu, cpu, TOL_FP64)
