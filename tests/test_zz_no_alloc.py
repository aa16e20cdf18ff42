"""crp_void_fraction_noalloc (C ABI) against the void fraction a simulation forms.

The entry point takes device arrays and allocates nothing; its scratch is a
fixed static device array.  It must reproduce the initial void fraction of
crp_create, and a second call in a row (reusing the scratch the first left
behind) must give the same result.  This file is collected last so that the
entry point also runs after every other test in the same process.
"""
import ctypes

import numpy as np
import pytest

import _bind as B
import crp

pytestmark = pytest.mark.gpu

CRP_ERR_UNSUPPORTED = 2
CRP_ERR_TOO_LARGE = 11
SCRATCH_BYTES = 16 << 20
TOL = 1e-12


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _noalloc(cfg, x, y, r, nb, out):
    import torch

    lib = crp.load()
    n = int(x.numel())
    stream = torch.cuda.current_stream().cuda_stream
    return lib.crp_void_fraction_noalloc(ctypes.byref(cfg), n, x.data_ptr(), y.data_ptr(), r.data_ptr(),
                                         nb.data_ptr(), out.data_ptr(), ctypes.c_void_p(stream))


def _check_against_sim(cfg, bub):
    import torch

    with crp.Sim(cfg, bub) as sim:
        ref = sim.field("f_g")
        x, y, r, nb = (_dev(sim.bubbles(k)) for k in ("x", "y", "R0", "n_B"))
    outs = []
    for _ in range(2):  # two calls in a row on the same scratch
        out = torch.full(ref.shape, float("nan"), dtype=torch.float64, device="cuda")
        assert _noalloc(cfg, x, y, r, nb, out) == 0
        torch.cuda.synchronize()
        outs.append(out.cpu().numpy())
    scale = max(np.abs(ref).max(), 1e-300)
    for got in outs:
        assert np.all(np.isfinite(got))
        assert np.abs(got - ref).max() <= TOL * scale, np.abs(got - ref).max() / scale
    assert np.array_equal(outs[0], outs[1])
    return ref


def test_matches_simulation_cylindrical():
    cfg = B.small_config(ext_bubble_count=300, ext_bubble_seed=7, ext_r0_sigma_ln=0.3, ext_cloud_r=1.0e-3,
                         ext_cloud_h=2.0e-3, ext_n_b=4.0, bub_R0=3.0e-6)
    ref = _check_against_sim(cfg, crp.seed_bubbles(cfg))
    assert ref.max() > 0


def test_matches_simulation_planar_lattice():
    cfg = B.small_config(tr_cylindrical=0, tr_box_size=1.6e-3)
    ref = _check_against_sim(cfg, None)
    assert ref.max() > 0


def test_edge_bubbles_and_empty_population():
    """Bubbles in the first/last cells and on the ghost rows; then n = 0 (all zeros)."""
    import torch

    cfg = B.small_config(tr_cylindrical=0)
    d = cfg.grid_lx / cfg.grid_x
    xs = np.array([0.3 * d, 0.5 * d, cfg.grid_lx - 0.2 * d, 2.5 * d, cfg.grid_lx * 0.5, 1.1 * d])
    ys = np.array([0.4 * d, cfg.grid_ly - 0.3 * d, 0.5 * d, cfg.grid_ly * 0.5, cfg.grid_ly - 0.5 * d, 3.0 * d])
    bub = crp.Bubbles(xs, ys, np.full(6, 2e-6), np.full(6, 3.0))
    _check_against_sim(cfg, bub)
    out = torch.full(((cfg.grid_y + 2), (cfg.grid_x + 2)), float("nan"), dtype=torch.float64, device="cuda")
    e = torch.empty(0, dtype=torch.float64, device="cuda")
    assert _noalloc(cfg, e, e, e, e, out) == 0
    torch.cuda.synchronize()
    assert torch.count_nonzero(out).item() == 0


def test_rejects_oversize_and_unsupported():
    import torch

    lib = crp.load()
    assert lib.crp_void_fraction_noalloc_scratch(48, 96, 300) <= SCRATCH_BYTES
    assert lib.crp_void_fraction_noalloc_scratch(2048, 2048, 1) > SCRATCH_BYTES
    assert lib.crp_void_fraction_noalloc_scratch(64, 64, 1 << 20) > SCRATCH_BYTES
    small = _dev(np.full(4, 1e-3))
    out = torch.zeros(16, dtype=torch.float64, device="cuda")
    big_grid = B.small_config(grid_x=2048, grid_y=2048, grid_lx=0.2, grid_ly=0.2)
    assert _noalloc(big_grid, small, small, small, small, out) == CRP_ERR_TOO_LARGE
    band = B.small_config(sim_smooth_delta_band=3)
    assert _noalloc(band, small, small, small, small, out) == CRP_ERR_UNSUPPORTED
    torch.cuda.synchronize()
    assert torch.count_nonzero(out).item() == 0
