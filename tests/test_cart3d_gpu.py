"""The 3-D Cartesian path (ext.grid_z > 0) on the GPU against the 3-D oracle,
through the C ABI: the bowl source without bubbles, with a bubble cloud at
its focus (reference radius scheme and rk45), the mixed precision form, a
seeded-phase bowl focused elsewhere, and determinism."""
import numpy as np
import pytest

import _bind as B
import crp
from test_cart3d import cart3d_small
from test_mixed_gpu import TOL_BUBBLE, TOL_FIELD, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-9
FLOOR = {"p0": 1e-3, "px": 1e-3, "py": 1e-3, "pz": 1e-3, "vx": 1e-9, "vy": 1e-9, "vz": 1e-9, "f_g": 1e-12,
         "f_gn": 1e-12, "f_gm": 1e-12, "rho_m": 1.0}
BUB = {"x": 1e-9, "y": 1e-9, "z": 1e-9, "R_t": 1e-9, "R_p": 1e-9, "d1_R_p": 1e-6, "PG_p": 1e-3, "PL_p": 1e-3,
       "PL_n": 1e-3, "Q_B": 1e-12, "v_x": 1e-9, "v_y": 1e-9, "v_z": 1e-9}


def rel_err(a, b, floor):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), floor))


def compare(gpu, cpu, skip=()):
    worst = {}
    for k, fl in FLOOR.items():
        a, b = gpu.field(k), cpu.field(k)
        assert a.shape == b.shape, (k, a.shape, b.shape)
        worst[k] = rel_err(a, b, fl)
    if cpu.dims3.num_bubbles:
        for k, fl in BUB.items():
            if k not in skip:
                worst["bub_" + k] = rel_err(gpu.bubbles(k), cpu.bubbles(k), fl)
        for k in ("ibn_x", "ibn_y", "ibn_z", "ibm_x", "ibm_y", "ibm_z"):
            assert np.array_equal(gpu.bubbles(k), cpu.bubbles(k)), k
    print({k: f"{v:.2e}" for k, v in worst.items()})
    bad = {k: v for k, v in worst.items() if not v <= TOL}
    assert not bad, bad


CASES = {
    "bowl": (dict(), 0, 80),
    "bowl_offaxis_seeded": (dict(ext_array_focus_dx=1e-3, ext_array_phases=1, ext_array_seed=9), 0, 60),
    # A 1 MPa burst collapses the cloud within 70 steps, and the reference
    # scheme's rounding differences then grow about 1e6-fold (9e-10 at step 70,
    # 1.2e-9 in PL at step 60, measured): the reference scheme is compared
    # under a 0.6 MPa burst, the rk45 scheme (1e-10 at step 70) under 1 MPa.
    "cloud_ref": (dict(tr_amp=0.6e6 / (998 * 1482)), 300, 70),
    "cloud_rk45": (dict(tr_amp=1.0e6 / (998 * 1482), ext_rp_scheme=1), 300, 70),
    "cloud_gaussian": (dict(ext_cloud_shape=2, ext_cloud_r=0.6e-3, N=36), 400, 60),
}


@pytest.mark.parametrize("name", list(CASES))
def test_3d_fp64_matches_oracle(name):
    over, nb, steps = CASES[name]
    over = dict(over)
    N = over.pop("N", 40)
    cfg = cart3d_small(N=N, bubbles=nb, **over)
    bub = crp.seed_bubbles3(cfg) if nb else None
    cpu = B.OracleSim3(cfg, bub)
    with crp.Sim(cfg, bub) as gpu:
        assert gpu.dims3.source_cells == cpu.dims3.source_cells
        compare(gpu, cpu)  # initial state
        for chunk in (steps // 2, steps - steps // 2):
            gpu.step(chunk)
            cpu.step(chunk)
        gs, cs = gpu.stats(), cpu.stats()
        print(name, "picard", gs.picard_total, cs.picard_total, "substeps", gs.rp_substeps_max, cs.rp_substeps_max)
        assert gs.steps == cs.steps == steps
        assert abs(gs.picard_total - cs.picard_total) <= max(2, cs.picard_total // 50)
        compare(gpu, cpu)
        assert np.abs(cpu.field("p0")).max() > 1e5  # the burst has reached the focus


def test_3d_mixed_matches_oracle():
    # A 0.05 MPa drive (0.5 MPa at the focus): the bowl's focal gain drives
    # the cloud to collapse at 0.2 MPa and above, and a collapsing cloud
    # amplifies the FP32 void-fraction storage error (6e-8) as it amplifies
    # FP64 rounding (1e5-fold over 70 steps, measured): 8e-4 at 0.2 MPa.
    cfg = cart3d_small(bubbles=300, tr_amp=0.05e6 / (998 * 1482))
    bub = crp.seed_bubbles3(cfg)
    cpu = B.OracleSim3(cfg, bub)
    cpu.step(70)
    cfg.ext_precision = 1
    with crp.Sim(cfg, bub) as gpu:
        gpu.step(70)
        errs = {k: rel_l2(gpu.field(k), cpu.field(k)) for k in ("p0", "vx", "vy", "vz", "f_g")}
        errs["R_t"] = rel_l2(gpu.bubbles("R_t"), cpu.bubbles("R_t"))
        print(errs)
        assert max(errs[k] for k in ("p0", "vx", "vy", "vz")) < TOL_FIELD, errs
        assert errs["f_g"] < TOL_BUBBLE and errs["R_t"] < TOL_BUBBLE, errs


def test_3d_is_deterministic():
    cfg = cart3d_small(bubbles=300, tr_amp=1.0e6 / (998 * 1482))
    bub = crp.seed_bubbles3(cfg)
    out = []
    for _ in range(2):
        with crp.Sim(cfg, bub) as gpu:
            gpu.step(50)
            out.append([gpu.field("p0"), gpu.field("f_g"), gpu.bubbles("R_t")])
    for a, b in zip(*out):
        assert np.array_equal(a, b)
