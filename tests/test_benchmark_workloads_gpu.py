"""Parity on the benchmark's own workloads, not only on small grids.

The 256 x 512 workload (axisym_256x512: 256 x 512 axisymmetric grid, 4096 seeded
bubbles, 0.5 MPa focused burst) is run from t = 0 on the CUDA path in FP64 and
in the mixed form, and on the FP64 oracle, in lockstep, until each stops.  The
drive grows the bubble cloud until the mixture model stops converging; the
oracle does the same, so the CUDA path must stop at the same step.

Measured (one B200, 16 host cores for the oracle), relative to the oracle:
FP64 p0 ~1e-15 through the quiet phase, 8e-12 (R_t 2e-10) at the focal arrival
(step 1000, focal pressure 1.9 MPa), then growing about tenfold per ten steps
once the cloud is driven (R/R0 > 20): 5e-8 at step 1100, 1e-3 at 1200; both
stop with CRP_ERR_PICARD at step 1220.  The mixed form's focal-pressure error
is 5e-7 at the focal arrival and 4e-5 fifty steps later (the 1e-4 target), and
grows past it from step 1060; it stops at step 1172 (its Picard threshold is
1e-5, since FP32 storage of f_g leaves a residual floor near 7e-7).  FP64 runs
whose bubble radii or positions differ by one FP32 rounding diverge from the
FP64 run as fast as the mixed form does.

The 1024 x 2048 workload (axisym_1024x2048, 262144 bubbles) is compared over a bounded
window from t = 0, the oracle's time being about 0.1 s per step; so is the 3-D
workload cart3d_256 (256^3 Cartesian grid, 64-element hemispherical bowl, 65536
bubbles), every field and bubble variable, at about 2 s per oracle step.
"""
import os

import numpy as np
import pytest

import _bind as B
import crp

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CONF = os.path.join(ROOT, "cuda-rp_b200", "configs")
TOL = 1e-9
FOCAL_ARRIVAL = 1000  # mixture step at which the burst reaches the focus (40 mm / 1482 m/s / dt)


def rel_l2(a, b):
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / n) if n > 0 else float(np.linalg.norm(a))


def rel_max(a, b, floor):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), floor))


def focal_mask(dims, cfg, radius=2e-3):
    fy = cfg.tr_focal_dist * 0.5 * np.sqrt(3.0)
    ii, jj = np.meshgrid(np.arange(dims.i1m), np.arange(dims.j1m))
    return np.hypot((ii - 0.5) * dims.dx, (jj - 0.5) * dims.dy - fy) <= radius


@pytest.fixture(scope="module")
def run_256x512():
    """Lockstep run of the 256 x 512 workload: errors at checkpoints and the steps at
    which each path stopped."""
    path = os.path.join(CONF, "axisym_256x512.conf")
    cfg = crp.parse_file(path)
    bub = crp.seed_bubbles(cfg)
    ocfg = B.oracle_parse_file(path)
    oracle = B.OracleSim(ocfg, B.oracle_seed_bubbles(ocfg), threads=os.cpu_count() or 1)
    mcfg = crp.Config.from_buffer_copy(cfg)
    mcfg.ext_precision = 1
    sims = {"fp64": crp.Sim(cfg, bub), "mixed": crp.Sim(mcfg, bub), "oracle": oracle}
    mask = focal_mask(sims["fp64"].dims, cfg)
    stopped, status, records = {}, {}, {}
    checkpoints = [500, FOCAL_ARRIVAL, 1050, 1100]
    step = 0
    try:
        while len(stopped) < 3 and step < 1400:
            n = 100 if step < 900 else 10
            for name, s in sims.items():
                if name in stopped:
                    continue
                try:
                    s.step(n)
                except crp.CrpError as e:
                    stopped[name] = int(s.stats().steps) + 1
                    status[name] = e.status
            step += n
            if step in checkpoints and "oracle" not in stopped:
                po, vo, ro = oracle.field("p0"), oracle.field("vx"), oracle.bubbles("R_t")
                rec = {"picard_oracle": int(oracle.stats().picard_total)}
                for name in ("fp64", "mixed"):
                    if name in stopped:
                        continue
                    s = sims[name]
                    p = s.field("p0")
                    rec[name] = {"p0": rel_max(p, po, 1e-3), "vx": rel_max(s.field("vx"), vo, 1e-9),
                                 "R_t": rel_max(s.bubbles("R_t"), ro, 1e-9), "focal_l2": rel_l2(p[mask], po[mask]),
                                 "picard": int(s.stats().picard_total)}
                records[step] = rec
    finally:
        for name in ("fp64", "mixed"):
            sims[name].close()
        oracle.close()
    print("256x512 checkpoints", records, "stopped", stopped)
    return {"records": records, "stopped": stopped, "status": status}


def test_256x512_fp64_matches_oracle_through_focal_arrival(run_256x512):
    for step in (500, FOCAL_ARRIVAL):
        r = run_256x512["records"][step]["fp64"]
        assert r["p0"] < TOL and r["vx"] < TOL and r["R_t"] < TOL, (step, r)
        assert r["picard"] == run_256x512["records"][step]["picard_oracle"]


def test_256x512_driven_phase_stays_close_until_the_cloud_amplifies(run_256x512):
    # 100 steps after the arrival the driven cloud has amplified rounding
    # differences by about 1e3 (measured 5e-8); still far below the physics.
    r = run_256x512["records"][1100]["fp64"]
    assert r["p0"] < 1e-5 and r["R_t"] < 1e-5, r
    assert abs(r["picard"] - run_256x512["records"][1100]["picard_oracle"]) <= 2


def test_256x512_cuda_and_oracle_stop_at_the_same_step(run_256x512):
    st, code = run_256x512["stopped"], run_256x512["status"]
    assert "fp64" in st and "oracle" in st, st
    assert code["fp64"] == 6 and code["oracle"] == 6  # CRP_ERR_PICARD
    assert st["fp64"] == st["oracle"], st


def test_256x512_mixed_focal_error_at_arrival(run_256x512):
    for step in (FOCAL_ARRIVAL, 1050):
        r = run_256x512["records"][step]["mixed"]
        assert r["focal_l2"] < 1e-4, (step, r)


def test_256x512_mixed_error_is_amplified_fp32_sized_differences():
    # After the focal arrival the driven cloud amplifies any difference about
    # tenfold per ten steps.  FP64 runs whose bubble radii or positions differ
    # from the workload's by one FP32 rounding (a factor 1 + 2^-24) leave the
    # unperturbed FP64 run as fast as the mixed form does (measured focal
    # rel. L2 against the FP64 run: mixed 3.5e-5 / 2.8e-3 / 1.3e-2 at steps
    # 1050 / 1075 / 1100; radii x (1 + 2^-24) 4.4e-5 / 9.6e-4 / 3.2e-3;
    # positions 2.2e-5 / 2.5e-3 / 5.5e-3), and a 2^-40 difference grows the
    # same way from a 1e5-fold smaller start (1.3e-7 at step 1100).  The
    # mixed form's error past the 1e-4 target is therefore what FP32-sized
    # differences become in this flow, not a fault of the mixed arithmetic.
    path = os.path.join(CONF, "axisym_256x512.conf")
    cfg = crp.parse_file(path)
    bub = crp.seed_bubbles(cfg)
    mcfg = crp.Config.from_buffer_copy(cfg)
    mcfg.ext_precision = 1

    def perturbed(fx=1.0, fr=1.0):
        return crp.Bubbles(bub.x * fx, bub.y.copy(), bub.r0 * fr, bub.n_b.copy(), None)

    sims = {"fp64": crp.Sim(cfg, bub), "mixed": crp.Sim(mcfg, bub),
            "r0_2^-24": crp.Sim(cfg, perturbed(fr=1.0 + 2.0 ** -24)),
            "x_2^-24": crp.Sim(cfg, perturbed(fx=1.0 + 2.0 ** -24)),
            "r0_2^-40": crp.Sim(cfg, perturbed(fr=1.0 + 2.0 ** -40))}
    try:
        mask = focal_mask(sims["fp64"].dims, cfg)
        for step in (1050, 1075, 1100):
            for sim in sims.values():
                sim.step(step - int(sim.stats().steps))
            base = sims["fp64"].field("p0")[mask]
            err = {k: rel_l2(s.field("p0")[mask], base) for k, s in sims.items() if k != "fp64"}
            print("256x512 focal rel. L2 against the FP64 run at step", step, err)
            fp32_sized = max(err["r0_2^-24"], err["x_2^-24"])
            assert err["mixed"] / 10 <= fp32_sized <= 10 * err["mixed"], (step, err)
            assert err["r0_2^-40"] < 1e-3 * fp32_sized, (step, err)
        assert fp32_sized > 1e-4  # such differences alone pass the mixed target
    finally:
        for sim in sims.values():
            sim.close()


def test_1024x2048_fp64_window_matches_oracle():
    path = os.path.join(CONF, "axisym_1024x2048.conf")
    cfg = crp.parse_file(path)
    ocfg = B.oracle_parse_file(path)
    oracle = B.OracleSim(ocfg, B.oracle_seed_bubbles(ocfg), threads=os.cpu_count() or 1)
    try:
        with crp.Sim(cfg, crp.seed_bubbles(cfg)) as gpu:
            # The first steps' pressure is a ramped source of millipascals; the
            # comparison starts once it has grown (floor 1 Pa for p0).
            for n in (60, 60):
                gpu.step(n)
                oracle.step(n)
                errs = {"p0": rel_max(gpu.field("p0"), oracle.field("p0"), 1.0),
                        "vx": rel_max(gpu.field("vx"), oracle.field("vx"), 1e-9),
                        "vy": rel_max(gpu.field("vy"), oracle.field("vy"), 1e-9),
                        "f_g": rel_max(gpu.field("f_g"), oracle.field("f_g"), 1e-12),
                        "R_t": rel_max(gpu.bubbles("R_t"), oracle.bubbles("R_t"), 1e-9)}
                print("1024x2048 step", gpu.stats().steps, errs)
                assert all(v < TOL for v in errs.values()), errs
                assert gpu.stats().picard_total == oracle.stats().picard_total
    finally:
        oracle.close()


def test_cart3d_256_fp64_window_matches_oracle():
    # In this window the burst has not reached the cloud (about 250 steps from
    # the bowl), so the pressure the bubbles gather is the grid's far field,
    # some 1e8 below the pressure near the bowl.  The grid fields agree to
    # rounding of their own maxima (1e-14, measured); the gathered bubble
    # quantities are compared against the same scale: the field's maximum
    # pressure and velocity, and the radius rate and heat flow a pressure of
    # that size would drive (measured: 1e-7 to 3e-5 of their own tiny maxima,
    # i.e. 1e-14 of the field scale).
    from test_cart3d_gpu import FLOOR, rel_err

    path = os.path.join(CONF, "cart3d_256.conf")
    cfg = crp.parse_file(path)
    ocfg = B.oracle_parse_file(path)
    oracle = B.OracleSim3(ocfg, B.oracle_seed_bubbles3(ocfg), threads=os.cpu_count() or 1)
    try:
        with crp.Sim(cfg, crp.seed_bubbles3(cfg)) as gpu:
            assert gpu.dims3.num_bubbles == oracle.dims3.num_bubbles == 65536
            for n in (10, 10):
                gpu.step(n)
                oracle.step(n)
                worst = {k: rel_err(gpu.field(k), oracle.field(k), fl) for k, fl in FLOOR.items()}
                pmax = float(np.abs(oracle.field("p0")).max())
                vmax = max(float(np.abs(oracle.field(k)).max()) for k in ("vx", "vy", "vz"))
                scale = {"x": 1e-9, "y": 1e-9, "z": 1e-9, "R_t": 1e-9, "R_p": 1e-9, "PG_p": 1e-3,
                         "PL_p": pmax, "PL_n": pmax, "v_x": vmax, "v_y": vmax, "v_z": vmax,
                         "d1_R_p": pmax / (cfg.ext_rho_inf * cfg.ext_c_inf),
                         "Q_B": 4.0 * np.pi * cfg.bub_R0 * cfg.bub_K0 * cfg.bub_T0 * pmax / cfg.bub_P0}
                for k, fl in scale.items():
                    worst["bub_" + k] = rel_err(gpu.bubbles(k), oracle.bubbles(k), fl)
                for k in ("ibn_x", "ibn_y", "ibn_z", "ibm_x", "ibm_y", "ibm_z"):
                    assert np.array_equal(gpu.bubbles(k), oracle.bubbles(k)), k
                print("cart3d_256 step", gpu.stats().steps, {k: f"{v:.2e}" for k, v in worst.items()})
                bad = {k: v for k, v in worst.items() if not v <= TOL}
                assert not bad, bad
                assert gpu.stats().picard_total == oracle.stats().picard_total
    finally:
        oracle.close()
