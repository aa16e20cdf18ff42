"""Whole runs against the reference's own kernels.

tests/golden/ref_run_<case>.npz hold the state after N steps of the
reference's unmodified CUDA kernels, driven in the order of solve_bubbles
(tests/golden/make_ref_golden.py gpu, run on a B200).  The oracle (CPU) and the
CUDA path (GPU) both replay each case from the same configuration and are
compared field by field.

Tolerance: the reference sums the void fraction with unordered CAS atomics and
its build contracts multiply-adds, so its last bits vary run to run; the
comparison allows REL_TOL of each field's maximum.
"""
import os

import numpy as np
import pytest

import _bind as B
import crp

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")

# Same cases as make_ref_golden.RUN_CASES (kept in one place there).
import importlib.util  # noqa: E402

_spec = importlib.util.spec_from_file_location("make_ref_golden", os.path.join(GOLD, "make_ref_golden.py"))
_mrg = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_mrg)
CASES = [c for c in _mrg.RUN_CASES if os.path.exists(os.path.join(GOLD, f"ref_run_{c}.npz"))]


def test_fixtures_are_p0_consistent():
    """Every committed fixture comes from a grid where the reference's p0 indexing
    quirk (inc/bubble_CUDA_kernel.cuh:862-864) is inactive: p0 = px + py inside."""
    for c in CASES:
        g = np.load(os.path.join(GOLD, f"ref_run_{c}.npz"))
        p = g["p"]
        assert np.array_equal(g["p0"][1:-1, 1:-1], (p[:, 0::2] + p[:, 1::2])[1:-1, 1:-1]), c

REL_TOL = 1e-9
# Rates and their integrals (radial velocity, bubble heat) are differences of
# nearly equal radii over sub-steps; they carry ~100x the relative rounding.
REL_TOL_RATES = {"bub_d1_R_p": 1e-7, "bub_Q_B": 1e-7}


def ref_fields(g):
    out = {"p0": g["p0"], "px": g["p"][:, 0::2], "py": g["p"][:, 1::2], "pnx": g["pn"][:, 0::2],
           "pny": g["pn"][:, 1::2], "vx": g["vx"], "vy": g["vy"], "f_g": g["f_g"], "f_gn": g["f_gn"],
           "f_gm": g["f_gm"], "rho_m": g["rho_m"]}
    if "T" in g:
        out["T"] = g["T"]
    return out


def ref_bubbles(g):
    if "bub_R_t" not in g:
        return {}
    return {"x": g["bub_pos"][0::2], "y": g["bub_pos"][1::2], "R_t": g["bub_R_t"], "R_p": g["bub_R_p"],
            "R_n": g["bub_R_n"], "d1_R_p": g["bub_d1_R_p"], "PG_p": g["bub_PG_p"], "PL_p": g["bub_PL_p"],
            "PL_n": g["bub_PL_n"], "dt": g["bub_dt"], "Q_B": g["bub_Q_B"], "n_B": g["bub_n_B"],
            "ibn_x": g["bub_ibn"][0::2], "ibn_y": g["bub_ibn"][1::2], "ibm_x": g["bub_ibm"][0::2],
            "ibm_y": g["bub_ibm"][1::2]}


from test_parity_gpu import FLOOR, rel_err  # noqa: E402


def compare(sim, g, tol):
    errs = {}
    for k, ref in ref_fields(g).items():
        a = sim.field(k)
        assert a.shape == ref.shape, (k, a.shape, ref.shape)
        errs[k] = rel_err(a, ref, FLOOR[k])
    for k, ref in ref_bubbles(g).items():
        a = sim.bubbles(k)
        if k.startswith("ib"):
            assert np.array_equal(a, ref), k
            continue
        errs["bub_" + k] = rel_err(a, ref, FLOOR.get("bub_" + k, 1e-12))
    print({k: f"{v:.1e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if not v <= max(tol, REL_TOL_RATES.get(k, 0.0))}
    assert not bad, bad


@pytest.mark.skipif(not CASES, reason="no reference run fixtures")
@pytest.mark.parametrize("case", CASES)
def test_oracle_replays_reference_run(case):
    g = np.load(os.path.join(GOLD, f"ref_run_{case}.npz"))
    cfg, steps = _mrg.case_config(case)
    assert steps == int(g["steps"])
    o = B.OracleSim(cfg)
    picard = []
    for _ in range(steps):
        o.step(1)
        picard.append(o.stats().picard_last)
    assert abs(o.stats().time - float(g["time"])) <= 1e-15 * float(g["time"])
    # Picard iteration counts per step follow the reference's (the convergence
    # test sits on a threshold, so allow a rare one-iteration difference).
    d = np.abs(np.array(picard) - g["picard"])
    assert d.max() <= 1 and d.sum() <= max(2, steps // 50), (d.sum(), d.max())
    compare(o, g, REL_TOL)


@pytest.mark.gpu
@pytest.mark.skipif(not CASES, reason="no reference run fixtures")
@pytest.mark.parametrize("case", CASES)
def test_cuda_path_replays_reference_run(case):
    g = np.load(os.path.join(GOLD, f"ref_run_{case}.npz"))
    cfg, steps = _mrg.case_config(case)
    with crp.Sim(cfg) as sim:
        sim.step(steps)
        s = sim.stats()
        assert abs(s.picard_total - int(g["picard"].sum())) <= max(2, steps // 50)
        compare(sim, g, REL_TOL)
