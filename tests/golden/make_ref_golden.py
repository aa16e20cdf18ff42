"""Generate golden fixtures from the reference's own code (oracle/_ref/libcrp_ref.so,
built by oracle/build_ref.sh from the reference sources).

  python tests/golden/make_ref_golden.py host           # CPU: initialisers + bubble physics
  python tests/golden/make_ref_golden.py gpu OUTDIR     # GPU: whole runs of the reference kernels

`host` writes tests/golden/ref_host.npz: the reference's derived scalars, index
layout, PML profiles, lattice bubble seeding, and its Rayleigh-Plesset /
thermal-model functions evaluated on a seeded set of inputs.

`gpu` runs the reference's unmodified kernels (VelocityKernel, MixturePressureKernel,
BubbleRadiusKernel, ... driven in the order of solve_bubbles) on the cases in
RUN_CASES, each in its own process, and writes OUTDIR/ref_run_<case>.npz plus the
reference's own rawdata text files for the `tiny` case.  The cases keep PML on the
y1 face and X <= Y, where every reference kernel stays inside its arrays.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "tests"), os.path.join(ROOT, "cuda-rp_b200")]

import crp  # noqa: E402
import _bind as B  # noqa: E402

vp = ctypes.c_void_p


def _p(a):
    return a.ctypes.data_as(vp)


# Overrides of tests/golden/small.conf for each whole-run case.
RUN_CASES = {
    # axisymmetric, focused pressure source on the y=0 boundary, bubbles at the focus
    "focus_p": dict(steps=240),
    # planar, plane pressure source, bubbles in every cell
    "plane_p": dict(steps=120, grid_x=32, grid_y=64, grid_lx=3.2e-3, grid_ly=6.4e-3, tr_cylindrical=0,
                    tr_focused_p=0, tr_plane_p=1, tr_box_size=0.0, bub_fg0=2.0e-6, tr_amp=0.05),
    # axisymmetric, focused velocity source, rigid x1 wall, 1-on/1-off burst
    "focus_v_wall": dict(steps=200, pml_x1=0, tr_focused_p=0, tr_focused_v=1, tr_on_wave=1, tr_off_wave=1,
                         tr_amp=0.1),
    # PML on x0 too, plane velocity source, bubbles off
    "plane_v_nobub": dict(steps=150, pml_x0=1, tr_focused_p=0, tr_plane_v=1, bub_enable=0),
    # small grid for the rawdata text comparison.  38 columns give i1m = 40, where
    # the pitched widths of p (double2) and p0 (double) coincide; MixturePressureKernel
    # indexes p0 with p's index (inc/bubble_CUDA_kernel.cuh:862-864), which scrambles
    # p0 when they differ (with 512-byte pitch alignment, when i1m mod 64 is in [1, 32]).
    "tiny": dict(steps=60, grid_x=38, grid_y=38, grid_lx=3.8e-3, grid_ly=3.8e-3, pml_grid_number=6,
                 tr_focal_dist=3.0e-3, tr_box_size=1.0e-3, sim_save_interval=60),
}

FIELDS = ["p0", "p", "pn", "vx", "vy", "f_g", "f_gn", "f_gm", "rho_m", "T"]
BUBBLE_FIELDS = ["pos", "R_t", "R_p", "R_n", "d1_R_p", "PG_p", "PL_p", "PL_n", "dt", "re", "Q_B", "n_B", "ibm",
                 "ibn"]


def case_config(name: str) -> tuple[crp.Config, int]:
    over = dict(RUN_CASES[name])
    steps = over.pop("steps")
    return B.small_config(**over), steps


# ---------------------------------------------------------------------------
def make_host() -> dict:
    r = B.ref_lib()
    out = {}
    cases = {"small": B.small_config(),
             "planar_pml_all": B.small_config(pml_x0=1, pml_y0=1, tr_cylindrical=0, pml_order=3,
                                              pml_sigma=0.01, pml_grid_number=5),
             "sample_like": B.small_config(grid_x=300, grid_y=600, grid_lx=30e-3, grid_ly=60e-3,
                                           pml_grid_number=10, sim_cfl=0.1, tr_amp=1.5e-2,
                                           tr_focal_dist=40e-3, tr_box_size=30e-3, bub_fg0=1e-7,
                                           bub_R0=6.5e-7, bub_mu=891e-6, tr_pid=1, tr_pid_start_step=5000)}
    for name, cfg in cases.items():
        rp = B.ref_params(cfg)
        sc = np.zeros(21)
        r.crp_ref_host_scalars(ctypes.byref(rp), _p(sc))
        ai = np.zeros(28, np.int32)
        r.crp_ref_host_array_index(ctypes.byref(rp), _p(ai))
        X, Y = cfg.grid_x, cfg.grid_y
        arrs = [np.zeros(n) for n in (X + 2, Y + 2, X + 3, Y + 3, X + 3, X + 2)]
        r.crp_ref_host_sigma(ctypes.byref(rp), *[_p(a) for a in arrs])
        cap = X * Y
        rows = np.zeros((cap, 6))
        n = r.crp_ref_host_bubbles(ctypes.byref(rp), _p(rows), cap)
        out[f"{name}/scalars"] = sc
        out[f"{name}/array_index"] = ai
        for k, a in zip(["mx", "my", "nx", "ny", "xu", "rxp"], arrs):
            out[f"{name}/{k}"] = a
        out[f"{name}/bubbles"] = rows[:n:max(1, n // 500)]
        out[f"{name}/bubble_count"] = np.int64(n)
    # Bubble physics on seeded inputs around the states the simulations visit.
    rng = np.random.default_rng(0xC0DA)
    m = 400
    R0 = 10 ** rng.uniform(-6.5, -5.0, m)
    PL0 = np.full(m, 0.1e6)
    sig, mu, rho, K0, T0, gam = 7.2e-2, 1.0e-3, 1.0e3, 26.2e-3, 293.15, 1.4
    PG0 = PL0 + 2 * sig / R0
    dt0 = 10 ** rng.uniform(-10, -8.5, m)
    bp = np.stack([R0, PG0, PL0, np.full(m, T0), np.full(m, gam), np.full(m, sig), np.full(m, mu),
                   np.full(m, rho), np.full(m, K0), dt0], axis=1)
    R = R0 * rng.uniform(0.2, 3.0, m)
    PG = PG0 * rng.uniform(0.2, 20.0, m)
    PL = rng.uniform(-0.5e6, 2.0e6, m)
    d1R = rng.normal(0, 5.0, m) * (rng.uniform(size=m) < 0.8)
    dt = dt0 * rng.uniform(0.5, 1.0, m)
    remain = dt * rng.uniform(0.3, 12.0, m)
    rp_in = np.stack([R, R * rng.uniform(0.98, 1.02, m), R, d1R, dt, remain], axis=1)
    rp_out = rp_in.copy()
    omega = np.zeros(m)
    alpha = np.zeros((m, 2))
    for k in range(m):
        st = rp_out[k].copy()
        r.crp_ref_rp_step(_p(bp[k].copy()), _p(st), PG[k], PL[k])
        rp_out[k] = st
        a = np.zeros(2)
        omega[k] = r.crp_ref_omega_n(_p(bp[k].copy()), PG[k], R[k], _p(a))
        alpha[k] = a
    # Upsilon / Lp on both sides of the |alpha| = 0.1 branch.
    mag = np.concatenate([10 ** rng.uniform(-3, 2, m), rng.uniform(0.05, 0.15, 100)])
    ang = rng.uniform(0, 2 * np.pi, len(mag))
    a_re, a_im = mag * np.cos(ang), mag * np.sin(ang)
    ul = np.zeros((len(mag), 4))
    for k in range(len(mag)):
        o = np.zeros(4)
        r.crp_ref_upsilon_lp(a_re[k], a_im[k], gam, R[k % m], _p(o))
        ul[k] = o
    pg = np.zeros(m)
    lp = ul[:m, 2:4]
    for k in range(m):
        pg[k] = r.crp_ref_solve_pg(_p(bp[k].copy()), PG[k], rp_in[k, 1], R[k], omega[k] + 1.0, dt[k],
                                   lp[k, 0], lp[k, 1])
    out.update({"phys/bp": bp, "phys/PG": PG, "phys/PL": PL, "phys/R": R, "phys/rp_in": rp_in,
                "phys/rp_out": rp_out, "phys/omega": omega, "phys/alpha": alpha, "phys/a_re": a_re,
                "phys/a_im": a_im, "phys/ups_lp": ul, "phys/pg": pg})
    return out


# ---------------------------------------------------------------------------
def run_case(name: str, outdir: str) -> None:
    r = B.ref_lib()
    cfg, steps = case_config(name)
    rp = B.ref_params(cfg)
    dims = np.zeros(7, np.int32)
    st = r.crp_ref_setup(ctypes.byref(rp), _p(dims))
    assert st == 0, st
    i1m, j1m, i2m, j2m, i2n, j2n, nb = (int(v) for v in dims)
    picard = np.zeros(steps, np.int32)
    rc = r.crp_ref_run(steps, 1000, _p(picard))
    assert rc == 0, rc
    shapes = {"p0": (j1m, i1m), "p": (j1m, 2 * i1m), "pn": (j1m, 2 * i1m), "vx": (j2m, i2n), "vy": (j2n, i2m),
              "f_g": (j2m, i2m), "f_gn": (j2m, i2m), "f_gm": (j2m, i2m), "rho_m": (j1m, i1m), "T": (j2m, i2m)}
    out = {"steps": np.int64(steps), "picard": picard, "time": np.float64(r.crp_ref_time())}
    for fname in FIELDS:
        a = np.zeros(shapes[fname])
        assert r.crp_ref_read_field(fname.encode(), _p(a)) == 0
        out[fname] = a
    # p0 must equal px + py on interior cells; it does not when the p0 index quirk
    # above is active for this grid, and the fixture is then not a comparison target.
    p = out["p"]
    ok = np.array_equal(out["p0"][1:-1, 1:-1], (p[:, 0::2] + p[:, 1::2])[1:-1, 1:-1])
    out["p0_consistent"] = np.bool_(ok)
    if cfg.bub_enable:
        for bname in BUBBLE_FIELDS:
            a = np.zeros(2 * nb if bname in ("pos", "ibm", "ibn") else nb)
            assert r.crp_ref_read_bubbles(bname.encode(), _p(a)) == 0
            out["bub_" + bname] = a
    if name == "tiny":
        d = os.path.join(outdir, "ref_rawdata_tiny") + "/"
        os.makedirs(d, exist_ok=True)
        assert r.crp_ref_save_ascii(d.encode()) == 0
        d = os.path.join(outdir, "ref_sph_tiny") + "/"
        os.makedirs(d, exist_ok=True)
        assert r.crp_ref_save_sph(d.encode()) == 0
    r.crp_ref_teardown()
    np.savez_compressed(os.path.join(outdir, f"ref_run_{name}.npz"), **out)
    print(f"{name}: steps={steps} picard total={int(picard.sum())} max={int(picard.max())} bubbles={nb}")


def main(argv):
    if not B.ref_available():
        print("reference harness not built (oracle/build_ref.sh)")
        return 1
    if argv[1] == "host":
        np.savez_compressed(os.path.join(HERE, "ref_host.npz"), **make_host())
        print("wrote ref_host.npz")
        return 0
    if argv[1] == "gpu":
        outdir = argv[2]
        os.makedirs(outdir, exist_ok=True)
        rc = 0
        for name in RUN_CASES:
            p = subprocess.run([sys.executable, __file__, "case", name, outdir])
            rc |= p.returncode
        return rc
    if argv[1] == "case":
        run_case(argv[2], argv[3])
        return 0
    return 2


if __name__ == "__main__":
    sys.exit(main(sys.argv))
