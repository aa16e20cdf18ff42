"""Benchmark of the CUDA-RP simulation path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload axisym_1024x2048|axisym_256x512|sweep_64] [--chunk S]

One bench step is S mixture time steps of the full hot path: fused FDTD/PML
update, bubble motion and binning, and every Picard iteration of
Rayleigh-Plesset + void-fraction gather + pressure re-evaluation the step
needs.  The run starts at t = 0; W untimed bench steps, then K timed ones.

The timed window stays inside the quiet phase of the workload whatever W and K
are (`window`): S = min(100, QUIET_END // (W + K + 1)), so mixture steps
[W S, (W + K) S) plus one profiling chunk end before the burst drives the
bubble cloud (QUIET_END: mixture step 1700 of the 1024 x 2048 workload, 900 of
256 x 512).  Both benchmark drives later grow the cloud until the mixture model
stops converging (the Picard loop at step 2187 of 1024 x 2048, 1219 of
256 x 512; the FP64 oracle does the same), so a window that reached there would
time a failing run.  The "driven" object then continues the same run untimed to
DRIVEN_START and times chunks of 10 mixture steps one by one (bounded by
--driven-seconds), recording where the run stops if a step fails.  The state
(about 200 MB at 1024 x 2048) is larger than L2, so no flush is needed between
steps.

metric: Mcell-upd/s of the plain FP64 path (the reference's precision) -
interior cells x mixture steps / device time (CUDA events on the simulation's
stream, max over ranks).  Also reported: bubble-steps/s; the mixed-precision
path's rate with its relative L2 against the FP64 path and the oracle; the
roofline of the fused FDTD kernel; a bounded CPU-oracle baseline and the error
of the GPU state against the FP64 oracle on that sample; an end-to-end number
through the C ABI with host buffers; clocks sampled during the timed region.

Multi-GPU (--gpus N under torchrun): independent replicas, one per GPU, no
data-path collective ("replicas only": the simulation does not shard across
GPUs here); value = all ranks' cell updates / max rank time.

--impl reference: the reference simulator has no CPU implementation (its
simulation is CUDA-only), so the reference arm times the FP64 host oracle -
the restatement of the reference's kernels - on all host cores, over the same
window start as this arm: untimed to mixture step W S, then K timed bench steps
of one mixture step each (a bounded sample of the window).  Its inputs come
from the oracle's own parser and seeding; it loads no product library.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "cuda-rp_b200")
sys.path[:0] = [PKG, os.path.join(ROOT, "tests")]

import numpy as np  # noqa: E402

# Mixture step at which the burst begins to drive the bubble cloud (the
# largest bubble radius leaves R0 by more than 1 %), measured with the FP64
# path; the Picard loop of both workloads stops converging about 500 and 300
# steps later (steps 2187 and 1219).
DRIVEN_START = {"axisym_1024x2048": 1700, "axisym_256x512": 900, "sweep_64": 500,
                # 3-D: the burst from the bowl reaches the cloud's inner bubbles
                "cart3d_384": 150, "cart3d_256": 200}
# Timed windows end here (see the module docstring).
QUIET_END = dict(DRIVEN_START)
MAX_CHUNK = {"axisym_1024x2048": 100, "axisym_256x512": 100, "sweep_64": 25, "cart3d_384": 25, "cart3d_256": 25}
WORKLOADS = {
    "axisym_1024x2048": os.path.join(PKG, "configs", "axisym_1024x2048.conf"),
    "axisym_256x512": os.path.join(PKG, "configs", "axisym_256x512.conf"),
    "cart3d_384": os.path.join(PKG, "configs", "cart3d_384.conf"),
    "cart3d_256": os.path.join(PKG, "configs", "cart3d_256.conf"),
}
# Compulsory HBM traffic of the fused FDTD pass per cell: FP64
# reads px, py, vx, vy, f_g, f_gn, f_gm and writes px, py, vx, vy, predicted f_g;
# mixed stores each velocity/pressure value as two FP32 words and f_g as FP32.
BYTES_PER_CELL = {"fp64": 96, "mixed": 80}
# 3-D: vz and pz besides, each read and written.
BYTES_PER_CELL_3D = {"fp64": 128, "mixed": 112}


def is3d(cfg):
    return cfg.ext_grid_z > 0


def cell_count(cfg):
    return cfg.grid_x * cfg.grid_y * (cfg.ext_grid_z if is3d(cfg) else 1)
DTYPE = {"fp64": "f64", "mixed": "f32 fields + f32 compensation (f64 arithmetic), f32 void fraction, "
                                  "f32 thermal model while |R/R0-1| <= 1e-3, f64 RP"}


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="axisym_1024x2048", choices=list(WORKLOADS) + ["sweep_64"])
    ap.add_argument("--chunk", type=int, default=None,
                    help="mixture steps per bench step (default: the largest that keeps the window quiet, "
                         "at most 100; 25 for sweep_64)")
    ap.add_argument("--driven-start", type=int, default=None)
    ap.add_argument("--driven-chunks", type=int, default=10)
    ap.add_argument("--driven-chunk", type=int, default=10)
    ap.add_argument("--driven-seconds", type=float, default=60.0)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"])
    ap.add_argument("--primary", default="fp64", choices=["fp64", "mixed"])
    args = ap.parse_args(argv)
    args.chunk, args.window = window(args.workload, args.warmup, args.steps, args.chunk)
    return args


def window(workload, warmup, steps, chunk=None):
    """Mixture steps per bench step and the timed window [start, end) of mixture
    steps: the window and one profiling chunk after it end by QUIET_END for any
    warm-up and step counts (chunk >= 1 always; an explicit chunk is kept)."""
    if chunk is None:
        chunk = max(1, min(MAX_CHUNK[workload], QUIET_END[workload] // (warmup + steps + 1)))
    start = warmup * chunk
    return chunk, (start, start + steps * chunk)


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu_index: int, period_ms: int = 20):
        self.gpu = gpu_index
        self.period = period_ms
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", str(self.period)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[0]))
                smax.append(float(s[1]))
                for n, v in zip(names, s[4:8]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "period_ms": self.period}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def grid_of(cfg):
    return [cfg.grid_x, cfg.grid_y] + ([cfg.ext_grid_z] if is3d(cfg) else [])


def traffic(kernel, workload, precision):
    """DRAM bytes (read + write) of one launch of the FDTD kernel from the
    committed ncu summary of this workload and precision, or None when there is none."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}_{precision}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("| traffic per launch (read + write) |"):
            mb = float(line.split("|")[2].split()[0])
            return int(mb * 1e6)
    return None


def load_workload(name):
    """Configuration and seeded bubbles of a workload, through the product's parser."""
    import crp

    cfg = crp.parse_file(WORKLOADS[name])
    seed = crp.seed_bubbles3 if is3d(cfg) else crp.seed_bubbles
    bub = seed(cfg) if cfg.ext_bubble_count > 0 else None
    return cfg, bub


def load_workload_oracle(name):
    """The same inputs built by the oracle's own parser and seeding (bit-equal to
    load_workload's, tests/test_oracle_workload.py); loads no product library."""
    import _bind as B

    cfg = B.oracle_parse_file(WORKLOADS[name])
    seed = B.oracle_seed_bubbles3 if is3d(cfg) else B.oracle_seed_bubbles
    bub = seed(cfg) if cfg.ext_bubble_count > 0 else None
    return cfg, bub


def oracle_sim(cfg, bub, threads):
    import _bind as B

    return (B.OracleSim3 if is3d(cfg) else B.OracleSim)(cfg, bub, threads=threads)


def cpu_baseline(cfg, bub, seconds, threads):
    """Oracle on the host cores: returns (cell-updates/s, steps, wall s, oracle sim)."""
    import _bind as B

    o = oracle_sim(cfg, bub, threads)
    t0 = time.perf_counter()
    o.step(1)
    t1 = time.perf_counter()
    n = max(1, min(200, int(seconds / max(t1 - t0, 1e-6))))
    t2 = time.perf_counter()
    o.step(n)
    t3 = time.perf_counter()
    rate = cell_count(cfg) * n / (t3 - t2)
    return rate, n + 1, t3 - t2, o


def state_error(g, oracle):
    """Relative L2 and max errors of a simulation's state against the oracle's."""
    out = {}
    for k in ("p0", "vx", "vy", "f_g"):
        a, b = g.field(k), oracle.field(k)
        out[k] = {"rel_l2": rel_l2(a, b), "rel_max": float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))}
    if g.dims.num_bubbles:
        a, b = g.bubbles("R_t"), oracle.bubbles("R_t")
        out["R_t"] = {"rel_l2": rel_l2(a, b), "rel_max": float(np.abs(a - b).max() / np.abs(b).max())}
    return out


def reference_sample(args, world):
    """Reference arm: the host oracle on all cores over the start of this
    workload's timed window (see the module docstring)."""
    import _bind as B

    if args.workload == "sweep_64":
        cfgs, _ = sweep_configs(B.oracle_parse_file)
        cfg = cfgs[0]
        bub = B.oracle_seed_bubbles(cfg)
    else:
        cfg, bub = load_workload_oracle(args.workload)
    threads = os.cpu_count() or 1
    o = oracle_sim(cfg, bub, threads)
    start = args.window[0]
    pre = max(0, start - args.warmup)
    o.step(pre) if pre else None
    for _ in range(args.warmup):
        o.step(1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step(1)
    dt = time.perf_counter() - t0
    cells = cell_count(cfg)
    nb_ref = o.dims3.num_bubbles if is3d(cfg) else o.dims.num_bubbles
    value = cells * args.steps / dt / 1e6
    t_start = int(o.stats().steps) - args.steps
    sample = (f"mixture steps {t_start}-{t_start + args.steps} of {args.workload} (untimed from t=0 to step "
              f"{t_start}), one per bench step, FP64 oracle with OpenMP")
    return {
        "impl": "reference", "metric": "Mcell-upd/s", "value": value, "unit": "Mcell-upd/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded bubbles, Philox-4x32-10)",
        "config": {"workload": args.workload, "grid": grid_of(cfg), "bubbles": nb_ref,
                   "mixture_steps_per_step": 1, "window_start": t_start, "precision": "fp64"},
        "bubble_steps_per_s": nb_ref * args.steps / dt,
        "cpu_baseline": {"value": value, "unit": "Mcell-upd/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "Mcell-upd/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_reference(args, rank, world):
    if rank != 0:
        return None
    return reference_sample(args, world)


def timed_run(cfg, bub, args, dist, dev):
    """Warm up, then time args.steps bench steps on the simulation's stream
    (CUDA events, max over ranks).  Returns a dict: ms, stats before/after,
    the simulation and the clocks; or {"error": ...} naming the failing step."""
    import torch

    import crp

    sim = crp.Sim(cfg, bub)
    stream = torch.cuda.ExternalStream(sim.stream)
    phase = "warm-up"
    try:
        for _ in range(args.warmup):
            sim.step(args.chunk)
        s0 = sim.stats()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        phase = "timed window"
        with Clocks(dev) as clk:
            e0.record(stream)
            for _ in range(args.steps):
                sim.step(args.chunk)
            e1.record(stream)
            e1.synchronize()
        torch.cuda.synchronize()
    except crp.CrpError as e:
        torch.cuda.synchronize()
        step = int(sim.stats().steps) + 1
        sim.close()
        return {"error": f"{phase}: mixture step {step}: {e}"}
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    return {"ms": ms, "s0": s0, "s1": sim.stats(), "sim": sim, "clocks": clk.summary(),
            "p0": sim.field("p0"), "R_t": sim.bubbles("R_t")}


def driven_sample(sim, args, cells, nb):
    """Further chunks of the primary run, timed one by one with CUDA events,
    until args.driven_chunks are done, the wall budget is spent or a step fails."""
    import torch

    import crp

    stream = torch.cuda.ExternalStream(sim.stream)
    start = DRIVEN_START[args.workload] if args.driven_start is None else args.driven_start
    out = {"chunks": [], "stopped": None}
    try:
        if sim.stats().steps < start:
            sim.step(start - sim.stats().steps)
    except crp.CrpError as e:
        out["stopped"] = f"before the sample, step {sim.stats().steps + 1}: {e}"
        return out
    out["start_step"] = int(sim.stats().steps)
    t_wall = time.perf_counter()
    ms_tot, steps_tot = 0.0, 0
    for _ in range(args.driven_chunks):
        if time.perf_counter() - t_wall > args.driven_seconds:
            out["stopped"] = "wall budget"
            break
        s0 = sim.stats()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        try:
            sim.step(args.driven_chunk)
        except crp.CrpError as e:
            torch.cuda.synchronize()
            out["stopped"] = f"step {sim.stats().steps + 1}: {e}"
            break
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        s1 = sim.stats()
        ms_tot += ms
        steps_tot += args.driven_chunk
        out["chunks"].append({"ms": ms, "picard_per_step": (s1.picard_total - s0.picard_total) / args.driven_chunk,
                              "rp_substeps_max": int(s1.rp_substeps_max),
                              "R_max_over_R0": float(np.max(sim.bubbles("R_t") / sim.bubbles("R0")))})
    if steps_tot:
        out["value"] = cells * steps_tot / (ms_tot * 1e-3) / 1e6
        out["unit"] = "Mcell-upd/s"
        out["bubble_steps_per_s"] = nb * steps_tot / (ms_tot * 1e-3)
    return out


def driven_rk45_sample(cfg, bub, args, cells, nb, ref_sim, rtol=1e-6, acc_sim=None, keep=False):
    """The driven sample of the same workload with the radius integrated by the
    rk45 scheme (ext.rp_scheme = rk45, relative tolerance rtol), in the primary
    precision: a fresh run taken untimed to the sample's start, then the same
    chunks timed one by one; its radii compared with the reference scheme's run
    at the same step (the difference is mostly the reference scheme's
    truncation error) and, with acc_sim, with a tighter-tolerance rk45 run (this
    run's own error).  keep: also return the simulation, left open."""
    import crp

    c = crp.Config.from_buffer_copy(cfg)
    c.ext_rp_scheme = 1
    c.ext_rp_tol = rtol
    sim = crp.Sim(c, bub)
    try:
        out = driven_sample(sim, args, cells, nb)
    except Exception:
        sim.close()
        raise
    out["scheme"] = "rk45"
    out["rtol"] = rtol
    steps = sim.stats().steps
    if ref_sim is not None and ref_sim.stats().steps == steps:
        out["R_t_rel_l2_vs_reference_scheme"] = rel_l2(sim.bubbles("R_t"), ref_sim.bubbles("R_t"))
        out["p0_rel_l2_vs_reference_scheme"] = rel_l2(sim.field("p0"), ref_sim.field("p0"))
    if acc_sim is not None and acc_sim.stats().steps == steps:
        key = f"vs_rk45_rtol_{acc_sim._keep[0].ext_rp_tol:g}"
        out["R_t_rel_l2_" + key] = rel_l2(sim.bubbles("R_t"), acc_sim.bubbles("R_t"))
        out["p0_rel_l2_" + key] = rel_l2(sim.field("p0"), acc_sim.field("p0"))
    if keep:
        return out, sim
    sim.close()
    return out


def driven_rk45_legs(cfg, bub, args, cells, nb, ref_sim):
    """rk45 at its default tolerance (1e-6) and at 1e-4, the second compared
    with the first: the accuracy a faster tolerance keeps."""
    accurate, acc_sim = driven_rk45_sample(cfg, bub, args, cells, nb, ref_sim, 1e-6, keep=True)
    try:
        fast = guarded(driven_rk45_sample, cfg, bub, args, cells, nb, ref_sim, 1e-4, acc_sim)
    finally:
        acc_sim.close()
    return accurate, fast


def max_over_ranks(x, dist):
    """The largest of every rank's x (the job's time is its slowest rank's);
    x itself without a process group.  NCCL reduces a CUDA tensor, gloo a CPU one."""
    if not dist:
        return x
    import torch

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, ms):
    """Whole-job throughput in units/s: every rank's units over the slowest rank's time."""
    return units_per_rank * world / (ms * 1e-3)


def focal_mask(sim, cfg, radius=2e-3):
    d = sim.dims
    fy = cfg.tr_focal_dist * 0.5 * np.sqrt(3.0)
    ii, jj = np.meshgrid(np.arange(d.i1m), np.arange(d.j1m))
    return np.hypot((ii - 0.5) * d.dx, (jj - 0.5) * d.dy - fy) <= radius


def adjoint_cost(cfg):
    """Cost of crp_adjoint against the forward it differentiates, on the same
    grid without bubbles (the adjoint's scope), FP64, 64 source elements: the
    device time of focal_compare_step(cfg) forward steps from t = 0, then of
    crp_adjoint over the same steps (its own forward with the focal record, the
    objective and the reverse sweep), both with CUDA events on the simulation's
    stream."""
    import torch

    import crp

    c = crp.Config.from_buffer_copy(cfg)
    c.bub_enable = 0
    c.ext_precision = 0
    c.ext_elements = 64
    c.dbg_T = 0
    steps = focal_compare_step(cfg)
    rng = np.random.default_rng(0xC0DA0004)
    amp, phase = rng.uniform(0.8, 1.2, 64), rng.uniform(-0.3, 0.3, 64)

    def timed(fn, sim):
        st = torch.cuda.ExternalStream(sim.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        out = fn()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    with crp.Sim(c) as fwd:
        fwd.set_source_elements(amp, phase)
        fwd.step(1)  # first-step set-up outside the timing, as below
        ms_fwd, _ = timed(lambda: fwd.step(steps - 1), fwd)
    with crp.Sim(c) as adj:
        adj.set_source_elements(amp, phase)
        ms_adj, (J, ga, gp) = timed(lambda: adj.adjoint(steps, 2.0e-3, 64), adj)
    ms_fwd *= steps / (steps - 1)
    return {"steps": steps, "focal_radius_m": 2.0e-3, "elements": 64, "precision": "fp64", "bubbles": 0,
            "forward_ms": ms_fwd, "adjoint_ms": ms_adj, "adjoint_over_forward": ms_adj / ms_fwd,
            "J": J, "grad_amp_norm": float(np.linalg.norm(ga)), "grad_phase_norm": float(np.linalg.norm(gp)),
            "note": "crp_adjoint (its forward with the focal record, the objective and the reverse sweep) over "
                    "the forward's device time on the same grid and steps; gradients checked against finite "
                    "differences and the oracle in tests/test_adjoint_gpu.py"}


def adjoint_cost3(cfg):
    """adjoint_cost on a 3-D grid: the bowl's own elements (amplitude 1, focusing
    phases), FP64, bubbles off, over the steps until 100 after the burst reaches
    the focus (array radius / c)."""
    import torch

    import crp

    c = crp.Config.from_buffer_copy(cfg)
    c.bub_enable = 0
    c.ext_precision = 0
    ne = c.ext_array_elements
    with crp.Sim(c) as probe:
        dt = probe.dims3.dt
    steps = int(np.ceil(c.ext_array_radius / c.ext_c_inf / dt)) + 100

    def timed(fn, sim):
        st = torch.cuda.ExternalStream(sim.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        out = fn()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    with crp.Sim(c) as fwd:
        fwd.step(1)
        ms_fwd, _ = timed(lambda: fwd.step(steps - 1), fwd)
    with crp.Sim(c) as adj:
        ms_adj, (J, ga, gp) = timed(lambda: adj.adjoint(steps, 2.0e-3, ne), adj)
    ms_fwd *= steps / (steps - 1)
    return {"steps": steps, "focal_radius_m": 2.0e-3, "elements": ne, "precision": "fp64", "bubbles": 0,
            "forward_ms": ms_fwd, "adjoint_ms": ms_adj, "adjoint_over_forward": ms_adj / ms_fwd,
            "J": J, "grad_amp_norm": float(np.linalg.norm(ga)), "grad_phase_norm": float(np.linalg.norm(gp)),
            "note": "crp_adjoint on the 3-D grid (its forward with the focal record, the objective and the reverse "
                    "sweep) over the forward's device time on the same grid and steps; gradients checked against "
                    "finite differences and the oracle in tests/test_adjoint3_gpu.py"}


def focal_compare_step(cfg):
    """Mixture step 100 steps after the focused burst reaches the focus: the
    source delays make every element's wave arrive there at t = focal_dist / c."""
    dt = cfg.sim_cfl * min(cfg.grid_lx / cfg.grid_x, cfg.grid_ly / cfg.grid_y) / cfg.ext_c_inf
    return int(np.ceil(cfg.tr_focal_dist / cfg.ext_c_inf / dt)) + 100


def compare_at(sims, cfg):
    """Advance the FP64 and mixed simulations (untimed) to the focal arrival and
    50 and 100 steps after it (focal_compare_step), comparing the mixed p0 with
    the FP64 p0 over the grid and within 2 mm of the focus, and the bubble radii,
    at each; the last comparison is the result, the earlier ones its history."""
    import crp

    last = focal_compare_step(cfg)
    history = []
    for step in (last - 100, last - 50, last):
        step = max(step, max(int(s.stats().steps) for s in sims.values()))
        for prec, sim in sims.items():
            try:
                if sim.stats().steps < step:
                    sim.step(step - int(sim.stats().steps))
            except crp.CrpError as e:
                out = {"at_step": step, "error": f"{prec} path: {e}"}
                if history:
                    out["history"] = history
                return out
        a, b = sims["mixed"].field("p0"), sims["fp64"].field("p0")
        m = focal_mask(sims["fp64"], cfg)
        history.append({"at_step": step, "p0_rel_l2": rel_l2(a, b), "p0_focal_rel_l2": rel_l2(a[m], b[m]),
                        "p0_focal_max_pa": float(np.max(np.abs(b[m]))),
                        "R_t_rel_l2": rel_l2(sims["mixed"].bubbles("R_t"), sims["fp64"].bubbles("R_t"))})
    out = dict(history[-1])
    out["history"] = history[:-1]
    return out


def rel_l2(a, b):
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / n) if n > 0 else float(np.linalg.norm(a))


def e2e_run(cfg, bub, args, nb):
    """End to end through the C ABI: crp_create from pinned host inputs (config
    and seeded bubbles), then the warm-up and timed bench steps from t = 0 with
    p0 and R_t read back into pinned host buffers after every bench step; wall
    clock over all of it (the teardown is not included)."""
    import torch

    import crp

    def pinned(a):
        t = torch.empty(a.shape if hasattr(a, "shape") else a, dtype=torch.float64, pin_memory=True).numpy()
        if hasattr(a, "shape"):
            t[...] = a
        return t

    bub_pinned = None
    if bub is not None:
        bub_pinned = crp.Bubbles(*(pinned(a) for a in (bub.x, bub.y, bub.r0, bub.n_b)),
                                 pinned(bub.z) if bub.z is not None else None)
    p0_shape = (cfg.ext_grid_z + 2, cfg.grid_y + 2, cfg.grid_x + 2) if is3d(cfg) else (cfg.grid_y + 2, cfg.grid_x + 2)
    p0_host = pinned(p0_shape)
    r_host = pinned((nb,)) if nb > 0 else None
    n_steps = args.warmup + args.steps
    t_steps = t_read = 0.0
    t0 = time.perf_counter()
    with crp.Sim(cfg, bub_pinned) as s2:
        t_create = time.perf_counter() - t0
        d = s2.dims
        for _ in range(n_steps):
            ta = time.perf_counter()
            s2.step(args.chunk)
            tb = time.perf_counter()
            s2.field("p0", out=p0_host)
            if r_host is not None:
                s2.bubbles("R_t", out=r_host)
            t_steps += tb - ta
            t_read += time.perf_counter() - tb
        wall = time.perf_counter() - t0
    h2d = (5 if is3d(cfg) else 4) * 8 * nb
    return {"value": cell_count(cfg) * n_steps * args.chunk / wall / 1e6, "unit": "Mcell-upd/s",
            "h2d_bytes_per_step": h2d // n_steps, "d2h_bytes_per_step": 8 * (int(np.prod(p0_shape)) + nb),
            "seconds": {"create": t_create, "steps": t_steps, "read_back": t_read, "total": wall},
            "mixture_steps": [0, n_steps * args.chunk],
            "note": "wall clock: crp_create (seeded bubbles uploaded from pinned host memory) + the warm-up and "
                    "timed bench steps from t=0 (the window's own steps and the ones before it) + p0 and R_t read "
                    "back into pinned host buffers after every bench step; the teardown is not included"}


def guarded(fn, *a, **k):
    """fn's result, or {"error": ...} if it raised: one failing leg of the bench
    does not cost the others their numbers."""
    try:
        return fn(*a, **k)
    except Exception as e:  # noqa: BLE001 - reported in the JSON line
        return {"error": f"{type(e).__name__}: {e}"}


def run_ours(args, rank, world, dist):
    import torch

    import crp

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    cfg, bub = load_workload(args.workload)
    cells = cell_count(cfg)
    S = args.chunk
    mix_steps = args.steps * S
    base = {
        "metric": "Mcell-upd/s", "unit": "Mcell-upd/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "data": "synthetic (seeded bubbles, Philox-4x32-10)",
        "config": {"workload": args.workload, "grid": grid_of(cfg),
                   "mixture_steps_per_step": S, "window": list(args.window), "precision": args.primary,
                   "parallelism": f"replicas x{world}", "l2": "state > L2 (no flush needed)"},
    }

    # Both forms of the workload: the plain FP64 path and the mixed form.
    runs = {}
    for prec in (["fp64", "mixed"] if args.precision == "both" else [args.precision]):
        cfg.ext_precision = 1 if prec == "mixed" else 0
        runs[prec] = timed_run(cfg, bub, args, dist, dev)
    primary = args.primary if args.primary in runs else next(iter(runs))
    run = runs[primary]
    cfg.ext_precision = 1 if primary == "mixed" else 0
    if "error" in run:
        for r in runs.values():
            if r.get("sim") is not None:
                r["sim"].close()
        return dict(base, value=None, error=f"{primary} path: {run['error']}", dtype=DTYPE[primary])
    sim = run["sim"]
    nb = sim.dims3.num_bubbles if is3d(cfg) else sim.dims.num_bubbles
    ms, s0, s1 = run["ms"], run["s0"], run["s1"]
    value = job_rate(cells * mix_steps, world, ms) / 1e6
    # The other path's simulation stays open when a driven sample follows: the
    # two are compared again once the burst has reached the focus.
    with_driven = rank == 0 and args.driven_chunks > 0 and world == 1

    # Roofline of the fused FDTD kernel: device time per launch from profiling
    # events over one more chunk (still before QUIET_END).
    sim.set_profiling(True)
    p0s = sim.stats()
    prof_err = guarded(sim.step, S)
    p1s = sim.stats()
    sim.set_profiling(False)
    n_fdtd = p1s.fdtd_launches - p0s.fdtd_launches
    fdtd_ms = (p1s.ms_fdtd - p0s.ms_fdtd) / max(n_fdtd, 1)
    prof = {k: (getattr(p1s, k) - getattr(p0s, k)) for k in ("ms_fdtd", "ms_rp", "ms_couple", "ms_other")}

    e2e = guarded(e2e_run, cfg, bub, args, nb) if rank == 0 and not args.no_e2e else None
    adjoint = (guarded(adjoint_cost3 if is3d(cfg) else adjoint_cost, cfg)
               if rank == 0 and world == 1 and not args.no_adjoint else None)
    driven = guarded(driven_sample, sim, args, cells, nb) if with_driven else None
    legs = guarded(driven_rk45_legs, cfg, bub, args, cells, nb, sim) if with_driven else None
    driven_rk45, driven_rk45_fast = legs if isinstance(legs, tuple) else (legs, None)
    focal = None
    if with_driven and all("sim" in r for r in runs.values()) and len(runs) > 1 and not is3d(cfg):
        focal = guarded(compare_at, {p: r["sim"] for p, r in runs.items()}, cfg)
    hbm, kind = peaks()
    bpc = (BYTES_PER_CELL_3D if is3d(cfg) else BYTES_PER_CELL)[primary]
    kernel = "fdtd3" if is3d(cfg) else "fdtd_strip"
    achieved = bpc * cells / (fdtd_ms * 1e-3) / 1e9 if n_fdtd else None
    result = None
    if rank == 0:
        result = dict(base)
        result.update({
            "value": value, "ms_per_step": ms / args.steps, "dtype": DTYPE[primary],
            "bubble_steps_per_s": nb * mix_steps * world / (ms * 1e-3),
            "picard_iterations_per_step": (s1.picard_total - s0.picard_total) / mix_steps,
            "gpu_launches": int(s1.kernel_launches - s0.kernel_launches),
            "roofline": {"kernel": kernel, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm if achieved else None, "peak_kind": kind,
                         "traffic": traffic(kernel, args.workload, primary), "bytes_per_cell": bpc,
                         "ms_per_launch": fdtd_ms if n_fdtd else None,
                         "launches": int(n_fdtd)},
            "kernel_ms_per_chunk": prof,
            "clocks": run["clocks"],
        })
        result["config"]["bubbles"] = nb
        if prof_err:
            result["roofline"]["error"] = prof_err["error"]
        for key, obj in (("driven", driven), ("driven_rk45", driven_rk45), ("driven_rk45_rtol_1e-4", driven_rk45_fast),
                         ("e2e", e2e), ("adjoint", adjoint)):
            if obj is not None:
                result[key] = obj
        for prec, r in runs.items():
            if "error" in r:
                result[f"{prec}_path"] = {"error": r["error"]}
                continue
            result[f"{prec}_path"] = {"value": cells * mix_steps * world / (r["ms"] * 1e-3) / 1e6,
                                      "ms_per_step": r["ms"] / args.steps,
                                      "picard_iterations_per_step": (r["s1"].picard_total - r["s0"].picard_total)
                                      / mix_steps,
                                      "rp_substeps_max": int(r["s1"].rp_substeps_max), "clocks": r["clocks"]}
        if "ms" in runs.get("fp64", {}) and "ms" in runs.get("mixed", {}):
            a, b = runs["mixed"], runs["fp64"]
            result["mixed_path"].update({
                "speedup_over_fp64": b["ms"] / a["ms"],
                "vs_fp64_at_window_end": {"at_step": int(args.window[1]),
                                          "p0_rel_l2": rel_l2(a["p0"], b["p0"]),
                                          "R_t_rel_l2": rel_l2(a["R_t"], b["R_t"])},
                "vs_fp64_at_focus": focal,
                "note": "relative L2 of the mixed path against the FP64 GPU path (which matches the FP64 oracle, "
                        "oracle_error); the focal figure is over the cells within 2 mm of the focus once the burst "
                        "has reached it"})
    for r in runs.values():
        if r.get("sim") is not None:
            r["sim"].close()

    if rank == 0 and not args.no_cpu_baseline:
        cpu = guarded(cpu_leg, args, cfg, bub)
        if "error" in cpu:
            result["cpu_baseline"] = cpu
        else:
            result.update(cpu)
    return result


def cpu_leg(args, cfg, bub):
    """The oracle on all host cores from t = 0 (inputs from its own parser and
    seeding), then fresh GPU runs of the same steps in both precisions compared
    with its state."""
    import crp

    threads = os.cpu_count() or 1
    ocfg, obub = load_workload_oracle(args.workload)
    rate, n, wall, oracle = cpu_baseline(ocfg, obub, args.cpu_seconds, threads)
    errors = {"steps": n}
    for prec in ("fp64", "mixed"):
        c = crp.Config.from_buffer_copy(cfg)
        c.ext_precision = 1 if prec == "mixed" else 0
        with crp.Sim(c, bub) as g:
            g.step(n)
            errors[prec] = state_error(g, oracle)
    oracle.close()
    return {"cpu_baseline": {"value": rate / 1e6, "unit": "Mcell-upd/s", "cores": threads, "kind": "port",
                             "sample": f"{n} mixture steps of {args.workload} from t=0 ({wall:.1f} s, OpenMP)"},
            "oracle_error": errors}


SWEEP_SEED = 0xC0DA0004


def sweep_configs(parse_file, n=64):
    """The batched-sweep workload: n axisymmetric simulations with grids X in
    [128, 512] (Y = 2X, dx = 0.1 mm), 1k-64k seeded bubbles (log-uniform), R0
    median 2-5 um (sigma_ln 0.3), 0.2-2.5 MPa surface drive at 0.5-2 MHz, the
    focus at 60 % of the length, and 2000-8000 steps each (the nominal length;
    the bench times a bounded number of them)."""
    import crp

    rng = np.random.default_rng(SWEEP_SEED)
    base = parse_file(WORKLOADS["axisym_256x512"])
    cfgs, steps = [], []
    for k in range(n):
        c = crp.Config.from_buffer_copy(base)
        X = int(rng.integers(128, 513)) // 8 * 8
        c.grid_x, c.grid_y = X, 2 * X
        c.grid_lx, c.grid_ly = X * 1e-4, 2 * X * 1e-4
        c.tr_amp = float(rng.uniform(0.2e6, 2.5e6)) / (998.0 * 1482.0)
        c.tr_freq = float(rng.uniform(0.5e6, 2.0e6))
        c.tr_focal_dist = 0.6 * c.grid_ly * 2.0 / np.sqrt(3.0)
        c.ext_bubble_count = int(round(np.exp(rng.uniform(np.log(1e3), np.log(6.4e4)))))
        c.bub_R0 = float(rng.uniform(2e-6, 5e-6))
        c.ext_bubble_seed = SWEEP_SEED + 1 + k
        c.ext_cloud_r = 0.1 * c.grid_lx
        c.ext_cloud_h = 0.2 * c.grid_ly
        cfgs.append(c)
        steps.append(int(rng.integers(2000, 8001)))
    return cfgs, steps


def run_sweep(args, rank, world):
    """Batched sweep on one GPU (crp_batch): every simulation advances
    args.chunk mixture steps per bench step from t = 0; device time from
    events on every simulation's stream (first start to last end)."""
    import torch

    import crp

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    cfgs, nominal = sweep_configs(crp.parse_file)
    n = len(cfgs)
    for c in cfgs:
        c.ext_precision = 1 if args.primary == "mixed" else 0
    with crp.Batch(cfgs) as batch:
        streams = [torch.cuda.ExternalStream(s.stream) for s in batch.sims]
        failed = {}

        def run(k_steps):
            try:
                batch.run([k_steps] * n)
            except crp.CrpError:
                for k, s in enumerate(batch.sims):
                    if k not in failed and s.stats().steps < batch_done[k] + k_steps:
                        failed[k] = int(s.stats().steps)

        batch_done = [0] * n
        run(args.warmup * args.chunk)
        batch_done = [s.stats().steps for s in batch.sims]
        # Per-simulation error against the FP64 oracle after the warm-up steps,
        # on four simulations (smallest and largest grid, most bubbles,
        # strongest drive; oracle seeding and parser, all host cores).
        oracle_err = {}
        if not args.no_cpu_baseline:
            import _bind as B

            ocfgs, _ = sweep_configs(B.oracle_parse_file)
            picks = sorted({min(range(n), key=lambda k: cfgs[k].grid_x), max(range(n), key=lambda k: cfgs[k].grid_x),
                            max(range(n), key=lambda k: cfgs[k].ext_bubble_count),
                            max(range(n), key=lambda k: cfgs[k].tr_amp)})
            for k in picks:
                if k in failed:
                    continue
                o = oracle_sim(ocfgs[k], B.oracle_seed_bubbles(ocfgs[k]), os.cpu_count() or 1)
                o.step(batch_done[k])
                oracle_err[str(k)] = {"grid": [cfgs[k].grid_x, cfgs[k].grid_y], "bubbles": cfgs[k].ext_bubble_count,
                                      "at_step": batch_done[k], **state_error(batch.sims[k], o)}
        # The autotuner (untimed): candidate settings timed on the batch itself,
        # every simulation's state restored after each trial.
        t0 = time.perf_counter()
        best, tried = batch.tune(trial_steps=10)
        tune_s = time.perf_counter() - t0
        s0 = [s.stats() for s in batch.sims]
        e0 = [torch.cuda.Event(enable_timing=True) for _ in range(n)]
        e1 = [torch.cuda.Event(enable_timing=True) for _ in range(n)]
        torch.cuda.synchronize()
        with Clocks(int(os.environ.get("LOCAL_RANK", 0))) as clk:
            for k in range(n):
                e0[k].record(streams[k])
            t0 = time.perf_counter()
            run(args.steps * args.chunk)
            wall = time.perf_counter() - t0
            for k in range(n):
                e1[k].record(streams[k])
            torch.cuda.synchronize()
        s1 = [s.stats() for s in batch.sims]
        ms = max(e0[0].elapsed_time(e1[k]) for k in range(n)) - min(
            e0[0].elapsed_time(e0[k]) for k in range(n))
        cell_steps = sum(c.grid_x * c.grid_y * (b.steps - a.steps) for c, a, b in zip(cfgs, s0, s1))
        bub_steps = sum(sim.dims.num_bubbles * (b.steps - a.steps) for sim, a, b in zip(batch.sims, s0, s1))
        launches = sum(b.kernel_launches - a.kernel_launches for a, b in zip(s0, s1))
        value = cell_steps / (ms * 1e-3) / 1e6
        return {
            "metric": "Mcell-upd/s", "value": value, "unit": "Mcell-upd/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPE[args.primary], "data": "synthetic (seeded sweep and bubbles)",
            "config": {"workload": "sweep_64", "simulations": n,
                       "cells": int(sum(c.grid_x * c.grid_y for c in cfgs)),
                       "bubbles": int(sum(sim.dims.num_bubbles for sim in batch.sims)),
                       "mixture_steps_per_step": args.chunk, "window": list(args.window),
                       "nominal_steps": [min(nominal), max(nominal)],
                       "parallelism": f"concurrent streams x{n}, {best.as_dict()['mode']} (autotuned)",
                       "l2": "state > L2 (no flush needed)"},
            "bubble_steps_per_s": bub_steps / (ms * 1e-3), "gpu_launches": int(launches),
            "failed_simulations": failed, "wall_s": wall, "clocks": clk.summary(),
            "tuning": {"chosen": best.as_dict(), "tried": [t.as_dict() for t in tried], "seconds": tune_s},
            "oracle_error": oracle_err,
        }


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    dist = None
    if args.impl == "reference":
        # The CPU reference arm runs on rank 0 only; other ranks exit without work.
        res = run_reference(args, rank, world)
        if res is not None:
            print(json.dumps(res), flush=True)
        return 0
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    rc = 0
    try:
        res = run_sweep(args, rank, world) if args.workload == "sweep_64" else run_ours(args, rank, world, dist)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
            rc = 1 if res.get("value") is None else 0
    finally:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
