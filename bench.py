"""Benchmark of the CUDA-RP simulation path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload axisym_1024x2048|axisym_256x512] [--chunk S] [--preroll P]

One bench step is S mixture time steps (default 100, one save interval of the
workload) of the full hot path: fused FDTD/PML update, bubble motion and
binning, and every Picard iteration of Rayleigh-Plesset + void-fraction
gather + pressure re-evaluation the step needs.  The run starts at t = 0 (or
after P untimed mixture steps, --preroll), takes W untimed bench steps and
times K: with the defaults, mixture steps 300-1300 of the workload, which end
as the burst's leading edge reaches the bubble cloud.  The "driven" object then
advances the same run untimed to --driven-start (default: where the burst
starts to drive the cloud) and times up to D chunks of 10 mixture steps there
(--driven-chunks, --driven-chunk, bounded by --driven-seconds of wall time),
recording where the run stops if a step fails (the workloads' drive grows the
bubbles until the mixture model stops converging).  The state (about 200 MB at
1024 x 2048) is larger than L2, so no flush is needed between steps.

metric: Mcell-upd/s — interior cells x mixture steps / device time (CUDA events
on the simulation's stream, max over ranks).  Also reported: bubble-steps/s,
the roofline of the fused FDTD kernel, a bounded CPU-oracle baseline and the
error of the GPU state against the FP64 oracle on that sample, an end-to-end
number through the C ABI with host buffers, clocks sampled during the timed
region.

Multi-GPU (--gpus N under torchrun): independent replicas, one per GPU, no
data-path collective ("replicas only": the simulation does not shard across
GPUs here); value = all ranks' cell updates / max rank time.

--impl reference: the reference simulator has no CPU implementation (its
simulation is CUDA-only), so the reference arm times the FP64 host oracle —
the restatement of the reference's kernels — on all host cores, each bench
step one mixture step of the same workload.
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
DRIVEN_START = {"axisym_1024x2048": 1700, "axisym_256x512": 900}
WORKLOADS = {
    "axisym_1024x2048": os.path.join(PKG, "configs", "axisym_1024x2048.conf"),
    "axisym_256x512": os.path.join(PKG, "configs", "axisym_256x512.conf"),
}
# Compulsory HBM traffic of the fused FDTD pass per cell: FP64
# reads px, py, vx, vy, f_g, f_gn, f_gm and writes px, py, vx, vy, predicted f_g;
# mixed stores each velocity/pressure value as two FP32 words and f_g as FP32.
BYTES_PER_CELL = {"fp64": 96, "mixed": 80}
DTYPE = {"fp64": "f64", "mixed": "f32 fields + f32 compensation (f64 arithmetic), f32 void fraction, "
                                  "f32 thermal model while |R/R0-1| <= 1e-3, f64 RP"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="axisym_1024x2048", choices=list(WORKLOADS) + ["sweep_64"])
    ap.add_argument("--chunk", type=int, default=None,
                    help="mixture steps per bench step (default 100; 25 for sweep_64, whose strongest drives "
                         "reach cavitation and stop converging from about step 500)")
    ap.add_argument("--preroll", type=int, default=0)
    ap.add_argument("--driven-start", type=int, default=None)
    ap.add_argument("--driven-chunks", type=int, default=10)
    ap.add_argument("--driven-chunk", type=int, default=10)
    ap.add_argument("--driven-seconds", type=float, default=60.0)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"])
    ap.add_argument("--primary", default="mixed", choices=["fp64", "mixed"])
    args = ap.parse_args()
    if args.chunk is None:
        args.chunk = 25 if args.workload == "sweep_64" else 100
    return args


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
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
                "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def traffic(workload, precision):
    """DRAM bytes (read + write) of one fdtd_strip launch from the committed ncu
    summary of this workload and precision, or None when there is none."""
    p = os.path.join(ROOT, "profiles", f"fdtd_strip_{workload}_{precision}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("| traffic per launch (read + write) |"):
            mb = float(line.split("|")[2].split()[0])
            return int(mb * 1e6)
    return None


def load_workload(name):
    import crp

    cfg = crp.parse_file(WORKLOADS[name])
    bub = crp.seed_bubbles(cfg) if cfg.ext_bubble_count > 0 else None
    return cfg, bub


def cpu_baseline(cfg, bub, seconds, threads):
    """Oracle on the host cores: returns (cell-updates/s, steps, wall s, oracle sim)."""
    import _bind as B

    o = B.OracleSim(cfg, bub, threads=threads)
    t0 = time.perf_counter()
    o.step(1)
    t1 = time.perf_counter()
    n = max(1, min(200, int(seconds / max(t1 - t0, 1e-6))))
    t2 = time.perf_counter()
    o.step(n)
    t3 = time.perf_counter()
    rate = cfg.grid_x * cfg.grid_y * n / (t3 - t2)
    return rate, n + 1, t3 - t2, o


def oracle_error(gpu_sim_factory, oracle, steps):
    """Relative errors of a fresh GPU run of `steps` steps against the oracle state."""
    with gpu_sim_factory() as g:
        g.step(steps)
        out = {}
        for k in ("p0", "vx", "vy", "f_g"):
            a, b = g.field(k), oracle.field(k)
            nrm = np.linalg.norm(b)
            out[k] = {"rel_l2": float(np.linalg.norm(a - b) / nrm) if nrm > 0 else float(np.linalg.norm(a)),
                      "rel_max": float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))}
        if g.dims.num_bubbles:
            a, b = g.bubbles("R_t"), oracle.bubbles("R_t")
            out["R_t"] = {"rel_l2": float(np.linalg.norm(a - b) / np.linalg.norm(b)),
                          "rel_max": float(np.abs(a - b).max() / np.abs(b).max())}
        out["steps"] = steps
        return out


def run_reference(args, rank, world):
    """Reference arm: the host oracle on all cores, one mixture step per bench step."""
    if rank != 0:
        return None
    import _bind as B

    if args.workload == "sweep_64":
        import crp

        cfgs, _ = sweep_configs()
        cfg = cfgs[0]
        bub = crp.seed_bubbles(cfg)
    else:
        cfg, bub = load_workload(args.workload)
    threads = os.cpu_count() or 1
    o = B.OracleSim(cfg, bub, threads=threads)
    for _ in range(args.warmup):
        o.step(1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step(1)
    dt = time.perf_counter() - t0
    cells = cfg.grid_x * cfg.grid_y
    value = cells * args.steps / dt / 1e6
    return {
        "impl": "reference", "metric": "Mcell-upd/s", "value": value, "unit": "Mcell-upd/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded bubbles)",
        "config": {"workload": args.workload, "grid": [cfg.grid_x, cfg.grid_y], "bubbles": o.dims.num_bubbles,
                   "mixture_steps_per_step": 1, "start": "t=0"},
        "bubble_steps_per_s": o.dims.num_bubbles * args.steps / dt,
        "cpu_baseline": {"value": value, "unit": "Mcell-upd/s", "cores": threads, "kind": "port",
                         "sample": f"{args.warmup}+{args.steps} mixture steps of {args.workload} from t=0"},
        "e2e": {"value": value, "unit": "Mcell-upd/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def timed_run(cfg, bub, args, preroll, dist, dev):
    """Pre-roll, warm up, then time args.steps bench steps on the simulation's
    stream (CUDA events, max over ranks).  Returns (ms, stats0, stats1, sim)."""
    import torch

    import crp

    sim = crp.Sim(cfg, bub)
    stream = torch.cuda.ExternalStream(sim.stream)
    sim.step(preroll)
    for _ in range(args.warmup):
        sim.step(args.chunk)
    s0 = sim.stats()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            sim.step(args.chunk)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(ms, dist)
    return ms, s0, sim.stats(), sim, clk.summary()


def driven_sample(sim, args, cells, nb):
    """Further chunks of the primary run, timed one by one with CUDA events,
    until args.driven_chunks are done, the wall budget is spent or a step fails."""
    import torch

    import crp

    stream = torch.cuda.ExternalStream(sim.stream)
    start = DRIVEN_START[args.workload] if args.driven_start is None else args.driven_start
    if sim.stats().steps < start:
        sim.step(start - sim.stats().steps)
    out = {"start_step": int(sim.stats().steps), "chunks": [], "stopped": None}
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


def adjoint_cost(cfg, args):
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


def focal_compare_step(cfg):
    """Mixture step 100 steps after the focused burst reaches the focus: the
    source delays make every element's wave arrive there at t = focal_dist / c."""
    dt = cfg.sim_cfl * min(cfg.grid_lx / cfg.grid_x, cfg.grid_ly / cfg.grid_y) / cfg.ext_c_inf
    return int(np.ceil(cfg.tr_focal_dist / cfg.ext_c_inf / dt)) + 100


def compare_at(primary_sim, other_sim, cfg, primary):
    """Advance both paths' simulations (untimed) to focal_compare_step and
    compare p0 over the grid and within 2 mm of the focus, and the bubble radii."""
    import crp

    step = max(int(primary_sim.stats().steps), focal_compare_step(cfg))
    for name, sim in (("primary", primary_sim), ("other", other_sim)):
        try:
            if sim.stats().steps < step:
                sim.step(step - int(sim.stats().steps))
        except crp.CrpError as e:
            path = primary if name == "primary" else ("fp64" if primary == "mixed" else "mixed")
            return {"at_step": step, "error": f"{path} path: {e}"}
    a, b = primary_sim.field("p0"), other_sim.field("p0")
    if primary != "mixed":
        a, b = b, a
    ra, rb = primary_sim.bubbles("R_t"), other_sim.bubbles("R_t")
    if primary != "mixed":
        ra, rb = rb, ra
    m = focal_mask(primary_sim, cfg)
    return {"at_step": step, "p0_rel_l2": rel_l2(a, b), "p0_focal_rel_l2": rel_l2(a[m], b[m]),
            "p0_focal_max_pa": float(np.max(np.abs(b[m]))), "R_t_rel_l2": rel_l2(ra, rb)}


def rel_l2(a, b):
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / n) if n > 0 else float(np.linalg.norm(a))


def run_ours(args, rank, world, dist):
    import torch

    import crp

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    cfg, bub = load_workload(args.workload)
    cells = cfg.grid_x * cfg.grid_y
    preroll = args.preroll
    S = args.chunk
    mix_steps = args.steps * S

    # Both forms of the workload: the plain FP64 path and the mixed form.
    runs = {}
    for prec in (["mixed", "fp64"] if args.precision == "both" else [args.precision]):
        cfg.ext_precision = 1 if prec == "mixed" else 0
        ms, s0, s1, sim, clocks = timed_run(cfg, bub, args, preroll, dist, dev)
        runs[prec] = {"ms": ms, "s0": s0, "s1": s1, "clocks": clocks,
                      "p0": sim.field("p0"), "R_t": sim.bubbles("R_t"), "sim": sim}
    # The other path's simulation stays open when a driven sample follows: the
    # two are compared again once the burst has reached the focus.
    with_driven = rank == 0 and args.driven_chunks > 0 and world == 1
    for prec, r in runs.items():
        if prec != args.primary and len(runs) > 1 and not with_driven:
            r["sim"].close()
            r["sim"] = None
    primary = args.primary if args.primary in runs else next(iter(runs))
    run = runs[primary]
    sim = run["sim"]
    cfg.ext_precision = 1 if primary == "mixed" else 0
    nb = sim.dims.num_bubbles
    ms, s0, s1 = run["ms"], run["s0"], run["s1"]
    value = job_rate(cells * mix_steps, world, ms) / 1e6
    launches = s1.kernel_launches - s0.kernel_launches
    picard = s1.picard_total - s0.picard_total

    # Roofline of the fused FDTD kernel: device time per launch from profiling events.
    sim.set_profiling(True)
    p0s = sim.stats()
    sim.step(S)
    p1s = sim.stats()
    sim.set_profiling(False)
    n_fdtd = p1s.fdtd_launches - p0s.fdtd_launches
    fdtd_ms = (p1s.ms_fdtd - p0s.ms_fdtd) / max(n_fdtd, 1)
    prof = {k: (getattr(p1s, k) - getattr(p0s, k)) for k in ("ms_fdtd", "ms_rp", "ms_couple", "ms_other")}
    # End to end through the C ABI: host inputs in, host rawdata arrays out.
    # Measured before the driven sample, so that no collapse phase precedes it.
    e2e = None
    if rank == 0 and not args.no_e2e:
        # Pinned host memory for the inputs and the read-backs, prepared before
        # the timed region.
        def pinned(a):
            t = torch.empty(a.shape if hasattr(a, "shape") else a, dtype=torch.float64, pin_memory=True).numpy()
            if hasattr(a, "shape"):
                t[...] = a
            return t

        bub_pinned = crp.Bubbles(*(pinned(a) for a in (bub.x, bub.y, bub.r0, bub.n_b))) if bub is not None else None
        p0_host = pinned((cfg.grid_y + 2, cfg.grid_x + 2))
        r_host = pinned((nb,)) if nb > 0 else None
        t0 = time.perf_counter()
        e2e_steps = 0
        t_steps = t_read = 0.0
        with crp.Sim(cfg, bub_pinned) as s2:
            t_create = time.perf_counter() - t0
            d = s2.dims
            h2d = 4 * 8 * nb
            for _ in range(args.steps):
                ta = time.perf_counter()
                s2.step(S)
                tb = time.perf_counter()
                e2e_steps += S
                s2.field("p0", out=p0_host)
                if r_host is not None:
                    s2.bubbles("R_t", out=r_host)
                t_steps += tb - ta
                t_read += time.perf_counter() - tb
            wall = time.perf_counter() - t0  # teardown (freeing the device memory) is not part of it
        e2e = {"value": cells * e2e_steps / wall / 1e6, "unit": "Mcell-upd/s",
               "h2d_bytes_per_step": h2d // max(args.steps, 1),
               "d2h_bytes_per_step": 8 * (d.i1m * d.j1m + nb),
               "seconds": {"create": t_create, "steps": t_steps, "read_back": t_read, "total": wall},
               "note": "wall clock: crp_create (seeded bubbles uploaded from pinned host memory) + steps from "
                       "t=0 + p0 and R_t read back into pinned host buffers every bench step; the simulation's "
                       "teardown is not included"}

    adjoint = adjoint_cost(cfg, args) if rank == 0 and world == 1 and not args.no_adjoint else None
    driven = driven_sample(sim, args, cells, nb) if with_driven else None
    focal = None
    if driven is not None and len(runs) > 1:
        other = next(r for prec, r in runs.items() if prec != primary)
        focal = compare_at(sim, other["sim"], cfg, primary)
    hbm, kind = peaks()
    bpc = BYTES_PER_CELL[primary]
    achieved = bpc * cells / (fdtd_ms * 1e-3) / 1e9
    result = None
    if rank == 0:
        result = {
            "metric": "Mcell-upd/s", "value": value, "unit": "Mcell-upd/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPE[primary], "data": "synthetic (seeded bubbles, Philox-4x32-10)",
            "config": {"workload": args.workload, "grid": [cfg.grid_x, cfg.grid_y], "bubbles": nb,
                       "mixture_steps_per_step": S, "preroll_steps": preroll, "precision": primary,
                       "parallelism": f"replicas x{world}", "l2": "state > L2 (no flush needed)"},
            "bubble_steps_per_s": nb * mix_steps * world / (ms * 1e-3),
            "picard_iterations_per_step": picard / mix_steps,
            "gpu_launches": int(launches),
            "roofline": {"kernel": "fdtd_strip", "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "peak_kind": kind, "traffic": traffic(args.workload, primary),
                         "bytes_per_cell": bpc,
                         "ms_per_launch": fdtd_ms},
            "kernel_ms_per_chunk": prof,
            "clocks": run["clocks"],
        }
        if driven is not None:
            result["driven"] = driven
        if e2e is not None:
            result["e2e"] = e2e
        if adjoint is not None:
            result["adjoint"] = adjoint
        for prec, r in runs.items():
            result[f"{prec}_path"] = {"value": cells * mix_steps * world / (r["ms"] * 1e-3) / 1e6,
                                      "ms_per_step": r["ms"] / args.steps,
                                      "picard_iterations_per_step": (r["s1"].picard_total - r["s0"].picard_total)
                                      / mix_steps,
                                      "rp_substeps_max": int(r["s1"].rp_substeps_max)}
        if "fp64" in runs and "mixed" in runs:
            a, b = runs["mixed"], runs["fp64"]
            result["mixed_vs_fp64"] = {
                "speedup": b["ms"] / a["ms"],
                "quiet": {"at_step": int(preroll + (args.warmup + args.steps) * S),
                          "p0_rel_l2": rel_l2(a["p0"], b["p0"]), "R_t_rel_l2": rel_l2(a["R_t"], b["R_t"])},
                "driven": focal,
                "note": "relative L2 of the mixed path against the FP64 GPU path, which matches the FP64 "
                        "oracle to ~1e-14 (oracle_error, tests/test_parity_gpu.py); the focal figure is over "
                        "the cells within 2 mm of the focus, once the burst has reached it"}
    for r in runs.values():
        if r["sim"] is not None:
            r["sim"].close()

    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cfg64 = crp.parse_file(WORKLOADS[args.workload])
        rate, n, wall, oracle = cpu_baseline(cfg64, bub, args.cpu_seconds, threads)
        result["cpu_baseline"] = {"value": rate / 1e6, "unit": "Mcell-upd/s", "cores": threads, "kind": "port",
                                  "sample": f"{n} mixture steps of {args.workload} from t=0 "
                                            f"({wall:.1f} s, OpenMP)"}
        result["oracle_error"] = oracle_error(lambda: crp.Sim(cfg, bub), oracle, n)
    return result


SWEEP_SEED = 0xC0DA0004


def sweep_configs(n=64):
    """The batched-sweep workload: n axisymmetric simulations with grids X in
    [128, 512] (Y = 2X, dx = 0.1 mm), 1k-64k seeded bubbles (log-uniform), R0
    median 2-5 um (sigma_ln 0.3), 0.2-2.5 MPa surface drive at 0.5-2 MHz, the
    focus at 60 % of the length, and 2000-8000 steps each (the nominal length;
    the bench times a bounded number of them)."""
    import crp

    rng = np.random.default_rng(SWEEP_SEED)
    base = crp.parse_file(WORKLOADS["axisym_256x512"])
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
    cfgs, nominal = sweep_configs()
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
                       "mixture_steps_per_step": args.chunk, "start": f"t = 0 + {args.warmup * args.chunk} steps",
                       "nominal_steps": [min(nominal), max(nominal)], "parallelism": "concurrent streams x64",
                       "l2": "state > L2 (no flush needed)"},
            "bubble_steps_per_s": bub_steps / (ms * 1e-3), "gpu_launches": int(launches),
            "failed_simulations": failed, "wall_s": wall, "clocks": clk.summary(),
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
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    try:
        res = run_sweep(args, rank, world) if args.workload == "sweep_64" else run_ours(args, rank, world, dist)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        if dist:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
