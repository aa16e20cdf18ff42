"""The multi-process side of bench.py on CPU: replicas report the slowest
rank's time (gloo, world size 2), and the reference arm under torchrun runs on
rank 0 alone while the other ranks exit without work."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    ms = bench.max_over_ranks(10.0 * (rank + 1), dist)
    rate = bench.job_rate(1000.0, world, ms)
    with open(os.path.join(out, f"rank{rank}.json"), "w") as f:
        json.dump({"ms": ms, "rate": rate}, f)
    dist.barrier()
    dist.destroy_process_group()


def test_slowest_rank_sets_the_job_time(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        d = json.load(open(tmp_path / f"rank{r}.json"))
        assert d["ms"] == 20.0
        assert abs(d["rate"] - 1000.0 * 2 / 0.020) < 1e-9


def test_reference_arm_under_torchrun_prints_once():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"), "--impl", "reference",
           "--workload", "axisym_256x512", "--steps", "1", "--warmup", "0", "--gpus", "2"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
