"""bench.py's timed window and its reference arm, on CPU.

The window must stay inside the quiet phase for any warm-up and step counts
(the workloads' drive later grows the bubble cloud until the Picard loop stops
converging), and the reference arm must build and run its workload with the
oracle alone: no product library in the process."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


@pytest.mark.parametrize("workload", ["axisym_1024x2048", "axisym_256x512", "sweep_64"])
@pytest.mark.parametrize("wk", [(5, 20), (3, 10), (1, 2), (0, 1), (50, 200), (3000, 3000)])
def test_window_stays_quiet(workload, wk):
    w, k = wk
    chunk, (start, end) = bench.window(workload, w, k)
    assert chunk >= 1
    assert start == w * chunk and end == start + k * chunk
    assert chunk <= bench.MAX_CHUNK[workload]
    if w + k + 1 <= bench.QUIET_END[workload]:
        # The window and the profiling chunk after it end in the quiet phase.
        assert end + chunk <= bench.QUIET_END[workload]


def test_driver_window_values():
    assert bench.window("axisym_1024x2048", 5, 20) == (65, (325, 1625))
    assert bench.window("axisym_1024x2048", 3, 10) == (100, (300, 1300))
    assert bench.window("axisym_256x512", 5, 20) == (34, (170, 850))


def test_explicit_chunk_is_kept():
    assert bench.window("axisym_1024x2048", 5, 20, 7) == (7, (35, 175))


def test_reference_arm_loads_no_product_library():
    code = (
        "import json, sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'axisym_256x512', "
        "'--steps', '2', '--warmup', '1']\n"
        "import bench\n"
        "res = bench.run_reference(bench.parse(sys.argv[1:]), 0, 1)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'res': res, 'libcrp': 'libcrp.so' in maps, 'oracle': 'liboracle.so' in maps}))\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["oracle"] and not d["libcrp"]
    res = d["res"]
    chunk, (start, _) = bench.window("axisym_256x512", 1, 2)
    assert res["config"]["window_start"] == start
    assert res["steps"] == 2 and res["warmup"] == 1 and res["value"] > 0
    assert res["impl"] == "reference" and res["cpu_baseline"]["kind"] == "port"
