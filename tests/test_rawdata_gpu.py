"""Plain-text rawdata and the `bubbles` program against the reference's own
save_ascii output (tests/golden/ref_rawdata_tiny, written by the reference's
src/output_styles.cpp for the `tiny` case of make_ref_golden.py)."""
import os
import subprocess

import numpy as np
import pytest

import crp

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLD = os.path.join(HERE, "golden", "ref_rawdata_tiny")
import importlib.util  # noqa: E402

_spec = importlib.util.spec_from_file_location("mrg", os.path.join(HERE, "golden", "make_ref_golden.py"))
_mrg = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_mrg)

_, STEPS = _mrg.case_config("tiny")
FILES = [f"{stem}{STEPS:05d}.txt" for stem in ("fg_step_", "T_step_", "p0_step_", "vx_step_", "vy_step_",
                                               "bubble_radii_", "bubble_PG_")]

# crp.Config field -> (section, key) of the configuration file, for the keys the
# tiny case overrides.
KEYS = {"grid_x": ("grid", "x"), "grid_y": ("grid", "y"), "grid_lx": ("grid", "lx"), "grid_ly": ("grid", "ly"),
        "pml_grid_number": ("pml", "grid_number"), "tr_focal_dist": ("transducer", "focal_dist"),
        "tr_box_size": ("transducer", "box_size"), "sim_save_interval": ("simulation", "save_interval")}


def tiny_conf_text():
    """tests/golden/small.conf with the tiny case's overrides applied."""
    over = dict(_mrg.RUN_CASES["tiny"])
    steps = over.pop("steps")
    lines, section = [], None
    for line in open(os.path.join(HERE, "golden", "small.conf")).read().splitlines():
        t = line.strip()
        if t.startswith("["):
            section = t[1:-1]
        elif "=" in t and not t.startswith("#"):
            key = t.split("=")[0].strip()
            for field, (sec, k) in KEYS.items():
                if sec == section and k == key and field in over:
                    line = f"{key}\t=\t{over[field]!r}"
            if section == "simulation" and key == "n_step_max":
                line = f"{key}\t=\t{steps}"
        lines.append(line)
    return "\n".join(lines) + "\n"


def compare_text(ours, ref):
    a, b = open(ours).read().split("\n"), open(ref).read().split("\n")
    assert len(a) == len(b)
    vals_a, vals_b = [], []
    for la, lb in zip(a, b):
        if not lb:
            assert not la  # blank row separators in the same places
            continue
        ca, cb = la.split("\t"), lb.split("\t")
        assert len(ca) == len(cb) == 3
        assert ca[0] == cb[0] and ca[1] == cb[1], (la, lb)  # coordinates print identically
        vals_a.append(float(ca[2]))
        vals_b.append(float(cb[2]))
    va, vb = np.array(vals_a), np.array(vals_b)
    scale = max(np.abs(vb).max(), 1e-300)
    # 6 significant digits on both sides: differences are last-digit rounding at most
    assert np.abs(va - vb).max() <= 1e-5 * scale + 1e-12, np.abs(va - vb).max() / scale


def test_rawdata_matches_reference_save_ascii(tmp_path):
    cfg, steps = _mrg.case_config("tiny")
    with crp.Sim(cfg) as sim:
        sim.step(steps)
        sim.write_rawdata(str(tmp_path))
    for name in FILES:
        compare_text(os.path.join(tmp_path, name), os.path.join(GOLD, name))


def test_bubbles_program(tmp_path):
    cfg, steps = _mrg.case_config("tiny")
    conf = tmp_path / "tiny.conf"
    conf.write_text(tiny_conf_text())
    parsed = crp.parse_file(str(conf))
    for field in KEYS:
        assert getattr(parsed, field) == getattr(cfg, field), field
    assert parsed.sim_n_step_max == steps
    out = tmp_path / "out"
    exe = os.path.join(ROOT, "cuda-rp_b200", "build", "bubbles")
    r = subprocess.run([exe, "-a", "-d", str(out), str(conf)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "Input file is" in r.stdout
    for name in FILES:
        compare_text(os.path.join(out, name), os.path.join(GOLD, name))
    assert (out / "runtime.txt").read_text().startswith("Finished in ")
    lo, hi = [float(v) for v in (out / "p0_minmax.txt").read_text().split()]
    assert lo <= hi
    # The tracker ran with debug.T: one line per step plus the initial 0.
    lines = (out / "focalpoint_actual_T.txt").read_text().splitlines()
    assert len(lines) == steps + 1 and lines[0] == "0\t0"
    assert (out / "focalpoint_controller_T.txt").read_text().splitlines() == [f"1\t{cfg.tr_focal_dist * 3 ** 0.5 / 2:g}"]


def test_bubbles_program_pid_passes(tmp_path):
    """transducer.pid_iterate = 2 with -d: two passes into <dir>_I/ and
    <dir>_II/, the second starting from the first one's last control point."""
    conf = tmp_path / "pid.conf"
    text = tiny_conf_text().replace("[transducer]", "[transducer]\npid\t=\t1\npid_start_step\t=\t10\npid_iterate\t=\t2")
    conf.write_text(text)
    exe = os.path.join(ROOT, "cuda-rp_b200", "build", "bubbles")
    r = subprocess.run([exe, "-d", str(tmp_path / "out"), str(conf)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "0 pass took" in r.stdout and "1 pass took" in r.stdout
    ctl = []
    for d in ("out_I", "out_II"):
        rows = [ln.split("\t") for ln in (tmp_path / d / "focalpoint_controller_T.txt").read_text().splitlines()]
        assert rows[0][0] == "10"
        ctl.append([float(v) for _, v in rows])
    assert len(ctl[0]) == 1 + STEPS - 10
    assert abs(ctl[1][0] - ctl[0][-1]) <= 1e-5 * abs(ctl[0][-1])


def test_run_writes_what_a_step_loop_writes(tmp_path):
    """crp_run with a save interval writes the files a manual step loop writes."""
    cfg, steps = _mrg.case_config("tiny")
    a, b = tmp_path / "run", tmp_path / "loop"
    a.mkdir()
    b.mkdir()
    seen = []
    with crp.Sim(cfg) as sim:
        sim.run(n_steps=steps, save_interval=20, directory=str(a), progress=lambda s, t: seen.append(s))
        assert sim.stats().steps == steps
    with crp.Sim(cfg) as sim:
        for k in range(steps // 20):
            sim.step(20)
            sim.write_rawdata(str(b))
    assert seen == [20, 40, 60][: steps // 20]
    names = sorted(os.listdir(b))
    assert names and sorted(os.listdir(a)) == names
    for name in names:
        assert open(a / name).read() == open(b / name).read(), name


SPH = os.path.join(HERE, "golden", "ref_sph_tiny")


def _read_sph(path):
    """Records of an SPH file: each is (int length, bytes, int length)."""
    raw = open(path, "rb").read()
    recs, k = [], 0
    while k < len(raw):
        n = int(np.frombuffer(raw[k:k + 4], np.int32)[0])
        recs.append(raw[k + 4:k + 4 + n])
        assert raw[k + 4 + n:k + 8 + n] == raw[k:k + 4]
        k += 8 + n
    return recs


@pytest.mark.skipif(not os.path.isdir(SPH), reason="no SPH fixture")
def test_sph_matches_reference_save_sph(tmp_path):
    """SPH files against the reference's own save_sph output for the tiny case:
    identical headers; values as floats within one float rounding."""
    cfg, steps = _mrg.case_config("tiny")
    with crp.Sim(cfg) as sim:
        sim.step(steps)
        sim.write_sph(str(tmp_path))
    names = sorted(os.listdir(SPH))
    assert names == sorted(f"{s}{steps:05d}.sph" for s in ("fg_step_", "p0_step_", "T_step_"))
    for name in names:
        ours, ref = _read_sph(os.path.join(tmp_path, name)), _read_sph(os.path.join(SPH, name))
        assert len(ours) == len(ref) == 6
        for a, b in zip(ours[:5], ref[:5]):
            assert a == b, name
        va, vb = np.frombuffer(ours[5], np.float32), np.frombuffer(ref[5], np.float32)
        assert va.shape == vb.shape
        scale = max(float(np.abs(vb).max()), 1e-30)
        assert float(np.abs(va.astype(np.float64) - vb).max()) <= 2.4e-7 * scale, name
