"""The `bubbles` program's command line (no GPU needed for these paths)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "cuda-rp_b200", "build", "bubbles")


def test_no_input_file():
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Please specify an input configuration file" in r.stdout


def test_help():
    for flag in ("-h", "--help"):
        r = subprocess.run([EXE, flag], capture_output=True, text=True, timeout=60)
        assert r.returncode == 0 and "--ascii" in r.stdout and "--directory" in r.stdout
    r = subprocess.run([EXE, "--help-all"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "bubbles.liquid_surface_tension" in r.stdout


def test_bad_config_reports_error(tmp_path):
    conf = tmp_path / "bad.conf"
    conf.write_text("[grid]\nx = 3.5\n")
    r = subprocess.run([EXE, str(conf)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "invalid value" in r.stderr


def test_missing_config_file(tmp_path):
    r = subprocess.run([EXE, str(tmp_path / "nope.conf")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "cannot open" in r.stderr
