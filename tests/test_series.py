"""The `bubbles_series` program's command line and file discovery (no GPU
needed for these paths): the reference's scripts/executor.sh NAME lists
confs/NAME_*.txt in `ls` order and writes into results/<date>/<HH:MM>/."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "cuda-rp_b200", "build", "bubbles_series")


def test_no_name():
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Please specify the name of a configuration series" in r.stdout


def test_help_and_unknown_option():
    r = subprocess.run([EXE, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "--confs" in r.stdout and "--results" in r.stdout
    r = subprocess.run([EXE, "--bogus", "x"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "unknown option --bogus" in r.stderr


def test_no_matching_files(tmp_path):
    (tmp_path / "confs").mkdir()
    (tmp_path / "confs" / "other_1.txt").write_text("[grid]\nx = 8\n")
    r = subprocess.run([EXE, "run"], capture_output=True, text=True, timeout=60, cwd=tmp_path)
    assert r.returncode == 1 and "no configuration file confs/run_*.txt" in r.stderr
    assert not (tmp_path / "results").exists()


def test_dry_run_plan(tmp_path):
    confs = tmp_path / "c"
    confs.mkdir()
    for name in ("run_2.txt", "run_10.txt", "run_a.txt", "run_1.conf", "runx_3.txt", "other_1.txt"):
        (confs / name).write_text("[grid]\nx = 8\n")
    r = subprocess.run([EXE, "--dry-run", "--confs", str(confs), "--results", str(tmp_path / "r"), "run"],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    m = re.fullmatch(r"results: (.*)/(\d{4}-\d{2}-\d{2})/(\d{2}:\d{2})", lines[0])
    assert m and m.group(1) == str(tmp_path / "r")
    run_dir = f"{m.group(1)}/{m.group(2)}/{m.group(3)}"
    # `ls` order of the names (bytewise): run_10 before run_2
    assert lines[1:] == [f"{confs}/run_{i}.txt -> {run_dir}/rawdata_{i}/" for i in ("10", "2", "a")]
    assert not (tmp_path / "r").exists()


def test_failed_runs_report(tmp_path):
    """A configuration that does not make a simulation fails alone: its error is
    reported with its file name, the file is still copied into the results, and
    the exit status is 1."""
    confs = tmp_path / "confs"
    confs.mkdir()
    (confs / "bad_1.txt").write_text("[grid]\nx = 3.5\n")
    r = subprocess.run([EXE, "bad"], capture_output=True, text=True, timeout=60, cwd=tmp_path)
    assert r.returncode == 1
    assert "[bad_1.txt] error: " in r.stderr and "invalid value" in r.stderr
    assert "1 of 1 configurations failed" in r.stderr
    copied = list((tmp_path / "results").glob("*/*/bad_1.txt"))
    assert len(copied) == 1 and copied[0].read_text() == "[grid]\nx = 3.5\n"
