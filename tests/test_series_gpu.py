"""`bubbles_series` on the GPU: configurations run concurrently write, file
for file, what `bubbles -a -d <dir> <conf>` writes for each one alone."""
import importlib.util
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(ROOT, "cuda-rp_b200", "build")

_spec = importlib.util.spec_from_file_location("trg", os.path.join(HERE, "test_rawdata_gpu.py"))
_trg = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_trg)


def test_series_matches_single_runs(tmp_path):
    base = _trg.tiny_conf_text()
    steps = _trg.STEPS
    assert f"n_step_max\t=\t{steps}" in base and "amp\t=\t0.12" in base
    texts = {
        "1": base,
        "2": base.replace(f"n_step_max\t=\t{steps}", f"n_step_max\t=\t{2 * steps}"),  # two saves
        "3": base.replace("amp\t=\t0.12", "amp\t=\t0.2"),  # another drive amplitude
    }
    confs = tmp_path / "confs"
    confs.mkdir()
    for i, t in texts.items():
        (confs / f"tiny_{i}.txt").write_text(t)
    r = subprocess.run([os.path.join(BUILD, "bubbles_series"), "-a", "--confs", str(confs), "--results",
                        str(tmp_path / "results"), "tiny"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    (run_dir,) = list((tmp_path / "results").glob("*/*"))
    for i, t in texts.items():
        assert (run_dir / f"tiny_{i}.txt").read_text() == t
        assert f"Processing tiny_{i}.txt" in r.stdout
        single = tmp_path / f"single_{i}"
        s = subprocess.run([os.path.join(BUILD, "bubbles"), "-a", "-d", str(single), str(confs / f"tiny_{i}.txt")],
                           capture_output=True, text=True, timeout=300)
        assert s.returncode == 0, s.stderr
        ours = run_dir / f"rawdata_{i}"
        names = sorted(p.name for p in single.iterdir() if p.name != "runtime.txt")
        assert names and names == sorted(p.name for p in ours.iterdir() if p.name != "runtime.txt")
        assert any(n.startswith("p0_step_") for n in names)
        for n in names:
            assert (ours / n).read_bytes() == (single / n).read_bytes(), (i, n)
        assert (ours / "runtime.txt").read_text().startswith("Finished in ")
