"""The oracle's own workload inputs (oracle/workload.cpp) against the product's:
configuration defaults, config-file parsing and the seeded bubble population
must agree bit for bit, so that the CPU arms of the bench, which build their
inputs with the oracle alone, run exactly the workload the CUDA path runs."""
import ctypes
import glob
import os

import numpy as np
import pytest

import crp
import _bind as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CONFS = sorted(glob.glob(os.path.join(ROOT, "cuda-rp_b200", "configs", "*.conf"))) + [
    os.path.join(ROOT, "tests", "golden", "small.conf")]


def raw(cfg):
    return bytes(memoryview(cfg))


def test_defaults_match():
    c = crp.Config()
    B.oracle_lib().crpo_config_defaults(ctypes.byref(c))
    assert raw(c) == raw(crp.defaults())


@pytest.mark.parametrize("path", CONFS, ids=os.path.basename)
def test_parse_matches(path):
    assert raw(B.oracle_parse_file(path)) == raw(crp.parse_file(path))


def test_grammar_matches(tmp_path):
    text = ("sph = 1\n# c\n[grid]\nx\t=\t300  # t\nlx = 30e-3\n[pml]\nx1 = true\ny1 = yes\nx0 = off\n"
            "[ext]\nprecision = mixed\ncloud_shape = Gaussian\nbubble_seed = 0xC0DA0002\nunknown_key = 3\n")
    p = tmp_path / "g.conf"
    p.write_text(text)
    assert raw(B.oracle_parse_file(str(p))) == raw(crp.parse_file(str(p)))
    p.write_text("[grid]\nx = 3\nx = 4\n")
    for parse in (B.oracle_parse_file, crp.parse_file):
        with pytest.raises(crp.CrpError):
            parse(str(p))


@pytest.mark.parametrize("shape", [0, 1, 2])
@pytest.mark.parametrize("cyl", [1, 0])
def test_seeding_matches(shape, cyl):
    cfg = crp.parse_file(CONFS[0])
    cfg.ext_cloud_shape = shape
    cfg.tr_cylindrical = cyl
    cfg.ext_bubble_count = 4099
    cfg.ext_bubble_seed = 0xC0DA0002 + 7 * shape + cyl
    a, b = crp.seed_bubbles(cfg), B.oracle_seed_bubbles(cfg)
    for u, v in zip((a.x, a.y, a.r0, a.n_b), (b.x, b.y, b.r0, b.n_b)):
        assert np.array_equal(u.view(np.uint64), v.view(np.uint64))
