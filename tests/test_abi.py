"""The C-ABI libraries load and export what the headers declare (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import pytest

import _bind as B
import crp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(crpo?_[a-z_0-9]+)\s*\(", text)))


def exported(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_libcrp_exports_every_declared_symbol():
    crp.load()
    names = declared("include/crp.h")
    assert "crp_create" in names and "crp_step" in names
    missing = [n for n in names if n not in exported(crp.LIB_PATH)]
    assert not missing, missing


def test_oracle_exports_every_declared_symbol():
    B.oracle_lib()
    names = declared("oracle/crp_oracle.h")
    missing = [n for n in names if n not in exported(B.ORACLE_LIB)]
    assert not missing, missing


def test_create_without_device_fails_cleanly():
    """Without a GPU, crp_create returns an error status instead of crashing."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    cfg = B.small_config()
    with pytest.raises(crp.CrpError) as e:
        crp.Sim(cfg)
    assert e.value.status == 10  # CRP_ERR_NO_DEVICE


def test_batch_without_device_fails_cleanly():
    """Without a GPU, crp_batch_create returns the first simulation's error."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(crp.CrpError) as e:
        crp.Batch([B.small_config(), B.small_config()])
    assert e.value.status == 10  # CRP_ERR_NO_DEVICE


def test_struct_sizes_match_c(tmp_path):
    """ctypes mirrors have the C layout (offset of the last member + size)."""
    src = str(tmp_path / "sizes.c")
    exe = str(tmp_path / "sizes")
    with open(src, "w") as f:
        f.write('#include "crp.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                'int main(){printf("%zu %zu %zu %zu\\n", sizeof(crp_config), sizeof(crp_stats), '
                'sizeof(crp_dims), sizeof(crp_bubbles_in));return 0;}\n')
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
    sizes = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    assert sizes == [ctypes.sizeof(crp.Config), ctypes.sizeof(crp.Stats), ctypes.sizeof(crp.Dims),
                     ctypes.sizeof(crp.BubblesIn)]
