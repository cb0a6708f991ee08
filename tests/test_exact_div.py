"""The force pass's exact division (recip_rn, div_by in csrc/lsp_device.cuh) against the
device's own IEEE reciprocal and division: every float in [2^-126, 2^126] for the reciprocal,
6.4 billion pairs for the quotient (tests/cpp/exact_div_check.cu). Bit equality required."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.gpu
def test_exact_division_matches_ieee(tmp_path):
    exe = tmp_path / "exact_div_check"
    nvcc = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc"
    cmd = [nvcc, "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-fmad=false",
           "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
           "-I", os.path.join(ROOT, "liquidsimulation_b200", "csrc"),
           os.path.join(ROOT, "tests", "cpp", "exact_div_check.cu"), "-o", str(exe)]
    if os.path.exists("/usr/bin/g++"):
        cmd[1:1] = ["-ccbin", "/usr/bin/g++"]
    subprocess.run(cmd, check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count(" 0 mismatches") == 3, r.stdout
