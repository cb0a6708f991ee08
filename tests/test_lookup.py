"""The division-free table lookup of the device kernels checked against IEEE division for
EVERY float distance in [0, h) (about 1e9 values per kernel radius), and its squared-distance
form against the IEEE square root for every float below the cutoff, on the CPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    exe = tmp_path_factory.mktemp("lookup") / "lookup_exhaustive"
    nvcc = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc"
    cmd = [nvcc, "-O2", "-std=c++17", "-Wno-deprecated-gpu-targets", "-Xcompiler", "-ffp-contract=off",
           "-I", os.path.join(ROOT, "liquidsimulation_b200", "csrc"),
           os.path.join(ROOT, "tests", "cpp", "lookup_exhaustive.cu"), "-o", str(exe)]
    if os.path.exists("/usr/bin/g++"):
        cmd[1:1] = ["-ccbin", "/usr/bin/g++"]
    subprocess.run(cmd, check=True)
    return exe


@pytest.mark.parametrize("radius,factor", [(0.0125, 3.2), (0.00459375, 3.2), (0.017, 2.688)])
def test_slot_equals_ieee_division_for_every_float(program, radius, factor):
    r = subprocess.run([str(program), str(radius), str(factor)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count(" 0 mismatches") == 2, r.stdout
