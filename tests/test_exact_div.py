"""The force pass's exact division and square root (recip_rn, div_by, sqrt_rn in
csrc/lsp_device.cuh) against the device's own IEEE reciprocal, division and square root:
every float in [2^-126, 2^126] for the reciprocal, 10.7 billion pairs for the quotient (the
force pass's and the non-pressure pass's operand ranges), every float from 2^-102 up for the
square root (tests/cpp/exact_div_check.cu). Bit equality."""
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
    assert r.stdout.count(" 0 mismatches") == 4, r.stdout


@pytest.mark.gpu
def test_force_pass_fallback_gives_the_same_bits():
    """A lone particle far outside the range where the reciprocal-based division is exact
    (x = 1e8 m) makes the force pass and the non-pressure pass use IEEE division for the whole
    step; it interacts with nothing, so every other particle must end each step with the same
    bits as in the same scene without it (reciprocal-based division and square root), and
    both scenes match the oracle."""
    import numpy as np
    from liquidsimulation_b200 import abi, scenes
    from liquidsimulation_b200.solver import from_scene
    from oracle import oracle as O
    base = scenes.small_box_scene(n_side=(8, 9, 8), obstacles=False, pci_min_iterations=3, pci_max_iterations=20)
    base.colliders = []                        # free fall: nothing pulls the far particle back
    far = scenes.Scene("far", base.params, np.concatenate([base.positions, [[1.0e8, 0.5, 0.5]]]).astype(np.float32),
                       np.zeros((base.n + 1, 3), np.float32), [], base.dt, 3, domain=base.domain)
    a, b = from_scene(base), from_scene(far)
    oa, ob = O.OracleSolver(base), O.OracleSolver(far)
    fields = (abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_PRESSURE, abi.FIELD_PRED_PRESSURE_FORCE)
    for step in range(3):
        sa, sb = a.update(base.dt), b.update(base.dt)
        oa.step(base.dt)
        ob.step(base.dt)
        assert sa.iterations == sb.iterations
        for f in fields:
            ga, gb = a.read(f), b.read(f)
            assert np.array_equal(ga.view(np.uint32), gb[:base.n].view(np.uint32)), (step, f)
            assert np.array_equal(ga.view(np.uint32), oa.get(f).view(np.uint32)), (step, f)
            assert np.array_equal(gb.view(np.uint32), ob.get(f).view(np.uint32)), (step, f)
    for s in (a, b, oa, ob):
        s.close()
