"""Golden fixtures produced by the reference's own CPU solver (tests/golden/make_golden.py).

The CPU test pins the oracle restatement to them; the GPU test pins the CUDA path
to them directly, so a GPU machine without the reference sources still checks
against the reference's outputs. Tolerance: exact float32 bit equality.
"""
import json
import os

import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KINDS = ["sph", "pcisph"]


def load(kind):
    z = np.load(os.path.join(HERE, f"{kind}_small.npz"))
    p = abi.default_params(**json.loads(str(z["params"])))
    cols = [scenes.Collider(k, tuple(c), s if k == "sphere" else tuple(s), b)
            for k, c, s, b in json.loads(str(z["colliders"]))]
    sc = scenes.Scene(f"golden_{kind}", p, z["positions0"], z["velocities0"], cols, float(z["dt"]), 4,
                      domain=((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)))
    return z, sc


def same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


FIELDS = (("x", abi.FIELD_POSITION), ("v", abi.FIELD_VELOCITY), ("half", abi.FIELD_HALF_VELOCITY),
          ("rho", abi.FIELD_DENSITY), ("p", abi.FIELD_PRESSURE))


@pytest.mark.parametrize("kind", KINDS)
def test_oracle_matches_golden(oracle_mod, kind):
    z, sc = load(kind)
    orc = oracle_mod.OracleSolver(sc)
    for s in range(4):
        st = orc.step(sc.dt)
        if kind == "pcisph":
            assert st.iterations == z["iterations"][s]
        for name, f in FIELDS:
            assert same_bits(orc.get(f), z[f"{name}_{s}"]), f"step {s} {name}"
        if s == 0:
            off, idx = orc.neighbors()
            assert np.array_equal(off, z["nbr_offsets_0"]) and np.array_equal(idx, z["nbr_index_0"])


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
def test_cuda_matches_golden(kind):
    from liquidsimulation_b200.solver import from_scene
    z, sc = load(kind)
    gpu = from_scene(sc)
    for s in range(4):
        st = gpu.update(sc.dt)
        if kind == "pcisph":
            assert st.iterations == z["iterations"][s]
        for name, f in FIELDS:
            assert same_bits(gpu.read(f), z[f"{name}_{s}"]), f"step {s} {name}"
        if s == 0:
            off, idx = gpu.neighbors()
            assert np.array_equal(off, z["nbr_offsets_0"]) and np.array_equal(idx, z["nbr_index_0"])
    gpu.close()
