"""Bit-exact parity at the benchmark sizes, not only at small ones: the 417,792-particle
PCISPH dam break, the 991,440-particle wave breaker and the 64-scene batch (1,350,776
particles) against the oracle (oracle/sph_oracle.cpp, pinned to the compiled reference by
tests/test_oracle.py), every field and the neighbour lists, tolerance 0 ulp.
"""
import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes
from liquidsimulation_b200.solver import batch_from_scenes, from_scene

pytestmark = pytest.mark.gpu

FIELDS = [abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_HALF_VELOCITY, abi.FIELD_OLD_HALF_VELOCITY,
          abi.FIELD_DENSITY, abi.FIELD_PRESSURE, abi.FIELD_FIRST_STEP, abi.FIELD_PRED_DENSITY,
          abi.FIELD_DENSITY_ERROR, abi.FIELD_PRED_POSITION, abi.FIELD_PRED_HALF_VELOCITY,
          abi.FIELD_PRED_PRESSURE_FORCE]


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def run(oracle_mod, sc, steps):
    gpu = from_scene(sc)
    orc = oracle_mod.OracleSolver(sc)
    try:
        for step in range(steps):
            sg, so = gpu.update(sc.dt), orc.step(sc.dt)
            assert sg.iterations == so.iterations, (step, sg.iterations, so.iterations)
            for f in FIELDS:
                a, b = bits(gpu.read(f)), bits(orc.get(f))
                assert np.array_equal(a, b), f"step {step} field {f}: {int((a != b).sum())} of {a.size} differ"
        og, ig = gpu.neighbors()
        oo, io = orc.neighbors()
        assert np.array_equal(og, oo) and np.array_equal(ig, io), "neighbour lists differ"
    finally:
        gpu.close()
        orc.close()


def test_dam_break_pcisph_417k(oracle_mod):
    sc = scenes.dam_break_pcisph(seed=2)
    assert sc.n == 417_792
    run(oracle_mod, sc, steps=4)


def test_wave_breaker_991k(oracle_mod):
    sc = scenes.wave_breaker(seed=3)
    assert sc.n == 991_440
    run(oracle_mod, sc, steps=3)


def test_batched_64_scenes(oracle_mod):
    scs = scenes.batched_dam_breaks(seed=4)
    batch = batch_from_scenes(scs)
    orcs = [oracle_mod.OracleSolver(sc) for sc in scs]
    try:
        for step in range(2):
            st = batch.update(scs[0].dt)
            for k, (sc, o) in enumerate(zip(scs, orcs)):
                so = o.step(sc.dt)
                assert st[k].iterations == so.iterations, (step, k)
                for f in (abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_DENSITY, abi.FIELD_PRESSURE):
                    assert np.array_equal(bits(batch.read(k, f)), bits(o.get(f))), (step, k, f)
    finally:
        batch.close()
        for o in orcs:
            o.close()
