"""Seeded random scenes against the oracle, bit for bit: random solver, particle radius,
kernel radius factor, viscosity, stiffness, negative-pressure factor, surface tension,
restitution, friction, gravity, iteration bounds, block placement, initial velocities,
boundary box or sphere, obstacles, with or without a user grid box, and in some PCISPH
scenes particles repeated at exactly the same position. Each scene runs a few
steps through the CUDA path and the oracle (pinned to the reference by test_oracle.py);
every field, the neighbour lists and the iteration counts must match exactly.
"""
import numpy as np
import pytest

from fuzz_scenes import random_scene
from liquidsimulation_b200 import abi
from liquidsimulation_b200.solver import from_scene

pytestmark = pytest.mark.gpu

FIELDS = [abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_HALF_VELOCITY, abi.FIELD_OLD_HALF_VELOCITY,
          abi.FIELD_DENSITY, abi.FIELD_PRESSURE, abi.FIELD_FIRST_STEP]
FIELDS_PCI = FIELDS + [abi.FIELD_PRED_DENSITY, abi.FIELD_DENSITY_ERROR, abi.FIELD_PRED_POSITION,
                       abi.FIELD_PRED_PRESSURE_FORCE]


@pytest.mark.parametrize("seed", range(40))
def test_random_scene_bit_exact(oracle_mod, seed):
    sc, pci = random_scene(seed)
    gpu = from_scene(sc)
    orc = oracle_mod.OracleSolver(sc)
    try:
        for step in range(3):
            sg, so = gpu.update(sc.dt), orc.step(sc.dt)
            assert sg.iterations == so.iterations, (seed, step, sg.iterations, so.iterations)
            for f in (FIELDS_PCI if pci else FIELDS):
                a = np.ascontiguousarray(gpu.read(f), np.float32).view(np.uint32)
                b = np.ascontiguousarray(orc.get(f), np.float32).view(np.uint32)
                assert np.array_equal(a, b), f"seed {seed} step {step} field {f}: {int((a != b).sum())} differ"
        og, ig = gpu.neighbors()
        oo, io = orc.neighbors()
        assert np.array_equal(og, oo) and np.array_equal(ig, io), f"seed {seed}: neighbour lists differ"
    finally:
        gpu.close()
        orc.close()
