"""The waterfall (an empty 2 x 2 x 1 box with a ledge, sheets of 40 x 50 particles appended at
1.5 m/s, PCISPH eta 1 %, dt 0.0005) on the GPU against the oracle, bit for bit, for both
emission cadences: the reference scenario's (a sheet once the accumulated time reaches one
lattice spacing of travel, WaterfallScenario.cpp:55-74) over its first 40 steps, and a sheet
before every step over the first 5 steps, the last of which runs the PCISPH loop to its
50-iteration bound (tests/test_workload_limits.py pins that on the CPU). Every step appends
on the device (lsp_add_particles), so the emitter path is checked in the scene that uses it.
"""
import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes
from liquidsimulation_b200.solver import from_scene

pytestmark = pytest.mark.gpu

FIELDS = [abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_HALF_VELOCITY, abi.FIELD_OLD_HALF_VELOCITY,
          abi.FIELD_DENSITY, abi.FIELD_PRESSURE, abi.FIELD_FIRST_STEP, abi.FIELD_PRED_DENSITY,
          abi.FIELD_DENSITY_ERROR, abi.FIELD_PRED_POSITION, abi.FIELD_PRED_PRESSURE_FORCE]


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("cadence,steps", [("reference", 40), ("every_step", 5)])
def test_waterfall_emission_bit_exact(oracle_mod, cadence, steps):
    sc = scenes.waterfall(seed=5)
    gpu, orc = from_scene(sc), oracle_mod.OracleSolver(sc)
    interval = np.float32(np.float32(sc.spacing) / np.float32(1.5))
    acc, sheet, capped = np.float32(0.0), 0, 0
    try:
        for k in range(steps):
            emit = True
            if cadence == "reference":
                acc = np.float32(acc + np.float32(sc.dt))
                emit = bool(acc >= interval)
                if emit:
                    acc = np.float32(0.0)
            if emit:
                x, v = scenes.waterfall_sheet(sheet, seed=5)
                gpu.add_particles(x, v)
                orc.add_particles(x, v)
                sheet += 1
            sg, so = gpu.update(sc.dt), orc.step(sc.dt)
            if gpu.get_particle_count() == 0:
                # The reference cadence starts with empty steps: nothing changes on either
                # side, and the library reports 0 iterations for a step with no particles
                # (test_empty_and_tiny_scenes) where the oracle counts its loop's minimum.
                assert sg.iterations == 0 and orc.n == 0
                continue
            assert sg.iterations == so.iterations, (k, sg.iterations, so.iterations)
            capped += sg.iterations == sc.params.pci_max_iterations
            for f in FIELDS:
                assert np.array_equal(_bits(gpu.read(f)), _bits(orc.get(f))), (k, f)
        og, ig = gpu.neighbors()
        oo, io = orc.neighbors()
        assert np.array_equal(og, oo) and np.array_equal(ig, io)
        assert sheet >= 3 and gpu.get_particle_count() == sheet * 2000
        if cadence == "every_step":
            assert capped == 1   # the fifth step runs to the iteration bound, as on the CPU
    finally:
        gpu.close()
        orc.close()
