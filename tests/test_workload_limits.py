"""Where the configured workloads leave the range the reference's solvers handle, pinned.

The benchmark departs from two configured workloads because of these limits, so they are
checked here, on the CPU, with the oracle (the restatement pinned bit for bit to the
reference) and, where it has been built, with the reference's own solver:

- the plain SPH dam break (12,000 particles, k = 3, dt = 0.002) produces non-finite positions
  at step index 56, after its density has climbed past 1.8 rho0: the bench times it after a
  20-step lead-in, well before that;
- the waterfall (sheets of 40 x 50 particles, spacing 0.008 m, 1.5 m/s, PCISPH eta 1 %, dt
  0.0005): appending a sheet before every step, as the workload text says, packs the stream
  about 11 times denser than the lattice and PCISPH hits its 50-iteration bound by step 4;
  appending one sheet per lattice spacing of travel, the reference scenario's cadence
  (WaterfallScenario.cpp:55-74), converges until the falling stream hits the basin at step
  472, where the loop runs away as well.
"""
import os

import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes


def _first_non_finite(step, get, limit):
    for k in range(limit):
        step()
        if not np.all(np.isfinite(get(abi.FIELD_POSITION))):
            return k
    return None


def test_sph_dam_break_goes_non_finite_at_step_56(oracle_mod, ref_available):
    sc = scenes.dam_break_sph(seed=1)
    o = oracle_mod.OracleSolver(sc)
    assert _first_non_finite(lambda: o.step(sc.dt), o.get, 70) == 56
    o.close()
    if ref_available:
        r = oracle_mod.RefSolver(sc)
        assert _first_non_finite(lambda: r.step(sc.dt), r.get, 70) == 56
        r.close()


def _waterfall(oracle_mod, reference_cadence, steps):
    oracle_mod.set_threads(os.cpu_count() or 1)
    sc = scenes.waterfall(seed=5)
    o = oracle_mod.OracleSolver(sc)
    interval = np.float32(np.float32(sc.spacing) / np.float32(1.5))
    acc, sheet, its = np.float32(0.0), 0, []
    for _ in range(steps):
        emit = True
        if reference_cadence:
            acc = np.float32(acc + np.float32(sc.dt))
            emit = bool(acc >= interval)
            if emit:
                acc = np.float32(0.0)
        if emit:
            o.add_particles(*scenes.waterfall_sheet(sheet, seed=5))
            sheet += 1
        st = o.step(sc.dt)
        its.append((st.iterations, st.converged, st.max_density_error_ratio))
        if st.iterations >= sc.params.pci_max_iterations:
            break
    o.close()
    return its


def test_waterfall_every_step_emission_fails_at_once(oracle_mod):
    its = _waterfall(oracle_mod, False, 20)
    assert len(its) == 5 and its[-1][0] == 50 and its[-1][2] > 0.1
    assert all(c for _, c, _ in its[:-1])


def test_waterfall_reference_cadence_converges_until_the_impact(oracle_mod):
    its = _waterfall(oracle_mod, True, 600)
    assert len(its) == 473 and its[-1][0] == 50 and its[-1][2] > 0.1
    assert all(c and e <= 0.01 for _, c, e in its[:-1])
    assert max(i for i, _, _ in its[:-1]) < 50
