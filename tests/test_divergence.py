"""The wave breaker at its configured time step dt = 0.0008 makes PCISPH diverge.

Fixture tests/golden/wave_breaker_dt0008.npz comes from the REFERENCE's own CPU solver
(tests/golden/make_golden.py): the wave breaker on the 0.01 m lattice (396,000 particles),
zero initial pressure, its loop rule (no minimum, at most 50 iterations, eta 1 %). Per step
it holds the iteration count and the maximum |density error|. The reference converges for
13 steps and then runs to the 50-iteration bound with a 65 % error at step 13
(PCISPHSolver.cpp:64-163): the predict-correct iteration itself diverges at this time step,
so the configured run cannot be timed as a converging benchmark. The oracle and the CUDA
path must reproduce the fixture exactly (iteration counts equal, error bits equal).
"""
import os

import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "wave_breaker_dt0008.npz")


def _scene(min_iterations=1):
    sc = scenes.wave_breaker(seed=3, s=0.01, dt=0.0008)
    sc.params.pci_min_iterations = min_iterations
    return sc


def _check_run(step, read_error, z):
    its, errs = [], []
    for _ in range(len(z["iterations"])):
        its.append(step())
        errs.append(np.float32(np.max(np.abs(read_error()))))
    its, errs = np.array(its, np.int32), np.array(errs, np.float32)
    assert np.array_equal(its, z["iterations"]), (its, z["iterations"])
    assert np.array_equal(errs.view(np.uint32), z["max_abs_error"].view(np.uint32))
    return its, errs


def test_fixture_records_the_divergence():
    z = np.load(FIXTURE)
    its, err = z["iterations"], z["max_abs_error"] / 1000.0
    first = int(np.argmax(its >= 50))
    assert first == 13 and int(z["n"]) == 396000
    assert np.all(its[:first] < 50) and np.all(err[:first] < 0.01)
    assert err[first] > 0.5 and np.all(its[first:] == 50)


def test_oracle_reproduces_the_reference_divergence(oracle_mod):
    z = np.load(FIXTURE)
    oracle_mod.set_threads(os.cpu_count() or 1)
    o = oracle_mod.OracleSolver(_scene())
    _check_run(lambda: o.step(0.0008).iterations, lambda: o.get(abi.FIELD_DENSITY_ERROR), z)
    o.close()


def test_oracle_diverges_with_the_workload_iteration_rule(oracle_mod):
    """With the workload's rule (min 3 / max 50) the same scene converges at 3 iterations per
    step for 11 steps and runs to the bound at step 11."""
    oracle_mod.set_threads(os.cpu_count() or 1)
    o = oracle_mod.OracleSolver(_scene(min_iterations=3))
    stats = [o.step(0.0008) for _ in range(12)]
    o.close()
    assert [s.iterations for s in stats[:11]] == [3] * 11 and all(s.converged for s in stats[:11])
    assert stats[11].iterations == 50 and not stats[11].converged and stats[11].max_density_error_ratio > 0.1


@pytest.mark.gpu
def test_gpu_reproduces_the_reference_divergence():
    from liquidsimulation_b200.solver import from_scene
    z = np.load(FIXTURE)
    s = from_scene(_scene())
    _check_run(lambda: s.update(0.0008).iterations, lambda: s.read(abi.FIELD_DENSITY_ERROR), z)
    s.close()
