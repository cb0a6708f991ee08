"""Refusals and strict convergence at the step call, on the GPU, against the oracle.

lsp_step and lsp_batch_step refuse a time step that is not finite and positive with
LSP_ERR_INVALID and leave every solver as it was: the next valid step still matches the
oracle's first step bit for bit. With strict_convergence set, a PCISPH step that ends at its
iteration cap above eta still advances the particles exactly as the reference's update does
(it has no failure path, PCISPHSolver.cpp:64-170), fills the step's stats, and then returns
LSP_ERR_NOT_CONVERGED; without the flag the same step returns 0.
"""
import ctypes

import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes
from liquidsimulation_b200.solver import batch_from_scenes, from_scene

pytestmark = pytest.mark.gpu

BAD_DT = [0.0, -0.001, float("nan"), float("inf"), float("-inf")]
FIELDS = [abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_HALF_VELOCITY, abi.FIELD_PRESSURE,
          abi.FIELD_DENSITY]


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _scene(seed, **kw):
    sc = scenes.dam_break_pcisph(seed=seed, counts=(8, 10, 8), s=0.02)
    for k, v in kw.items():
        setattr(sc.params, k, v)
    return sc


def test_bad_time_steps_are_refused_and_change_nothing(oracle_mod):
    sc = _scene(4)
    gpu, orc = from_scene(sc), oracle_mod.OracleSolver(sc)
    batch = batch_from_scenes([sc, _scene(5)])
    try:
        for dt in BAD_DT:
            with pytest.raises(abi.LspError) as e:
                gpu.update(dt)
            assert e.value.code == abi.LSP_ERR_INVALID, dt
            with pytest.raises(abi.LspError) as e:
                batch.update(dt)
            assert e.value.code == abi.LSP_ERR_INVALID, dt
        sg, so = gpu.update(sc.dt), orc.step(sc.dt)
        sb = batch.update(sc.dt)[0]
        assert sg.iterations == so.iterations == sb.iterations
        for f in FIELDS:
            assert np.array_equal(_bits(gpu.read(f)), _bits(orc.get(f))), f
            assert np.array_equal(_bits(batch.read(0, f)), _bits(orc.get(f))), f
    finally:
        gpu.close()
        orc.close()
        batch.close()


def test_strict_convergence_reports_the_capped_step(oracle_mod):
    # eta far below what two iterations reach: every step ends at the cap, unconverged.
    kw = dict(pci_eta=1e-7, pci_min_iterations=1, pci_max_iterations=2)
    sc = _scene(6, **kw)
    strict = _scene(6, strict_convergence=1, **kw)
    plain, gpu, orc = from_scene(sc), from_scene(strict), oracle_mod.OracleSolver(sc)
    lib = abi.load_library()
    try:
        for step in range(2):
            st = abi.LspStepStats()
            rc = lib.lsp_step(gpu._h, ctypes.c_float(sc.dt), ctypes.byref(st))
            assert rc == abi.LSP_ERR_NOT_CONVERGED, (step, rc)
            assert b"max iterations" in lib.lsp_last_error()
            assert st.iterations == 2 and st.converged == 0 and st.max_density_error_ratio > 1e-7
            sp, so = plain.update(sc.dt), orc.step(sc.dt)
            assert sp.iterations == so.iterations == 2 and sp.converged == 0
            for f in FIELDS:
                assert np.array_equal(_bits(gpu.read(f)), _bits(orc.get(f))), (step, f)
                assert np.array_equal(_bits(plain.read(f)), _bits(orc.get(f))), (step, f)
    finally:
        plain.close()
        gpu.close()
        orc.close()


def test_strict_convergence_in_a_batch(oracle_mod):
    """One strict scene that stops at its cap makes the batch step return
    LSP_ERR_NOT_CONVERGED after every scene has stepped; its neighbour, which converges,
    still matches its own oracle."""
    kw = dict(pci_eta=1e-7, pci_min_iterations=1, pci_max_iterations=2)
    capped, easy = _scene(7, strict_convergence=1, **kw), _scene(8)
    batch = batch_from_scenes([capped, easy])
    oc, oe = oracle_mod.OracleSolver(_scene(7, **kw)), oracle_mod.OracleSolver(easy)
    lib = abi.load_library()
    try:
        st = (abi.LspStepStats * 2)()
        rc = lib.lsp_batch_step(batch._h, ctypes.c_float(easy.dt), st)
        assert rc == abi.LSP_ERR_NOT_CONVERGED
        sc_, se = oc.step(easy.dt), oe.step(easy.dt)
        assert st[0].iterations == sc_.iterations == 2 and st[0].converged == 0
        assert st[1].iterations == se.iterations and st[1].converged == 1
        for f in FIELDS:
            assert np.array_equal(_bits(batch.read(0, f)), _bits(oc.get(f))), f
            assert np.array_equal(_bits(batch.read(1, f)), _bits(oe.get(f))), f
    finally:
        batch.close()
        oc.close()
        oe.close()
