"""The rest of the reference-facing surface, on the GPU, against the oracle bit for bit.

- lsp_step_many: k steps in one call equal k calls of lsp_step.
- SPHSolver::removeParticles / removeStaticCollisionObjects / cleanUp
  (SPHSolver.cpp:137-184): a solver emptied and refilled steps exactly like a fresh one.
- setHasCollisionObjectDataChanged with a sphere (SPHSolver.cpp:612-615): a sphere moved and
  resized between steps, in a single solver and in a batch.
- Read-back (SPHSolver.cpp:384-429): lsp_read_particles gives the position and velocity
  fields in caller order; the batch's counts, masses and read-back agree with its scenes.
- lsp_device_info reports the device the library runs on.
- The products of a step (neighbour lists, grid, recorded features) describe the particles of
  that step: after particles are added or removed they are refused (LSP_ERR_STATE) until the
  next step.
"""
import ctypes

import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes
from liquidsimulation_b200.solver import batch_from_scenes, from_scene

pytestmark = pytest.mark.gpu

FIELDS = [abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_HALF_VELOCITY, abi.FIELD_OLD_HALF_VELOCITY,
          abi.FIELD_DENSITY, abi.FIELD_PRESSURE, abi.FIELD_FIRST_STEP]


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _same(gpu, orc, what):
    for f in FIELDS:
        assert np.array_equal(_bits(gpu.read(f)), _bits(orc.get(f))), (what, f)


def test_step_many_equals_single_steps(oracle_mod):
    sc = scenes.small_box_scene(n_side=(8, 9, 8))
    gpu, orc = from_scene(sc), oracle_mod.OracleSolver(sc)
    try:
        st = gpu.step_many(sc.dt, 4)
        for _ in range(4):
            so = orc.step(sc.dt)
        assert st.iterations == so.iterations
        _same(gpu, orc, "step_many(4)")
        before = _bits(gpu.read(abi.FIELD_POSITION)).copy()
        gpu.step_many(sc.dt, 0)
        assert np.array_equal(_bits(gpu.read(abi.FIELD_POSITION)), before)
        with pytest.raises(abi.LspError) as e:
            gpu.step_many(sc.dt, -1)
        assert e.value.code == abi.LSP_ERR_INVALID
    finally:
        gpu.close()
        orc.close()


@pytest.mark.parametrize("how", ["remove", "clean_up"])
def test_emptied_solver_steps_like_a_fresh_one(oracle_mod, how):
    a = scenes.small_box_scene(n_side=(8, 8, 8), seed=3)
    b = scenes.small_box_scene(n_side=(7, 9, 6), seed=4, obstacles=False)
    gpu = from_scene(a)
    for _ in range(3):
        gpu.update(a.dt)
    if how == "remove":
        gpu.remove_particles()
        gpu.remove_static_collision_objects()
    else:
        gpu.clean_up()
    assert gpu.get_particle_count() == 0
    st = gpu.update(a.dt)
    assert st.iterations == 0 and st.converged == 1
    gpu.add_particles(b.positions, b.velocities)
    for c in b.colliders:
        gpu.add_static_collision_object(c)
    orc = oracle_mod.OracleSolver(b)
    try:
        for step in range(3):
            sg, so = gpu.update(b.dt), orc.step(b.dt)
            assert sg.iterations == so.iterations, step
            _same(gpu, orc, f"refilled, step {step}")
        og, ig = gpu.neighbors()
        oo, io = orc.neighbors()
        assert np.array_equal(og, oo) and np.array_equal(ig, io)
    finally:
        gpu.close()
        orc.close()


def test_moving_sphere(oracle_mod):
    sc = scenes.small_box_scene(n_side=(8, 8, 8), seed=5)
    # From its place into the top of the block (z 0.05-0.21), resized on the way.
    path = [((0.3, 0.08, 0.6), 0.1), ((0.2, 0.1, 0.35), 0.12), ((0.15, 0.1, 0.3), 0.12), ((0.13, 0.1, 0.27), 0.1)]
    gpu, orc = from_scene(sc), oracle_mod.OracleSolver(sc)
    batch = batch_from_scenes([scenes.small_box_scene(n_side=(6, 6, 6), seed=6), sc])
    try:
        for step, (c, r) in enumerate(path):
            gpu.update_static_collision_sphere(2, c, r)
            orc.update_sphere(2, c, r)
            batch.update_sphere(1, 2, c, r)
            sg, so = gpu.update(sc.dt), orc.step(sc.dt)
            sb = batch.update(sc.dt)[1]
            assert sg.iterations == so.iterations == sb.iterations, step
            _same(gpu, orc, f"sphere step {step}")
            for f in FIELDS:
                assert np.array_equal(_bits(batch.read(1, f)), _bits(orc.get(f))), (step, f)
    finally:
        gpu.close()
        orc.close()
        batch.close()


def test_read_particles_and_batch_read_back():
    lib = abi.load_library()
    sc = scenes.small_box_scene(n_side=(6, 7, 5), seed=8)
    other = scenes.small_box_scene(n_side=(5, 5, 5), seed=9)
    gpu = from_scene(sc)
    batch = batch_from_scenes([other, sc])
    try:
        gpu.update(sc.dt)
        batch.update(sc.dt)
        n = sc.n
        x = np.empty((n, 3), np.float32)
        v = np.empty((n, 3), np.float32)
        assert lib.lsp_read_particles(gpu._h, x.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                      v.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n) == 0
        assert np.array_equal(_bits(x), _bits(gpu.read(abi.FIELD_POSITION)))
        assert np.array_equal(_bits(v), _bits(gpu.read(abi.FIELD_VELOCITY)))
        assert lib.lsp_read_particles(gpu._h, x.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                      None, n - 1) == abi.LSP_ERR_INVALID
        scenes_, total = ctypes.c_int32(), ctypes.c_int64()
        assert lib.lsp_batch_info(batch._h, ctypes.byref(scenes_), ctypes.byref(total)) == 0
        assert (scenes_.value, total.value) == (2, other.n + sc.n)
        for k, s in enumerate((other, sc)):
            cnt, mass = ctypes.c_int64(), ctypes.c_float()
            assert lib.lsp_batch_scene_count(batch._h, k, ctypes.byref(cnt)) == 0 and cnt.value == s.n
            assert lib.lsp_batch_particle_mass(batch._h, k, ctypes.byref(mass)) == 0
            single = from_scene(s)
            assert np.float32(mass.value).view(np.uint32) == np.float32(single.get_particle_mass()).view(np.uint32)
            single.close()
        xb = np.empty((n, 3), np.float32)
        vb = np.empty((n, 3), np.float32)
        assert lib.lsp_batch_read_particles(batch._h, 1, xb.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                            vb.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n) == 0
        assert np.array_equal(_bits(xb), _bits(x)) and np.array_equal(_bits(vb), _bits(v))
    finally:
        gpu.close()
        batch.close()


def test_device_info():
    import torch
    lib = abi.load_library()
    sms, major, minor = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert lib.lsp_device_info(ctypes.byref(sms), ctypes.byref(major), ctypes.byref(minor)) == 0
    props = torch.cuda.get_device_properties(0)
    assert (sms.value, major.value, minor.value) == (props.multi_processor_count, props.major, props.minor)
    assert major.value == 10


def test_step_products_need_a_step_on_the_current_particles():
    sc = scenes.small_box_scene(n_side=(6, 6, 6), seed=10)
    gpu = from_scene(sc)
    try:
        gpu.mlp_record(True)
        gpu.update(sc.dt)
        gpu.neighbors()
        gpu.grid()
        extra = scenes.lattice((0.5, 0.5, 0.5), (3, 3, 3), 0.02, 11)
        gpu.add_particles(extra)
        for call in (gpu.neighbors, gpu.grid, lambda: gpu.mlp_train(iterations=1, batch=64)):
            with pytest.raises(abi.LspError) as e:
                call()
            assert e.value.code == abi.LSP_ERR_STATE
        gpu.update(sc.dt)
        off, idx = gpu.neighbors()
        assert off.size == sc.n + extra.shape[0] + 1 and idx.size == off[-1]
        gpu.mlp_train(iterations=1, batch=64)
        gpu.remove_particles()
        with pytest.raises(abi.LspError) as e:
            gpu.neighbors()
        assert e.value.code == abi.LSP_ERR_STATE
    finally:
        gpu.close()
