"""Warm-start MLP: the FP64 oracle against finite differences (CPU), and the tensor-core
forward (tcgen05) / backward (mma.sync) kernels against the oracle (GPU).

Tolerances. Forward: |y_gpu - y_oracle| <= 2e-2 * (1 + |y|) per output (BF16 operands
rounded at the same points, FP32 vs FP64 accumulation, occasional one-ulp BF16 flips of
a hidden activation). Gradient: relative L2 error <= 2e-2 over the whole vector, and
<= 5e-2 per parameter block.
"""
import ctypes

import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes
from oracle import mlp_oracle as M


def batch(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0.0, 1.0, (n, 8)).astype(np.float32)
    x[:, 4] = rng.uniform(0.5, 1.2, n)          # neighbour-count-like feature
    t = (0.8 * x[:, 1] + 0.3 * np.tanh(x[:, 0]) - 0.1 * x[:, 4]).astype(np.float32)
    return x, t


def test_oracle_backward_matches_finite_differences():
    w = M.init(3)
    x, t = batch(64, 1)
    _, g = M.loss_and_grad(w, x.astype(np.float64), t, bf16_points=False)
    rng = np.random.default_rng(0)
    picks = list(rng.choice(M.N_PARAMS, 40, replace=False)) + [M.OFF["b3"], M.OFF["W3"], M.OFF["b1"]]
    fd = M.finite_difference(w, x.astype(np.float64), t, params=picks)
    for p, v in fd.items():
        assert abs(g[p] - v) <= 1e-6 + 1e-5 * abs(v), (p, g[p], v)


def test_bf16_rounding_helper():
    v = np.array([1.0, 1.00390625, 1.001953125, 3.0e-3, -2.5], np.float64)
    r = M.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0   # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even wins
    assert r[2] == 1.0
    assert abs(r[3] - 3.0e-3) / 3.0e-3 < 2 ** -8
    assert r[4] == -2.5


def _solver():
    from liquidsimulation_b200.solver import PCISPHSolver
    return PCISPHSolver()


def _set(s, w):
    w32 = np.ascontiguousarray(w, np.float32)
    s._call("lsp_mlp_set_weights", w32.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), w32.size)


@pytest.mark.gpu
def test_gpu_forward_matches_oracle():
    s = _solver()
    w = M.init(5)
    _set(s, w)
    x, _ = batch(1000, 2)
    out = np.empty(1000, np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    s._call("lsp_mlp_forward", x.ctypes.data_as(fp), 1000, out.ctypes.data_as(fp))
    ref, _ = M.forward(np.asarray(w, np.float32).astype(np.float64), x)
    assert np.all(np.abs(out - ref) <= 2e-2 * (1 + np.abs(ref))), np.max(np.abs(out - ref))
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 127, 129, 100_003])
def test_tensor_core_forward_tiles(n):
    """The tcgen05 inference in 128-row tiles: a single row, ragged tails and more tiles than
    resident blocks (grid-stride), against the oracle with a non-trivial output layer."""
    s = _solver()
    w = M.init(11)
    w[M.OFF["W3"]:M.OFF["W3"] + 32] *= 10.0
    w[M.OFF["b1"]:M.OFF["b1"] + 32] = np.linspace(-0.5, 0.5, 32)
    _set(s, w)
    x, _ = batch(n, 12)
    out = np.empty(n, np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    s._call("lsp_mlp_forward", x.ctypes.data_as(fp), n, out.ctypes.data_as(fp))
    ref, _ = M.forward(np.asarray(w, np.float32).astype(np.float64), x)
    err = np.abs(out - ref) / (1 + np.abs(ref))
    assert np.all(err <= 2e-2), float(err.max())
    assert np.median(err) < 2e-3
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [16, 100, 4096])
def test_gpu_gradient_matches_oracle(n):
    s = _solver()
    w = M.init(7)
    w[M.OFF["W3"]:M.OFF["W3"] + 32] *= 10.0      # a non-trivial output layer
    w32 = np.asarray(w, np.float32)
    _set(s, w32)
    x, t = batch(n, 3)
    g = np.empty(M.N_PARAMS, np.float32)
    loss = ctypes.c_float()
    fp = ctypes.POINTER(ctypes.c_float)
    s._call("lsp_mlp_gradient", x.ctypes.data_as(fp), t.ctypes.data_as(fp), n, g.ctypes.data_as(fp),
            ctypes.byref(loss))
    lref, gref = M.loss_and_grad(w32.astype(np.float64), x, t)
    assert abs(loss.value - lref) <= 1e-2 * (1 + abs(lref))
    rel = np.linalg.norm(g - gref) / np.linalg.norm(gref)
    assert rel < 2e-2, rel
    for name, size in (("W1", 256), ("b1", 32), ("W2", 1024), ("b2", 32), ("W3", 32), ("b3", 1)):
        a, b = g[M.OFF[name]:M.OFF[name] + size], gref[M.OFF[name]:M.OFF[name] + size]
        assert np.linalg.norm(a - b) <= 5e-2 * np.linalg.norm(b) + 1e-7, name
    # Deterministic: the partial-gradient reduction has a fixed order.
    g2 = np.empty_like(g)
    s._call("lsp_mlp_gradient", x.ctypes.data_as(fp), t.ctypes.data_as(fp), n, g2.ctypes.data_as(fp), None)
    assert np.array_equal(g.view(np.uint32), g2.view(np.uint32))
    s.close()


@pytest.mark.gpu
def test_weights_roundtrip_and_reset():
    s = _solver()
    w = M.init(9).astype(np.float32)
    _set(s, w)
    back = np.empty_like(w)
    s._call("lsp_mlp_get_weights", back.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), back.size)
    assert np.array_equal(w, back)
    with pytest.raises(abi.LspError):
        s._call("lsp_mlp_set_weights", w.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 10)
    s._call("lsp_mlp_reset", ctypes.c_uint64(1))
    s.close()


# ---------------------------------------------------------------- warm start in the solver

def _warm_scene(**kw):
    sc = scenes.dam_break_pcisph(seed=5, counts=(14, 22, 14), s=0.02)
    sc.params.pci_min_iterations = 1
    for k, v in kw.items():
        setattr(sc.params, k, v)
    return sc


@pytest.mark.gpu
@pytest.mark.parametrize("loop_mode", [abi.LSP_LOOP_PERSISTENT, abi.LSP_LOOP_HOST])
def test_rejected_guess_is_bit_identical_to_plain(loop_mode):
    """A network that guesses an absurd pressure raises the first error; the step restarts
    from zero pressure and must end with exactly the plain solver's bits."""
    from liquidsimulation_b200.solver import from_scene
    sc = _warm_scene(loop_mode=loop_mode)
    plain = from_scene(sc)
    warm = from_scene(sc)
    w = M.init(1).astype(np.float32)
    w[M.OFF["b3"]] = 400.0          # p_guess = 400 corrections' worth of pressure everywhere
    warm.mlp_set_weights(w)
    warm.set_warm_start(abi.LSP_WARM_MLP)
    for step in range(3):
        sp = plain.update(sc.dt)
        sw = warm.update(sc.dt)
        assert sw.warm_start_used == 0
        assert sw.iterations == sp.iterations + 2   # the two checked passes, then the plain loop
        for f in (abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_DENSITY, abi.FIELD_PRESSURE,
                  abi.FIELD_PRED_PRESSURE_FORCE):
            assert np.array_equal(plain.read(f).view(np.uint32), warm.read(f).view(np.uint32)), (step, f)
    plain.close()
    warm.close()


@pytest.mark.gpu
def test_features_follow_their_definitions():
    from liquidsimulation_b200.solver import from_scene
    sc = _warm_scene()
    s = from_scene(sc)
    s.mlp_record(True)
    prev_p = None
    delta = ctypes.c_float()
    s._call("lsp_pcisph_delta", ctypes.c_float(sc.dt), ctypes.byref(delta))
    p_scale = np.float32(delta.value) * np.float32(0.01) * np.float32(sc.params.rest_density)
    for step in range(3):
        s.update(sc.dt)
        f = s.read_features()
        counts = s.read(abi.FIELD_NEIGHBOR_COUNT)
        assert np.allclose(f[:, 4], counts / 32.0)
        if prev_p is not None:
            assert np.allclose(f[:, 1], prev_p / p_scale, rtol=1e-5, atol=1e-6)
        assert np.all(f[:, 7] >= 0) and np.all(f[:, 7] <= 1)
        prev_p = s.read(abi.FIELD_PRESSURE)
    s.close()


@pytest.mark.gpu
def test_trained_warm_start_converges():
    """Train on plain-PCISPH pressures, then warm-start: every step still meets eta, the
    guess is kept on most steps, and the persistent and per-phase loops give identical bits."""
    from liquidsimulation_b200.solver import from_scene
    solvers = []
    for mode in (abi.LSP_LOOP_PERSISTENT, abi.LSP_LOOP_HOST):
        sc = _warm_scene(loop_mode=mode, pci_min_iterations=3)
        s = from_scene(sc)
        s.mlp_record(True)
        losses = []
        for step in range(25):
            s.update(sc.dt)
            losses.append(s.mlp_train(iterations=20, batch=4096, lr=3e-3, seed=step))
        assert losses[-1] < losses[0]
        s.mlp_record(False)
        s.set_warm_start(abi.LSP_WARM_MLP)
        kept = 0
        for step in range(8):
            st = s.update(sc.dt)
            assert st.converged == 1 and st.max_density_error_ratio < sc.params.pci_eta
            kept += st.warm_start_used
        assert kept >= 4
        solvers.append(s)
    a, b = solvers
    for f in (abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_PRESSURE):
        assert np.array_equal(a.read(f).view(np.uint32), b.read(f).view(np.uint32)), f
    assert np.array_equal(a.mlp_get_weights(), b.mlp_get_weights())
    for s in solvers:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("loop_mode", [abi.LSP_LOOP_PERSISTENT, abi.LSP_LOOP_HOST])
def test_auto_warm_start_is_plain_until_its_switch_point(loop_mode):
    """LSP_WARM_AUTO with a switch point the scene never reaches runs the zero start: the
    same bits and iteration counts as LSP_WARM_ZERO, and no step tries the guess."""
    from liquidsimulation_b200.solver import from_scene
    sc = _warm_scene(loop_mode=loop_mode, pci_min_iterations=3)
    plain = from_scene(sc)
    auto = from_scene(sc)
    auto.mlp_set_weights(M.init(2).astype(np.float32))
    auto.set_params(warm_start=abi.LSP_WARM_AUTO, warm_auto_iterations=1000)
    for step in range(4):
        sp, sa = plain.update(sc.dt), auto.update(sc.dt)
        assert sa.iterations == sp.iterations and sa.warm_start_tried == 0 and sa.warm_start_used == 0
        for f in (abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_DENSITY, abi.FIELD_PRESSURE):
            assert np.array_equal(plain.read(f).view(np.uint32), auto.read(f).view(np.uint32)), (step, f)
    plain.close()
    auto.close()


@pytest.mark.gpu
@pytest.mark.parametrize("loop_mode", [abi.LSP_LOOP_PERSISTENT, abi.LSP_LOOP_HOST])
def test_auto_warm_start_switches_after_a_slow_step(loop_mode):
    """A step above the switch point turns the learned guess on from the next step: the run
    matches a solver that records features on the first step and is set to LSP_WARM_MLP
    after it, bit for bit, and stays on."""
    from liquidsimulation_b200.solver import from_scene
    sc = _warm_scene(loop_mode=loop_mode, pci_min_iterations=3)
    w = M.init(4).astype(np.float32)
    auto = from_scene(sc)
    auto.mlp_set_weights(w)
    auto.set_params(warm_start=abi.LSP_WARM_AUTO, warm_auto_iterations=2)
    ref = from_scene(sc)
    ref.mlp_set_weights(w)
    ref.mlp_record(True)
    for step in range(4):
        sa, sr = auto.update(sc.dt), ref.update(sc.dt)
        assert sa.warm_start_tried == (1 if step > 0 else 0)
        assert (sa.iterations, sa.warm_start_used) == (sr.iterations, sr.warm_start_used)
        for f in (abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_DENSITY, abi.FIELD_PRESSURE):
            assert np.array_equal(ref.read(f).view(np.uint32), auto.read(f).view(np.uint32)), (step, f)
        if step == 0:
            ref.set_warm_start(abi.LSP_WARM_MLP)
    with pytest.raises(abi.LspError):
        auto.set_params(warm_start=3)
    with pytest.raises(abi.LspError):
        auto.set_params(warm_auto_iterations=-1)
    auto.close()
    ref.close()
