"""Steps that start from the learned warm start, checked against the oracle bit for bit.

The warm start replaces the zero initial pressure of PCISPHSolver.cpp:58-62: iteration 0
predicts from zero pressure force, measures the density error, and then takes the
network's guess (p = y * p_scale, clamped at zero without negative pressure) in place of
its own correction (:117-125). The loop then runs as the reference's (:64-163); at
iteration 1 the guess is rejected, and the step restarts from the zero start, if the
maximum density error rose. The oracle restates exactly that (OracleSolver.step with
initial_pressure), so a step whose guess was KEPT is compared with the oracle started from
the same guess: every field to 0 ulp, the same iteration count and the same decision to
keep or reject the guess. The guess itself is recomputed here from the step's recorded features with
lsp_mlp_forward, which runs the same tensor-core tile as the warm-start kernel.
"""
import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes
from oracle import oracle as O

FIELDS = (abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_HALF_VELOCITY, abi.FIELD_OLD_HALF_VELOCITY,
          abi.FIELD_FIRST_STEP, abi.FIELD_DENSITY, abi.FIELD_PRESSURE, abi.FIELD_PRED_DENSITY, abi.FIELD_DENSITY_ERROR,
          abi.FIELD_PRED_POSITION, abi.FIELD_PRED_HALF_VELOCITY, abi.FIELD_PRED_PRESSURE_FORCE)


def _scene(**kw):
    sc = scenes.dam_break_pcisph(seed=5, counts=(14, 22, 14), s=0.02)
    sc.params.pci_min_iterations = 3
    for k, v in kw.items():
        setattr(sc.params, k, v)
    return sc


def _guess(y, delta, rho0, neg):
    """store_guess (mlp_tc.cu) in float32: p = y * (delta * 0.01 * rho0), clamped at zero
    when negative pressure is switched off."""
    p_scale = np.float32(delta) * np.float32(0.01) * np.float32(rho0)
    p = (np.asarray(y, np.float32) * p_scale).astype(np.float32)
    if neg == 0.0:
        p = np.where(p < 0, np.float32(0), p).astype(np.float32)
    return p


def _same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


# ---------------------------------------------------------------- oracle alone (CPU)

def test_oracle_rejected_guess_reproduces_the_zero_start():
    """An absurd initial pressure raises the error at iteration 1: the oracle restarts from
    the zero start and ends with the plain step's bits, two passes later."""
    sc = _scene(pci_min_iterations=1)
    plain, warm = O.OracleSolver(sc), O.OracleSolver(sc)
    for step in range(3):
        sp = plain.step(sc.dt)
        sw = warm.step(sc.dt, initial_pressure=np.full(sc.n, 1.0e5, np.float32))
        assert (sw.warm_start_tried, sw.warm_start_used) == (1, 0)
        assert sw.iterations == sp.iterations + 2
        for f in FIELDS:
            assert _same_bits(plain.get(f), warm.get(f)), (step, f)
    plain.close()
    warm.close()


def test_oracle_kept_guess_takes_the_given_pressure():
    """A modest guess is kept: iteration 0 holds exactly the given pressure (one iteration,
    the loop's upper bound), and a warm step never stops at iteration 0."""
    sc = _scene(pci_min_iterations=1, pci_max_iterations=1)
    o = O.OracleSolver(sc)
    o.step(sc.dt)
    p0 = np.linspace(0.0, 1.0, sc.n, dtype=np.float32)
    st = o.step(sc.dt, initial_pressure=p0)
    assert (st.iterations, st.warm_start_tried, st.warm_start_used) == (1, 1, 1)
    assert _same_bits(o.get(abi.FIELD_PRESSURE), p0)
    sc2 = _scene(pci_min_iterations=1)
    o2 = O.OracleSolver(sc2)
    o2.step(sc2.dt)
    st2 = o2.step(sc2.dt, initial_pressure=np.zeros(sc2.n, np.float32))
    assert st2.iterations >= 2 and st2.warm_start_tried == 1
    with pytest.raises(ValueError):
        o2.step(sc2.dt, initial_pressure=np.zeros(sc2.n + 1, np.float32))
    o.close()
    o2.close()


# ---------------------------------------------------------------- device vs oracle (GPU)

def _train(s, dt, steps=20):
    s.mlp_record(True)
    s.mlp_set_loss_asymmetry(4.0)
    for k in range(steps):
        st = s.update(dt)
        if st.converged if hasattr(st, "converged") else all(x.converged for x in st):
            s.mlp_train(iterations=20, batch=4096, lr=3e-3, seed=k)
    s.mlp_record(False)


@pytest.mark.gpu
@pytest.mark.parametrize("loop_mode", [abi.LSP_LOOP_PERSISTENT, abi.LSP_LOOP_HOST])
def test_kept_guess_matches_oracle(loop_mode):
    from liquidsimulation_b200.solver import from_scene
    sc = _scene(loop_mode=loop_mode)
    s = from_scene(sc)
    _train(s, sc.dt)
    s.set_warm_start(abi.LSP_WARM_MLP)
    o = O.OracleSolver(sc)
    delta = o.delta(sc.dt)
    kept = 0
    for step in range(6):
        x, v, h, old, first = s.read_state()
        sg = s.update(sc.dt)
        y = s.mlp_forward(s.read_features())
        o.set_state(x, v, h, old, first)
        so = o.step(sc.dt, initial_pressure=_guess(y, delta, sc.params.rest_density,
                                                   sc.params.negative_pressure_factor))
        assert (sg.iterations, sg.warm_start_used, sg.converged) == (so.iterations, so.warm_start_used,
                                                                     so.converged), step
        for f in FIELDS:
            assert _same_bits(s.read(f), o.get(f)), (step, f)
        kept += sg.warm_start_used
    assert kept >= 3, kept   # the comparison covers steps whose guess was kept
    s.close()
    o.close()


@pytest.mark.gpu
def test_batch_kept_guess_matches_oracle():
    from liquidsimulation_b200.solver import PCISPHSolver, batch_from_scenes
    scs = scenes.batched_dam_breaks(seed=4, scenes=3, nmin=800, nmax=2500)
    for sc in scs:
        sc.params.pci_min_iterations = 3
    dt = scs[0].dt
    b = batch_from_scenes(scs)
    _train(b, dt)
    b.set_warm_start(abi.LSP_WARM_MLP)
    net = PCISPHSolver()               # evaluates the batch's network on recorded features
    net.mlp_set_weights(b.mlp_get_weights())
    orcs = [O.OracleSolver(sc) for sc in scs]
    bounds = np.cumsum([0] + [sc.n for sc in scs])
    kept = 0
    for step in range(4):
        x, v, h, old, first = b.read_state()
        st = b.update(dt)
        for k, (sc, o) in enumerate(zip(scs, orcs)):
            lo, hi = bounds[k], bounds[k + 1]
            y = net.mlp_forward(b.read_features(k))
            o.set_state(x[lo:hi], v[lo:hi], h[lo:hi], old[lo:hi], first[lo:hi])
            so = o.step(dt, initial_pressure=_guess(y, o.delta(dt), sc.params.rest_density,
                                                    sc.params.negative_pressure_factor))
            assert (st[k].iterations, st[k].warm_start_used) == (so.iterations, so.warm_start_used), (step, k)
            for f in FIELDS:
                assert _same_bits(b.read(k, f), o.get(f)), (step, k, f)
            kept += st[k].warm_start_used
    assert kept >= 4, kept
    for o in orcs:
        o.close()
    net.close()
    b.close()
