"""What the trained warm start gains over the reference's zero start, measured.

The wave breaker on a 0.015 m lattice (115,434 particles) at the configured dt = 0.0008,
eta = 1 %, min 3 / max 50 iterations. The plain solver (zero initial pressure,
PCISPHSolver.cpp:58-62) meets eta for about 300 steps and then its loop runs away (50
iterations per step, error far above eta). The learned solver trains its network on the
converged plain steps of a 60-step lead-in and warm-starts every later step: its run stays
converged. That is the gain the network brings here, stability of the run; on equal inputs
(the same state stepped both ways) it costs about one iteration per step instead, which
bench.py's same_state block reports.
"""
import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes

STEPS, LEAD = 400, 60


def _run(learned):
    from liquidsimulation_b200.solver import from_scene
    sc = scenes.wave_breaker(seed=3, s=0.015, dt=0.0008)
    s = from_scene(sc)
    eta = sc.params.pci_eta
    if learned:
        s.mlp_record(True)
        s.mlp_set_loss_asymmetry(4.0)
    lead = LEAD
    ok, its = [], []
    for t in range(STEPS):
        st = s.update(sc.dt)
        good = bool(st.converged and st.max_density_error_ratio <= eta + 1e-12)
        ok.append(good)
        its.append(st.iterations)
        if learned and t < lead:
            if good:
                s.mlp_train(iterations=8, batch=65536, lr=2e-3, seed=t)
            if t == lead - 1 or not good:
                s.mlp_record(False)
                s.set_warm_start(abi.LSP_WARM_MLP)
                lead = t
    s.close()
    return np.array(ok), np.array(its)


@pytest.mark.gpu
def test_trained_warm_start_keeps_the_run_converged():
    plain_ok, plain_its = _run(False)
    learned_ok, learned_its = _run(True)
    print(f"\nplain: {plain_ok.sum()}/{STEPS} steps at <= 1 %, {plain_its.mean():.1f} iterations per step; "
          f"learned: {learned_ok.sum()}/{STEPS}, {learned_its.mean():.1f}")
    assert learned_ok.all()
    assert plain_ok.sum() < STEPS - 50            # the zero start runs away well before the end
    assert learned_its.mean() < 0.7 * plain_its.mean()
