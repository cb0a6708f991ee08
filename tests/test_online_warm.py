"""OnlineWarmStart: the learned warm start retrained online with the zero start as fallback.

CPU: the policy's schedule on a scripted stand-in for the solver (which steps train, when
the guess is used, that a warm step missing eta falls back to the zero start until the next
training step, and that unconverged training steps do not train). GPU: the policy on a real
solver, where every step still meets eta and training steps match a plain solver bit for bit.
"""
import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes
from liquidsimulation_b200.solver import OnlineWarmStart


class _Stats:
    def __init__(self, converged, err=0.005, warm=0):
        self.converged = converged
        self.max_density_error_ratio = err
        self.iterations = 3
        self.warm_start_used = warm


class _FakeSolver:
    """Records the calls OnlineWarmStart makes; `fail` holds the step indices that miss eta."""

    def __init__(self, fail=()):
        self.fail = set(fail)
        self.k = 0
        self.mode = abi.LSP_WARM_ZERO
        self.recording = False
        self.log = []
        self.trains = []
        p = abi.default_params(solver=abi.LSP_SOLVER_PCISPH, pci_eta=0.01)
        self._p = p

    @property
    def params(self):
        self._p.warm_start = self.mode
        return self._p

    def mlp_set_loss_asymmetry(self, w):
        pass

    def set_warm_start(self, mode):
        self.mode = mode

    def mlp_record(self, on):
        self.recording = on

    def mlp_train(self, iterations, batch, lr, seed):
        self.trains.append(self.k - 1)
        return 0.1

    def update(self, dt):
        ok = self.k not in self.fail
        self.log.append((self.k, self.mode, self.recording))
        self.k += 1
        return _Stats(ok, 0.005 if ok else 0.3, warm=int(self.mode == abi.LSP_WARM_MLP and ok))


def test_schedule_trains_on_lead_and_every_interval():
    s = _FakeSolver()
    pol = OnlineWarmStart(s, every=5, lead=3)
    for _ in range(20):
        pol.update(0.001)
    training = [k for k, mode, rec in s.log if rec]
    assert training == [0, 1, 2, 7, 12, 17]
    assert all(mode == abi.LSP_WARM_ZERO for k, mode, rec in s.log if rec)
    assert all(mode == abi.LSP_WARM_MLP for k, mode, rec in s.log if not rec)
    assert s.trains == training and pol.trained_steps == 6 and pol.warm_steps == 14


def test_missed_eta_falls_back_until_the_next_training_step():
    s = _FakeSolver(fail={4})
    pol = OnlineWarmStart(s, every=5, lead=3)
    for _ in range(13):
        pol.update(0.001)
    modes = {k: mode for k, mode, rec in s.log}
    assert modes[3] == abi.LSP_WARM_MLP and modes[4] == abi.LSP_WARM_MLP      # step 4 misses eta
    assert modes[5] == abi.LSP_WARM_ZERO and modes[6] == abi.LSP_WARM_ZERO    # fallback: zero start
    assert modes[8] == abi.LSP_WARM_MLP                                       # after training at 7
    assert pol.fallback_steps == 2


def test_unconverged_training_steps_do_not_train_and_nothing_is_warm_before_training():
    s = _FakeSolver(fail={0, 1, 2})
    pol = OnlineWarmStart(s, every=4, lead=3)
    for _ in range(8):
        pol.update(0.001)
    assert s.trains == [6]
    modes = {k: mode for k, mode, rec in s.log}
    assert modes[3] == abi.LSP_WARM_ZERO and modes[4] == abi.LSP_WARM_ZERO and modes[7] == abi.LSP_WARM_MLP
    with pytest.raises(ValueError):
        OnlineWarmStart(s, every=0)


@pytest.mark.gpu
def test_online_warm_start_on_a_solver():
    from liquidsimulation_b200.solver import from_scene
    sc = scenes.dam_break_pcisph(seed=5, counts=(14, 22, 14), s=0.02)
    a, plain = from_scene(sc), from_scene(sc)
    pol = OnlineWarmStart(a, every=6, lead=4, iterations=10, batch=4096, lr=3e-3)
    tried = []
    for k in range(16):
        x, v, h, old, first = a.read_state()
        st = pol.update(sc.dt)
        assert st.converged == 1 and st.max_density_error_ratio <= sc.params.pci_eta
        tried.append(st.warm_start_tried)
        if pol.is_training_step(k):
            # A training step is the plain solver's step from the same state, bit for bit.
            plain.write_state(x, v, h, old, first)
            sp = plain.update(sc.dt)
            assert st.iterations == sp.iterations and st.warm_start_tried == 0
            for f in (abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_PRESSURE):
                assert np.array_equal(a.read(f).view(np.uint32), plain.read(f).view(np.uint32)), (k, f)
    assert pol.trained_steps == pol.training_steps == 6 and sum(tried) == 10
    a.close()
    plain.close()


@pytest.mark.gpu
def test_set_warm_start_switches_mode_only():
    """lsp_set_warm_start changes params.warm_start and nothing else; an unknown mode is
    refused with LSP_ERR_INVALID and leaves the solver as it was."""
    from liquidsimulation_b200.solver import from_scene
    sc = scenes.dam_break_pcisph(seed=5, counts=(8, 10, 8), s=0.02)
    s = from_scene(sc)
    before = s.params
    s.set_warm_start(abi.LSP_WARM_MLP)
    after = s.params
    assert after.warm_start == abi.LSP_WARM_MLP
    after.warm_start = before.warm_start
    assert bytes(after) == bytes(before)
    with pytest.raises(abi.LspError) as e:
        s.set_warm_start(7)
    assert e.value.code == abi.LSP_ERR_INVALID and s.params.warm_start == abi.LSP_WARM_MLP
    s.close()
