"""Batches of independent scenes (lsp_batch_*): every scene of a batch must carry exactly the
bits of the same scene stepped alone by a single-scene handle, which tests/test_gpu_parity.py
pins to the oracle bit for bit; one scene is also checked against the oracle directly.

Compared per step and scene: iteration counts and convergence, every per-particle field
(0 ulp), neighbour lists, sorted keys, caller ids and the cell table. Launch shapes (graph
or direct launches, 128/256/512/1024 particles per block, persistent-kernel grid sizes) and the
autotuner must not change a bit.
"""
import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes
from liquidsimulation_b200.solver import batch_from_scenes, from_scene, SceneBatch

pytestmark = pytest.mark.gpu

FIELDS_PCI = [abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_HALF_VELOCITY, abi.FIELD_OLD_HALF_VELOCITY,
              abi.FIELD_DENSITY, abi.FIELD_PRESSURE, abi.FIELD_FIRST_STEP, abi.FIELD_PRED_DENSITY,
              abi.FIELD_DENSITY_ERROR, abi.FIELD_PRED_POSITION, abi.FIELD_PRED_HALF_VELOCITY,
              abi.FIELD_PRED_PRESSURE_FORCE, abi.FIELD_NEIGHBOR_COUNT]
FIELDS_SPH = FIELDS_PCI[:7] + [abi.FIELD_NEIGHBOR_COUNT]


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def small_batch(seed=4, count=5, nmin=300, nmax=3000):
    return scenes.batched_dam_breaks(seed=seed, scenes=count, nmin=nmin, nmax=nmax)


def compare_scene(batch, k, single, pci=True, grid=True, nbrs=True, tag=""):
    for f in (FIELDS_PCI if pci else FIELDS_SPH):
        a, b = batch.read(k, f), single.read(f)
        assert np.array_equal(bits(a), bits(b)), f"{tag} scene {k} field {f}: {int((bits(a) != bits(b)).sum())} differ"
    if nbrs:
        ob, ib = batch.neighbors(k)
        os_, is_ = single.neighbors()
        assert np.array_equal(ob, os_) and np.array_equal(ib, is_), f"{tag} scene {k}: neighbour lists differ"
    if grid:
        db, ob, kb, idb, cb = batch.grid(k)
        ds, os_, ks, ids, cs = single.grid()
        assert np.array_equal(db, ds) and np.array_equal(ob, os_), f"{tag} scene {k}: grid box differs"
        assert np.array_equal(kb, ks), f"{tag} scene {k}: sorted keys differ"
        assert np.array_equal(idb, ids), f"{tag} scene {k}: sorted caller ids differ"
        assert np.array_equal(cb, cs), f"{tag} scene {k}: cell tables differ"


def run_against_singles(scene_list, steps, launch=None, check_every=1):
    batch = batch_from_scenes(scene_list)
    if launch:
        batch.set_launch(**launch)
    singles = [from_scene(sc) for sc in scene_list]
    pci = scene_list[0].params.solver == abi.LSP_SOLVER_PCISPH
    dt = scene_list[0].dt
    try:
        for step in range(steps):
            sb = batch.update(dt)
            for k, s in enumerate(singles):
                ss = s.update(dt)
                assert sb[k].iterations == ss.iterations, (step, k, sb[k].iterations, ss.iterations)
                assert sb[k].converged == ss.converged
                assert sb[k].max_density_error_ratio == ss.max_density_error_ratio
                assert sb[k].max_neighbors == ss.max_neighbors
                if step % check_every == 0 or step == steps - 1:
                    compare_scene(batch, k, s, pci=pci, tag=f"step {step}")
        return batch, singles
    except Exception:
        batch.close()
        for s in singles:
            s.close()
        raise


def close_all(batch, singles):
    batch.close()
    for s in singles:
        s.close()


def test_batch_matches_single_scenes():
    b, s = run_against_singles(small_batch(), steps=6)
    info = b.get_launch()
    assert info["graph_active"] == 1, "the step did not run as a captured CUDA graph"
    close_all(b, s)


def test_scene_matches_oracle_directly(oracle_mod):
    scs = small_batch(seed=7, count=3, nmin=200, nmax=800)
    batch = batch_from_scenes(scs)
    orc = oracle_mod.OracleSolver(scs[1])
    for step in range(3):
        st = batch.update(scs[1].dt)[1]
        so = orc.step(scs[1].dt)
        assert st.iterations == so.iterations
        for f in FIELDS_PCI[:-1]:
            assert np.array_equal(bits(batch.read(1, f)), bits(orc.get(f))), (step, f)
        ob, ib = batch.neighbors(1)
        oo, io = orc.neighbors()
        assert np.array_equal(ob, oo) and np.array_equal(ib, io)
    batch.close()


@pytest.mark.parametrize("launch", [
    dict(use_graph=False, threads=256, loop_blocks=0),
    dict(use_graph=True, threads=128, loop_blocks=0),
    dict(use_graph=True, threads=512, loop_blocks=0),
    dict(use_graph=True, threads=1024, loop_blocks=0),
    dict(use_graph=False, threads=1024, loop_blocks=2),
    dict(use_graph=True, threads=256, loop_blocks=3),
])
def test_launch_shape_does_not_change_bits(launch):
    b, s = run_against_singles(small_batch(seed=5, count=4), steps=3, launch=launch, check_every=2)
    close_all(b, s)


def test_per_scene_iteration_rules():
    """Scenes with different eta, minimum and maximum iterations converge on their own."""
    scs = small_batch(seed=6, count=4)
    scs[0].params.pci_eta = 0.002
    scs[1].params.pci_min_iterations = 7
    scs[2].params.pci_max_iterations = 2
    scs[3].params.pci_eta = 0.05
    b, s = run_against_singles(scs, steps=4, check_every=3)
    close_all(b, s)


def test_sph_batch_matches_single_scenes():
    scs = [scenes.dam_break_sph(seed=11 + k, scale=0.3 + 0.1 * k) for k in range(3)]
    b, s = run_against_singles(scs, steps=4)
    close_all(b, s)


def test_autotune_keeps_results_and_advances_one_step():
    scs = small_batch(seed=8, count=4)
    batch = batch_from_scenes(scs)
    singles = [from_scene(sc) for sc in scs]
    dt = scs[0].dt
    batch.update(dt)
    for s in singles:
        s.update(dt)
    tuning, stats = batch.autotune(dt, repeats=2)
    for k, s in enumerate(singles):
        ss = s.update(dt)
        assert stats[k].iterations == ss.iterations
        compare_scene(batch, k, s, tag="autotuned step")
    assert tuning.candidates >= 3
    chosen = (tuning.threads, tuning.loop_blocks)
    cands = [(tuning.cand_threads[i], tuning.cand_loop_blocks[i]) for i in range(tuning.candidates)]
    assert chosen in cands
    best = min(tuning.cand_ms[i] for i in range(tuning.candidates))
    assert tuning.cand_ms[cands.index(chosen)] == best
    launch = batch.get_launch()
    assert launch["threads"] == tuning.threads
    for step in range(2):
        batch.update(dt)
        for k, s in enumerate(singles):
            s.update(dt)
    for k, s in enumerate(singles):
        compare_scene(batch, k, s, tag="after autotune")
    close_all(batch, singles)


def test_moving_collider_matches_single():
    scs = small_batch(seed=9, count=3)
    for sc in scs:
        sc.colliders.append(scenes.Collider("box", (0.8, 0.1, 0.5), (0.05, 0.1, 0.05), False))
    batch = batch_from_scenes(scs)
    singles = [from_scene(sc) for sc in scs]
    dt = scs[0].dt
    for step in range(4):
        cx = 0.8 - 0.1 * step
        batch.update_box(1, 1, (cx, 0.1, 0.5), (0.05, 0.1, 0.05))
        singles[1].update_static_collision_box(1, (cx, 0.1, 0.5), (0.05, 0.1, 0.05))
        batch.update(dt)
        for s in singles:
            s.update(dt)
    for k, s in enumerate(singles):
        compare_scene(batch, k, s, grid=False, tag="moving collider")
    close_all(batch, singles)


def test_neighbor_list_growth_in_batch():
    """A compressed scene overflows the first list capacity (2 x the lattice estimate of 33.5
    neighbours + 16, rounded up to 8 = 88); the step is redone with longer lists and must
    still match the single-scene run."""
    scs = small_batch(seed=10, count=3)
    squeeze = scs[2]
    c = squeeze.positions.mean(axis=0)
    squeeze.positions = (c + (squeeze.positions - c) * 0.6).astype(np.float32)
    batch = batch_from_scenes(scs)
    singles = [from_scene(sc) for sc in scs]
    dt = scs[0].dt
    for step in range(2):
        sb = batch.update(dt)
        for k, s in enumerate(singles):
            ss = s.update(dt)
            assert sb[k].iterations == ss.iterations and sb[k].max_neighbors == ss.max_neighbors
            compare_scene(batch, k, s, tag=f"step {step}")
        if step == 0:
            assert sb[2].max_neighbors > 88
    close_all(batch, singles)


def test_state_roundtrip_and_errors():
    scs = small_batch(seed=12, count=3)
    batch = batch_from_scenes(scs)
    dt = scs[0].dt
    batch.update(dt)
    x, v, h, o, f = batch.read_state()
    assert x.shape == (batch.total, 3)
    assert np.array_equal(bits(x[: scs[0].n]), bits(batch.positions(0)))
    batch.write_state(x, v, h, o, f)
    x2, *_ = batch.read_state()
    assert np.array_equal(bits(x), bits(x2))
    with pytest.raises(abi.LspError) as e:
        batch.add_scene(scs[0].params, scs[0].positions)
    assert e.value.code == abi.LSP_ERR_STATE
    with pytest.raises(abi.LspError):
        batch._call("lsp_batch_read_field", 7, abi.FIELD_POSITION, None, 1)
    batch.close()
    fresh = SceneBatch()
    fresh.add_scene(scs[0].params, scs[0].positions)
    sph = scenes.dam_break_sph(seed=1, scale=0.2)
    with pytest.raises(abi.LspError) as e:
        fresh.add_scene(sph.params, sph.positions)
    assert e.value.code == abi.LSP_ERR_INVALID
    warm = scenes.dam_break_pcisph(seed=2, counts=(4, 4, 4), s=0.02)
    warm.params.warm_start = abi.LSP_WARM_MLP
    with pytest.raises(abi.LspError):
        fresh.add_scene(warm.params, warm.positions)
    with pytest.raises(abi.LspError):
        fresh.set_launch(True, 192, 0)
    fresh.close()


def _trained_weights(sc, steps=8):
    trainer = from_scene(sc)
    trainer.mlp_record(True)
    for t in range(steps):
        trainer.update(sc.dt)
        trainer.mlp_train(iterations=10, batch=4096, lr=3e-3, seed=t)
    w = trainer.mlp_get_weights()
    trainer.close()
    return w


@pytest.mark.parametrize("guess", ["trained", "absurd"])
def test_batch_warm_start_matches_single_scenes(guess):
    """Learned warm start in a batch: per scene, the features, the kept/rejected decision,
    the iteration count and every field equal the single-scene warm start's bits."""
    from oracle import mlp_oracle as M
    scs = small_batch(seed=13, count=4)
    if guess == "trained":
        w = _trained_weights(scs[0])
    else:
        w = M.init(1).astype(np.float32)
        w[M.OFF["b3"]] = 400.0   # every guess raises the error: every scene restarts from zero
    batch = batch_from_scenes(scs)
    batch.mlp_set_weights(w)
    batch.set_warm_start(abi.LSP_WARM_MLP)
    singles = [from_scene(sc) for sc in scs]
    for s in singles:
        s.mlp_set_weights(w)
        s.set_warm_start(abi.LSP_WARM_MLP)
    dt = scs[0].dt
    kept = 0
    for step in range(5):
        sb = batch.update(dt)
        for k, s in enumerate(singles):
            ss = s.update(dt)
            assert (sb[k].iterations, sb[k].warm_start_used, sb[k].converged) == \
                   (ss.iterations, ss.warm_start_used, ss.converged), (step, k)
            kept += sb[k].warm_start_used
            compare_scene(batch, k, s, grid=False, nbrs=(step == 4), tag=f"{guess} step {step}")
            assert np.array_equal(bits(batch.read_features(k)), bits(s.read_features())), (step, k)
    if guess == "absurd":
        assert kept == 0
    close_all(batch, singles)


def test_batch_records_and_trains():
    scs = small_batch(seed=14, count=4)
    batch = batch_from_scenes(scs)
    batch.mlp_record(True)
    batch.mlp_set_loss_asymmetry(4.0)
    dt = scs[0].dt
    losses = []
    for step in range(10):
        batch.update(dt)
        losses.append(batch.mlp_train(iterations=10, batch=8192, lr=3e-3, seed=step))
    assert np.isfinite(losses).all() and losses[-1] < losses[0]
    f = batch.read_features(2)
    assert f.shape == (scs[2].n, 8) and np.isfinite(f).all()
    batch.mlp_record(False)
    batch.set_warm_start(abi.LSP_WARM_MLP)
    st = batch.update(dt)
    assert all(s.converged for s in st)
    batch.close()


def test_batch_auto_warm_start_switches_per_scene():
    """LSP_WARM_AUTO in a batch: each scene switches to the learned guess after its own slow
    step (scene 0 at a low switch point, the others never) and matches a single-scene solver
    in LSP_WARM_AUTO with the same switch point, bit for bit, including which steps tried the
    guess."""
    scs = small_batch(seed=15, count=4)
    w = _trained_weights(scs[0])
    for k, sc in enumerate(scs):
        sc.params.warm_auto_iterations = 2 if k == 0 else 1000
    batch = batch_from_scenes(scs)
    batch.mlp_set_weights(w)
    batch.set_warm_start(abi.LSP_WARM_AUTO)
    singles = [from_scene(sc) for sc in scs]
    for s in singles:
        s.mlp_set_weights(w)
        s.set_params(warm_start=abi.LSP_WARM_AUTO)
    dt = scs[0].dt
    for step in range(4):
        sb = batch.update(dt)
        for k, s in enumerate(singles):
            ss = s.update(dt)
            assert (sb[k].iterations, sb[k].warm_start_used, sb[k].warm_start_tried, sb[k].converged) == \
                   (ss.iterations, ss.warm_start_used, ss.warm_start_tried, ss.converged), (step, k)
            compare_scene(batch, k, s, grid=False, nbrs=(step == 3), tag=f"auto step {step}")
        assert sb[0].warm_start_tried == (1 if step > 0 else 0)
        assert all(sb[k].warm_start_tried == 0 for k in range(1, len(scs)) if sb[k].converged)
    close_all(batch, singles)
