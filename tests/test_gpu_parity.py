"""CUDA path (liblsp.so through its C ABI) against the oracle, bit for bit.

The oracle (oracle/sph_oracle.cpp) is pinned to the compiled reference CPU solver by
tests/test_oracle.py. Here every per-particle field of every step must carry the same
bits as the oracle's FP32 result: positions, velocities, half velocities, densities,
pressures, predicted densities/errors/positions/pressure forces, neighbour lists,
iteration counts. Tolerance: 0 ulp (exact equality of the float32 bit patterns).
"""
import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes
from liquidsimulation_b200.solver import from_scene

pytestmark = pytest.mark.gpu

FIELDS_SPH = [abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_HALF_VELOCITY, abi.FIELD_OLD_HALF_VELOCITY,
              abi.FIELD_DENSITY, abi.FIELD_PRESSURE, abi.FIELD_FIRST_STEP]
FIELDS_PCI = FIELDS_SPH + [abi.FIELD_PRED_DENSITY, abi.FIELD_DENSITY_ERROR, abi.FIELD_PRED_POSITION,
                           abi.FIELD_PRED_HALF_VELOCITY, abi.FIELD_PRED_PRESSURE_FORCE]


def bits_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def mismatch_report(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    bad = a.view(np.uint32) != b.view(np.uint32)
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))
    return f"{int(bad.sum())} of {bad.size} differ, max |diff| {d.max() if d.size else 0:.3e}"


def run_pair(O, scene, steps, fields=None, check_neighbors=True):
    gpu = from_scene(scene)
    orc = O.OracleSolver(scene)
    pci = scene.params.solver == abi.LSP_SOLVER_PCISPH
    fields = fields or (FIELDS_PCI if pci else FIELDS_SPH)
    try:
        for s in range(steps):
            sg = gpu.update(scene.dt)
            so = orc.step(scene.dt)
            assert sg.iterations == so.iterations, f"step {s}: iterations {sg.iterations} vs {so.iterations}"
            assert sg.converged == so.converged
            if check_neighbors:
                og, ig = gpu.neighbors()
                oo, io = orc.neighbors()
                assert np.array_equal(og, oo), f"step {s}: neighbour offsets differ"
                assert np.array_equal(ig, io), f"step {s}: neighbour lists differ"
            for f in fields:
                a, b = gpu.read(f), orc.get(f)
                assert bits_equal(a, b), f"step {s} field {f}: {mismatch_report(a, b)}"
        return gpu, orc
    except Exception:
        gpu.close()
        raise


def test_tables_mass_delta(oracle_mod):
    sc = scenes.small_box_scene()
    gpu = from_scene(sc)
    orc = oracle_mod.OracleSolver(sc)
    assert bits_equal(gpu.kernel_tables(), orc.tables())
    assert np.float32(gpu.get_particle_mass()).view(np.uint32) == np.float32(orc.mass()).view(np.uint32)
    assert np.float32(gpu.get_kernel_radius()).view(np.uint32) == np.float32(orc.kernel_radius()).view(np.uint32)
    d = ctypes_delta(gpu, sc.dt)
    assert np.float32(d).view(np.uint32) == np.float32(orc.delta(sc.dt)).view(np.uint32)
    gpu.close()


def ctypes_delta(gpu, dt):
    import ctypes
    out = ctypes.c_float()
    gpu._call("lsp_pcisph_delta", ctypes.c_float(dt), ctypes.byref(out))
    return out.value


def test_grid_build_matches_spec(oracle_mod):
    sc = scenes.small_box_scene(n_side=(14, 16, 12))
    gpu = from_scene(sc)
    gpu.update(sc.dt)
    dims, org, keys, ids, start = gpu.grid()
    k2, i2, s2, esc = oracle_mod.grid_build(sc.positions, gpu.get_kernel_radius(), org, dims)
    assert esc == 0
    assert np.array_equal(keys, k2)
    assert np.array_equal(ids, i2)
    assert np.array_equal(start, s2)
    # Dense lower-bound table property.
    assert np.array_equal(start[:-1], np.searchsorted(keys, np.arange(start.size - 1), side="left"))
    assert start[-1] == sc.n
    gpu.close()


def _edge_scene(O, solver):
    """Particles at the edges of the neighbour search (SPHSpatialGrid.cpp:39-82): a block
    straddling the origin (negative cells, and cell 0, which spans (-h, h) under the
    truncating cell coordinate), particles exactly on cell faces and one ulp either side, and
    pairs whose distance lies within a few ulp of h in random directions. (Particles clamped
    into the border cells of a user grid box are covered by test_particles_outside_grid_box.)"""
    s = 0.02
    params = scenes._params(s, solver, pci_min_iterations=1, pci_max_iterations=4)
    block = scenes.lattice((-0.1, -0.08, -0.06), (10, 8, 7), s, 11)
    probe = O.OracleSolver(scenes.Scene("probe", params, block, np.zeros_like(block), [], 0.0005, 1))
    h = np.float32(probe.kernel_radius())
    probe.close()
    rng = np.random.default_rng(12)
    pts = [block]
    for k in range(-3, 4):
        f = np.float32(k) * h
        for v in (np.nextafter(f, np.float32(-1)), f, np.nextafter(f, np.float32(1))):
            p = rng.uniform(-0.09, 0.09, (3, 3)).astype(np.float32)
            for a in range(3):
                p[a, a] = v
            pts.append(p)
    base = rng.uniform(-0.09, 0.09, (120, 3)).astype(np.float32)
    d = rng.normal(size=(120, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.float64(h) * (1.0 + rng.integers(-3, 4, (120, 1)) * 2.0 ** -23)
    pts += [base, (base + d * r).astype(np.float32)]
    pos = np.concatenate(pts).astype(np.float32)
    cols = [scenes.Collider("box", (0.0, 0.0, 0.0), (0.3, 0.3, 0.3), True)]
    return scenes.Scene("search_edges", params, pos, np.zeros_like(pos), cols, 0.0005, 2, spacing=s), h


@pytest.mark.parametrize("solver", [abi.LSP_SOLVER_SPH, abi.LSP_SOLVER_PCISPH])
def test_neighbour_search_edges(oracle_mod, solver):
    sc, h = _edge_scene(oracle_mod, solver)
    gpu, orc = from_scene(sc), oracle_mod.OracleSolver(sc)
    fields = FIELDS_PCI if solver == abi.LSP_SOLVER_PCISPH else FIELDS_SPH
    try:
        for step in range(3):
            sg, so = gpu.update(sc.dt), orc.step(sc.dt)
            assert sg.iterations == so.iterations, step
            og, ig = gpu.neighbors()
            oo, io = orc.neighbors()
            assert np.array_equal(og, oo) and np.array_equal(ig, io), f"step {step}: neighbour lists differ"
            for f in fields:
                a, b = gpu.read(f), orc.get(f)
                assert bits_equal(a, b), f"step {step} field {f}: {mismatch_report(a, b)}"
            if step == 0:
                # The scene does reach the edges: accepted pairs of the first step's lists
                # whose squared distance lies within 2^-20 of h^2, and particles in cell 0
                # from both sides of the origin.
                assert (np.abs(sc.positions) < h).all(axis=1).sum() > 0
                assert (sc.positions < -h).all(axis=1).sum() > 0
                owner = np.repeat(np.arange(sc.n), np.diff(og))
                d2 = ((sc.positions[ig].astype(np.float64) - sc.positions[owner]) ** 2).sum(axis=1)
                assert (np.abs(d2 / np.float64(h) ** 2 - 1.0) < 2.0 ** -20).sum() > 0
    finally:
        gpu.close()
        orc.close()


def test_grid_build_with_many_scan_tiles(oracle_mod):
    """A grid box of 225^3 = 11.4M cells (5,563 scan tiles of 2,048 cells, more than the 4,096
    whose prefixes the apply kernel sums itself): the tile prefixes come from the separate
    top-level scan. Same keys, order and cell table as the specification, and the step
    matches the oracle."""
    sc = scenes.small_box_scene(n_side=(10, 12, 10))
    sc.domain = ((0.0, 0.0, 0.0), (9.0, 9.0, 9.0))
    gpu = from_scene(sc)
    orc = oracle_mod.OracleSolver(sc)
    gpu.update(sc.dt)
    orc.step(sc.dt)
    dims, org, keys, ids, start = gpu.grid()
    assert int(np.prod(dims.astype(np.int64))) > 4096 * 2048
    k2, i2, s2, esc = oracle_mod.grid_build(sc.positions, gpu.get_kernel_radius(), org, dims)
    assert esc == 0
    assert np.array_equal(keys, k2) and np.array_equal(ids, i2) and np.array_equal(start, s2)
    for f in (abi.FIELD_POSITION, abi.FIELD_DENSITY, abi.FIELD_PRESSURE):
        assert bits_equal(gpu.read(f), orc.get(f)), f
    gpu.close()
    orc.close()


@pytest.mark.parametrize("solver", [abi.LSP_SOLVER_SPH, abi.LSP_SOLVER_PCISPH])
def test_small_scene_bit_exact(oracle_mod, solver):
    sc = scenes.small_box_scene(solver=solver)
    gpu, orc = run_pair(oracle_mod, sc, 6)
    gpu.close()


def test_dam_break_sph_12k_bit_exact(oracle_mod):
    sc = scenes.dam_break_sph()
    gpu, orc = run_pair(oracle_mod, sc, 4, check_neighbors=True)
    gpu.close()


@pytest.mark.parametrize("loop_mode", [abi.LSP_LOOP_PERSISTENT, abi.LSP_LOOP_HOST])
def test_pcisph_min_max_iterations(oracle_mod, loop_mode):
    sc = scenes.small_box_scene(n_side=(12, 14, 12), pci_min_iterations=3, pci_max_iterations=50,
                                loop_mode=loop_mode)
    gpu, orc = run_pair(oracle_mod, sc, 4, check_neighbors=False)
    gpu.close()


@pytest.mark.parametrize("loop_mode", [abi.LSP_LOOP_PERSISTENT, abi.LSP_LOOP_HOST])
def test_pcisph_loop_modes_many_iterations(oracle_mod, loop_mode):
    """A tight tolerance forces long loops (the persistent kernel crosses many grid barriers)."""
    sc = scenes.small_box_scene(n_side=(16, 16, 16), pci_eta=1e-4, pci_min_iterations=1,
                                pci_max_iterations=40, loop_mode=loop_mode)
    gpu, orc = run_pair(oracle_mod, sc, 3, check_neighbors=False)
    st = gpu.update(sc.dt)
    assert st.iterations > 5
    gpu.close()


def test_negative_pressure_and_surface_tension(oracle_mod):
    sc = scenes.small_box_scene(negative_pressure_factor=0.4, surface_tension_threshold=0.5,
                                surface_tension=0.5)
    gpu, orc = run_pair(oracle_mod, sc, 5, check_neighbors=False)
    gpu.close()
    sc = scenes.small_box_scene(solver=abi.LSP_SOLVER_SPH, negative_pressure_factor=0.4,
                                surface_tension_threshold=0.5, surface_tension=0.5)
    gpu, orc = run_pair(oracle_mod, sc, 5, check_neighbors=False)
    gpu.close()


def test_boundary_sphere_and_keep_velocity(oracle_mod):
    sc = scenes.small_box_scene(keep_initial_velocity=1)
    sc.colliders.append(scenes.Collider("sphere", (0.3, 0.3, 0.3), 0.45, True))
    sc.velocities[:] = np.array([0.3, -0.2, 0.1], np.float32)
    gpu, orc = run_pair(oracle_mod, sc, 5, check_neighbors=False)
    gpu.close()


def test_initial_velocity_wipe(oracle_mod):
    sc = scenes.small_box_scene()
    sc.velocities[:] = np.array([1.0, 0.0, -0.5], np.float32)
    gpu, orc = run_pair(oracle_mod, sc, 3, check_neighbors=False)
    gpu.close()


def test_injected_state(oracle_mod):
    """Per-step parity from the same injected state (not a trajectory comparison)."""
    sc = scenes.small_box_scene(n_side=(10, 10, 10))
    gpu = from_scene(sc)
    orc = oracle_mod.OracleSolver(sc)
    rng = np.random.default_rng(11)
    n = sc.n
    x = sc.positions + rng.uniform(-0.004, 0.004, (n, 3)).astype(np.float32)
    v = rng.normal(0, 0.3, (n, 3)).astype(np.float32)
    h = rng.normal(0, 0.3, (n, 3)).astype(np.float32)
    o = rng.normal(0, 0.3, (n, 3)).astype(np.float32)
    first = (rng.uniform(size=n) < 0.3).astype(np.int32)
    gpu.write_state(x, v, h, o, first)
    orc.set_state(x, v, h, o, first)
    xs = gpu.read_state()
    for a, b in zip(xs[:4], (x, v, h, o)):
        assert bits_equal(a, b)
    assert np.array_equal(xs[4], first)
    for _ in range(3):
        sg, so = gpu.update(sc.dt), orc.step(sc.dt)
        assert sg.iterations == so.iterations
        for f in FIELDS_PCI:
            assert bits_equal(gpu.read(f), orc.get(f)), f"field {f}"
    gpu.close()


def test_speed_squared_field(oracle_mod):
    """The headless colour source: |v|^2 as Vector3D::squareMagnitude rounds it
    (Vector3D.cpp:55-58, read by SPHParticleDrawable.cpp:10-27), from the oracle's v."""
    sc = scenes.small_box_scene(n_side=(8, 8, 8))
    gpu, orc = run_pair(oracle_mod, sc, 3, check_neighbors=False)
    v = orc.get(abi.FIELD_VELOCITY).astype(np.float32)
    want = (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]
    assert bits_equal(gpu.read(abi.FIELD_SPEED_SQUARED), want)
    gpu.close()


def test_add_particles_mid_run_and_moving_collider(oracle_mod):
    sc = scenes.small_box_scene(n_side=(8, 8, 8))
    gpu = from_scene(sc)
    orc = oracle_mod.OracleSolver(sc)
    for s in range(6):
        if s == 2:
            extra = scenes.lattice((0.5, 0.5, 0.5), (5, 4, 6), 0.02, 99)
            vel = np.tile(np.array([[0.5, -1.0, 0.0]], np.float32), (extra.shape[0], 1))
            gpu.add_particles(extra, vel)
            orc.add_particles(extra, vel)
        if s == 3:
            gpu.update_static_collision_box(1, (0.5, 0.12, 0.35), (0.1, 0.12, 0.08))
            orc.update_box(1, (0.5, 0.12, 0.35), (0.1, 0.12, 0.08))
        sg, so = gpu.update(sc.dt), orc.step(sc.dt)
        assert sg.iterations == so.iterations
        for f in FIELDS_PCI:
            assert bits_equal(gpu.read(f), orc.get(f)), f"step {s} field {f}"
    gpu.close()


def test_neighbor_capacity_regrow(oracle_mod):
    """Particles packed 2.5x denser than the radius implies overflow the first neighbour
    capacity; the step is redone with a larger one and still matches."""
    s = 0.008
    pos = scenes.lattice((0.3, 0.3, 0.3), (12, 12, 12), s, 5)
    p = abi.default_params(particle_radius=0.02 / 1.6, kernel_radius_factor=3.2, rest_density=1000.0,
                           solver=abi.LSP_SOLVER_SPH, viscosity=0.1)
    sc = scenes.Scene("dense", p, pos, np.zeros_like(pos),
                      [scenes.Collider("box", (0.5, 0.5, 0.5), (0.5, 0.5, 0.5), True)], 0.0005, 2,
                      domain=((0, 0, 0), (1, 1, 1)))
    gpu, orc = run_pair(oracle_mod, sc, 2)
    st = gpu.update(sc.dt)
    assert st.max_neighbors > 100
    gpu.close()


def test_particles_outside_grid_box(oracle_mod):
    """A grid box smaller than the fluid: outside particles are clamped into edge cells.
    Neighbour sets and all per-particle results still match; only the order of an
    edge particle's list may differ, so sets are compared and fields to 1e-5 relative."""
    sc = scenes.small_box_scene(n_side=(10, 10, 10), solver=abi.LSP_SOLVER_SPH, obstacles=False)
    sc.domain = ((0.1, 0.1, 0.1), (0.2, 0.2, 0.2))
    gpu = from_scene(sc)
    orc = oracle_mod.OracleSolver(sc)
    st = gpu.update(sc.dt)
    orc.step(sc.dt)
    assert st.escaped > 0
    og, ig = gpu.neighbors()
    oo, io = orc.neighbors()
    assert np.array_equal(og, oo)
    for i in range(sc.n):
        assert sorted(ig[og[i]:og[i + 1]]) == sorted(io[oo[i]:oo[i + 1]])
    rho_g, rho_o = gpu.read(abi.FIELD_DENSITY), orc.get(abi.FIELD_DENSITY)
    assert np.allclose(rho_g, rho_o, rtol=1e-5, atol=0)
    gpu.close()


def test_empty_and_tiny_scenes(oracle_mod):
    sc = scenes.small_box_scene(n_side=(1, 1, 1))
    gpu, orc = run_pair(oracle_mod, sc, 3)
    gpu.close()
    sc2 = scenes.small_box_scene(n_side=(2, 1, 1))
    gpu, orc = run_pair(oracle_mod, sc2, 3)
    gpu.close()
    from liquidsimulation_b200.solver import PCISPHSolver
    s = PCISPHSolver()
    st = s.update(0.001)
    assert st.iterations == 0 and s.get_particle_count() == 0
    s.close()


def test_errors_are_reported():
    from liquidsimulation_b200.solver import PCISPHSolver
    s = PCISPHSolver()
    with pytest.raises(abi.LspError) as e:
        s.update(-1.0)
    assert e.value.code == abi.LSP_ERR_INVALID
    with pytest.raises(abi.LspError):
        s.set_params(particle_radius=-1.0)
    pos = np.array([[0.1, 0.1, 0.1], [np.nan, 0.2, 0.2]], np.float32)
    s.add_particles(pos)
    s.add_static_collision_box((0.5, 0.5, 0.5), (0.5, 0.5, 0.5), boundary=True)
    with pytest.raises(abi.LspError) as e:
        s.update(0.001)
    assert e.value.code == abi.LSP_ERR_DEVICE_STATUS
    s.close()


@pytest.mark.parametrize("loop_mode", [abi.LSP_LOOP_PERSISTENT, abi.LSP_LOOP_HOST])
def test_coincident_particles(oracle_mod, loop_mode):
    """Particles added twice at exactly the same position (and some offset along one axis
    only): their pressure-force direction is 0/0, so the reference's NaN reset zeroes the
    whole pressure force of those particles (PCISPHSolver.cpp:129-150), and coordinates that
    differ in one axis give exact zero components elsewhere. Every field must still match
    the oracle bit for bit."""
    import dataclasses
    sc = scenes.dam_break_pcisph(seed=9, counts=(10, 14, 10), s=0.02)
    sc.params.loop_mode = loop_mode
    rng = np.random.default_rng(9)
    pick = rng.choice(sc.n, 40, replace=False)
    twins = sc.positions[pick].copy()
    shifted = sc.positions[pick[:10]].copy()
    shifted[:, 1] += np.float32(0.001)
    pos = np.concatenate([sc.positions, twins, shifted]).astype(np.float32)
    sc = dataclasses.replace(sc, positions=pos, velocities=np.zeros_like(pos))
    gpu, orc = run_pair(oracle_mod, sc, steps=3)
    pf = gpu.read(abi.FIELD_PRED_PRESSURE_FORCE).reshape(-1, 3)
    assert np.all(pf[pick] == 0) and np.all(pf[sc.n - 50:sc.n - 10] == 0)
    gpu.close()
    orc.close()


def test_bounded_barrier_gives_up_and_device_stays_usable():
    """The persistent loops' grid barrier waits with a bounded spin: a round that cannot
    complete (fewer blocks than parties) ends with the timeout bit instead of a hang, only
    the block left waiting gives up, and the device keeps working afterwards."""
    import ctypes
    lib = abi.load_library()
    done, flags = ctypes.c_int32(), ctypes.c_uint32()
    timeout_bit = 4
    assert lib.lsp_barrier_probe(-1, 4, 4, ctypes.byref(done), ctypes.byref(flags)) == 0
    assert (done.value, flags.value & timeout_bit) == (4, 0)
    assert lib.lsp_barrier_probe(-1, 1, 2, ctypes.byref(done), ctypes.byref(flags)) == 0
    assert (done.value, flags.value & timeout_bit) == (0, timeout_bit)
    assert lib.lsp_barrier_probe(-1, 3, 2, ctypes.byref(done), ctypes.byref(flags)) == 0
    assert (done.value, flags.value & timeout_bit) == (2, timeout_bit)
    assert lib.lsp_barrier_probe(-1, 9, 2, ctypes.byref(done), ctypes.byref(flags)) == abi.LSP_ERR_INVALID
    sc = scenes.dam_break_pcisph(seed=3, counts=(8, 8, 8), s=0.02)
    s = from_scene(sc)
    assert s.update(sc.dt).iterations >= 1
    s.close()
