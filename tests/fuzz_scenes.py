"""Seeded random scenes for the fuzz parity tests (test_fuzz_parity.py on the GPU,
test_oracle.py against the compiled reference)."""
import numpy as np

from liquidsimulation_b200 import abi, scenes


def random_scene(seed):
    rng = np.random.default_rng(seed)
    pci = bool(rng.integers(2))
    s = float(rng.uniform(0.015, 0.03))
    kw = dict(
        particle_radius=s / float(rng.uniform(1.4, 2.0)),
        kernel_radius_factor=float(rng.uniform(2.5, 4.0)),
        viscosity=float(rng.choice([0.0, 0.01, 0.1, 3.5])),
        stiffness=float(rng.uniform(1.0, 20.0)),
        negative_pressure_factor=float(rng.choice([0.0, 0.0, 0.3, 1.0])),
        surface_tension=float(rng.choice([0.0, 0.0728, 0.5])),
        surface_tension_threshold=float(rng.choice([0.5, 7.065, 50.0])),
        restitution=float(rng.uniform(0.0, 1.0)),
        friction=float(rng.uniform(0.0, 1.0)),
        gravity=tuple(float(g) for g in rng.normal(0.0, 5.0, 3)),
    )
    if pci:
        kw.update(pci_eta=float(rng.choice([0.005, 0.01, 0.05])), pci_min_iterations=int(rng.integers(1, 4)),
                  pci_max_iterations=int(rng.integers(3, 12)), keep_initial_velocity=int(rng.integers(2)))
    params = scenes._params(s, abi.LSP_SOLVER_PCISPH if pci else abi.LSP_SOLVER_SPH, **kw)
    counts = tuple(int(c) for c in rng.integers(5, 12, 3))
    lo = tuple(float(v) for v in rng.uniform(0.1, 0.4, 3))
    pos = scenes.lattice(lo, counts, s, int(rng.integers(1 << 30)))
    vel = rng.normal(0.0, 0.3, pos.shape).astype(np.float32) if rng.integers(2) else np.zeros_like(pos)
    if rng.integers(3) == 0:
        cols = [scenes.Collider("sphere", (0.5, 0.5, 0.5), 0.5, True)]
    else:
        cols = [scenes.Collider("box", (0.5, 0.5, 0.5), (0.5, 0.5, 0.5), True)]
    for _ in range(int(rng.integers(0, 3))):
        c = tuple(float(v) for v in rng.uniform(0.2, 0.8, 3))
        if rng.integers(2):
            cols.append(scenes.Collider("box", c, tuple(float(v) for v in rng.uniform(0.03, 0.1, 3)), False))
        else:
            cols.append(scenes.Collider("sphere", c, float(rng.uniform(0.03, 0.1)), False))
    domain = ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)) if rng.integers(2) else None
    dt = float(rng.choice([0.0005, 0.001, 0.002]))
    # Drawn last so the draws above stay those of earlier versions of this generator. Some
    # PCISPH scenes repeat a few particles at exactly the same position (0/0 pressure-force
    # directions, reset by the reference's NaN test); SPH has no such reset, so it gets none.
    if pci and rng.integers(4) == 0:
        dup = rng.choice(pos.shape[0], max(1, pos.shape[0] // 50), replace=False)
        pos = np.concatenate([pos, pos[dup]]).astype(np.float32)
        vel = np.concatenate([vel, vel[dup]]).astype(np.float32)
    return scenes.Scene(f"fuzz_{seed}", params, pos, vel, cols, dt, 3, domain=domain, spacing=s), pci
