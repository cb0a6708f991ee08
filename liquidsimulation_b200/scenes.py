"""Seeded synthetic scenes: the dam-break, wave-breaker, batched and waterfall workloads.

The reference ships no scene files or datasets; its demo builds scenes in code
(LiquidSimulation/src/Scenarios/*.cpp) with a lattice emitter
(LiquidPhysics/src/Particles/SPHParticleEmitter.cpp). These generators stand in
for them with seeded lattices: lattice point (i, j, k) sits at
``lo + (i + 0.5) * s`` and is jittered uniformly by +-1 % of the spacing per axis,
drawn from ``numpy.random.Generator(PCG64(seed))`` in x, y, z order per particle.
Particles are emitted x-fastest (i inner, then j, then k). Blocks that rest against
the walls start one particle radius plus the jitter amplitude from each wall
(``wall_lattice``), so their first layer is not moved by the first collision pass.

Particle radius is ``s / 1.6`` (the emitter's spacing is 1.6 radii,
SPHParticleEmitter.cpp) and the smoothing length ``h = 2 s``, i.e. a kernel-radius
factor of 3.2. Mass is the reference's derived mass
(SPHSolver::recalcParticleMass, SPHSolver.cpp:480-507) unless a workload fixes it.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import abi


@dataclasses.dataclass
class Collider:
    kind: str            # "box" or "sphere"
    center: tuple
    size: object         # half extents (box) or radius (sphere)
    boundary: bool


@dataclasses.dataclass
class Scene:
    name: str
    params: abi.LspParams
    positions: np.ndarray          # float32 [N, 3], caller order
    velocities: np.ndarray         # float32 [N, 3]
    colliders: list
    dt: float
    steps: int
    domain: tuple | None = None    # (lo[3], hi[3]) grid box, or None
    spacing: float = 0.0

    @property
    def n(self) -> int:
        return int(self.positions.shape[0])


def lattice(lo, counts, s, seed, jitter=0.01, rng=None, first=None):
    """Jittered lattice: counts=(nx, ny, nz) points at lo + (idx + 0.5) * s, x fastest, or at
    first + idx * s when ``first`` (the first point per axis) is given."""
    nx, ny, nz = (int(c) for c in counts)
    rng = rng if rng is not None else np.random.Generator(np.random.PCG64(seed))
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    base = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64)
    if first is not None:
        pts = np.asarray(first, np.float64)[None, :] + base * s
    else:
        pts = np.asarray(lo, np.float64)[None, :] + (base + 0.5) * s
    pts += rng.uniform(-jitter * s, jitter * s, size=pts.shape)
    return pts.astype(np.float32)


def wall_lattice(lo, counts, s, seed, rng=None, hi=None):
    """A block resting in a corner of the walls at ``lo`` (walls up to ``hi``, if given: the
    block is clipped to fit them): its first layer sits one particle
    radius (s / 1.6) plus the jitter amplitude from each wall, so the boundary collision
    (which keeps particles r inside, StaticCollisionBox.cpp:77-114) does not move it. A
    block starting at lo + s/2 would have its first layer pinned 1/8 spacing inward by the
    first collision pass, which compresses the corner by ~20 % and makes the reference's
    PCISPH loop run to its iteration cap."""
    off = s / 1.6 + 0.01 * s
    first = tuple(float(l) + off for l in lo)
    if hi is not None:
        # Layers that would fall inside the far walls' margin are dropped.
        counts = [min(int(c), int(math.floor((float(u) - off - f) / s + 1e-9)) + 1)
                  for c, f, u in zip(counts, first, hi)]
    return lattice(lo, counts, s, seed, rng=rng, first=first)


def _params(s, solver, **kw):
    base = dict(
        particle_radius=s / 1.6,
        kernel_radius_factor=3.2,
        rest_density=1000.0,
        viscosity=0.1,
        stiffness=3.0,
        negative_pressure_factor=0.0,
        surface_tension=0.0728,
        surface_tension_threshold=7.065,
        restitution=0.5,
        friction=1.0,
        gravity=(0.0, -9.81, 0.0),
        solver=solver,
    )
    base.update(kw)
    return abi.default_params(**base)


def dam_break_sph(seed: int = 1, scale: float = 1.0) -> Scene:
    """Plain SPH dam break: unit box walls, 20x30x20 block at s = 0.02 (12,000 particles),
    mass 0.008, h = 0.04, k = 3, mu = 0.1, dt = 0.002. ``scale`` < 1 shrinks the block."""
    s = 0.02
    counts = [max(2, int(round(c * scale))) for c in (20, 30, 20)]
    pos = wall_lattice((0.0, 0.0, 0.0), counts, s, seed, hi=(1.0, 1.0, 1.0))
    p = _params(s, abi.LSP_SOLVER_SPH, mass_override=0.008)
    box = Collider("box", (0.5, 0.5, 0.5), (0.5, 0.5, 0.5), True)
    return Scene("dam_break_sph_12k", p, pos, np.zeros_like(pos), [box], 0.002, 1000,
                 domain=((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)), spacing=s)


def dam_break_pcisph(seed: int = 2, counts=(64, 102, 64), s: float = 0.00625) -> Scene:
    """PCISPH dam break: unit box walls, 64x102x64 block at s = 0.00625 (417,792 particles),
    h = 2 s, eta = 1 %, min 3 / max 50 iterations, zero initial pressure, dt = 0.001."""
    pos = wall_lattice((0.0, 0.0, 0.0), counts, s, seed, hi=(1.0, 1.0, 1.0))
    p = _params(s, abi.LSP_SOLVER_PCISPH, pci_eta=0.01, pci_min_iterations=3, pci_max_iterations=50)
    box = Collider("box", (0.5, 0.5, 0.5), (0.5, 0.5, 0.5), True)
    n = pos.shape[0]
    return Scene(f"dam_break_pcisph_{n}", p, pos, np.zeros_like(pos), [box], 0.001, 2000,
                 domain=((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)), spacing=s)


def wave_breaker(seed: int = 3, s: float = 0.00735, block=(0.8, 0.5, 1.0), dt: float = 0.0004) -> Scene:
    """PCISPH wave breaker, ~1M particles: 2x1x1 walls, block [0,0.8]x[0,0.5]x[0,1] at
    s = 0.00735 (108x68x135 = 991,440 particles: the block spans the full depth, so one
    layer is dropped to clear the far wall's margin); two 0.2x0.3x0.2 box obstacles and a
    r = 0.15 sphere obstacle resting on the floor at seeded x in [1, 1.8]; eta = 1 %,
    min 3 / max 50, dt = 0.0004. At dt = 0.0008 the reference's own PCISPH (zero initial
    pressure each step) diverges at step 11 on this lattice, and on the 0.01 m lattice as
    well: the loop cannot rebuild the 0.5 m column's hydrostatic pressure to 1 %."""
    rng = np.random.Generator(np.random.PCG64(seed))
    counts = [int(math.floor(b / s + 1e-9)) for b in block]
    pos = wall_lattice((0.0, 0.0, 0.0), counts, s, seed, rng=rng, hi=(2.0, 1.0, 1.0))
    p = _params(s, abi.LSP_SOLVER_PCISPH, pci_eta=0.01, pci_min_iterations=3, pci_max_iterations=50)
    cols = [Collider("box", (1.0, 0.5, 0.5), (1.0, 0.5, 0.5), True)]
    for _ in range(2):
        cx = float(rng.uniform(1.1, 1.7))
        cz = float(rng.uniform(0.15, 0.85))
        cols.append(Collider("box", (cx, 0.15, cz), (0.1, 0.15, 0.1), False))
    cx = float(rng.uniform(1.15, 1.65))
    cz = float(rng.uniform(0.2, 0.8))
    cols.append(Collider("sphere", (cx, 0.15, cz), 0.15, False))
    return Scene(f"wave_breaker_{pos.shape[0]}", p, pos, np.zeros_like(pos), cols, dt, 3000,
                 domain=((0.0, 0.0, 0.0), (2.0, 1.0, 1.0)), spacing=s)


def batched_dam_breaks(seed: int = 4, scenes: int = 64, nmin: int = 2000, nmax: int = 64000):
    """64 independent PCISPH dam breaks: N log-uniform in [2000, 64000], block edges uniform
    in [0.2, 0.6], spacing (V_block / N)^(1/3), unit box walls, eta = 1 %, dt = 0.001."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for b in range(scenes):
        n_target = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
        edges = rng.uniform(0.2, 0.6, size=3)
        s = float((np.prod(edges) / n_target) ** (1.0 / 3.0))
        counts = [max(2, int(e / s)) for e in edges]
        pos = wall_lattice((0.0, 0.0, 0.0), counts, s, int(rng.integers(1 << 30)), hi=(1.0, 1.0, 1.0))
        p = _params(s, abi.LSP_SOLVER_PCISPH, pci_eta=0.01, pci_min_iterations=3, pci_max_iterations=50)
        box = Collider("box", (0.5, 0.5, 0.5), (0.5, 0.5, 0.5), True)
        out.append(Scene(f"batch_{b}", p, pos, np.zeros_like(pos), [box], 0.001, 100,
                         domain=((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)), spacing=s))
    return out


def waterfall_sheet(step: int, seed: int = 5, s: float = 0.008, nx: int = 40, ny: int = 50):
    """One emitted sheet of the waterfall: a 40x50 lattice in the y-z plane at the ledge lip
    (x = 0.02), spacing 0.008, velocity 1.5 m/s along +x, jittered +-1 % from (seed, step)."""
    rng = np.random.Generator(np.random.PCG64([seed, step]))
    j, k = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    y = 0.55 + (j.ravel() + 0.5) * s
    z = 0.3 + (k.ravel() + 0.5) * s
    pos = np.stack([np.full_like(y, 0.02), y, z], axis=1)
    pos += rng.uniform(-0.01 * s, 0.01 * s, size=pos.shape)
    vel = np.zeros_like(pos)
    vel[:, 0] = 1.5
    return pos.astype(np.float32), vel.astype(np.float32)


def waterfall(seed: int = 5, s: float = 0.008) -> Scene:
    """Waterfall: 2x2x1 walls, a 0.5 m-high ledge box the sheets fall from, PCISPH eta = 1 %,
    dt = 0.0005; the scene starts empty and the caller appends waterfall_sheet(step)."""
    p = _params(s, abi.LSP_SOLVER_PCISPH, pci_eta=0.01, pci_min_iterations=3, pci_max_iterations=50,
                keep_initial_velocity=1)
    cols = [Collider("box", (1.0, 1.0, 0.5), (1.0, 1.0, 0.5), True),
            Collider("box", (0.25, 0.25, 0.5), (0.25, 0.25, 0.5), False)]
    empty = np.zeros((0, 3), np.float32)
    return Scene("waterfall", p, empty, empty.copy(), cols, 0.0005, 0,
                 domain=((0.0, 0.0, 0.0), (2.0, 2.0, 1.0)), spacing=s)


def small_box_scene(n_side=(10, 12, 10), s=0.02, solver=abi.LSP_SOLVER_PCISPH, seed=7, obstacles=True,
                    **param_overrides) -> Scene:
    """A small test scene: a block in a unit box with a box and a sphere obstacle, of
    either solver; used by the parity tests at sizes the oracle finishes in seconds."""
    pos = lattice((0.05, 0.05, 0.05), n_side, s, seed)
    kw = dict(pci_eta=0.01, pci_min_iterations=1, pci_max_iterations=8) if solver == abi.LSP_SOLVER_PCISPH else {}
    kw.update(param_overrides)
    p = _params(s, solver, **kw)
    cols = [Collider("box", (0.5, 0.5, 0.5), (0.5, 0.5, 0.5), True)]
    if obstacles:
        cols.append(Collider("box", (0.55, 0.1, 0.3), (0.08, 0.1, 0.08), False))
        cols.append(Collider("sphere", (0.3, 0.08, 0.6), 0.1, False))
    return Scene("small_box", p, pos, np.zeros_like(pos), cols, 0.002, 10,
                 domain=((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)), spacing=s)
