"""Generates the golden fixtures from the REFERENCE's own CPU solver.

Runs oracle/_ref/libref_sph.so (LiquidPhysics/src compiled unmodified by
oracle/Makefile, needs the reference sources at build time) on two small seeded
scenes and stores inputs and per-step outputs in tests/golden/*.npz:

  sph_small.npz     SPH, 8x9x8 block in a unit box with a box and a sphere obstacle
  pcisph_small.npz  PCISPH (eta 1 %, <= 8 iterations), same scene

Each file holds the scene's parameters, initial positions/velocities, colliders,
dt, and for each of 4 steps: positions, velocities, half velocities, densities,
pressures, PCISPH iteration counts, plus the neighbour lists of step 0.

  wave_breaker_dt0008.npz  the wave breaker on the 0.01 m lattice (396,000 particles) at its
                           configured dt = 0.0008 with the reference's own iteration rule
                           (no minimum, at most 50, eta 1 %): per step, the iteration count
                           and the maximum |density error| (float32). It converges for 13 steps
                           and runs to the 50-iteration bound with a 65 % error at step 13.

    python tests/golden/make_golden.py REF_DIR [sph pcisph divergence]
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from liquidsimulation_b200 import abi, scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402

STEPS = 4


def scene(kind):
    solver = abi.LSP_SOLVER_PCISPH if kind == "pcisph" else abi.LSP_SOLVER_SPH
    return scenes.small_box_scene(n_side=(8, 9, 8), solver=solver, seed=21)


def generate(kind):
    sc = scene(kind)
    ref = O.RefSolver(sc, capture_neighbors=True)
    out = {"positions0": sc.positions, "velocities0": sc.velocities, "dt": np.float32(sc.dt),
           "params": json.dumps(abi.params_dict(sc.params)),
           "colliders": json.dumps([[c.kind, list(c.center), c.size if c.kind == "sphere" else list(c.size),
                                     c.boundary] for c in sc.colliders])}
    its = []
    for s in range(STEPS):
        its.append(ref.step(sc.dt))
        for name, f in (("x", abi.FIELD_POSITION), ("v", abi.FIELD_VELOCITY), ("half", abi.FIELD_HALF_VELOCITY),
                        ("rho", abi.FIELD_DENSITY), ("p", abi.FIELD_PRESSURE)):
            out[f"{name}_{s}"] = ref.get(f)
        if s == 0:
            off, idx = ref.neighbors()
            out["nbr_offsets_0"] = off.astype(np.int32)
            out["nbr_index_0"] = idx.astype(np.int32)
    out["iterations"] = np.array(its, np.int32)
    path = os.path.join(HERE, f"{kind}_small.npz")
    np.savez_compressed(path, **out)
    return path


DIVERGENCE_STEPS = 15


def divergence_scene():
    sc = scenes.wave_breaker(seed=3, s=0.01, dt=0.0008)
    sc.params.pci_min_iterations = 1          # the reference's loop has no minimum
    return sc


def generate_divergence():
    sc = divergence_scene()
    ref = O.RefSolver(sc)
    its, errs = [], []
    for _ in range(DIVERGENCE_STEPS):
        its.append(ref.step(sc.dt))
        errs.append(np.float32(np.max(np.abs(ref.get(abi.FIELD_DENSITY_ERROR)))))
        print(len(its) - 1, its[-1], errs[-1] / sc.params.rest_density, flush=True)
    path = os.path.join(HERE, "wave_breaker_dt0008.npz")
    np.savez_compressed(path, iterations=np.array(its, np.int32), max_abs_error=np.array(errs, np.float32),
                        n=np.int64(sc.n), dt=np.float32(sc.dt))
    return path


if __name__ == "__main__":
    ref_dir = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF_DIR")
    if not ref_dir:
        sys.exit("usage: make_golden.py REF_DIR (the reference checkout; or set REF_DIR)")
    O.build(ref_dir=ref_dir)
    kinds = sys.argv[2:] or ["sph", "pcisph", "divergence"]
    for k in kinds:
        path = generate_divergence() if k == "divergence" else generate(k)
        print(path, os.path.getsize(path))
