"""Generates the golden fixtures from the REFERENCE's own CPU solver.

Runs oracle/_ref/libref_sph.so (LiquidPhysics/src compiled unmodified by
oracle/Makefile, needs the reference sources at build time) on two small seeded
scenes and stores inputs and per-step outputs in tests/golden/*.npz:

  sph_small.npz     SPH, 8x9x8 block in a unit box with a box and a sphere obstacle
  pcisph_small.npz  PCISPH (eta 1 %, <= 8 iterations), same scene

Each file holds the scene's parameters, initial positions/velocities, colliders,
dt, and for each of 4 steps: positions, velocities, half velocities, densities,
pressures, PCISPH iteration counts, plus the neighbour lists of step 0.

    python tests/golden/make_golden.py
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


if __name__ == "__main__":
    ref_dir = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF_DIR")
    if not ref_dir:
        sys.exit("usage: make_golden.py REF_DIR (the reference checkout; or set REF_DIR)")
    O.build(ref_dir=ref_dir)
    for k in ("sph", "pcisph"):
        print(generate(k), os.path.getsize(os.path.join(HERE, f"{k}_small.npz")))
