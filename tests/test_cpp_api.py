"""The C++ solver API (include/lsp_solver.hpp) compiled against liblsp.so: a program that
drives PCISPHSolver like a reference application must reproduce the oracle bit for bit."""
import os
import subprocess

import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "liquidsimulation_b200")


def compile_program(tmp_path):
    exe = tmp_path / "solver_api"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "solver_api.cpp"), "-L", PKG, "-llsp",
                    f"-Wl,-rpath,{PKG}", "-o", str(exe)], check=True)
    return exe


def test_cpp_api_compiles(tmp_path):
    from liquidsimulation_b200 import build
    build.build()
    assert compile_program(tmp_path).exists()


@pytest.mark.gpu
def test_cpp_api_matches_oracle(tmp_path, oracle_mod):
    exe = compile_program(tmp_path)
    sc = scenes.small_box_scene(n_side=(9, 10, 9), obstacles=False)
    p = sc.params
    # The C++ program sets only these parameters; the rest keep the reference defaults.
    q = abi.default_params(solver=abi.LSP_SOLVER_PCISPH, particle_radius=p.particle_radius,
                           kernel_radius_factor=p.kernel_radius_factor, rest_density=p.rest_density,
                           viscosity=p.viscosity, pci_eta=p.pci_eta, pci_max_iterations=p.pci_max_iterations)
    steps = 4
    scene_file = tmp_path / "scene.bin"
    with open(scene_file, "wb") as f:
        np.array([sc.n, steps], np.int32).tofile(f)
        np.array([sc.dt, q.particle_radius, q.kernel_radius_factor, q.rest_density, q.viscosity, q.pci_eta],
                 np.float32).tofile(f)
        np.array([q.pci_max_iterations], np.int32).tofile(f)
        np.array([0.5, 0.5, 0.5, 0.5, 0.5, 0.5], np.float32).tofile(f)
        sc.positions.astype(np.float32).tofile(f)
    out = tmp_path / "out.bin"
    subprocess.run([str(exe), str(scene_file), str(out)], check=True)
    got = np.fromfile(out, np.float32)
    x, rho = got[: 3 * sc.n].reshape(-1, 3), got[3 * sc.n:]
    sc2 = scenes.Scene("cpp", q, sc.positions, np.zeros_like(sc.positions),
                       [scenes.Collider("box", (0.5, 0.5, 0.5), (0.5, 0.5, 0.5), True)], sc.dt, steps)
    orc = oracle_mod.OracleSolver(sc2)
    for _ in range(steps):
        orc.step(sc.dt)
    assert np.array_equal(x.view(np.uint32), orc.get(abi.FIELD_POSITION).view(np.uint32))
    assert np.array_equal(rho.view(np.uint32), orc.get(abi.FIELD_DENSITY).view(np.uint32))


def compile_batch_program(tmp_path):
    exe = tmp_path / "batch_api"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "batch_api.cpp"), "-L", PKG, "-llsp",
                    f"-Wl,-rpath,{PKG}", "-o", str(exe)], check=True)
    return exe


def test_cpp_batch_api_compiles(tmp_path):
    from liquidsimulation_b200 import build
    build.build()
    assert compile_batch_program(tmp_path).exists()


@pytest.mark.gpu
def test_cpp_batch_api_matches_single_scenes(tmp_path):
    """lsp::SceneBatch from C++ (autotuned first step) equals single-scene solvers bit for bit."""
    from liquidsimulation_b200.solver import from_scene
    exe = compile_batch_program(tmp_path)
    scs = scenes.batched_dam_breaks(seed=21, scenes=3, nmin=300, nmax=2000)
    steps = 3
    scene_file = tmp_path / "batch.bin"
    with open(scene_file, "wb") as f:
        np.array([len(scs), steps], np.int32).tofile(f)
        np.array([scs[0].dt], np.float32).tofile(f)
        for sc in scs:
            f.write(bytes(sc.params))
            np.array([sc.n], np.int32).tofile(f)
            np.array([0.5, 0.5, 0.5, 0.5, 0.5, 0.5], np.float32).tofile(f)
            sc.positions.astype(np.float32).tofile(f)
    out = tmp_path / "out.bin"
    subprocess.run([str(exe), str(scene_file), str(out)], check=True)
    got = np.fromfile(out, np.float32)
    off = 0
    for sc in scs:
        x = got[off: off + 3 * sc.n]
        rho = got[off + 3 * sc.n: off + 4 * sc.n]
        off += 4 * sc.n
        ref_scene = scenes.Scene("single", sc.params, sc.positions, np.zeros_like(sc.positions),
                                 [scenes.Collider("box", (0.5, 0.5, 0.5), (0.5, 0.5, 0.5), True)], sc.dt, steps)
        s = from_scene(ref_scene)
        for _ in range(steps):
            s.update(sc.dt)
        assert np.array_equal(x.view(np.uint32), s.read(abi.FIELD_POSITION).ravel().view(np.uint32))
        assert np.array_equal(rho.view(np.uint32), s.read(abi.FIELD_DENSITY).view(np.uint32))
        s.close()
    assert off == got.size
