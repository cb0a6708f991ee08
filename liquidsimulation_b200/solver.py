"""Python mirror of the reference solver API over the C ABI (liblsp.so).

``SPHSolver`` and ``PCISPHSolver`` keep the method set of LiquidPhysics'
``LiPhEn::SPHSolver`` (LiquidPhysics/include/SPHSolver.h:25-168) and
``LiPhEn::PCISPHSolver`` (PCISPHSolver.h:7-44) in snake_case: scene setup
(particles, static collision boxes/spheres), parameter setters/getters, one
``update(dt)`` per step (PhysicSolver::update, PhysicSolver.h:10) and particle
read-back. Arrays are numpy, in caller order. There is no CPU fallback: without
``liblsp.so`` or a B200 the constructor raises.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, byref, c_float, c_int32, c_int64, c_uint32

import numpy as np

from . import abi

_fp = POINTER(c_float)


def _f32(a, shape_last=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a


def _ptr(a, typ=_fp):
    return a.ctypes.data_as(typ) if a is not None else None


class SPHSolver:
    """LiPhEn::SPHSolver on the GPU (ParallelizationType extended with CUDA)."""

    SOLVER = abi.LSP_SOLVER_SPH

    def __init__(self, params: abi.LspParams | None = None, device: int = -1, **overrides):
        self._lib = abi.load_library()
        p = params if params is not None else abi.default_params()
        p = abi.default_params(**{**abi.params_dict(p), **overrides})
        p.solver = self.SOLVER
        h = ctypes.c_void_p()
        abi.check(self._lib, self._lib.lsp_create(byref(p), device, byref(h)))
        self._h = h
        self._colliders = []

    # ------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.lsp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _call(self, name, *args):
        return abi.check(self._lib, getattr(self._lib, name)(self._h, *args))

    # ------------------------------------------------------------ parameters
    @property
    def params(self) -> abi.LspParams:
        p = abi.LspParams()
        self._call("lsp_get_params", byref(p))
        return p

    def set_params(self, **fields):
        """Changes parameters by field name; on an error the solver keeps the previous ones."""
        p = self.params
        for k, v in fields.items():
            if k == "gravity":
                p.gravity[:] = tuple(v)
            else:
                setattr(p, k, v)
        self._call("lsp_set_params", byref(p))

    # Setters / getters of SPHSolver.h:79-109.
    def set_gravity(self, g): self.set_params(gravity=g)
    def set_particle_radius(self, r): self.set_params(particle_radius=r)
    def set_kernel_radius_factor(self, f): self.set_params(kernel_radius_factor=f)
    def set_rest_density(self, rho0): self.set_params(rest_density=rho0)
    def set_viscosity_coefficient(self, mu): self.set_params(viscosity=mu)
    def set_pressure_stiffness_coefficient(self, k): self.set_params(stiffness=k)
    def set_negative_pressure_factor(self, f): self.set_params(negative_pressure_factor=f)
    def set_surface_tension_coefficient(self, s): self.set_params(surface_tension=s)
    def set_surface_tension_threshold(self, t): self.set_params(surface_tension_threshold=t)
    def set_restitution_coefficient(self, e): self.set_params(restitution=e)
    def set_friction_coefficient(self, f): self.set_params(friction=f)

    def set_has_collision_object_data_changed(self, changed: bool = True):
        """Colliders are re-uploaded whenever changed through this API; kept for parity."""

    def get_gravity(self): return tuple(self.params.gravity)
    def get_particle_radius(self): return self.params.particle_radius
    def get_kernel_radius_factor(self): return self.params.kernel_radius_factor
    def get_rest_density(self): return self.params.rest_density
    def get_viscosity_coefficient(self): return self.params.viscosity
    def get_pressure_stiffness_coefficient(self): return self.params.stiffness
    def get_negative_pressure_factor(self): return self.params.negative_pressure_factor
    def get_surface_tension_coefficient(self): return self.params.surface_tension
    def get_surface_tension_threshold(self): return self.params.surface_tension_threshold
    def get_restitution_coefficient(self): return self.params.restitution
    def get_friction_coefficient(self): return self.params.friction

    def get_particle_mass(self) -> float:
        m = c_float()
        self._call("lsp_particle_mass", byref(m))
        return m.value

    def get_kernel_radius(self) -> float:
        h = c_float()
        self._call("lsp_kernel_radius", byref(h))
        return h.value

    def get_particle_count(self) -> int:
        n = c_int64()
        self._call("lsp_particle_count", byref(n))
        return n.value

    def kernel_tables(self) -> np.ndarray:
        out = np.empty(5 * abi.TABLE_SIZE, np.float32)
        self._call("lsp_kernel_tables", _ptr(out), out.size)
        return out.reshape(5, abi.TABLE_SIZE)

    # ------------------------------------------------------------ scene
    def add_particles(self, positions, velocities=None):
        """SPHSolver::addParticle for each row (SPHSolver.cpp:129-135)."""
        pos = _f32(positions).reshape(-1, 3)
        vel = None if velocities is None else _f32(velocities).reshape(-1, 3)
        if vel is not None and vel.shape != pos.shape:
            raise ValueError("velocities must match positions")
        self._call("lsp_add_particles", _ptr(pos), _ptr(vel), pos.shape[0])

    def add_particle(self, position, velocity=None):
        self.add_particles(np.asarray(position, np.float32)[None, :],
                           None if velocity is None else np.asarray(velocity, np.float32)[None, :])

    def remove_particles(self):
        self._call("lsp_remove_particles")

    def add_static_collision_box(self, center, half_extent, boundary: bool = False) -> int:
        c = _f32(center)
        h = _f32(half_extent)
        self._call("lsp_add_box", _ptr(c), _ptr(h), abi.LSP_BOUNDARY if boundary else abi.LSP_OBSTACLE)
        self._colliders.append("box")
        return len(self._colliders) - 1

    def add_static_collision_sphere(self, center, radius: float, boundary: bool = False) -> int:
        c = _f32(center)
        self._call("lsp_add_sphere", _ptr(c), float(radius), abi.LSP_BOUNDARY if boundary else abi.LSP_OBSTACLE)
        self._colliders.append("sphere")
        return len(self._colliders) - 1

    def add_static_collision_object(self, collider) -> int:
        """Takes a scenes.Collider (kind 'box' or 'sphere')."""
        if collider.kind == "box":
            return self.add_static_collision_box(collider.center, collider.size, collider.boundary)
        return self.add_static_collision_sphere(collider.center, collider.size, collider.boundary)

    def update_static_collision_box(self, index, center, half_extent):
        self._call("lsp_update_box", int(index), _ptr(_f32(center)), _ptr(_f32(half_extent)))

    def update_static_collision_sphere(self, index, center, radius):
        self._call("lsp_update_sphere", int(index), _ptr(_f32(center)), float(radius))

    def remove_static_collision_objects(self):
        self._call("lsp_remove_colliders")
        self._colliders = []

    def clean_up(self):
        """SPHSolver::cleanUp (SPHSolver.cpp:180-184)."""
        self.remove_particles()
        self.remove_static_collision_objects()

    def set_domain(self, lo, hi):
        self._call("lsp_set_domain", _ptr(_f32(lo)), _ptr(_f32(hi)))

    # ------------------------------------------------------------ stepping
    def update(self, dt: float) -> abi.LspStepStats:
        """PhysicSolver::update (PhysicSolver.cpp:12-21)."""
        st = abi.LspStepStats()
        self._call("lsp_step", c_float(dt), byref(st))
        return st

    def step_many(self, dt: float, steps: int) -> abi.LspStepStats:
        st = abi.LspStepStats()
        self._call("lsp_step_many", c_float(dt), int(steps), byref(st))
        return st

    def synchronize(self):
        self._call("lsp_synchronize")

    # ------------------------------------------------------------ read-back
    def read(self, field: int) -> np.ndarray:
        n = self.get_particle_count()
        shape = (n, 3) if field in abi.VECTOR_FIELDS else (n,)
        out = np.empty(shape, np.float32)
        self._call("lsp_read_field", int(field), _ptr(out), n)
        return out

    def positions(self) -> np.ndarray:
        return self.read(abi.FIELD_POSITION)

    def velocities(self) -> np.ndarray:
        return self.read(abi.FIELD_VELOCITY)

    def read_state(self):
        n = self.get_particle_count()
        x, v, h, o = (np.empty((n, 3), np.float32) for _ in range(4))
        first = np.empty(n, np.int32)
        self._call("lsp_read_state", _ptr(x), _ptr(v), _ptr(h), _ptr(o), _ptr(first, POINTER(c_int32)), n)
        return x, v, h, o, first

    def write_state(self, x, v, half, old_half, first):
        n = self.get_particle_count()
        arrs = [_f32(a).reshape(n, 3) for a in (x, v, half, old_half)]
        f = np.ascontiguousarray(first, np.int32).reshape(n)
        self._call("lsp_write_state", *(_ptr(a) for a in arrs), _ptr(f, POINTER(c_int32)), n)

    def save_state(self, path: str, seed: int = 0):
        """Writes the scene and its state to a file (lsp_save_state)."""
        self._call("lsp_save_state", str(path).encode(), ctypes.c_uint64(seed))

    def load_state(self, path: str):
        """Replaces parameters, particles, colliders and grid box from a file (lsp_load_state)."""
        self._call("lsp_load_state", str(path).encode())
        self._colliders = []

    def neighbors(self):
        """Start-of-step neighbour lists of the last step: (offsets[n+1], caller ids)."""
        n = self.get_particle_count()
        off = np.empty(n + 1, np.int64)
        self._call("lsp_read_neighbors", _ptr(off, POINTER(c_int64)), None, n, 0)
        idx = np.empty(max(int(off[-1]), 1), np.int32)
        self._call("lsp_read_neighbors", _ptr(off, POINTER(c_int64)), _ptr(idx, POINTER(c_int32)), n, idx.size)
        return off, idx[: int(off[-1])]

    # ------------------------------------------------------------ learned warm start
    def mlp_reset(self, seed: int = 0):
        self._call("lsp_mlp_reset", ctypes.c_uint64(seed))

    def mlp_set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32).reshape(-1)
        self._call("lsp_mlp_set_weights", _ptr(w), w.size)

    def mlp_get_weights(self) -> np.ndarray:
        w = np.empty(abi.MLP_PARAMS, np.float32)
        self._call("lsp_mlp_get_weights", _ptr(w), w.size)
        return w

    def mlp_record(self, on: bool = True):
        self._call("lsp_mlp_record", 1 if on else 0)

    def mlp_set_loss_asymmetry(self, over_weight: float):
        self._call("lsp_mlp_set_loss_asymmetry", c_float(over_weight))

    def mlp_train(self, iterations: int = 4, batch: int = 65536, lr: float = 1e-3, seed: int = 0) -> float:
        """Adam steps on the last recorded step (features -> final pressure); returns the loss."""
        loss = c_float()
        self._call("lsp_mlp_train", int(iterations), int(batch), c_float(lr), ctypes.c_uint64(seed), byref(loss))
        return loss.value

    def mlp_forward(self, features) -> np.ndarray:
        x = np.ascontiguousarray(features, np.float32).reshape(-1, abi.MLP_FEATURES)
        out = np.empty(x.shape[0], np.float32)
        self._call("lsp_mlp_forward", _ptr(x), x.shape[0], _ptr(out))
        return out

    def read_features(self) -> np.ndarray:
        n = self.get_particle_count()
        out = np.empty((n, abi.MLP_FEATURES), np.float32)
        self._call("lsp_read_features", _ptr(out), n)
        return out

    def set_warm_start(self, mode: int):
        """params.warm_start alone (lsp_set_warm_start: no table rebuild)."""
        self._call("lsp_set_warm_start", int(mode))

    def grid_cells(self) -> int:
        """Cells of the grid box of the last step (the dense cell table has one entry more)."""
        dims = np.empty(3, np.int32)
        org = np.empty(3, np.int32)
        cells = c_int64()
        self._call("lsp_grid_info", _ptr(dims, POINTER(c_int32)), _ptr(org, POINTER(c_int32)), byref(cells))
        return int(cells.value)

    def grid(self):
        """(dims, origin, sorted keys, sorted caller ids, dense cell table) of the last step."""
        n = self.get_particle_count()
        dims = np.empty(3, np.int32)
        org = np.empty(3, np.int32)
        cells = c_int64()
        self._call("lsp_grid_info", _ptr(dims, POINTER(c_int32)), _ptr(org, POINTER(c_int32)), byref(cells))
        keys = np.empty(max(n, 1), np.uint32)
        ids = np.empty(max(n, 1), np.int32)
        start = np.empty(cells.value + 1, np.uint32)
        self._call("lsp_read_grid", _ptr(keys, POINTER(c_uint32)), _ptr(ids, POINTER(c_int32)), n,
                   _ptr(start, POINTER(c_uint32)), cells.value + 1)
        return dims, org, keys[:n], ids[:n], start


class PCISPHSolver(SPHSolver):
    """LiPhEn::PCISPHSolver on the GPU."""

    SOLVER = abi.LSP_SOLVER_PCISPH

    def set_min_iterations(self, n: int):
        """PCISPHSolver::setMinIterations (PCISPHSolver.cpp:342-345). The reference's loop runs
        at most this many iterations (PCISPHSolver.cpp:64), so it sets pci_max_iterations."""
        self.set_params(pci_max_iterations=int(n))

    def get_min_iterations(self) -> int:
        return self.params.pci_max_iterations

    def set_max_density_error_ratio(self, eta: float):
        self.set_params(pci_eta=float(eta))

    def get_max_density_error_ratio(self) -> float:
        return self.params.pci_eta

    def set_minimum_iteration_floor(self, n: int):
        """Extension: no convergence exit before n iterations (the reference has none)."""
        self.set_params(pci_min_iterations=int(n))


class OnlineWarmStart:
    """Learned warm start retrained online, with the reference's zero start as fallback.

    Drives one PCISPH solver step by step. A training step runs the plain solver (zero
    initial pressure, PCISPHSolver.cpp:58-62) with its features recorded and, if it met eta,
    takes `iterations` Adam steps on its final pressures: the first `lead` steps, then every
    `every`-th step. Every other step starts from the network's guess (LSP_WARM_MLP), once the
    network has been trained at least once; a warm step that misses eta switches the solver
    back to the zero start until the next training step (the fallback). The network never
    trains on warm-started outputs. A scene that grows (particles appended between steps)
    is handled: features are recorded per step."""

    def __init__(self, solver, every: int = 500, lead: int = 50, iterations: int = 8, batch: int = 65536,
                 lr: float = 2e-3, loss_asymmetry: float = 4.0):
        if every < 1 or lead < 0:
            raise ValueError("every must be >= 1 and lead >= 0")
        self.s = solver
        self.every, self.lead, self.iterations, self.batch, self.lr = every, lead, iterations, batch, lr
        self.k = 0
        self.trained_steps = 0
        self.training_steps = 0
        self.fallback_steps = 0
        self.warm_steps = 0
        self._healthy = True
        solver.mlp_set_loss_asymmetry(loss_asymmetry)
        solver.set_warm_start(abi.LSP_WARM_ZERO)

    def _mode(self, mode):
        if self.s.params.warm_start != mode:
            self.s.set_warm_start(mode)

    def is_training_step(self, k: int) -> bool:
        return k < self.lead or (k - self.lead) % self.every == self.every - 1

    def update(self, dt: float) -> abi.LspStepStats:
        k = self.k
        self.k += 1
        s = self.s
        if self.is_training_step(k):
            self._mode(abi.LSP_WARM_ZERO)
            s.mlp_record(True)
            st = s.update(dt)
            s.mlp_record(False)
            self.training_steps += 1
            eta = s.params.pci_eta
            if st.converged and st.max_density_error_ratio <= eta + 1e-12:
                s.mlp_train(iterations=self.iterations, batch=self.batch, lr=self.lr, seed=k)
                self.trained_steps += 1
            self._healthy = True
            return st
        warm = self.trained_steps > 0 and self._healthy
        self._mode(abi.LSP_WARM_MLP if warm else abi.LSP_WARM_ZERO)
        st = s.update(dt)
        if warm:
            self.warm_steps += 1
            if not st.converged:
                self._healthy = False
        else:
            self.fallback_steps += 1
        return st


def state_file_info(path: str) -> dict:
    """Header of a state file (no device needed): params, particle count, colliders, seed."""
    lib = abi.load_library()
    p = abi.LspParams()
    n = c_int64()
    cols = c_int32()
    seed = ctypes.c_uint64()
    abi.check(lib, lib.lsp_state_file_info(str(path).encode(), byref(p), byref(n), byref(cols), byref(seed)))
    return {"params": p, "n": n.value, "colliders": cols.value, "seed": seed.value}


def from_scene(scene, device: int = -1) -> SPHSolver:
    """Builds a solver for a scenes.Scene: parameters, particles, colliders, grid box."""
    cls = PCISPHSolver if scene.params.solver == abi.LSP_SOLVER_PCISPH else SPHSolver
    s = cls(scene.params, device=device)
    if scene.domain is not None:
        s.set_domain(*scene.domain)
    if scene.n:
        s.add_particles(scene.positions, scene.velocities)
    for c in scene.colliders:
        s.add_static_collision_object(c)
    return s


class SceneBatch:
    """Many independent scenes stepped together (lsp_batch_* in include/lsp.h).

    The reference runs one solver object per scene; a batch holds them all in one set of
    device arrays and advances every scene with one CUDA graph per step, the PCISPH loops of
    all scenes in one persistent kernel. Each scene's results are bit-identical to a
    single-scene solver given the same inputs. Scenes and colliders are added before the
    first step."""

    def __init__(self, device: int = -1):
        self._lib = abi.load_library()
        h = ctypes.c_void_p()
        abi.check(self._lib, self._lib.lsp_batch_create(device, byref(h)))
        self._h = h
        self._counts = []

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.lsp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _call(self, name, *args):
        return abi.check(self._lib, getattr(self._lib, name)(self._h, *args))

    # ------------------------------------------------------------ scenes
    def add_scene(self, params: abi.LspParams, positions, velocities=None, domain=None) -> int:
        x = _f32(positions).reshape(-1, 3)
        v = None if velocities is None else _f32(velocities).reshape(-1, 3)
        lo = hi = None
        if domain is not None:
            lo, hi = (np.ascontiguousarray(d, np.float32).reshape(3) for d in domain)
        idx = c_int32()
        self._call("lsp_batch_add_scene", byref(params), _ptr(x), _ptr(v), x.shape[0], _ptr(lo), _ptr(hi),
                   byref(idx))
        self._counts.append(x.shape[0])
        return idx.value

    def add_box(self, scene: int, center, half_extent, boundary: bool = False):
        c = np.ascontiguousarray(center, np.float32)
        h = np.ascontiguousarray(half_extent, np.float32)
        self._call("lsp_batch_add_box", scene, _ptr(c), _ptr(h), abi.LSP_BOUNDARY if boundary else abi.LSP_OBSTACLE)

    def add_sphere(self, scene: int, center, radius: float, boundary: bool = False):
        c = np.ascontiguousarray(center, np.float32)
        self._call("lsp_batch_add_sphere", scene, _ptr(c), c_float(radius),
                   abi.LSP_BOUNDARY if boundary else abi.LSP_OBSTACLE)

    def add_collider(self, scene: int, collider):
        """Takes a scenes.Collider (kind 'box' or 'sphere')."""
        if collider.kind == "box":
            self.add_box(scene, collider.center, collider.size, collider.boundary)
        else:
            self.add_sphere(scene, collider.center, collider.size, collider.boundary)

    def update_box(self, scene: int, index: int, center, half_extent):
        c = np.ascontiguousarray(center, np.float32)
        h = np.ascontiguousarray(half_extent, np.float32)
        self._call("lsp_batch_update_box", scene, index, _ptr(c), _ptr(h))

    def update_sphere(self, scene: int, index: int, center, radius: float):
        c = np.ascontiguousarray(center, np.float32)
        self._call("lsp_batch_update_sphere", scene, index, _ptr(c), c_float(radius))

    @property
    def scenes(self) -> int:
        return len(self._counts)

    @property
    def total(self) -> int:
        return int(sum(self._counts))

    def count(self, scene: int) -> int:
        return self._counts[scene]

    # ------------------------------------------------------------ stepping
    def update(self, dt: float):
        """One step of every scene; returns the per-scene LspStepStats."""
        st = (abi.LspStepStats * max(self.scenes, 1))()
        self._call("lsp_batch_step", c_float(dt), st)
        return list(st)[: self.scenes]

    def set_launch(self, use_graph: bool = True, threads: int = 256, loop_blocks: int = 0):
        self._call("lsp_batch_set_launch", int(use_graph), int(threads), int(loop_blocks))

    def get_launch(self) -> dict:
        vals = [ctypes.c_int() for _ in range(4)]
        self._call("lsp_batch_get_launch", *(byref(v) for v in vals))
        return dict(zip(("use_graph", "threads", "loop_blocks", "graph_active"), (v.value for v in vals)))

    def autotune(self, dt: float, repeats: int = 3):
        """Tunes the launch shape on the next step and performs that step. Returns
        (LspBatchTuning, per-scene stats)."""
        t = abi.LspBatchTuning()
        st = (abi.LspStepStats * max(self.scenes, 1))()
        self._call("lsp_batch_autotune", c_float(dt), int(repeats), byref(t), st)
        return t, list(st)[: self.scenes]

    # ------------------------------------------------------------ learned warm start
    def set_warm_start(self, mode: int):
        self._call("lsp_batch_set_warm_start", int(mode))

    def mlp_reset(self, seed: int = 0):
        self._call("lsp_batch_mlp_reset", ctypes.c_uint64(seed))

    def mlp_set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        self._call("lsp_batch_mlp_set_weights", _ptr(w), w.size)

    def mlp_get_weights(self) -> np.ndarray:
        w = np.empty(abi.MLP_PARAMS, np.float32)
        self._call("lsp_batch_mlp_get_weights", _ptr(w), w.size)
        return w

    def mlp_record(self, on: bool = True):
        self._call("lsp_batch_mlp_record", int(on))

    def mlp_set_loss_asymmetry(self, over_weight: float):
        self._call("lsp_batch_mlp_set_loss_asymmetry", c_float(over_weight))

    def mlp_train(self, iterations: int = 4, batch: int = 65536, lr: float = 1e-3, seed: int = 0) -> float:
        loss = c_float()
        self._call("lsp_batch_mlp_train", int(iterations), int(batch), c_float(lr), ctypes.c_uint64(seed),
                   byref(loss))
        return loss.value

    def read_features(self, scene: int) -> np.ndarray:
        n = self._counts[scene]
        out = np.empty((n, abi.MLP_FEATURES), np.float32)
        self._call("lsp_batch_read_features", scene, _ptr(out), n)
        return out

    # ------------------------------------------------------------ read-back
    def read(self, scene: int, field: int) -> np.ndarray:
        n = self._counts[scene]
        shape = (n, 3) if field in abi.VECTOR_FIELDS else (n,)
        out = np.empty(shape, np.float32)
        self._call("lsp_batch_read_field", scene, int(field), _ptr(out), n)
        return out

    def positions(self, scene: int) -> np.ndarray:
        return self.read(scene, abi.FIELD_POSITION)

    def neighbors(self, scene: int):
        n = self._counts[scene]
        off = np.empty(n + 1, np.int64)
        self._call("lsp_batch_read_neighbors", scene, _ptr(off, POINTER(c_int64)), None, n, 0)
        idx = np.empty(max(int(off[-1]), 1), np.int32)
        self._call("lsp_batch_read_neighbors", scene, _ptr(off, POINTER(c_int64)), _ptr(idx, POINTER(c_int32)), n,
                   idx.size)
        return off, idx[: int(off[-1])]

    def grid(self, scene: int):
        n = self._counts[scene]
        dims = np.empty(3, np.int32)
        org = np.empty(3, np.int32)
        cells = c_int64()
        self._call("lsp_batch_grid_info", scene, _ptr(dims, POINTER(c_int32)), _ptr(org, POINTER(c_int32)),
                   byref(cells))
        keys = np.empty(n, np.uint32)
        ids = np.empty(n, np.int32)
        start = np.empty(cells.value + 1, np.uint32)
        self._call("lsp_batch_read_grid", scene, _ptr(keys, POINTER(c_uint32)), _ptr(ids, POINTER(c_int32)), n,
                   _ptr(start, POINTER(c_uint32)), cells.value + 1)
        return dims, org, keys, ids, start

    def read_state(self):
        n = self.total
        x, v, h, o = (np.empty((n, 3), np.float32) for _ in range(4))
        first = np.empty(n, np.int32)
        self._call("lsp_batch_read_state", _ptr(x), _ptr(v), _ptr(h), _ptr(o), _ptr(first, POINTER(c_int32)), n)
        return x, v, h, o, first

    def write_state(self, x, v, half, old_half, first):
        n = self.total
        arrs = [_f32(a).reshape(n, 3) for a in (x, v, half, old_half)]
        f = np.ascontiguousarray(first, np.int32).reshape(n)
        self._call("lsp_batch_write_state", *(_ptr(a) for a in arrs), _ptr(f, POINTER(c_int32)), n)

    def launch_count(self) -> int:
        v = c_int64()
        self._call("lsp_batch_launch_count", byref(v))
        return v.value


def batch_from_scenes(scene_list, device: int = -1) -> SceneBatch:
    """A SceneBatch holding scenes.Scene objects in order (same dt expected)."""
    b = SceneBatch(device)
    for sc in scene_list:
        k = b.add_scene(sc.params, sc.positions, sc.velocities, sc.domain)
        for c in sc.colliders:
            b.add_collider(k, c)
    return b
