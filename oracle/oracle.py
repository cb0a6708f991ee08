"""Python front-end of the oracle (test infrastructure, not product code).

Two CPU solvers with one interface:

* ``RefSolver``: the reference's own sequential CPU solver, compiled unmodified
  from LiquidPhysics/src by ``oracle/Makefile`` into ``oracle/_ref/libref_sph.so``.
* ``OracleSolver``: the project's restatement, ``oracle/liblsp_oracle.so``
  (``oracle/sph_oracle.cpp``), pinned bit for bit to ``RefSolver`` by the CPU tests;
  it also runs in FP64 and supports the minimum-iteration rule.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module. The product never does.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_float, c_int, c_int32, c_int64, c_uint32, c_void_p

import numpy as np

from liquidsimulation_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libref_sph.so")
ORACLE_LIB = os.path.join(HERE, "liblsp_oracle.so")

_fp = POINTER(c_float)
_i32p = POINTER(c_int32)
_i64p = POINTER(c_int64)


def _f(a):
    return a.ctypes.data_as(_fp) if a is not None else None


def build(ref_dir: str | None = None, quiet: bool = True) -> None:
    """Runs oracle/Makefile (the restatement always; the reference when its sources exist)."""
    import subprocess
    cmd = ["make", "-C", HERE]
    if ref_dir:
        cmd.append(f"REF_DIR={ref_dir}")
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL if quiet else None)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


_ref = None
_orc = None


def _ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError(f"{REF_LIB} missing: run `make -C oracle ref` where the reference sources exist")
        L = ctypes.CDLL(REF_LIB)
        V = c_void_p
        sigs = {
            "ref_create": (c_void_p, [c_int]), "ref_destroy": (None, [V]),
            "ref_parallelization_type": (c_int, [V]),
            "ref_set_gravity": (None, [V, c_float, c_float, c_float]),
            "ref_set_particle_radius": (None, [V, c_float]), "ref_set_kernel_radius_factor": (None, [V, c_float]),
            "ref_set_rest_density": (None, [V, c_float]), "ref_set_viscosity": (None, [V, c_float]),
            "ref_set_stiffness": (None, [V, c_float]), "ref_set_negative_pressure_factor": (None, [V, c_float]),
            "ref_set_surface_tension": (None, [V, c_float]), "ref_set_surface_tension_threshold": (None, [V, c_float]),
            "ref_set_restitution": (None, [V, c_float]), "ref_set_friction": (None, [V, c_float]),
            "ref_set_pci_iterations": (None, [V, c_int]), "ref_set_pci_eta": (None, [V, c_float]),
            "ref_force_mass": (None, [V, c_float]), "ref_capture_neighbors": (None, [V, c_int]),
            "ref_mass": (c_float, [V]), "ref_kernel_radius": (c_float, [V]), "ref_division_step": (c_float, [V]),
            "ref_tables": (None, [V, _fp]),
            "ref_add_particles": (None, [V, _fp, _fp, c_int]),
            "ref_add_box": (None, [V, _fp, _fp, c_int]), "ref_add_sphere": (None, [V, _fp, c_float, c_int]),
            "ref_add_iteration_counter": (None, [V]),
            "ref_count": (c_int, [V]), "ref_step": (None, [V, c_float]), "ref_steps": (None, [V, c_float, c_int]),
            "ref_last_iterations": (c_int, [V]),
            "ref_get": (c_int, [V, c_int, _fp]),
            "ref_set_state": (None, [V, _fp, _fp, _fp, _fp, POINTER(c_int)]),
            "ref_neighbor_total": (c_int, [V]), "ref_neighbor_lists": (None, [V, POINTER(c_int), POINTER(c_int)]),
        }
        for k, (r, a) in sigs.items():
            fn = getattr(L, k)
            fn.restype = r
            fn.argtypes = a
        _ref = L
    return _ref


def _orc_lib():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            build()
        L = ctypes.CDLL(ORACLE_LIB)
        V = c_void_p
        P = POINTER(abi.LspParams)
        sigs = {
            "orc_create": (c_void_p, [P, c_int]), "orc_destroy": (None, [V]),
            "orc_set_params": (c_int, [V, P]),
            "orc_add_particles": (c_int, [V, _fp, _fp, c_int64]),
            "orc_add_box": (c_int, [V, _fp, _fp, c_int]), "orc_add_sphere": (c_int, [V, _fp, c_float, c_int]),
            "orc_update_box": (c_int, [V, c_int, _fp, _fp]), "orc_update_sphere": (c_int, [V, c_int, _fp, c_float]),
            "orc_count": (c_int64, [V]),
            "orc_step": (c_int, [V, c_float, POINTER(abi.LspStepStats)]),
            "orc_set_initial_pressure": (c_int, [V, _fp, c_int64]),
            "orc_set_delta_override": (c_int, [V, c_double]),
            "orc_get": (c_int, [V, c_int, _fp]), "orc_get_f64": (c_int, [V, c_int, POINTER(c_double)]),
            "orc_set_state": (c_int, [V, _fp, _fp, _fp, _fp, _i32p]),
            "orc_mass": (c_float, [V]), "orc_kernel_radius": (c_float, [V]), "orc_delta": (c_float, [V, c_float]),
            "orc_tables": (None, [V, _fp]),
            "orc_neighbor_total": (c_int64, [V]), "orc_neighbor_lists": (None, [V, _i64p, _i32p]),
            "orc_set_threads": (None, [c_int]),
            "orc_grid_build": (c_int, [_fp, c_int64, c_float, _i32p, _i32p, POINTER(c_uint32), _i32p,
                                       POINTER(c_uint32), _i64p]),
        }
        for k, (r, a) in sigs.items():
            fn = getattr(L, k)
            fn.restype = r
            fn.argtypes = a
        _orc = L
    return _orc


def _vec(a):
    return np.ascontiguousarray(a, dtype=np.float32).reshape(-1)


class RefSolver:
    """The reference CPU solver (SPHSolver / PCISPHSolver, ParallelizationType::NONE)."""

    def __init__(self, scene, count_iterations: bool = True, capture_neighbors: bool = False):
        L = self.L = _ref_lib()
        p = scene.params
        self.pcisph = p.solver == abi.LSP_SOLVER_PCISPH
        self.h = L.ref_create(1 if self.pcisph else 0)
        assert L.ref_parallelization_type(self.h) == 0, "reference did not select its CPU path"
        L.ref_set_gravity(self.h, *p.gravity)
        L.ref_set_particle_radius(self.h, p.particle_radius)
        L.ref_set_kernel_radius_factor(self.h, p.kernel_radius_factor)
        L.ref_set_rest_density(self.h, p.rest_density)
        L.ref_set_viscosity(self.h, p.viscosity)
        L.ref_set_stiffness(self.h, p.stiffness)
        L.ref_set_negative_pressure_factor(self.h, p.negative_pressure_factor)
        L.ref_set_surface_tension(self.h, p.surface_tension)
        L.ref_set_surface_tension_threshold(self.h, p.surface_tension_threshold)
        L.ref_set_restitution(self.h, p.restitution)
        L.ref_set_friction(self.h, p.friction)
        if self.pcisph:
            if p.pci_min_iterations > 1:
                raise ValueError("the reference has no minimum iteration count; use OracleSolver")
            L.ref_set_pci_iterations(self.h, p.pci_max_iterations)
            L.ref_set_pci_eta(self.h, p.pci_eta)
        if p.mass_override > 0:
            L.ref_force_mass(self.h, p.mass_override)
        pos = _vec(scene.positions)
        vel = _vec(scene.velocities)
        if pos.size:
            L.ref_add_particles(self.h, _f(pos), _f(vel), pos.size // 3)
        for c in scene.colliders:
            center = np.asarray(c.center, np.float32)
            if c.kind == "box":
                L.ref_add_box(self.h, _f(center), _f(np.asarray(c.size, np.float32)), int(c.boundary))
            else:
                L.ref_add_sphere(self.h, _f(center), float(c.size), int(c.boundary))
        if count_iterations and self.pcisph:
            L.ref_add_iteration_counter(self.h)
        if capture_neighbors:
            L.ref_capture_neighbors(self.h, 1)

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    __del__ = close

    @property
    def n(self):
        return self.L.ref_count(self.h)

    def step(self, dt):
        self.L.ref_step(self.h, dt)
        return self.L.ref_last_iterations(self.h) if self.pcisph else 0

    def steps(self, dt, k):
        self.L.ref_steps(self.h, dt, k)

    def get(self, field):
        shape = (self.n, 3) if field in abi.VECTOR_FIELDS else (self.n,)
        out = np.empty(shape, np.float32)
        rc = self.L.ref_get(self.h, field, _f(out))
        if rc != 0:
            raise ValueError(f"field {field} not available")
        return out

    def set_state(self, x, v, half, old_half, first):
        first = np.ascontiguousarray(first, np.int32)
        self.L.ref_set_state(self.h, _f(_vec(x)), _f(_vec(v)), _f(_vec(half)), _f(_vec(old_half)),
                             first.ctypes.data_as(POINTER(c_int)))

    def neighbors(self):
        total = self.L.ref_neighbor_total(self.h)
        off = np.empty(self.n + 1, np.int32)
        idx = np.empty(max(total, 1), np.int32)
        self.L.ref_neighbor_lists(self.h, off.ctypes.data_as(POINTER(c_int)), idx.ctypes.data_as(POINTER(c_int)))
        return off.astype(np.int64), idx[:total]

    def mass(self):
        return self.L.ref_mass(self.h)

    def kernel_radius(self):
        return self.L.ref_kernel_radius(self.h)

    def tables(self):
        out = np.empty(5 * abi.TABLE_SIZE, np.float32)
        self.L.ref_tables(self.h, _f(out))
        return out.reshape(5, abi.TABLE_SIZE)


class OracleSolver:
    """The project's CPU restatement of the reference step (FP32 or FP64)."""

    def __init__(self, scene, fp64: bool = False, params=None):
        L = self.L = _orc_lib()
        self.params = params if params is not None else scene.params
        self.h = L.orc_create(ctypes.byref(self.params), 1 if fp64 else 0)
        self.fp64 = fp64
        pos = _vec(scene.positions)
        vel = _vec(scene.velocities)
        if pos.size:
            L.orc_add_particles(self.h, _f(pos), _f(vel), pos.size // 3)
        for c in scene.colliders:
            center = np.asarray(c.center, np.float32)
            if c.kind == "box":
                L.orc_add_box(self.h, _f(center), _f(np.asarray(c.size, np.float32)), int(c.boundary))
            else:
                L.orc_add_sphere(self.h, _f(center), float(c.size), int(c.boundary))

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    __del__ = close

    @property
    def n(self):
        return self.L.orc_count(self.h)

    def add_particles(self, pos, vel=None):
        pos = _vec(pos)
        vel = _vec(vel) if vel is not None else np.zeros_like(pos)
        self.L.orc_add_particles(self.h, _f(pos), _f(vel), pos.size // 3)

    def update_box(self, index, center, half):
        self.L.orc_update_box(self.h, index, _f(np.asarray(center, np.float32)), _f(np.asarray(half, np.float32)))

    def update_sphere(self, index, center, radius):
        self.L.orc_update_sphere(self.h, index, _f(np.asarray(center, np.float32)), float(radius))

    def step(self, dt, initial_pressure=None):
        """One step. initial_pressure (caller order, float32[n]): the pressure iteration 0
        takes in place of its own correction, as the device's learned warm start does
        (checked at iteration 1 and dropped for the zero start if the error rose)."""
        if initial_pressure is not None:
            p0 = np.ascontiguousarray(initial_pressure, np.float32).reshape(-1)
            if self.L.orc_set_initial_pressure(self.h, _f(p0), p0.size) != 0:
                raise ValueError("initial_pressure must hold one value per particle")
        st = abi.LspStepStats()
        self.L.orc_step(self.h, dt, ctypes.byref(st))
        return st

    def set_delta(self, delta):
        """Use this PCISPH pressure scaling instead of the derived one (None: derive it)."""
        self.L.orc_set_delta_override(self.h, float(delta) if delta else 0.0)

    def get(self, field, fp64=False):
        shape = (self.n, 3) if field in abi.VECTOR_FIELDS else (self.n,)
        if fp64:
            out = np.empty(shape, np.float64)
            rc = self.L.orc_get_f64(self.h, field, out.ctypes.data_as(POINTER(c_double)))
        else:
            out = np.empty(shape, np.float32)
            rc = self.L.orc_get(self.h, field, _f(out))
        if rc != 0:
            raise ValueError(f"field {field} not available")
        return out

    def set_state(self, x, v, half, old_half, first):
        first = np.ascontiguousarray(first, np.int32)
        self.L.orc_set_state(self.h, _f(_vec(x)), _f(_vec(v)), _f(_vec(half)), _f(_vec(old_half)),
                             first.ctypes.data_as(_i32p))

    def neighbors(self):
        total = self.L.orc_neighbor_total(self.h)
        off = np.empty(self.n + 1, np.int64)
        idx = np.empty(max(total, 1), np.int32)
        self.L.orc_neighbor_lists(self.h, off.ctypes.data_as(_i64p), idx.ctypes.data_as(_i32p))
        return off, idx[:total]

    def mass(self):
        return self.L.orc_mass(self.h)

    def kernel_radius(self):
        return self.L.orc_kernel_radius(self.h)

    def delta(self, dt):
        return self.L.orc_delta(self.h, dt)

    def tables(self):
        out = np.empty(5 * abi.TABLE_SIZE, np.float32)
        self.L.orc_tables(self.h, _f(out))
        return out.reshape(5, abi.TABLE_SIZE)


def set_threads(n: int) -> None:
    _orc_lib().orc_set_threads(int(n))


def grid_build(positions, h, origin, dims):
    """Device grid-build specification: (keys_sorted, ids_sorted, cell_start, escaped)."""
    L = _orc_lib()
    pos = _vec(positions)
    n = pos.size // 3
    origin = np.ascontiguousarray(origin, np.int32)
    dims = np.ascontiguousarray(dims, np.int32)
    cells = int(np.prod(dims.astype(np.int64)))
    keys = np.empty(max(n, 1), np.uint32)
    ids = np.empty(max(n, 1), np.int32)
    start = np.empty(cells + 1, np.uint32)
    esc = c_int64(0)
    L.orc_grid_build(_f(pos), n, float(h), origin.ctypes.data_as(_i32p), dims.ctypes.data_as(_i32p),
                     keys.ctypes.data_as(POINTER(c_uint32)), ids.ctypes.data_as(_i32p),
                     start.ctypes.data_as(POINTER(c_uint32)), ctypes.byref(esc))
    return keys[:n], ids[:n], start, int(esc.value)
