"""ctypes mirror of include/lsp.h and the loader of the CUDA library.

The structures and constants here are the C ABI of ``liblsp.so``; they must stay
field-for-field identical to ``include/lsp.h`` (a CPU test checks the sizes).
Defaults follow the reference's constructors: ``SPHSolver::SPHSolver``
(LiquidPhysics/src/SPHSolver.cpp:11-23) and ``PCISPHSolver::PCISPHSolver``
(LiquidPhysics/src/PCISPHSolver.cpp:6-7).
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_uint32, c_void_p

LSP_OK = 0
LSP_ERR_INVALID = -1
LSP_ERR_CUDA = -2
LSP_ERR_NO_DEVICE = -3
LSP_ERR_DEVICE_STATUS = -4
LSP_ERR_NOT_CONVERGED = -5
LSP_ERR_TIMEOUT = -6
LSP_ERR_CAPACITY = -7
LSP_ERR_STATE = -8

LSP_SOLVER_SPH = 0
LSP_SOLVER_PCISPH = 1
LSP_OBSTACLE = 0
LSP_BOUNDARY = 1
LSP_WARM_ZERO = 0
LSP_WARM_MLP = 1
LSP_WARM_AUTO = 2
LSP_LOOP_PERSISTENT = 0
LSP_LOOP_HOST = 1

FIELD_POSITION = 0
FIELD_VELOCITY = 1
FIELD_HALF_VELOCITY = 2
FIELD_DENSITY = 3
FIELD_PRESSURE = 4
FIELD_FIRST_STEP = 5
FIELD_PRED_DENSITY = 6
FIELD_DENSITY_ERROR = 7
FIELD_PRED_POSITION = 8
FIELD_PRED_HALF_VELOCITY = 9
FIELD_PRED_PRESSURE_FORCE = 10
FIELD_OLD_HALF_VELOCITY = 11
FIELD_NEIGHBOR_COUNT = 12
FIELD_SPEED_SQUARED = 13

VECTOR_FIELDS = {FIELD_POSITION, FIELD_VELOCITY, FIELD_HALF_VELOCITY, FIELD_PRED_POSITION,
                 FIELD_PRED_HALF_VELOCITY, FIELD_PRED_PRESSURE_FORCE, FIELD_OLD_HALF_VELOCITY}

PROF_NAMES = ["grid_keys", "neighbors", "density", "nonpressure", "sph_pressure", "pci_predict",
              "pci_density", "pci_force", "integrate_collide", "pci_loop", "warm_start", "grid_scan",
              "grid_scatter", "grid_gather"]

MLP_PARAMS = 1377
MLP_FEATURES = 8

TABLE_SIZE = 1001  # SPHKernel m_subdivision = 1000 -> 1001 entries (SPHKernel.cpp:4-7, :124)


class LspParams(ctypes.Structure):
    _fields_ = [
        ("gravity", c_float * 3),
        ("particle_radius", c_float),
        ("kernel_radius_factor", c_float),
        ("rest_density", c_float),
        ("viscosity", c_float),
        ("stiffness", c_float),
        ("negative_pressure_factor", c_float),
        ("surface_tension", c_float),
        ("surface_tension_threshold", c_float),
        ("restitution", c_float),
        ("friction", c_float),
        ("mass_override", c_float),
        ("solver", c_int32),
        ("pci_max_iterations", c_int32),
        ("pci_min_iterations", c_int32),
        ("pci_eta", c_float),
        ("warm_start", c_int32),
        ("strict_convergence", c_int32),
        ("keep_initial_velocity", c_int32),
        ("loop_mode", c_int32),
        ("warm_auto_iterations", c_int32),
        ("reserved", c_int32 * 5),
    ]


class LspStepStats(ctypes.Structure):
    _fields_ = [
        ("iterations", c_int32),
        ("converged", c_int32),
        ("max_density_error_ratio", c_double),
        ("max_neighbors", c_int32),
        ("escaped", c_int32),
        ("warm_start_used", c_int32),
        ("warm_start_tried", c_int32),
    ]


class LspBatchTuning(ctypes.Structure):
    _fields_ = [
        ("threads", c_int32),
        ("loop_blocks", c_int32),
        ("candidates", c_int32),
        ("reserved", c_int32),
        ("cand_threads", c_int32 * 16),
        ("cand_loop_blocks", c_int32 * 16),
        ("cand_ms", c_float * 16),
    ]


def default_params(**overrides) -> LspParams:
    """The reference's constructor defaults, then ``overrides`` by field name."""
    p = LspParams()
    p.gravity[:] = (0.0, -9.81, 0.0)
    p.particle_radius = 0.017
    p.kernel_radius_factor = 2.688
    p.rest_density = 998.29
    p.viscosity = 3.5
    p.stiffness = 3.0
    p.negative_pressure_factor = 0.0
    p.surface_tension = 0.0728
    p.surface_tension_threshold = 7.065
    p.restitution = 0.5
    p.friction = 1.0
    p.mass_override = 0.0
    p.solver = LSP_SOLVER_SPH
    p.pci_max_iterations = 4
    p.pci_min_iterations = 1
    p.pci_eta = 0.1
    p.warm_start = LSP_WARM_ZERO
    p.strict_convergence = 0
    p.keep_initial_velocity = 0
    p.loop_mode = LSP_LOOP_PERSISTENT
    for k, v in overrides.items():
        if k == "gravity":
            p.gravity[:] = tuple(v)
        else:
            setattr(p, k, v)
    return p


def params_dict(p: LspParams) -> dict:
    out = {}
    for name, _ in LspParams._fields_:
        if name == "reserved":
            continue
        v = getattr(p, name)
        out[name] = tuple(v) if name == "gravity" else v
    return out


# ---------------------------------------------------------------- CUDA library

_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG_DIR, "liblsp.so")
_lib = None


class LspError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"liblsp error {code}: {message}")
        self.code = code


def load_library(path: str | None = None):
    """Loads liblsp.so (the CUDA build). Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(
            f"{p} not found: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `python -m liquidsimulation_b200.build`")
    lib = ctypes.CDLL(p)
    _declare(lib)
    if path is None:
        _lib = lib
    return lib


def _declare(lib):
    S = c_void_p
    fp = POINTER(c_float)
    i32p = POINTER(c_int32)
    i64p = POINTER(c_int64)
    u32p = POINTER(c_uint32)
    sig = {
        "lsp_params_default": (None, [POINTER(LspParams)]),
        "lsp_last_error": (c_char_p, []),
        "lsp_device_info": (c_int, [POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
        "lsp_barrier_probe": (c_int, [c_int, c_int, c_int, POINTER(c_int32), POINTER(c_uint32)]),
        "lsp_create": (c_int, [POINTER(LspParams), c_int, POINTER(c_void_p)]),
        "lsp_destroy": (c_int, [S]),
        "lsp_set_params": (c_int, [S, POINTER(LspParams)]),
        "lsp_get_params": (c_int, [S, POINTER(LspParams)]),
        "lsp_particle_mass": (c_int, [S, fp]),
        "lsp_kernel_radius": (c_int, [S, fp]),
        "lsp_particle_count": (c_int, [S, i64p]),
        "lsp_pcisph_delta": (c_int, [S, c_float, fp]),
        "lsp_kernel_tables": (c_int, [S, fp, c_int]),
        "lsp_add_particles": (c_int, [S, fp, fp, c_int64]),
        "lsp_remove_particles": (c_int, [S]),
        "lsp_add_box": (c_int, [S, fp, fp, c_int]),
        "lsp_add_sphere": (c_int, [S, fp, c_float, c_int]),
        "lsp_remove_colliders": (c_int, [S]),
        "lsp_update_box": (c_int, [S, c_int, fp, fp]),
        "lsp_update_sphere": (c_int, [S, c_int, fp, c_float]),
        "lsp_set_domain": (c_int, [S, fp, fp]),
        "lsp_step": (c_int, [S, c_float, POINTER(LspStepStats)]),
        "lsp_step_many": (c_int, [S, c_float, c_int, POINTER(LspStepStats)]),
        "lsp_synchronize": (c_int, [S]),
        "lsp_read_particles": (c_int, [S, fp, fp, c_int64]),
        "lsp_read_field": (c_int, [S, c_int, fp, c_int64]),
        "lsp_read_state": (c_int, [S, fp, fp, fp, fp, i32p, c_int64]),
        "lsp_write_state": (c_int, [S, fp, fp, fp, fp, i32p, c_int64]),
        "lsp_read_neighbors": (c_int, [S, i64p, i32p, c_int64, c_int64]),
        "lsp_grid_info": (c_int, [S, i32p, i32p, i64p]),
        "lsp_read_grid": (c_int, [S, u32p, i32p, c_int64, u32p, c_int64]),
        "lsp_timer_mark": (c_int, [S, c_int]),
        "lsp_timer_elapsed": (c_int, [S, c_int, c_int, fp]),
        "lsp_profile": (c_int, [S, c_int]),
        "lsp_profile_read": (c_int, [S, POINTER(c_double), i64p, c_int]),
        "lsp_launch_count": (c_int, [S, i64p]),
        "lsp_host_alloc": (c_int, [ctypes.c_size_t, POINTER(c_void_p)]),
        "lsp_host_free": (c_int, [c_void_p]),
        "lsp_mlp_reset": (c_int, [S, ctypes.c_uint64]),
        "lsp_mlp_set_weights": (c_int, [S, fp, c_int]),
        "lsp_mlp_get_weights": (c_int, [S, fp, c_int]),
        "lsp_mlp_record": (c_int, [S, c_int]),
        "lsp_set_warm_start": (c_int, [S, c_int]),
        "lsp_mlp_set_loss_asymmetry": (c_int, [S, c_float]),
        "lsp_mlp_train": (c_int, [S, c_int, c_int, c_float, ctypes.c_uint64, fp]),
        "lsp_mlp_forward": (c_int, [S, fp, c_int64, fp]),
        "lsp_mlp_gradient": (c_int, [S, fp, fp, c_int64, fp, fp]),
        "lsp_read_features": (c_int, [S, fp, c_int64]),
        "lsp_save_state": (c_int, [S, c_char_p, ctypes.c_uint64]),
        "lsp_load_state": (c_int, [S, c_char_p]),
        "lsp_state_file_info": (c_int, [c_char_p, POINTER(LspParams), i64p, i32p, POINTER(ctypes.c_uint64)]),
        # batches of independent scenes
        "lsp_batch_create": (c_int, [c_int, POINTER(c_void_p)]),
        "lsp_batch_destroy": (c_int, [c_void_p]),
        "lsp_batch_add_scene": (c_int, [c_void_p, POINTER(LspParams), fp, fp, c_int64, fp, fp, i32p]),
        "lsp_batch_add_box": (c_int, [c_void_p, c_int32, fp, fp, c_int]),
        "lsp_batch_add_sphere": (c_int, [c_void_p, c_int32, fp, c_float, c_int]),
        "lsp_batch_update_box": (c_int, [c_void_p, c_int32, c_int32, fp, fp]),
        "lsp_batch_update_sphere": (c_int, [c_void_p, c_int32, c_int32, fp, c_float]),
        "lsp_batch_info": (c_int, [c_void_p, i32p, i64p]),
        "lsp_batch_scene_count": (c_int, [c_void_p, c_int32, i64p]),
        "lsp_batch_particle_mass": (c_int, [c_void_p, c_int32, fp]),
        "lsp_batch_step": (c_int, [c_void_p, c_float, POINTER(LspStepStats)]),
        "lsp_batch_read_particles": (c_int, [c_void_p, c_int32, fp, fp, c_int64]),
        "lsp_batch_read_field": (c_int, [c_void_p, c_int32, c_int, fp, c_int64]),
        "lsp_batch_read_neighbors": (c_int, [c_void_p, c_int32, i64p, i32p, c_int64, c_int64]),
        "lsp_batch_grid_info": (c_int, [c_void_p, c_int32, i32p, i32p, i64p]),
        "lsp_batch_read_grid": (c_int, [c_void_p, c_int32, u32p, i32p, c_int64, u32p, c_int64]),
        "lsp_batch_read_state": (c_int, [c_void_p, fp, fp, fp, fp, i32p, c_int64]),
        "lsp_batch_write_state": (c_int, [c_void_p, fp, fp, fp, fp, i32p, c_int64]),
        "lsp_batch_set_launch": (c_int, [c_void_p, c_int, c_int, c_int]),
        "lsp_batch_get_launch": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
        "lsp_batch_autotune": (c_int, [c_void_p, c_float, c_int, POINTER(LspBatchTuning), POINTER(LspStepStats)]),
        "lsp_batch_set_warm_start": (c_int, [c_void_p, c_int]),
        "lsp_batch_mlp_reset": (c_int, [c_void_p, ctypes.c_uint64]),
        "lsp_batch_mlp_set_weights": (c_int, [c_void_p, fp, c_int]),
        "lsp_batch_mlp_get_weights": (c_int, [c_void_p, fp, c_int]),
        "lsp_batch_mlp_record": (c_int, [c_void_p, c_int]),
        "lsp_batch_mlp_set_loss_asymmetry": (c_int, [c_void_p, c_float]),
        "lsp_batch_mlp_train": (c_int, [c_void_p, c_int, c_int, c_float, ctypes.c_uint64, fp]),
        "lsp_batch_read_features": (c_int, [c_void_p, c_int32, fp, c_int64]),
        "lsp_batch_timer_mark": (c_int, [c_void_p, c_int]),
        "lsp_batch_timer_elapsed": (c_int, [c_void_p, c_int, c_int, fp]),
        "lsp_batch_launch_count": (c_int, [c_void_p, i64p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    # Optional entry points (declared when the loaded library exports them).
    for name, (res, args) in EXTRA_SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is not None:
            fn.restype = res
            fn.argtypes = args


EXTRA_SIGNATURES: dict = {}


def check(lib, code: int):
    if code != LSP_OK:
        msg = lib.lsp_last_error()
        raise LspError(code, msg.decode() if msg else "")
    return code
