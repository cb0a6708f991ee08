"""State files (lsp_save_state / lsp_load_state / lsp_state_file_info).

CPU: a file written here from the documented layout is read back by the library's header
reader; damaged files are rejected with LSP_ERR_INVALID. GPU: a run saved mid-way and
resumed in a new handle continues bit-identically to the original run, warm start included.
"""
import ctypes
import struct

import numpy as np
import pytest

from liquidsimulation_b200 import abi, scenes
from liquidsimulation_b200.solver import from_scene, state_file_info, PCISPHSolver

MAGIC = b"LSPSTAT1"


def write_file(path, params, pos, seed=77, colliders=(), domain=None, flags_extra=0, magic=MAGIC, truncate=0):
    n = pos.shape[0]
    flags = 2 | (4 if domain is not None else 0) | flags_extra
    lo, hi = domain if domain is not None else ((0, 0, 0), (0, 0, 0))
    blob = bytearray()
    blob += magic + struct.pack("<IIQqiI", 1, flags, seed, n, len(colliders), ctypes.sizeof(abi.LspParams))
    blob += bytes(params)
    blob += struct.pack("<6f", *lo, *hi)
    for sphere, boundary, c, h, r in colliders:
        blob += struct.pack("<2i7f", sphere, boundary, *c, *h, r)
    x = pos.astype(np.float32)
    blob += x.tobytes() + np.zeros_like(x).tobytes() * 3 + np.ones(n, np.int32).tobytes()
    blob += np.zeros(abi.MLP_PARAMS, np.float32).tobytes()
    if truncate:
        blob = blob[:-truncate]
    path.write_bytes(bytes(blob))


def test_header_reader_follows_the_documented_layout(tmp_path):
    sc = scenes.small_box_scene(n_side=(4, 5, 6))
    f = tmp_path / "s.lspstate"
    write_file(f, sc.params, sc.positions, seed=12345,
               colliders=[(0, 1, (0.5, 0.5, 0.5), (0.5, 0.5, 0.5), 0.0), (1, 0, (0.3, 0.1, 0.2), (0, 0, 0), 0.1)],
               domain=((0, 0, 0), (1, 1, 1)))
    info = state_file_info(f)
    assert info["n"] == 120 and info["colliders"] == 2 and info["seed"] == 12345
    assert bytes(info["params"]) == bytes(sc.params)


@pytest.mark.parametrize("damage", ["magic", "version", "truncated_header"])
def test_damaged_files_are_rejected(tmp_path, damage):
    sc = scenes.small_box_scene(n_side=(3, 3, 3))
    f = tmp_path / "bad.lspstate"
    write_file(f, sc.params, sc.positions, magic=b"NOTSTATE" if damage == "magic" else MAGIC)
    if damage == "version":
        b = bytearray(f.read_bytes())
        b[8:12] = struct.pack("<I", 99)
        f.write_bytes(bytes(b))
    if damage == "truncated_header":
        f.write_bytes(f.read_bytes()[:40])
    with pytest.raises(abi.LspError) as e:
        state_file_info(f)
    assert e.value.code == abi.LSP_ERR_INVALID


FIELDS = [abi.FIELD_POSITION, abi.FIELD_VELOCITY, abi.FIELD_HALF_VELOCITY, abi.FIELD_OLD_HALF_VELOCITY,
          abi.FIELD_DENSITY, abi.FIELD_PRESSURE, abi.FIELD_FIRST_STEP]


@pytest.mark.gpu
@pytest.mark.parametrize("warm", [False, True])
def test_saved_run_resumes_bit_identically(tmp_path, warm):
    from oracle import mlp_oracle as M
    sc = scenes.dam_break_pcisph(seed=5, counts=(14, 22, 14), s=0.02)
    a = from_scene(sc)
    if warm:
        a.mlp_set_weights(M.init(3).astype(np.float32))
        a.set_warm_start(abi.LSP_WARM_MLP)
    for _ in range(4):
        a.update(sc.dt)
    f = tmp_path / "run.lspstate"
    a.save_state(f, seed=5)
    info = state_file_info(f)
    assert info["n"] == sc.n and info["seed"] == 5 and info["colliders"] == len(sc.colliders)
    b = PCISPHSolver()
    b.load_state(f)
    assert b.get_particle_count() == sc.n
    for step in range(3):
        sa, sb = a.update(sc.dt), b.update(sc.dt)
        assert (sa.iterations, sa.warm_start_used) == (sb.iterations, sb.warm_start_used), step
        for fld in FIELDS:
            assert np.array_equal(a.read(fld).view(np.uint32), b.read(fld).view(np.uint32)), (step, fld)
    a.close()
    b.close()


def read_file(path):
    """The state file's contents, parsed on the CPU from the layout documented in
    csrc/state_io.cpp: (flags, seed, params, domain, colliders, x, v, v_half, v_half_old, first)."""
    b = path.read_bytes()
    assert b[:8] == MAGIC
    version, flags, seed, n, ncol, psize = struct.unpack_from("<IIQqiI", b, 8)
    assert version == 1 and psize == ctypes.sizeof(abi.LspParams)
    off = 8 + struct.calcsize("<IIQqiI")
    params = abi.LspParams.from_buffer_copy(b[off:off + psize])
    off += psize
    lo_hi = struct.unpack_from("<6f", b, off)
    off += 24
    cols = []
    for _ in range(ncol):
        sphere, boundary, *rest = struct.unpack_from("<2i7f", b, off)
        off += struct.calcsize("<2i7f")
        c, h, r = rest[0:3], rest[3:6], rest[6]
        cols.append(scenes.Collider("sphere", tuple(c), r, bool(boundary)) if sphere
                    else scenes.Collider("box", tuple(c), tuple(h), bool(boundary)))
    arrs = []
    for _ in range(4):
        arrs.append(np.frombuffer(b, np.float32, 3 * n, off).reshape(n, 3).copy())
        off += 12 * n
    first = np.frombuffer(b, np.int32, n, off).copy()
    return flags, seed, params, (lo_hi[:3], lo_hi[3:]), cols, arrs, first


@pytest.mark.gpu
def test_resumed_run_matches_the_oracle_from_the_file(tmp_path):
    """A state file saved mid-run is parsed here on the CPU; the oracle starts from its
    caller-order state, parameters and colliders, the library from lsp_load_state, and both
    take three steps: 0 ulp on every field, equal iteration counts."""
    from oracle import oracle as O
    sc = scenes.dam_break_pcisph(seed=6, counts=(14, 22, 14), s=0.02)
    a = from_scene(sc)
    for _ in range(5):
        a.update(sc.dt)
    f = tmp_path / "mid.lspstate"
    a.save_state(f, seed=6)
    a.close()
    flags, seed, params, domain, cols, (x, v, h, old), first = read_file(f)
    assert seed == 6 and x.shape == (sc.n, 3) and first.max() == 0
    b = PCISPHSolver()
    b.load_state(f)
    file_scene = scenes.Scene("from_file", params, x, v, cols, sc.dt, 3, domain=domain)
    o = O.OracleSolver(file_scene)
    o.set_state(x, v, h, old, first)
    for step in range(3):
        sb, so = b.update(sc.dt), o.step(sc.dt)
        assert sb.iterations == so.iterations, step
        for fld in FIELDS:
            assert np.array_equal(b.read(fld).view(np.uint32), o.get(fld).view(np.uint32)), (step, fld)
    b.close()
    o.close()
