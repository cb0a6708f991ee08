"""The C ABI without a GPU: the library loads, exports every symbol include/lsp.h
declares, the ctypes structures match the C layout, defaults match the reference
constructors, and calls fail cleanly (status codes, no crash) when no device exists."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from liquidsimulation_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = sorted(os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
                 if f.endswith(".h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(lsp_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from liquidsimulation_b200 import build
    build.build()
    return abi.load_library()


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_struct_layout_matches_c(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "lsp.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(lsp_params), offsetof(lsp_params, solver),
         offsetof(lsp_params, pci_eta), offsetof(lsp_params, keep_initial_velocity),
         sizeof(lsp_step_stats), offsetof(lsp_step_stats, max_neighbors),
         sizeof(lsp_batch_tuning), offsetof(lsp_batch_tuning, cand_ms));
  return 0;
}''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    got = [int(x) for x in out]
    want = [ctypes.sizeof(abi.LspParams), abi.LspParams.solver.offset, abi.LspParams.pci_eta.offset,
            abi.LspParams.keep_initial_velocity.offset, ctypes.sizeof(abi.LspStepStats),
            abi.LspStepStats.max_neighbors.offset, ctypes.sizeof(abi.LspBatchTuning),
            abi.LspBatchTuning.cand_ms.offset]
    assert got == want


def test_defaults_match_reference_constructors(lib):
    c = abi.LspParams()
    lib.lsp_params_default(ctypes.byref(c))
    py = abi.default_params()
    assert bytes(c) == bytes(py)
    # SPHSolver.cpp:11-23 and PCISPHSolver.cpp:6-7.
    assert np.float32(c.kernel_radius_factor) == np.float32(2.688)
    assert np.float32(c.rest_density) == np.float32(998.29)
    assert c.pci_max_iterations == 4 and np.float32(c.pci_eta) == np.float32(0.1)


def test_calls_fail_cleanly_without_device(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    p = abi.default_params()
    h = ctypes.c_void_p()
    rc = lib.lsp_create(ctypes.byref(p), -1, ctypes.byref(h))
    assert rc == abi.LSP_ERR_NO_DEVICE
    assert b"device" in lib.lsp_last_error()
    assert lib.lsp_step(None, ctypes.c_float(0.001), None) == abi.LSP_ERR_INVALID
    assert lib.lsp_destroy(None) == abi.LSP_OK
    b = ctypes.c_void_p()
    assert lib.lsp_batch_create(-1, ctypes.byref(b)) == abi.LSP_ERR_NO_DEVICE
    assert lib.lsp_batch_step(None, ctypes.c_float(0.001), None) == abi.LSP_ERR_INVALID
    assert lib.lsp_batch_destroy(None) == abi.LSP_OK


def test_product_has_no_cpu_fallback():
    """The product package never imports, loads or links the oracle or the reference build."""
    pkg = os.path.join(ROOT, "liquidsimulation_b200")
    pat = re.compile(r"(^\s*(from|import)\s+oracle\b)|liblsp_oracle|libref_sph|orc_\w+\(|ref_\w+\(", re.M)
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cpp", ".h", ".cuh")):
                text = open(os.path.join(dirpath, f)).read()
                assert not pat.search(text), f
