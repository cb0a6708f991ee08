"""lsp_mlp_gradient_static, the entry point that allocates no device memory, against the
allocating lsp_mlp_gradient on the same weights and batches, two calls in a row.

Callers that may not allocate device memory while they run (a training loop inside a
framework that owns the GPU's memory pool, a process under a hard memory budget) pass
device buffers they already own; the partial sums go to a fixed scratch array in the
library. The two entry points partition the batch over different grids, so their FP32
sums differ only by rounding order: relative L2 error of the gradient <= 1e-4, loss
within 1e-5 relative (the tensor-core gradient tests against the FP64 oracle allow 2e-2).

This file is named to run last: it checks a path that shares one scratch array across
calls, and must pass both alone in a fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

from liquidsimulation_b200 import abi

pytestmark = pytest.mark.gpu


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0.0, 1.0, (n, 8)).astype(np.float32)
    t = (0.7 * x[:, 1] - 0.2 * np.tanh(x[:, 0]) + 0.05 * x[:, 6]).astype(np.float32)
    return x, t


def test_static_gradient_matches_allocating_entry_point():
    import torch
    from liquidsimulation_b200.solver import PCISPHSolver

    lib = abi.load_library()
    lib.lsp_mlp_gradient_static.restype = ctypes.c_int
    lib.lsp_mlp_gradient_static.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                            ctypes.c_void_p, ctypes.c_void_p]
    s = PCISPHSolver()
    rng = np.random.default_rng(3)
    w = (rng.normal(0.0, 0.3, abi.MLP_PARAMS)).astype(np.float32)
    s.mlp_set_weights(w)
    fp = ctypes.POINTER(ctypes.c_float)
    dev = torch.device("cuda", torch.cuda.current_device())
    cases = [(5000, 11), (777, 12)]
    refs, bufs = [], []
    for n, seed in cases:
        x, t = _batch(n, seed)
        # Reference: the allocating entry point on host arrays.
        g_ref = np.empty(abi.MLP_PARAMS, np.float32)
        l_ref = ctypes.c_float()
        s._call("lsp_mlp_gradient", x.ctypes.data_as(fp), t.ctypes.data_as(fp), n, g_ref.ctypes.data_as(fp),
                ctypes.byref(l_ref))
        refs.append((g_ref, l_ref.value))
        # Device buffers owned by the caller, all created before the allocation-free calls.
        bufs.append((torch.from_numpy(x).to(dev), torch.from_numpy(t).to(dev),
                     torch.full((abi.MLP_PARAMS,), float("nan"), dtype=torch.float32, device=dev),
                     torch.full((1,), float("nan"), dtype=torch.float32, device=dev)))
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    for call, ((n, _), (dx, dt, dg, dl)) in enumerate(zip(cases, bufs)):
        rc = lib.lsp_mlp_gradient_static(s._h, dx.data_ptr(), dt.data_ptr(), n, dg.data_ptr(), dl.data_ptr())
        assert rc == abi.LSP_OK, lib.lsp_last_error()
        s.synchronize()
    # Nothing was allocated on the device by the two calls (the scratch was set up when the
    # solver was created).
    assert torch.cuda.mem_get_info(dev)[0] == free_before
    for call, ((g_ref, l_ref), (dx, dt, dg, dl)) in enumerate(zip(refs, bufs)):
        g = dg.cpu().numpy()
        loss = float(dl.cpu().numpy()[0])
        rel = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
        assert rel <= 1e-4, (call, rel)
        assert abs(loss - l_ref) <= 1e-5 * abs(l_ref), (call, loss, l_ref)
    # Sizes beyond the fixed scratch are refused with a clear error, and host buffers too.
    rc = lib.lsp_mlp_gradient_static(s._h, dx.data_ptr(), dt.data_ptr(), (1 << 24) + 1, dg.data_ptr(),
                                     dl.data_ptr())
    assert rc == abi.LSP_ERR_CAPACITY and b"16777216" in lib.lsp_last_error()
    host = np.zeros(8 * 16, np.float32)
    rc = lib.lsp_mlp_gradient_static(s._h, host.ctypes.data, dt.data_ptr(), 16, dg.data_ptr(), dl.data_ptr())
    assert rc == abi.LSP_ERR_INVALID
    if torch.cuda.device_count() > 1:
        # A buffer on another GPU is refused before anything is launched (the pointer is
        # only inspected, never read).
        other = (torch.cuda.current_device() + 1) % torch.cuda.device_count()
        far = torch.zeros(8 * 16, dtype=torch.float32, device=torch.device("cuda", other))
        rc = lib.lsp_mlp_gradient_static(s._h, far.data_ptr(), dt.data_ptr(), 16, dg.data_ptr(), dl.data_ptr())
        assert rc == abi.LSP_ERR_INVALID and b"solver's GPU" in lib.lsp_last_error()
    s.close()
