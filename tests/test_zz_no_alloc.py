"""lym_cdot_batch_noalloc: the dot-product entry point for callers that cannot
allocate device memory (code running under a framework's pooling allocator or a
fixed device-memory budget).  It must give what the allocating entry point
lym_cdot gives, call after call, while its scratch lives in a static device array.

This file is collected last on purpose, so a run that stops at the first
failure has already run every other test; it also passes on its own in a
fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative; both entry points sum in FP64, in different orders


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_dot_matches_allocating_dot(cuda_device):
    from tfleonardym_b200 import _dev, _lib
    lib = _lib.lib()
    rng = np.random.default_rng(20261203)
    nvec, n = 7, 4 * 3 * 4096 + 5  # seven spinors of a 16^3 x 4 SU(3) lattice, plus a ragged tail
    a = torch.from_numpy(rng.normal(size=(nvec, n)) + 1j * rng.normal(size=(nvec, n))).to(cuda_device)
    b = torch.from_numpy(rng.normal(size=(nvec, n)) + 1j * rng.normal(size=(nvec, n))).to(cuda_device)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    expect = [_dev.cdot(a[i], b[i]) for i in range(nvec)]  # the existing entry point, lym_cdot
    for call in range(2):  # the scratch keeps the previous call's contents
        out = (ctypes.c_double * (2 * nvec))()
        rc = lib.lym_cdot_batch_noalloc(nvec, n, _ptr(a), _ptr(b), out, stream)
        assert rc == _lib.LYM_OK, lib.lym_last_error()
        for i in range(nvec):
            got = complex(out[2 * i], out[2 * i + 1])
            assert abs(got - expect[i]) <= TOL * abs(expect[i]), (call, i, got, expect[i])


def test_noalloc_dot_rejects_more_vectors_than_its_scratch(cuda_device):
    from tfleonardym_b200 import _lib
    lib = _lib.lib()
    a = torch.zeros((65, 8), dtype=torch.complex128, device=cuda_device)
    out = (ctypes.c_double * (2 * 65))()
    rc = lib.lym_cdot_batch_noalloc(65, 8, _ptr(a), _ptr(a), out, None)
    assert rc == _lib.LYM_ERR_BAD_ARG
    assert b"static scratch" in lib.lym_last_error()
