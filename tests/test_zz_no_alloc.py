"""The allocation-free dot product, b2p_dot_noalloc, against the ordinary one.

b2p_dot_noalloc serves callers that cannot let a library allocate device
memory: code that records a CUDA graph (cudaMalloc is not allowed while a
stream is being captured) or an application that hands out all device memory
from its own pool.  The caller owns the device buffers; the library uses only a
fixed scratch array reserved at load time.  This test gives it device buffers,
calls it twice in a row through the C ABI, and checks both results against
b2p_dot (the entry point that stages host buffers through its own context
memory).  This file is named so that pytest collects it last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_dot(b2p, torch, a_dev, b_dev, out_dev, n, stream):
    return b2p.lib().b2p_dot_noalloc(C.c_void_p(a_dev.data_ptr()), C.c_void_p(b_dev.data_ptr()), n,
                                     C.c_void_p(out_dev.data_ptr()), C.c_void_p(stream.cuda_stream))


def test_dot_noalloc_matches_dot_twice(b2p):
    import torch
    rng = np.random.default_rng(2024)
    stream = torch.cuda.Stream()
    with b2p.Context(0) as ctx:
        for n in (1_000_003, 4096):  # two calls in a row, different sizes share the scratch array
            a = rng.standard_normal(n)
            b = rng.standard_normal(n)
            want = ctx.dot(a, b)
            a_dev = torch.from_numpy(a).cuda()
            b_dev = torch.from_numpy(b).cuda()
            out_dev = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            assert _noalloc_dot(b2p, torch, a_dev, b_dev, out_dev, n, stream) == b2p.OK
            stream.synchronize()
            if n != 1_000_003:  # after the first call (its set-up) no device memory moves
                assert torch.cuda.mem_get_info()[0] == free_before
            got = float(out_dev.item())
            # same two-pass FP64 algorithm, different block partition: agree to rounding
            assert abs(got - want) <= 1e-12 * float(np.abs(a) @ np.abs(b)), (n, got, want)


def test_dot_noalloc_rejects_too_large(b2p):
    import torch
    n = b2p.DOT_NOALLOC_MAX_N + 1
    a_dev = torch.zeros(n, dtype=torch.float64, device="cuda")
    out_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = b2p.lib().b2p_dot_noalloc(C.c_void_p(a_dev.data_ptr()), C.c_void_p(a_dev.data_ptr()), n,
                                   C.c_void_p(out_dev.data_ptr()), None)
    assert st == b2p.TOO_LARGE
