"""The allocation-free dot product, gb_dot_f64_noalloc.

Some callers cannot allocate device memory during a call: their HBM is
already owned by another allocator (a framework's caching pool), or they run
latency-critical loops where cudaMalloc/cudaFree would synchronise the device.
gb_dot_f64_noalloc serves them by keeping its partial sums in a fixed device
array compiled into the library.  This file checks it through the C ABI
against the allocating gb_dot_f64, on two calls in a row (so the second call
runs over the array the first one left behind), and that sizes above its
stated maximum are refused.  It sits in its own file named to be collected
last, and passes both alone in a fresh process and after the other tests.
"""
from __future__ import annotations


import numpy as np
import pytest

import gooseberry_b200 as gb
from gooseberry_b200 import workloads as W

pytestmark = pytest.mark.gpu

MAX_N = 16384 * 8192  # GB_DOT_NOALLOC_MAX_N in include/gooseberry_b200.h


def _dot_both(torch, a, b):
    L = gb.lib()
    stream = torch.cuda.current_stream().cuda_stream
    ref = torch.empty(1, dtype=torch.float64, device="cuda")
    got = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    assert L.gb_dot_f64(a.numel(), a.data_ptr(), b.data_ptr(), ref.data_ptr(), stream) == 1, \
        gb.last_error()
    assert L.gb_dot_f64_noalloc(a.numel(), a.data_ptr(), b.data_ptr(), got.data_ptr(),
                                stream) == 1, gb.last_error()
    torch.cuda.synchronize()
    return float(ref.item()), float(got.item())


def test_noalloc_dot_matches_allocating_dot_on_two_calls():
    import torch
    assert torch.cuda.is_available()
    # a large call (many chunks) then a smaller one over the same scratch
    for n, seed in ((3_000_017, 5), (40_001, 6)):
        a = torch.from_numpy(W.dense_x(n, seed)).cuda()
        b = torch.from_numpy(W.rhs(n, seed)).cuda()
        ref, got = _dot_both(torch, a, b)
        scale = float(torch.sum(torch.abs(a * b)).item())
        # same tolerance as the BLAS-1 device test: both sums are fixed-order
        # double reductions that differ only in grouping
        assert abs(got - ref) <= 1e-12 * scale, (n, got, ref)
        exact = float(np.dot(a.cpu().numpy(), b.cpu().numpy()))
        assert abs(got - exact) <= 1e-12 * scale
    # repeated call on the same input gives the same bits
    a = torch.from_numpy(W.dense_x(777_777, 8)).cuda()
    b = torch.from_numpy(W.rhs(777_777, 8)).cuda()
    r1 = _dot_both(torch, a, b)[1]
    r2 = _dot_both(torch, a, b)[1]
    assert r1 == r2


def test_noalloc_dot_refuses_sizes_above_its_maximum():
    import torch
    a = torch.zeros(4, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = gb.lib().gb_dot_f64_noalloc(MAX_N + 1, a.data_ptr(), a.data_ptr(), out.data_ptr(),
                                     torch.cuda.current_stream().cuda_stream)
    assert rc == 3  # GOOSEBERRY_ERROR_INVALIDINPUT, refused before any kernel runs
    assert "exceeds" in gb.last_error()
    # and zero elements gives zero
    rc = gb.lib().gb_dot_f64_noalloc(0, None, None, out.data_ptr(),
                                     torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rc == 1 and float(out.item()) == 0.0
