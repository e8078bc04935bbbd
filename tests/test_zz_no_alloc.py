"""llg_dot_multi_noalloc: the multi-dot for callers that cannot allocate.

Applications whose device memory is owned by another allocator, and solver
loops that allow no allocation after set-up (cudaMalloc/cudaFree may
synchronise the device), cannot let a library call cudaMalloc when they ask
for K dot products.  This entry point keeps its reduction scratch in a fixed
device array instead; the test checks it against the allocating
llg_dot_multi through the C ABI on two calls in a row (the scratch array
keeps the previous call's contents): bit for bit where both reduce the same
vectors, within 1e-13 of a host sum for the shorter prefixes.  It also
checks the size limit.  This file sorts last so a stop-at-first-failure run
has already run every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import llg

pytestmark = pytest.mark.gpu


def _fn():
    lib = llg.load()
    fn = lib.llg_dot_multi_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_int, C.c_void_p, C.POINTER(C.c_void_p), C.c_int64, C.c_void_p, C.c_void_p]
    return fn


def test_noalloc_multi_dot_matches_allocating_entry_point(gpu):
    import torch
    fn = _fn()
    ctx = llg.Context(llg.default_params(211, 97))
    n = 3 * 211 * 97
    rng = np.random.default_rng(123)
    cases = [(7, n), (3, n), (16, 1000), (1, 5)]  # different shapes back to back
    for nvec, length in cases:
        x = torch.from_numpy(rng.standard_normal(n)).cuda()
        Ys = [torch.from_numpy(rng.standard_normal(n)).cuda() for _ in range(nvec)]
        if length == n:
            ref = np.array(ctx.dot_multi(x, Ys))
        else:
            xs = x[:length].cpu().numpy()
            ref = np.array([np.dot(xs, y[:length].cpu().numpy()) for y in Ys])
        arr = (C.c_void_p * nvec)(*[y.data_ptr() for y in Ys])
        out = torch.full((nvec,), np.nan, dtype=torch.float64, device="cuda")
        for call in range(2):
            rc = fn(nvec, x.data_ptr(), arr, length, out.data_ptr(), None)
            assert rc == 0, llg.load().llg_last_error()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            if length == n:   # same partition, order and tree as llg_dot_multi
                assert np.array_equal(got, ref), (nvec, length, call, got, ref)
            else:             # against a host sum in another order
                scale = max(np.abs(ref).max(), 1.0)
                assert np.abs(got - ref).max() <= 1e-13 * scale, (nvec, length, call, got, ref)
            out.fill_(np.nan)


def test_noalloc_multi_dot_rejects_oversize(gpu):
    import torch
    fn = _fn()
    x = torch.zeros(10, dtype=torch.float64, device="cuda")
    ys = [torch.zeros(10, dtype=torch.float64, device="cuda") for _ in range(17)]
    arr = (C.c_void_p * 17)(*[y.data_ptr() for y in ys])
    out = torch.zeros(17, dtype=torch.float64, device="cuda")
    assert fn(17, x.data_ptr(), arr, 10, out.data_ptr(), None) == -100
    assert b"LLG_NOALLOC_MAX_VECS" in llg.load().llg_last_error()
