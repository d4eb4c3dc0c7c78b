"""GPU test of psbx_dot_noalloc, the dot-product entry point that allocates
nothing (for callers that cannot let a library call cudaMalloc: code that
owns all device memory through its own pool or budget, and latency-critical
loops where an allocation would synchronise the device).

It is compared through the C-ABI with the existing entry point
dotMultiVecDeviceDouble, on two calls in a row with different sizes (the
shared scratch keeps the previous call's contents), within the reduction
tolerance the other tests use: |d_new - d_ref| <= 1e-13 * sum|x_i y_i|.
This file is collected last so that a run stopping at its first failure has
run every other test already; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_dot_noalloc_matches_dot_entry(psb):
    import torch
    from psblas3_b200._lib import lib

    stream = lib.psb_cudaGetStream()
    for call, (n, cnt) in enumerate([(1_000_003, 3), (4097, 1)]):
        rng = np.random.default_rng(50 + call)
        a = rng.uniform(-1, 1, (n, cnt))
        b = rng.standard_normal((n, cnt))
        A, B = psb.DVect.bld(a if cnt > 1 else a[:, 0]), psb.DVect.bld(b if cnt > 1 else b[:, 0])
        ref = np.atleast_1d(psb.psb_gedot(A, B))  # existing entry: dotMultiVecDeviceDouble
        res = torch.full((cnt,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.psbx_dot_noalloc(C.c_void_p(res.data_ptr()), n, cnt, C.c_void_p(lib.psbx_multivec_data(A.h)),
                                  C.c_void_p(lib.psbx_multivec_data(B.h)), A.pitch, C.c_void_p(stream))
        assert rc == 0
        torch.cuda.synchronize()
        got = res.cpu().numpy()
        for k in range(cnt):
            scale = np.sum(np.abs(a[:, k] * b[:, k]))
            assert abs(got[k] - ref[k]) <= 1e-13 * scale, (call, k, got[k], ref[k])


def test_dot_noalloc_rejects_more_vectors_than_its_scratch(psb):
    import torch
    from psblas3_b200._lib import lib

    res = torch.zeros(9, dtype=torch.float64, device="cuda")
    x = torch.zeros(9 * 64, dtype=torch.float64, device="cuda")
    rc = lib.psbx_dot_noalloc(C.c_void_p(res.data_ptr()), 64, 9, C.c_void_p(x.data_ptr()),
                              C.c_void_p(x.data_ptr()), 64, None)
    assert rc == 1
    assert b"count must be between 1 and 8" in lib.psbx_last_error()
