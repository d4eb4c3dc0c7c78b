"""GPU tests of psbx_dot_noalloc, the dot-product entry point that allocates
nothing.  It exists for callers that cannot let a library call cudaMalloc:
code that owns all device memory through its own pool or a fixed budget, and
latency-critical loops where an allocation would synchronise the device.

The results are compared through the C-ABI with the existing entry point
dotMultiVecDeviceDouble, on two calls in a row with different sizes (the
shared scratch keeps the previous call's contents).  Both run the same
reduction kernel on the same grid, so the results must be the same bits; the
reduction tolerance the other tests use (|d_new - d_ref| <= 1e-13 *
sum|x_i y_i|) is checked as well, so a failure says which bar broke.
A second test runs the entry point in a fresh process that never creates the
library's context and checks that free device memory does not move.
This file is collected last so that a run stopping at its first failure has
run every other test already; it also passes on its own in a fresh process.
"""
import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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
            assert got[k] == ref[k], (call, k, got[k], ref[k])


def test_dot_noalloc_rejects_more_vectors_than_its_scratch(psb):
    import torch
    from psblas3_b200._lib import lib

    res = torch.zeros(9, dtype=torch.float64, device="cuda")
    x = torch.zeros(9 * 64, dtype=torch.float64, device="cuda")
    rc = lib.psbx_dot_noalloc(C.c_void_p(res.data_ptr()), 64, 9, C.c_void_p(x.data_ptr()),
                              C.c_void_p(x.data_ptr()), 64, None)
    assert rc == 1
    assert b"count must be between 1 and 8" in lib.psbx_last_error()


_CHILD = textwrap.dedent(r"""
    import ctypes as C, os, sys
    sys.path.insert(0, sys.argv[1])
    # load the library before the CUDA context exists, so that (with eager
    # module loading) its device code and static arrays are placed when the
    # context is created, not at the first call
    lib = C.CDLL(os.path.join(sys.argv[1], "psblas3_b200", "libpsbx.so"))
    lib.psbx_dot_noalloc.restype = C.c_int
    lib.psbx_dot_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                     C.c_void_p]
    import torch
    n = 3_000_001
    g = torch.Generator(device="cuda").manual_seed(7)
    x = torch.rand(4 * n, dtype=torch.float64, device="cuda", generator=g)
    y = torch.rand(4 * n, dtype=torch.float64, device="cuda", generator=g)
    res = torch.zeros(8, dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    out = []
    for k, (m, cnt) in enumerate([(n, 1), (n, 4), (1000, 2), (n, 3), (17, 1)]):
        rc = lib.psbx_dot_noalloc(res.data_ptr(), m, cnt, x.data_ptr(), y.data_ptr(), n, s)
        assert rc == 0, rc
        torch.cuda.synchronize()
        out.append(res[:cnt].cpu().tolist())
    free1 = torch.cuda.mem_get_info()[0]
    ref = [float(torch.dot(x[:n], y[:n])), float(torch.dot(x[:17], y[:17]))]
    print("FREE", free0, free1)
    assert free0 == free1, (free0, free1)
    assert abs(out[0][0] - ref[0]) <= 1e-12 * ref[0]
    assert abs(out[4][0] - ref[1]) <= 1e-12 * ref[1]
    assert out[3] == out[1][:3], (out[3], out[1])
    print("NOALLOC_OK")
""")


def test_dot_noalloc_allocates_no_device_memory():
    """In a process that never creates the library's context (no gpuInit, no
    other entry point), several calls leave the device's free memory exactly
    where it was: the entry point allocates nothing, on its first call or
    later ones."""
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    p = subprocess.run([sys.executable, "-c", _CHILD, ROOT], env=env, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0 and "NOALLOC_OK" in p.stdout, p.stdout + p.stderr
