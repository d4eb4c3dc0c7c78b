"""Our HLL SpMV against the reference's own GPU kernel, executed.

The reference's SPGPU HLL SpMV (spgpuDhellspmv, cuda/spgpu/kernels/
hell_dspmv.cu) is compiled from the psblas3 sources for sm_100a into
oracle/_ref/ and called on device copies of the same HLL arrays, the way
spmvHllDeviceDouble calls it (cuda/hlldev.c:185-207, y updated in place,
avgNzr = ceil(nnz/rows) as hlldev.c:45).  That build keeps nvcc's default
multiply-add contraction, so its sums round differently from the CPU
reference (and from ours, which follow the CPU reference bit for bit); the
bar is the FP64 SpMV tolerance |dy_i| <= 1e-13 * sum_j |a_ij x_j|."""
import numpy as np
import pytest

import oracle as O
from psblas3_b200 import gen

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _cases():
    yield "c1_pde3d_40", gen.pde3d(40, a=(1, 1, 1), b=(1 / np.sqrt(3),) * 3)
    yield "stencil27_40", gen.stencil27(40)
    irp, ja, va = gen.powerlaw(20000, kmax=300, seed=3)
    yield "powerlaw_20k", (irp, ja, va)


@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.0, 1.0), (3.0, 0.5)])
def test_hll_spmv_matches_reference_gpu_kernel(psb, alpha, beta):
    import torch
    ref = O.ref_gpu()
    if ref is None:
        pytest.skip("reference GPU kernel not built (psblas3 sources absent when building)")
    try:
        for name, (irp, ja, va) in _cases():
            n = len(irp) - 1
            ia, _, _ = gen.csr_to_coo(irp, ja, va)
            h = O.hll_from_coo(n, ia, ja, va, 32)
            rng = np.random.default_rng(7)
            x, y0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
            # the reference kernel on device copies of the HLL arrays
            dv = {k: torch.from_numpy(np.ascontiguousarray(h[k])).cuda() for k in ("val", "ja", "hkoffs", "irn")}
            dx = torch.from_numpy(x).cuda()
            dz = torch.from_numpy(y0.copy()).cuda()
            torch.cuda.synchronize()
            ref.hll_spmv(dz.data_ptr(), dz.data_ptr(), alpha, dv["val"].data_ptr(), dv["ja"].data_ptr(), 32,
                         dv["hkoffs"].data_ptr(), dv["irn"].data_ptr(), -(-len(ja) // n), n, dx.data_ptr(), beta)
            torch.cuda.synchronize()
            y_ref = dz.cpu().numpy()
            # ours through the C-ABI
            A = psb.HllMat.from_host_hll(n, 32, h["irn"], h["hkoffs"], h["ja"], h["val"], h["idiag"])
            X, Y = psb.DVect.bld(x), psb.DVect.bld(y0)
            A.spmv(alpha, X, beta, Y)
            y = Y.get_vect()
            scale = O.csr_csmv(irp, ja, np.abs(va), abs(alpha), np.abs(x), abs(beta), np.abs(y0))
            assert np.all(np.abs(y - y_ref) <= TOL * scale + 1e-300), name
            # and ours in the exact mode equals the CPU reference bit for bit
            A.set_wide_split(False)
            Y = psb.DVect.bld(y0)
            A.spmv(alpha, X, beta, Y)
            assert np.array_equal(Y.get_vect(), O.csr_csmv(irp, ja, va, alpha, x, beta, y0)), name
    finally:
        ref.close()


def test_cg_matches_reference_gpu_path(psb):
    """psb_dcg run on the reference's own GPU kernels (oracle/ref_cg.c over
    SPGPU) and this library's device CG reach the same tolerance within +-2
    iterations on an SPD 7-point operator with DIAG, and agree on x."""
    import torch
    ref = O.ref_gpu()
    if ref is None:
        pytest.skip("reference GPU kernels not built (psblas3 sources absent when building)")
    try:
        irp, ja, va = gen.poisson7(24)
        n = len(irp) - 1
        ia, _, _ = gen.csr_to_coo(irp, ja, va)
        h = O.hll_from_coo(n, ia, ja, va, 32)
        dinv = O.diag_prec_build(O.hll_get_diag(h, n))
        b = np.random.default_rng(9).uniform(-1, 1, n)
        dv = {k: torch.from_numpy(np.ascontiguousarray(h[k])).cuda() for k in ("val", "ja", "hkoffs", "irn")}
        d_dinv, d_b = torch.from_numpy(dinv).cuda(), torch.from_numpy(b).cuda()
        d_x = torch.zeros(n, dtype=torch.float64, device="cuda")
        it_ref, err_ref = ref.cg(n, dv["val"].data_ptr(), dv["ja"].data_ptr(), dv["hkoffs"].data_ptr(),
                                 dv["irn"].data_ptr(), -(-len(ja) // n), d_dinv.data_ptr(), d_b.data_ptr(),
                                 d_x.data_ptr(), 1e-9, 1000)
        x_ref = d_x.cpu().numpy()
        A = psb.HllMat.from_host_hll(n, 32, h["irn"], h["hkoffs"], h["ja"], h["val"], h["idiag"])
        P = psb.DiagPrec("DIAG").build(A)
        B, X = psb.DVect.bld(b), psb.DVect.bld(np.zeros(n))
        it, err = psb.psb_krylov("CG", A, P, B, X, eps=1e-9, itmax=1000)
        assert abs(it - it_ref) <= 2, (it, it_ref)
        assert err <= 1e-9 and err_ref <= 1e-9
        assert np.max(np.abs(X.get_vect() - x_ref)) <= 1e-7
    finally:
        ref.close()
