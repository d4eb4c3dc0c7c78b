"""GPU tests of psbx_dmixed_cg, the single-system mixed-precision CG (FP32
iterations with FP64-accumulated dots, FP64 residual replacement and stop
test).

Bar: the true relative residual ||b - A x|| / ||b||, recomputed here by the
oracle's FP64 CSR product, is at most the tolerance (1e-10); the solution
agrees with the oracle's FP64 CG solution within cond-scaled bounds; the
inner iterations stay close to the FP64 CG's (the replacement keeps the
Krylov space instead of restarting it).  Operators: the 7-point Poisson
operator (short rows), the anisotropic 2-D operator of the batched
workload at eps 1e-2 and 1e-3, and a power-law SPD matrix stored with its
rows in length order (wide hacks).
"""
import numpy as np
import pytest

import oracle as O
from psblas3_b200 import gen

pytestmark = pytest.mark.gpu


def _setup(psb, irp, ja, va, seed=0, perm=False):
    import torch
    n = len(irp) - 1
    d = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
    dp = None
    if perm:
        dp = torch.from_numpy(np.argsort(-np.diff(irp), kind="stable").astype(np.int32)).cuda()
    A = psb.HllMat.from_csr_device(n, n, len(ja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), 32,
                                   None if dp is None else dp.data_ptr())
    P = psb.DiagPrec("DIAG").build(A)
    ustar = np.random.default_rng(seed).uniform(0, 1, n)
    b = O.csr_csmv(irp, ja, va, 1.0, ustar, 0.0, np.zeros(n))
    return n, A, P, b


def _true_rel_res(irp, ja, va, b, x):
    r = O.csr_csmv(irp, ja, va, -1.0, x, 1.0, b)
    return np.linalg.norm(r) / np.linalg.norm(b)


@pytest.mark.parametrize("case", ["poisson40", "aniso_1e-2", "aniso_1e-3", "powerlaw_sorted"])
def test_mixed_cg_reaches_fp64_tolerance(psb, case):
    if case == "poisson40":
        irp, ja, va = gen.poisson7(40)
        perm = False
    elif case.startswith("aniso"):
        irp, ja, va = gen.aniso2d(160, float(case.split("_")[1]))
        perm = False
    else:
        irp, ja, va = gen.powerlaw_spd(60_000, kmax=2000, seed=3)
        perm = True
    n, A, P, b = _setup(psb, irp, ja, va, perm=perm)
    X = psb.DVect(n)
    it, err, nref = psb.psb_mixed_cg(A, P, psb.DVect.bld(b), X, eps=1e-10, itmax=20000)
    x = X.get_vect()
    rr = _true_rel_res(irp, ja, va, b, x)
    assert err <= 1e-10 and rr <= 1e-10 * (1 + 1e-6), (err, rr)
    # the FP64 device CG on the same system
    X64 = psb.DVect(n)
    it64, err64 = psb.psb_krylov("CG", A, P, psb.DVect.bld(b), X64, eps=1e-10, itmax=20000)
    assert err64 <= 1e-10
    assert it <= 1.25 * it64 + 10, (it, it64, nref)
    assert nref >= 2
    print(f"{case}: mixed {it} inner / {nref} replacements, FP64 CG {it64}")


def test_mixed_cg_matches_oracle_solution(psb):
    irp, ja, va = gen.poisson7(30)
    n, A, P, b = _setup(psb, irp, ja, va, seed=4)
    X = psb.DVect(n)
    it, err, nref = psb.psb_mixed_cg(A, P, psb.DVect.bld(b), X, eps=1e-10)
    xo, ito, erro = O.krylov("CG", irp, ja, va, b, dinv=O.diag_prec_build(np.full(n, 6.0)), eps=1e-10)
    # both have relative residual <= 1e-10; cond(A) ~ 4 (n+1)^2 / pi^2 ~ 390
    assert np.max(np.abs(X.get_vect() - xo)) <= 390 * 2e-10 * np.max(np.abs(xo))
    assert abs(it - ito) <= 0.1 * ito + 5, (it, ito)


def test_mixed_cg_nonzero_start_and_no_prec(psb):
    irp, ja, va = gen.poisson7(20)
    n, A, P, b = _setup(psb, irp, ja, va, seed=5)
    x0 = np.random.default_rng(9).uniform(-1, 1, n)
    X = psb.DVect.bld(x0)
    it, err, nref = psb.psb_mixed_cg(A, None, psb.DVect.bld(b), X, eps=1e-10, delta=0.05)
    assert err <= 1e-10 and _true_rel_res(irp, ja, va, b, X.get_vect()) <= 1e-10 * (1 + 1e-6)


def test_mixed_cg_itmax_and_errors(psb):
    from psblas3_b200._lib import PsbxError
    irp, ja, va = gen.poisson7(20)
    n, A, P, b = _setup(psb, irp, ja, va)
    X = psb.DVect(n)
    it, err, nref = psb.psb_mixed_cg(A, P, psb.DVect.bld(b), X, eps=1e-10, itmax=5)
    assert it == 5 and err > 1e-10
    # the returned x is the FP64 solution after the last replacement
    assert abs(_true_rel_res(irp, ja, va, b, X.get_vect()) - err) <= 1e-12
    with pytest.raises(PsbxError):
        psb.psb_mixed_cg(A, P, psb.DVect.bld(b), X, delta=1.5)
