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


def _random_spd(seed):
    """Symmetric, diagonally dominant: rows of 0 .. 12 random off-diagonal
    entries mirrored, diagonal = absolute row sum + 1 (1-based CSR)."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(500, 5000))
    k = rng.integers(0, 13, n)
    ia = np.repeat(np.arange(1, n + 1), k)
    ja = rng.integers(1, n + 1, len(ia))
    va = rng.standard_normal(len(ia))
    ii, jj, vv = np.concatenate([ia, ja]), np.concatenate([ja, ia]), np.concatenate([va, va])
    keep = ii != jj
    ii, jj, vv = ii[keep], jj[keep], vv[keep]
    absum = np.bincount(ii - 1, weights=np.abs(vv), minlength=n)
    ii = np.concatenate([ii, np.arange(1, n + 1)])
    jj = np.concatenate([jj, np.arange(1, n + 1)])
    vv = np.concatenate([vv, absum + 1.0])
    fi, fj, fv = O.coo_fix(n, ii, jj, vv)
    return O.csr_from_coo(n, fi, fj, fv)


def test_mixed_cg_random_systems(psb):
    """Seeded random SPD systems, in stored order and with the rows in length
    order (permuted layout): the mixed solve reaches ||b - Ax|| <= 1e-10 ||b||
    (checked in FP64 on the host) and the batch engine (stored order; it
    takes no permuted layout), one and eight right-hand sides, does too."""
    import torch
    for seed in range(4):
        irp, ja, va = _random_spd(5000 + seed)
        for perm in (True, False):  # the engine takes the stored order (the last one)
            n, A, P, b = _setup(psb, irp, ja, va, seed=seed, perm=perm)
            B, X = psb.DVect.bld(b), psb.DVect(n)
            it, err, nref = psb.psb_mixed_cg(A, P, B, X, eps=1e-10, itmax=5000)
            assert err <= 1e-10 and _true_rel_res(irp, ja, va, b, X.get_vect()) <= 1.01e-10, (seed, perm)
        A.make_single()
        for k in (1, 8):
            rhs = np.random.default_rng(seed).uniform(-1, 1, (n, k))
            db = torch.from_numpy(np.ascontiguousarray(rhs.reshape(-1))).cuda()
            dx = torch.zeros_like(db)
            eng = psb.BatchSolver(1, n, k)
            s = eng.add(A, db, dx, P.dv.data_ptr, eps=1e-10)
            eng.run()
            st, outer, its, errs = eng.poll(s)
            x = dx.cpu().numpy().reshape(n, k)
            assert st == 1, (seed, k, st)
            for j in range(k):
                assert _true_rel_res(irp, ja, va, rhs[:, j], x[:, j]) <= 1.01e-10, (seed, k, j)
            eng.free()
