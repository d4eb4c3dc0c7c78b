"""GPU parity of the device-resident Krylov solvers against the oracle's
restatement of psb_dcg / psb_dfcg / psb_dcgstab / psb_drgmres.

Bar (from the reference's own behaviour): same stop test; iteration count
within +-2 of the oracle's; final error estimate <= eps; the true residual
of the returned x within a small factor of eps*||b||."""
import numpy as np
import pytest

import oracle as O
from psblas3_b200 import gen

pytestmark = pytest.mark.gpu


def _mats(psb, irp, ja, va, fmt):
    n = len(irp) - 1
    ia, _, _ = gen.csr_to_coo(irp, ja, va)
    if fmt == "HLL":
        h = O.hll_from_coo(n, ia, ja, va, 32)
        return psb.HllMat.from_host_hll(n, 32, h["irn"], h["hkoffs"], h["ja"], h["val"], h["idiag"])
    if fmt == "ELL":
        e = O.ell_from_coo(n, ia, ja, va)
        return psb.EllMat.from_host_ell(n, e["nzm"], e["irn"], e["ja"], e["val"], e["idiag"], e["ldv"])
    return psb.CsrMat(n, irp, ja, va)


def _solve_both(psb, method, irp, ja, va, b, fmt="HLL", eps=1e-9, itmax=1000, istop=2, prec=True, irst=10):
    n = len(irp) - 1
    A = _mats(psb, irp, ja, va, fmt)
    P = psb.DiagPrec("DIAG" if prec else "NONE").build(A)
    B, X = psb.DVect.bld(b), psb.DVect.bld(np.zeros(n))
    it, err = psb.psb_krylov(method, A, P, B, X, eps=eps, itmax=itmax, istop=istop, irst=irst)
    x = X.get_vect()
    dinv = None
    if prec:
        ia, _, _ = gen.csr_to_coo(irp, ja, va)
        h = O.hll_from_coo(n, ia, ja, va, 32)
        dinv = O.diag_prec_build(O.hll_get_diag(h, n))
        assert np.array_equal(P.dv.get_vect(), dinv)  # prec build is bit-exact
    xo, ito, erro = O.krylov(method, irp, ja, va, b, dinv=dinv, eps=eps, itmax=itmax, istop=istop, irst=irst)
    return (x, it, err), (xo, ito, erro)


def test_bicgstab_c1(psb):
    """C1: pde3d 40^3 (a=1, b=(1,1,1)/sqrt3), HLL-32, DIAG, b = A*1, x0 = 0,
    eps = 1e-9, istop 2."""
    irp, ja, va = gen.pde3d(40, a=(1, 1, 1), b=(1 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    b = O.csr_csmv(irp, ja, va, 1.0, np.ones(n), 0.0, np.zeros(n))
    (x, it, err), (xo, ito, erro) = _solve_both(psb, "BICGSTAB", irp, ja, va, b)
    assert abs(it - ito) <= 2, (it, ito)
    assert err <= 1e-9 and erro <= 1e-9
    r = b - gen.csr_matvec(irp, ja, va, x)
    assert np.linalg.norm(r) <= 2e-9 * np.linalg.norm(b)
    assert np.max(np.abs(x - xo)) <= 1e-6


@pytest.mark.parametrize("fmt", ["HLL", "ELL", "CSR"])
@pytest.mark.parametrize("method", ["CG", "BICGSTAB"])
def test_methods_formats_poisson(psb, fmt, method):
    irp, ja, va = gen.poisson7(24)
    n = len(irp) - 1
    b = np.random.default_rng(3).uniform(-1, 1, n)
    (x, it, err), (xo, ito, erro) = _solve_both(psb, method, irp, ja, va, b, fmt=fmt, eps=1e-8)
    assert abs(it - ito) <= 2, (it, ito)
    assert err <= 1e-8
    r = b - gen.csr_matvec(irp, ja, va, x)
    assert np.linalg.norm(r) <= 2e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("istop", [1, 2, 3])
def test_stop_criteria(psb, istop):
    irp, ja, va = gen.pde3d(14, b=(0.5, 0.25, 0.0))
    n = len(irp) - 1
    b = np.random.default_rng(4).uniform(-1, 1, n)
    (x, it, err), (xo, ito, erro) = _solve_both(psb, "BICGSTAB", irp, ja, va, b, eps=1e-7, istop=istop)
    assert abs(it - ito) <= 2, (istop, it, ito)
    assert err <= 1e-7


def test_cg_no_prec_and_itmax(psb):
    irp, ja, va = gen.poisson7(16)
    n = len(irp) - 1
    b = np.random.default_rng(5).uniform(-1, 1, n)
    (x, it, err), (xo, ito, erro) = _solve_both(psb, "CG", irp, ja, va, b, prec=False, eps=1e-10)
    assert abs(it - ito) <= 2
    # itmax stops the solve with iter == itmax, err above eps (as the reference)
    (x, it, err), (xo, ito, erro) = _solve_both(psb, "CG", irp, ja, va, b, eps=1e-14, itmax=7)
    assert it == 7 and ito == 7 and err > 1e-14
    assert abs(err - erro) <= 1e-6 * erro


def test_zero_rhs_returns_at_once(psb):
    irp, ja, va = gen.poisson7(8)
    n = len(irp) - 1
    for method in ("CG", "BICGSTAB", "FCG", "RGMRES", "CGS", "BICG", "BICGSTABL"):
        (x, it, err), (xo, ito, erro) = _solve_both(psb, method, irp, ja, va, np.zeros(n))
        assert np.all(x == 0)
        assert it == ito


def test_unknown_method_is_an_error(psb):
    irp, ja, va = gen.poisson7(4)
    n = len(irp) - 1
    A = _mats(psb, irp, ja, va, "HLL")
    from psblas3_b200._lib import PsbxError
    with pytest.raises(PsbxError):
        psb.psb_krylov("QMR", A, None, psb.DVect.bld(np.ones(n)), psb.DVect(n))
    with pytest.raises(PsbxError):
        psb.psb_krylov("CG", A, None, psb.DVect.bld(np.ones(n)), psb.DVect(n), istop=7)
    # RGMRES: only istop 2 here; irst must be positive
    for istop, irst in ((1, 10), (3, 10), (2, 0)):
        with pytest.raises(PsbxError):
            psb.psb_krylov("RGMRES", A, None, psb.DVect.bld(np.ones(n)), psb.DVect(n), istop=istop, irst=irst)


@pytest.mark.parametrize("fmt", ["HLL", "ELL", "CSR"])
@pytest.mark.parametrize("irst", [4, 10, 30])
def test_rgmres_c1(psb, fmt, irst):
    """RGMRES (psb_drgmres.f90) on the nonsymmetric C1 operator with DIAG:
    iterations within +-2 of the oracle, the estimated and the true residual
    at the tolerance, the solution close to the oracle's."""
    irp, ja, va = gen.pde3d(20, a=(1, 1, 1), b=(1 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    b = O.csr_csmv(irp, ja, va, 1.0, np.ones(n), 0.0, np.zeros(n))
    (x, it, err), (xo, ito, erro) = _solve_both(psb, "RGMRES", irp, ja, va, b, fmt=fmt, eps=1e-9, irst=irst)
    assert abs(it - ito) <= 2, (it, ito)
    assert err <= 1e-9 and erro <= 1e-9
    r = b - gen.csr_matvec(irp, ja, va, x)
    assert np.linalg.norm(r) <= 2e-9 * np.linalg.norm(b)
    assert np.max(np.abs(x - xo)) <= 1e-6


@pytest.mark.parametrize("istop", [1, 2, 3])
@pytest.mark.parametrize("fmt", ["HLL", "CSR"])
def test_fcg_spd(psb, istop, fmt):
    """FCG (psb_dfcg.F90) on an SPD 7-point operator: iterations within +-2
    of the oracle, error at the tolerance; FCG and CG agree on SPD input."""
    irp, ja, va = gen.poisson7(22)
    n = len(irp) - 1
    b = np.random.default_rng(11).uniform(-1, 1, n)
    (x, it, err), (xo, ito, erro) = _solve_both(psb, "FCG", irp, ja, va, b, fmt=fmt, eps=1e-9, istop=istop)
    assert abs(it - ito) <= 2, (it, ito)
    assert err <= 1e-9
    ia, _, _ = gen.csr_to_coo(irp, ja, va)
    dinv = O.diag_prec_build(O.hll_get_diag(O.hll_from_coo(n, ia, ja, va, 32), n))
    _, ito_cg, _ = O.krylov("CG", irp, ja, va, b, dinv=dinv, eps=1e-9, istop=istop)
    assert abs(ito_cg - ito) <= 2, (ito_cg, ito)
    r = b - gen.csr_matvec(irp, ja, va, x)
    assert np.linalg.norm(r) <= 1e-6 * np.linalg.norm(b)


def test_itmax_fcg_and_rgmres(psb):
    """itmax: FCG stops at itmax; RGMRES tests itmax only at a restart, so
    it finishes the running cycle (irst = 10 -> 10 iterations for itmax 7),
    as the reference does."""
    irp, ja, va = gen.poisson7(16)
    n = len(irp) - 1
    b = np.random.default_rng(5).uniform(-1, 1, n)
    (x, it, err), (xo, ito, erro) = _solve_both(psb, "FCG", irp, ja, va, b, eps=1e-14, itmax=7)
    assert it == 7 and ito == 7 and err > 1e-14
    assert abs(err - erro) <= 1e-6 * erro
    (x, it, err), (xo, ito, erro) = _solve_both(psb, "RGMRES", irp, ja, va, b, eps=1e-14, itmax=7, irst=10)
    assert it == 10 and ito == 10 and err > 1e-14
    assert abs(err - erro) <= 1e-6 * erro


@pytest.mark.parametrize("method", ["CG", "FCG", "CGS", "BICG", "BICGSTAB", "BICGSTABL", "RGMRES"])
def test_wide_hacks_in_solvers(psb, method):
    """Row-sorted SPD power-law matrix whose leading hacks take the wide-hack
    path (products formed by all blocks, then each row added in order by a
    warp per hack, before every product): every method matches the oracle's
    iteration count within +-2 and reaches the tolerance."""
    irp, ja, va = gen.powerlaw_spd(40000, kmax=3000, seed=8)
    irp, ja, va, _ = gen.sort_rows_by_length(irp, ja, va)
    n = len(irp) - 1
    b = np.random.default_rng(6).uniform(-1, 1, n)
    (x, it, err), (xo, ito, erro) = _solve_both(psb, method, irp, ja, va, b, eps=1e-10, itmax=2000)
    assert abs(it - ito) <= 2, (it, ito)
    assert err <= 1e-10
    r = b - gen.csr_matvec(irp, ja, va, x)
    assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("istop", [1, 2, 3])
@pytest.mark.parametrize("fmt", ["HLL", "ELL", "CSR"])
@pytest.mark.parametrize("method", ["CGS", "BICG"])
def test_cgs_bicg_c1(psb, method, istop, fmt):
    """CGS (psb_dcgs.f90) and BiCG (psb_dbicg.f90, A^T products on a
    transposed copy) on the nonsymmetric C1-type operator with DIAG:
    iterations within +-2 of the oracle, tolerance reached, x close."""
    irp, ja, va = gen.pde3d(20, a=(1, 1, 1), b=(1 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    b = O.csr_csmv(irp, ja, va, 1.0, np.ones(n), 0.0, np.zeros(n))
    (x, it, err), (xo, ito, erro) = _solve_both(psb, method, irp, ja, va, b, fmt=fmt, eps=1e-9, istop=istop)
    assert abs(it - ito) <= 2, (it, ito)
    assert err <= 1e-9
    assert np.max(np.abs(x - xo)) <= 1e-6


@pytest.mark.parametrize("irst", [1, 2, 4])
@pytest.mark.parametrize("istop", [1, 2])
def test_bicgstabl_c1(psb, irst, istop):
    """BiCGSTAB(L) (psb_dcgstabl.f90, L = irst, left preconditioned, stop test
    on the preconditioned residual) on the C1-type operator: iterations
    within +-2 of the oracle (they move in steps of L), tolerance reached,
    x equal to the oracle's to 1e-8."""
    irp, ja, va = gen.pde3d(20, a=(1, 1, 1), b=(1 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    b = O.csr_csmv(irp, ja, va, 1.0, np.ones(n), 0.0, np.zeros(n))
    (x, it, err), (xo, ito, erro) = _solve_both(psb, "BICGSTABL", irp, ja, va, b, eps=1e-9, istop=istop, irst=irst)
    assert abs(it - ito) <= 2, (it, ito)
    assert err <= 1e-9
    assert np.max(np.abs(x - xo)) <= 1e-8


@pytest.mark.parametrize("method", ["CG", "BICGSTAB"])
def test_repeated_solves_replay_kept_graph(psb, method):
    """Calls with the same matrix view and vectors replay the iteration graph
    kept from the first call: the same iterations, error and bits; new values
    in the same right-hand side vector solve the new system; a nonzero
    initial guess is honoured; another vector is another graph."""
    irp, ja, va = gen.pde3d(14, a=(1, 1, 1), b=(1 / np.sqrt(3),) * 3) if method == "BICGSTAB" else gen.poisson7(14)
    n = len(irp) - 1
    import torch
    d = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
    A = psb.HllMat.from_csr_device(n, n, len(ja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), 32)
    P = psb.DiagPrec("DIAG").build(A)
    rng = np.random.default_rng(11)
    b1, b2, x0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    B, X = psb.DVect.bld(b1), psb.DVect(n)
    runs = []
    for _ in range(3):
        X.zero()
        it, err = psb.psb_krylov(method, A, P, B, X, eps=1e-10, itmax=2000)
        runs.append((it, err, X.get_vect()))
    for it, err, x in runs[1:]:
        assert it == runs[0][0] and err == runs[0][1] and np.array_equal(x, runs[0][2])
    B.set_vect(b2)
    X.set_vect(x0)
    it, err = psb.psb_krylov(method, A, P, B, X, eps=1e-10, itmax=2000)
    assert err <= 1e-10
    r = b2 - gen.csr_matvec(irp, ja, va, X.get_vect())
    assert np.linalg.norm(r) <= 1e-9 * np.linalg.norm(b2)
    # a second solution vector: its own graph, same answer as the first one's
    X2 = psb.DVect(n)
    X.zero()
    it_a, err_a = psb.psb_krylov(method, A, P, B, X, eps=1e-10, itmax=2000)
    it_b, err_b = psb.psb_krylov(method, A, P, B, X2, eps=1e-10, itmax=2000)
    assert (it_a, err_a) == (it_b, err_b) and np.array_equal(X.get_vect(), X2.get_vect())


@pytest.mark.parametrize("fmt", ["HLL", "ELL", "CSR"])
def test_random_systems_cg_bicgstab(psb, fmt):
    """Seeded random diagonally dominant systems (rows of 0 .. 12 random
    off-diagonal entries, the diagonal their absolute sum plus 1): CG on the
    symmetric ones (A + A^T), BiCGSTAB on the nonsymmetric ones, DIAG: the
    device solver and the oracle reach the tolerance within +-2 iterations
    and agree on x."""
    for seed in range(4):
        rng = np.random.default_rng(4000 + seed)
        n = int(rng.integers(200, 3000))
        k = rng.integers(0, 13, n)
        ia = np.repeat(np.arange(1, n + 1), k)
        ja = rng.integers(1, n + 1, len(ia))
        va = rng.standard_normal(len(ia))
        for sym, method in ((True, "CG"), (False, "BICGSTAB")):
            ii, jj, vv = (np.concatenate([ia, ja]), np.concatenate([ja, ia]), np.concatenate([va, va])) if sym \
                else (ia, ja, va)
            keep = ii != jj
            ii, jj, vv = ii[keep], jj[keep], vv[keep]
            absum = np.bincount(ii - 1, weights=np.abs(vv), minlength=n)
            ii = np.concatenate([ii, np.arange(1, n + 1)])
            jj = np.concatenate([jj, np.arange(1, n + 1)])
            vv = np.concatenate([vv, absum + 1.0])
            fi, fj, fv = O.coo_fix(n, ii, jj, vv)
            irp, cja, cva = O.csr_from_coo(n, fi, fj, fv)
            b = rng.uniform(-1, 1, n)
            (x, it, err), (xo, ito, erro) = _solve_both(psb, method, irp, cja, cva, b, fmt=fmt, eps=1e-9)
            assert abs(it - ito) <= 2, (seed, method, it, ito)
            assert err <= 1e-9 and erro <= 1e-9
            assert np.max(np.abs(x - xo)) <= 1e-7 * max(1.0, np.max(np.abs(xo)))
