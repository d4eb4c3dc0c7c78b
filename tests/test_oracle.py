"""CPU tests of the oracle (the restated reference CPU path) against the
reference's own known-answer tests and structural facts of its formats.
No GPU needed."""
import json
import os

import numpy as np
import pytest

import oracle as O
from psblas3_b200 import gen

HERE = os.path.dirname(os.path.abspath(__file__))


def _kats():
    with open(os.path.join(HERE, "golden", "usmv_kats.json")) as f:
        return json.load(f)["cases"]


def _vecops():
    with open(os.path.join(HERE, "golden", "vecop_kats.json")) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("fmt", ["CSR", "HLL", "ELL"])
def test_usmv_kats_all_formats(fmt):
    """test/torture/psb_d_mvsv_tester.f90: every d_usmv case, exact equality,
    through each format's csmv (the tester reads afmt from stdin)."""
    cases = _kats()
    assert len(cases) == 24
    for c in cases:
        m = c["m"]
        ia, ja, va = O.coo_fix(m, c["ia"], c["ja"], c["val"])
        y = np.array(c["y_before"], float)
        x = np.array(c["x"], float)
        t = c["trans"].upper()
        if fmt == "CSR":
            irp, cja, cv = O.csr_from_coo(m, ia, ja, va)
            out = O.csr_csmv(irp, cja, cv, c["alpha"], x, c["beta"], y, trans=t)
        elif fmt == "HLL":
            h = O.hll_from_coo(m, ia, ja, va, hksz=4)
            out = O.hll_csmv(h, m, c["alpha"], x, c["beta"], y, trans=t)
        else:
            e = O.ell_from_coo(m, ia, ja, va)
            out = O.ell_csmv(e, m, c["alpha"], x, c["beta"], y, trans=t)
        assert np.array_equal(out, np.array(c["y_after"], float)), (fmt, c["name"], out, c["y_after"])


def test_vecoperation_kats():
    """test/kernel/vecoperation.f90 constant-vector checks (exact)."""
    n = 17
    for c in _vecops():
        x = np.full(n, c["x"])
        if c["op"] == "axpby":
            out = O.axpby(c["alpha"], x, c["beta"], np.full(n, c["y"]))
            assert np.all(out == c["expect"]), c
        elif c["op"] == "axpbyz":
            out = O.axpbyz(c["alpha"], x, c["beta"], np.full(n, c["y"]))
            assert np.all(out == c["expect"]), c
        elif c["op"] == "mlt":
            out = O.mlt(c["alpha"], x, np.full(n, c["y"]), c["beta"], np.zeros(n))
            assert np.all(out == c["expect"]), c
        elif c["op"] == "dot":
            assert O.dot(x, np.full(n, c["y"])) == n * c["expect_per_entry"]
        elif c["op"] == "amax":
            assert O.amax(x) == c["expect"]


def test_coo_fix_sorts_and_adds_duplicates():
    ia = [3, 1, 2, 1, 3, 1]
    ja = [1, 2, 2, 2, 3, 1]
    va = [1.0, 2.0, 3.0, 4.0, 5.0, 6.0]
    ia2, ja2, va2 = O.coo_fix(3, ia, ja, va)
    assert list(ia2) == [1, 1, 2, 3, 3]
    assert list(ja2) == [1, 2, 2, 1, 3]
    assert list(va2) == [6.0, 6.0, 3.0, 1.0, 5.0]


def test_hll_layout_c1_sizes():
    """C1 operator (7-pt, 40^3): n = 64,000, nnz = 438,400, HLL-32
    allocation 442,240 slots; hack offsets multiples of 32; padding = last
    column of the row, value 0."""
    irp, ja, va = gen.pde3d(40, a=(1, 1, 1), b=(1 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    assert n == 64000 and len(ja) == 438400
    ia, _, _ = gen.csr_to_coo(irp, ja, va)
    h = O.hll_from_coo(n, ia, ja, va, hksz=32)
    assert h["hkoffs"][-1] == 442240
    assert np.all(h["hkoffs"] % 32 == 0)
    assert np.array_equal(h["irn"], np.diff(irp))
    # padding check on every hack
    for k in range(len(h["hkoffs"]) - 1):
        w = (h["hkoffs"][k + 1] - h["hkoffs"][k]) // 32
        blk_ja = h["ja"][h["hkoffs"][k]: h["hkoffs"][k + 1]].reshape(w, 32)
        blk_v = h["val"][h["hkoffs"][k]: h["hkoffs"][k + 1]].reshape(w, 32)
        for ii in range(32):
            r = k * 32 + ii
            L = h["irn"][r]
            assert np.array_equal(blk_ja[:L, ii], ja[irp[r] - 1: irp[r + 1] - 1])
            if L < w:
                assert np.all(blk_ja[L:, ii] == ja[irp[r + 1] - 2])
                assert np.all(blk_v[L:, ii] == 0.0)
        if k > 40:
            break
    # diagonal positions
    for r in range(0, n, 997):
        row = ja[irp[r] - 1: irp[r + 1] - 1]
        assert h["idiag"][r] == int(np.where(row == r + 1)[0][0]) + 1


def test_hll_last_hack_and_empty_rows():
    """Last hack pre-filled with ja = nr, val = 0 (psi_d_convert_hll_from_coo
    :94-96); an empty row pads with the hack's first COO column."""
    nr = 37  # two hacks of 32, the second one ragged
    ia = [1, 1, 2, 5, 33, 33, 37]
    ja = [1, 4, 2, 9, 30, 33, 1]
    va = [1.0, 2, 3, 4, 5, 6, 7]
    h = O.hll_from_coo(nr, ia, ja, va, hksz=32)
    assert list(h["hkoffs"]) == [0, 64, 64 + 64]
    # row 3 (empty) pads with jac(1) of hack 1 = 1
    blk = h["ja"][0:64].reshape(2, 32)
    assert blk[0, 2] == 1 and blk[1, 2] == 1
    # second hack: rows 33..37 stored, rows 38..64 keep ja = nr
    blk2 = h["ja"][64:128].reshape(2, 32)
    assert list(blk2[:, 0]) == [30, 33]
    assert blk2[0, 5] == 37 and blk2[1, 5] == 37
    assert np.all(h["val"][64:128].reshape(2, 32)[:, 5:] == 0)
    # row 34 (empty) pads with the hack's first COO column (30)
    assert blk2[0, 1] == 30
    assert h["idiag"][32] == 2 and h["idiag"][0] == 1 and h["idiag"][1] == 1


@pytest.mark.parametrize("maker", ["pde3d", "stencil27", "powerlaw"])
def test_formats_agree_bitwise(maker):
    """HLL, ELL and CSR csmv give identical bits (same per-row order)."""
    if maker == "pde3d":
        irp, ja, va = gen.pde3d(12, b=(1 / np.sqrt(3),) * 3)
    elif maker == "stencil27":
        irp, ja, va = gen.stencil27(10)
    else:
        irp, ja, va = gen.powerlaw(3000, kmax=600, seed=3)
    n = len(irp) - 1
    ia, _, _ = gen.csr_to_coo(irp, ja, va)
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, n)
    y0 = rng.uniform(-1, 1, n)
    h = O.hll_from_coo(n, ia, ja, va, 32)
    e = O.ell_from_coo(n, ia, ja, va)
    for a, b in [(1.0, 0.0), (-1.0, 1.0), (2.5, -0.5)]:
        yc = O.csr_csmv(irp, ja, va, a, x, b, y0)
        yh = O.hll_csmv(h, n, a, x, b, y0)
        ye = O.ell_csmv(e, n, a, x, b, y0)
        assert np.array_equal(yc, yh) and np.array_equal(yc, ye)
        ref = a * gen.csr_matvec(irp, ja, va, x) + b * y0
        assert np.allclose(yc, ref, rtol=1e-12, atol=1e-12)


def test_hll_get_diag_and_prec():
    irp, ja, va = gen.pde3d(8, b=(0.3, 0.2, 0.1))
    n = len(irp) - 1
    ia, _, _ = gen.csr_to_coo(irp, ja, va)
    h = O.hll_from_coo(n, ia, ja, va, 32)
    d = O.hll_get_diag(h, n)
    dd = np.array([va[irp[i] - 1 + np.where(ja[irp[i] - 1: irp[i + 1] - 1] == i + 1)[0][0]] for i in range(n)])
    assert np.array_equal(d, dd)
    dinv = O.diag_prec_build(np.concatenate([d, [0.0]]))
    assert dinv[-1] == 1.0 and np.array_equal(dinv[:-1], 1.0 / d)


def test_oracle_bicgstab_c1_small():
    """BiCGSTAB + DIAG on the pde3d operator (a=1, b=(1,1,1)/sqrt3), b = A*1,
    x0 = 0, istop 2 (C1 at a reduced grid)."""
    irp, ja, va = gen.pde3d(16, b=(1 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    ia, _, _ = gen.csr_to_coo(irp, ja, va)
    h = O.hll_from_coo(n, ia, ja, va, 32)
    dinv = O.diag_prec_build(O.hll_get_diag(h, n))
    b = O.csr_csmv(irp, ja, va, 1.0, np.ones(n), 0.0, np.zeros(n))
    x, it, err = O.krylov("BICGSTAB", irp, ja, va, b, dinv=dinv, eps=1e-9, itmax=1000)
    assert err <= 1e-9 and 5 < it < 200
    r = b - gen.csr_matvec(irp, ja, va, x)
    assert np.linalg.norm(r) <= 1.01e-9 * np.linalg.norm(b)
    assert np.max(np.abs(x - 1)) < 1e-6


@pytest.mark.parametrize("istop", [1, 2, 3])
def test_oracle_cg_poisson(istop):
    irp, ja, va = gen.poisson7(12)
    n = len(irp) - 1
    rng = np.random.default_rng(1)
    b = rng.uniform(-1, 1, n)
    dinv = 1.0 / np.full(n, 6.0)
    x, it, err = O.krylov("CG", irp, ja, va, b, dinv=dinv, eps=1e-8, itmax=500, istop=istop)
    assert err <= 1e-8 and it > 5
    if istop == 2:
        r = b - gen.csr_matvec(irp, ja, va, x)
        assert np.linalg.norm(r) <= 1.01e-8 * np.linalg.norm(b)


def test_oracle_itmax_and_zero_rhs():
    irp, ja, va = gen.poisson7(6)
    n = len(irp) - 1
    b = np.random.default_rng(2).uniform(-1, 1, n)
    _, it, err = O.krylov("CG", irp, ja, va, b, eps=1e-30, itmax=3)
    assert it == 3 and err > 1e-30
    # b = 0 with x0 = 0: ||b|| = 0 so the test is ||r|| <= eps at once
    _, it, err = O.krylov("BICGSTAB", irp, ja, va, np.zeros(n), eps=1e-9, itmax=50)
    assert it == 0 and err == 0.0


def test_oracle_fcg_and_rgmres():
    """FCG equals CG on an SPD operator (same iterations, same error to a
    few ulps of the tolerance); RGMRES converges on the nonsymmetric C1-type
    operator with its estimated residual equal to the true one; the
    restated drotg gives the rotation of (3, 4) to rounding."""
    import ctypes as C
    from psblas3_b200 import gen
    irp, ja, va = gen.poisson7(12)
    n = len(irp) - 1
    b = np.random.default_rng(2).uniform(-1, 1, n)
    ia, _, _ = gen.csr_to_coo(irp, ja, va)
    dinv = O.diag_prec_build(O.hll_get_diag(O.hll_from_coo(n, ia, ja, va, 32), n))
    _, it_cg, e_cg = O.krylov("CG", irp, ja, va, b, dinv=dinv, eps=1e-10)
    x, it_f, e_f = O.krylov("FCG", irp, ja, va, b, dinv=dinv, eps=1e-10)
    assert it_f == it_cg and abs(e_f - e_cg) <= 1e-3 * e_cg
    irp, ja, va = gen.pde3d(10, a=(1, 1, 1), b=(1 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    b = O.csr_csmv(irp, ja, va, 1.0, np.ones(n), 0.0, np.zeros(n))
    # the reference keeps the rotation cosines in single precision, so over
    # long cycles its residual estimate drifts from the true residual; up to
    # 30 steps per cycle they agree here
    for irst in (3, 10, 30):
        x, it, err = O.krylov("RGMRES", irp, ja, va, b, eps=1e-10, itmax=2000, irst=irst)
        r = b - O.csr_csmv(irp, ja, va, 1.0, x, 0.0, np.zeros(n))
        assert err <= 1e-10
        assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.5e-10
    a, bb, c, s = (C.c_double(v) for v in (3.0, 4.0, 0.0, 0.0))
    O.lib().or_drotg(C.byref(a), C.byref(bb), C.byref(c), C.byref(s))
    assert np.allclose((a.value, c.value, s.value), (5.0, 0.6, 0.8), rtol=4e-16, atol=0)
    assert abs(c.value ** 2 + s.value ** 2 - 1.0) <= 1e-15
    with pytest.raises(ValueError):
        O.krylov("RGMRES", irp, ja, va, b, istop=1)


def _random_coo(draw_seed, nr, nc, density, dup):
    rng = np.random.default_rng(draw_seed)
    nz = int(nr * nc * density)
    ia = rng.integers(1, nr + 1, nz)
    ja = rng.integers(1, nc + 1, nz)
    if dup and nz:  # repeat some entries: coo_fix adds them
        k = rng.integers(0, nz, max(1, nz // 5))
        ia, ja = np.concatenate([ia, ia[k]]), np.concatenate([ja, ja[k]])
    val = rng.standard_normal(len(ia))
    return ia, ja, val


def test_random_matrices_formats_agree():
    """Seeded random matrices (rectangular, empty rows, duplicate entries,
    hack sizes 1 .. 64): after psb_d_fix_coo every format's csmv gives the
    CSR csmv's bits, and the HLL layout keeps the reference's invariants --
    hack width = its longest row, padding value 0 repeating the row's last
    column (the hack's first COO column for an empty row), idiag = 1-based
    diagonal position where the row has one."""
    for seed in range(40):
        rng = np.random.default_rng(1000 + seed)
        nr, nc = int(rng.integers(1, 90)), int(rng.integers(1, 90))
        ia, ja, val = _random_coo(seed, nr, nc, float(rng.uniform(0.0, 0.3)), bool(seed % 2))
        ia, ja, val = O.coo_fix(nr, ia, ja, val)
        assert np.all(np.diff(ia.astype(np.int64) * (nc + 1) + ja) > 0)  # sorted, no duplicates left
        irp, cja, cval = O.csr_from_coo(nr, ia, ja, val)
        x, y0 = rng.uniform(-1, 1, nc), rng.uniform(-1, 1, nr)
        a, b = float(rng.choice([1.0, -1.0, 2.5])), float(rng.choice([0.0, 1.0, -0.5]))
        yc = O.csr_csmv(irp, cja, cval, a, x, b, y0, nc=nc)
        lens = np.diff(irp)
        for hksz in (1, 4, 32, 64):
            h = O.hll_from_coo(nr, ia, ja, val, hksz)
            assert np.array_equal(h["irn"], lens)
            assert np.array_equal(O.hll_csmv(h, nr, a, x, b, y0, nc=nc), yc), (seed, hksz)
            for k in range(len(h["hkoffs"]) - 1):
                rows = np.arange(k * hksz, min(nr, (k + 1) * hksz))
                w = (h["hkoffs"][k + 1] - h["hkoffs"][k]) // hksz
                assert w == (lens[rows].max() if len(rows) else 0)
                blk_j = h["ja"][h["hkoffs"][k]:h["hkoffs"][k + 1]].reshape(w, hksz)
                blk_v = h["val"][h["hkoffs"][k]:h["hkoffs"][k + 1]].reshape(w, hksz)
                for li, r in enumerate(rows):
                    n_r = lens[r]
                    row_j = cja[irp[r] - 1:irp[r + 1] - 1]
                    assert np.array_equal(blk_j[:n_r, li], row_j)
                    assert np.all(blk_v[n_r:, li] == 0.0)
                    if n_r:
                        assert np.all(blk_j[n_r:, li] == row_j[-1])
                    d = np.nonzero(row_j == r + 1)[0]
                    if len(d):
                        assert h["idiag"][r] == d[0] + 1
        e = O.ell_from_coo(nr, ia, ja, val)
        assert np.array_equal(O.ell_csmv(e, nr, a, x, b, y0, nc=nc), yc), seed
