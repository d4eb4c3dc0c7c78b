"""GPU parity of the sparse formats and SpMV kernels against the oracle.

Bar: conversions bit-exact (irn, hkoffs, ja, val including padding; idiag
on rows that hold a diagonal); HLL / ELL / CSR-stream SpMV bit-exact against
the oracle's csmv (same per-row order, rounded multiply then add); the CSR
warp-per-row path for rows longer than 2048 entries within the FP64
tolerance |dy_i| <= 1e-13 * sum_j |a_ij x_j| (componentwise, so rows whose
sum cancels are judged on the scale of their terms)."""
import json
import os

import numpy as np
import pytest

import oracle as O
from psblas3_b200 import gen

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-13


def _host_hll(irp, ja, va, hksz=32):
    n = len(irp) - 1
    ia, _, _ = gen.csr_to_coo(irp, ja, va)
    return O.hll_from_coo(n, ia, ja, va, hksz)


def _c1():
    return gen.pde3d(40, a=(1, 1, 1), b=(1 / np.sqrt(3),) * 3)


def test_usmv_kats_on_device(psb):
    """psb_d_mvsv_tester.f90 non-transposed usmv cases through the GPU
    HLL / ELL / CSR paths, exact equality."""
    cases = [c for c in json.load(open(os.path.join(HERE, "golden", "usmv_kats.json")))["cases"]
             if c["trans"] == "n"]
    assert len(cases) == 8
    for c in cases:
        m = c["m"]
        ia, ja, va = O.coo_fix(m, c["ia"], c["ja"], c["val"])
        irp, cja, cv = O.csr_from_coo(m, ia, ja, va)
        h = O.hll_from_coo(m, ia, ja, va, 32)
        e = O.ell_from_coo(m, ia, ja, va)
        mats = [psb.HllMat.from_host_hll(m, 32, h["irn"], h["hkoffs"], h["ja"], h["val"], h["idiag"]),
                psb.EllMat.from_host_ell(m, e["nzm"], e["irn"], e["ja"], e["val"], e["idiag"], e["ldv"]),
                psb.CsrMat(m, irp, cja, cv)]
        for A in mats:
            x = psb.DVect.bld(np.array(c["x"], float))
            y = psb.DVect.bld(np.array(c["y_before"], float))
            psb.psb_spmm(c["alpha"], A, x, c["beta"], y)
            assert np.array_equal(y.get_vect(), np.array(c["y_after"], float)), (type(A).__name__, c["name"])


@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.0, 1.0), (3.0, 1.0), (0.5, -2.0), (0.0, 2.0)])
def test_hll_spmv_c1_bitexact(psb, alpha, beta):
    """C1 operator, x ~ U[-1,1] seed 0: GPU HLL SpMV == oracle HLL csmv."""
    irp, ja, va = _c1()
    n = len(irp) - 1
    h = _host_hll(irp, ja, va)
    A = psb.HllMat.from_host_hll(n, 32, h["irn"], h["hkoffs"], h["ja"], h["val"], h["idiag"])
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, n)
    y0 = rng.uniform(-1, 1, n)
    ref = O.hll_csmv(h, n, alpha, x, beta, y0)
    X, Y = psb.DVect.bld(x), psb.DVect.bld(y0)
    psb.psb_spmm(alpha, A, X, beta, Y)
    assert np.array_equal(Y.get_vect(), ref)


def test_hll_beta0_does_not_read_y(psb):
    irp, ja, va = gen.stencil27(9)
    n = len(irp) - 1
    h = _host_hll(irp, ja, va)
    A = psb.HllMat.from_host_hll(n, 32, h["irn"], h["hkoffs"], h["ja"], h["val"], h["idiag"])
    x = np.random.default_rng(1).uniform(-1, 1, n)
    Y = psb.DVect.bld(np.full(n, np.nan))
    psb.psb_spmm(2.0, A, psb.DVect.bld(x), 0.0, Y)
    assert np.array_equal(Y.get_vect(), O.hll_csmv(h, n, 2.0, x, 0.0, np.zeros(n)))


def test_device_hll_build_matches_cpu_converter(psb):
    """psbx_hll_from_csr_device == psi_d_convert_hll_from_coo byte for byte,
    padding included (C1 operator plus a ragged power-law matrix)."""
    import torch
    for irp, ja, va in (_c1(), gen.powerlaw(5000, kmax=300, seed=5)):
        n = len(irp) - 1
        h = _host_hll(irp, ja, va)
        d_irp = torch.from_numpy(irp).cuda()
        d_ja = torch.from_numpy(ja).cuda()
        d_va = torch.from_numpy(va).cuda()
        A = psb.HllMat.from_csr_device(n, n, len(ja), d_irp.data_ptr(), d_ja.data_ptr(), d_va.data_ptr(), 32)
        g = A.read()
        assert np.array_equal(g["hkoffs"], h["hkoffs"])
        assert np.array_equal(g["irn"], h["irn"])
        assert np.array_equal(g["ja"], h["ja"])
        assert np.array_equal(g["val"].view(np.uint64), h["val"].view(np.uint64))
        has = h["idiag"] > 0
        assert np.array_equal(g["idiag"][has], h["idiag"][has])
        assert np.all(g["idiag"][~has] == 0)


def _drop_rows(irp, ja, va, rows):
    """CSR with the entries of `rows` (0-based) removed (empty rows)."""
    keep = np.ones(len(ja), bool)
    for r in rows:
        keep[irp[r] - 1:irp[r + 1] - 1] = False
    cnt = np.diff(irp).copy()
    cnt[rows] = 0
    nirp = np.concatenate([[1], 1 + np.cumsum(cnt)]).astype(np.int32)
    return nirp, ja[keep].copy(), va[keep].copy()


def _permute_rows(irp, ja, va, perm):
    cnt = np.diff(irp)[perm]
    nirp = np.concatenate([[1], 1 + np.cumsum(cnt)]).astype(np.int32)
    idx = np.concatenate([np.arange(irp[r] - 1, irp[r + 1] - 1) for r in perm])
    return nirp, ja[idx].copy(), va[idx].copy()


def test_device_hll_build_large_empty_rows_and_perm(psb):
    """The device build over more than one scan chunk (4,394 hacks), with
    empty rows (padding from the hack's first stored column, including hacks
    whose first rows are empty) and with a row permutation (hack rows taken
    in perm order == the CPU converter on the row-permuted matrix)."""
    import torch
    irp, ja, va = gen.pde3d(52)
    n = len(irp) - 1
    rng = np.random.default_rng(12)
    empty = np.unique(np.concatenate([rng.choice(n, n // 20, replace=False), np.arange(64, 70), [n - 1]]))
    irp, ja, va = _drop_rows(irp, ja, va, empty)
    for perm in (None, rng.permutation(n).astype(np.int32)):
        if perm is None:
            h = _host_hll(irp, ja, va)
        else:
            h = _host_hll(*_permute_rows(irp, ja, va, perm))
        d = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
        d_perm = None if perm is None else torch.from_numpy(perm).cuda()
        A = psb.HllMat.from_csr_device(n, n, len(ja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), 32,
                                       None if d_perm is None else d_perm.data_ptr())
        g = A.read()
        assert np.array_equal(g["hkoffs"], h["hkoffs"])
        assert np.array_equal(g["irn"], h["irn"])
        assert np.array_equal(g["ja"], h["ja"])
        assert np.array_equal(g["val"].view(np.uint64), h["val"].view(np.uint64))
        if perm is None:
            want = np.where(h["idiag"] > 0, h["idiag"], 0)
        else:  # idiag points at the diagonal of the original row held in each slot
            want = np.zeros(n, np.int32)
            for slot, r in enumerate(perm):
                pos = np.nonzero(ja[irp[r] - 1:irp[r + 1] - 1] == r + 1)[0]
                want[slot] = pos[0] + 1 if len(pos) else 0
        assert np.array_equal(g["idiag"], want)
        # and the SpMV through the permuted layout gives y in the original row order
        x = rng.uniform(-1, 1, n)
        X, Y = psb.DVect.bld(x), psb.DVect(n)
        A.spmv(1.0, X, 0.0, Y)
        assert np.array_equal(Y.get_vect(), O.csr_csmv(irp, ja, va, 1.0, x, 0.0, np.zeros(n)))


def test_psi_copy_coo_to_hlg(psb):
    """GPU conversion variant (psi_cuda_CopyCooToHlg.cuh): same offsets, row
    lengths, stored entries and diagonal positions as the CPU converter;
    padding column = column of the first entry of row 2, value 0."""
    irp, ja, va = gen.pde3d(13, b=(0.2, 0.1, 0.3))
    n = len(irp) - 1
    ia, _, _ = gen.csr_to_coo(irp, ja, va)
    h = _host_hll(irp, ja, va)
    A = psb.HllMat.from_coo_gpu(n, ia, ja, va, 32)
    g = A.read()
    assert np.array_equal(g["hkoffs"], h["hkoffs"]) and np.array_equal(g["irn"], h["irn"])
    jc = ja[irp[1] - 1]
    for k in range(len(h["hkoffs"]) - 1):
        w = (h["hkoffs"][k + 1] - h["hkoffs"][k]) // 32
        gj = g["ja"][h["hkoffs"][k]: h["hkoffs"][k + 1]].reshape(w, 32)
        cj = h["ja"][h["hkoffs"][k]: h["hkoffs"][k + 1]].reshape(w, 32)
        gv = g["val"][h["hkoffs"][k]: h["hkoffs"][k + 1]].reshape(w, 32)
        for ii in range(min(32, n - 32 * k)):
            L = h["irn"][32 * k + ii]
            assert np.array_equal(gj[:L, ii], cj[:L, ii])
            assert np.all(gj[L:, ii] == jc) and np.all(gv[L:, ii] == 0)
    assert np.array_equal(g["idiag"], h["idiag"])
    x = np.random.default_rng(2).uniform(-1, 1, n)
    Y = psb.DVect(n)
    psb.psb_spmm(1.0, A, psb.DVect.bld(x), 0.0, Y)
    assert np.array_equal(Y.get_vect(), O.hll_csmv(h, n, 1.0, x, 0.0, np.zeros(n)))


@pytest.mark.parametrize("maker", ["pde3d", "stencil27", "ragged"])
def test_ell_spmv_and_conversion(psb, maker):
    if maker == "pde3d":
        irp, ja, va = gen.pde3d(11, b=(1 / np.sqrt(3),) * 3)
    elif maker == "stencil27":
        irp, ja, va = gen.stencil27(9)
    else:
        irp, ja, va = gen.powerlaw(777, kmax=60, seed=7)
    n = len(irp) - 1
    ia, _, _ = gen.csr_to_coo(irp, ja, va)
    e = O.ell_from_coo(n, ia, ja, va)
    x = np.random.default_rng(3).uniform(-1, 1, n)
    y0 = np.random.default_rng(4).uniform(-1, 1, n)
    ref = O.ell_csmv(e, n, -1.5, x, 0.25, y0)
    for A in (psb.EllMat.from_host_ell(n, e["nzm"], e["irn"], e["ja"], e["val"], e["idiag"], e["ldv"]),
              psb.EllMat.from_coo_gpu(n, ia, ja, va)):
        g = A.read()
        nzm, ldv = g["nzm"], g["ldv"]
        assert nzm == e["nzm"] and ldv == ((n + 31) // 32) * 32
        gj = g["ja"].reshape(nzm, ldv)[:, :n]
        gv = g["val"].reshape(nzm, ldv)[:, :n]
        assert np.array_equal(gj, e["ja"].reshape(nzm, n))
        assert np.array_equal(gv, e["val"].reshape(nzm, n))
        Y = psb.DVect.bld(y0)
        psb.psb_spmm(-1.5, A, psb.DVect.bld(x), 0.25, Y)
        assert np.array_equal(Y.get_vect(), ref)


@pytest.mark.parametrize("maker", ["pde3d", "stencil27", "powerlaw_long"])
def test_csr_spmv(psb, maker):
    if maker == "pde3d":
        irp, ja, va = gen.pde3d(21, b=(1 / np.sqrt(3),) * 3)
    elif maker == "stencil27":
        irp, ja, va = gen.stencil27(17)
    else:
        irp, ja, va = gen.powerlaw(60000, kmax=4096, seed=11)
    n = len(irp) - 1
    x = np.random.default_rng(5).uniform(-1, 1, n)
    y0 = np.random.default_rng(6).uniform(-1, 1, n)
    ref = O.csr_csmv(irp, ja, va, 1.0, x, -1.0, y0)
    A = psb.CsrMat(n, irp, ja, va)
    Y = psb.DVect.bld(y0)
    psb.psb_spmm(1.0, A, psb.DVect.bld(x), -1.0, Y)
    got = Y.get_vect()
    lens = np.diff(irp)
    short = lens <= 2048
    assert np.array_equal(got[short], ref[short])
    if (~short).any():
        ia, _, _ = gen.csr_to_coo(irp, ja, va)
        scale = np.bincount(ia - 1, weights=np.abs(va * x[ja - 1]), minlength=n) + np.abs(y0)
        assert np.all(np.abs(got - ref)[~short] <= TOL * scale[~short])
    irp2, ja2, va2 = A.read()
    assert np.array_equal(irp2, irp) and np.array_equal(ja2, ja) and np.array_equal(va2, va)


def test_edge_shapes(psb):
    """1-row matrix, an empty row, n not a multiple of 32, hack size 64."""
    cases = [(1, [1], [1], [2.5]), (5, [1, 2, 2, 5], [1, 1, 2, 5], [1.0, -2.0, 3.0, 4.0]),
             (45, list(range(1, 46)), list(range(1, 46)), list(np.arange(1.0, 46.0)))]
    for n, ia, ja, va in cases:
        ia, ja, va = O.coo_fix(n, ia, ja, va)
        x = np.random.default_rng(n).uniform(-1, 1, n)
        for hk in (32, 64):
            h = O.hll_from_coo(n, ia, ja, va, hk)
            A = psb.HllMat.from_host_hll(n, hk, h["irn"], h["hkoffs"], h["ja"], h["val"], h["idiag"])
            Y = psb.DVect(n)
            psb.psb_spmm(1.0, A, psb.DVect.bld(x), 0.0, Y)
            assert np.array_equal(Y.get_vect(), O.hll_csmv(h, n, 1.0, x, 0.0, np.zeros(n)))
        irp, cja, cv = O.csr_from_coo(n, ia, ja, va)
        A = psb.CsrMat(n, irp, cja, cv)
        Y = psb.DVect(n)
        psb.psb_spmm(1.0, A, psb.DVect.bld(x), 0.0, Y)
        assert np.array_equal(Y.get_vect(), O.csr_csmv(irp, cja, cv, 1.0, x, 0.0, np.zeros(n)))


def test_size_mismatch_is_an_error(psb):
    irp, ja, va = gen.poisson7(4)
    n = len(irp) - 1
    h = _host_hll(irp, ja, va)
    A = psb.HllMat.from_host_hll(n, 32, h["irn"], h["hkoffs"], h["ja"], h["val"], h["idiag"])
    from psblas3_b200._lib import PsbxError
    with pytest.raises(PsbxError) as ei:
        psb.psb_spmm(1.0, A, psb.DVect(n), 0.0, psb.DVect(n - 1))
    assert ei.value.code == 1  # SPGPU_UNSUPPORTED


def test_full_size_27pt_properties(psb):
    """C2a operator at full size (200^3, 213,847,192 entries), built on the
    device: A*1 equals the exact row sums (26 - neighbours, integers), and
    A*(x+y) - (A*x + A*y) stays at rounding level."""
    import torch
    irp, ja, va = gen.stencil27(200)
    n = len(irp) - 1
    assert len(ja) == 213847192
    d_irp, d_ja, d_va = (torch.from_numpy(a).cuda() for a in (irp, ja, va))
    A = psb.HllMat.from_csr_device(n, n, len(ja), d_irp.data_ptr(), d_ja.data_ptr(), d_va.data_ptr(), 32)
    del d_irp, d_ja, d_va
    p = A.params()
    assert p["allocsize"] == 214591104
    ones = psb.DVect.bld(np.ones(n))
    Y = psb.DVect(n)
    psb.psb_spmm(1.0, A, ones, 0.0, Y)
    rowsum = 27.0 - np.diff(irp)  # 26 - (len - 1)
    assert np.array_equal(Y.get_vect(), rowsum)
    rng = np.random.default_rng(0)
    x, z = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    Ax, Az, Axz = psb.DVect(n), psb.DVect(n), psb.DVect(n)
    psb.psb_spmm(1.0, A, psb.DVect.bld(x), 0.0, Ax)
    psb.psb_spmm(1.0, A, psb.DVect.bld(z), 0.0, Az)
    psb.psb_spmm(1.0, A, psb.DVect.bld(x + z), 0.0, Axz)
    d = Axz.get_vect() - (Ax.get_vect() + Az.get_vect())
    assert np.max(np.abs(d)) <= 1e-12 * 27 * 4
    A.free()


def test_distributed_parts_on_device(psb):
    """Row-block SpMV of psb_dspmm.f90:196-216 with 3 ranks' parts on one
    GPU (one process; the exchange is a device copy between the parts'
    buffers): per rank, y = A_d x_own then y += A_nd x_halo, bit-exact
    against the oracle doing the same two products; assembled, the global
    product within the FP64 tolerance."""
    import torch
    from psblas3_b200 import dist
    irp, ja, va = _c1()
    n, world = len(irp) - 1, 3
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, n)
    y0 = rng.uniform(-1, 1, n)
    alpha, beta = 1.5, -0.5
    blocks = dist.partition_rows(n, world)
    parts = [dist.local_part(irp, ja, va, *b) for b in blocks]
    halos = [p.halo for p in parts]
    plans = [dist.exchange_plan(r, blocks, halos) for r in range(world)]
    ops = [dist.DistSpMV(p, pl) for p, pl in zip(parts, plans)]
    X = []
    for p in parts:
        xe = np.zeros(p.ncol)
        xe[:p.nl] = x[p.lo:p.hi]           # halo entries start as zeros: the exchange fills them
        X.append(psb.DVect.bld(xe))
    for op, xv in zip(ops, X):
        op.gather(xv)

    def exchange_for(r):
        def ex(sendbuf, recvbuf, plan):
            pos = 0
            for q in range(world):
                cnt = plan.recv_counts[q]
                if cnt:
                    off = int(sum(plans[q].send_counts[:r]))
                    recvbuf[pos:pos + cnt].copy_(ops[q].sendbuf[off:off + cnt])
                    pos += cnt
        return ex

    y_all = np.zeros(n)
    for r, (p, op) in enumerate(zip(parts, ops)):
        Y = psb.DVect.bld(y0[p.lo:p.hi])
        op(alpha, X[r], beta, Y, exchange=exchange_for(r))
        torch.cuda.synchronize()
        got = Y.get_vect()
        xe = np.concatenate([x[p.lo:p.hi], x[p.halo]])
        ref = O.csr_csmv(*p.ad, alpha, xe, beta, y0[p.lo:p.hi], nc=p.ncol)
        ref = O.csr_csmv(*p.and_, alpha, xe, 1.0, ref, nc=p.ncol)
        assert np.array_equal(got, ref), r
        assert np.array_equal(X[r].get_vect()[p.nl:], x[p.halo]), r
        y_all[p.lo:p.hi] = got
    glob = O.csr_csmv(irp, ja, va, alpha, x, beta, y0)
    scale = O.csr_csmv(irp, ja, np.abs(va), abs(alpha), np.abs(x), abs(beta), np.abs(y0))
    assert np.all(np.abs(y_all - glob) <= TOL * scale)


@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.0, 1.0), (2.5, -0.5)])
def test_hll_wide_hacks_bitexact(psb, alpha, beta):
    """Exact mode on a row-sorted power-law matrix (rows up to 4,000 entries
    at the front): the products of the wide hacks are formed by all blocks
    and each row's products added in entry order by a warp per hack, so the
    HLL SpMV stays bit-identical to the CPU csmv for every row mapping;
    host-written, device-built and permuted (perm = the length order)
    layouts alike."""
    import torch
    irp, ja, va = gen.powerlaw(60000, kmax=4000, seed=21)
    sirp, sja, sva, order = gen.sort_rows_by_length(irp, ja, va)
    n = len(irp) - 1
    rng = np.random.default_rng(4)
    x, y0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    h = _host_hll(sirp, sja, sva)
    assert np.any(np.diff(h["hkoffs"]) // 32 > 256)
    mats = [psb.HllMat.from_host_hll(n, 32, h["irn"], h["hkoffs"], h["ja"], h["val"], h["idiag"])]
    d = [torch.from_numpy(a).cuda() for a in (sirp, sja, sva)]
    mats.append(psb.HllMat.from_csr_device(n, n, len(sja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), 32))
    want = O.csr_csmv(sirp, sja, sva, alpha, x, beta, y0)
    for A in mats:
        A.set_wide_split(False)  # exact mode
        for tpr in (0, 1, -2, 2):  # two threads per row falls back to the stored order here
            A.set_threads_per_row(tpr)
            X, Y = psb.DVect.bld(x), psb.DVect.bld(y0)
            A.spmv(alpha, X, beta, Y)
            assert np.array_equal(Y.get_vect(), want), tpr
    # the unsorted matrix stored in length order through a permutation
    e = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
    d_perm = torch.from_numpy(np.ascontiguousarray(order, dtype=np.int32)).cuda()
    P = psb.HllMat.from_csr_device(n, n, len(ja), e[0].data_ptr(), e[1].data_ptr(), e[2].data_ptr(), 32,
                                   d_perm.data_ptr())
    P.set_wide_split(False)
    X, Y = psb.DVect.bld(x), psb.DVect.bld(y0)
    P.spmv(alpha, X, beta, Y)
    assert np.array_equal(Y.get_vect(), O.csr_csmv(irp, ja, va, alpha, x, beta, y0))


@pytest.mark.parametrize("wide", [0, 1, 33, 200])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.5, 0.5)])
def test_hll_wide_split_tolerance(psb, wide, alpha, beta):
    """Tolerance mode (the default): each wide hack is summed
    in 64-column chunks by all SMs, in the launch of the other rows; every
    row agrees with the CPU csmv within 1e-13 (|A||x| + |beta y|)_i, also
    on a second call (the per-hack tickets reset); host-built, device-built and permuted
    layouts; the CG over the same matrix converges as in the stored-order
    mode (iterations within 2)."""
    import torch
    irp, ja, va = gen.powerlaw(60000, kmax=4000, seed=21)
    sirp, sja, sva, order = gen.sort_rows_by_length(irp, ja, va)
    n = len(irp) - 1
    rng = np.random.default_rng(14)
    x, y0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    h = _host_hll(sirp, sja, sva)
    d = [torch.from_numpy(a).cuda() for a in (sirp, sja, sva)]
    e = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
    d_perm = torch.from_numpy(np.ascontiguousarray(order, dtype=np.int32)).cuda()
    cases = [
        (psb.HllMat.from_host_hll(n, 32, h["irn"], h["hkoffs"], h["ja"], h["val"], h["idiag"]), (sirp, sja, sva)),
        (psb.HllMat.from_csr_device(n, n, len(sja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), 32),
         (sirp, sja, sva)),
        (psb.HllMat.from_csr_device(n, n, len(ja), e[0].data_ptr(), e[1].data_ptr(), e[2].data_ptr(), 32,
                                    d_perm.data_ptr()), (irp, ja, va)),
    ]
    for A, (ri, rj, rv) in cases:
        A.set_wide(wide)
        assert A.layout()["split"] == 1  # the default
        want = O.csr_csmv(ri, rj, rv, alpha, x, beta, y0)
        scale = O.csr_csmv(ri, rj, np.abs(rv), abs(alpha), np.abs(x), abs(beta), np.abs(y0))
        X = psb.DVect.bld(x)
        for _ in range(2):  # a second call reuses the per-hack tickets
            Y = psb.DVect.bld(y0)
            A.spmv(alpha, X, beta, Y)
            got = Y.get_vect()
            assert np.all(np.abs(got - want) <= TOL * scale)
        A.free()
    sirp, sja, sva = gen.powerlaw_spd(20000, kmax=3000, seed=6)
    sirp, sja, sva, _ = gen.sort_rows_by_length(sirp, sja, sva)
    n = len(sirp) - 1
    f = [torch.from_numpy(a).cuda() for a in (sirp, sja, sva)]
    S = psb.HllMat.from_csr_device(n, n, len(sja), f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(), 32)
    S.set_wide(wide)
    P = psb.DiagPrec("DIAG").build(S)
    b = rng.uniform(-1, 1, n)
    its = []
    for split in (0, 1):
        S.set_wide_split(split)
        B, Xs = psb.DVect.bld(b), psb.DVect(n)
        it, err = psb.psb_krylov("CG", S, P, B, Xs, eps=1e-10, itmax=1000)
        assert err <= 1e-10
        its.append(it)
    assert abs(its[1] - its[0]) <= 2


@pytest.mark.parametrize("tpr", [0, 1, 2, -2])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.5, 0.5)])
def test_hll_threads_per_row(psb, tpr, alpha, beta):
    """Every row mapping of the standalone HLL SpMV (auto, one or two
    threads per row, two rows per thread) on a stencil, a row-sorted
    power-law matrix with wide hacks, and an odd row count: within 1e-13 of
    the CPU csmv in the tolerance mode, its bits in the exact mode (two
    threads per row then runs as two rows per thread)."""
    import torch
    mats = [gen.stencil27(13), gen.sort_rows_by_length(*gen.powerlaw(30007, kmax=3000, seed=9))[:3],
            gen.powerlaw(1037, kmax=90, seed=2)]
    for irp, ja, va in mats:
        n = len(irp) - 1
        d = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
        A = psb.HllMat.from_csr_device(n, n, len(ja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), 32)
        A.set_threads_per_row(tpr)
        assert A.layout()["tpr"] == tpr
        rng = np.random.default_rng(n)
        x, y0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
        want = O.csr_csmv(irp, ja, va, alpha, x, beta, y0)
        scale = O.csr_csmv(irp, ja, np.abs(va), abs(alpha), np.abs(x), abs(beta), np.abs(y0))
        X = psb.DVect.bld(x)
        Y = psb.DVect.bld(y0)
        A.spmv(alpha, X, beta, Y)
        assert np.all(np.abs(Y.get_vect() - want) <= TOL * scale), (n, tpr)
        A.set_wide_split(False)
        Y = psb.DVect.bld(y0)
        A.spmv(alpha, X, beta, Y)
        assert np.array_equal(Y.get_vect(), want), (n, tpr)
        A.free()
    with pytest.raises(RuntimeError):
        irp, ja, va = gen.stencil27(5)
        n = len(irp) - 1
        d = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
        psb.HllMat.from_csr_device(n, n, len(ja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                   64).set_threads_per_row(2)


def test_hll_autotune(psb):
    """The autotuned layout (hack size, wide-hack threshold, threads per
    row) comes back in the tolerance mode, within 1e-13 of the CPU csmv, and
    in the exact mode gives its bits, for a stencil and a skewed row-sorted
    matrix; its choice lies in the candidate set."""
    import torch
    for irp, ja, va in (gen.stencil27(40), gen.sort_rows_by_length(*gen.powerlaw(80000, kmax=4000, seed=2))[:3]):
        n = len(irp) - 1
        d = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
        A, info = psb.HllMat.autotune_from_csr_device(n, n, len(ja), d[0].data_ptr(), d[1].data_ptr(),
                                                     d[2].data_ptr())
        assert info["hksz"] in (32, 64, 128) and info["ms"] > 0
        assert info["wide_w"] in ((32, 64, 128, 256, 1024, -1) if info["hksz"] == 32 else (0,))
        assert info["tpr"] in ((-2, 1, 2) if info["hksz"] == 32 else (0,))
        assert A.layout()["split"] == 1
        x = np.random.default_rng(3).uniform(-1, 1, n)
        X, Y = psb.DVect.bld(x), psb.DVect(n)
        A.spmv(1.0, X, 0.0, Y)
        want = O.csr_csmv(irp, ja, va, 1.0, x, 0.0, np.zeros(n))
        scale = O.csr_csmv(irp, ja, np.abs(va), 1.0, np.abs(x), 0.0, np.zeros(n))
        assert np.all(np.abs(Y.get_vect() - want) <= TOL * scale), info
        A.set_wide_split(False)  # the exact mode: the same bits whatever the layout
        A.spmv(1.0, X, 0.0, Y)
        assert np.array_equal(Y.get_vect(), want), info


@pytest.mark.parametrize("wide", [-1, 0, 1, 33, 64, 200])
def test_hll_wide_threshold_same_bits(psb, wide):
    """In the exact mode every wide-hack threshold gives the CPU csmv's bits: 1 sends almost
    every hack down the wide path (partial product blocks, partial ring
    chunks, rows ending inside a chunk), -1 none; an unsorted power-law
    matrix puts wide hacks between narrow ones."""
    import torch
    irp, ja, va = gen.powerlaw(20000, kmax=3000, seed=5)
    n = len(irp) - 1
    d = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
    A = psb.HllMat.from_csr_device(n, n, len(ja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), 32)
    A.set_wide(wide).set_wide_split(False)
    rng = np.random.default_rng(8)
    x, y0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    X, Y = psb.DVect.bld(x), psb.DVect.bld(y0)
    A.spmv(-1.5, X, 0.5, Y)
    assert np.array_equal(Y.get_vect(), O.csr_csmv(irp, ja, va, -1.5, x, 0.5, y0))
    # and the CG over the same matrix made SPD (its products go the same way)
    sirp, sja, sva = gen.powerlaw_spd(20000, kmax=3000, seed=6)
    e = [torch.from_numpy(a).cuda() for a in (sirp, sja, sva)]
    S = psb.HllMat.from_csr_device(n, n, len(sja), e[0].data_ptr(), e[1].data_ptr(), e[2].data_ptr(), 32)
    S.set_wide_split(False)
    P = psb.DiagPrec("DIAG").build(S)
    b = rng.uniform(-1, 1, n)
    runs = []
    for w in (-1, wide):
        S.set_wide(w)
        B, Xs = psb.DVect.bld(b), psb.DVect(n)
        it, err = psb.psb_krylov("CG", S, P, B, Xs, eps=1e-10, itmax=1000)
        runs.append((it, err, Xs.get_vect().copy()))
    assert runs[1][0] == runs[0][0] and runs[1][1] == runs[0][1]
    assert np.array_equal(runs[1][2], runs[0][2])  # same products, same reductions
    assert runs[1][1] <= 1e-10
    r = O.csr_csmv(sirp, sja, sva, -1.0, runs[1][2], 1.0, b)
    assert np.linalg.norm(r) <= 1e-9 * np.linalg.norm(b)


def test_probe_gather(psb):
    """The gather-floor probe (psbx_probe_gather) reads x at every index
    pair (an odd last index skipped) and returns a positive time."""
    import ctypes as C

    import torch
    from psblas3_b200._lib import check, lib
    n = 1001
    idx = np.random.default_rng(1).integers(1, 5001, n).astype(np.int32)
    X = psb.DVect.bld(np.ones(5000))
    d_idx = torch.from_numpy(idx).cuda()
    out = torch.zeros((n + 7) // 8, dtype=torch.float64, device="cuda")
    ms = C.c_double(0.0)
    check(lib.psbx_probe_gather(C.c_void_p(d_idx.data_ptr()), n, 1, C.c_void_p(X.data_ptr),
                                C.c_void_p(out.data_ptr()), 3, C.byref(ms)), "psbx_probe_gather")
    assert ms.value > 0
    assert out.sum().item() == 2 * (n // 2)  # every pair read once, x = 1


@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.5, 0.5), (0.0, 2.0)])
def test_hll_spmv_host(psb, alpha, beta):
    """psbx_hll_spmv_host (host x and y, copies overlapped with the product
    block by block) gives the bits of write + spmvHllDeviceDouble + read for
    every block count, with pageable and page-locked host arrays (beta = 0
    and page-locked y: the row blocks store into y directly), on banded
    operators (overlapped) and on handles that take the three steps in turn
    (wide hacks, a row permutation); x may be the same array as y."""
    import torch
    rng = np.random.default_rng(17)
    cases = []
    for irp, ja, va in (gen.stencil27(30), gen.pde3d(21, a=(1, 1, 1), b=(0.5, 0.5, 0.5))):
        n = len(irp) - 1
        d = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
        cases.append((psb.HllMat.from_csr_device(n, n, len(ja), d[0].data_ptr(), d[1].data_ptr(),
                                                 d[2].data_ptr(), 32), n))
    sirp, sja, sva, order = gen.sort_rows_by_length(*gen.powerlaw(20011, kmax=3000, seed=4))
    n = len(sirp) - 1
    d = [torch.from_numpy(a).cuda() for a in (sirp, sja, sva)]
    cases.append((psb.HllMat.from_csr_device(n, n, len(sja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                             32), n))
    irp, ja, va = gen.pde3d(17)
    n = len(irp) - 1
    perm = torch.from_numpy(rng.permutation(n).astype(np.int32)).cuda()
    d = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
    cases.append((psb.HllMat.from_csr_device(n, n, len(ja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), 32,
                                             perm.data_ptr()), n))
    # rectangular: more columns than rows, and fewer
    for nr, nc in ((5000, 5517), (5000, 4700)):
        rows = [np.unique(np.append(rng.choice(nc, 5, replace=False), min(i, nc - 1))) + 1 for i in range(nr)]
        ja = np.concatenate(rows).astype(np.int32)
        irp = np.concatenate([[1], 1 + np.cumsum([len(r) for r in rows])]).astype(np.int32)
        va = rng.standard_normal(len(ja))
        d = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
        cases.append((psb.HllMat.from_csr_device(nr, nc, len(ja), d[0].data_ptr(), d[1].data_ptr(),
                                                 d[2].data_ptr(), 32), (nr, nc)))
    for A, n in cases:
        nr, nc = n if isinstance(n, tuple) else (n, n)
        x, y0 = rng.uniform(-1, 1, nc), rng.uniform(-1, 1, nr)
        X, Y = psb.DVect.bld(x), psb.DVect.bld(y0)
        A.spmv(alpha, X, beta, Y)
        want = Y.get_vect()
        for chunks in (0, 1, 3, 7, 10 ** 6):
            y = y0.copy()
            A.spmv_host(alpha, x, beta, y, chunks=chunks)
            assert np.array_equal(y, want), (n, chunks)
            xp = torch.from_numpy(x).pin_memory()
            yp = torch.from_numpy(y0.copy()).pin_memory()
            A.spmv_host(alpha, xp, beta, yp, chunks=chunks)
            assert np.array_equal(yp.numpy(), want), (n, chunks, "pinned")
        if beta == 0.0 and nr == nc:  # y = A y in place, pageable and page-locked
            yy = x.copy()
            A.spmv_host(alpha, yy, 0.0, yy)
            assert np.array_equal(yy, want)
            yp = torch.from_numpy(x.copy()).pin_memory()
            for _ in range(2):
                yp.copy_(torch.from_numpy(x))
                A.spmv_host(alpha, yp, 0.0, yp)
                assert np.array_equal(yp.numpy(), want)
        A.free()


def test_device_build_random_matrices(psb):
    """Seeded random matrices (rectangular, empty rows, after psb_d_fix_coo):
    the device CSR -> HLL build gives the CPU converter's arrays byte for
    byte for hack sizes 32 and 64, and the device product (exact mode) the
    CPU csmv's bits."""
    import torch
    for seed in range(12):
        rng = np.random.default_rng(2000 + seed)
        nr, nc = int(rng.integers(1, 300)), int(rng.integers(1, 300))
        nz = max(1, int(nr * nc * float(rng.uniform(0.0, 0.1))))
        ia, ja, va = O.coo_fix(nr, rng.integers(1, nr + 1, nz), rng.integers(1, nc + 1, nz), rng.standard_normal(nz))
        irp, cja, cva = O.csr_from_coo(nr, ia, ja, va)
        x, y0 = rng.uniform(-1, 1, nc), rng.uniform(-1, 1, nr)
        want = O.csr_csmv(irp, cja, cva, -1.5, x, 0.5, y0, nc=nc)
        for hksz in (32, 64):
            h = O.hll_from_coo(nr, ia, ja, va, hksz)
            d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (irp, cja, cva)]
            A = psb.HllMat.from_csr_device(nr, nc, len(cja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), hksz)
            g = A.read()
            for k in ("hkoffs", "irn", "ja"):
                assert np.array_equal(g[k], h[k]), (seed, hksz, k)
            assert np.array_equal(g["val"].view(np.uint64), h["val"].view(np.uint64)), (seed, hksz)
            has = np.array([np.any(cja[irp[r] - 1:irp[r + 1] - 1] == r + 1) for r in range(nr)], bool)
            assert np.array_equal(g["idiag"][has], h["idiag"][has])
            A.set_wide_split(False)
            X, Y = psb.DVect.bld(x), psb.DVect.bld(y0)
            A.spmv(-1.5, X, 0.5, Y)
            assert np.array_equal(Y.get_vect(), want), (seed, hksz)
            A.free()


def test_random_matrices_ell_csr_products(psb):
    """Seeded random rectangular matrices with empty rows: the ELL (host
    arrays of the CPU converter) and CSR device products give the CPU csmv's
    bits; CSR rows longer than a block (none here) would be the only
    tolerance case."""
    for seed in range(12):
        rng = np.random.default_rng(3000 + seed)
        nr, nc = int(rng.integers(1, 400)), int(rng.integers(1, 400))
        nz = max(1, int(nr * nc * float(rng.uniform(0.0, 0.08))))
        ia, ja, va = O.coo_fix(nr, rng.integers(1, nr + 1, nz), rng.integers(1, nc + 1, nz), rng.standard_normal(nz))
        irp, cja, cva = O.csr_from_coo(nr, ia, ja, va)
        x, y0 = rng.uniform(-1, 1, nc), rng.uniform(-1, 1, nr)
        for a, b in ((1.0, 0.0), (-1.5, 0.5)):
            want = O.csr_csmv(irp, cja, cva, a, x, b, y0, nc=nc)
            Cm = psb.CsrMat(nr, irp, cja, cva, cols=nc)
            X, Y = psb.DVect.bld(x), psb.DVect.bld(y0)
            Cm.spmv(a, X, b, Y)
            assert np.array_equal(Y.get_vect(), want), (seed, "csr", a, b)
            Cm.free()
            e = O.ell_from_coo(nr, ia, ja, va)
            E = psb.EllMat.from_host_ell(nr, e["nzm"], e["irn"], e["ja"], e["val"], e["idiag"], e["ldv"],
                                         nnz=len(cja))
            X, Y = psb.DVect.bld(x), psb.DVect.bld(y0)
            E.spmv(a, X, b, Y)
            assert np.array_equal(Y.get_vect(), want), (seed, "ell", a, b)
            E.free()
