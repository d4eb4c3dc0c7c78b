"""GPU tests of the entry points that complete the link of the reference's
Fortran GPU modules: the plain device buffers and mapped host memory of the
vector types, geins, the integer (psb_i_vect_cuda) and FP32
(psb_s_vect_cuda) multivector sets, the FP32 HLL / ELL products and
conversions, the ELL value update (csput), the parameter blocks, and the CSR
triangular solve.

Bars: element-wise operations, copies, gathers, scatters and conversions
bit-exact; FP32 products bit-exact against the oracle's restatement of the
library's documented FP32 form (FP64 row sums rounded once) and within the
FP32 error bound gamma_k * sum|a_ij x_j| (gamma_k = k u / (1 - k u),
u = 2^-24, k = row length + 2) of the reference's FP32-accumulated product;
FP32 dot / nrm2 / amax bit-exact, asum within one FP32 ulp; the triangular
solve bit-exact against the CPU restatement of psb_d_csr_cssv.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from psblas3_b200 import gen

pytestmark = pytest.mark.gpu
F = np.float32


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


# ------------------------------------------------------------ plain buffers
@pytest.mark.parametrize("tname,dt", [("Double", np.float64), ("Float", np.float32), ("Int", np.int32)])
def test_device_buffers_roundtrip(psb, tname, dt):
    from psblas3_b200._lib import lib
    f = lambda s: getattr(lib, s.format(t=tname))  # noqa: E731
    n = 1000
    h = (np.arange(n) * 3 - 7).astype(dt)
    d = C.c_void_p()
    assert f("allocate{t}")(C.byref(d), n) == 0
    assert f("write{t}")(d, _p(h), n) == 0
    back = np.zeros(n, dt)
    assert f("read{t}")(d, _p(back), n) == 0
    assert np.array_equal(back, h)
    # 1-based first: entries first..first+9 of the device buffer
    part = (np.arange(10) + 500).astype(dt)
    assert f("write{t}First")(101, d, _p(part), 10, 1) == 0
    got = np.zeros(10, dt)
    assert f("read{t}First")(101, d, _p(got), 10, 1) == 0
    assert np.array_equal(got, part)
    assert f("read{t}")(d, _p(back), n) == 0
    ref = h.copy()
    ref[100:110] = part
    assert np.array_equal(back, ref)
    f("free{t}")(d)
    # m x n
    dm = C.c_void_p()
    hm = np.arange(6 * 7).astype(dt)
    assert f("allocateMulti{t}")(C.byref(dm), 6, 7) == 0
    assert f("writeMulti{t}")(dm, _p(hm), 6, 7) == 0
    gm = np.zeros_like(hm)
    assert f("readMulti{t}")(dm, _p(gm), 6, 7) == 0
    assert np.array_equal(gm, hm)
    f("free{t}")(dm)


def test_mapped_host_memory(psb):
    """registerMappedDouble gives a device alias of a host buffer; the
    library's dot reads it in place; unregisterMapped releases it."""
    from psblas3_b200._lib import lib
    n = 4096
    rng = np.random.default_rng(5)
    host = np.ascontiguousarray(rng.uniform(-1, 1, n))
    other = rng.uniform(-1, 1, n)
    dptr = C.c_void_p()
    assert lib.registerMappedDouble(_p(host), C.byref(dptr), n, C.c_double(0.0)) == 0
    assert dptr.value
    w = C.c_void_p()
    assert lib.psbx_wrapMultiVecDevice(C.byref(w), dptr, n, 2) == 0
    Y = psb.DVect.bld(other)
    res = C.c_double(0)
    assert lib.dotMultiVecDeviceDouble(C.byref(res), n, w, Y.h) == 0
    assert res.value == O.dot(host, other)
    lib.freeMultiVecDevice(w)
    assert lib.unregisterMapped(_p(host)) == 0


# ------------------------------------------------------------------- geins
@pytest.mark.parametrize("dt", [np.float64, np.float32, np.int32])
def test_geins(psb, dt):
    from psblas3_b200._lib import lib
    name = {np.float64: "Double", np.float32: "Float", np.int32: "Int"}[dt]
    fn = getattr(lib, f"geinsMultiVecDevice{name}")
    n, m = 500, 120
    rng = np.random.default_rng(9)
    x0 = (rng.integers(-50, 50, n)).astype(dt)
    irl = rng.choice(n, m, replace=False).astype(np.int32) + 1   # 1-based, distinct
    val = (rng.integers(-9, 9, m)).astype(dt)
    for dupl in (0, 1):
        X, Irl, Val = psb.DVect.bld(x0), psb.DVect.bld(irl), psb.DVect.bld(val)
        assert fn(m, Irl.h, Val.h, dupl, 1, X.h) == 0
        ref = x0.copy()
        ref[irl - 1] = val if dupl == 0 else ref[irl - 1] + val
        assert np.array_equal(X.get_vect(), ref), dupl
    Irl = psb.DVect.bld(irl)
    assert fn(m + 1, Irl.h, psb.DVect.bld(val).h, 0, 1, psb.DVect.bld(x0).h) == 1  # n beyond the index vector


# ---------------------------------------------------------- integer vectors
def test_int_vectors(psb):
    from psblas3_b200._lib import lib
    n = 3000
    rng = np.random.default_rng(2)
    x = rng.integers(-1000, 1000, n).astype(np.int32)
    X = psb.DVect.bld(x)
    assert np.array_equal(X.get_vect(), x)
    assert lib.setscalMultiVecDeviceInt(7, 11, 20, 1, X.h) == 0
    ref = x.copy()
    ref[10:20] = 7
    assert np.array_equal(X.get_vect(), ref)
    idx = rng.choice(n, 400, replace=False).astype(np.int32) + 1
    I = psb.DVect.bld(idx)
    import torch
    buf = torch.zeros(400, dtype=torch.int32, device="cuda")
    assert lib.igathMultiVecDeviceIntVecIdx(X.h, 0, 400, 1, I.h, 1, C.c_void_p(buf.data_ptr()), 1) == 0
    assert np.array_equal(buf.cpu().numpy(), ref[idx - 1])
    src = torch.from_numpy(rng.integers(-5, 5, 400).astype(np.int32)).cuda()
    dI = torch.from_numpy(idx).cuda()
    for beta in (0, 1):
        Y = psb.DVect.bld(ref)
        assert lib.iscatMultiVecDeviceInt(Y.h, 0, 400, 1, C.c_void_p(dI.data_ptr()), 1,
                                          C.c_void_p(src.data_ptr()), 1, beta) == 0
        exp = ref.copy()
        exp[idx - 1] = src.cpu().numpy() + (beta * ref[idx - 1])
        assert np.array_equal(Y.get_vect(), exp), beta


# ------------------------------------------------------------ FP32 vectors
def test_float_vectors_elementwise(psb):
    from psblas3_b200._lib import lib
    n = 100_003
    rng = np.random.default_rng(3)
    x, y, z, w = (rng.uniform(-2, 2, n).astype(F) for _ in range(4))
    for a, b in [(1.5, -0.25), (0.0, 2.0), (0.0, 0.0), (3.0, 0.0), (0.0, 1.0), (-1.0, 1.0)]:
        X, Y = psb.DVect.bld(x), psb.DVect.bld(y)
        assert lib.axpbyMultiVecDeviceFloat(n, a, X.h, b, Y.h) == 0
        assert np.array_equal(Y.get_vect(), O.saxpby(a, x, b, y)), (a, b)
    X, Y, Z = psb.DVect.bld(x), psb.DVect.bld(y), psb.DVect.bld(z)
    assert lib.upd_xyzMultiVecDeviceFloat(n, 0.5, -1.5, 2.0, 0.75, X.h, Y.h, Z.h) == 0
    ry, rz = O.supd_xyz(0.5, -1.5, 2.0, 0.75, x, y, z)
    assert np.array_equal(Y.get_vect(), ry) and np.array_equal(Z.get_vect(), rz)
    X, Y, Z, W = (psb.DVect.bld(v) for v in (x, y, z, w))
    assert lib.xyzwMultiVecDeviceFloat(n, 1.25, -0.5, 0.3, 2.0, -1.0, 0.125, X.h, Y.h, Z.h, W.h) == 0
    ry, rz, rw = O.sxyzw(1.25, -0.5, 0.3, 2.0, -1.0, 0.125, x, y, z, w)
    assert all(np.array_equal(V.get_vect(), r) for V, r in ((Y, ry), (Z, rz), (W, rw)))
    A, B, Z = psb.DVect.bld(x), psb.DVect.bld(y), psb.DVect.bld(z)
    assert lib.axybzMultiVecDeviceFloat(n, 1.0, A.h, B.h, 0.0, Z.h) == 0
    assert np.array_equal(Z.get_vect(), O.smlt(1.0, x, y, 0.0, z))
    assert lib.axybzMultiVecDeviceFloat(n, -0.5, A.h, B.h, 1.5, Z.h) == 0
    assert np.array_equal(Z.get_vect(), O.smlt(-0.5, x, y, 1.5, O.smlt(1.0, x, y, 0.0, z)))
    assert lib.axyMultiVecDeviceFloat(n, 2.0, A.h, B.h) == 0
    assert np.array_equal(B.get_vect(), O.smlt(2.0, x, y, 0.0, y))
    A2, B2 = psb.DVect.bld(x), psb.DVect(n, dtype=F)
    assert lib.absMultiVecDeviceFloat2(n, 3.0, A2.h, B2.h) == 0
    assert np.array_equal(B2.get_vect(), F(3.0) * np.abs(x))
    assert lib.absMultiVecDeviceFloat(n, -1.0, A2.h) == 0
    assert np.array_equal(A2.get_vect(), F(-1.0) * np.abs(x))
    S = psb.DVect.bld(x)
    assert lib.scalMultiVecDeviceFloat(F(0.1), S.h) == 0
    assert np.array_equal(S.get_vect(), F(0.1) * x)
    assert lib.setscalMultiVecDeviceFloat(F(2.5), 3, 9, 1, S.h) == 0
    exp = F(0.1) * x
    exp[2:9] = F(2.5)
    assert np.array_equal(S.get_vect(), exp)


def test_float_vectors_reductions(psb):
    from psblas3_b200._lib import lib
    rng = np.random.default_rng(4)
    for n in (1, 1000, 1_000_003):
        x = rng.uniform(-1, 1, n).astype(F)
        y = rng.standard_normal(n).astype(F)
        X, Y = psb.DVect.bld(x), psb.DVect.bld(y)
        r = C.c_float(0)
        assert lib.dotMultiVecDeviceFloat(C.byref(r), n, X.h, Y.h) == 0
        assert F(r.value) == O.sdot(x, y), n
        assert lib.nrm2MultiVecDeviceFloat(C.byref(r), n, X.h) == 0
        assert F(r.value) == O.snrm2(x), n
        assert lib.amaxMultiVecDeviceFloat(C.byref(r), n, Y.h) == 0
        assert F(r.value) == O.samax(y), n
        assert lib.asumMultiVecDeviceFloat(C.byref(r), n, Y.h) == 0
        ref = O.sasum(y)
        assert abs(F(r.value) - ref) <= np.spacing(ref), n
    # several vectors at once
    xm = rng.uniform(-1, 1, (777, 3)).astype(F)
    ym = rng.uniform(-1, 1, (777, 3)).astype(F)
    X, Y = psb.DVect.bld(xm), psb.DVect.bld(ym)
    r3 = (C.c_float * 3)()
    assert lib.dotMultiVecDeviceFloat(r3, 777, X.h, Y.h) == 0
    assert [F(v) for v in r3] == [O.sdot(xm[:, k], ym[:, k]) for k in range(3)]


def test_float_gather_scatter(psb):
    import torch
    from psblas3_b200._lib import lib
    n, m = 5000, 800
    rng = np.random.default_rng(8)
    x = rng.uniform(-1, 1, n).astype(F)
    idx = rng.choice(n, m, replace=False).astype(np.int32) + 1
    X, I = psb.DVect.bld(x), psb.DVect.bld(idx)
    buf = torch.zeros(m, dtype=torch.float32, device="cuda")
    assert lib.igathMultiVecDeviceFloatVecIdx(X.h, 0, m, 1, I.h, 1, C.c_void_p(buf.data_ptr()), 1) == 0
    assert np.array_equal(buf.cpu().numpy(), x[idx - 1])
    src = rng.uniform(-1, 1, m).astype(F)
    dsrc, dI = torch.from_numpy(src).cuda(), torch.from_numpy(idx).cuda()
    assert lib.iscatMultiVecDeviceFloat(X.h, 0, m, 1, C.c_void_p(dI.data_ptr()), 1, C.c_void_p(dsrc.data_ptr()), 1,
                                        F(0.5)) == 0
    exp = x.copy()
    exp[idx - 1] = F(0.5) * x[idx - 1] + src
    assert np.array_equal(X.get_vect(), exp)


# ------------------------------------------------------- FP32 HLL and ELL
def _fp32_matrix():
    irp, ja, va = gen.powerlaw(20_000, kmax=300, seed=4)
    n = len(irp) - 1
    ia, _, _ = gen.csr_to_coo(irp, ja, va)
    return n, irp, ia, ja, va.astype(F)


def _fp32_bound(h, n, alpha, x, beta, y0, y_ref32):
    """|y - y_ref32| may be up to twice the FP32 accumulation bound."""
    absA = dict(h, val=np.abs(np.asarray(h["val"], np.float64)))
    scale = O.hll_csmv(absA, n, abs(alpha), np.abs(x.astype(np.float64)), abs(beta), np.abs(y0.astype(np.float64)))
    k = np.asarray(h["irn"], np.float64) + 2
    u = 2.0 ** -24
    return 2 * (k * u / (1 - k * u)) * scale


def test_hll_float_spmv(psb):
    from psblas3_b200._lib import lib
    n, irp, ia, ja, va32 = _fp32_matrix()
    h = O.hll_from_coo(n, ia, ja, va32.astype(np.float64), 32)
    h32 = dict(h, val=np.asarray(h["val"], F))
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, n).astype(F)
    y0 = rng.uniform(-1, 1, n).astype(F)
    # the FP32 object written from host arrays, and built by the device scatter
    hdl = C.c_void_p()
    assert lib.FallocHllDevice(C.byref(hdl), 32, n, len(ja), len(h["val"]), 1, 1) == 0
    assert lib.writeHllDeviceFloat(hdl, _p(np.ascontiguousarray(h32["val"])), _p(h["ja"]), _p(h["hkoffs"]),
                                   _p(h["irn"]), _p(h["idiag"])) == 0
    rb = np.zeros(len(h["val"]), F)
    rj = np.zeros(len(h["ja"]), np.int32)
    rh, rn, rd = np.zeros_like(h["hkoffs"]), np.zeros_like(h["irn"]), np.zeros_like(h["idiag"])
    assert lib.readHllDeviceFloat(hdl, _p(rb), _p(rj), _p(rh), _p(rn), _p(rd)) == 0
    assert np.array_equal(rb, h32["val"]) and np.array_equal(rj, h["ja"])
    scat = psb.HllMat.from_coo_gpu(n, ia, ja, va32.astype(np.float64))  # FP64 object, used for its layout
    p = scat.params()
    hdl2 = C.c_void_p()
    assert lib.FallocHllDevice(C.byref(hdl2), 32, n, len(ja), p["allocsize"], 1, 1) == 0
    irn = np.bincount(ia - 1, minlength=n).astype(np.int32)
    noffs = (n + 31) // 32
    width = np.zeros(noffs * 32, np.int64)
    width[:n] = irn
    hk = np.zeros(noffs + 1, np.int64)
    np.cumsum(width.reshape(noffs, 32).max(axis=1) * 32, out=hk[1:])
    idisp = np.zeros(n + 1, np.int64)
    np.cumsum(irn, out=idisp[1:])
    hk32, idisp32, ja32 = hk.astype(np.int32), idisp.astype(np.int32), np.ascontiguousarray(ja, np.int32)
    assert lib.psiCopyCooToHlgFloat(n, n, len(ja), 32, noffs, int(hk[-1]), _p(irn), _p(hk32), _p(idisp32), _p(ja32),
                                    _p(np.ascontiguousarray(va32)), hdl2) == 0
    g64 = scat.read()
    rb = np.zeros(p["allocsize"], F)
    rj = np.zeros(p["allocsize"], np.int32)
    rh, rn, rd = np.zeros(noffs + 1, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)
    assert lib.readHllDeviceFloat(hdl2, _p(rb), _p(rj), _p(rh), _p(rn), _p(rd)) == 0
    assert np.array_equal(rj, g64["ja"]) and np.array_equal(rb, np.asarray(g64["val"], F))
    for a, b in [(1.0, 0.0), (-0.75, 1.5), (2.0, -1.0), (0.0, 0.5)]:
        for H in (hdl, hdl2):
            X, Y = psb.DVect.bld(x), psb.DVect.bld(y0)
            assert lib.spmvHllDeviceFloat(H, F(a), X.h, F(b), Y.h) == 0
            got = Y.get_vect()
            assert np.array_equal(got, O.hll_csmv_f32(h32, n, a, x, b, y0)), (a, b)
            ref32 = O.hll_csmv_f32(h32, n, a, x, b, y0, reference_fp32=True)
            bound = _fp32_bound(h32, n, a, x, b, y0, ref32)
            assert np.all(np.abs(got.astype(np.float64) - ref32) <= bound + 2 * np.spacing(np.abs(ref32)))
    # the FP32 copy of an FP64 object (the mixed-precision solver's operand)
    scat.make_single()
    X, Y = psb.DVect.bld(x), psb.DVect.bld(y0)
    assert lib.spmvHllDeviceFloat(scat.h, F(1.0), X.h, F(0.0), Y.h) == 0
    assert np.array_equal(Y.get_vect(), O.hll_csmv_f32(h32, n, 1.0, x, 0.0, y0))
    lib.freeHllDevice(hdl)
    lib.freeHllDevice(hdl2)


def test_ell_float_and_params(psb):
    from psblas3_b200._lib import lib
    n, irp, ia, ja, va32 = _fp32_matrix()
    irn = np.bincount(ia - 1, minlength=n).astype(np.int32)
    nzm = int(irn.max())
    prm = lib.getEllDeviceParams(n, nzm, len(ja), n, 1, 1)
    hdl = C.c_void_p()
    assert lib.FallocEllDevice(C.byref(hdl), n, nzm, len(ja), n, 1, 1) == 0
    pitch = lib.getEllDevicePitch(hdl)
    assert prm.pitch == pitch and prm.maxRowSize == nzm and prm.rows == n and prm.avgRowSize == -(-len(ja) // n)
    idisp = np.zeros(n + 1, np.int64)
    np.cumsum(irn, out=idisp[1:])
    assert lib.psiCopyCooToElgFloat(n, n, len(ja), 1, pitch, nzm, _p(irn), _p(idisp.astype(np.int32)),
                                    _p(np.ascontiguousarray(ja, np.int32)), _p(np.ascontiguousarray(va32)), hdl) == 0
    val = np.zeros(pitch * nzm, F)
    eja = np.zeros(pitch * nzm, np.int32)
    rn, rd = np.zeros(n, np.int32), np.zeros(n, np.int32)
    assert lib.readEllDeviceFloat(hdl, _p(val), _p(eja), pitch, _p(rn), _p(rd)) == 0
    e64 = O.ell_from_coo(n, ia, ja, va32.astype(np.float64), ldv=pitch)
    first_n = lambda a: np.asarray(a).reshape(nzm, pitch)[:, :n]  # noqa: E731  (rows past n are padding)
    assert np.array_equal(first_n(eja), first_n(e64["ja"]))
    assert np.array_equal(first_n(val), first_n(np.asarray(e64["val"], F)))
    e32 = dict(e64, val=val, ja=eja, irn=rn, ldv=pitch)
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, n).astype(F)
    y0 = rng.uniform(-1, 1, n).astype(F)
    for a, b in [(1.0, 0.0), (-1.25, 0.5)]:
        X, Y = psb.DVect.bld(x), psb.DVect.bld(y0)
        assert lib.spmvEllDeviceFloat(hdl, F(a), X.h, F(b), Y.h) == 0
        assert np.array_equal(Y.get_vect(), O.ell_csmv_f32(e32, n, a, x, b, y0)), (a, b)
    # write / read back the FP32 arrays
    hdl2 = C.c_void_p()
    assert lib.FallocEllDevice(C.byref(hdl2), n, nzm, len(ja), n, 1, 1) == 0
    assert lib.writeEllDeviceFloat(hdl2, _p(val), _p(eja), pitch, _p(rn), _p(rd)) == 0
    v2 = np.zeros_like(val)
    j2 = np.zeros_like(eja)
    assert lib.readEllDeviceFloat(hdl2, _p(v2), _p(j2), pitch, _p(np.zeros(n, np.int32)),
                                  _p(np.zeros(n, np.int32))) == 0
    assert np.array_equal(v2, val) and np.array_equal(j2, eja)
    lib.freeEllDevice(hdl)
    lib.freeEllDevice(hdl2)
    hp = lib.bldHllDeviceParams(32, n, len(ja), 12345, 2, 1)
    assert (hp.hackSize, hp.rows, hp.nzt, hp.allocsize, hp.elementType, hp.firstIndex) == (32, n, len(ja), 12345, 2, 1)
    assert hp.avgNzr == -(-len(ja) // n)
    lib.resetEllTimer()
    assert lib.getEllTimer() == 0.0
    assert lib.FcusparseCreate() == 0 and lib.FcusparseDestroy() == 0


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_ell_csput(psb, dt):
    """dev_csputEllDevice*: values of stored entries overwritten in place;
    entries not in the pattern (and rows outside the matrix) change nothing."""
    from psblas3_b200._lib import lib
    irp, ja, va = gen.poisson7(10)
    n = len(irp) - 1
    ia, _, _ = gen.csr_to_coo(irp, ja, va)
    et = 2 if dt == np.float64 else 1
    e = O.ell_from_coo(n, ia, ja, va)
    hdl = C.c_void_p()
    assert lib.FallocEllDevice(C.byref(hdl), n, e["nzm"], len(ja), n, et, 1) == 0
    pitch = lib.getEllDevicePitch(hdl)
    e = O.ell_from_coo(n, ia, ja, va, ldv=pitch)
    ev = np.ascontiguousarray(e["val"], dt)
    fw = lib.writeEllDeviceDouble if dt == np.float64 else lib.writeEllDeviceFloat
    fr = lib.readEllDeviceDouble if dt == np.float64 else lib.readEllDeviceFloat
    assert fw(hdl, _p(ev), _p(np.ascontiguousarray(e["ja"], np.int32)), pitch, _p(e["irn"]), _p(e["idiag"])) == 0
    rng = np.random.default_rng(6)
    sel = rng.choice(len(ja), 300, replace=False)
    ui, uj = ia[sel].astype(np.int32), ja[sel].astype(np.int32)
    uv = rng.uniform(-5, 5, 300).astype(dt)
    # two entries that are not in the pattern, one row outside the matrix
    ui = np.concatenate([ui, [1, 5, n + 3]]).astype(np.int32)
    uj = np.concatenate([uj, [n, n - 1, 1]]).astype(np.int32)
    uv = np.concatenate([uv, np.array([99, 98, 97], dt)])
    I, J, V = psb.DVect.bld(ui), psb.DVect.bld(uj), psb.DVect.bld(uv)
    fput = lib.dev_csputEllDeviceDouble if dt == np.float64 else lib.dev_csputEllDeviceFloat
    assert fput(hdl, len(ui), I.h, J.h, V.h) == 0
    got = np.zeros(pitch * e["nzm"], dt)
    gja = np.zeros(pitch * e["nzm"], np.int32)
    assert fr(hdl, _p(got), _p(gja), pitch, _p(np.zeros(n, np.int32)), _p(np.zeros(n, np.int32))) == 0
    exp = ev.copy().reshape(e["nzm"], pitch)
    ejr = np.asarray(e["ja"]).reshape(e["nzm"], pitch)
    for r, c, v in zip(ui[:300], uj[:300], uv[:300]):
        k = np.flatnonzero(ejr[: e["irn"][r - 1], r - 1] == c)[0]
        exp[k, r - 1] = v
    assert np.array_equal(got, exp.reshape(-1))
    lib.freeEllDevice(hdl)


# ------------------------------------------------------- triangular solve
def _triangles(n3=12, seed=0):
    """The lower and upper triangles of a 7-point operator with random
    values, in the CPU type's storage (diagonal last / first) and with a
    strengthened diagonal."""
    irp, ja, va = gen.poisson7(n3)
    n = len(irp) - 1
    rng = np.random.default_rng(seed)
    va = rng.uniform(-1, 1, len(va))
    rows = np.repeat(np.arange(n), np.diff(irp))
    cols = ja - 1
    out = {}
    for lower in (True, False):
        keep = cols <= rows if lower else cols >= rows
        r, c, v = rows[keep], cols[keep], va[keep]
        v = np.where(r == c, 4.0 + np.abs(v), v)
        # CPU storage: off-diagonals ascending, diagonal last (lower) / first (upper)
        key = np.where(r == c, (n if lower else -1), c)
        o = np.lexsort((key, r))
        r, c, v = r[o], c[o], v[o]
        rp = np.zeros(n + 1, np.int64)
        np.add.at(rp, r + 1, 1)
        rp = np.cumsum(rp) + 1
        out[lower] = (rp.astype(np.int32), (c + 1).astype(np.int32), v)
    return n, out


def _strict(irp, ja, va):
    n = len(irp) - 1
    rows = np.repeat(np.arange(n), np.diff(irp))
    keep = ja - 1 != rows
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, rows[keep] + 1, 1)
    return (np.cumsum(rp) + 1).astype(np.int32), ja[keep], va[keep]


def _solve(psb, irp, ja, va, lower, unit, alpha, x):
    from psblas3_b200._lib import lib
    Cm = psb.CsrMat(len(irp) - 1, irp, ja, va)
    assert lib.d_CSRGIsNullSvBuffer(C.byref(Cm.cm)) == 1
    assert lib.d_CSRGDeviceSetMatFillMode(C.byref(Cm.cm), 0 if lower else 1) == 0
    assert lib.d_CSRGDeviceSetMatDiagType(C.byref(Cm.cm), 1 if unit else 0) == 0
    X, Y = psb.DVect.bld(x), psb.DVect(len(x))
    assert lib.d_spsvCSRGDevice(C.byref(Cm.cm), alpha, X.h, 0.0, Y.h) == 0
    assert lib.d_CSRGIsNullSvBuffer(C.byref(Cm.cm)) == 0
    y = Y.get_vect()
    # a second solve on the same handle (next generation of the row flags)
    assert lib.d_spsvCSRGDevice(C.byref(Cm.cm), alpha, X.h, 0.0, Y.h) == 0
    assert np.array_equal(Y.get_vect(), y)
    Cm.free()
    return y


@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("unit", [False, True])
@pytest.mark.parametrize("alpha", [1.0, -1.0, 2.5])
def test_csr_triangular_solve(psb, lower, unit, alpha):
    n, tri = _triangles()
    irp, ja, va = tri[lower]
    x = np.random.default_rng(1).uniform(-1, 1, n)
    if unit:
        cpu = _strict(irp, ja, va)   # the CPU type stores no diagonal when unit
        ref = O.csr_trsv(*cpu, lower, True, alpha, x)
        # the device matrix as the GPU glue builds it (diagonal stored, ignored)
        got = _solve(psb, irp, ja, va, lower, True, alpha, x)
        assert np.array_equal(got, ref)
        got2 = _solve(psb, *cpu, lower, True, alpha, x)
        assert np.array_equal(got2, ref)
    else:
        ref = O.csr_trsv(irp, ja, va, lower, False, alpha, x)
        got = _solve(psb, irp, ja, va, lower, False, alpha, x)
        assert np.array_equal(got, ref)


def test_csr_triangular_solve_long_chain(psb):
    """A bidiagonal matrix: every row waits for the one before it (a
    dependency chain as long as the matrix)."""
    n = 200_000
    rng = np.random.default_rng(7)
    irp = np.concatenate([[1], 2 * np.arange(1, n + 1)]).astype(np.int32)  # row 0: 1 entry, the others 2
    ja = np.empty(2 * n - 1, np.int32)
    va = np.empty(2 * n - 1)
    ja[0], va[0] = 1, 2.0
    k = np.arange(1, n)
    ja[2 * k - 1], ja[2 * k] = k, k + 1
    va[2 * k - 1], va[2 * k] = rng.uniform(-1, 1, n - 1), 2.0 + rng.uniform(0, 1, n - 1)
    assert irp[-1] == 2 * n
    x = rng.uniform(-1, 1, n)
    ref = O.csr_trsv(irp, ja, va, True, False, 1.0, x)
    got = _solve(psb, irp, ja, va, True, False, 1.0, x)
    assert np.array_equal(got, ref)
