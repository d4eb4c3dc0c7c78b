"""CPU oracle for the PSBLAS single-GPU sparse Krylov path.

TEST INFRASTRUCTURE ONLY.  This package restates the reference's CPU path
(conversion COO->CSR/HLL/ELL, csmv, vector kernels, diagonal preconditioner,
CG and BiCGSTAB) in plain C (``oracle.c``).  Only ``tests/``, the smoke check
and the CPU-baseline leg of ``bench.py`` may import it; the product library
never calls it and has no CPU fallback.

All index arrays are 1-based int32 like the reference Fortran; values FP64.

``ref_gpu()`` loads the reference's own GPU kernels (SPGPU HLL SpMV, dot,
nrm2, axpby, diagonal product), compiled from the psblas3 sources for sm_100a
into ``oracle/_ref/`` by ``make -C oracle ref``, with ``ref_cg.c`` driving
them in psb_dcg's call sequence: a second, executed reference for the GPU
SpMV (tests) and the reference's GPU timings beside the CPU path (bench.py's
reference arm).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile liboracle.so with the committed Makefile (CPU only)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_REF_GPU_PATH = os.path.join(_HERE, "_ref", "libspgpu_ref.so")


def ref_source_dir() -> str:
    """Location of the psblas3 source tree: $PSBLAS_SRC, else the checkout
    this build recipe was written against (/root/reference)."""
    return os.environ.get("PSBLAS_SRC", "/root/reference")


def build_ref() -> bool:
    """Compile the reference's SPGPU kernels into oracle/_ref/ when the
    psblas3 sources are present (they are not on every machine: without them
    an existing oracle/_ref/ build is used, and the tests that need it skip)."""
    src = ref_source_dir()
    if not os.path.exists(os.path.join(src, "cuda", "spgpu", "kernels", "hell_dspmv.cu")):
        if not os.path.exists(_REF_GPU_PATH):
            print(f"oracle: psblas3 sources not found at {src} (set PSBLAS_SRC); "
                  "oracle/_ref/ not built")
        return os.path.exists(_REF_GPU_PATH)
    subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={src}"], check=True)
    return True


class RefGpu:
    """ctypes handle on spgpuCreate / spgpuDhellspmv / spgpuGetStream
    (cuda/spgpu/core.h, cuda/spgpu/hell.h:74-107)."""

    def __init__(self, path, device=0):
        L = C.CDLL(path)
        P, I, D = C.c_void_p, C.c_int, C.c_double
        L.spgpuCreate.restype = I
        L.spgpuCreate.argtypes = [C.POINTER(P), I]
        L.spgpuDestroy.restype = None
        L.spgpuDestroy.argtypes = [P]
        L.spgpuGetStream.restype = P
        L.spgpuGetStream.argtypes = [P]
        L.spgpuDhellspmv.restype = None
        L.spgpuDhellspmv.argtypes = [P, P, P, D, P, P, I, P, P, P, I, I, P, D, I]
        L.refg_cg.restype = I
        L.refg_cg.argtypes = [I, P, P, P, P, I, P, P, P, D, I, C.POINTER(I), C.POINTER(D)]
        self.L = L
        self.h = P()
        if L.spgpuCreate(C.byref(self.h), int(device)) != 0:
            raise RuntimeError("spgpuCreate failed")

    @property
    def stream(self):
        return self.L.spgpuGetStream(self.h)

    def hll_spmv(self, z, y, alpha, cM, rP, hksz, hkoffs, rS, avg_nzr, rows, x, beta, base=1):
        """z = alpha*A*x + beta*y exactly as spmvHllDeviceDouble calls it
        (cuda/hlldev.c:185-207: no row permutation); device pointers (int)."""
        self.L.spgpuDhellspmv(self.h, z, y, float(alpha), cM, rP, int(hksz), hkoffs, rS, None, int(avg_nzr),
                              int(rows), x, float(beta), int(base))

    def cg(self, n, cM, rP, hkoffs, rS, avg_nzr, dinv, b, x, eps, itmax):
        """psb_dcg on the reference's GPU kernels (ref_cg.c); device pointers
        (int; dinv may be None); returns (iter, err)."""
        it, err = C.c_int(0), C.c_double(0.0)
        rc = self.L.refg_cg(int(n), cM, rP, hkoffs, rS, int(avg_nzr), dinv, b, x, float(eps), int(itmax),
                            C.byref(it), C.byref(err))
        if rc != 0:
            raise RuntimeError(f"refg_cg failed rc={rc}")
        return it.value, err.value

    def close(self):
        if self.h:
            self.L.spgpuDestroy(self.h)
            self.h = C.c_void_p()


def ref_gpu(device=0):
    """The reference's GPU kernels, or None when oracle/_ref/ holds no build."""
    if not os.path.exists(_REF_GPU_PATH):
        return None
    return RefGpu(_REF_GPU_PATH, device)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        I, D, I64, CH = C.c_int, C.c_double, C.c_int64, C.c_char
        sig = {
            "or_set_threads": (None, [I]),
            "or_get_threads": (I, []),
            "or_coo_fix": (I64, [I, I64, _i32p, _i32p, _f64p]),
            "or_csr_from_coo": (None, [I, I64, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p]),
            "or_hll_alloc_size": (I64, [I, I64, _i32p, I]),
            "or_hll_from_coo": (I, [I, I64, _i32p, _i32p, _f64p, I, _i32p, _i32p, _i32p, _f64p, _i32p]),
            "or_ell_max_row": (I, [I, I64, _i32p]),
            "or_ell_from_coo": (I, [I, I64, _i32p, _i32p, _f64p, I, I, _i32p, _i32p, _f64p, _i32p]),
            "or_csr_csmv": (I, [CH, I, I, _i32p, _i32p, _f64p, D, _f64p, D, _f64p]),
            "or_hll_csmv": (I, [CH, I, I, I, _i32p, _i32p, _i32p, _f64p, D, _f64p, D, _f64p]),
            "or_ell_csmv": (I, [CH, I, I, I, I, _i32p, _i32p, _f64p, D, _f64p, D, _f64p]),
            "or_hll_get_diag": (I, [I, I, _i32p, _i32p, _f64p, _i32p, _f64p]),
            "or_axpby": (None, [I, D, _f64p, D, _f64p]),
            "or_axpbyz": (None, [I, D, _f64p, D, _f64p, _f64p]),
            "or_dot": (D, [I, _f64p, _f64p]),
            "or_nrm2": (D, [I, _f64p]),
            "or_amax": (D, [I, _f64p]),
            "or_asum": (D, [I, _f64p]),
            "or_mlt": (None, [I, D, _f64p, _f64p, D, _f64p]),
            "or_upd_xyz": (None, [I, D, D, D, D, _f64p, _f64p, _f64p]),
            "or_xyzw": (None, [I, D, D, D, D, D, D, _f64p, _f64p, _f64p, _f64p]),
            "or_diag_prec_build": (None, [I, _f64p, _f64p]),
            "or_hll_csmv_f32": (I, [I, I, I, _i32p, _i32p, _i32p, _f32p, C.c_float, _f32p, C.c_float, _f32p]),
            "or_ell_csmv_f32": (I, [I, I, _i32p, _i32p, _f32p, C.c_float, _f32p, C.c_float, _f32p]),
            "or_csr_trsv": (I, [I, _i32p, _i32p, _f64p, I, I, D, _f64p, _f64p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        for name in ("or_cg", "or_bicgstab", "or_fcg", "or_cgs", "or_bicg"):
            f = getattr(L, name)
            f.restype = I
            f.argtypes = [I, _i32p, _i32p, _f64p, C.c_void_p, _f64p, _f64p, D, I, I,
                          C.POINTER(I), C.POINTER(D), C.c_void_p]
        for name in ("or_rgmres", "or_bicgstabl"):
            f = getattr(L, name)
            f.restype = I
            f.argtypes = [I, _i32p, _i32p, _f64p, C.c_void_p, _f64p, _f64p, D, I, I, I,
                          C.POINTER(I), C.POINTER(D), C.c_void_p]
        L.or_drotg.restype = None
        L.or_drotg.argtypes = [C.POINTER(D)] * 4
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---------------------------------------------------------------- assembly
def coo_fix(nr, ia, ja, val):
    """Sort by (row, col) stably and add duplicates (psb_d_fix_coo)."""
    ia, ja, val = _i32(ia).copy(), _i32(ja).copy(), _f64(val).copy()
    nz = lib().or_coo_fix(int(nr), len(ia), ia, ja, val)
    return ia[:nz], ja[:nz], val[:nz]


def csr_from_coo(nr, ia, ja, val):
    ia, ja, val = _i32(ia), _i32(ja), _f64(val)
    irp = np.zeros(nr + 1, np.int32)
    cja = np.zeros(len(ja), np.int32)
    cval = np.zeros(len(val), np.float64)
    lib().or_csr_from_coo(int(nr), len(ia), ia, ja, val, irp, cja, cval)
    return irp, cja, cval


def hll_from_coo(nr, ia, ja, val, hksz=32):
    """Row-sorted COO -> HLL (psi_d_convert_hll_from_coo)."""
    ia, ja, val = _i32(ia), _i32(ja), _f64(val)
    isz = lib().or_hll_alloc_size(int(nr), len(ia), ia, int(hksz))
    noffs = (nr + hksz - 1) // hksz
    irn = np.zeros(nr, np.int32)
    hkoffs = np.zeros(noffs + 1, np.int32)
    hja = np.zeros(max(isz, 1), np.int32)
    hval = np.zeros(max(isz, 1), np.float64)
    idiag = np.zeros(nr, np.int32)
    lib().or_hll_from_coo(int(nr), len(ia), ia, ja, val, int(hksz), irn, hkoffs, hja, hval, idiag)
    return dict(irn=irn, hkoffs=hkoffs, ja=hja[:isz], val=hval[:isz], idiag=idiag, hksz=hksz)


def ell_from_coo(nr, ia, ja, val, ldv=None):
    """Row-sorted COO -> ELL (psi_d_convert_ell_from_coo); ldv >= nr rows."""
    ia, ja, val = _i32(ia), _i32(ja), _f64(val)
    ldv = nr if ldv is None else int(ldv)
    nzm = lib().or_ell_max_row(int(nr), len(ia), ia)
    irn = np.zeros(nr, np.int32)
    idiag = np.zeros(nr, np.int32)
    eja = np.zeros(max(ldv * nzm, 1), np.int32)
    eval_ = np.zeros(max(ldv * nzm, 1), np.float64)
    lib().or_ell_from_coo(int(nr), len(ia), ia, ja, val, ldv, nzm, irn, eja, eval_, idiag)
    return dict(irn=irn, ja=eja[: ldv * nzm], val=eval_[: ldv * nzm], idiag=idiag, ldv=ldv, nzm=nzm)


# ---------------------------------------------------------------- SpMV
def csr_csmv(irp, ja, val, alpha, x, beta, y, trans="N", nc=None):
    nr = len(irp) - 1
    nc = nr if nc is None else nc
    y = _f64(y).copy()
    lib().or_csr_csmv(trans.encode(), nr, int(nc), _i32(irp), _i32(ja), _f64(val),
                      float(alpha), _f64(x), float(beta), y)
    return y


def hll_csmv(h, nr, alpha, x, beta, y, trans="N", nc=None):
    nc = nr if nc is None else nc
    y = _f64(y).copy()
    lib().or_hll_csmv(trans.encode(), int(nr), int(nc), int(h["hksz"]), h["irn"], h["hkoffs"],
                      _i32(h["ja"]) if len(h["ja"]) else np.zeros(1, np.int32),
                      _f64(h["val"]) if len(h["val"]) else np.zeros(1),
                      float(alpha), _f64(x), float(beta), y)
    return y


def ell_csmv(e, nr, alpha, x, beta, y, trans="N", nc=None):
    nc = nr if nc is None else nc
    y = _f64(y).copy()
    lib().or_ell_csmv(trans.encode(), int(nr), int(nc), int(e["ldv"]), int(e["nzm"]), e["irn"],
                      _i32(e["ja"]) if len(e["ja"]) else np.zeros(1, np.int32),
                      _f64(e["val"]) if len(e["val"]) else np.zeros(1),
                      float(alpha), _f64(x), float(beta), y)
    return y


def hll_csmv_f32(h, nr, alpha, x, beta, y, reference_fp32=False):
    """FP32 HLL product (not transposed).  By default the library's
    documented form (FP64 sums of exact products, rounded once); with
    reference_fp32 the reference's FP32 accumulation (psb_s_hll_csmv)."""
    y = np.ascontiguousarray(y, np.float32).copy()
    lib().or_hll_csmv_f32(1 if reference_fp32 else 0, int(nr), int(h["hksz"]), _i32(h["irn"]), _i32(h["hkoffs"]),
                          _i32(h["ja"]) if len(h["ja"]) else np.zeros(1, np.int32),
                          np.ascontiguousarray(h["val"], np.float32) if len(h["val"]) else np.zeros(1, np.float32),
                          float(alpha), np.ascontiguousarray(x, np.float32), float(beta), y)
    return y


def ell_csmv_f32(e, nr, alpha, x, beta, y):
    """FP32 ELL product in the library's documented form (as hll_csmv_f32)."""
    y = np.ascontiguousarray(y, np.float32).copy()
    lib().or_ell_csmv_f32(int(nr), int(e["ldv"]), _i32(e["irn"]), _i32(e["ja"]),
                          np.ascontiguousarray(e["val"], np.float32), float(alpha),
                          np.ascontiguousarray(x, np.float32), float(beta), y)
    return y


def csr_trsv(irp, ja, val, lower, unit, alpha, x):
    """psb_d_csr_cssv restated (not transposed, beta 0): y = alpha*T^{-1}x
    with the CPU type's triangle storage (diagonal last in a lower row, first
    in an upper row, absent when unit)."""
    n = len(irp) - 1
    y = np.zeros(n)
    lib().or_csr_trsv(n, _i32(irp), _i32(ja), _f64(val), int(bool(lower)), int(bool(unit)), float(alpha),
                      _f64(x), y)
    return y


def hll_get_diag(h, nr):
    d = np.zeros(nr, np.float64)
    lib().or_hll_get_diag(int(nr), int(h["hksz"]), h["irn"], h["hkoffs"],
                          _f64(h["val"]) if len(h["val"]) else np.zeros(1), h["idiag"], d)
    return d


# ---------------------------------------------------------------- vectors
def axpby(alpha, x, beta, y):
    y = _f64(y).copy()
    lib().or_axpby(len(y), float(alpha), _f64(x), float(beta), y)
    return y


def axpbyz(alpha, x, beta, y):
    z = np.zeros(len(y))
    lib().or_axpbyz(len(y), float(alpha), _f64(x), float(beta), _f64(y), z)
    return z


def dot(x, y):
    return lib().or_dot(len(x), _f64(x), _f64(y))


def nrm2(x):
    return lib().or_nrm2(len(x), _f64(x))


def amax(x):
    return lib().or_amax(len(x), _f64(x))


def asum(x):
    return lib().or_asum(len(x), _f64(x))


def mlt(alpha, d, x, beta, z):
    z = _f64(z).copy()
    lib().or_mlt(len(z), float(alpha), _f64(d), _f64(x), float(beta), z)
    return z


def upd_xyz(alpha, beta, gamma, delta, x, y, z):
    y, z = _f64(y).copy(), _f64(z).copy()
    lib().or_upd_xyz(len(y), alpha, beta, gamma, delta, _f64(x), y, z)
    return y, z


def xyzw(a, b, c, d, e, f, x, y, z, w):
    y, z, w = _f64(y).copy(), _f64(z).copy(), _f64(w).copy()
    lib().or_xyzw(len(y), a, b, c, d, e, f, _f64(x), y, z, w)
    return y, z, w


# FP32 vectors (the s type): the CPU loops of psi_s_serial_impl.F90 are the
# FP64 ones with real(psb_spk_) -- every multiply and add rounded to FP32,
# which numpy's float32 operations do one at a time.  The reductions restate
# the library's documented form: dot and nrm2 are the compensated FP64 sums
# of the (exact) FP64 products rounded to FP32 once, asum the FP64 sum
# rounded once, amax exact.
_F = np.float32


def saxpby(alpha, x, beta, y):
    x, y = np.asarray(x, _F), np.asarray(y, _F)
    a, b = _F(alpha), _F(beta)
    if a == 0:
        return np.zeros_like(y) if b == 0 else (y.copy() if b == 1 else b * y)
    return a * x if b == 0 else a * x + b * y


def _axpby_el(a, x, b, y):
    if a == 0:
        return np.zeros_like(y) if b == 0 else b * y
    return a * x if b == 0 else a * x + b * y


def supd_xyz(alpha, beta, gamma, delta, x, y, z):
    x, y, z = (np.asarray(v, _F) for v in (x, y, z))
    yy = _axpby_el(_F(alpha), x, _F(beta), y)
    return yy, _axpby_el(_F(gamma), yy, _F(delta), z)


def sxyzw(a, b, c, d, e, f, x, y, z, w):
    x, y, z, w = (np.asarray(v, _F) for v in (x, y, z, w))
    yy = _F(a) * x + _F(b) * y
    zz = _F(c) * yy + _F(d) * z
    return yy, zz, _F(e) * zz + _F(f) * w


def smlt(alpha, d, x, beta, z):
    t = _F(alpha) * (np.asarray(d, _F) * np.asarray(x, _F))
    return t if _F(beta) == 0 else t + _F(beta) * np.asarray(z, _F)


def sdot(x, y):
    return _F(dot(np.asarray(x, _F).astype(np.float64), np.asarray(y, _F).astype(np.float64)))


def snrm2(x):
    return _F(nrm2(np.asarray(x, _F).astype(np.float64)))


def sasum(x):
    return _F(asum(np.asarray(x, _F).astype(np.float64)))


def samax(x):
    return _F(np.max(np.abs(np.asarray(x, _F)))) if len(x) else _F(0)


def diag_prec_build(diag):
    d = np.zeros(len(diag))
    lib().or_diag_prec_build(len(diag), _f64(diag), d)
    return d


# ---------------------------------------------------------------- Krylov
def krylov(method, irp, ja, val, b, x0=None, dinv=None, eps=1e-6, itmax=1000, istop=2,
           history=False, irst=10):
    """psb_krylov('CG'|'FCG'|'CGS'|'BICG'|'BICGSTAB'|'BICGSTABL'|'RGMRES') restated; returns
    (x, iter, err[, hist]).  irst is the GMRES restart length."""
    n = len(irp) - 1
    x = np.zeros(n) if x0 is None else _f64(x0).copy()
    it, err = C.c_int(0), C.c_double(0.0)
    hist = np.full(itmax + irst + 2, np.nan) if history else None
    d = None if dinv is None else _f64(dinv)
    m = method.upper()
    args = [n, _i32(irp), _i32(ja), _f64(val), None if d is None else d.ctypes.data_as(C.c_void_p),
            _f64(b), x, float(eps), int(itmax), int(istop)]
    if m in ("RGMRES", "GMRES", "BICGSTABL"):
        args.append(int(irst))
        f = lib().or_bicgstabl if m == "BICGSTABL" else lib().or_rgmres
    else:
        f = {"CG": lib().or_cg, "BICGSTAB": lib().or_bicgstab, "FCG": lib().or_fcg, "CGS": lib().or_cgs,
             "BICG": lib().or_bicg}[m]
    rc = f(*args, C.byref(it), C.byref(err), None if hist is None else hist.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise ValueError(f"oracle krylov failed rc={rc}")
    if history:
        return x, it.value, err.value, hist
    return x, it.value, err.value
