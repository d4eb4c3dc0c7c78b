"""Host-side mirror of the PSBLAS objects on this path, over the C-ABI.

Names and argument meaning follow the reference so tests read like its
drivers:

* ``DVect``        -- psb_d_vect_cuda (cuda/psb_d_cuda_vect_mod.F90:48-106):
                      a device multivector handle plus a host copy.
* ``HllMat``       -- psb_d_cuda_hlg_sparse_mat (HLL on the device), built
                      from host HLL arrays (to_gpu / writeHllDevice), from
                      row-sorted COO via psiCopyCooToHlg, or on the device
                      from CSR (psbx_hll_from_csr_device).
* ``EllMat``       -- psb_d_cuda_elg_sparse_mat.
* ``CsrMat``       -- psb_d_cuda_csrg_sparse_mat (d_CSRG* entry points).
* ``DiagPrec``     -- prec%init('DIAG') / prec%build (psb_d_diagprec).
* ``psb_spmm``, ``psb_geaxpby``, ``psb_gedot``, ``psb_genrm2``, ``psb_geamax``,
  ``psb_geasum``, ``psb_gemlt``, ``psb_krylov`` -- base/psblas/* and
  krylov/psb_dkrylov.f90 entry points (np = 1: no halo, no allreduce).

Every call goes through libpsbx.so; there is no CPU fallback.  Errors raise
PsbxError carrying the C-ABI status code (the reference's ``info``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import check, lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def init(dev: int = 0) -> None:
    """psb_cuda_init -> gpuInit (cuda/psb_cuda_env_mod.F90:43-60)."""
    check(lib.gpuInit(int(dev)), "gpuInit")


# ------------------------------------------------------------------ vectors
_VT = {np.dtype(np.float64): ("Double", L.SPGPU_TYPE_DOUBLE), np.dtype(np.float32): ("Float", L.SPGPU_TYPE_FLOAT),
       np.dtype(np.int32): ("Int", L.SPGPU_TYPE_INT)}


class DVect:
    """One (count=1) or several (count>1) device vectors of FP64 (the d
    type), FP32 (the s type) or int32 (the i type) entries."""

    def __init__(self, n: int, count: int = 1, dtype=np.float64, zero: bool = True):
        """zero: start from zeros (psb_geall + psb_geasb); the C entry point
        FallocMultiVecDevice itself leaves the memory as cudaMalloc gives it,
        as the reference's does."""
        self.n = int(n)
        self.count = int(count)
        self.dtype = np.dtype(dtype)
        self.tname, et = _VT[self.dtype]
        h = C.c_void_p()
        check(lib.FallocMultiVecDevice(C.byref(h), self.count, self.n, et), "FallocMultiVecDevice")
        self.h = h
        self.pitch = lib.getMultiVecDevicePitch(self.h)
        if zero:
            self.zero()

    @classmethod
    def bld(cls, x):
        """psb_d_vect_cuda%bld(x): allocate and copy host data to the device."""
        x = np.asarray(x)
        dt = x.dtype if x.dtype in (np.float32, np.int32) else np.float64
        v = cls(x.shape[0], 1 if x.ndim == 1 else x.shape[1], dt, zero=False)
        v.set_vect(x)
        return v

    def _host(self, x):
        x = np.asarray(x, dtype=self.dtype)
        if self.count == 1:
            return np.ascontiguousarray(x.reshape(self.n))
        buf = np.zeros((self.count, self.pitch), self.dtype)
        buf[:, : self.n] = x.reshape(self.n, self.count).T
        return buf

    def set_vect(self, x):
        buf = self._host(x)
        check(getattr(lib, "writeMultiVecDevice" + self.tname)(self.h, _ptr(buf)), "writeMultiVecDevice")

    def get_vect(self):
        buf = np.zeros((self.count, self.pitch), self.dtype)
        check(getattr(lib, "readMultiVecDevice" + self.tname)(self.h, _ptr(buf)), "readMultiVecDevice")
        out = buf[:, : self.n]
        return out[0].copy() if self.count == 1 else out.T.copy()

    @property
    def data_ptr(self):
        """Device address of the vector data (int)."""
        return lib.psbx_multivec_data(self.h)

    def set_scal(self, val, first=1, last=None):
        last = self.n if last is None else last
        v = int(val) if self.dtype == np.int32 else float(val)
        check(getattr(lib, "setscalMultiVecDevice" + self.tname)(v, int(first), int(last), 1, self.h), "setscal")

    def zero(self):
        """Every element of every vector (padding included) to 0."""
        self.set_scal(0, 1, self.pitch * self.count)

    def scal(self, alpha):
        check(getattr(lib, "scalMultiVecDevice" + self.tname)(float(alpha), self.h), "scal")

    def free(self):
        if self.h:
            lib.freeMultiVecDevice(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ------------------------------------------------------------------ matrices
class HllMat:
    fmt = L.PSBX_FMT_HLL

    def __init__(self, h, rows):
        self.h = h
        self.rows = rows

    @classmethod
    def from_host_hll(cls, rows, hksz, irn, hkoffs, ja, val, idiag, nnz=None):
        """to_gpu: FallocHllDevice + writeHllDeviceDouble with host HLL arrays
        (psb_d_cuda_hlg_to_gpu.F90:56-58)."""
        ja = np.ascontiguousarray(ja, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        irn = np.ascontiguousarray(irn, np.int32)
        hkoffs = np.ascontiguousarray(hkoffs, np.int32)
        idiag = np.ascontiguousarray(idiag, np.int32)
        nnz = int(irn.sum()) if nnz is None else nnz
        h = C.c_void_p()
        check(lib.FallocHllDevice(C.byref(h), hksz, rows, nnz, len(val), L.SPGPU_TYPE_DOUBLE, 1), "FallocHllDevice")
        check(lib.writeHllDeviceDouble(h, _ptr(val), _ptr(ja), _ptr(hkoffs), _ptr(irn), _ptr(idiag)),
              "writeHllDeviceDouble")
        return cls(h, rows)

    @classmethod
    def from_coo_gpu(cls, rows, ia, ja, val, hksz=32):
        """psb_d_cuda_cp_hlg_from_coo (GPU scatter path): host hack offsets
        and idisp (psb_d_cuda_cp_hlg_from_coo.F90:117-188), then
        psiCopyCooToHlgDouble."""
        ia = np.ascontiguousarray(ia, np.int32)
        ja = np.ascontiguousarray(ja, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        irn = np.bincount(ia - 1, minlength=rows).astype(np.int32)
        noffs = (rows + hksz - 1) // hksz
        pad = np.zeros(noffs * hksz, np.int64)
        pad[:rows] = irn
        width = pad.reshape(noffs, hksz).max(axis=1) if noffs else np.zeros(0, np.int64)
        hkoffs = np.zeros(noffs + 1, np.int64)
        np.cumsum(width * hksz, out=hkoffs[1:])
        idisp = np.zeros(rows + 1, np.int64)
        np.cumsum(irn, out=idisp[1:])
        isz = int(hkoffs[-1])
        hkoffs32, idisp32 = hkoffs.astype(np.int32), idisp.astype(np.int32)
        h = C.c_void_p()
        check(lib.FallocHllDevice(C.byref(h), hksz, rows, len(ia), isz, L.SPGPU_TYPE_DOUBLE, 1), "FallocHllDevice")
        check(lib.psiCopyCooToHlgDouble(rows, rows, len(ia), hksz, noffs, isz, _ptr(irn), _ptr(hkoffs32),
                                        _ptr(idisp32), _ptr(ja), _ptr(val), h), "psiCopyCooToHlgDouble")
        return cls(h, rows)

    @classmethod
    def from_csr_device(cls, rows, cols, nnz, d_irp, d_ja, d_val, hksz=32, d_perm=None):
        """Device CSR (raw device pointers, 1-based) -> device HLL."""
        h = C.c_void_p()
        check(lib.psbx_hll_from_csr_device(C.byref(h), rows, cols, nnz, C.c_void_p(d_irp), C.c_void_p(d_ja),
                                           C.c_void_p(d_val), hksz,
                                           None if d_perm is None else C.c_void_p(d_perm)),
              "psbx_hll_from_csr_device")
        return cls(h, rows)

    @classmethod
    def autotune_from_csr_device(cls, rows, cols, nnz, d_irp, d_ja, d_val, d_perm=None):
        """Device CSR (raw device pointers, 1-based) -> the HLL layout with the
        fastest SpMV among hack sizes 32/64/128, wide-hack thresholds and
        threads per row; returns (HllMat, {"hksz", "wide_w", "tpr", "ms"}),
        the matrix in the tolerance mode."""
        h = C.c_void_p()
        hk, ww, ms = C.c_int(0), C.c_int(0), C.c_double(0.0)
        check(lib.psbx_hll_autotune_from_csr_device(C.byref(h), rows, cols, nnz, C.c_void_p(d_irp),
                                                    C.c_void_p(d_ja), C.c_void_p(d_val),
                                                    None if d_perm is None else C.c_void_p(d_perm),
                                                    C.byref(hk), C.byref(ww), C.byref(ms)),
              "psbx_hll_autotune_from_csr_device")
        mat = cls(h, rows)
        return mat, {"hksz": hk.value, "wide_w": ww.value, "tpr": mat.layout()["tpr"], "ms": ms.value}

    def set_wide(self, wide_w):
        """Wide-hack threshold (hack size 32): 0 default, < 0 never; in the
        exact mode the same bits for every choice."""
        check(lib.psbx_hll_set_wide(self.h, int(wide_w)), "psbx_hll_set_wide")
        return self

    def set_wide_split(self, split=True):
        """Tolerance mode (True, the default: wide hacks summed split over 8
        warps, two threads per row allowed; every row within 1e-13 of
        (|A||x|)_i) or exact mode (False: every row in stored order, the CPU
        csmv's bits)."""
        check(lib.psbx_hll_set_wide_split(self.h, int(bool(split))), "psbx_hll_set_wide_split")
        return self

    def spmv_host(self, alpha, x, beta, y, chunks=0):
        """y = alpha*A*x + beta*y for host arrays (numpy float64, or pinned
        torch tensors for overlapped copies): copies up, the product and the
        copy down in one call, overlapped block by block
        (psbx_hll_spmv_host)."""
        def ptr(a):
            return C.c_void_p(a.data_ptr()) if hasattr(a, "data_ptr") else a.ctypes.data_as(C.c_void_p)
        check(lib.psbx_hll_spmv_host(self.h, float(alpha), ptr(x), float(beta), ptr(y), int(chunks)),
              "psbx_hll_spmv_host")
        return y

    def set_threads_per_row(self, tpr):
        """Row mapping of the standalone SpMV (hack size 32): 0 auto, 1 or 2
        threads per row (2: tolerance mode only), -2 two rows per thread."""
        check(lib.psbx_hll_set_threads_per_row(self.h, int(tpr)), "psbx_hll_set_threads_per_row")
        return self

    def layout(self):
        hk, ww, sp, tp = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
        check(lib.psbx_hll_get_layout(self.h, C.byref(hk), C.byref(ww), C.byref(sp), C.byref(tp)),
              "psbx_hll_get_layout")
        return {"hksz": hk.value, "wide_w": ww.value, "split": sp.value, "tpr": tp.value}

    def params(self):
        v = [C.c_int() for _ in range(7)]
        check(lib.getHllDeviceParams(self.h, *[C.byref(t) for t in v]), "getHllDeviceParams")
        keys = ("hksz", "rows", "nzeros", "allocsize", "hackOffsLength", "firstIndex", "avgnzr")
        return dict(zip(keys, (t.value for t in v)))

    def read(self):
        """from_gpu: readHllDeviceDouble into host arrays."""
        p = self.params()
        val = np.zeros(max(p["allocsize"], 1))
        ja = np.zeros(max(p["allocsize"], 1), np.int32)
        hk = np.zeros(p["hackOffsLength"] + 1, np.int32)
        irn = np.zeros(max(p["rows"], 1), np.int32)
        idg = np.zeros(max(p["rows"], 1), np.int32)
        check(lib.readHllDeviceDouble(self.h, _ptr(val), _ptr(ja), _ptr(hk), _ptr(irn), _ptr(idg)), "readHll")
        n, a = p["rows"], p["allocsize"]
        return dict(val=val[:a], ja=ja[:a], hkoffs=hk, irn=irn[:n], idiag=idg[:n], hksz=p["hksz"])

    def make_single(self):
        check(lib.psbx_hll_make_single(self.h), "psbx_hll_make_single")

    def spmv(self, alpha, x, beta, y):
        f = lib.spmvHllDeviceDouble if x.dtype == np.float64 else lib.spmvHllDeviceFloat
        check(f(self.h, alpha, x.h, beta, y.h), "spmvHllDevice")

    def free(self):
        if self.h:
            lib.freeHllDevice(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class EllMat:
    fmt = L.PSBX_FMT_ELL

    def __init__(self, h, rows):
        self.h = h
        self.rows = rows

    @classmethod
    def from_host_ell(cls, rows, nzm, irn, ja, val, idiag, ldv, nnz=None):
        """psb_d_cuda_elg_to_gpu: reallocate host arrays to (pitch, nzm) and
        writeEllDeviceDouble (psb_d_cuda_elg_to_gpu.F90:60-90)."""
        h = C.c_void_p()
        nnz = int(np.sum(irn)) if nnz is None else nnz
        check(lib.FallocEllDevice(C.byref(h), rows, nzm, nnz, rows, L.SPGPU_TYPE_DOUBLE, 1), "FallocEllDevice")
        pitch = lib.getEllDevicePitch(h)
        ja2 = np.ones((nzm, pitch), np.int32)
        va2 = np.zeros((nzm, pitch), np.float64)
        ja2[:, :rows] = np.asarray(ja, np.int32).reshape(nzm, ldv)[:, :rows]
        va2[:, :rows] = np.asarray(val, np.float64).reshape(nzm, ldv)[:, :rows]
        irn = np.ascontiguousarray(irn, np.int32)
        idiag = np.ascontiguousarray(idiag, np.int32)
        check(lib.writeEllDeviceDouble(h, _ptr(va2), _ptr(ja2), pitch, _ptr(irn), _ptr(idiag)), "writeEll")
        return cls(h, rows)

    @classmethod
    def from_coo_gpu(cls, rows, ia, ja, val):
        ia = np.ascontiguousarray(ia, np.int32)
        ja = np.ascontiguousarray(ja, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        irn = np.bincount(ia - 1, minlength=rows).astype(np.int32)
        nzm = int(irn.max()) if rows else 0
        idisp = np.zeros(rows + 1, np.int64)
        np.cumsum(irn, out=idisp[1:])
        idisp = idisp.astype(np.int32)
        h = C.c_void_p()
        check(lib.FallocEllDevice(C.byref(h), rows, nzm, len(ia), rows, L.SPGPU_TYPE_DOUBLE, 1), "FallocEllDevice")
        pitch = lib.getEllDevicePitch(h)
        check(lib.psiCopyCooToElgDouble(rows, rows, len(ia), 1, pitch, nzm, _ptr(irn), _ptr(idisp), _ptr(ja),
                                        _ptr(val), h), "psiCopyCooToElgDouble")
        return cls(h, rows)

    def read(self):
        pitch = lib.getEllDevicePitch(self.h)
        nzm = lib.getEllDeviceMaxRowSize(self.h)
        val = np.zeros(max(pitch * nzm, 1))
        ja = np.zeros(max(pitch * nzm, 1), np.int32)
        irn = np.zeros(max(self.rows, 1), np.int32)
        idg = np.zeros(max(self.rows, 1), np.int32)
        check(lib.readEllDeviceDouble(self.h, _ptr(val), _ptr(ja), pitch, _ptr(irn), _ptr(idg)), "readEll")
        return dict(val=val[: pitch * nzm], ja=ja[: pitch * nzm], irn=irn[: self.rows], idiag=idg[: self.rows],
                    ldv=pitch, nzm=nzm)

    def spmv(self, alpha, x, beta, y):
        check(lib.spmvEllDeviceDouble(self.h, alpha, x.h, beta, y.h), "spmvEllDeviceDouble")

    def free(self):
        if self.h:
            lib.freeEllDevice(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class CsrMat:
    fmt = L.PSBX_FMT_CSR

    def __init__(self, rows, irp, ja, val, cols=None):
        """to_gpu of psb_d_cuda_csrg_sparse_mat: d_CSRGDeviceAlloc +
        d_CSRGHost2Device (1-based arrays)."""
        self.rows = int(rows)
        self.cm = L.Cmat()
        irp = np.ascontiguousarray(irp, np.int32)
        ja = np.ascontiguousarray(ja, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        nz = len(ja)
        check(lib.d_CSRGDeviceAlloc(C.byref(self.cm), self.rows, cols or self.rows, nz), "d_CSRGDeviceAlloc")
        check(lib.d_CSRGDeviceSetMatIndexBase(C.byref(self.cm), 1), "SetMatIndexBase")
        check(lib.d_CSRGHost2Device(C.byref(self.cm), self.rows, cols or self.rows, nz, _ptr(irp), _ptr(ja),
                                    _ptr(val)), "d_CSRGHost2Device")
        self.nz = nz

    @property
    def h(self):
        return C.addressof(self.cm)

    def spmv(self, alpha, x, beta, y):
        check(lib.d_spmvCSRGDevice(C.byref(self.cm), alpha, x.h, beta, y.h), "d_spmvCSRGDevice")

    def read(self):
        irp = np.zeros(self.rows + 1, np.int32)
        ja = np.zeros(max(self.nz, 1), np.int32)
        val = np.zeros(max(self.nz, 1))
        check(lib.d_CSRGDevice2Host(C.byref(self.cm), self.rows, self.rows, self.nz, _ptr(irp), _ptr(ja),
                                    _ptr(val)), "d_CSRGDevice2Host")
        return irp, ja[: self.nz], val[: self.nz]

    def free(self):
        if self.cm.mat:
            lib.d_CSRGDeviceFree(C.byref(self.cm))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ------------------------------------------------------------------ psblas
def psb_spmm(alpha, a, x, beta, y):
    """psb_spmm(alpha, a, x, beta, y, desc_a, info) at np=1 (psb_dspmm.f90:57-310)."""
    a.spmv(float(alpha), x, float(beta), y)


def psb_geaxpby(alpha, x, beta, y, n=None):
    check(lib.axpbyMultiVecDeviceDouble(int(n or y.n), float(alpha), x.h, float(beta), y.h), "axpby")


def _red(f, name, *vs, n=None):
    out = (C.c_double * vs[0].count)()
    check(f(out, int(n or vs[0].n), *[v.h for v in vs]), name)
    return out[0] if vs[0].count == 1 else np.array(out[:])


def psb_gedot(x, y, n=None):
    return _red(lib.dotMultiVecDeviceDouble, "dot", x, y, n=n)


def psb_genrm2(x, n=None):
    return _red(lib.nrm2MultiVecDeviceDouble, "nrm2", x, n=n)


def psb_geamax(x, n=None):
    return _red(lib.amaxMultiVecDeviceDouble, "amax", x, n=n)


def psb_geasum(x, n=None):
    return _red(lib.asumMultiVecDeviceDouble, "asum", x, n=n)


def psb_gemlt(alpha, d, x, beta, z, n=None):
    """z = alpha*d.*x + beta*z (the y%mlt(alpha, dv, x, beta) of the DIAG
    apply, via axybzMultiVecDevice)."""
    check(lib.axybzMultiVecDeviceDouble(int(n or z.n), float(alpha), d.h, x.h, float(beta), z.h), "axybz")


class DiagPrec:
    """prec%init('DIAG') + prec%build(a) (psb_d_diagprec_impl.f90:229-292)."""

    def __init__(self, ptype="DIAG"):
        ptype = ptype.upper()
        if ptype not in ("DIAG", "NONE", "NOPREC"):
            raise ValueError(f"preconditioner {ptype} is not provided by this library")
        self.ptype = ptype
        self.dv = None

    def build(self, a):
        if self.ptype == "DIAG":
            self.dv = DVect(a.rows)
            check(lib.psbx_diag_prec_build(a.h if a.fmt != L.PSBX_FMT_CSR else C.c_void_p(a.h), a.fmt, self.dv.h),
                  "psbx_diag_prec_build")
        return self

    def apply(self, x, y):
        if self.dv is None:
            psb_geaxpby(1.0, x, 0.0, y)
        else:
            psb_gemlt(1.0, self.dv, x, 0.0, y)


def psb_krylov(method, a, prec, b, x, eps=1e-6, itmax=1000, istop=2, itrace=0, irst=10):
    """psb_krylov(method, a, prec, b, x, eps, desc_a, info, itmax, iter, err,
    itrace, irst, istop) for 'CG', 'FCG', 'BICGSTAB' and 'RGMRES' (irst = restart
    length), device-resident.
    Returns (iter, err); raises PsbxError on failure."""
    opt = L.SolverOptions()
    lib.psbx_DefaultSolverOptions(C.byref(opt))
    opt.eps, opt.itmax, opt.istop, opt.itrace, opt.irst = float(eps), int(itmax), int(istop), int(itrace), int(irst)
    dinv = None if (prec is None or prec.dv is None) else prec.dv.h
    mh = a.h if a.fmt != L.PSBX_FMT_CSR else C.c_void_p(a.h)
    check(lib.psbx_dkrylov(method.upper().encode(), mh, a.fmt, dinv, b.h, x.h, C.byref(opt)), "psbx_dkrylov")
    return opt.iter, opt.err


def psb_mixed_cg(a, prec, b, x, eps=1e-10, itmax=100000, delta=0.1):
    """Mixed-precision CG for one system (psbx_dmixed_cg): FP32 iterations
    with FP64-accumulated dots, FP64 residual replacement, FP64 stop test
    ||b - A x|| <= eps ||b||.  a: HllMat (hack size 32).  Returns
    (inner iterations, relative true residual, residual replacements)."""
    opt = L.SolverOptions()
    lib.psbx_DefaultSolverOptions(C.byref(opt))
    opt.eps, opt.itmax, opt.istop = float(eps), int(itmax), 2
    dinv = None if (prec is None or prec.dv is None) else prec.dv.h
    nref = C.c_int(0)
    check(lib.psbx_dmixed_cg(a.h, dinv, b.h, x.h, C.byref(opt), float(delta), C.byref(nref)), "psbx_dmixed_cg")
    return opt.iter, opt.err, nref.value


class BatchSolver:
    """Batched mixed-precision CG engine (psbx_batch_*): FP32 inner Jacobi-CG
    with FP64-accumulated dots inside FP64 iterative refinement, many
    systems advancing together; systems join and leave between steps."""

    def __init__(self, max_systems, max_rows_total, nrhs=1, inner_fp64=False):
        """inner_fp64: inner iterations in FP64 instead of FP32 (the batched
        FP64 solve)."""
        self.nrhs = int(nrhs)
        h = C.c_void_p()
        check(lib.psbx_batch_create_prec(C.byref(h), int(max_systems), int(max_rows_total), self.nrhs,
                                         64 if inner_fp64 else 32), "batch_create")
        self.h = h
        self.keep = {}
        self.max_systems = int(max_systems)
        self._fin = (C.c_int * max(1, self.max_systems))()

    def add(self, A, d_b, d_x, d_dinv=None, eps=1e-10, inner_tol=1e-2, itmax=100000, keep=None):
        """A: HllMat (hack 32); d_b, d_x, d_dinv: device pointers (ints) or
        torch tensors (rows*nrhs doubles, interleaved).  Returns the slot."""
        def ptr(t):
            return None if t is None else C.c_void_p(t if isinstance(t, int) else t.data_ptr())
        slot = C.c_int(-1)
        check(lib.psbx_batch_add(self.h, A.h, ptr(d_b), ptr(d_x), ptr(d_dinv), float(eps), float(inner_tol),
                                 int(itmax), C.byref(slot)), "batch_add")
        self.keep[slot.value] = keep
        return slot.value

    def step(self, replays=1):
        n = C.c_int(0)
        check(lib.psbx_batch_step(self.h, int(replays), C.byref(n)), "batch_step")
        return n.value

    def launch(self, replays=1):
        """Enqueue replays and the state read-back; returns at once."""
        check(lib.psbx_batch_launch(self.h, int(replays)), "batch_launch")

    def wait(self):
        """Wait for the last launch; returns the number of running slots."""
        n = C.c_int(0)
        check(lib.psbx_batch_wait(self.h, C.byref(n)), "batch_wait")
        return n.value

    def poll(self, slot):
        st, outer = C.c_int(0), C.c_int(0)
        its = (C.c_int * self.nrhs)()
        err = (C.c_double * self.nrhs)()
        check(lib.psbx_batch_poll(self.h, int(slot), C.byref(st), C.byref(outer), its, err), "batch_poll")
        return st.value, outer.value, list(its), list(err)

    def finished(self):
        """Slots whose solve has ended as of the last wait, in slot order (one
        call; poll them for their results)."""
        cnt = C.c_int(0)
        check(lib.psbx_batch_finished(self.h, self._fin, len(self._fin), C.byref(cnt)), "batch_finished")
        return list(self._fin[:min(cnt.value, len(self._fin))])

    def remove(self, slot):
        check(lib.psbx_batch_remove(self.h, int(slot)), "batch_remove")
        self.keep.pop(slot, None)

    def run(self, replays_per_step=4, max_steps=100000):
        for _ in range(max_steps):
            if self.step(replays_per_step) == 0:
                return
        raise RuntimeError("batch did not finish")

    def free(self):
        if self.h:
            lib.psbx_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def kernel_launches() -> int:
    return int(lib.psbx_kernel_launches())
