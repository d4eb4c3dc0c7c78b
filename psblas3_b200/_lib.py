"""ctypes binding of libpsbx.so (the C-ABI declared in include/psbx.h).

The shared library is built in-tree (``python -m psblas3_b200.build`` or
``__graft_entry__.build()``).  There is no fallback: if the library is
missing or cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpsbx.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"libpsbx.so not built at {LIB_PATH}; run __graft_entry__.build()")

lib = C.CDLL(LIB_PATH)

I, U, D, F, P, CH = C.c_int, C.c_uint, C.c_double, C.c_float, C.c_void_p, C.c_char_p
PI = C.POINTER(C.c_int)
PD = C.POINTER(C.c_double)
PP = C.POINTER(C.c_void_p)


class SolverOptions(C.Structure):
    """psbx_SolverOptions == psb_c_SolverOptions (cbind/krylov/psb_krylov_cbind.h:17-27)."""
    _fields_ = [("iter", C.c_int), ("itmax", C.c_int), ("itrace", C.c_int), ("irst", C.c_int),
                ("istop", C.c_int), ("eps", C.c_double), ("err", C.c_double)]


class Cmat(C.Structure):
    """psbx_d_Cmat == the interoperable d_Cmat of cuda/d_cusparse_mod.F90:36-38."""
    _fields_ = [("mat", C.c_void_p)]


PC = C.POINTER(Cmat)
PF = C.POINTER(C.c_float)


class HllDeviceParams(C.Structure):
    """psbx_HllDeviceParams == HllDeviceParams of cuda/hlldev.h:70-93."""
    _fields_ = [(k, C.c_uint) for k in ("elementType", "hackSize", "rows", "avgNzr", "nzt", "allocsize",
                                        "firstIndex")]


class EllDeviceParams(C.Structure):
    """psbx_EllDeviceParams == EllDeviceParams of cuda/elldev.h:75-97."""
    _fields_ = [(k, C.c_uint) for k in ("elementType", "pitch", "rows", "columns", "maxRowSize", "avgRowSize",
                                        "firstIndex")]

_SIGS = {
    # environment
    "gpuInit": (I, [I]), "gpuClose": (None, []), "setDevice": (I, [I]), "getDevice": (I, []),
    "getDeviceCount": (I, []), "getDeviceHasUVA": (I, []), "DeviceHasUVA": (I, []),
    "getGPUMultiProcessors": (I, []), "getGPUMemoryBusWidth": (I, []), "getGPUMemoryClockRate": (I, []),
    "getGPUWarpSize": (I, []), "getGPUMaxThreadsPerBlock": (I, []), "getGPUMaxThreadsPerMP": (I, []),
    "getGPUMaxRegistersPerBlock": (I, []), "cpyGPUNameString": (None, [C.c_char_p]),
    "cudaSync": (None, []), "cudaReset": (None, []), "psb_cudaGetHandle": (P, []),
    "psb_cudaCreateHandle": (None, []), "psb_cudaDestroyHandle": (None, []),
    "psb_cudaGetStream": (P, []), "psb_cudaSetStream": (None, [P]),
    # multivectors
    "FallocMultiVecDevice": (I, [PP, U, U, U]), "freeMultiVecDevice": (None, [P]),
    "getMultiVecDeviceSize": (I, [P]), "getMultiVecDeviceCount": (I, [P]), "getMultiVecDevicePitch": (I, [P]),
    "writeMultiVecDeviceDouble": (I, [P, P]), "writeMultiVecDeviceDoubleR2": (I, [P, P, I]),
    "readMultiVecDeviceDouble": (I, [P, P]), "readMultiVecDeviceDoubleR2": (I, [P, P, I]),
    "writeMultiVecDeviceFloat": (I, [P, P]), "readMultiVecDeviceFloat": (I, [P, P]),
    "setscalMultiVecDeviceDouble": (I, [D, I, I, I, P]), "scalMultiVecDeviceDouble": (I, [D, P]),
    "nrm2MultiVecDeviceDouble": (I, [PD, I, P]), "amaxMultiVecDeviceDouble": (I, [PD, I, P]),
    "asumMultiVecDeviceDouble": (I, [PD, I, P]), "dotMultiVecDeviceDouble": (I, [PD, I, P, P]),
    "axpbyMultiVecDeviceDouble": (I, [I, D, P, D, P]),
    "upd_xyzMultiVecDeviceDouble": (I, [I, D, D, D, D, P, P, P]),
    "xyzwMultiVecDeviceDouble": (I, [I, D, D, D, D, D, D, P, P, P, P]),
    "axyMultiVecDeviceDouble": (I, [I, D, P, P]), "axybzMultiVecDeviceDouble": (I, [I, D, P, P, D, P]),
    "absMultiVecDeviceDouble2": (I, [I, D, P, P]), "absMultiVecDeviceDouble": (I, [I, D, P]),
    "igathMultiVecDeviceDouble": (I, [P, I, I, I, P, I, P, I]),
    "igathMultiVecDeviceDoubleVecIdx": (I, [P, I, I, I, P, I, P, I]),
    "iscatMultiVecDeviceDouble": (I, [P, I, I, I, P, I, P, I, D]),
    "iscatMultiVecDeviceDoubleVecIdx": (I, [P, I, I, I, P, I, P, I, D]),
    "geinsMultiVecDeviceDouble": (I, [I, P, P, I, I, P]),
    # plain device buffers and mapped host memory
    "unregisterMapped": (I, [P]),
    # FP32 vectors
    "writeMultiVecDeviceFloatR2": (I, [P, P, I]), "readMultiVecDeviceFloatR2": (I, [P, P, I]),
    "setscalMultiVecDeviceFloat": (I, [F, I, I, I, P]), "scalMultiVecDeviceFloat": (I, [F, P]),
    "nrm2MultiVecDeviceFloat": (I, [PF, I, P]), "amaxMultiVecDeviceFloat": (I, [PF, I, P]),
    "asumMultiVecDeviceFloat": (I, [PF, I, P]), "dotMultiVecDeviceFloat": (I, [PF, I, P, P]),
    "axpbyMultiVecDeviceFloat": (I, [I, F, P, F, P]),
    "upd_xyzMultiVecDeviceFloat": (I, [I, F, F, F, F, P, P, P]),
    "xyzwMultiVecDeviceFloat": (I, [I, F, F, F, F, F, F, P, P, P, P]),
    "axyMultiVecDeviceFloat": (I, [I, F, P, P]), "axybzMultiVecDeviceFloat": (I, [I, F, P, P, F, P]),
    "absMultiVecDeviceFloat2": (I, [I, F, P, P]), "absMultiVecDeviceFloat": (I, [I, F, P]),
    "igathMultiVecDeviceFloat": (I, [P, I, I, I, P, I, P, I]),
    "igathMultiVecDeviceFloatVecIdx": (I, [P, I, I, I, P, I, P, I]),
    "iscatMultiVecDeviceFloat": (I, [P, I, I, I, P, I, P, I, F]),
    "iscatMultiVecDeviceFloatVecIdx": (I, [P, I, I, I, P, I, P, I, F]),
    "geinsMultiVecDeviceFloat": (I, [I, P, P, I, I, P]),
    # integer vectors
    "writeMultiVecDeviceInt": (I, [P, P]), "writeMultiVecDeviceIntR2": (I, [P, P, I]),
    "readMultiVecDeviceInt": (I, [P, P]), "readMultiVecDeviceIntR2": (I, [P, P, I]),
    "setscalMultiVecDeviceInt": (I, [I, I, I, I, P]),
    "igathMultiVecDeviceInt": (I, [P, I, I, I, P, I, P, I]),
    "igathMultiVecDeviceIntVecIdx": (I, [P, I, I, I, P, I, P, I]),
    "iscatMultiVecDeviceInt": (I, [P, I, I, I, P, I, P, I, I]),
    "iscatMultiVecDeviceIntVecIdx": (I, [P, I, I, I, P, I, P, I, I]),
    "geinsMultiVecDeviceInt": (I, [I, P, P, I, I, P]),
    # HLL
    "bldHllDeviceParams": (HllDeviceParams, [U, U, U, U, U, U]),
    "psiCopyCooToHlgFloat": (I, [I, I, I, I, I, I, P, P, P, P, P, P]),
    "FallocHllDevice": (I, [PP, U, U, U, U, U, U]), "freeHllDevice": (None, [P]),
    "getHllDeviceParams": (I, [P, PI, PI, PI, PI, PI, PI, PI]),
    "writeHllDeviceDouble": (I, [P, P, P, P, P, P]), "readHllDeviceDouble": (I, [P, P, P, P, P, P]),
    "writeHllDeviceFloat": (I, [P, P, P, P, P, P]), "readHllDeviceFloat": (I, [P, P, P, P, P, P]),
    "psiCopyCooToHlgDouble": (I, [I, I, I, I, I, I, P, P, P, P, P, P]),
    "spmvHllDeviceDouble": (I, [P, D, P, D, P]), "spmvHllDeviceFloat": (I, [P, F, P, F, P]),
    # ELL
    "FallocEllDevice": (I, [PP, U, U, U, U, U, U]), "freeEllDevice": (None, [P]), "zeroEllDevice": (None, [P]),
    "getEllDevicePitch": (I, [P]), "getEllDeviceMaxRowSize": (I, [P]),
    "writeEllDeviceDouble": (I, [P, P, P, I, P, P]), "readEllDeviceDouble": (I, [P, P, P, I, P, P]),
    "psiCopyCooToElgDouble": (I, [I, I, I, I, I, I, P, P, P, P, P]),
    "spmvEllDeviceDouble": (I, [P, D, P, D, P]),
    "getEllDeviceParams": (EllDeviceParams, [U, U, U, U, U, U]),
    "resetEllTimer": (None, []), "getEllTimer": (D, []),
    "writeEllDeviceFloat": (I, [P, P, P, I, P, P]), "readEllDeviceFloat": (I, [P, P, P, I, P, P]),
    "psiCopyCooToElgFloat": (I, [I, I, I, I, I, I, P, P, P, P, P]),
    "spmvEllDeviceFloat": (I, [P, F, P, F, P]),
    "dev_csputEllDeviceDouble": (I, [P, I, P, P, P]), "dev_csputEllDeviceFloat": (I, [P, I, P, P, P]),
    # CSR
    "d_CSRGDeviceAlloc": (I, [PC, I, I, I]), "d_CSRGDeviceFree": (I, [PC]),
    "d_CSRGDeviceGetParms": (I, [PC, PI, PI, PI]), "d_CSRGDeviceSetMatType": (I, [PC, I]),
    "d_CSRGDeviceSetMatFillMode": (I, [PC, I]), "d_CSRGDeviceSetMatDiagType": (I, [PC, I]),
    "d_CSRGDeviceSetMatIndexBase": (I, [PC, I]),
    "d_CSRGHost2Device": (I, [PC, I, I, I, P, P, P]), "d_CSRGDevice2Host": (I, [PC, I, I, I, P, P, P]),
    "d_spmvCSRGDevice": (I, [PC, D, P, D, P]),
    "d_spsvCSRGDevice": (I, [PC, D, P, D, P]), "d_CSRGIsNullSvBuffer": (I, [PC]),
    "FcusparseCreate": (I, []), "FcusparseDestroy": (I, []),
    # additions
    "psbx_DefaultSolverOptions": (I, [C.POINTER(SolverOptions)]),
    "psbx_dkrylov": (I, [CH, P, I, P, P, P, C.POINTER(SolverOptions)]),
    "psbx_diag_prec_build": (I, [P, I, P]),
    "psbx_dmixed_cg": (I, [P, P, P, P, C.POINTER(SolverOptions), D, PI]),
    "psbx_hll_from_csr_device": (I, [PP, I, I, I, P, P, P, I, P]),
    "psbx_hll_autotune_from_csr_device": (I, [PP, I, I, I, P, P, P, P, PI, PI, PD]),
    "psbx_hll_make_single": (I, [P]), "psbx_hll_set_wide": (I, [P, I]), "psbx_hll_set_wide_split": (I, [P, I]),
    "psbx_hll_set_threads_per_row": (I, [P, I]), "psbx_hll_spmv_host": (I, [P, D, P, D, P, I]), "psbx_probe_gather": (I, [P, C.c_longlong, I, P, P, I, PD]), "psbx_hll_get_layout": (I, [P, PI, PI, PI, PI]),
    "psbx_wrapMultiVecDevice": (I, [PP, P, U, U]), "psbx_multivec_data": (P, [P]),
    "psbx_hll_spmv_raw": (I, [P, D, P, D, P]),
    "psbx_dot_noalloc": (I, [P, I, I, P, P, I, P]),
    "psbx_batch_create": (I, [PP, I, I, I]), "psbx_batch_create_prec": (I, [PP, I, I, I, I]),
    "psbx_batch_add": (I, [P, P, P, P, P, D, D, I, PI]),
    "psbx_batch_step": (I, [P, I, PI]),
    "psbx_batch_launch": (I, [P, I]), "psbx_batch_wait": (I, [P, PI]),
    "psbx_batch_poll": (I, [P, I, PI, PI, PI, PD]), "psbx_batch_finished": (I, [P, PI, I, PI]),
    "psbx_batch_remove": (I, [P, I]),
    "psbx_batch_destroy": (I, [P]),
    "psbx_kernel_launches": (C.c_uint64, []), "psbx_last_error": (C.c_char_p, []),
}

for _t, _c in (("Int", C.c_int), ("Float", C.c_float), ("Double", C.c_double)):
    _SIGS.update({
        f"allocate{_t}": (I, [PP, I]), f"allocateMulti{_t}": (I, [PP, I, I]),
        f"write{_t}": (I, [P, P, I]), f"read{_t}": (I, [P, P, I]),
        f"write{_t}First": (I, [I, P, P, I, I]), f"read{_t}First": (I, [I, P, P, I, I]),
        f"writeMulti{_t}": (I, [P, P, I, I]), f"readMulti{_t}": (I, [P, P, I, I]),
        f"free{_t}": (None, [P]), f"registerMapped{_t}": (I, [P, PP, I, _c]),
    })

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args

EXPORTED = tuple(_SIGS)

SPGPU_SUCCESS, SPGPU_UNSUPPORTED, SPGPU_UNSPECIFIED, SPGPU_OUTOFMEMORY = 0, 1, 2, 3
PSBX_TIMEOUT, PSBX_BREAKDOWN, PSBX_NOT_CONVERGED = 4, 5, 6
SPGPU_TYPE_INT, SPGPU_TYPE_FLOAT, SPGPU_TYPE_DOUBLE = 0, 1, 2
PSBX_FMT_HLL, PSBX_FMT_ELL, PSBX_FMT_CSR = 0, 1, 2


class PsbxError(RuntimeError):
    def __init__(self, where, code):
        msg = lib.psbx_last_error().decode(errors="replace")
        super().__init__(f"{where} returned {code} ({msg})")
        self.code = code


def check(rc, where):
    if rc != 0:
        raise PsbxError(where, rc)
    return rc
