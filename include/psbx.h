/*
 * psbx.h -- C-ABI of the B200 sparse Krylov library (libpsbx.so).
 *
 * The first part exports, with the same names, argument meaning and return
 * codes, the C glue entry points that PSBLAS 3.9's Fortran GPU types bind to
 * through iso_c_binding (psb_d_cuda_hlg_sparse_mat, psb_d_cuda_elg_sparse_mat,
 * psb_d_cuda_csrg_sparse_mat, psb_d_vect_cuda, psb_cuda_env_mod).  Linking
 * the unmodified Fortran modules against libpsbx.so in place of the
 * reference's libpsb_cuda routes psb_spmm / psb_geaxpby / psb_gedot /
 * psb_genrm2 to the kernels of this library.  Each declaration cites the
 * reference interface it replaces (path within the psblas3 tree).
 *
 * The second part (psbx_*) adds entry points that have no one-to-one
 * counterpart in the reference glue: the device-resident Krylov solver that a
 * psb_krylov shim calls, the mixed-precision solver, the batched solver and
 * device-side format builders.  Each says which reference routine it stands
 * in for.
 *
 * Conventions (as in the reference): matrix and vector handles are opaque
 * void*, owned by the caller and freed with the matching free routine; index
 * arrays passed in are int32 with firstIndex (normally 1, Fortran); host
 * arrays are borrowed for the duration of the call only; every call runs on
 * the library's stream and returns after the host-visible result is ready.
 * Return codes: 0 success, 1 unsupported / size mismatch, 2 unspecified CUDA
 * error, 3 out of device memory, plus the solver codes below.
 * The library is not thread-safe, like the reference's global handle.
 */
#ifndef PSBX_H
#define PSBX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status and element codes: cuda/spgpu/core.h:69-80 ------------------ */
#define SPGPU_SUCCESS        0
#define SPGPU_UNSUPPORTED    1
#define SPGPU_UNSPECIFIED    2
#define SPGPU_OUTOFMEMORY    3
#define PSBX_TIMEOUT         4   /* a bounded device wait ran out           */
#define PSBX_BREAKDOWN       5   /* Krylov breakdown (rho/sigma/omega == 0) */
#define PSBX_NOT_CONVERGED   6   /* itmax reached above tolerance           */

#define SPGPU_TYPE_INT            0
#define SPGPU_TYPE_FLOAT          1
#define SPGPU_TYPE_DOUBLE         2
#define SPGPU_TYPE_COMPLEX_FLOAT  3
#define SPGPU_TYPE_COMPLEX_DOUBLE 4

/* ======================================================================== */
/* Environment: cuda/psb_cuda_env_mod.F90:43-175, cuda/cuda_util.c:220-440   */
/* ======================================================================== */
int   gpuInit(int dev);                       /* cuda_util.c:220 */
void  gpuClose(void);                         /* cuda_util.c:244 */
int   setDevice(int dev);                     /* cuda_util.c:261 */
int   getDevice(void);                        /* cuda_util.c:289 */
int   getDeviceCount(void);                   /* cuda_util.c:366 */
int   getDeviceHasUVA(void);                  /* cuda_util.c:296 */
int   DeviceHasUVA(void);                     /* cuda_util.c:360 */
int   getGPUMultiProcessors(void);            /* cuda_util.c:303 */
int   getGPUMemoryBusWidth(void);             /* cuda_util.c:311 */
int   getGPUMemoryClockRate(void);            /* cuda_util.c:319 */
int   getGPUWarpSize(void);                   /* cuda_util.c:327 */
int   getGPUMaxThreadsPerBlock(void);         /* cuda_util.c:333 */
int   getGPUMaxThreadsPerMP(void);            /* cuda_util.c:339 */
int   getGPUMaxRegistersPerBlock(void);       /* cuda_util.c:345 */
void  cpyGPUNameString(char *cstring);        /* cuda_util.c:352 (>= 256 bytes) */
void  cudaSync(void);                         /* cuda_util.c:377 */
void  cudaReset(void);                        /* cuda_util.c:396 */
void *psb_cudaGetHandle(void);                /* cuda_util.c:414 */
void  psb_cudaCreateHandle(void);             /* cuda_util.c:419 */
void  psb_cudaDestroyHandle(void);            /* cuda_util.c:426 */
void *psb_cudaGetStream(void);                /* cuda_util.c:433 (cudaStream_t) */
void  psb_cudaSetStream(void *stream);        /* cuda_util.c:438 */

/* ======================================================================== */
/* Dense multivectors: cuda/vectordev.h:76-86, cuda/dvectordev.h,            */
/* Fortran side cuda/psb_base_vectordev_mod.F90, psb_d_vectordev_mod.F90     */
/* Layout: count vectors of size elements, pitch = size when count == 1,     */
/* else size rounded up to 256 bytes (vectordev.c:40-70).                    */
/* ======================================================================== */
int  FallocMultiVecDevice(void **deviceMultiVec, unsigned count,
                          unsigned size, unsigned elementType);
void freeMultiVecDevice(void *deviceVec);
int  getMultiVecDeviceSize(void *deviceVec);
int  getMultiVecDeviceCount(void *deviceVec);
int  getMultiVecDevicePitch(void *deviceVec);
int  writeMultiVecDeviceDouble(void *deviceVec, double *hostVec);
int  writeMultiVecDeviceDoubleR2(void *deviceVec, double *hostVec, int ld);
int  readMultiVecDeviceDouble(void *deviceVec, double *hostVec);
int  readMultiVecDeviceDoubleR2(void *deviceVec, double *hostVec, int ld);
int  writeMultiVecDeviceFloat(void *deviceVec, float *hostVec);
int  readMultiVecDeviceFloat(void *deviceVec, float *hostVec);
/* cuda/psb_base_vectordev_mod.F90 (unregisterMapped), vectordev.c:145 */
int  unregisterMapped(void *buf);
/* cuda/psb_d_vectordev_mod.F90:85-160 / cuda_util.c:601-665: plain device
 * buffers (raw pointers) for the gather/scatter buffers of the vector types:
 * allocate n (or m*n) entries; write/read n entries, from the
 * IndexBase-based entry first, or m*n entries; free.  registerMapped pins a
 * host buffer of n entries and returns its device alias (cuda_util.c:104). */
int  allocateDouble(void **d, int n);
int  allocateMultiDouble(void **d, int m, int n);
int  writeDouble(void *d, double *h, int n);
int  readDouble(void *d, double *h, int n);
int  writeDoubleFirst(int first, void *d, double *h, int n, int IndexBase);
int  readDoubleFirst(int first, void *d, double *h, int n, int IndexBase);
int  writeMultiDouble(void *d, double *h, int m, int n);
int  readMultiDouble(void *d, double *h, int m, int n);
void freeDouble(void *d);
int  registerMappedDouble(void *buf, void **d_p, int n, double dummy);
/* the same for the FP32 (psb_s_vectordev_mod.F90) and integer
 * (psb_i_vectordev_mod.F90) vector types */
int  allocateFloat(void **d, int n);
int  allocateMultiFloat(void **d, int m, int n);
int  writeFloat(void *d, float *h, int n);
int  readFloat(void *d, float *h, int n);
int  writeFloatFirst(int first, void *d, float *h, int n, int IndexBase);
int  readFloatFirst(int first, void *d, float *h, int n, int IndexBase);
int  writeMultiFloat(void *d, float *h, int m, int n);
int  readMultiFloat(void *d, float *h, int m, int n);
void freeFloat(void *d);
int  registerMappedFloat(void *buf, void **d_p, int n, float dummy);
int  allocateInt(void **d, int n);
int  allocateMultiInt(void **d, int m, int n);
int  writeInt(void *d, int *h, int n);
int  readInt(void *d, int *h, int n);
int  writeIntFirst(int first, void *d, int *h, int n, int IndexBase);
int  readIntFirst(int first, void *d, int *h, int n, int IndexBase);
int  writeMultiInt(void *d, int *h, int m, int n);
int  readMultiInt(void *d, int *h, int m, int n);
void freeInt(void *d);
int  registerMappedInt(void *buf, void **d_p, int n, int dummy);
/* dvectordev.c:101-112: x(first:last) = val (indexBase-relative) */
int  setscalMultiVecDeviceDouble(double val, int first, int last,
                                 int indexBase, void *devVecX);
/* dvectordev.c:189-198: x = alpha*x over the whole pitch*count */
int  scalMultiVecDeviceDouble(double alpha, void *devVecA);
/* dvectordev.c:200-236: reductions over the first n entries of each of the
 * count vectors; y_res[count] on the host.  Deterministic order on device,
 * no host-side partial sums. */
int  nrm2MultiVecDeviceDouble(double *y_res, int n, void *devVecA);
int  amaxMultiVecDeviceDouble(double *y_res, int n, void *devVecA);
int  asumMultiVecDeviceDouble(double *y_res, int n, void *devVecA);
int  dotMultiVecDeviceDouble(double *y_res, int n, void *devVecA, void *devVecB);
/* dvectordev.c:238-255: y = alpha*x + beta*y (beta == 0: y not read) */
int  axpbyMultiVecDeviceDouble(int n, double alpha, void *devVecX,
                               double beta, void *devVecY);
/* dvectordev.c:257-273: y = alpha*x + beta*y; z = gamma*y + delta*z */
int  upd_xyzMultiVecDeviceDouble(int n, double alpha, double beta,
                                 double gamma, double delta, void *devVecX,
                                 void *devVecY, void *devVecZ);
/* dvectordev.c:275-292 with the CPU semantics of psi_dxyzw
 * (base/serial/psi_d_serial_impl.F90:1853-1855):
 * y = a*x + b*y; z = c*y + d*z; w = e*z + f*w */
int  xyzwMultiVecDeviceDouble(int n, double a, double b, double c, double d,
                              double e, double f, void *devVecX, void *devVecY,
                              void *devVecZ, void *devVecW);
/* dvectordev.c:294-306: b = alpha*a.*b */
int  axyMultiVecDeviceDouble(int n, double alpha, void *devVecA, void *devVecB);
/* dvectordev.c:308-322: z = alpha*a.*b + beta*z (the diagonal prec apply) */
int  axybzMultiVecDeviceDouble(int n, double alpha, void *devVecA,
                               void *devVecB, double beta, void *devVecZ);
/* dvectordev.c:324-345: b = alpha*|a| ; a = alpha*|a| */
int  absMultiVecDeviceDouble2(int n, double alpha, void *devVecA, void *devVecB);
int  absMultiVecDeviceDouble(int n, double alpha, void *devVecA);
/* dvectordev.h:51-61 / dvectordev.c:127-177 (spgpuDgath, spgpuDscat of
 * cuda/spgpu/vector.h:620-653): the halo-exchange halves of the vector type
 * (psb_d_cuda_vect_mod.F90 gthzv / sctb).  Vector vectorId of the
 * multivector; idx holds n indexBase-based positions starting at entry
 * first; buf (device memory) starts at entry hfirst.
 *   gath: buf[i] = v[idx[i]]
 *   scat: v[idx[i]] = beta*v[idx[i]] + buf[i]   (beta == 0: v not read) */
int  igathMultiVecDeviceDouble(void *deviceVec, int vectorId, int n, int first,
                               void *indexes, int hfirst, void *host_values,
                               int indexBase);
int  igathMultiVecDeviceDoubleVecIdx(void *deviceVec, int vectorId, int n,
                                     int first, void *deviceIdx, int hfirst,
                                     void *host_values, int indexBase);
int  iscatMultiVecDeviceDouble(void *deviceVec, int vectorId, int n, int first,
                               void *indexes, int hfirst, void *host_values,
                               int indexBase, double beta);
int  iscatMultiVecDeviceDoubleVecIdx(void *deviceVec, int vectorId, int n,
                                     int first, void *deviceIdx, int hfirst,
                                     void *host_values, int indexBase,
                                     double beta);
/* dvectordev.c:98-125 (psb_d_vectordev_mod.F90:176-178): x(irl(i)) = val(i)
 * (dupl 0, overwrite) or x(irl(i)) += val(i) (dupl 1); irl, val, x device
 * multivectors, irl indexBase-based. */
int  geinsMultiVecDeviceDouble(int n, void *devMultiVecIrl,
                               void *devMultiVecVal, int dupl, int indexBase,
                               void *devMultiVecX);

/* ---- FP32 vectors: cuda/svectordev.h:40-80, psb_s_vectordev_mod.F90.
 * Same layouts and meanings as the FP64 entries.  Element-wise operations
 * round each FP32 multiply and add; dot and nrm2 accumulate the (exact) FP64
 * products with the compensated sum and round to FP32 once; asum sums in
 * FP64 and rounds once (the reference's SPGPU kernels accumulate in FP32). */
int  writeMultiVecDeviceFloatR2(void *deviceVec, float *hostVec, int ld);
int  readMultiVecDeviceFloatR2(void *deviceVec, float *hostVec, int ld);
int  setscalMultiVecDeviceFloat(float val, int first, int last,
                                int indexBase, void *devVecX);
int  scalMultiVecDeviceFloat(float alpha, void *devVecA);
int  nrm2MultiVecDeviceFloat(float *y_res, int n, void *devVecA);
int  amaxMultiVecDeviceFloat(float *y_res, int n, void *devVecA);
int  asumMultiVecDeviceFloat(float *y_res, int n, void *devVecA);
int  dotMultiVecDeviceFloat(float *y_res, int n, void *devVecA, void *devVecB);
int  axpbyMultiVecDeviceFloat(int n, float alpha, void *devVecX, float beta,
                              void *devVecY);
int  upd_xyzMultiVecDeviceFloat(int n, float alpha, float beta, float gamma,
                                float delta, void *devVecX, void *devVecY,
                                void *devVecZ);
int  xyzwMultiVecDeviceFloat(int n, float a, float b, float c, float d,
                             float e, float f, void *devVecX, void *devVecY,
                             void *devVecZ, void *devVecW);
int  axyMultiVecDeviceFloat(int n, float alpha, void *devVecA, void *devVecB);
int  axybzMultiVecDeviceFloat(int n, float alpha, void *devVecA,
                              void *devVecB, float beta, void *devVecZ);
int  absMultiVecDeviceFloat2(int n, float alpha, void *devVecA, void *devVecB);
int  absMultiVecDeviceFloat(int n, float alpha, void *devVecA);
int  igathMultiVecDeviceFloat(void *deviceVec, int vectorId, int n, int first,
                              void *indexes, int hfirst, void *host_values,
                              int indexBase);
int  igathMultiVecDeviceFloatVecIdx(void *deviceVec, int vectorId, int n,
                                    int first, void *deviceIdx, int hfirst,
                                    void *host_values, int indexBase);
int  iscatMultiVecDeviceFloat(void *deviceVec, int vectorId, int n, int first,
                              void *indexes, int hfirst, void *host_values,
                              int indexBase, float beta);
int  iscatMultiVecDeviceFloatVecIdx(void *deviceVec, int vectorId, int n,
                                    int first, void *deviceIdx, int hfirst,
                                    void *host_values, int indexBase,
                                    float beta);
int  geinsMultiVecDeviceFloat(int n, void *devMultiVecIrl,
                              void *devMultiVecVal, int dupl, int indexBase,
                              void *devMultiVecX);

/* ---- integer vectors: cuda/ivectordev.c, psb_i_vectordev_mod.F90 (the
 * index vectors of psb_i_vect_cuda). */
int  writeMultiVecDeviceInt(void *deviceVec, int *hostVec);
int  writeMultiVecDeviceIntR2(void *deviceVec, int *hostVec, int ld);
int  readMultiVecDeviceInt(void *deviceVec, int *hostVec);
int  readMultiVecDeviceIntR2(void *deviceVec, int *hostVec, int ld);
int  setscalMultiVecDeviceInt(int val, int first, int last, int indexBase,
                              void *devVecX);
int  igathMultiVecDeviceInt(void *deviceVec, int vectorId, int n, int first,
                            void *indexes, int hfirst, void *host_values,
                            int indexBase);
int  igathMultiVecDeviceIntVecIdx(void *deviceVec, int vectorId, int n,
                                  int first, void *deviceIdx, int hfirst,
                                  void *host_values, int indexBase);
int  iscatMultiVecDeviceInt(void *deviceVec, int vectorId, int n, int first,
                            void *indexes, int hfirst, void *host_values,
                            int indexBase, int beta);
int  iscatMultiVecDeviceIntVecIdx(void *deviceVec, int vectorId, int n,
                                  int first, void *deviceIdx, int hfirst,
                                  void *host_values, int indexBase, int beta);
int  geinsMultiVecDeviceInt(int n, void *devMultiVecIrl, void *devMultiVecVal,
                            int dupl, int indexBase, void *devMultiVecX);

/* ======================================================================== */
/* HLL (hacked ELLPACK): cuda/hlldev.h:96-153, cuda/hlldev_mod.F90:37-259    */
/* Layout (ext/psb_d_hll_mat_mod.f90:38-104): rows in hacks of hksz; hack k  */
/* stores ja/val column-major with leading dimension hksz starting at        */
/* hkoffs[k]; irn[i] = stored entries of row i; idiag[i] = 1-based position  */
/* of the diagonal in row i (0 if none).                                     */
/* ======================================================================== */
/* cuda/hlldev.h:70-93 */
typedef struct psbx_HllDeviceParams {
  unsigned elementType, hackSize, rows, avgNzr, nzt, allocsize, firstIndex;
} psbx_HllDeviceParams;
/* cuda/hlldev.c:34-49 */
psbx_HllDeviceParams bldHllDeviceParams(unsigned hksize, unsigned rows,
                                        unsigned nzeros, unsigned allocsize,
                                        unsigned elementType,
                                        unsigned firstIndex);
int  FallocHllDevice(void **deviceMat, unsigned hksize, unsigned rows,
                     unsigned nzeros, unsigned allocsize, unsigned elementType,
                     unsigned firstIndex);
void freeHllDevice(void *deviceMat);
int  getHllDeviceParams(void *deviceMat, int *hksize, int *rows, int *nzeros,
                        int *allocsize, int *hackOffsLength, int *firstIndex,
                        int *avgnzr);
int  writeHllDeviceDouble(void *deviceMat, double *val, int *ja, int *hkoffs,
                          int *irn, int *idiag);
int  readHllDeviceDouble(void *deviceMat, double *val, int *ja, int *hkoffs,
                         int *irn, int *idiag);
int  writeHllDeviceFloat(void *deviceMat, float *val, int *ja, int *hkoffs,
                         int *irn, int *idiag);
int  readHllDeviceFloat(void *deviceMat, float *val, int *ja, int *hkoffs,
                        int *irn, int *idiag);
/* cuda/hlldev.c:420-462: row-sorted COO on the host (1-based), hack offsets
 * and row lengths precomputed by the caller (psb_d_cuda_cp_hlg_from_coo.F90:
 * 117-188), scattered into the HLL layout on the device.  Padding follows
 * psi_cuda_CopyCooToHlg.cuh:59-64 (column of the first entry of row 2). */
int  psiCopyCooToHlgDouble(int nr, int nc, int nza, int hacksz, int noffs,
                           int isz, int *irn, int *hoffs, int *idisp, int *ja,
                           double *val, void *deviceMat);
int  psiCopyCooToHlgFloat(int nr, int nc, int nza, int hacksz, int noffs,
                          int isz, int *irn, int *hoffs, int *idisp, int *ja,
                          float *val, void *deviceMat);
/* cuda/hlldev.c:185-207: y = alpha*A*x + beta*y (beta == 0: y not read) */
int  spmvHllDeviceDouble(void *deviceMat, double alpha, void *deviceX,
                         double beta, void *deviceY);
/* cuda/hlldev.c:160-183: the FP32 product.  Each row's products (exact in
 * FP64) are added in FP64 in stored order and rounded to FP32 once; then
 * y = alpha*sum + beta*y in FP32 (the reference's kernel accumulates in
 * FP32). */
int  spmvHllDeviceFloat(void *deviceMat, float alpha, void *deviceX,
                        float beta, void *deviceY);

/* ======================================================================== */
/* ELL: cuda/elldev.h, cuda/elldev_mod.F90:37-313.  Device pitch = rows     */
/* rounded up to 32 (cuda/spgpu/ell.c:33-37); host arrays are pitch x        */
/* maxRowSize column-major (psb_d_cuda_elg_to_gpu.F90:60-90).                */
/* ======================================================================== */
/* cuda/elldev.h:75-97 */
typedef struct psbx_EllDeviceParams {
  unsigned elementType, pitch, rows, columns, maxRowSize, avgRowSize,
      firstIndex;
} psbx_EllDeviceParams;
/* cuda/elldev.c:36-64.  pitch is the one FallocEllDevice allocates (rows
 * rounded up to 32), so psb_d_cuda_elg_to_gpu.F90:65 finds it equal. */
psbx_EllDeviceParams getEllDeviceParams(unsigned rows, unsigned maxRowSize,
                                        unsigned nnzeros, unsigned columns,
                                        unsigned elementType,
                                        unsigned firstIndex);
/* elldev_mod.F90:175-185 (no definition in the reference's C glue, no
 * caller): no ELL timer is kept; getEllTimer returns 0. */
void resetEllTimer(void);
double getEllTimer(void);
int  FallocEllDevice(void **deviceMat, unsigned rows, unsigned maxRowSize,
                     unsigned nnzeros, unsigned columns, unsigned elementType,
                     unsigned firstIndex);
void freeEllDevice(void *deviceMat);
void zeroEllDevice(void *deviceMat);
int  getEllDevicePitch(void *deviceMat);
int  getEllDeviceMaxRowSize(void *deviceMat);
int  writeEllDeviceDouble(void *deviceMat, double *val, int *ja, int ldj,
                          int *irn, int *idiag);
int  readEllDeviceDouble(void *deviceMat, double *val, int *ja, int ldj,
                         int *irn, int *idiag);
/* cuda/elldev.c (psiCopyCooToElgDouble) */
int  psiCopyCooToElgDouble(int nr, int nc, int nza, int hacksz, int ldv,
                           int nzm, int *irn, int *idisp, int *ja, double *val,
                           void *deviceMat);
int  spmvEllDeviceDouble(void *deviceMat, double alpha, void *deviceX,
                         double beta, void *deviceY);
/* FP32 ELL (elldev.c:172-192, 317-330; psiCopyCooToElgFloat); the product
 * sums rows like spmvHllDeviceFloat. */
int  writeEllDeviceFloat(void *deviceMat, float *val, int *ja, int ldj,
                         int *irn, int *idiag);
int  readEllDeviceFloat(void *deviceMat, float *val, int *ja, int ldj,
                        int *irn, int *idiag);
int  psiCopyCooToElgFloat(int nr, int nc, int nza, int hacksz, int ldv,
                          int nzm, int *irn, int *idisp, int *ja, float *val,
                          void *deviceMat);
int  spmvEllDeviceFloat(void *deviceMat, float alpha, void *deviceX,
                        float beta, void *deviceY);
/* elldev.c:607-644 (ell_csput_base.cuh): for i < nnz, the stored entry of
 * row ia[i] (1-based) in column ja[i] takes the value val[i] (a binary
 * search over the row's ascending columns; absent entries are skipped).
 * ia, ja: integer device multivectors; val: a device multivector of the
 * matrix's type. */
int  dev_csputEllDeviceDouble(void *deviceMat, int nnz, void *ia, void *ja,
                              void *val);
int  dev_csputEllDeviceFloat(void *deviceMat, int nnz, void *ia, void *ja,
                             void *val);

/* ======================================================================== */
/* CSR (replaces the cuSPARSE-backed CSRG of cuda/d_cusparse_mod.F90:36-190; */
/* the matrix handle is the interoperable struct d_Cmat {void *mat;}).       */
/* ======================================================================== */
typedef struct psbx_d_Cmat { void *mat; } psbx_d_Cmat;
int d_CSRGDeviceAlloc(psbx_d_Cmat *Mat, int nr, int nc, int nz);
int d_CSRGDeviceFree(psbx_d_Cmat *Mat);
int d_CSRGDeviceGetParms(psbx_d_Cmat *Mat, int *nr, int *nc, int *nz);
int d_CSRGDeviceSetMatType(psbx_d_Cmat *Mat, int type);
int d_CSRGDeviceSetMatFillMode(psbx_d_Cmat *Mat, int type);
int d_CSRGDeviceSetMatDiagType(psbx_d_Cmat *Mat, int type);
int d_CSRGDeviceSetMatIndexBase(psbx_d_Cmat *Mat, int type); /* 0 or 1 */
int d_CSRGHost2Device(psbx_d_Cmat *Mat, int m, int n, int nz, int *irp,
                      int *ja, double *val);
int d_CSRGDevice2Host(psbx_d_Cmat *Mat, int m, int n, int nz, int *irp,
                      int *ja, double *val);
/* y = alpha*A*x + beta*y with x, y MultiVectDevice handles */
int d_spmvCSRGDevice(psbx_d_Cmat *Mat, double alpha, void *deviceX,
                     double beta, void *deviceY);
/* fcusparse_fct.h:132-220 (cusparseSpSV): y = alpha * T^{-1} x, T the
 * triangle selected by d_CSRGDeviceSetMatFillMode (0 lower, 1 upper), with a
 * unit diagonal when d_CSRGDeviceSetMatDiagType set 1 (the stored diagonal
 * is then ignored); entries outside the triangle are ignored, a row without
 * a stored diagonal (non-unit) is divided by 1.  Rows are solved in order
 * with the sums of base/serial/impl/psb_d_csr_impl.F90:890-940, alpha
 * applied after (:862-873).  beta is not used (as in cusparseSpSV).  Returns
 * PSBX_TIMEOUT if a row's wait for its dependencies ran past its bound. */
int d_spsvCSRGDevice(psbx_d_Cmat *Mat, double alpha, void *deviceX,
                     double beta, void *deviceY);
/* fcusparse_fct.h:465-471: 1 until the first d_spsvCSRGDevice call. */
int d_CSRGIsNullSvBuffer(psbx_d_Cmat *Mat);
/* base_cusparse_mod.F90:83-96 (fcusparse.c:44-70): no cuSPARSE handle is
 * needed; Create initialises the library context, both return 0. */
int FcusparseCreate(void);
int FcusparseDestroy(void);

/* ======================================================================== */
/* Additions (no one-to-one counterpart in the reference glue)               */
/* ======================================================================== */

/* Solver options: mirrors psb_c_SolverOptions
 * (cbind/krylov/psb_krylov_cbind.h:17-27) field for field. */
typedef struct psbx_SolverOptions {
  int    iter;    /* out: iterations performed                       */
  int    itmax;   /* in:  maximum iterations (reference default 1000) */
  int    itrace;  /* in:  unused (no host printing on the device path) */
  int    irst;    /* in:  unused by CG / BiCGSTAB                     */
  int    istop;   /* in:  1 backward error, 2 ||r||/||b||, 3 ||r||/||r0|| */
  double eps;     /* in:  stopping tolerance                          */
  double err;     /* out: final error estimate                        */
} psbx_SolverOptions;

int psbx_DefaultSolverOptions(psbx_SolverOptions *opt);

/* Matrix formats accepted by the solver entry points. */
#define PSBX_FMT_HLL 0
#define PSBX_FMT_ELL 1
#define PSBX_FMT_CSR 2

/* Device-resident psb_krylov('CG'|'FCG'|'CGS'|'BICG'|'BICGSTAB'|
 * 'BICGSTABL'|'RGMRES') (krylov/psb_dkrylov.f90:179-210 dispatch,
 * psb_dcg.F90:218-295, psb_dfcg.F90, psb_dcgs.f90, psb_dbicg.f90 -- its A^T
 * products on a transposed copy built at the start of the solve --,
 * psb_dcgstab.f90:226-365, psb_dcgstabl.f90 with L = opt->irst,
 * psb_drgmres.f90) with the diagonal
 * preconditioner (prec/impl/psb_d_diagprec_impl.f90:116).  RGMRES (also
 * 'GMRES') restarts every opt->irst steps and takes istop 2 only (the
 * reference also accepts 1); other method names return 1.
 *   mat   HLL / ELL handle, or a psbx_d_Cmat* for CSR (fmt selects)
 *   dinv  MultiVectDevice with the inverse diagonal, or NULL for no prec
 *   b, x  MultiVectDevice (x holds x0 on entry, the solution on exit)
 * Scalars stay on the device; the stop test runs every iteration on the
 * device; the host reads a status word once per captured batch of
 * iterations.  Returns 0 (converged or itmax reached, as the reference),
 * or an error code; opt->iter and opt->err are filled like psb_krylov's
 * iter and err. */
int psbx_dkrylov(const char *method, void *mat, int fmt, void *dinv,
                 void *b, void *x, psbx_SolverOptions *opt);

/* Mixed-precision psb_krylov('CG') for one system (krylov/psb_dcg.F90:218-295
 * with the DIAG preconditioner; no single reference entry): the iterations
 * run in FP32 -- the matrix's FP32 value copy (made here if absent), FP32
 * vectors, dot products accumulated in FP64 -- and the residual
 * r = b - A x, the solution x and the stop test ||r|| <= eps ||b|| (istop 2
 * only) in FP64.  The FP32 recursive residual is replaced by the FP64 true
 * residual whenever it has fallen by the factor delta (0 < delta < 1, e.g.
 * 0.1) since the last replacement, keeping the search direction.
 *   mat   FP64 HLL handle, hack size 32;  dinv  FP64 inverse diagonal or NULL
 *   b, x  FP64 MultiVectDevice (x = x0 on entry, the solution on exit)
 * opt->iter = inner iterations, opt->err = ||b - A x|| / ||b|| (FP64, true
 * residual); *refreshes (nullable) = residual replacements.  Returns 0
 * (converged or itmax) or an error code. */
int psbx_dmixed_cg(void *mat, void *dinv, void *b, void *x,
                   psbx_SolverOptions *opt, double delta, int *refreshes);

/* psb_d_diag_precbld (prec/impl/psb_d_diagprec_impl.f90:229-292) on the
 * device: dinv(i) = 1/a_ii, 1 where a_ii == 0 (HLL uses idiag). */
int psbx_diag_prec_build(void *mat, int fmt, void *dinv);

/* Device-side CSR -> HLL build (the conversion of
 * ext/impl/psi_d_convert_hll_from_coo.f90:31-122 with the padding of
 * psi_d_xtr_ell_from_coo.f90:53-60) from a CSR matrix already on the device
 * (irp/ja 1-based int32, val FP64).  *deviceMat receives a new HLL handle.
 * perm (device int32[rows] or NULL): when given, hack rows are taken in the
 * order perm[0..rows-1] (0-based row ids) and the SpMV scatters y through
 * it; this is the row-sorted HLL variant for skewed row lengths. */
int psbx_hll_from_csr_device(void **deviceMat, int rows, int cols, int nnz,
                             const int *d_irp, const int *d_ja,
                             const double *d_val, int hksz, const int *d_perm);

/* Autotuned device CSR -> HLL (the "autotuned hack size and threads per
 * row" of the GPU HLL SpMV; the reference fixes hksz = 32,
 * psb_d_cuda_cp_hlg_from_coo.F90:60): builds each candidate layout -- hack
 * size 32, 64 or 128 and, for hack size 32, the width above which a hack
 * takes the wide path (32, 64, 128, 256, 1024 or never) and the threads per
 * row of the other hacks (two rows per thread, one, or two threads per row)
 * -- times its SpMV on the library stream and keeps the fastest.  The handle
 * comes back in the tolerance mode; after psbx_hll_set_wide_split(m, 0)
 * every layout gives the CPU csmv's bits.  *hksz, *wide_w (-1 never, 0 not
 * applicable) and *ms (one SpMV) describe the choice, psbx_hll_get_layout
 * the row mapping.  Arguments otherwise as psbx_hll_from_csr_device. */
int psbx_hll_autotune_from_csr_device(void **deviceMat, int rows, int cols,
                                      int nnz, const int *d_irp,
                                      const int *d_ja, const double *d_val,
                                      const int *d_perm, int *hksz,
                                      int *wide_w, double *ms);

/* Sets the wide-hack threshold of a hack-32 HLL matrix built by this
 * library (0: default -- 64 or four times the mean hack width, whichever is
 * larger; < 0: never) and rebuilds its wide-hack lists.  In the exact mode
 * every threshold gives the same bits; only the time changes.  Returns SPGPU_UNSUPPORTED for
 * another hack size unless wide_w is 0. */
int psbx_hll_set_wide(void *deviceMat, int wide_w);

/* Tolerance or exact mode of an HLL handle.  1 (the default), tolerance:
 * each 64-column chunk of a wide hack (hack size 32) is summed by a block
 * (its 8 warps taking interleaved columns) and the chunks' row partials are
 * added in column order, in the same launch as the other rows -- no product
 * buffer, no long serial chain -- and the standalone SpMV may take two
 * threads per row (psbx_hll_set_threads_per_row); every row is then within
 * |dy_i| <= len_i u sum_j |a_ij x_j| of the stored-order sum.  0, exact:
 * every row in stored order (wide hacks: products by all blocks, then a warp
 * per hack adds them in order), the CPU csmv's bits.  Every solver and
 * product on the handle follows it.  The reference's own GPU HLL kernels
 * (fused multiply-add, two-thread rows) are a tolerance mode too. */
int psbx_hll_set_wide_split(void *deviceMat, int split);

/* y = alpha*A*x + beta*y with x and y in HOST memory (page-locked for the
 * copies to overlap; pageable works, serialised): the composition of
 * writeMultiVecDeviceDouble (x, and y when beta != 0), spmvHllDeviceDouble
 * and readMultiVecDeviceDouble (hlldev.c:185-207, dvectordev.c) in one
 * call, with the copies overlapped with the product: the rows are cut into
 * `chunks` blocks of whole hacks (0: 8; 1: no overlap), x goes up block by
 * block, each row block starts once the part of x holding its largest
 * column is on the device, and its part of y goes down as soon as it is
 * done -- or, when beta is 0 and y is page-locked, each row block stores
 * its part of y straight into it (no copy down), so the two directions of
 * the link carry x and y at the same time.  The same bits as the three
 * calls.  Overlap needs hack size 32, no wide hacks and no row permutation;
 * other handles take the three steps one after the other.  Device staging
 * vectors are kept in the handle.  x may be the same array as y.  Returns
 * once y is on the host. */
int psbx_hll_spmv_host(void *deviceMat, double alpha, const double *x, double beta, double *y, int chunks);

/* Row mapping of the standalone SpMV on a hack-32 HLL handle: 0 auto (two
 * rows per thread when there are wide hacks, one otherwise), 1 one thread
 * per row, 2 two threads per row (entries of even and odd position summed
 * apart and then added -- the reference's two-thread HLL mode,
 * hell_spmv_base_template.cuh:63; tolerance mode only, the exact mode takes
 * -2 instead), -2 two adjacent rows per thread (double2/int2 loads, stored
 * order).  Other hack sizes accept 0 and 1.  The solvers' fused kernels keep
 * their own mapping.  psbx_hll_autotune_from_csr_device picks it. */
int psbx_hll_set_threads_per_row(void *deviceMat, int tpr);

/* The layout of an HLL handle: hack size, wide threshold as set (0
 * default), tolerance (1) or exact (0) mode, row mapping. */
int psbx_hll_get_layout(void *deviceMat, int *hksz, int *wide_w, int *split, int *tpr);

/* Adds an FP32 copy of the values of an FP64 HLL handle (for the FP32 inner
 * iterations of the mixed-precision solver). */
int psbx_hll_make_single(void *deviceMat);

/* Wraps caller-owned device memory (double, n entries) as a one-vector
 * MultiVectDevice without allocating; freeMultiVecDevice on it releases the
 * descriptor only. */
int psbx_wrapMultiVecDevice(void **deviceVec, void *devPtr, unsigned size,
                            unsigned elementType);
void *psbx_multivec_data(void *deviceVec);

/* Runs y = alpha*A*x + beta*y for an HLL handle on raw device pointers
 * (x, y: double, y may not alias x) on the library stream, asynchronously. */
int psbx_hll_spmv_raw(void *deviceMat, double alpha, const double *x,
                      double beta, double *y);
/* Batched mixed-precision CG engine (stands in for many psb_krylov('CG')
 * calls of krylov/psb_dcg.F90 with the DIAG preconditioner; no single
 * reference entry).  Each system is an FP64 HLL handle with hack size 32 and
 * 1-based indices (an FP32 copy of its values is made if absent) and nrhs
 * (1 or 8) right-hand sides interleaved as v[row*nrhs + k].  Per rhs: outer
 * FP64 refinement r = b - A x, stop at ||r|| <= eps ||b||, inner Jacobi-CG
 * in FP32 (FP64-accumulated dots) to a relative reduction inner_tol, then
 * x += ||r|| d; the next inner loop keeps the search direction (residual
 * replacement; restarted only after a breakdown or when the true residual
 * has drifted from the recursive one).  inner_tol 1e-2 suits it: with 1e-4
 * the FP32 recursion can lose accuracy before it gets there, and the
 * safeguards then spend iterations.  All systems advance together in one persistent grid whose
 * iterations are captured in a CUDA graph; each system has its own
 * convergence state and leaves the work when done; systems can be added
 * and removed between steps.  A system's results do not depend on which
 * other systems share the engine.
 *   create : max_systems slots, max_rows_total rows over all slots
 *   add    : d_b, d_x device arrays (rows*nrhs doubles, x = x0 on entry and
 *            the solution on exit, owned by the caller; 16-byte aligned
 *            when nrhs is 8), d_dinv the FP64 inverse diagonal or NULL;
 *            *slot receives the slot id
 *   step   : replays the captured iterations `replays` times (8 iterations
 *            each), then reports how many slots are still running
 *   poll   : state 0 running / 1 converged / 2 stopped (itmax, breakdown);
 *            outer steps, inner iterations and ||b-Ax||/||b|| per rhs */
int psbx_batch_create(void **eng, int max_systems, int max_rows_total, int nrhs);
/* The same engine with the inner iterations in FP32 (inner_bits 32, as
 * psbx_batch_create) or in FP64 (64: FP64 values and vectors throughout --
 * the batched FP64 solve, to tell the gain of batching from that of the
 * FP32 inner iterations). */
int psbx_batch_create_prec(void **eng, int max_systems, int max_rows_total, int nrhs, int inner_bits);
int psbx_batch_add(void *eng, void *hllMat, const double *d_b, double *d_x, const double *d_dinv, double eps,
                   double inner_tol, int itmax, int *slot);
int psbx_batch_step(void *eng, int replays, int *n_running);
/* psbx_batch_step in two halves: launch enqueues the replays and the state
 * read-back and returns at once (1 if a launch is already in flight); wait
 * blocks until it is done.  Between them the host may read finished slots'
 * solutions (their phase is done, so the running replays do not touch
 * them), add requests and remove slots; adds and removes take effect at the
 * next launch.  poll reports the state as of the last wait. */
int psbx_batch_launch(void *eng, int replays);
int psbx_batch_wait(void *eng, int *n_running);
int psbx_batch_poll(void *eng, int slot, int *state, int *outer, int *iters, double *err);
/* The slots whose solve has ended as of the last wait (phase done, not yet
 * removed), in slot order: the first `max` go to slots[], *count receives
 * how many there are (call again with a larger array if it exceeds max).
 * One call instead of a poll per running slot. */
int psbx_batch_finished(void *eng, int *slots, int max, int *count);
int psbx_batch_remove(void *eng, int slot);
int psbx_batch_destroy(void *eng);

/* Allocation-free dot products.  No counterpart in the reference: it is a
 * variant of dotMultiVecDeviceDouble for callers that cannot let a library
 * call cudaMalloc -- code that owns all device memory through its own pool or
 * a fixed budget, and latency-critical loops where an allocation would
 * synchronise the device.  It allocates nothing: its scratch is a fixed
 * file-scope device array (512 KiB of partial sums plus 8 counters, held on
 * every GPU that loads the library until the process exits).
 *   d_res   device pointer to count doubles: d_res[k] = sum_i x_k[i]*y_k[i]
 *   n       entries per vector; count 1..8 vectors (more is rejected with
 *           SPGPU_UNSUPPORTED and a message), pitch = entries between the
 *           vectors of x and of y (ignored when count == 1)
 *   x, y    device pointers; stream: cudaStream_t (NULL: default stream)
 * The call is asynchronous on the stream and allocates nothing.  The first
 * call on each device looks up the scratch's device address and zeroes its
 * counters (a synchronous cudaMemset), so make that first call before any
 * stream capture.  Each later call leaves the counters at zero when its
 * kernel ends.  gpuClose, cudaReset and psb_cudaDestroyHandle drop the
 * looked-up addresses; a caller that resets the device itself
 * (cudaDeviceReset) calls gpuClose before the next call here.  All calls
 * share the one scratch array: calls whose kernels overlap on the GPU
 * (different streams, or different host threads) race and give wrong
 * results; order them.  Results are bit for bit those of
 * dotMultiVecDeviceDouble on the same vectors (same kernel, same grid, same
 * compensated sum). */
int psbx_dot_noalloc(double *d_res, int n, int count, const double *x, const double *y, int pitch,
                     void *stream);

/* Number of kernels launched by the library since load (for accounting). */
uint64_t psbx_kernel_launches(void);
/* Last CUDA error string seen by the library (static storage). */
const char *psbx_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* PSBX_H */
