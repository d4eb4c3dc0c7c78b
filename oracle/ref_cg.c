/* ref_cg.c -- TEST AND BASELINE INFRASTRUCTURE, not part of the product.
 *
 * The reference's GPU CG path driven the way its Fortran layer drives it:
 * psb_dcg_vect (krylov/psb_dcg.F90:218-295) with psb_d_vect_cuda vectors and
 * an HLL matrix, i.e. one SPGPU kernel per PSBLAS call through the C glue of
 * cuda/dvectordev.c and cuda/hlldev.c:
 *   psb_geaxpby      -> spgpuDaxpby     (dvectordev.c:229-243)
 *   psb_spmm         -> spgpuDhellspmv  (hlldev.c:185-207)
 *   psb_gedot        -> spgpuDmdot      (dvectordev.c:217-225, host result)
 *   psb_genrm2       -> spgpuDmnrm2     (dvectordev.c:189-195, host result)
 *   DIAG apply       -> spgpuDmaxypbz   (dvectordev.c:296-306)
 * The SPGPU kernels are the reference's own sources, compiled into the same
 * library (oracle/Makefile, target ref).  Stop test istop 2 as
 * psb_d_check_conv_vect (krylov/psb_d_krylov_conv_mod.f90:300-341).  The
 * Fortran dispatch and the host/device dirty-flag bookkeeping of the
 * reference are not replayed, so this is a lower bound of its time.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stddef.h>

#include "core.h"
#include "hell.h"
#include "vector.h"

/* The reference's axpby kernel sizes its grid from the environment layer's
 * device queries (cuda/cuda_util.c:303-344, answered from the device
 * properties that gpuInit caches); the same answers, for the current device. */
static int prop_mp = 0, prop_thr = 0;
static void load_props(void) {
  if (prop_mp) return;
  int dev = 0;
  struct cudaDeviceProp p;
  cudaGetDevice(&dev);
  if (cudaGetDeviceProperties(&p, dev) == cudaSuccess) {
    prop_mp = p.multiProcessorCount;
    prop_thr = p.maxThreadsPerMultiProcessor;
  }
}
int getGPUMultiProcessors(void) { load_props(); return prop_mp; }
int getGPUMaxThreadsPerMP(void) { load_props(); return prop_thr; }

typedef struct {
  spgpuHandle_t h;
  int n, avg;
  const double *cM;
  const int *rP, *hkoffs, *rS;
} refmat;

static void axpby(const refmat *A, double alpha, const double *x, double beta, double *y) {
  spgpuDaxpby(A->h, y, A->n, beta, y, alpha, (double *)x);
}

static void spmm(const refmat *A, double alpha, const double *x, double beta, double *y) {
  spgpuDhellspmv(A->h, y, y, alpha, (double *)A->cM, A->rP, 32, A->hkoffs, A->rS, NULL, A->avg, A->n,
                 (double *)x, beta, 1);
}

static double dot(const refmat *A, const double *x, const double *y) {
  double r = 0.0;
  spgpuDmdot(A->h, &r, A->n, (double *)x, (double *)y, 1, A->n);
  return r;
}

static double nrm2(const refmat *A, const double *x) {
  double r = 0.0;
  spgpuDmnrm2(A->h, &r, A->n, (double *)x, 1, A->n);
  return r;
}

static void prec(const refmat *A, const double *dinv, const double *x, double *y) {
  if (dinv)
    spgpuDmaxypbz(A->h, y, A->n, 0.0, y, 1.0, (double *)dinv, (double *)x, 1, A->n);
  else
    axpby(A, 1.0, x, 0.0, y);
}

/* Returns 0, or 2 on a CUDA error; *iter and *err as psb_krylov's. */
int refg_cg(int n, const double *cM, const int *rP, const int *hkoffs, const int *rS, int avg_nzr,
            const double *dinv, const double *b, double *x, double eps, int itmax, int *iter, double *err) {
  refmat A;
  if (spgpuCreate(&A.h, 0) != SPGPU_SUCCESS) return 2;
  A.n = n;
  A.avg = avg_nzr;
  A.cM = cM;
  A.rP = rP;
  A.hkoffs = hkoffs;
  A.rS = rS;
  double *w = NULL;
  if (cudaMalloc((void **)&w, sizeof(double) * 4 * (size_t)n) != cudaSuccess) {
    spgpuDestroy(A.h);
    return 2;
  }
  cudaMemset(w, 0, sizeof(double) * 4 * (size_t)n);
  double *p = w, *q = w + n, *r = w + 2 * (size_t)n, *z = w + 3 * (size_t)n;
  int itx = 0;
  double rho = 0.0, rho_old, alpha, beta, sigma, errnum = 0.0, errden = 1.0;
  const double bn2 = nrm2(&A, b);
  for (;;) { /* restart */
    if (itx >= itmax) break;
    int it = 0, conv = 0;
    axpby(&A, 1.0, b, 0.0, r);
    spmm(&A, -1.0, x, 1.0, r);
    rho = 0.0;
    for (;;) {
      it++;
      itx++;
      prec(&A, dinv, r, z);
      rho_old = rho;
      rho = dot(&A, r, z);
      if (it == 1) {
        axpby(&A, 1.0, z, 0.0, p);
      } else {
        if (rho_old == 0.0) break;
        beta = rho / rho_old;
        axpby(&A, 1.0, z, beta, p);
      }
      spmm(&A, 1.0, p, 0.0, q);
      sigma = dot(&A, p, q);
      if (sigma == 0.0) break;
      alpha = rho / sigma;
      axpby(&A, alpha, p, 1.0, x);
      axpby(&A, -alpha, q, 1.0, r);
      errnum = nrm2(&A, r);
      errden = bn2;
      int stop = (errden == 0.0) ? (errnum <= eps) : (errnum <= eps * errden);
      if (stop || itmax <= itx) {
        conv = 1;
        break;
      }
    }
    if (conv) break;
  }
  cudaError_t e = cudaDeviceSynchronize();
  cudaFree(w);
  spgpuDestroy(A.h);
  *iter = itx;
  *err = errden == 0.0 ? errnum : errnum / errden;
  return e == cudaSuccess ? 0 : 2;
}
