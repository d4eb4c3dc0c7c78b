/*
 * oracle.c -- CPU restatement of the PSBLAS 3.9 CPU path (test
 * infrastructure; see oracle.h).  Every function names the reference routine
 * it restates, by file:line within the psblas3 source tree.
 *
 * Compiled with -O2 -fopenmp -ffp-contract=off.  Row-parallel loops keep the
 * per-row summation order of the reference, so their results do not depend
 * on the thread count.  Reductions (dot, nrm2, asum) run left to right when
 * one thread is set; with more threads they sum static per-thread partials in
 * thread order (deterministic for a fixed count), which is only used for
 * timing the CPU baseline.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 1;

void or_set_threads(int nthreads) { g_threads = nthreads > 0 ? nthreads : 1; }
int  or_get_threads(void) { return g_threads; }

/* ------------------------------------------------------------------------ */
/* COO fix: stable sort by (row, col), add duplicates.                       */
/* base/serial/impl/psb_d_coo_impl.F90:4094 (psb_d_fix_coo, dupl = add,     */
/* psb_dupl_def_ = psb_dupl_add_ at base/modules/psb_const_mod.F90:225-228). */
/* Counting sort by column then by row (both stable) gives the (row, col)    */
/* order with ties kept in insertion order, so duplicates add in that order. */
/* ------------------------------------------------------------------------ */
int64_t or_coo_fix(int nr, int64_t nnz, int *ia, int *ja, double *val)
{
  if (nnz <= 0) return 0;
  int nc = 0;
  for (int64_t k = 0; k < nnz; k++) if (ja[k] > nc) nc = ja[k];
  int64_t *cnt = (int64_t *)calloc((size_t)(nc > nr ? nc : nr) + 2, sizeof(int64_t));
  int *ia2 = (int *)malloc(nnz * sizeof(int));
  int *ja2 = (int *)malloc(nnz * sizeof(int));
  double *v2 = (double *)malloc(nnz * sizeof(double));
  /* pass 1: stable by column */
  for (int64_t k = 0; k < nnz; k++) cnt[ja[k]]++;
  int64_t s = 0;
  for (int c = 0; c <= nc; c++) { int64_t t = cnt[c]; cnt[c] = s; s += t; }
  for (int64_t k = 0; k < nnz; k++) {
    int64_t p = cnt[ja[k]]++;
    ia2[p] = ia[k]; ja2[p] = ja[k]; v2[p] = val[k];
  }
  /* pass 2: stable by row */
  memset(cnt, 0, ((size_t)(nc > nr ? nc : nr) + 2) * sizeof(int64_t));
  for (int64_t k = 0; k < nnz; k++) cnt[ia2[k]]++;
  s = 0;
  for (int r = 0; r <= nr; r++) { int64_t t = cnt[r]; cnt[r] = s; s += t; }
  for (int64_t k = 0; k < nnz; k++) {
    int64_t p = cnt[ia2[k]]++;
    ia[p] = ia2[k]; ja[p] = ja2[k]; val[p] = v2[k];
  }
  free(cnt); free(ia2); free(ja2); free(v2);
  /* add duplicates in order */
  int64_t w = 0;
  for (int64_t k = 0; k < nnz; k++) {
    if (w > 0 && ia[w - 1] == ia[k] && ja[w - 1] == ja[k]) {
      val[w - 1] = val[w - 1] + val[k];
    } else {
      ia[w] = ia[k]; ja[w] = ja[k]; val[w] = val[k]; w++;
    }
  }
  return w;
}

/* COO (row-sorted) -> CSR.  base/serial/impl/psb_d_csr_impl.F90:3154
 * (psb_d_cp_csr_from_coo): irp(1)=1, irp(i+1)=irp(i)+rowcount(i). */
void or_csr_from_coo(int nr, int64_t nnz, const int *ia, const int *ja,
                     const double *val, int *irp, int *cja, double *cval)
{
  for (int i = 0; i <= nr; i++) irp[i] = 0;
  for (int64_t k = 0; k < nnz; k++) irp[ia[k]]++;
  irp[0] = 1;
  for (int i = 1; i <= nr; i++) irp[i] += irp[i - 1];
  memcpy(cja, ja, nnz * sizeof(int));
  memcpy(cval, val, nnz * sizeof(double));
}

/* ------------------------------------------------------------------------ */
/* HLL conversion: ext/impl/psi_d_convert_hll_from_coo.f90:31-122 and        */
/* ext/impl/psi_d_xtr_ell_from_coo.f90:31-62.                                */
/*   irn(i)      = number of entries of row i                  (:59-64)     */
/*   hkoffs(1)=0, hkoffs(j+1)=hkoffs(j)+hksz*max(irn in hack j)  (:69-82)   */
/*   last hack pre-filled with val=0, ja=nr                      (:94-96)   */
/*   inside hack: ja(ii,jj) with leading dimension hksz (column major)      */
/*   padding: ja = last column of the row (jac(1) of the hack if the row is */
/*   empty), val = 0                                        (xtr:53-60)     */
/*   idiag(ii) = 1-based position of the diagonal in the row     (xtr:48)   */
/* idiag is left at 0 for rows without a diagonal (the reference leaves it  */
/* undefined there; psi_cuda_CopyCooToHlg.cuh:46 writes 0).                 */
/* ------------------------------------------------------------------------ */
int64_t or_hll_alloc_size(int nr, int64_t nnz, const int *ia, int hksz)
{
  int *irn = (int *)calloc(nr > 0 ? nr : 1, sizeof(int));
  for (int64_t k = 0; k < nnz; k++) irn[ia[k] - 1]++;
  int64_t off = 0;
  for (int i = 0; i < nr; i += hksz) {
    int ir = (hksz < nr - i) ? hksz : nr - i;
    int mx = irn[i];
    for (int k = 1; k < ir; k++) if (irn[i + k] > mx) mx = irn[i + k];
    off += (int64_t)mx * hksz;
  }
  free(irn);
  return off;
}

static void xtr_ell_from_coo(int i0, int nrh, int mxrwl, const int *iac,
                             const int *jac, const double *valc, int *hja,
                             double *hval, const int *irn, int *idiag, int ld)
{
  int64_t kc = 0;
  for (int ii = 0; ii < nrh; ii++) {
    int nc = irn[ii];
    int ic = 0;
    for (int jj = 0; jj < nc; jj++) {
      int ir = iac[kc];
      ic = jac[kc];
      if (ir == ic) idiag[ii] = jj + 1;
      hja[(int64_t)jj * ld + ii] = ic;
      hval[(int64_t)jj * ld + ii] = valc[kc];
      kc++;
    }
    if (nc == 0) ic = jac[0];
    for (int jj = nc; jj < mxrwl; jj++) {
      hja[(int64_t)jj * ld + ii] = ic;
      hval[(int64_t)jj * ld + ii] = 0.0;
    }
  }
  (void)i0;
}

int or_hll_from_coo(int nr, int64_t nnz, const int *ia, const int *ja,
                    const double *val, int hksz, int *irn, int *hkoffs,
                    int *hja, double *hval, int *idiag)
{
  for (int i = 0; i < nr; i++) { irn[i] = 0; idiag[i] = 0; }
  for (int64_t k = 0; k < nnz; k++) irn[ia[k] - 1]++;
  int noffs = (nr + hksz - 1) / hksz;
  hkoffs[0] = 0;
  int j = 0;
  for (int i = 0; i < nr; i += hksz) {
    int ir = (hksz < nr - i) ? hksz : nr - i;
    int mx = irn[i];
    for (int k = 1; k < ir; k++) if (irn[i + k] > mx) mx = irn[i + k];
    hkoffs[j + 1] = hkoffs[j] + mx * hksz;
    j++;
  }
  if (noffs > 0) {
    int64_t isz = hkoffs[noffs];
    int64_t nzm = hkoffs[noffs] - hkoffs[noffs - 1];
    for (int64_t k = isz - nzm; k < isz; k++) { hval[k] = 0.0; hja[k] = nr; }
  }
  int64_t kc = 0, k = 0;
  for (int i = 0; i < nr; i += hksz) {
    int ir = (hksz < nr - i) ? hksz : nr - i;
    int hk = i / hksz;
    int64_t isz = hkoffs[hk + 1] - hkoffs[hk];
    int mxrwl = (int)(isz / hksz);
    int64_t nza = 0;
    for (int t = 0; t < ir; t++) nza += irn[i + t];
    if (isz > 0)
      xtr_ell_from_coo(i, ir, mxrwl, ia + kc, ja + kc, val + kc, hja + k,
                       hval + k, irn + i, idiag + i, hksz);
    k += isz;
    kc += nza;
  }
  return 0;
}

/* ELL conversion: ext/impl/psi_d_convert_ell_from_coo.f90:31-86 (nzm = max
 * row length, ldv rows per column, padding as xtr_ell_from_coo).  Rows
 * nr+1..ldv are filled with val=0, ja=1 (the reference leaves them undefined
 * and never reads them). */
int or_ell_max_row(int nr, int64_t nnz, const int *ia)
{
  int *irn = (int *)calloc(nr > 0 ? nr : 1, sizeof(int));
  for (int64_t k = 0; k < nnz; k++) irn[ia[k] - 1]++;
  int mx = 0;
  for (int i = 0; i < nr; i++) if (irn[i] > mx) mx = irn[i];
  free(irn);
  return mx;
}

int or_ell_from_coo(int nr, int64_t nnz, const int *ia, const int *ja,
                    const double *val, int ldv, int nzm, int *irn, int *eja,
                    double *eval, int *idiag)
{
  if (ldv < nr) return 1;
  for (int i = 0; i < nr; i++) { irn[i] = 0; idiag[i] = 0; }
  for (int64_t k = 0; k < nnz; k++) irn[ia[k] - 1]++;
  for (int64_t c = 0; c < nzm; c++)
    for (int i = nr; i < ldv; i++) { eja[c * ldv + i] = 1; eval[c * ldv + i] = 0.0; }
  if (nnz > 0 && nzm > 0)
    xtr_ell_from_coo(0, nr, nzm, ia, ja, val, eja, eval, irn, idiag, ldv);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* SpMV.  Non-transposed rows follow the inner form of the reference:       */
/*   ext/impl/psb_d_hll_csmv.f90:291-371 (psb_d_hll_csmv_inner),            */
/*   ext/impl/psb_d_ell_csmv.f90:91-200,                                    */
/*   base/serial/impl/psb_d_csr_impl.F90:113-270 (psb_d_csr_csmv_inner):    */
/*   acc = 0; acc = acc + val*x(ja) over the row's stored entries in order; */
/*   alpha == 0: y = beta*y (y = 0 when beta == 0), x not read;             */
/*   beta == 0: y = alpha*acc, y not read; otherwise y = alpha*acc+beta*y.  */
/* The reference's special cases alpha,beta in {+1,-1} give the same bits   */
/* as this generic form for finite data.                                    */
/* Transposed: y = beta*y first, then y(ja) += alpha*val*x(row)             */
/* (psb_d_hll_csmv.f90:70-105; psb_d_csr_impl.F90:271-330).                 */
/* ------------------------------------------------------------------------ */
static inline double finish_row(double alpha, double acc, double beta, double yold)
{
  if (beta == 0.0) return alpha * acc;
  return alpha * acc + beta * yold;
}

static void scale_y(int m, double beta, double *y)
{
  if (beta == 0.0) { for (int i = 0; i < m; i++) y[i] = 0.0; }
  else if (beta != 1.0) { for (int i = 0; i < m; i++) y[i] = beta * y[i]; }
}

int or_csr_csmv(char trans, int nr, int nc, const int *irp, const int *ja,
                const double *val, double alpha, const double *x, double beta,
                double *y)
{
  int tra = (trans == 'T' || trans == 't' || trans == 'C' || trans == 'c');
  int m = tra ? nc : nr;
  if (alpha == 0.0) { scale_y(m, beta, y); return 0; }
  if (!tra) {
#pragma omp parallel for schedule(static) num_threads(g_threads)
    for (int i = 0; i < nr; i++) {
      double acc = 0.0;
      for (int j = irp[i]; j < irp[i + 1]; j++) acc = acc + val[j - 1] * x[ja[j - 1] - 1];
      y[i] = finish_row(alpha, acc, beta, beta == 0.0 ? 0.0 : y[i]);
    }
  } else {
    scale_y(m, beta, y);
    for (int i = 0; i < nr; i++)
      for (int j = irp[i]; j < irp[i + 1]; j++)
        y[ja[j - 1] - 1] = y[ja[j - 1] - 1] + alpha * val[j - 1] * x[i];
  }
  return 0;
}

int or_hll_csmv(char trans, int nr, int nc, int hksz, const int *irn,
                const int *hkoffs, const int *hja, const double *hval,
                double alpha, const double *x, double beta, double *y)
{
  int tra = (trans == 'T' || trans == 't' || trans == 'C' || trans == 'c');
  int nhk = (nr + hksz - 1) / hksz;
  if (!tra) {
    if (alpha == 0.0) { scale_y(nr, beta, y); return 0; }
#pragma omp parallel for schedule(static) num_threads(g_threads)
    for (int h = 0; h < nhk; h++) {
      int i0 = h * hksz;
      int ir = (hksz < nr - i0) ? hksz : nr - i0;
      const int *hj = hja + hkoffs[h];
      const double *hv = hval + hkoffs[h];
      for (int ii = 0; ii < ir; ii++) {
        double acc = 0.0;
        for (int jj = 0; jj < irn[i0 + ii]; jj++)
          acc = acc + hv[(int64_t)jj * hksz + ii] * x[hj[(int64_t)jj * hksz + ii] - 1];
        y[i0 + ii] = finish_row(alpha, acc, beta, beta == 0.0 ? 0.0 : y[i0 + ii]);
      }
    }
  } else {
    scale_y(nc, beta, y);
    for (int h = 0; h < nhk; h++) {
      int i0 = h * hksz;
      int ir = (hksz < nr - i0) ? hksz : nr - i0;
      const int *hj = hja + hkoffs[h];
      const double *hv = hval + hkoffs[h];
      for (int ii = 0; ii < ir; ii++)
        for (int jj = 0; jj < irn[i0 + ii]; jj++) {
          int jc = hj[(int64_t)jj * hksz + ii] - 1;
          y[jc] = y[jc] + alpha * hv[(int64_t)jj * hksz + ii] * x[i0 + ii];
        }
    }
  }
  return 0;
}

/* FP32 HLL / ELL products y = alpha*A*x + beta*y (not transposed).
 * mode 0 restates the library's documented form (include/psbx.h,
 * spmvHllDeviceFloat): each product of two floats is formed exactly in
 * FP64, the products are added in FP64 in stored order, the sum is rounded
 * to FP32 once, then y = alpha*sum + beta*y in FP32 (beta == 0: y not read;
 * alpha == 0: y = beta*y, 0 when beta == 0).
 * mode 1 restates the reference's FP32 CPU product psb_s_hll_csmv
 * (ext/impl/psb_s_hll_csmv.f90, the inner form of psb_d_hll_csmv.f90:345-360
 * with real(psb_spk_)): acc = acc + val*x(ja) in FP32 -- the bar the
 * library's FP32 product is compared with through the FP32 error bound. */
static float f32_finish(float alpha, float acc, float beta, float y)
{
  float t = alpha * acc;
  return beta == 0.0f ? t : t + beta * y;
}

int or_hll_csmv_f32(int mode, int nr, int hksz, const int *irn, const int *hkoffs,
                    const int *hja, const float *hval, float alpha, const float *x,
                    float beta, float *y)
{
  int nhk = (nr + hksz - 1) / hksz;
  if (alpha == 0.0f) {
    for (int i = 0; i < nr; i++) y[i] = beta == 0.0f ? 0.0f : beta * y[i];
    return 0;
  }
#pragma omp parallel for schedule(static) num_threads(g_threads)
  for (int h = 0; h < nhk; h++) {
    int i0 = h * hksz;
    int ir = (hksz < nr - i0) ? hksz : nr - i0;
    const int *hj = hja + hkoffs[h];
    const float *hv = hval + hkoffs[h];
    for (int ii = 0; ii < ir; ii++) {
      float acc;
      if (mode == 0) {
        double a = 0.0;
        for (int jj = 0; jj < irn[i0 + ii]; jj++)
          a = a + (double)hv[(int64_t)jj * hksz + ii] * (double)x[hj[(int64_t)jj * hksz + ii] - 1];
        acc = (float)a;
      } else {
        acc = 0.0f;
        for (int jj = 0; jj < irn[i0 + ii]; jj++)
          acc = acc + hv[(int64_t)jj * hksz + ii] * x[hj[(int64_t)jj * hksz + ii] - 1];
      }
      y[i0 + ii] = f32_finish(alpha, acc, beta, beta == 0.0f ? 0.0f : y[i0 + ii]);
    }
  }
  return 0;
}

int or_ell_csmv_f32(int nr, int ldv, const int *irn, const int *eja, const float *eval,
                    float alpha, const float *x, float beta, float *y)
{
  if (alpha == 0.0f) {
    for (int i = 0; i < nr; i++) y[i] = beta == 0.0f ? 0.0f : beta * y[i];
    return 0;
  }
#pragma omp parallel for schedule(static) num_threads(g_threads)
  for (int i = 0; i < nr; i++) {
    double a = 0.0;
    for (int j = 0; j < irn[i]; j++)
      a = a + (double)eval[(int64_t)j * ldv + i] * (double)x[eja[(int64_t)j * ldv + i] - 1];
    y[i] = f32_finish(alpha, (float)a, beta, beta == 0.0f ? 0.0f : y[i]);
  }
  return 0;
}

/* Triangular solve of psb_d_csr_cssv (base/serial/impl/psb_d_csr_impl.F90:
 * 782-1041), not transposed, beta == 0: inner_csrsv (:890-940) then
 * y = alpha*y (:862-873).  The storage is the CPU type's: a lower triangle
 * keeps its diagonal as the last entry of each row and an upper one as the
 * first, unless unit (no diagonal stored).  1-based irp/ja. */
int or_csr_trsv(int n, const int *irp, const int *ja, const double *val, int lower,
                int unit, double alpha, const double *x, double *y)
{
  if (lower) {
    for (int i = 0; i < n; i++) {
      double acc = 0.0;
      int e = unit ? irp[i + 1] - 1 : irp[i + 1] - 2;
      for (int j = irp[i]; j <= e; j++) acc = acc + val[j - 1] * y[ja[j - 1] - 1];
      y[i] = unit ? x[i] - acc : (x[i] - acc) / val[irp[i + 1] - 2];
    }
  } else {
    for (int i = n - 1; i >= 0; i--) {
      double acc = 0.0;
      int b = unit ? irp[i] : irp[i] + 1;
      for (int j = b; j <= irp[i + 1] - 1; j++) acc = acc + val[j - 1] * y[ja[j - 1] - 1];
      y[i] = unit ? x[i] - acc : (x[i] - acc) / val[irp[i] - 1];
    }
  }
  if (alpha == -1.0) {
    for (int i = 0; i < n; i++) y[i] = -y[i];
  } else if (alpha != 1.0) {
    for (int i = 0; i < n; i++) y[i] = alpha * y[i];
  }
  return 0;
}

int or_ell_csmv(char trans, int nr, int nc, int ldv, int nzm, const int *irn,
                const int *eja, const double *eval, double alpha,
                const double *x, double beta, double *y)
{
  int tra = (trans == 'T' || trans == 't' || trans == 'C' || trans == 'c');
  (void)nzm;
  if (!tra) {
    if (alpha == 0.0) { scale_y(nr, beta, y); return 0; }
#pragma omp parallel for schedule(static) num_threads(g_threads)
    for (int i = 0; i < nr; i++) {
      double acc = 0.0;
      for (int jj = 0; jj < irn[i]; jj++)
        acc = acc + eval[(int64_t)jj * ldv + i] * x[eja[(int64_t)jj * ldv + i] - 1];
      y[i] = finish_row(alpha, acc, beta, beta == 0.0 ? 0.0 : y[i]);
    }
  } else {
    scale_y(nc, beta, y);
    for (int i = 0; i < nr; i++)
      for (int jj = 0; jj < irn[i]; jj++) {
        int jc = eja[(int64_t)jj * ldv + i] - 1;
        y[jc] = y[jc] + alpha * eval[(int64_t)jj * ldv + i] * x[i];
      }
  }
  return 0;
}

/* ext/impl/psb_d_hll_get_diag.f90:89-107: d(i) = val(i, idiag(i)) or 0. */
int or_hll_get_diag(int nr, int hksz, const int *irn, const int *hkoffs,
                    const double *hval, const int *idiag, double *d)
{
  (void)irn;
  for (int i = 0; i < nr; i++) {
    int h = i / hksz, ii = i % hksz;
    d[i] = idiag[i] != 0 ? hval[hkoffs[h] + (int64_t)(idiag[i] - 1) * hksz + ii] : 0.0;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Dense vector kernels.                                                     */
/* Element-wise loops run over threads for long vectors: each entry is      */
/* computed alone, so the results do not depend on the thread count.        */
/* axpby: base/serial/psi_d_serial_impl.F90:593-745 (psi_daxpbyv).  The      */
/* special cases there (alpha, beta in {0, +1, -1}) equal the generic form   */
/* bit for bit for finite data; what they change is which operand is read:   */
/* alpha == 0 never reads x, beta == 0 never reads y.                        */
/* ------------------------------------------------------------------------ */
void or_axpby(int n, double alpha, const double *x, double beta, double *y)
{
  if (alpha == 0.0) {
    if (beta == 0.0) {
#pragma omp parallel for schedule(static) num_threads(g_threads) if (n > 65536)
      for (int i = 0; i < n; i++) y[i] = 0.0;
    } else if (beta != 1.0) {
#pragma omp parallel for schedule(static) num_threads(g_threads) if (n > 65536)
      for (int i = 0; i < n; i++) y[i] = beta * y[i];
    }
    return;
  }
  if (beta == 0.0) {
#pragma omp parallel for schedule(static) num_threads(g_threads) if (n > 65536)
    for (int i = 0; i < n; i++) y[i] = alpha * x[i];
    return;
  }
#pragma omp parallel for schedule(static) num_threads(g_threads) if (n > 65536)
  for (int i = 0; i < n; i++) y[i] = alpha * x[i] + beta * y[i];
}

/* psi_daxpbyv2 (psi_d_serial_impl.F90:746-825): z = alpha*x + beta*y. */
void or_axpbyz(int n, double alpha, const double *x, double beta,
               const double *y, double *z)
{
#pragma omp parallel for schedule(static) num_threads(g_threads) if (n > 65536)
  for (int i = 0; i < n; i++) {
    double a = (alpha == 0.0) ? 0.0 : alpha * x[i];
    z[i] = (beta == 0.0) ? a : (alpha == 0.0 ? beta * y[i] : a + beta * y[i]);
  }
}

/* dot and nrm2: base/modules/serial/psb_d_base_vect_mod.F90:974-996 and
 * :1764-1774 call external BLAS ddot/dnrm2 (third party, version not pinned,
 * so the reference fixes no summation order).  The restatement computes the
 * dot product with the compensated algorithm Dot2 (Ogita, Rump, Oishi,
 * "Accurate sum and dot product", SIAM J. Sci. Comput. 26(6), 2005): every
 * product is split exactly into p + e with an FMA, the running sum is kept
 * as s + c with TwoSum, and the result is s + c, which is as accurate as a
 * sum in twice the working precision and then rounded.  It is at least as
 * accurate as any ordering a BLAS ddot could use, and it makes the result
 * (nearly always) independent of the summation order, which is what lets a
 * parallel device reduction agree with it bit for bit.  nrm2 = sqrt(dot(x,x))
 * as the reference's GPU kernel (cuda/spgpu/kernels/dnrm2.cu) computes it.
 * The FMA here is explicit (fma()), not a contraction. */
typedef struct { double s, c; } dd_t;

static inline dd_t dd_two_sum(double a, double b)
{
  dd_t r;
  r.s = a + b;
  double bb = r.s - a;
  r.c = (a - (r.s - bb)) + (b - bb);
  return r;
}

static inline void dd_add_prod(dd_t *acc, double a, double b)
{
  double p = a * b;
  double e = fma(a, b, -p);
  dd_t t = dd_two_sum(acc->s, p);
  acc->s = t.s;
  acc->c = acc->c + (t.c + e);
}

static inline dd_t dd_merge(dd_t x, dd_t y)
{
  dd_t t = dd_two_sum(x.s, y.s);
  t.c = t.c + (x.c + y.c);
  return t;
}

double or_dot(int n, const double *x, const double *y)
{
  if (g_threads <= 1) {
    dd_t acc = {0.0, 0.0};
    for (int i = 0; i < n; i++) dd_add_prod(&acc, x[i], y[i]);
    return acc.s + acc.c;
  }
  dd_t part[1024];
  int nt = g_threads > 1024 ? 1024 : g_threads;
#pragma omp parallel num_threads(nt)
  {
    int t = 0, T = 1;
#ifdef _OPENMP
    t = omp_get_thread_num(); T = omp_get_num_threads();
#endif
    int64_t lo = (int64_t)n * t / T, hi = (int64_t)n * (t + 1) / T;
    dd_t acc = {0.0, 0.0};
    for (int64_t i = lo; i < hi; i++) dd_add_prod(&acc, x[i], y[i]);
    part[t] = acc;
    if (t == 0) nt = T;
  }
  dd_t acc = {0.0, 0.0};
  for (int t = 0; t < nt; t++) acc = dd_merge(acc, part[t]);
  return acc.s + acc.c;
}

double or_nrm2(int n, const double *x) { return sqrt(or_dot(n, x, x)); }

double or_amax(int n, const double *x)
{
  double m = 0.0;
#pragma omp parallel for schedule(static) num_threads(g_threads) reduction(max : m) if (n > 65536)
  for (int i = 0; i < n; i++) { double a = fabs(x[i]); if (a > m) m = a; }
  return m;
}

double or_asum(int n, const double *x)
{
  double s = 0.0;
  for (int i = 0; i < n; i++) s = s + fabs(x[i]);
  return s;
}

/* mlt: z = alpha*d.*x + beta*z (psb_d_base_vect_mod mlt_a_2; GPU
 * cuda/spgpu/kernels/axy_base.cuh:110-210).  beta == 0 never reads z;
 * alpha == 1 gives d*x exactly. */
void or_mlt(int n, double alpha, const double *d, const double *x,
            double beta, double *z)
{
#pragma omp parallel for schedule(static) num_threads(g_threads) if (n > 65536)
  for (int i = 0; i < n; i++) {
    double t = alpha * (d[i] * x[i]);
    z[i] = (beta == 0.0) ? t : t + beta * z[i];
  }
}

/* psi_d_upd_xyz (psi_d_serial_impl.F90:1571-1794): y = alpha*x + beta*y;
 * z = gamma*y + delta*z. */
void or_upd_xyz(int n, double alpha, double beta, double gamma, double delta,
                const double *x, double *y, double *z)
{
  or_axpby(n, alpha, x, beta, y);
  or_axpby(n, gamma, y, delta, z);
}

/* psi_dxyzw (psi_d_serial_impl.F90:1853-1855): y = a*x+b*y; z = c*y+d*z;
 * w = e*z+f*w (the CPU semantics; the reference GPU kernel dxyzw.cu:47-49
 * computes a different expression, which is not followed). */
void or_xyzw(int n, double a, double b, double c, double d, double e,
             double f, const double *x, double *y, double *z, double *w)
{
#pragma omp parallel for schedule(static) num_threads(g_threads) if (n > 65536)
  for (int i = 0; i < n; i++) {
    y[i] = a * x[i] + b * y[i];
    z[i] = c * y[i] + d * z[i];
    w[i] = e * z[i] + f * w[i];
  }
}

/* prec/impl/psb_d_diagprec_impl.f90:261-267: d = 1/diag, 1 where diag==0. */
void or_diag_prec_build(int n, const double *diag, double *dinv)
{
  for (int i = 0; i < n; i++) dinv[i] = (diag[i] == 0.0) ? 1.0 : 1.0 / diag[i];
}

/* ------------------------------------------------------------------------ */
/* Krylov.  Stopping test: krylov/psb_d_krylov_conv_mod.f90:205-356.         */
/* ------------------------------------------------------------------------ */
typedef struct {
  int istop, itmax;
  double eps, ani, bni, bn2, r0n2, errnum, errden;
} conv_t;

static double csr_normi(int n, const int *irp, const double *val)
{
  double m = 0.0;
  for (int i = 0; i < n; i++) {
    double s = 0.0;
    for (int j = irp[i]; j < irp[i + 1]; j++) s += fabs(val[j - 1]);
    if (s > m) m = s;
  }
  return m;
}

static int init_conv(conv_t *c, int istop, int itmax, double eps, int n,
                     const int *irp, const int *ja, const double *val,
                     const double *b, const double *x)
{
  c->istop = istop; c->itmax = itmax; c->eps = eps;
  c->errnum = 0.0; c->errden = 1.0;
  if (istop == 1) {
    c->ani = csr_normi(n, irp, val);
    c->bni = or_amax(n, b);
  } else if (istop == 2) {
    c->bn2 = or_nrm2(n, b);
  } else if (istop == 3) {
    double *r = (double *)malloc(n * sizeof(double));
    memcpy(r, b, n * sizeof(double));
    or_csr_csmv('N', n, n, irp, ja, val, -1.0, x, 1.0, r);
    c->r0n2 = or_nrm2(n, r);
    free(r);
  } else {
    return 1;
  }
  return 0;
}

static int check_conv(conv_t *c, int it, int n, const double *x, const double *r)
{
  if (c->istop == 1) {
    c->errnum = or_amax(n, r);
    c->errden = c->ani * or_amax(n, x) + c->bni;
  } else if (c->istop == 2) {
    c->errnum = or_nrm2(n, r);
    c->errden = c->bn2;
  } else {
    c->errnum = or_nrm2(n, r);
    c->errden = c->r0n2;
  }
  int res;
  if (c->errden == 0.0) res = (c->errnum <= c->eps);
  else res = (c->errnum <= c->eps * c->errden);
  return res || (c->itmax <= it);
}

static double end_err(const conv_t *c)
{
  /* krylov/psb_base_krylov_conv_mod.f90:96-136 (log_end) */
  return c->errden == 0.0 ? c->errnum : c->errnum / c->errden;
}

static void prec_apply(int n, const double *dinv, const double *x, double *y)
{
  if (dinv) or_mlt(n, 1.0, dinv, x, 0.0, y);
  else memcpy(y, x, n * sizeof(double));
}

/* krylov/psb_dcg.F90:218-295 (psb_dcg_vect), restart loop included. */
int or_cg(int n, const int *irp, const int *ja, const double *val,
          const double *dinv, const double *b, double *x, double eps,
          int itmax, int istop, int *iter, double *err, double *res_hist)
{
  double *p = (double *)calloc(n, sizeof(double));
  double *q = (double *)calloc(n, sizeof(double));
  double *r = (double *)calloc(n, sizeof(double));
  double *z = (double *)calloc(n, sizeof(double));
  conv_t c;
  int itx = 0, rc = 0;
  double alpha = 0.0, rho, rho_old, beta, sigma;
  for (;;) {
    if (itx >= itmax) break;
    int it = 0;
    or_axpby(n, 1.0, b, 0.0, r);
    or_csr_csmv('N', n, n, irp, ja, val, -1.0, x, 1.0, r);
    rho = 0.0;
    if (init_conv(&c, istop, itmax, eps, n, irp, ja, val, b, x)) { rc = 1; goto done; }
    int conv = 0;
    for (;;) {
      it++; itx++;
      prec_apply(n, dinv, r, z);
      rho_old = rho;
      rho = or_dot(n, r, z);
      if (it == 1) {
        or_axpby(n, 1.0, z, 0.0, p);
      } else {
        if (rho_old == 0.0) break;
        beta = rho / rho_old;
        or_axpby(n, 1.0, z, beta, p);
      }
      or_csr_csmv('N', n, n, irp, ja, val, 1.0, p, 0.0, q);
      sigma = or_dot(n, p, q);
      if (sigma == 0.0) break;
      alpha = rho / sigma;
      or_axpby(n, alpha, p, 1.0, x);
      or_axpby(n, -alpha, q, 1.0, r);
      int stop = check_conv(&c, itx, n, x, r);
      if (res_hist && itx <= itmax) res_hist[itx] = end_err(&c);
      if (stop) { conv = 1; break; }
    }
    if (conv) break;
  }
  *iter = itx;
  *err = end_err(&c);
done:
  free(p); free(q); free(r); free(z);
  return rc;
}

/* krylov/psb_dcgstab.f90:226-365 (psb_dcgstab_vect), restart loop included. */
int or_bicgstab(int n, const int *irp, const int *ja, const double *val,
                const double *dinv, const double *b, double *x, double eps,
                int itmax, int istop, int *iter, double *err,
                double *res_hist)
{
  double *q = (double *)calloc(n, sizeof(double));
  double *r = (double *)calloc(n, sizeof(double));
  double *p = (double *)calloc(n, sizeof(double));
  double *v = (double *)calloc(n, sizeof(double));
  double *s = (double *)calloc(n, sizeof(double));
  double *t = (double *)calloc(n, sizeof(double));
  double *z = (double *)calloc(n, sizeof(double));
  double *f = (double *)calloc(n, sizeof(double));
  conv_t c;
  int itx = 0, rc = 0;
  double rho = 0.0, rho_old, alpha = 0.0, omega = 0.0, beta, sigma, tau;
  if (init_conv(&c, istop, itmax, eps, n, irp, ja, val, b, x)) { rc = 1; goto done; }
  for (;;) {
    if (itx >= itmax) break;
    int it = 0;
    or_axpby(n, 1.0, b, 0.0, r);
    or_csr_csmv('N', n, n, irp, ja, val, -1.0, x, 1.0, r);
    or_axpby(n, 1.0, r, 0.0, q);
    if (check_conv(&c, itx, n, x, r)) break;
    if (res_hist) res_hist[itx] = end_err(&c);
    rho = 0.0;
    int conv = 0;
    for (;;) {
      it++; itx++;
      rho_old = rho;
      rho = or_dot(n, q, r);
      if (rho == 0.0) break;
      if (it == 1) {
        or_axpby(n, 1.0, r, 0.0, p);
      } else {
        beta = (rho / rho_old) * (alpha / omega);
        or_axpby(n, -omega, v, 1.0, p);
        or_axpby(n, 1.0, r, beta, p);
      }
      prec_apply(n, dinv, p, f);
      or_csr_csmv('N', n, n, irp, ja, val, 1.0, f, 0.0, v);
      sigma = or_dot(n, q, v);
      if (sigma == 0.0) break;
      alpha = rho / sigma;
      or_axpby(n, 1.0, r, 0.0, s);
      or_axpby(n, -alpha, v, 1.0, s);
      prec_apply(n, dinv, s, z);
      or_csr_csmv('N', n, n, irp, ja, val, 1.0, z, 0.0, t);
      sigma = or_dot(n, t, t);
      if (sigma == 0.0) break;
      tau = or_dot(n, t, s);
      omega = tau / sigma;
      if (omega == 0.0) break;
      or_axpby(n, alpha, f, 1.0, x);
      or_axpby(n, omega, z, 1.0, x);
      or_axpby(n, 1.0, s, 0.0, r);
      or_axpby(n, -omega, t, 1.0, r);
      int stop = check_conv(&c, itx, n, x, r);
      if (res_hist && itx <= itmax) res_hist[itx] = end_err(&c);
      if (stop) { conv = 1; break; }
    }
    if (conv) break;
  }
  *iter = itx;
  *err = end_err(&c);
done:
  free(q); free(r); free(p); free(v); free(s); free(t); free(z); free(f);
  return rc;
}

/* krylov/psb_dfcg.F90 (psb_dfcg_vect): flexible CG, restart loop included.
 * init_conv runs once before the restart loop; each restart recomputes
 * r = b - A x; beta == 0 after a restart ends the solve, delta == 0 inside
 * the iteration goes back to the restart. */
int or_fcg(int n, const int *irp, const int *ja, const double *val,
           const double *dinv, const double *b, double *x, double eps,
           int itmax, int istop, int *iter, double *err, double *res_hist)
{
  double *v = (double *)calloc(n, sizeof(double));
  double *w = (double *)calloc(n, sizeof(double));
  double *d = (double *)calloc(n, sizeof(double));
  double *q = (double *)calloc(n, sizeof(double));
  double *r = (double *)calloc(n, sizeof(double));
  conv_t c;
  int itx = 0, rc = 0;
  double alpha, beta, gamma, delta, theta;
  if (init_conv(&c, istop, itmax, eps, n, irp, ja, val, b, x)) { rc = 1; goto done; }
  for (;;) {
    if (itx >= itmax) break;
    or_axpby(n, 1.0, b, 0.0, r);
    or_csr_csmv('N', n, n, irp, ja, val, -1.0, x, 1.0, r);
    if (check_conv(&c, itx, n, x, r)) break;
    if (res_hist) res_hist[itx] = end_err(&c);
    prec_apply(n, dinv, r, v);
    or_csr_csmv('N', n, n, irp, ja, val, 1.0, v, 0.0, w);
    alpha = or_dot(n, r, v);
    beta = or_dot(n, w, v);
    if (beta == 0.0) break;
    or_axpby(n, 1.0, v, 0.0, d);
    or_axpby(n, 1.0, w, 0.0, q);
    delta = beta;
    theta = alpha / delta;
    or_axpby(n, theta, d, 1.0, x);
    or_axpby(n, -theta, q, 1.0, r);
    int conv = 0;
    for (;;) {
      itx++;
      int stop = check_conv(&c, itx, n, x, r);
      if (res_hist && itx <= itmax) res_hist[itx] = end_err(&c);
      if (stop) { conv = 1; break; }
      prec_apply(n, dinv, r, v);
      or_csr_csmv('N', n, n, irp, ja, val, 1.0, v, 0.0, w);
      alpha = or_dot(n, r, v);
      beta = or_dot(n, w, v);
      gamma = or_dot(n, q, v);
      theta = gamma / delta;
      or_axpby(n, 1.0, v, -theta, d);
      or_axpby(n, 1.0, w, -theta, q);
      delta = beta - (gamma * gamma) / delta;
      if (delta == 0.0) break;
      theta = alpha / delta;
      or_axpby(n, theta, d, 1.0, x);
      or_axpby(n, -theta, q, 1.0, r);
    }
    if (conv) break;
  }
  *iter = itx;
  *err = end_err(&c);
done:
  free(v); free(w); free(d); free(q); free(r);
  return rc;
}

/* Plane rotations and the triangular solve that the reference takes from
 * external BLAS (third party, version not pinned): restated from the
 * classic netlib reference BLAS (drotg of LAPACK <= 3.9, drot, dtrsm
 * 'L','U','N','N' with one right-hand side), with rounded operations. */
void or_drotg(double *a, double *b, double *c, double *s)
{
  const double roe = fabs(*a) > fabs(*b) ? *a : *b;
  const double scale = fabs(*a) + fabs(*b);
  double r, z;
  if (scale == 0.0) {
    *c = 1.0; *s = 0.0; r = 0.0; z = 0.0;
  } else {
    const double ta = *a / scale, tb = *b / scale;
    r = scale * sqrt(ta * ta + tb * tb);
    r = (roe >= 0.0 ? 1.0 : -1.0) * r;
    *c = *a / r;
    *s = *b / r;
    z = 1.0;
    if (fabs(*a) > fabs(*b)) z = *s;
    if (fabs(*b) >= fabs(*a) && *c != 0.0) z = 1.0 / *c;
  }
  *a = r;
  *b = z;
}

static inline void drot1(double *x, double *y, double c, double s)
{
  const double t = c * *x + s * *y;
  *y = c * *y - s * *x;
  *x = t;
}

/* B(1:m) = U(1:m,1:m)^-1 B, U upper triangular column-major, leading dim ld */
static void trsm_upper(int m, const double *u, int ld, double *bv)
{
  for (int k = m - 1; k >= 0; k--) {
    if (bv[k] != 0.0) {
      bv[k] = bv[k] / u[k + (size_t)k * ld];
      for (int i = 0; i < k; i++) bv[i] = bv[i] - bv[k] * u[i + (size_t)k * ld];
    }
  }
}

/* krylov/psb_drgmres.f90 (psb_drgmres_vect): restarted right-preconditioned
 * GMRES(nl), modified Gram-Schmidt, Givens rotations, stop test istop 2
 * (||r||_2 <= eps ||b||_2 with the rotated residual estimate |rs(i+1)|).
 * The cosine is stored through cmplx(tmp, dzero) without a KIND argument
 * (psb_drgmres.f90, after drotg), which makes it default (single)
 * precision: c(i) = (double)(float)tmp here as well.  istop other than 2
 * returns 2 (the reference accepts 1 and 2; its istop 1 branch keeps
 * adding into xt across inner iterations and restarts). */
int or_rgmres(int n, const int *irp, const int *ja, const double *val,
              const double *dinv, const double *b, double *x, double eps,
              int itmax, int istop, int irst, int *iter, double *err,
              double *res_hist)
{
  if (istop != 2) return 2;
  if (irst <= 0) return 1;
  const int nl = irst, ld = irst + 1;
  double *V = (double *)calloc((size_t)(nl + 1) * n + 1, sizeof(double));
  double *w = (double *)calloc(n + 1, sizeof(double));
  double *w1 = (double *)calloc(n + 1, sizeof(double));
  double *h = (double *)calloc((size_t)ld * ld, sizeof(double));
  double *cs = (double *)calloc(ld, sizeof(double));
  double *sn = (double *)calloc(ld, sizeof(double));
  double *rs = (double *)calloc(ld, sizeof(double));
  const double bn2 = or_nrm2(n, b);
  double errnum = 0.0, errden = 1.0;
  int itx = 0;
#define VK(k) (V + (size_t)(k) * n)
#define H(r, c) h[(r) + (size_t)(c) * ld]
  for (;;) {
    double *v1 = VK(0);
    or_axpby(n, 1.0, b, 0.0, v1);
    or_csr_csmv('N', n, n, irp, ja, val, -1.0, x, 1.0, v1);
    rs[0] = or_nrm2(n, v1);
    for (int k = 1; k < ld; k++) rs[k] = 0.0;
    double scal = 1.0 / rs[0];
    errnum = or_nrm2(n, v1);
    errden = bn2;
    if (res_hist && itx <= itmax) res_hist[itx] = errden == 0.0 ? errnum : errnum / errden;
    if (errnum <= eps * errden) break;
    for (int j = 0; j < n; j++) v1[j] = scal * v1[j];
    if (itx >= itmax) break;
    int conv = 0, m = nl;
    for (int i = 1; i <= nl; i++) {
      itx++;
      prec_apply(n, dinv, VK(i - 1), w1);
      or_csr_csmv('N', n, n, irp, ja, val, 1.0, w1, 0.0, w);
      for (int k = 1; k <= i; k++) {
        H(k - 1, i - 1) = or_dot(n, VK(k - 1), w);
        or_axpby(n, -H(k - 1, i - 1), VK(k - 1), 1.0, w);
      }
      H(i, i - 1) = or_nrm2(n, w);
      scal = 1.0 / H(i, i - 1);
      or_axpby(n, scal, w, 0.0, VK(i));
      for (int k = 2; k <= i; k++) drot1(&H(k - 2, i - 1), &H(k - 1, i - 1), cs[k - 2], sn[k - 2]);
      double rti = H(i - 1, i - 1), rti1 = H(i, i - 1), tmp;
      or_drotg(&rti, &rti1, &tmp, &sn[i - 1]);
      cs[i - 1] = (double)(float)tmp;
      drot1(&H(i - 1, i - 1), &H(i, i - 1), cs[i - 1], sn[i - 1]);
      H(i, i - 1) = 0.0;
      drot1(&rs[i - 1], &rs[i], cs[i - 1], sn[i - 1]);
      errnum = fabs(rs[i]);
      errden = bn2;
      if (res_hist && itx <= itmax) res_hist[itx] = errden == 0.0 ? errnum : errnum / errden;
      if (errnum <= eps * errden) { conv = 1; m = i; break; }
    }
    trsm_upper(m, h, ld, rs);
    for (int j = 0; j < n; j++) w1[j] = 0.0;
    for (int k = 1; k <= m; k++) or_axpby(n, rs[k - 1], VK(k - 1), 1.0, w1);
    prec_apply(n, dinv, w1, w);
    or_axpby(n, 1.0, w, 1.0, x);
    if (conv) break;
  }
#undef VK
#undef H
  *iter = itx;
  *err = errden == 0.0 ? errnum : errnum / errden;
  free(V); free(w); free(w1); free(h); free(cs); free(sn); free(rs);
  return 0;
}

/* krylov/psb_dcgs.f90 (psb_dcgs_vect): conjugate gradient squared with the
 * restart loop; init_conv once before it; rho == 0 or sigma == 0 go back to
 * the restart (which recomputes r and rt = r). */
int or_cgs(int n, const int *irp, const int *ja, const double *val,
           const double *dinv, const double *b, double *x, double eps,
           int itmax, int istop, int *iter, double *err, double *res_hist)
{
  double *q = (double *)calloc(n + 1, sizeof(double));
  double *r = (double *)calloc(n + 1, sizeof(double));
  double *rt = (double *)calloc(n + 1, sizeof(double));
  double *p = (double *)calloc(n + 1, sizeof(double));
  double *v = (double *)calloc(n + 1, sizeof(double));
  double *uv = (double *)calloc(n + 1, sizeof(double));
  double *z = (double *)calloc(n + 1, sizeof(double));
  double *f = (double *)calloc(n + 1, sizeof(double));
  double *s = (double *)calloc(n + 1, sizeof(double));
  double *qt = (double *)calloc(n + 1, sizeof(double));
  conv_t c;
  int itx = 0, rc = 0;
  double rho = 0.0, rho_old, alpha, beta, sigma;
  if (init_conv(&c, istop, itmax, eps, n, irp, ja, val, b, x)) { rc = 1; goto done; }
  for (;;) {
    if (itx >= itmax) break;
    int it = 0, conv = 0;
    or_axpby(n, 1.0, b, 0.0, r);
    or_csr_csmv('N', n, n, irp, ja, val, -1.0, x, 1.0, r);
    or_axpby(n, 1.0, r, 0.0, rt);
    if (check_conv(&c, itx, n, x, r)) break;
    if (res_hist) res_hist[itx] = end_err(&c);
    rho = 0.0;
    for (;;) {
      it++;
      itx++;
      rho_old = rho;
      rho = or_dot(n, rt, r);
      if (rho == 0.0) break;
      if (it == 1) {
        or_axpby(n, 1.0, r, 0.0, uv);
        or_axpby(n, 1.0, r, 0.0, p);
      } else {
        beta = rho / rho_old;
        or_axpby(n, 1.0, r, 0.0, uv);
        or_axpby(n, beta, q, 1.0, uv);
        or_axpby(n, 1.0, q, beta, p);
        or_axpby(n, 1.0, uv, beta, p);
      }
      prec_apply(n, dinv, p, f);
      or_csr_csmv('N', n, n, irp, ja, val, 1.0, f, 0.0, v);
      sigma = or_dot(n, rt, v);
      if (sigma == 0.0) break;
      alpha = rho / sigma;
      or_axpby(n, 1.0, uv, 0.0, q);
      or_axpby(n, -alpha, v, 1.0, q);
      or_axpby(n, 1.0, uv, 0.0, s);
      or_axpby(n, 1.0, q, 1.0, s);
      prec_apply(n, dinv, s, z);
      or_axpby(n, alpha, z, 1.0, x);
      or_csr_csmv('N', n, n, irp, ja, val, 1.0, z, 0.0, qt);
      or_axpby(n, -alpha, qt, 1.0, r);
      int stop = check_conv(&c, itx, n, x, r);
      if (res_hist && itx <= itmax) res_hist[itx] = end_err(&c);
      if (stop) { conv = 1; break; }
    }
    if (conv) break;
  }
  *iter = itx;
  *err = end_err(&c);
done:
  free(q); free(r); free(rt); free(p); free(v); free(uv); free(z); free(f); free(s); free(qt);
  return rc;
}

/* krylov/psb_dbicg.f90 (psb_dbicg_vect): biconjugate gradient with the
 * restart loop; the transposed products go through csmv 'T' (the diagonal
 * preconditioner is its own transpose); rho == 0 or sigma == 0 go back to
 * the restart. */
int or_bicg(int n, const int *irp, const int *ja, const double *val,
            const double *dinv, const double *b, double *x, double eps,
            int itmax, int istop, int *iter, double *err, double *res_hist)
{
  double *r = (double *)calloc(n + 1, sizeof(double));
  double *rt = (double *)calloc(n + 1, sizeof(double));
  double *z = (double *)calloc(n + 1, sizeof(double));
  double *zt = (double *)calloc(n + 1, sizeof(double));
  double *p = (double *)calloc(n + 1, sizeof(double));
  double *pt = (double *)calloc(n + 1, sizeof(double));
  double *q = (double *)calloc(n + 1, sizeof(double));
  double *qt = (double *)calloc(n + 1, sizeof(double));
  conv_t c;
  int itx = 0, rc = 0;
  double rho = 0.0, rho_old, alpha, beta, sigma;
  if (init_conv(&c, istop, itmax, eps, n, irp, ja, val, b, x)) { rc = 1; goto done; }
  for (;;) {
    if (itx >= itmax) break;
    int it = 0, conv = 0;
    or_axpby(n, 1.0, b, 0.0, r);
    or_csr_csmv('N', n, n, irp, ja, val, -1.0, x, 1.0, r);
    or_axpby(n, 1.0, r, 0.0, rt);
    rho = 0.0;
    if (check_conv(&c, itx, n, x, r)) break;
    if (res_hist) res_hist[itx] = end_err(&c);
    for (;;) {
      it++;
      itx++;
      prec_apply(n, dinv, r, z);
      prec_apply(n, dinv, rt, zt);
      rho_old = rho;
      rho = or_dot(n, rt, z);
      if (rho == 0.0) break;
      if (it == 1) {
        or_axpby(n, 1.0, z, 0.0, p);
        or_axpby(n, 1.0, zt, 0.0, pt);
      } else {
        beta = rho / rho_old;
        or_axpby(n, 1.0, z, beta, p);
        or_axpby(n, 1.0, zt, beta, pt);
      }
      or_csr_csmv('N', n, n, irp, ja, val, 1.0, p, 0.0, q);
      or_csr_csmv('T', n, n, irp, ja, val, 1.0, pt, 0.0, qt);
      sigma = or_dot(n, pt, q);
      if (sigma == 0.0) break;
      alpha = rho / sigma;
      or_axpby(n, alpha, p, 1.0, x);
      or_axpby(n, -alpha, q, 1.0, r);
      or_axpby(n, -alpha, qt, 1.0, rt);
      int stop = check_conv(&c, itx, n, x, r);
      if (res_hist && itx <= itmax) res_hist[itx] = end_err(&c);
      if (stop) { conv = 1; break; }
    }
    if (conv) break;
  }
  *iter = itx;
  *err = end_err(&c);
done:
  free(r); free(rt); free(z); free(zt); free(p); free(pt); free(q); free(qt);
  return rc;
}

/* krylov/psb_dcgstabl.f90 (psb_dcgstabl_vect): BiCGSTAB(L), nl = irst, left
 * preconditioned (r and the new directions are preconditioned in place), the
 * stop test on the preconditioned residual; breakdowns go back to the
 * restart. */
int or_bicgstabl(int n, const int *irp, const int *ja, const double *val,
                 const double *dinv, const double *b, double *x, double eps,
                 int itmax, int istop, int irst, int *iter, double *err,
                 double *res_hist)
{
  if (irst <= 0) return 1;
  const int nl = irst;
  double *r = (double *)calloc(n + 1, sizeof(double));
  double *rt0 = (double *)calloc(n + 1, sizeof(double));
  double *uh = (double *)calloc((size_t)(nl + 1) * n + 1, sizeof(double));
  double *rh = (double *)calloc((size_t)(nl + 1) * n + 1, sizeof(double));
  double *tmp = (double *)calloc(n + 1, sizeof(double));
  double *gamma = (double *)calloc(nl + 1, sizeof(double));
  double *gamma1 = (double *)calloc(nl + 1, sizeof(double));
  double *gamma2 = (double *)calloc(nl + 1, sizeof(double));
  double *sigma = (double *)calloc(nl + 1, sizeof(double));
  double *taum = (double *)calloc((size_t)(nl + 1) * (nl + 1), sizeof(double));
#define UH(k) (uh + (size_t)(k) * n)
#define RH(k) (rh + (size_t)(k) * n)
#define TAU(i, j) taum[(i) + (size_t)(j) * (nl + 1)]
  conv_t c;
  int itx = 0, rc = 0;
  double rho, rho_old, alpha, beta, omega;
  if (init_conv(&c, istop, itmax, eps, n, irp, ja, val, b, x)) { rc = 1; goto done; }
  for (;;) {
    if (itx >= itmax) break;
    int conv = 0;
    or_axpby(n, 1.0, b, 0.0, r);
    or_csr_csmv('N', n, n, irp, ja, val, -1.0, x, 1.0, r);
    prec_apply(n, dinv, r, tmp);
    memcpy(r, tmp, sizeof(double) * n);
    or_axpby(n, 1.0, r, 0.0, rt0);
    or_axpby(n, 1.0, r, 0.0, RH(0));
    or_axpby(n, 0.0, r, 0.0, UH(0));
    rho = 1.0;
    alpha = 0.0;
    omega = 1.0;
    if (check_conv(&c, itx, n, x, r)) break;
    if (res_hist) res_hist[itx] = end_err(&c);
    for (;;) {
      itx += nl;
      rho = -omega * rho;
      int brk = 0;
      for (int j = 0; j < nl; j++) {
        rho_old = rho;
        rho = or_dot(n, RH(j), rt0);
        if (rho == 0.0) { brk = 1; break; }
        beta = alpha * rho / rho_old;
        rho_old = rho;
        for (int k = 0; k <= j; k++) or_axpby(n, 1.0, RH(k), -beta, UH(k));
        or_csr_csmv('N', n, n, irp, ja, val, 1.0, UH(j), 0.0, UH(j + 1));
        prec_apply(n, dinv, UH(j + 1), tmp);
        memcpy(UH(j + 1), tmp, sizeof(double) * n);
        gamma[j] = or_dot(n, UH(j + 1), rt0);
        if (gamma[j] == 0.0) { brk = 1; break; }
        alpha = rho / gamma[j];
        for (int k = 0; k <= j; k++) or_axpby(n, -alpha, UH(k + 1), 1.0, RH(k));
        or_axpby(n, alpha, UH(0), 1.0, x);
        or_csr_csmv('N', n, n, irp, ja, val, 1.0, RH(j), 0.0, RH(j + 1));
        prec_apply(n, dinv, RH(j + 1), tmp);
        memcpy(RH(j + 1), tmp, sizeof(double) * n);
      }
      if (brk) break;
      for (int j = 1; j <= nl; j++) {
        for (int i = 1; i <= j - 1; i++) {
          TAU(i, j) = or_dot(n, RH(i), RH(j));
          TAU(i, j) = TAU(i, j) / sigma[i];
          or_axpby(n, -TAU(i, j), RH(i), 1.0, RH(j));
        }
        sigma[j] = or_dot(n, RH(j), RH(j));
        gamma1[j] = or_dot(n, RH(0), RH(j));
        gamma1[j] = gamma1[j] / sigma[j];
      }
      gamma[nl] = gamma1[nl];
      omega = gamma[nl];
      for (int j = nl - 1; j >= 1; j--) {
        gamma[j] = gamma1[j];
        for (int i = j + 1; i <= nl; i++) gamma[j] = gamma[j] - TAU(j, i) * gamma[i];
      }
      for (int j = 1; j <= nl - 1; j++) {
        gamma2[j] = gamma[j + 1];
        for (int i = j + 1; i <= nl - 1; i++) gamma2[j] = gamma2[j] + TAU(j, i) * gamma[i + 1];
      }
      or_axpby(n, gamma[1], RH(0), 1.0, x);
      or_axpby(n, -gamma1[nl], RH(nl), 1.0, RH(0));
      or_axpby(n, -gamma[nl], UH(nl), 1.0, UH(0));
      for (int j = 1; j <= nl - 1; j++) {
        or_axpby(n, -gamma[j], UH(j), 1.0, UH(0));
        or_axpby(n, gamma2[j], RH(j), 1.0, x);
        or_axpby(n, -gamma1[j], RH(j), 1.0, RH(0));
      }
      int stop = check_conv(&c, itx, n, x, RH(0));
      if (res_hist && itx <= itmax) res_hist[itx] = end_err(&c);
      if (stop) { conv = 1; break; }
    }
    if (conv) break;
  }
  *iter = itx;
  *err = end_err(&c);
done:
#undef UH
#undef RH
#undef TAU
  free(r); free(rt0); free(uh); free(rh); free(tmp); free(gamma); free(gamma1); free(gamma2); free(sigma);
  free(taum);
  return rc;
}
