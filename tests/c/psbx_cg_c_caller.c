/*
 * A C program using only include/psbx.h: the calls a C or Fortran caller of
 * the reference's GPU glue makes, in the same order -- gpuInit, an HLL-32
 * matrix written from host arrays (FallocHllDevice + writeHllDeviceDouble,
 * the layout of psi_d_convert_hll_from_coo), device vectors
 * (FallocMultiVecDevice + writeMultiVecDeviceDouble), one product
 * (spmvHllDeviceDouble) and the device-resident psb_krylov('CG') with the
 * diagonal preconditioner (psbx_dkrylov).
 *
 * Matrix: the 2-D 5-point Laplacian on an m x m grid (4 on the diagonal,
 * -1 for each neighbour), CSR built row by row, then its HLL-32 form.
 * b = A * ones, so the solution is ones.  Prints one line:
 *   "rows <n> spmv_maxdiff <d> iters <it> err <e> resid <r> maxerr <x>"
 * and returns 0, or prints the failing call and returns 1.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "psbx.h"

#define CHECK(call)                                                   \
  do {                                                                \
    int rc_ = (call);                                                 \
    if (rc_ != 0) {                                                   \
      fprintf(stderr, "%s failed: %d (%s)\n", #call, rc_, psbx_last_error()); \
      return 1;                                                       \
    }                                                                 \
  } while (0)

int main(int argc, char **argv) {
  const int m = argc > 1 ? atoi(argv[1]) : 60;
  const int n = m * m, hk = 32, nh = (n + hk - 1) / hk;
  /* CSR, 1-based, columns in increasing order */
  int *irp = malloc(sizeof(int) * (n + 1)), *ja = malloc(sizeof(int) * 5 * n);
  double *va = malloc(sizeof(double) * 5 * n);
  int nz = 0;
  irp[0] = 1;
  for (int i = 0; i < m; i++)
    for (int j = 0; j < m; j++) {
      const int r = i * m + j;
      if (i > 0) { ja[nz] = r - m + 1; va[nz++] = -1.0; }
      if (j > 0) { ja[nz] = r - 1 + 1; va[nz++] = -1.0; }
      ja[nz] = r + 1; va[nz++] = 4.0;
      if (j < m - 1) { ja[nz] = r + 1 + 1; va[nz++] = -1.0; }
      if (i < m - 1) { ja[nz] = r + m + 1; va[nz++] = -1.0; }
      irp[r + 1] = nz + 1;
    }
  /* HLL-32: hack h holds rows 32h .. 32h+31 column-major (entry k of lane
   * l at hkoffs[h] + 32 k + l), width = its longest row; padding repeats
   * the row's last column with value 0; rows past n take column n */
  int *hkoffs = malloc(sizeof(int) * (nh + 1)), *irn = malloc(sizeof(int) * n), *idiag = malloc(sizeof(int) * n);
  hkoffs[0] = 0;
  for (int h = 0; h < nh; h++) {
    int w = 0;
    for (int l = 0; l < hk && h * hk + l < n; l++) {
      const int r = h * hk + l, len = irp[r + 1] - irp[r];
      if (len > w) w = len;
    }
    hkoffs[h + 1] = hkoffs[h] + hk * w;
  }
  const int alloc = hkoffs[nh];
  int *hja = malloc(sizeof(int) * alloc);
  double *hva = malloc(sizeof(double) * alloc);
  for (int h = 0; h < nh; h++) {
    const int w = (hkoffs[h + 1] - hkoffs[h]) / hk;
    for (int l = 0; l < hk; l++) {
      const int r = h * hk + l;
      for (int k = 0; k < w; k++) {
        const int p = hkoffs[h] + hk * k + l;
        if (r >= n) { hja[p] = n; hva[p] = 0.0; continue; }
        const int len = irp[r + 1] - irp[r], e = irp[r] - 1;
        hja[p] = k < len ? ja[e + k] : ja[e + len - 1];
        hva[p] = k < len ? va[e + k] : 0.0;
      }
      if (r < n) {
        irn[r] = irp[r + 1] - irp[r];
        idiag[r] = 0;
        for (int k = 0; k < irn[r]; k++)
          if (ja[irp[r] - 1 + k] == r + 1) idiag[r] = k + 1;
      }
    }
  }
  CHECK(gpuInit(0));
  void *A = NULL, *X = NULL, *B = NULL, *D = NULL, *Y = NULL;
  CHECK(FallocHllDevice(&A, hk, n, nz, alloc, SPGPU_TYPE_DOUBLE, 1));
  CHECK(writeHllDeviceDouble(A, hva, hja, hkoffs, irn, idiag));
  double *ones = malloc(sizeof(double) * n), *b = malloc(sizeof(double) * n), *dinv = malloc(sizeof(double) * n);
  double *x = malloc(sizeof(double) * n), *y = malloc(sizeof(double) * n);
  for (int r = 0; r < n; r++) {
    ones[r] = 1.0;
    double s = 0.0;
    for (int e = irp[r] - 1; e < irp[r + 1] - 1; e++) s += va[e];
    b[r] = s;            /* A * ones, exact in these small integers */
    dinv[r] = 1.0 / 4.0; /* the inverse diagonal (psb_d_diag_precbld) */
    x[r] = 0.0;
  }
  CHECK(FallocMultiVecDevice(&X, 1, n, SPGPU_TYPE_DOUBLE));
  CHECK(FallocMultiVecDevice(&B, 1, n, SPGPU_TYPE_DOUBLE));
  CHECK(FallocMultiVecDevice(&D, 1, n, SPGPU_TYPE_DOUBLE));
  CHECK(FallocMultiVecDevice(&Y, 1, n, SPGPU_TYPE_DOUBLE));
  /* one product y = A * ones, against b */
  CHECK(writeMultiVecDeviceDouble(X, ones));
  CHECK(spmvHllDeviceDouble(A, 1.0, X, 0.0, Y));
  CHECK(readMultiVecDeviceDouble(Y, y));
  double dmax = 0.0;
  for (int r = 0; r < n; r++) dmax = fmax(dmax, fabs(y[r] - b[r]));
  /* CG with the diagonal preconditioner, from x = 0 */
  CHECK(writeMultiVecDeviceDouble(X, x));
  CHECK(writeMultiVecDeviceDouble(B, b));
  CHECK(writeMultiVecDeviceDouble(D, dinv));
  psbx_SolverOptions opt;
  CHECK(psbx_DefaultSolverOptions(&opt));
  opt.eps = 1e-9;
  opt.itmax = 5000;
  opt.istop = 2;
  CHECK(psbx_dkrylov("CG", A, PSBX_FMT_HLL, D, B, X, &opt));
  CHECK(readMultiVecDeviceDouble(X, x));
  double rn = 0.0, bn = 0.0, xe = 0.0;
  for (int r = 0; r < n; r++) {
    double s = 0.0;
    for (int e = irp[r] - 1; e < irp[r + 1] - 1; e++) s += va[e] * x[ja[e] - 1];
    rn += (b[r] - s) * (b[r] - s);
    bn += b[r] * b[r];
    xe = fmax(xe, fabs(x[r] - 1.0));
  }
  printf("rows %d spmv_maxdiff %.17g iters %d err %.17g resid %.17g maxerr %.17g\n", n, dmax, opt.iter, opt.err,
         sqrt(rn / bn), xe);
  freeMultiVecDevice(X);
  freeMultiVecDevice(B);
  freeMultiVecDevice(D);
  freeMultiVecDevice(Y);
  freeHllDevice(A);
  gpuClose();
  free(irp); free(ja); free(va); free(hkoffs); free(irn); free(idiag); free(hja); free(hva);
  free(ones); free(b); free(dinv); free(x); free(y);
  return 0;
}
