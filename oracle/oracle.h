/*
 * oracle.h -- CPU restatement of the PSBLAS 3.9 CPU path that the B200
 * library replaces.  TEST INFRASTRUCTURE ONLY: only tests/, the smoke check
 * and the CPU-baseline leg of bench.py may load this library.  It is the
 * checker, never the thing measured as the product and never shipped as a
 * fallback.
 *
 * Conventions follow the reference Fortran: all index arrays are 1-based,
 * matrices are held row-sorted (COO sorted by row then column, duplicates
 * added), values are FP64, indices int32 (psb_ipk_ = 4 bytes, the setting the
 * reference's CUDA build requires).  Floating-point contraction is disabled
 * when this file is compiled (-ffp-contract=off), so every a*b+c below is a
 * rounded multiply followed by a rounded add, as in the reference's loops on
 * x86-64 without FMA.
 */
#ifndef PSBX_ORACLE_H
#define PSBX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

void    or_set_threads(int nthreads);
int     or_get_threads(void);

/* ---- assembly / conversion ---------------------------------------------- */
int64_t or_coo_fix(int nr, int64_t nnz, int *ia, int *ja, double *val);
void    or_csr_from_coo(int nr, int64_t nnz, const int *ia, const int *ja,
                        const double *val, int *irp, int *cja, double *cval);
int64_t or_hll_alloc_size(int nr, int64_t nnz, const int *ia, int hksz);
int     or_hll_from_coo(int nr, int64_t nnz, const int *ia, const int *ja,
                        const double *val, int hksz, int *irn, int *hkoffs,
                        int *hja, double *hval, int *idiag);
int     or_ell_max_row(int nr, int64_t nnz, const int *ia);
int     or_ell_from_coo(int nr, int64_t nnz, const int *ia, const int *ja,
                        const double *val, int ldv, int nzm, int *irn,
                        int *eja, double *eval, int *idiag);

/* ---- sparse matrix-vector products: y = alpha*op(A)*x + beta*y --------- */
int or_csr_csmv(char trans, int nr, int nc, const int *irp, const int *ja,
                const double *val, double alpha, const double *x, double beta,
                double *y);
int or_hll_csmv(char trans, int nr, int nc, int hksz, const int *irn,
                const int *hkoffs, const int *hja, const double *hval,
                double alpha, const double *x, double beta, double *y);
int or_ell_csmv(char trans, int nr, int nc, int ldv, int nzm, const int *irn,
                const int *eja, const double *eval, double alpha,
                const double *x, double beta, double *y);
int or_hll_csmv_f32(int mode, int nr, int hksz, const int *irn, const int *hkoffs,
                    const int *hja, const float *hval, float alpha, const float *x,
                    float beta, float *y);
int or_ell_csmv_f32(int nr, int ldv, const int *irn, const int *eja, const float *eval,
                    float alpha, const float *x, float beta, float *y);
int or_csr_trsv(int n, const int *irp, const int *ja, const double *val, int lower,
                int unit, double alpha, const double *x, double *y);
int or_hll_get_diag(int nr, int hksz, const int *irn, const int *hkoffs,
                    const double *hval, const int *idiag, double *d);

/* ---- dense vector kernels ------------------------------------------------ */
void   or_axpby(int n, double alpha, const double *x, double beta, double *y);
void   or_axpbyz(int n, double alpha, const double *x, double beta,
                 const double *y, double *z);
double or_dot(int n, const double *x, const double *y);
double or_nrm2(int n, const double *x);
double or_amax(int n, const double *x);
double or_asum(int n, const double *x);
void   or_mlt(int n, double alpha, const double *d, const double *x,
              double beta, double *z);
void   or_upd_xyz(int n, double alpha, double beta, double gamma, double delta,
                  const double *x, double *y, double *z);
void   or_xyzw(int n, double a, double b, double c, double d, double e,
               double f, const double *x, double *y, double *z, double *w);
void   or_diag_prec_build(int n, const double *diag, double *dinv);

/* ---- Krylov solvers (CSR operator, diagonal preconditioner) ------------- */
/* dinv == NULL means no preconditioner.  Returns 0, fills iter/err.
 * res_hist (optional, length itmax+1) receives errnum/errden per check. */
int or_cg(int n, const int *irp, const int *ja, const double *val,
          const double *dinv, const double *b, double *x, double eps,
          int itmax, int istop, int *iter, double *err, double *res_hist);
int or_bicgstab(int n, const int *irp, const int *ja, const double *val,
                const double *dinv, const double *b, double *x, double eps,
                int itmax, int istop, int *iter, double *err,
                double *res_hist);
int or_fcg(int n, const int *irp, const int *ja, const double *val,
           const double *dinv, const double *b, double *x, double eps,
           int itmax, int istop, int *iter, double *err, double *res_hist);
int or_rgmres(int n, const int *irp, const int *ja, const double *val,
              const double *dinv, const double *b, double *x, double eps,
              int itmax, int istop, int irst, int *iter, double *err,
              double *res_hist);
int or_cgs(int n, const int *irp, const int *ja, const double *val,
           const double *dinv, const double *b, double *x, double eps,
           int itmax, int istop, int *iter, double *err, double *res_hist);
int or_bicg(int n, const int *irp, const int *ja, const double *val,
            const double *dinv, const double *b, double *x, double eps,
            int itmax, int istop, int *iter, double *err, double *res_hist);
int or_bicgstabl(int n, const int *irp, const int *ja, const double *val,
                 const double *dinv, const double *b, double *x, double eps,
                 int itmax, int istop, int irst, int *iter, double *err,
                 double *res_hist);
void or_drotg(double *a, double *b, double *c, double *s);

#ifdef __cplusplus
}
#endif
#endif
