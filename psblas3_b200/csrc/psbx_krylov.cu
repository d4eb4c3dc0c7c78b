// psbx_krylov.cu -- device-resident CG and BiCGSTAB with the diagonal
// preconditioner: the psb_krylov('CG'|'BICGSTAB') path of
// krylov/psb_dkrylov.f90:179-210, krylov/psb_dcg.F90:218-295,
// krylov/psb_dcgstab.f90:226-365, stop test krylov/psb_d_krylov_conv_mod.f90:
// 205-356, prec apply prec/impl/psb_d_diagprec_impl.f90:116.
//
// The reference runs one kernel per BLAS-1 call and brings every dot and
// norm back to the host (3 blocking copies per CG iteration, 5 per
// BiCGSTAB iteration).  Here the scalars (rho, sigma, alpha, beta, omega,
// the stop-test numbers and the iteration counters) live in device memory:
//   CG iteration       = 3 kernels: p-update | SpMV + (p,q) | x,r,z update +
//                        (r,z) and the stop-test norm
//   BiCGSTAB iteration = 5 kernels: p,f | SpMV + (q,v) | s,z | SpMV + (t,t),
//                        (t,s) | x,r update + (q,r) and the stop-test norm
// Each reduction ends in the kernel that produces its operands: blocks write
// one partial each, the last block to finish sums the partials in a fixed
// order and updates the scalars (and the status word).  Every kernel first
// reads the status word and returns at once when the solve has stopped, so
// a CUDA graph of G iterations is replayed until the host, reading the
// status once per replay, sees convergence, itmax, or a breakdown (which
// restarts from r = b - A*x as the reference's restart loop does).
//
// The element-wise updates use the reference's exact operation sequence
// (e.g. x = alpha*p + x; r = -alpha*q + r; p = z + beta*p) with rounded
// multiplies and adds, so they match the CPU path bit for bit given the same
// scalars; only the reduction order differs.
#include "psbx_internal.cuh"

#include <string.h>
#include <strings.h>
#include <vector>

enum { ST_RUN = 0, ST_DONE = 1, ST_BREAK = 2 };

struct KState {
  double rho, rho_old, sigma, alpha, beta, omega, tau;
  double bn2, bni, ani, r0n2;
  double errnum, errden, eps;
  int itmax, istop;
  int it, itx;
  int status;
  int r0set;
};

#define KT 256
#define KLANES 4

struct KWork {
  int n = 0;
  int grid = 0;
  double *vec = nullptr;     // nvec * n doubles
  KState *S = nullptr;       // device
  KState *hS = nullptr;      // pinned host mirror
  double *part = nullptr;    // KLANES * grid
  unsigned *ticket = nullptr;  // 8
};

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ bool stopped(const KState *S) { return *((volatile const int *)&S->status) != ST_RUN; }

__device__ __forceinline__ double prec(const double *__restrict__ dinv, int i, double v) {
  return dinv ? rmul(ld_ro(dinv + i), v) : v;
}

// stop test of psb_d_check_conv_vect (psb_d_krylov_conv_mod.f90:300-341);
// returns 1 when the solve stops at iteration itx.
__device__ __forceinline__ int check_conv(KState *S, double sum_rr, double amax_r, double amax_x) {
  if (S->istop == 1) {
    S->errnum = amax_r;
    S->errden = S->ani * amax_x + S->bni;
  } else if (S->istop == 2) {
    S->errnum = sqrt(sum_rr);
    S->errden = S->bn2;
  } else {
    S->errnum = sqrt(sum_rr);
    S->errden = S->r0n2;
  }
  int res = (S->errden == 0.0) ? (S->errnum <= S->eps) : (S->errnum <= S->eps * S->errden);
  return res || (S->itmax <= S->itx);
}

// Partials: lane k of block b at part[2*(k*grid + b)] (pairs for the
// compensated sums, first slot only for maxima).  Lanes 0-1: sums; 2-3: max.
template <int NS>
__device__ __forceinline__ void publish_sums(double *part, int grid, const dd_t (&v)[NS]) {
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NS; k++) {
      part[2 * ((size_t)k * grid + blockIdx.x)] = v[k].s;
      part[2 * ((size_t)k * grid + blockIdx.x) + 1] = v[k].c;
    }
  }
}

__device__ __forceinline__ void publish_max2(double *part, int grid, const double (&m)[2]) {
  if (threadIdx.x == 0) {
    part[2 * ((size_t)2 * grid + blockIdx.x)] = m[0];
    part[2 * ((size_t)3 * grid + blockIdx.x)] = m[1];
  }
}

__device__ __forceinline__ void final_max2(const double *part, int grid, int n, double (&m)[2], double *smem) {
  m[0] = 0.0;
  m[1] = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    m[0] = fmax(m[0], __ldcg(part + 2 * ((size_t)2 * grid + i)));
    m[1] = fmax(m[1], __ldcg(part + 2 * ((size_t)3 * grid + i)));
  }
  block_max<2>(m, smem);
}

// ---------------------------------------------------------------- setup
// bn2 = ||b||_2, bni = ||b||_inf.
__global__ void __launch_bounds__(KT) k_kry_setup(int n, const double *__restrict__ b, KState *S,
                                                  double *__restrict__ part, unsigned *__restrict__ ticket,
                                                  int grid) {
  __shared__ double sm[128];
  dd_t s[1] = {{0.0, 0.0}};
  double m[2] = {0.0, 0.0};
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    const double v = b[i];
    dd_add_prod(s[0], v, v);
    m[0] = fmax(m[0], fabs(v));
  }
  block_sum_dd<1>(s, sm);
  block_max<2>(m, sm + 64);
  publish_sums<1>(part, grid, s);
  publish_max2(part, grid, m);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[1];
    double mm[2];
    final_sum_dd<1>(part, grid, gridDim.x, o, sm);
    final_max2(part, grid, gridDim.x, mm, sm + 64);
    if (threadIdx.x == 0) {
      S->bn2 = sqrt(dd_value(o[0]));
      S->bni = mm[0];
      *ticket = 0;
    }
  }
}

// ani = ||A||_inf from the stored entries (psb_spnrmi, for istop 1).
template <class View>
__global__ void __launch_bounds__(KT) k_kry_normi(View A, KState *S, double *__restrict__ part,
                                                  unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[64];
  double m[2] = {0.0, 0.0};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) m[0] = fmax(m[0], row_abs_sum(A, s));
  block_max<2>(m, sm);
  publish_max2(part, grid, m);
  if (psbx_last_block(ticket, gridDim.x)) {
    double o[2];
    final_max2(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      S->ani = o[0];
      *ticket = 0;
    }
  }
}

// ---------------------------------------------------------------- CG
// restart: r = b - A*x; z = M^-1 r; rho = (r,z); (r,r) for istop 3.
template <class View>
__global__ void __launch_bounds__(KT) k_cg_init(View A, KState *S, const double *__restrict__ b,
                                                const double *__restrict__ x, const double *__restrict__ dinv,
                                                double *__restrict__ r, double *__restrict__ z,
                                                double *__restrict__ part, unsigned *__restrict__ ticket,
                                                int grid) {
  __shared__ double sm[128];
  dd_t acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double ax = row_dot(A, s, x);
    const int i = out_row(A, s);
    // psb_geaxpby(1,b,0,r); psb_spmm(-1,a,x,1,r): r = (-1)*acc + 1*r
    const double ri = radd(rmul(-1.0, ax), b[i]);
    const double zi = prec(dinv, i, ri);
    r[i] = ri;
    z[i] = zi;
    dd_add_prod(acc[0], ri, zi);
    dd_add_prod(acc[1], ri, ri);
  }
  block_sum_dd<2>(acc, sm);
  publish_sums<2>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[2];
    final_sum_dd<2>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      if (S->istop == 3) S->r0n2 = sqrt(dd_value(o[1]));  // init_conv inside CG's restart loop
      S->rho_old = 0.0;
      S->rho = dd_value(o[0]);
      S->it = 1;
      S->itx = S->itx + 1;
      S->status = ST_RUN;
      *ticket = 0;
    }
  }
}

// p = z (it == 1) or p = z + beta*p
__global__ void __launch_bounds__(KT) k_cg_p(KState *S, int n, const double *__restrict__ z, double *__restrict__ p) {
  if (stopped(S)) return;
  const bool first = S->it == 1;
  const double beta = S->beta;
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT)
    p[i] = first ? z[i] : radd(z[i], rmul(beta, p[i]));
}

// q = A*p ; sigma = (p,q) ; alpha = rho/sigma
template <class View>
__global__ void __launch_bounds__(KT) k_cg_spmv(View A, KState *S, const double *__restrict__ p,
                                                double *__restrict__ q, double *__restrict__ part,
                                                unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[64];
  if (stopped(S)) return;
  dd_t acc[1] = {{0.0, 0.0}};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double t = row_dot(A, s, p);
    const int i = out_row(A, s);
    q[i] = t;
    dd_add_prod(acc[0], ld_ro(p + i), t);
  }
  block_sum_dd<1>(acc, sm);
  publish_sums<1>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[1];
    final_sum_dd<1>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      const double sigma = dd_value(o[0]);
      S->sigma = sigma;
      if (sigma == 0.0) S->status = ST_BREAK;  // psb_dcg.F90:265-270
      else S->alpha = S->rho / sigma;
      *ticket = 0;
    }
  }
}

// x = alpha*p + x ; r = -alpha*q + r ; z = M^-1 r ; (r,z), stop test
__global__ void __launch_bounds__(KT) k_cg_update(KState *S, int n, const double *__restrict__ p,
                                                  const double *__restrict__ q, const double *__restrict__ dinv,
                                                  double *__restrict__ x, double *__restrict__ r,
                                                  double *__restrict__ z, double *__restrict__ part,
                                                  unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[192];
  if (stopped(S)) return;
  const double alpha = S->alpha, malpha = -S->alpha;
  dd_t acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  double mx[2] = {0.0, 0.0};
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    const double xi = radd(rmul(alpha, p[i]), x[i]);
    const double ri = radd(rmul(malpha, q[i]), r[i]);
    const double zi = prec(dinv, i, ri);
    x[i] = xi;
    r[i] = ri;
    z[i] = zi;
    dd_add_prod(acc[0], ri, zi);
    dd_add_prod(acc[1], ri, ri);
    mx[0] = fmax(mx[0], fabs(ri));
    mx[1] = fmax(mx[1], fabs(xi));
  }
  block_sum_dd<2>(acc, sm);
  block_max<2>(mx, sm + 128);
  publish_sums<2>(part, grid, acc);
  publish_max2(part, grid, mx);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[2];
    double m[2];
    final_sum_dd<2>(part, grid, gridDim.x, o, sm);
    final_max2(part, grid, gridDim.x, m, sm + 128);
    if (threadIdx.x == 0) {
      if (check_conv(S, dd_value(o[1]), m[0], m[1])) {
        S->status = ST_DONE;
      } else {
        // next iteration: rho_old = rho; rho = (r,z); breakdown on rho_old
        S->it += 1;
        S->itx += 1;
        S->rho_old = S->rho;
        S->rho = dd_value(o[0]);
        if (S->rho_old == 0.0) S->status = ST_BREAK;  // psb_dcg.F90:253-258
        else S->beta = S->rho / S->rho_old;
      }
      *ticket = 0;
    }
  }
}

// ---------------------------------------------------------------- BiCGSTAB
// restart: r = b - A*x ; q = r ; stop test at itx ; rho = (q,r)
template <class View>
__global__ void __launch_bounds__(KT) k_bcg_init(View A, KState *S, const double *__restrict__ b,
                                                 const double *__restrict__ x, double *__restrict__ r,
                                                 double *__restrict__ q, double *__restrict__ part,
                                                 unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[192];
  dd_t acc[1] = {{0.0, 0.0}};
  double mx[2] = {0.0, 0.0};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double ax = row_dot(A, s, x);
    const int i = out_row(A, s);
    const double ri = radd(rmul(-1.0, ax), b[i]);
    r[i] = ri;
    q[i] = ri;
    dd_add_prod(acc[0], ri, ri);
    mx[0] = fmax(mx[0], fabs(ri));
    mx[1] = fmax(mx[1], fabs(ld_ro(x + i)));
  }
  block_sum_dd<1>(acc, sm);
  block_max<2>(mx, sm + 128);
  publish_sums<1>(part, grid, acc);
  publish_max2(part, grid, mx);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[1];
    double m[2];
    final_sum_dd<1>(part, grid, gridDim.x, o, sm);
    final_max2(part, grid, gridDim.x, m, sm + 128);
    if (threadIdx.x == 0) {
      const double rr = dd_value(o[0]);
      if (S->istop == 3 && !S->r0set) {  // init_conv outside the restart loop
        S->r0n2 = sqrt(rr);
        S->r0set = 1;
      }
      if (check_conv(S, rr, m[0], m[1])) {
        S->status = ST_DONE;
      } else {
        S->it = 1;
        S->itx += 1;
        S->rho_old = 0.0;
        S->rho = rr;  // (q,r) with q == r
        S->status = (rr == 0.0) ? ST_BREAK : ST_RUN;  // psb_dcgstab.f90:267
      }
      *ticket = 0;
    }
  }
}

// p = r (it == 1) or p = -omega*v + p ; p = r + beta*p ;  f = M^-1 p
__global__ void __launch_bounds__(KT) k_bcg_p(KState *S, int n, const double *__restrict__ r,
                                              const double *__restrict__ v, const double *__restrict__ dinv,
                                              double *__restrict__ p, double *__restrict__ f) {
  if (stopped(S)) return;
  const bool first = S->it == 1;
  const double beta = S->beta, momega = -S->omega;
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    double pi;
    if (first) {
      pi = r[i];
    } else {
      pi = radd(rmul(momega, v[i]), p[i]);
      pi = radd(r[i], rmul(beta, pi));
    }
    p[i] = pi;
    f[i] = prec(dinv, i, pi);
  }
}

// v = A*f ; sigma = (q,v) ; alpha = rho/sigma
template <class View>
__global__ void __launch_bounds__(KT) k_bcg_spmv1(View A, KState *S, const double *__restrict__ f,
                                                  const double *__restrict__ q, double *__restrict__ v,
                                                  double *__restrict__ part, unsigned *__restrict__ ticket,
                                                  int grid) {
  __shared__ double sm[64];
  if (stopped(S)) return;
  dd_t acc[1] = {{0.0, 0.0}};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double t = row_dot(A, s, f);
    const int i = out_row(A, s);
    v[i] = t;
    dd_add_prod(acc[0], ld_ro(q + i), t);
  }
  block_sum_dd<1>(acc, sm);
  publish_sums<1>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[1];
    final_sum_dd<1>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      const double sigma = dd_value(o[0]);
      S->sigma = sigma;
      if (sigma == 0.0) S->status = ST_BREAK;  // psb_dcgstab.f90:298
      else S->alpha = S->rho / sigma;
      *ticket = 0;
    }
  }
}

// s = -alpha*v + r ; z = M^-1 s
__global__ void __launch_bounds__(KT) k_bcg_s(KState *S, int n, const double *__restrict__ r,
                                              const double *__restrict__ v, const double *__restrict__ dinv,
                                              double *__restrict__ s, double *__restrict__ z) {
  if (stopped(S)) return;
  const double malpha = -S->alpha;
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    const double si = radd(rmul(malpha, v[i]), r[i]);
    s[i] = si;
    z[i] = prec(dinv, i, si);
  }
}

// t = A*z ; sigma = (t,t) ; tau = (t,s) ; omega = tau/sigma
template <class View>
__global__ void __launch_bounds__(KT) k_bcg_spmv2(View A, KState *S, const double *__restrict__ z,
                                                  const double *__restrict__ sv, double *__restrict__ t,
                                                  double *__restrict__ part, unsigned *__restrict__ ticket,
                                                  int grid) {
  __shared__ double sm[128];
  if (stopped(S)) return;
  dd_t acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double ti = row_dot(A, s, z);
    const int i = out_row(A, s);
    t[i] = ti;
    dd_add_prod(acc[0], ti, ti);
    dd_add_prod(acc[1], ti, ld_ro(sv + i));
  }
  block_sum_dd<2>(acc, sm);
  publish_sums<2>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[2];
    final_sum_dd<2>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      const double sigma = dd_value(o[0]);
      S->sigma = sigma;
      if (sigma == 0.0) {
        S->status = ST_BREAK;  // psb_dcgstab.f90:328
      } else {
        S->tau = dd_value(o[1]);
        S->omega = S->tau / sigma;
        if (S->omega == 0.0) S->status = ST_BREAK;  // psb_dcgstab.f90:346
      }
      *ticket = 0;
    }
  }
}

// x = alpha*f + x ; x = omega*z + x ; r = -omega*t + s ; rho' = (q,r) ;
// stop test ; beta = (rho/rho_old)*(alpha/omega)
__global__ void __launch_bounds__(KT) k_bcg_update(KState *S, int n, const double *__restrict__ f,
                                                   const double *__restrict__ z, const double *__restrict__ s,
                                                   const double *__restrict__ t, const double *__restrict__ q,
                                                   double *__restrict__ x, double *__restrict__ r,
                                                   double *__restrict__ part, unsigned *__restrict__ ticket,
                                                   int grid) {
  __shared__ double sm[192];
  if (stopped(S)) return;
  const double alpha = S->alpha, omega = S->omega, momega = -S->omega;
  dd_t acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  double mx[2] = {0.0, 0.0};
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    double xi = radd(rmul(alpha, f[i]), x[i]);
    xi = radd(rmul(omega, z[i]), xi);
    const double ri = radd(rmul(momega, t[i]), s[i]);
    x[i] = xi;
    r[i] = ri;
    dd_add_prod(acc[0], ld_ro(q + i), ri);
    dd_add_prod(acc[1], ri, ri);
    mx[0] = fmax(mx[0], fabs(ri));
    mx[1] = fmax(mx[1], fabs(xi));
  }
  block_sum_dd<2>(acc, sm);
  block_max<2>(mx, sm + 128);
  publish_sums<2>(part, grid, acc);
  publish_max2(part, grid, mx);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[2];
    double m[2];
    final_sum_dd<2>(part, grid, gridDim.x, o, sm);
    final_max2(part, grid, gridDim.x, m, sm + 128);
    if (threadIdx.x == 0) {
      if (check_conv(S, dd_value(o[1]), m[0], m[1])) {
        S->status = ST_DONE;
      } else {
        S->it += 1;
        S->itx += 1;
        S->rho_old = S->rho;
        S->rho = dd_value(o[0]);
        if (S->rho == 0.0) S->status = ST_BREAK;  // psb_dcgstab.f90:267
        else S->beta = (S->rho / S->rho_old) * (S->alpha / S->omega);
      }
      *ticket = 0;
    }
  }
}

// ---------------------------------------------------------------- prec build
// psb_d_diag_precbld (prec/impl/psb_d_diagprec_impl.f90:229-292) with the
// diagonal of psb_d_hll_get_diag (ext/impl/psb_d_hll_get_diag.f90:89-107):
// dinv(i) = 1/a_ii, or 1 where a_ii == 0 (also for rows without a diagonal).
__device__ __forceinline__ double inv_or_one(double d) { return d == 0.0 ? 1.0 : 1.0 / d; }

__global__ void k_diag_hll(HllView A, const int *__restrict__ idiag, double *__restrict__ dinv) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= A.rows) return;
  const int h = s / A.hksz, ii = s - h * A.hksz;
  const int p = idiag[s];
  const double d = p > 0 ? A.val[(size_t)A.hkoffs[h] + (size_t)(p - 1) * A.hksz + ii] : 0.0;
  dinv[out_row(A, s)] = inv_or_one(d);
}

__global__ void k_diag_ell(EllView A, const int *__restrict__ idiag, double *__restrict__ dinv) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.rows) return;
  const int p = idiag[r];
  const double d = p > 0 ? A.val[(size_t)r + (size_t)(p - 1) * A.pitch] : 0.0;
  dinv[r] = inv_or_one(d);
}

__global__ void k_diag_csr(CsrView A, double *__restrict__ dinv) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.rows) return;
  double d = 0.0;
  for (int k = A.irp[r] - A.base; k < A.irp[r + 1] - A.base; k++)
    if (A.ja[k] - A.base == r) d = A.val[k];
  dinv[r] = inv_or_one(d);
}

static int mat_rows(void *mat, int fmt) {
  if (fmt == PSBX_FMT_HLL) return ((HllDevice *)mat)->rows;
  if (fmt == PSBX_FMT_ELL) return ((EllDevice *)mat)->rows;
  CsrDevice *m = (CsrDevice *)((psbx_d_Cmat *)mat)->mat;
  return m ? m->m : -1;
}

extern "C" int psbx_diag_prec_build(void *mat, int fmt, void *dinv) {
  MultiVectDevice *d = (MultiVectDevice *)dinv;
  if (!mat || !d || d->elemType != SPGPU_TYPE_DOUBLE) return SPGPU_UNSUPPORTED;
  const int n = mat_rows(mat, fmt);
  if (n < 0 || d->size_ < n) return SPGPU_UNSUPPORTED;
  if (n == 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  const int g = (n + 255) / 256;
  if (fmt == PSBX_FMT_HLL) {
    HllDevice *m = (HllDevice *)mat;
    if (m->elemType != SPGPU_TYPE_DOUBLE) return SPGPU_UNSUPPORTED;
    k_diag_hll<<<g, 256, 0, c.stream>>>(hll_view(m), m->diag, (double *)d->v_);
  } else if (fmt == PSBX_FMT_ELL) {
    EllDevice *m = (EllDevice *)mat;
    k_diag_ell<<<g, 256, 0, c.stream>>>(ell_view(m), m->diag, (double *)d->v_);
  } else if (fmt == PSBX_FMT_CSR) {
    k_diag_csr<<<g, 256, 0, c.stream>>>(csr_view((CsrDevice *)((psbx_d_Cmat *)mat)->mat), (double *)d->v_);
  } else {
    return SPGPU_UNSUPPORTED;
  }
  PSBX_LAUNCH_CK("k_diag");
  PSBX_CK(cudaStreamSynchronize(c.stream));
  return SPGPU_SUCCESS;
}

// ---------------------------------------------------------------- driver
#define KGRAPH_ITERS 8

template <class View>
static int solve(const View &A, bool bicg, const double *dinv, const double *b, double *x, int n,
                 psbx_SolverOptions *opt) {
  PsbxCtx &c = psbx_ctx();
  cudaStream_t st = c.stream;
  const int nvec = bicg ? 8 : 4;
  int grid = (n + KT - 1) / KT;
  if (grid > c.sms * 8) grid = c.sms * 8;
  if (grid < 1) grid = 1;

  double *vec = nullptr, *part = nullptr;
  KState *S = nullptr;
  unsigned *ticket = nullptr;
  PSBX_CK(cudaMallocAsync(&vec, sizeof(double) * (size_t)nvec * (size_t)(n > 0 ? n : 1), st));
  PSBX_CK(cudaMallocAsync(&part, sizeof(double) * 2 * KLANES * (size_t)grid, st));
  PSBX_CK(cudaMallocAsync(&S, sizeof(KState), st));
  PSBX_CK(cudaMallocAsync(&ticket, sizeof(unsigned) * 8, st));
  PSBX_CK(cudaMemsetAsync(ticket, 0, sizeof(unsigned) * 8, st));
  PSBX_CK(cudaMemsetAsync(vec, 0, sizeof(double) * (size_t)nvec * (size_t)(n > 0 ? n : 1), st));

  static_assert(sizeof(KState) <= 64 * sizeof(double), "KState fits the pinned staging area");
  KState *hS = (KState *)c.h_res;
  KState init;
  memset(&init, 0, sizeof(init));
  init.eps = opt->eps;
  init.itmax = opt->itmax;
  init.istop = opt->istop;
  init.status = ST_RUN;
  PSBX_CK(cudaMemcpyAsync(S, &init, sizeof(KState), cudaMemcpyHostToDevice, st));

  int rc = SPGPU_SUCCESS;
  double *v0 = vec, *v1 = vec + n, *v2 = vec + 2 * (size_t)n, *v3 = vec + 3 * (size_t)n;
  double *v4 = vec + 4 * (size_t)n, *v5 = vec + 5 * (size_t)n, *v6 = vec + 6 * (size_t)n, *v7 = vec + 7 * (size_t)n;
  // CG: p=v0 q=v1 r=v2 z=v3 ; BiCGSTAB: q=v0 r=v1 p=v2 v=v3 s=v4 t=v5 z=v6 f=v7

  k_kry_setup<<<grid, KT, 0, st>>>(n, b, S, part, ticket, grid);
  psbx_count_launch();
  if (opt->istop == 1) {
    k_kry_normi<View><<<grid, KT, 0, st>>>(A, S, part, ticket, grid);
    psbx_count_launch();
  }

  // one captured batch of KGRAPH_ITERS iterations
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) rc = psbx_cuda_status(e, "BeginCapture");
  if (!rc) {
    for (int k = 0; k < KGRAPH_ITERS; k++) {
      if (!bicg) {
        k_cg_p<<<grid, KT, 0, st>>>(S, n, v3, v0);
        k_cg_spmv<View><<<grid, KT, 0, st>>>(A, S, v0, v1, part, ticket, grid);
        k_cg_update<<<grid, KT, 0, st>>>(S, n, v0, v1, dinv, x, v2, v3, part, ticket, grid);
      } else {
        k_bcg_p<<<grid, KT, 0, st>>>(S, n, v1, v3, dinv, v2, v7);
        k_bcg_spmv1<View><<<grid, KT, 0, st>>>(A, S, v7, v0, v3, part, ticket, grid);
        k_bcg_s<<<grid, KT, 0, st>>>(S, n, v1, v3, dinv, v4, v6);
        k_bcg_spmv2<View><<<grid, KT, 0, st>>>(A, S, v6, v4, v5, part, ticket, grid);
        k_bcg_update<<<grid, KT, 0, st>>>(S, n, v7, v6, v4, v5, v0, x, v1, part, ticket, grid);
      }
    }
    e = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "EndCapture");
  }
  if (!rc) {
    e = cudaGraphInstantiate(&gexec, graph, 0);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "GraphInstantiate");
  }
  const int per_graph = KGRAPH_ITERS * (bicg ? 5 : 3);

  auto fetch = [&]() -> int {
    PSBX_CK(cudaMemcpyAsync(hS, S, sizeof(KState), cudaMemcpyDeviceToHost, st));
    PSBX_CK(cudaStreamSynchronize(st));
    return SPGPU_SUCCESS;
  };

  if (!rc) rc = fetch();
  // restart loop (psb_dcg.F90:218-225 / psb_dcgstab.f90:226-237)
  while (!rc) {
    if (hS->itx >= opt->itmax) break;
    if (!bicg)
      k_cg_init<View><<<grid, KT, 0, st>>>(A, S, b, x, dinv, v2, v3, part, ticket, grid);
    else
      k_bcg_init<View><<<grid, KT, 0, st>>>(A, S, b, x, v1, v0, part, ticket, grid);
    psbx_count_launch();
    if ((rc = fetch())) break;
    if (hS->status == ST_DONE) break;
    if (hS->status == ST_BREAK) continue;
    // iteration loop: replay the captured batch until the status changes
    for (;;) {
      e = cudaGraphLaunch(gexec, st);
      if (e != cudaSuccess) {
        rc = psbx_cuda_status(e, "GraphLaunch");
        break;
      }
      psbx_count_launch(per_graph);
      if ((rc = fetch())) break;
      if (hS->status != ST_RUN) break;
    }
    if (rc || hS->status == ST_DONE) break;
    // ST_BREAK: back to the restart test
  }
  if (!rc) {
    opt->iter = hS->itx;
    opt->err = hS->errden == 0.0 ? hS->errnum : hS->errnum / hS->errden;
  }
  if (gexec) cudaGraphExecDestroy(gexec);
  if (graph) cudaGraphDestroy(graph);
  cudaFreeAsync(vec, st);
  cudaFreeAsync(part, st);
  cudaFreeAsync(S, st);
  cudaFreeAsync(ticket, st);
  cudaError_t e2 = cudaStreamSynchronize(st);
  if (!rc && e2 != cudaSuccess) rc = psbx_cuda_status(e2, "solve");
  return rc;
}

extern "C" int psbx_dkrylov(const char *method, void *mat, int fmt, void *dinv, void *b, void *x,
                            psbx_SolverOptions *opt) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  if (!method || !mat || !b || !x || !opt) return SPGPU_UNSUPPORTED;
  bool bicg;
  if (!strcasecmp(method, "CG")) bicg = false;
  else if (!strcasecmp(method, "BICGSTAB")) bicg = true;
  else return SPGPU_UNSUPPORTED;  // other methods are outside this library
  if (opt->istop < 1 || opt->istop > 3) return SPGPU_UNSUPPORTED;  // psb_err_invalid_istop_
  MultiVectDevice *B = (MultiVectDevice *)b, *X = (MultiVectDevice *)x, *D = (MultiVectDevice *)dinv;
  const int n = mat_rows(mat, fmt);
  if (n < 0 || B->size_ < n || X->size_ < n || (D && D->size_ < n)) return SPGPU_UNSUPPORTED;
  if (B->elemType != SPGPU_TYPE_DOUBLE || X->elemType != SPGPU_TYPE_DOUBLE) return SPGPU_UNSUPPORTED;
  const double *dv = D ? (const double *)D->v_ : nullptr;
  if (opt->itmax <= 0) {
    opt->iter = 0;
    opt->err = 0.0;
    return SPGPU_SUCCESS;
  }
  if (fmt == PSBX_FMT_HLL) {
    HllDevice *m = (HllDevice *)mat;
    if (m->elemType != SPGPU_TYPE_DOUBLE) return SPGPU_UNSUPPORTED;
    if (m->hackSize == 32)
      return solve(hll32_view(hll_view(m)), bicg, dv, (const double *)B->v_, (double *)X->v_, n, opt);
    return solve(hll_view(m), bicg, dv, (const double *)B->v_, (double *)X->v_, n, opt);
  }
  if (fmt == PSBX_FMT_ELL)
    return solve(ell_view((EllDevice *)mat), bicg, dv, (const double *)B->v_, (double *)X->v_, n, opt);
  if (fmt == PSBX_FMT_CSR)
    return solve(csr_view((CsrDevice *)((psbx_d_Cmat *)mat)->mat), bicg, dv, (const double *)B->v_,
                 (double *)X->v_, n, opt);
  return SPGPU_UNSUPPORTED;
}
