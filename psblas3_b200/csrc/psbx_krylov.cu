// psbx_krylov.cu -- device-resident Krylov solvers with the diagonal
// preconditioner: the psb_krylov('CG'|'FCG'|'CGS'|'BICG'|'BICGSTAB'|
// 'BICGSTABL'|'RGMRES') path of krylov/psb_dkrylov.f90:179-210,
// krylov/psb_dcg.F90:218-295, psb_dfcg.F90, psb_dcgs.f90, psb_dbicg.f90,
// krylov/psb_dcgstab.f90:226-365, psb_dcgstabl.f90, psb_drgmres.f90, stop
// test krylov/psb_d_krylov_conv_mod.f90:205-356, prec apply
// prec/impl/psb_d_diagprec_impl.f90:116.
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

// ST_XUPD: a GMRES cycle ended (converged or nl steps); x is updated next.
enum { ST_RUN = 0, ST_DONE = 1, ST_BREAK = 2, ST_XUPD = 3 };

struct KState {
  double rho, rho_old, sigma, alpha, beta, omega, tau;
  double bn2, bni, ani, r0n2;
  double errnum, errden, eps;
  double gamma, delta, theta1, theta2;  // FCG
  double scal;                          // GMRES: scale of the next basis vector
  int itmax, istop;
  int it, itx;
  int status;
  int r0set;
  int first;                            // FCG: first step after a restart
  int gm_m, gm_conv;                    // GMRES: basis vectors in the x update; converged
};

#define KT 256
#define KLANES 4

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

// ---------------------------------------------------------------- FCG
// krylov/psb_dfcg.F90: per iteration w = A v and three dots (one kernel),
// then d, q, x, r updates, v = M^-1 r and the stop-test norms (one kernel).

// restart: r = b - A*x ; v = M^-1 r ; stop test at itx (no increment)
template <class View>
__global__ void __launch_bounds__(KT) k_fcg_init(View A, KState *S, const double *__restrict__ b,
                                                 const double *__restrict__ x, const double *__restrict__ dinv,
                                                 double *__restrict__ r, double *__restrict__ v,
                                                 double *__restrict__ part, unsigned *__restrict__ ticket,
                                                 int grid) {
  __shared__ double sm[192];
  dd_t acc[1] = {{0.0, 0.0}};
  double mx[2] = {0.0, 0.0};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double ax = row_dot(A, s, x);
    const int i = out_row(A, s);
    const double ri = radd(rmul(-1.0, ax), b[i]);
    r[i] = ri;
    v[i] = prec(dinv, i, ri);
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
      if (S->istop == 3 && !S->r0set) {  // psb_init_conv runs once, before the restart loop
        S->r0n2 = sqrt(rr);
        S->r0set = 1;
      }
      S->status = check_conv(S, rr, m[0], m[1]) ? ST_DONE : ST_RUN;
      S->first = 1;
      *ticket = 0;
    }
  }
}

// w = A*v ; alpha = (r,v), beta = (w,v), gamma = (q,v) ; new delta and the
// two step lengths (psb_dfcg.F90 restart block and iteration block)
template <class View>
__global__ void __launch_bounds__(KT) k_fcg_spmv(View A, KState *S, const double *__restrict__ v,
                                                 const double *__restrict__ r, const double *__restrict__ q,
                                                 double *__restrict__ w, double *__restrict__ part,
                                                 unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[192];
  if (stopped(S)) return;
  const bool first = S->first;
  dd_t acc[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double wi = row_dot(A, s, v);
    const int i = out_row(A, s);
    const double vi = ld_ro(v + i);
    w[i] = wi;
    dd_add_prod(acc[0], ld_ro(r + i), vi);
    dd_add_prod(acc[1], wi, vi);
    if (!first) dd_add_prod(acc[2], ld_ro(q + i), vi);
  }
  block_sum_dd<3>(acc, sm);
  publish_sums<3>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[3];
    final_sum_dd<3>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      const double alpha = dd_value(o[0]), beta = dd_value(o[1]);
      if (first) {
        if (beta == 0.0) {
          S->status = ST_DONE;  // exit restart on beta == 0
        } else {
          S->delta = beta;
          S->theta2 = alpha / S->delta;
        }
      } else {
        const double gamma = dd_value(o[2]);
        S->theta1 = gamma / S->delta;
        S->delta = beta - (gamma * gamma) / S->delta;
        if (S->delta == 0.0) S->status = ST_BREAK;  // exit iteration: back to the restart
        else S->theta2 = alpha / S->delta;
      }
      *ticket = 0;
    }
  }
}

// d = v (first) or d = v - theta1 d ; q = w (first) or q = w - theta1 q ;
// x = theta2 d + x ; r = -theta2 q + r ; v = M^-1 r ; itx += 1 ; stop test
__global__ void __launch_bounds__(KT) k_fcg_update(KState *S, int n, const double *__restrict__ w,
                                                   const double *__restrict__ dinv, double *__restrict__ v,
                                                   double *__restrict__ d, double *__restrict__ q,
                                                   double *__restrict__ x, double *__restrict__ r,
                                                   double *__restrict__ part, unsigned *__restrict__ ticket,
                                                   int grid) {
  __shared__ double sm[192];
  if (stopped(S)) return;
  const bool first = S->first;
  const double mt1 = -S->theta1, t2 = S->theta2, mt2 = -S->theta2;
  dd_t acc[1] = {{0.0, 0.0}};
  double mx[2] = {0.0, 0.0};
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    double di, qi;
    if (first) {
      di = v[i];
      qi = w[i];
    } else {
      di = radd(v[i], rmul(mt1, d[i]));
      qi = radd(w[i], rmul(mt1, q[i]));
    }
    const double xi = radd(rmul(t2, di), x[i]);
    const double ri = radd(rmul(mt2, qi), r[i]);
    d[i] = di;
    q[i] = qi;
    x[i] = xi;
    r[i] = ri;
    v[i] = prec(dinv, i, ri);
    dd_add_prod(acc[0], ri, ri);
    mx[0] = fmax(mx[0], fabs(ri));
    mx[1] = fmax(mx[1], fabs(xi));
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
      S->first = 0;
      S->itx += 1;
      if (check_conv(S, dd_value(o[0]), m[0], m[1])) S->status = ST_DONE;
      *ticket = 0;
    }
  }
}

// ---------------------------------------------------------------- RGMRES
// krylov/psb_drgmres.f90, istop 2: one restart cycle of nl inner steps is
// resid | (next, SpMV + h(1,i), MGS steps k = 2..i, last MGS + ||w||) x nl
// | triangular solve | x update.  The small Hessenberg problem (h, c, s, rs)
// lives in device memory and is updated by one thread in the finalisers.
struct GmSmall {
  int ld;        // nl + 1
  double *h;     // ld*ld, column-major
  double *c, *s, *rs;  // ld each
};

// plane rotation of netlib drot with one element
__device__ __forceinline__ void drot1(double &x, double &y, double c, double s) {
  const double t = radd(rmul(c, x), rmul(s, y));
  y = radd(rmul(c, y), -rmul(s, x));
  x = t;
}

// netlib drotg (LAPACK <= 3.9); a <- r, b <- z
__device__ __forceinline__ void drotg(double &a, double &b, double &c, double &s) {
  const double roe = fabs(a) > fabs(b) ? a : b;
  const double scale = radd(fabs(a), fabs(b));
  double r, z;
  if (scale == 0.0) {
    c = 1.0;
    s = 0.0;
    r = 0.0;
    z = 0.0;
  } else {
    const double ta = a / scale, tb = b / scale;
    r = rmul(scale, sqrt(radd(rmul(ta, ta), rmul(tb, tb))));
    r = rmul(roe >= 0.0 ? 1.0 : -1.0, r);
    c = a / r;
    s = b / r;
    z = 1.0;
    if (fabs(a) > fabs(b)) z = s;
    if (fabs(b) >= fabs(a) && c != 0.0) z = 1.0 / c;
  }
  a = r;
  b = z;
}

// restart: v1 = b - A*x ; rs(1) = ||v1|| ; stop test ; scal = 1/rs(1)
template <class View>
__global__ void __launch_bounds__(KT) k_gm_resid(View A, KState *S, GmSmall G, const double *__restrict__ b,
                                                 const double *__restrict__ x, double *__restrict__ v1,
                                                 double *__restrict__ part, unsigned *__restrict__ ticket,
                                                 int grid) {
  __shared__ double sm[64];
  if (stopped(S)) return;
  dd_t acc[1] = {{0.0, 0.0}};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double ax = row_dot(A, s, x);
    const int i = out_row(A, s);
    const double vi = radd(rmul(-1.0, ax), b[i]);
    v1[i] = vi;
    dd_add_prod(acc[0], vi, vi);
  }
  block_sum_dd<1>(acc, sm);
  publish_sums<1>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[1];
    final_sum_dd<1>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      const double rn = sqrt(dd_value(o[0]));
      G.rs[0] = rn;
      for (int k = 1; k < G.ld; k++) G.rs[k] = 0.0;
      S->scal = 1.0 / rn;
      S->errnum = rn;
      S->errden = S->bn2;
      if (S->errnum <= S->eps * S->errden || S->itx >= S->itmax) S->status = ST_DONE;
      *ticket = 0;
    }
  }
}

// v_i = scal * src (src = v_1 for i = 1, else w) ; w1 = M^-1 v_i
__global__ void __launch_bounds__(KT) k_gm_next(KState *S, int n, const double *src, double *vi,
                                                const double *__restrict__ dinv, double *__restrict__ w1) {
  if (stopped(S)) return;
  const double scal = S->scal;
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    const double t = rmul(scal, src[i]);
    vi[i] = t;
    w1[i] = prec(dinv, i, t);
  }
}

// w = A*w1 ; h(1,i) = (v_1, w)
template <class View>
__global__ void __launch_bounds__(KT) k_gm_spmv(View A, KState *S, GmSmall G, int i, const double *__restrict__ w1,
                                                const double *__restrict__ v1, double *__restrict__ w,
                                                double *__restrict__ part, unsigned *__restrict__ ticket,
                                                int grid) {
  __shared__ double sm[64];
  if (stopped(S)) return;
  dd_t acc[1] = {{0.0, 0.0}};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double wi = row_dot(A, s, w1);
    const int r = out_row(A, s);
    w[r] = wi;
    dd_add_prod(acc[0], ld_ro(v1 + r), wi);
  }
  block_sum_dd<1>(acc, sm);
  publish_sums<1>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[1];
    final_sum_dd<1>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      G.h[(size_t)(i - 1) * G.ld] = dd_value(o[0]);
      *ticket = 0;
    }
  }
}

// MGS step k (2 <= k <= i): w = -h(k-1,i) v_{k-1} + w ; h(k,i) = (v_k, w)
__global__ void __launch_bounds__(KT) k_gm_mgs(KState *S, GmSmall G, int i, int k, int n,
                                               const double *__restrict__ vprev, const double *__restrict__ vk,
                                               double *__restrict__ w, double *__restrict__ part,
                                               unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[64];
  if (stopped(S)) return;
  const double mh = -G.h[(k - 2) + (size_t)(i - 1) * G.ld];
  dd_t acc[1] = {{0.0, 0.0}};
  for (int j = blockIdx.x * KT + threadIdx.x; j < n; j += gridDim.x * KT) {
    double wj = w[j];
    if (mh != 0.0) {  // psi_daxpby reads nothing for alpha == 0
      wj = radd(rmul(mh, vprev[j]), wj);
      w[j] = wj;
    }
    dd_add_prod(acc[0], ld_ro(vk + j), wj);
  }
  block_sum_dd<1>(acc, sm);
  publish_sums<1>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[1];
    final_sum_dd<1>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      G.h[(k - 1) + (size_t)(i - 1) * G.ld] = dd_value(o[0]);
      *ticket = 0;
    }
  }
}

// last MGS step: w = -h(i,i) v_i + w ; h(i+1,i) = ||w|| ; scal = 1/h(i+1,i);
// rotations of column i, new rotation, rs update, stop test on |rs(i+1)|
__global__ void __launch_bounds__(KT) k_gm_norm(KState *S, GmSmall G, int i, int nl, int n,
                                                const double *__restrict__ vi, double *__restrict__ w,
                                                double *__restrict__ part, unsigned *__restrict__ ticket,
                                                int grid) {
  __shared__ double sm[64];
  if (stopped(S)) return;
  const int ld = G.ld;
  const double mh = -G.h[(i - 1) + (size_t)(i - 1) * ld];
  dd_t acc[1] = {{0.0, 0.0}};
  for (int j = blockIdx.x * KT + threadIdx.x; j < n; j += gridDim.x * KT) {
    double wj = w[j];
    if (mh != 0.0) {
      wj = radd(rmul(mh, vi[j]), wj);
      w[j] = wj;
    }
    dd_add_prod(acc[0], wj, wj);
  }
  block_sum_dd<1>(acc, sm);
  publish_sums<1>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[1];
    final_sum_dd<1>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      double *hc = G.h + (size_t)(i - 1) * ld;  // column i
      hc[i] = sqrt(dd_value(o[0]));
      S->scal = 1.0 / hc[i];
      for (int k = 2; k <= i; k++) drot1(hc[k - 2], hc[k - 1], G.c[k - 2], G.s[k - 2]);
      double rti = hc[i - 1], rti1 = hc[i], tmp;
      drotg(rti, rti1, tmp, G.s[i - 1]);
      G.c[i - 1] = (double)(float)tmp;  // cmplx(tmp, dzero) without KIND: default precision
      drot1(hc[i - 1], hc[i], G.c[i - 1], G.s[i - 1]);
      hc[i] = 0.0;
      drot1(G.rs[i - 1], G.rs[i], G.c[i - 1], G.s[i - 1]);
      S->itx += 1;
      S->errnum = fabs(G.rs[i]);
      S->errden = S->bn2;
      if (S->errnum <= S->eps * S->errden) {
        S->gm_m = i;
        S->gm_conv = 1;
        S->status = ST_XUPD;
      } else if (i == nl) {
        S->gm_m = nl;
        S->gm_conv = 0;
        S->status = ST_XUPD;
      }
      *ticket = 0;
    }
  }
}

// rs(1:m) = H(1:m,1:m)^-1 rs(1:m)  (netlib dtrsm 'L','U','N','N', one column)
__global__ void k_gm_trsm(KState *S, GmSmall G) {
  if (threadIdx.x != 0 || *((volatile const int *)&S->status) != ST_XUPD) return;
  const int m = S->gm_m, ld = G.ld;
  for (int k = m - 1; k >= 0; k--) {
    if (G.rs[k] != 0.0) {
      G.rs[k] = G.rs[k] / G.h[k + (size_t)k * ld];
      for (int i = 0; i < k; i++) G.rs[i] = radd(G.rs[i], -rmul(G.rs[k], G.h[i + (size_t)k * ld]));
    }
  }
}

// w1 = sum_k rs(k) v_k (k in order, from zero) ; x = M^-1 w1 + x ; then the
// solve stops (converged) or the next cycle restarts
__global__ void __launch_bounds__(KT) k_gm_xupd(KState *S, GmSmall G, int n, const double *__restrict__ V,
                                                const double *__restrict__ dinv, double *__restrict__ x,
                                                unsigned *__restrict__ ticket) {
  if (*((volatile const int *)&S->status) != ST_XUPD) return;
  const int m = S->gm_m;
  for (int j = blockIdx.x * KT + threadIdx.x; j < n; j += gridDim.x * KT) {
    double acc = 0.0;
    for (int k = 0; k < m; k++) {
      const double a = G.rs[k];
      if (a != 0.0) acc = radd(rmul(a, V[(size_t)k * n + j]), acc);
    }
    x[j] = radd(prec(dinv, j, acc), x[j]);
  }
  if (psbx_last_block(ticket, gridDim.x)) {
    if (threadIdx.x == 0) {
      S->status = S->gm_conv ? ST_DONE : ST_RUN;
      *ticket = 0;
    }
  }
}

// ---------------------------------------------------------------- CGS
// krylov/psb_dcgs.f90: per iteration uv/p update and f = M^-1 p | SpMV v = A f
// with (rt,v) | q, s, z = M^-1 s, x update | SpMV A z fused with the r
// update, (rt,r), and the stop-test norms.

// restart: r = b - A*x ; rt = r ; stop test at itx ; first rho = (rt,r)
template <class View>
__global__ void __launch_bounds__(KT) k_cgs_init(View A, KState *S, const double *__restrict__ b,
                                                 const double *__restrict__ x, double *__restrict__ r,
                                                 double *__restrict__ rt, double *__restrict__ part,
                                                 unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[192];
  dd_t acc[1] = {{0.0, 0.0}};
  double mx[2] = {0.0, 0.0};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double ax = row_dot(A, s, x);
    const int i = out_row(A, s);
    const double ri = radd(rmul(-1.0, ax), b[i]);
    r[i] = ri;
    rt[i] = ri;
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
      if (S->istop == 3 && !S->r0set) {  // psb_init_conv runs once, before the restart loop
        S->r0n2 = sqrt(rr);
        S->r0set = 1;
      }
      if (check_conv(S, rr, m[0], m[1])) {
        S->status = ST_DONE;
      } else {
        S->it = 1;
        S->itx += 1;
        S->rho_old = 0.0;
        S->rho = rr;  // (rt,r) with rt == r
        S->status = rr == 0.0 ? ST_BREAK : ST_RUN;
      }
      *ticket = 0;
    }
  }
}

// it == 1: uv = r, p = r ; else uv = beta q + r, p = q + beta p, p = uv + beta p ;
// f = M^-1 p
__global__ void __launch_bounds__(KT) k_cgs_p(KState *S, int n, const double *__restrict__ r,
                                              const double *__restrict__ q, const double *__restrict__ dinv,
                                              double *__restrict__ uv, double *__restrict__ p,
                                              double *__restrict__ f) {
  if (stopped(S)) return;
  const bool first = S->it == 1;
  const double beta = S->beta;
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    const double ri = r[i];
    double ui, pi;
    if (first) {
      ui = ri;
      pi = ri;
    } else {
      const double qi = q[i];
      ui = radd(rmul(beta, qi), ri);
      pi = radd(qi, rmul(beta, p[i]));
      pi = radd(ui, rmul(beta, pi));
    }
    uv[i] = ui;
    p[i] = pi;
    f[i] = prec(dinv, i, pi);
  }
}

// v = A*f ; sigma = (rt,v) ; alpha = rho/sigma
template <class View>
__global__ void __launch_bounds__(KT) k_cgs_spmv1(View A, KState *S, const double *__restrict__ f,
                                                  const double *__restrict__ rt, double *__restrict__ v,
                                                  double *__restrict__ part, unsigned *__restrict__ ticket,
                                                  int grid) {
  __shared__ double sm[64];
  if (stopped(S)) return;
  dd_t acc[1] = {{0.0, 0.0}};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double t = row_dot(A, s, f);
    const int i = out_row(A, s);
    v[i] = t;
    dd_add_prod(acc[0], ld_ro(rt + i), t);
  }
  block_sum_dd<1>(acc, sm);
  publish_sums<1>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[1];
    final_sum_dd<1>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      const double sigma = dd_value(o[0]);
      S->sigma = sigma;
      if (sigma == 0.0) S->status = ST_BREAK;  // psb_dcgs.f90: breakdown s1
      else S->alpha = S->rho / sigma;
      *ticket = 0;
    }
  }
}

// q = -alpha v + uv ; s = q + uv ; z = M^-1 s ; x = alpha z + x
__global__ void __launch_bounds__(KT) k_cgs_q(KState *S, int n, const double *__restrict__ uv,
                                              const double *__restrict__ v, const double *__restrict__ dinv,
                                              double *__restrict__ q, double *__restrict__ z,
                                              double *__restrict__ x) {
  if (stopped(S)) return;
  const double alpha = S->alpha, malpha = -S->alpha;
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    const double ui = uv[i];
    const double qi = radd(rmul(malpha, v[i]), ui);
    const double zi = prec(dinv, i, radd(qi, ui));
    q[i] = qi;
    z[i] = zi;
    x[i] = radd(rmul(alpha, zi), x[i]);
  }
}

// r = -alpha (A z) + r ; stop test ; next rho = (rt,r), beta = rho/rho_old
template <class View>
__global__ void __launch_bounds__(KT) k_cgs_spmv2(View A, KState *S, const double *__restrict__ z,
                                                  const double *__restrict__ rt, const double *__restrict__ x,
                                                  double *__restrict__ r, double *__restrict__ part,
                                                  unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[192];
  if (stopped(S)) return;
  const double malpha = -S->alpha;
  const bool need_x = S->istop == 1;
  dd_t acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  double mx[2] = {0.0, 0.0};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double t = row_dot(A, s, z);
    const int i = out_row(A, s);
    const double ri = radd(rmul(malpha, t), r[i]);
    r[i] = ri;
    dd_add_prod(acc[0], ri, ri);
    dd_add_prod(acc[1], ld_ro(rt + i), ri);
    mx[0] = fmax(mx[0], fabs(ri));
    if (need_x) mx[1] = fmax(mx[1], fabs(x[i]));
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
      if (check_conv(S, dd_value(o[0]), m[0], m[1])) {
        S->status = ST_DONE;
      } else {
        S->it += 1;
        S->itx += 1;
        S->rho_old = S->rho;
        S->rho = dd_value(o[1]);
        if (S->rho == 0.0) S->status = ST_BREAK;  // psb_dcgs.f90: breakdown r
        else S->beta = S->rho / S->rho_old;
      }
      *ticket = 0;
    }
  }
}

// ---------------------------------------------------------------- BiCG
// krylov/psb_dbicg.f90.  The transposed product A^T pt runs on a CSR copy of
// A^T built once per solve (host counting sort, stable: the entries of each
// column in ascending row order), so y_c = sum over rows i of (1*a_ic)*x_i
// accumulates in the order of the reference's scatter loop (csmv 'T').

// qt = A^T pt, one thread per column
__global__ void __launch_bounds__(KT) k_spmv_t(KState *S, int n, const int *__restrict__ tirp,
                                               const int *__restrict__ tja, const double *__restrict__ tval,
                                               const double *__restrict__ x, double *__restrict__ y) {
  if (stopped(S)) return;
  for (int c = blockIdx.x * KT + threadIdx.x; c < n; c += gridDim.x * KT) {
    double acc = 0.0;
    for (int k = tirp[c]; k < tirp[c + 1]; k++) acc = radd(acc, rmul(ld_ro(tval + k), ld_ro(x + ld_ro(tja + k))));
    y[c] = acc;
  }
}

// restart: r = b - A*x ; rt = r ; stop test at itx
template <class View>
__global__ void __launch_bounds__(KT) k_bicg_init(View A, KState *S, const double *__restrict__ b,
                                                  const double *__restrict__ x, double *__restrict__ r,
                                                  double *__restrict__ rt, double *__restrict__ part,
                                                  unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[192];
  dd_t acc[1] = {{0.0, 0.0}};
  double mx[2] = {0.0, 0.0};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double ax = row_dot(A, s, x);
    const int i = out_row(A, s);
    const double ri = radd(rmul(-1.0, ax), b[i]);
    r[i] = ri;
    rt[i] = ri;
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
      if (S->istop == 3 && !S->r0set) {  // psb_init_conv runs once, before the restart loop
        S->r0n2 = sqrt(rr);
        S->r0set = 1;
      }
      S->status = check_conv(S, rr, m[0], m[1]) ? ST_DONE : ST_RUN;
      S->it = 0;
      S->rho = 0.0;
      *ticket = 0;
    }
  }
}

// iteration top after a restart: z = M^-1 r ; zt = M^-1 rt ; rho = (rt,z)
__global__ void __launch_bounds__(KT) k_bicg_top(KState *S, int n, const double *__restrict__ r,
                                                 const double *__restrict__ rt, const double *__restrict__ dinv,
                                                 double *__restrict__ z, double *__restrict__ zt,
                                                 double *__restrict__ part, unsigned *__restrict__ ticket,
                                                 int grid) {
  __shared__ double sm[64];
  if (stopped(S)) return;
  dd_t acc[1] = {{0.0, 0.0}};
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    const double zi = prec(dinv, i, r[i]);
    const double rti = rt[i];
    z[i] = zi;
    zt[i] = prec(dinv, i, rti);
    dd_add_prod(acc[0], rti, zi);
  }
  block_sum_dd<1>(acc, sm);
  publish_sums<1>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[1];
    final_sum_dd<1>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      S->it += 1;
      S->itx += 1;
      S->rho_old = S->rho;
      S->rho = dd_value(o[0]);
      if (S->rho == 0.0) S->status = ST_BREAK;  // psb_dbicg.f90: breakdown r
      else if (S->it > 1) S->beta = S->rho / S->rho_old;
      *ticket = 0;
    }
  }
}

// p = z, pt = zt (it == 1) or p = z + beta p, pt = zt + beta pt
__global__ void __launch_bounds__(KT) k_bicg_p(KState *S, int n, const double *__restrict__ z,
                                               const double *__restrict__ zt, double *__restrict__ p,
                                               double *__restrict__ pt) {
  if (stopped(S)) return;
  const bool first = S->it == 1;
  const double beta = S->beta;
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    p[i] = first ? z[i] : radd(z[i], rmul(beta, p[i]));
    pt[i] = first ? zt[i] : radd(zt[i], rmul(beta, pt[i]));
  }
}

// q = A*p ; sigma = (pt,q) ; alpha = rho/sigma
template <class View>
__global__ void __launch_bounds__(KT) k_bicg_spmv(View A, KState *S, const double *__restrict__ p,
                                                  const double *__restrict__ pt, double *__restrict__ q,
                                                  double *__restrict__ part, unsigned *__restrict__ ticket,
                                                  int grid) {
  __shared__ double sm[64];
  if (stopped(S)) return;
  dd_t acc[1] = {{0.0, 0.0}};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double t = row_dot(A, s, p);
    const int i = out_row(A, s);
    q[i] = t;
    dd_add_prod(acc[0], ld_ro(pt + i), t);
  }
  block_sum_dd<1>(acc, sm);
  publish_sums<1>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[1];
    final_sum_dd<1>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      const double sigma = dd_value(o[0]);
      S->sigma = sigma;
      if (sigma == 0.0) S->status = ST_BREAK;  // psb_dbicg.f90: breakdown s1
      else S->alpha = S->rho / sigma;
      *ticket = 0;
    }
  }
}

// x = alpha p + x ; r = -alpha q + r ; rt = -alpha qt + rt ; stop test ;
// next top: z = M^-1 r, zt = M^-1 rt, rho = (rt,z)
__global__ void __launch_bounds__(KT) k_bicg_update(KState *S, int n, const double *__restrict__ p,
                                                    const double *__restrict__ q, const double *__restrict__ qt,
                                                    const double *__restrict__ dinv, double *__restrict__ x,
                                                    double *__restrict__ r, double *__restrict__ rt,
                                                    double *__restrict__ z, double *__restrict__ zt,
                                                    double *__restrict__ part, unsigned *__restrict__ ticket,
                                                    int grid) {
  __shared__ double sm[192];
  if (stopped(S)) return;
  const double alpha = S->alpha, malpha = -S->alpha;
  dd_t acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  double mx[2] = {0.0, 0.0};
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    const double xi = radd(rmul(alpha, p[i]), x[i]);
    const double ri = radd(rmul(malpha, q[i]), r[i]);
    const double rti = radd(rmul(malpha, qt[i]), rt[i]);
    const double zi = prec(dinv, i, ri);
    x[i] = xi;
    r[i] = ri;
    rt[i] = rti;
    z[i] = zi;
    zt[i] = prec(dinv, i, rti);
    dd_add_prod(acc[0], ri, ri);
    dd_add_prod(acc[1], rti, zi);
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
      if (check_conv(S, dd_value(o[0]), m[0], m[1])) {
        S->status = ST_DONE;
      } else {
        S->it += 1;
        S->itx += 1;
        S->rho_old = S->rho;
        S->rho = dd_value(o[1]);
        if (S->rho == 0.0) S->status = ST_BREAK;
        else S->beta = S->rho / S->rho_old;
      }
      *ticket = 0;
    }
  }
}

// ---------------------------------------------------------------- BiCGSTAB(L)
// krylov/psb_dcgstabl.f90 with nl = irst, kernel by kernel: every axpby,
// dot and preconditioned product of the reference is one small kernel whose
// scalars live in device memory (LState), and one outer iteration (nl BiCG
// steps + the minimal-residual part) is one CUDA graph.
struct LState {
  double rho, rho_old, alpha, beta, omega;
  double *gamma, *gamma1, *gamma2, *sigma, *taum;  // [nl+1] each, taum [(nl+1)^2]
  int nl;
};

// y = a*x + b*y with the special cases of psi_daxpby (psi_d_serial_impl.F90:
// alpha == 0 reads no x, beta == 0 reads no y); a = ca * (*pa) when pa is
// given, else ca; b likewise
__global__ void __launch_bounds__(KT) k_l_axpby(KState *S, int n, const double *pa, double ca,
                                                const double *__restrict__ x, const double *pb, double cb,
                                                double *__restrict__ y) {
  if (stopped(S)) return;
  const double a = pa ? ca * *pa : ca, b = pb ? cb * *pb : cb;
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    if (a == 0.0) {
      if (b == 0.0) y[i] = 0.0;
      else if (b != 1.0) y[i] = rmul(b, y[i]);
    } else if (b == 0.0) {
      y[i] = rmul(a, x[i]);
    } else {
      y[i] = radd(rmul(a, x[i]), rmul(b, y[i]));
    }
  }
}

// y = M^-1 (A x): psb_spmm(1,a,x,0,y) followed by prec%apply(y) in place
template <class View>
__global__ void __launch_bounds__(KT) k_l_spmv(View A, KState *S, const double *__restrict__ x,
                                               const double *__restrict__ dinv, double *__restrict__ y) {
  if (stopped(S)) return;
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double t = row_dot(A, s, x);
    const int i = out_row(A, s);
    y[i] = prec(dinv, i, t);
  }
}

enum { LOP_RHO = 0, LOP_GAMMA = 1, LOP_TAU = 2, LOP_SIGMA = 3 };

// dot products and the scalar step that follows each one in the reference:
//   LOP_RHO    rho_old = rho; rho = (a,b); rho == 0 -> restart;
//              beta = alpha*rho/rho_old; rho_old = rho
//   LOP_GAMMA  gamma(j) = (a,b); == 0 -> restart; alpha = rho/gamma(j)
//   LOP_TAU    taum(i,j) = (a,b) / sigma(i)
//   LOP_SIGMA  sigma(j) = (a,a); gamma1(j) = (c,a) / sigma(j)   (c = rh(0))
__global__ void __launch_bounds__(KT) k_l_dot(KState *S, LState *L, int op, int i, int j, int n,
                                              const double *__restrict__ a, const double *__restrict__ b,
                                              const double *__restrict__ c, double *__restrict__ part,
                                              unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[128];
  if (stopped(S)) return;
  dd_t acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (int k = blockIdx.x * KT + threadIdx.x; k < n; k += gridDim.x * KT) {
    const double ak = a[k];
    dd_add_prod(acc[0], ak, op == LOP_SIGMA ? ak : b[k]);
    if (op == LOP_SIGMA) dd_add_prod(acc[1], c[k], ak);
  }
  block_sum_dd<2>(acc, sm);
  publish_sums<2>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[2];
    final_sum_dd<2>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      const double d = dd_value(o[0]);
      const int ld = L->nl + 1;
      if (op == LOP_RHO) {
        L->rho_old = L->rho;
        L->rho = d;
        if (d == 0.0) {
          S->status = ST_BREAK;
        } else {
          L->beta = L->alpha * L->rho / L->rho_old;
          L->rho_old = L->rho;
        }
      } else if (op == LOP_GAMMA) {
        L->gamma[j] = d;
        if (d == 0.0) S->status = ST_BREAK;
        else L->alpha = L->rho / d;
      } else if (op == LOP_TAU) {
        L->taum[i + (size_t)j * ld] = d / L->sigma[i];
      } else {
        L->sigma[j] = d;
        L->gamma1[j] = dd_value(o[1]) / d;
      }
      *ticket = 0;
    }
  }
}

// top of an outer iteration: itx += nl ; rho = -omega*rho
__global__ void k_l_top(KState *S, LState *L) {
  if (threadIdx.x != 0 || stopped(S)) return;
  S->itx += L->nl;
  L->rho = -L->omega * L->rho;
}

// the minimal-residual recurrences of gamma, omega and gamma2
__global__ void k_l_mr(KState *S, LState *L) {
  if (threadIdx.x != 0 || stopped(S)) return;
  const int nl = L->nl, ld = nl + 1;
  double *g = L->gamma, *g1 = L->gamma1, *g2 = L->gamma2, *tau = L->taum;
  g[nl] = g1[nl];
  L->omega = g[nl];
  for (int j = nl - 1; j >= 1; j--) {
    g[j] = g1[j];
    for (int i = j + 1; i <= nl; i++) g[j] = radd(g[j], -rmul(tau[j + (size_t)i * ld], g[i]));
  }
  for (int j = 1; j <= nl - 1; j++) {
    g2[j] = g[j + 1];
    for (int i = j + 1; i <= nl - 1; i++) g2[j] = radd(g2[j], rmul(tau[j + (size_t)i * ld], g[i + 1]));
  }
}

// restart: r = M^-1 (b - A x) ; rt0 = rh(0) = r ; uh(0) = 0 ; rho = 1,
// alpha = 0, omega = 1 ; stop test on r (no itx increment)
template <class View>
__global__ void __launch_bounds__(KT) k_l_init(View A, KState *S, LState *L, const double *__restrict__ b,
                                               const double *__restrict__ x, const double *__restrict__ dinv,
                                               double *__restrict__ rt0, double *__restrict__ rh0,
                                               double *__restrict__ uh0, double *__restrict__ part,
                                               unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[192];
  dd_t acc[1] = {{0.0, 0.0}};
  double mx[2] = {0.0, 0.0};
  for (int s = blockIdx.x * KT + threadIdx.x; s < A.rows; s += gridDim.x * KT) {
    const double ax = row_dot(A, s, x);
    const int i = out_row(A, s);
    const double ri = prec(dinv, i, radd(rmul(-1.0, ax), b[i]));
    rt0[i] = ri;
    rh0[i] = ri;
    uh0[i] = 0.0;
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
      if (S->istop == 3 && !S->r0set) {  // psb_init_conv runs once, before the restart loop
        S->r0n2 = sqrt(rr);
        S->r0set = 1;
      }
      L->rho = 1.0;
      L->alpha = 0.0;
      L->omega = 1.0;
      S->status = check_conv(S, rr, m[0], m[1]) ? ST_DONE : ST_RUN;
      *ticket = 0;
    }
  }
}

// stop test on (x, rh(0)) at the end of an outer iteration
__global__ void __launch_bounds__(KT) k_l_check(KState *S, int n, const double *__restrict__ x,
                                                const double *__restrict__ r, double *__restrict__ part,
                                                unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[192];
  if (stopped(S)) return;
  dd_t acc[1] = {{0.0, 0.0}};
  double mx[2] = {0.0, 0.0};
  for (int i = blockIdx.x * KT + threadIdx.x; i < n; i += gridDim.x * KT) {
    const double ri = r[i];
    dd_add_prod(acc[0], ri, ri);
    mx[0] = fmax(mx[0], fabs(ri));
    mx[1] = fmax(mx[1], fabs(x[i]));
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
      if (check_conv(S, dd_value(o[0]), m[0], m[1])) S->status = ST_DONE;
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

// The kernels that sum the wide hacks' rows before each product
// (psbx_long_rows): 2 (ordered), 1 (split), 0 without wide hacks.
template <class View> static inline int long_launch(const View &) { return 0; }
static inline int long_launch(const Hll32WView &A) { return A.wideSplit ? 1 : 2; }

// Replays a captured batch of iterations until running(status) is false,
// with 1, 2, 4, then 8 replays between two reads of the status word: a long
// solve pays one host round trip per 64 iterations, and the kernels of the
// replays queued after the stop return at once (they test the status).
template <class Pred>
static int replay_until(cudaGraphExec_t gexec, cudaStream_t st, int per_graph, KState *S, KState *hS,
                        Pred running) {
  int batch = 1;
  for (;;) {
    for (int k = 0; k < batch; k++) {
      cudaError_t e = cudaGraphLaunch(gexec, st);
      if (e != cudaSuccess) return psbx_cuda_status(e, "GraphLaunch");
      psbx_count_launch(per_graph);
    }
    PSBX_CK(cudaMemcpyAsync(hS, S, sizeof(KState), cudaMemcpyDeviceToHost, st));
    PSBX_CK(cudaStreamSynchronize(st));
    if (!running(*hS)) return SPGPU_SUCCESS;
    if (batch < 8) batch *= 2;
  }
}

// Captured iteration graphs of the CG / BiCGSTAB driver, kept with their
// workspaces.  A graph is a function of its kernels' arguments alone (matrix
// view, vectors, workspace, sizes; the solver options live in the state
// word, written at every call), so a later call whose arguments are the same
// replays the kept graph instead of capturing and instantiating it again --
// the repeated solves of a time-stepping loop.  The key holds every field of
// the view and every pointer and size the captured kernels receive.  At most
// KCACHE_N graphs, least recently used out; workspaces over KCACHE_MAX bytes
// are not kept (their solves are long enough not to notice the capture).
#define KCACHE_N 4
#define KCACHE_MAX ((size_t)64 << 20)

struct KCache {
  std::vector<uint64_t> key;
  cudaGraphExec_t gexec = nullptr;
  double *vec = nullptr, *part = nullptr;
  KState *S = nullptr;
  unsigned *ticket = nullptr;
  uint64_t used = 0;
};
static KCache g_kc[KCACHE_N];
static uint64_t g_kc_clock = 0;

static void key_hll(std::vector<uint64_t> &k, const HllView &v, uint64_t tag) {
  k.insert(k.end(), {tag, (uint64_t)v.val, (uint64_t)v.ja, (uint64_t)v.irn, (uint64_t)v.hkoffs, (uint64_t)v.perm,
                     (uint64_t)(uint32_t)v.rows, (uint64_t)(uint32_t)v.hksz, (uint64_t)(uint32_t)v.base,
                     (uint64_t)v.longHacks, (uint64_t)v.lres, (uint64_t)(uint32_t)v.nLong,
                     (uint64_t)(uint32_t)v.longW, (uint64_t)v.wideBase, (uint64_t)v.wchunk, (uint64_t)v.wprod,
                     (uint64_t)(uint32_t)v.nWChunks, (uint64_t)(uint32_t)v.wideSplit, (uint64_t)v.wpart,
                     (uint64_t)v.wticket, (uint64_t)v.wcbase});
}
static void key_view(std::vector<uint64_t> &k, const HllView &v) { key_hll(k, v, 0); }
static void key_view(std::vector<uint64_t> &k, const Hll32View &v) { key_hll(k, v, 1); }
static void key_view(std::vector<uint64_t> &k, const Hll32WView &v) { key_hll(k, v, 2); }
static void key_view(std::vector<uint64_t> &k, const Hll32SView &v) { key_hll(k, v, 5); }
static void key_view(std::vector<uint64_t> &k, const EllView &v) {
  k.insert(k.end(), {3, (uint64_t)v.val, (uint64_t)v.ja, (uint64_t)v.irn, (uint64_t)(uint32_t)v.rows,
                     (uint64_t)(uint32_t)v.pitch, (uint64_t)(uint32_t)v.base});
}
static void key_view(std::vector<uint64_t> &k, const CsrView &v) {
  k.insert(k.end(), {4, (uint64_t)v.val, (uint64_t)v.ja, (uint64_t)v.irp, (uint64_t)(uint32_t)v.rows,
                     (uint64_t)(uint32_t)v.base});
}

static void kc_release(KCache &e, cudaStream_t st) {
  if (e.gexec) {
    cudaStreamSynchronize(st);  // no replay of it in flight
    cudaGraphExecDestroy(e.gexec);
  }
  cudaFreeAsync(e.vec, st);
  cudaFreeAsync(e.part, st);
  cudaFreeAsync(e.S, st);
  cudaFreeAsync(e.ticket, st);
  e = KCache();
}

void psbx_krylov_cache_clear() {
  cudaStream_t st = psbx_ctx().stream;
  for (KCache &e : g_kc)
    if (!e.key.empty()) kc_release(e, st);
  cudaStreamSynchronize(st);
}

static KCache *kc_find(const std::vector<uint64_t> &key) {
  for (KCache &e : g_kc)
    if (!e.key.empty() && e.key == key) {
      e.used = ++g_kc_clock;
      return &e;
    }
  return nullptr;
}

static KCache *kc_slot(cudaStream_t st) {  // a free entry, else the least recently used one, released
  KCache *lru = &g_kc[0];
  for (KCache &e : g_kc) {
    if (e.key.empty()) return &e;
    if (e.used < lru->used) lru = &e;
  }
  kc_release(*lru, st);
  return lru;
}

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
  cudaGraphExec_t gexec = nullptr;
  const size_t vbytes = sizeof(double) * (size_t)nvec * (size_t)(n > 0 ? n : 1);
  std::vector<uint64_t> key;
  KCache *ce = nullptr;
  if (vbytes <= KCACHE_MAX) {
    key_view(key, A);
    key.insert(key.end(), {(uint64_t)bicg, (uint64_t)dinv, (uint64_t)b, (uint64_t)x, (uint64_t)(uint32_t)n,
                           (uint64_t)(uint32_t)grid});
    ce = kc_find(key);
  }
  if (ce) {
    vec = ce->vec;
    part = ce->part;
    S = ce->S;
    ticket = ce->ticket;
    gexec = ce->gexec;
  } else {
    PSBX_CK(psbx_malloc_async(&vec, vbytes, st));
    PSBX_CK(psbx_malloc_async(&part, sizeof(double) * 2 * KLANES * (size_t)grid, st));
    PSBX_CK(psbx_malloc_async(&S, sizeof(KState), st));
    PSBX_CK(psbx_malloc_async(&ticket, sizeof(unsigned) * 8, st));
  }
  PSBX_CK(cudaMemsetAsync(ticket, 0, sizeof(unsigned) * 8, st));
  PSBX_CK(cudaMemsetAsync(vec, 0, vbytes, st));

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

  // one captured batch of KGRAPH_ITERS iterations (kept from an earlier call
  // with the same arguments, or captured now)
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaSuccess;
  if (!gexec) {
    e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "BeginCapture");
  }
  if (!rc && !gexec) {
    for (int k = 0; k < KGRAPH_ITERS; k++) {
      if (!bicg) {
        k_cg_p<<<grid, KT, 0, st>>>(S, n, v3, v0);
        psbx_long_rows(A, v0, &S->status, st);
        k_cg_spmv<View><<<grid, KT, 0, st>>>(A, S, v0, v1, part, ticket, grid);
        k_cg_update<<<grid, KT, 0, st>>>(S, n, v0, v1, dinv, x, v2, v3, part, ticket, grid);
      } else {
        k_bcg_p<<<grid, KT, 0, st>>>(S, n, v1, v3, dinv, v2, v7);
        psbx_long_rows(A, v7, &S->status, st);
        k_bcg_spmv1<View><<<grid, KT, 0, st>>>(A, S, v7, v0, v3, part, ticket, grid);
        k_bcg_s<<<grid, KT, 0, st>>>(S, n, v1, v3, dinv, v4, v6);
        psbx_long_rows(A, v6, &S->status, st);
        k_bcg_spmv2<View><<<grid, KT, 0, st>>>(A, S, v6, v4, v5, part, ticket, grid);
        k_bcg_update<<<grid, KT, 0, st>>>(S, n, v7, v6, v4, v5, v0, x, v1, part, ticket, grid);
      }
    }
    e = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "EndCapture");
    if (!rc) {
      e = cudaGraphInstantiate(&gexec, graph, 0);
      if (e != cudaSuccess) rc = psbx_cuda_status(e, "GraphInstantiate");
    }
    if (!rc && !key.empty()) {  // keep it, with the workspace it was captured on
      ce = kc_slot(st);
      ce->key = key;
      ce->gexec = gexec;
      ce->vec = vec;
      ce->part = part;
      ce->S = S;
      ce->ticket = ticket;
      ce->used = ++g_kc_clock;
    }
  }
  const int per_graph = KGRAPH_ITERS * ((bicg ? 5 : 3) + (bicg ? 2 : 1) * long_launch(A));

  auto fetch = [&]() -> int {
    PSBX_CK(cudaMemcpyAsync(hS, S, sizeof(KState), cudaMemcpyDeviceToHost, st));
    PSBX_CK(cudaStreamSynchronize(st));
    return SPGPU_SUCCESS;
  };

  if (!rc) rc = fetch();
  // restart loop (psb_dcg.F90:218-225 / psb_dcgstab.f90:226-237)
  while (!rc) {
    if (hS->itx >= opt->itmax) break;
    if ((rc = psbx_long_rows(A, x, nullptr, st))) break;
    if (!bicg)
      k_cg_init<View><<<grid, KT, 0, st>>>(A, S, b, x, dinv, v2, v3, part, ticket, grid);
    else
      k_bcg_init<View><<<grid, KT, 0, st>>>(A, S, b, x, v1, v0, part, ticket, grid);
    psbx_count_launch(1 + long_launch(A));
    if ((rc = fetch())) break;
    if (hS->status == ST_DONE) break;
    if (hS->status == ST_BREAK) continue;
    // iteration loop: replay the captured batch until the status changes
    rc = replay_until(gexec, st, per_graph, S, hS, [](const KState &k) { return k.status == ST_RUN; });
    if (rc || hS->status == ST_DONE) break;
    // ST_BREAK: back to the restart test
  }
  if (!rc) {
    opt->iter = hS->itx;
    opt->err = hS->errden == 0.0 ? hS->errnum : hS->errnum / hS->errden;
  }
  if (graph) cudaGraphDestroy(graph);
  if (!ce) {  // not kept
    if (gexec) cudaGraphExecDestroy(gexec);
    cudaFreeAsync(vec, st);
    cudaFreeAsync(part, st);
    cudaFreeAsync(S, st);
    cudaFreeAsync(ticket, st);
  }
  cudaError_t e2 = cudaStreamSynchronize(st);
  if (!rc && e2 != cudaSuccess) rc = psbx_cuda_status(e2, "solve");
  return rc;
}

// FCG driver: restart kernel on the host loop, then a graph of
// KGRAPH_ITERS x (SpMV + dots | updates) replayed until the status changes.
template <class View>
static int solve_fcg(const View &A, const double *dinv, const double *b, double *x, int n, psbx_SolverOptions *opt) {
  PsbxCtx &c = psbx_ctx();
  cudaStream_t st = c.stream;
  int grid = (n + KT - 1) / KT;
  if (grid > c.sms * 8) grid = c.sms * 8;
  if (grid < 1) grid = 1;
  const size_t nn = (size_t)(n > 0 ? n : 1);
  double *vec = nullptr, *part = nullptr;
  KState *S = nullptr;
  unsigned *ticket = nullptr;
  PSBX_CK(psbx_malloc_async(&vec, sizeof(double) * 5 * nn, st));
  PSBX_CK(psbx_malloc_async(&part, sizeof(double) * 2 * KLANES * (size_t)grid, st));
  PSBX_CK(psbx_malloc_async(&S, sizeof(KState), st));
  PSBX_CK(psbx_malloc_async(&ticket, sizeof(unsigned) * 8, st));
  PSBX_CK(cudaMemsetAsync(ticket, 0, sizeof(unsigned) * 8, st));
  PSBX_CK(cudaMemsetAsync(vec, 0, sizeof(double) * 5 * nn, st));
  KState *hS = (KState *)c.h_res;
  KState init;
  memset(&init, 0, sizeof(init));
  init.eps = opt->eps;
  init.itmax = opt->itmax;
  init.istop = opt->istop;
  init.status = ST_RUN;
  PSBX_CK(cudaMemcpyAsync(S, &init, sizeof(KState), cudaMemcpyHostToDevice, st));
  double *v = vec, *w = vec + nn, *d = vec + 2 * nn, *q = vec + 3 * nn, *r = vec + 4 * nn;

  k_kry_setup<<<grid, KT, 0, st>>>(n, b, S, part, ticket, grid);
  psbx_count_launch();
  if (opt->istop == 1) {
    k_kry_normi<View><<<grid, KT, 0, st>>>(A, S, part, ticket, grid);
    psbx_count_launch();
  }
  int rc = SPGPU_SUCCESS;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) rc = psbx_cuda_status(e, "BeginCapture");
  if (!rc) {
    for (int k = 0; k < KGRAPH_ITERS; k++) {
      psbx_long_rows(A, v, &S->status, st);
      k_fcg_spmv<View><<<grid, KT, 0, st>>>(A, S, v, r, q, w, part, ticket, grid);
      k_fcg_update<<<grid, KT, 0, st>>>(S, n, w, dinv, v, d, q, x, r, part, ticket, grid);
    }
    e = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "EndCapture");
  }
  if (!rc) {
    e = cudaGraphInstantiate(&gexec, graph, 0);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "GraphInstantiate");
  }
  auto fetch = [&]() -> int {
    PSBX_CK(cudaMemcpyAsync(hS, S, sizeof(KState), cudaMemcpyDeviceToHost, st));
    PSBX_CK(cudaStreamSynchronize(st));
    return SPGPU_SUCCESS;
  };
  // restart loop of psb_dfcg.F90
  while (!rc) {
    if ((rc = psbx_long_rows(A, x, nullptr, st))) break;
    k_fcg_init<View><<<grid, KT, 0, st>>>(A, S, b, x, dinv, r, v, part, ticket, grid);
    psbx_count_launch(1 + long_launch(A));
    if ((rc = fetch())) break;
    if (hS->status == ST_DONE) break;
    rc = replay_until(gexec, st, (2 + long_launch(A)) * KGRAPH_ITERS, S, hS,
                      [](const KState &k) { return k.status == ST_RUN; });
    if (rc || hS->status == ST_DONE) break;
    // ST_BREAK (delta == 0): back to the restart, whose kernel resets the status
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
  if (!rc && e2 != cudaSuccess) rc = psbx_cuda_status(e2, "solve_fcg");
  return rc;
}

// RGMRES driver (istop 2): one graph per restart cycle, replayed until the
// status word says done.
template <class View>
static int solve_gmres(const View &A, const double *dinv, const double *b, double *x, int n,
                       psbx_SolverOptions *opt) {
  PsbxCtx &c = psbx_ctx();
  cudaStream_t st = c.stream;
  const int nl = opt->irst, ld = nl + 1;
  int grid = (n + KT - 1) / KT;
  if (grid > c.sms * 8) grid = c.sms * 8;
  if (grid < 1) grid = 1;
  const size_t nn = (size_t)(n > 0 ? n : 1);
  double *vec = nullptr, *part = nullptr, *small = nullptr;
  KState *S = nullptr;
  unsigned *ticket = nullptr;
  // V (ld vectors), w, w1
  PSBX_CK(psbx_malloc_async(&vec, sizeof(double) * (size_t)(ld + 2) * nn, st));
  PSBX_CK(psbx_malloc_async(&small, sizeof(double) * ((size_t)ld * ld + 3 * (size_t)ld), st));
  PSBX_CK(psbx_malloc_async(&part, sizeof(double) * 2 * KLANES * (size_t)grid, st));
  PSBX_CK(psbx_malloc_async(&S, sizeof(KState), st));
  PSBX_CK(psbx_malloc_async(&ticket, sizeof(unsigned) * 8, st));
  PSBX_CK(cudaMemsetAsync(ticket, 0, sizeof(unsigned) * 8, st));
  PSBX_CK(cudaMemsetAsync(vec, 0, sizeof(double) * (size_t)(ld + 2) * nn, st));
  PSBX_CK(cudaMemsetAsync(small, 0, sizeof(double) * ((size_t)ld * ld + 3 * (size_t)ld), st));
  KState *hS = (KState *)c.h_res;
  KState init;
  memset(&init, 0, sizeof(init));
  init.eps = opt->eps;
  init.itmax = opt->itmax;
  init.istop = opt->istop;
  init.status = ST_RUN;
  PSBX_CK(cudaMemcpyAsync(S, &init, sizeof(KState), cudaMemcpyHostToDevice, st));
  GmSmall G;
  G.ld = ld;
  G.h = small;
  G.c = small + (size_t)ld * ld;
  G.s = G.c + ld;
  G.rs = G.s + ld;
  double *V = vec, *w = vec + (size_t)ld * nn, *w1 = w + nn;
  auto Vk = [&](int k) { return V + (size_t)k * nn; };  // 0-based basis vector

  k_kry_setup<<<grid, KT, 0, st>>>(n, b, S, part, ticket, grid);
  psbx_count_launch();
  int rc = SPGPU_SUCCESS, per_graph = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) rc = psbx_cuda_status(e, "BeginCapture");
  if (!rc) {
    psbx_long_rows(A, x, &S->status, st);
    k_gm_resid<View><<<grid, KT, 0, st>>>(A, S, G, b, x, Vk(0), part, ticket, grid);
    per_graph += 1 + long_launch(A);
    for (int i = 1; i <= nl; i++) {
      k_gm_next<<<grid, KT, 0, st>>>(S, n, i == 1 ? Vk(0) : w, Vk(i - 1), dinv, w1);
      psbx_long_rows(A, w1, &S->status, st);
      k_gm_spmv<View><<<grid, KT, 0, st>>>(A, S, G, i, w1, Vk(0), w, part, ticket, grid);
      for (int k = 2; k <= i; k++)
        k_gm_mgs<<<grid, KT, 0, st>>>(S, G, i, k, n, Vk(k - 2), Vk(k - 1), w, part, ticket, grid);
      k_gm_norm<<<grid, KT, 0, st>>>(S, G, i, nl, n, Vk(i - 1), w, part, ticket, grid);
      per_graph += 3 + (i - 1) + long_launch(A);
    }
    k_gm_trsm<<<1, 32, 0, st>>>(S, G);
    k_gm_xupd<<<grid, KT, 0, st>>>(S, G, n, V, dinv, x, ticket);
    per_graph += 2;
    e = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "EndCapture");
  }
  if (!rc) {
    e = cudaGraphInstantiate(&gexec, graph, 0);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "GraphInstantiate");
  }
  // each replay is one restart cycle; the solve ends when the status says done
  if (!rc) rc = replay_until(gexec, st, per_graph, S, hS, [](const KState &k) { return k.status != ST_DONE; });
  if (!rc) {
    opt->iter = hS->itx;
    opt->err = hS->errden == 0.0 ? hS->errnum : hS->errnum / hS->errden;
  }
  if (gexec) cudaGraphExecDestroy(gexec);
  if (graph) cudaGraphDestroy(graph);
  cudaFreeAsync(vec, st);
  cudaFreeAsync(small, st);
  cudaFreeAsync(part, st);
  cudaFreeAsync(S, st);
  cudaFreeAsync(ticket, st);
  cudaError_t e2 = cudaStreamSynchronize(st);
  if (!rc && e2 != cudaSuccess) rc = psbx_cuda_status(e2, "solve_gmres");
  return rc;
}

// CGS driver: restart kernel on the host loop, then a graph of
// KGRAPH_ITERS x (uv,p,f | SpMV + (rt,v) | q,z,x | SpMV + r, (rt,r), stop test).
template <class View>
static int solve_cgs(const View &A, const double *dinv, const double *b, double *x, int n, psbx_SolverOptions *opt) {
  PsbxCtx &c = psbx_ctx();
  cudaStream_t st = c.stream;
  int grid = (n + KT - 1) / KT;
  if (grid > c.sms * 8) grid = c.sms * 8;
  if (grid < 1) grid = 1;
  const size_t nn = (size_t)(n > 0 ? n : 1);
  double *vec = nullptr, *part = nullptr;
  KState *S = nullptr;
  unsigned *ticket = nullptr;
  PSBX_CK(psbx_malloc_async(&vec, sizeof(double) * 8 * nn, st));
  PSBX_CK(psbx_malloc_async(&part, sizeof(double) * 2 * KLANES * (size_t)grid, st));
  PSBX_CK(psbx_malloc_async(&S, sizeof(KState), st));
  PSBX_CK(psbx_malloc_async(&ticket, sizeof(unsigned) * 8, st));
  PSBX_CK(cudaMemsetAsync(ticket, 0, sizeof(unsigned) * 8, st));
  PSBX_CK(cudaMemsetAsync(vec, 0, sizeof(double) * 8 * nn, st));
  KState *hS = (KState *)c.h_res;
  KState init;
  memset(&init, 0, sizeof(init));
  init.eps = opt->eps;
  init.itmax = opt->itmax;
  init.istop = opt->istop;
  init.status = ST_RUN;
  PSBX_CK(cudaMemcpyAsync(S, &init, sizeof(KState), cudaMemcpyHostToDevice, st));
  double *r = vec, *rt = vec + nn, *p = vec + 2 * nn, *q = vec + 3 * nn, *uv = vec + 4 * nn, *f = vec + 5 * nn,
         *v = vec + 6 * nn, *z = vec + 7 * nn;

  k_kry_setup<<<grid, KT, 0, st>>>(n, b, S, part, ticket, grid);
  psbx_count_launch();
  if (opt->istop == 1) {
    k_kry_normi<View><<<grid, KT, 0, st>>>(A, S, part, ticket, grid);
    psbx_count_launch();
  }
  int rc = SPGPU_SUCCESS;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) rc = psbx_cuda_status(e, "BeginCapture");
  if (!rc) {
    for (int k = 0; k < KGRAPH_ITERS; k++) {
      k_cgs_p<<<grid, KT, 0, st>>>(S, n, r, q, dinv, uv, p, f);
      psbx_long_rows(A, f, &S->status, st);
      k_cgs_spmv1<View><<<grid, KT, 0, st>>>(A, S, f, rt, v, part, ticket, grid);
      k_cgs_q<<<grid, KT, 0, st>>>(S, n, uv, v, dinv, q, z, x);
      psbx_long_rows(A, z, &S->status, st);
      k_cgs_spmv2<View><<<grid, KT, 0, st>>>(A, S, z, rt, x, r, part, ticket, grid);
    }
    e = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "EndCapture");
  }
  if (!rc) {
    e = cudaGraphInstantiate(&gexec, graph, 0);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "GraphInstantiate");
  }
  auto fetch = [&]() -> int {
    PSBX_CK(cudaMemcpyAsync(hS, S, sizeof(KState), cudaMemcpyDeviceToHost, st));
    PSBX_CK(cudaStreamSynchronize(st));
    return SPGPU_SUCCESS;
  };
  if (!rc) rc = fetch();
  // restart loop of psb_dcgs.f90
  while (!rc) {
    if (hS->itx >= opt->itmax) break;
    if ((rc = psbx_long_rows(A, x, nullptr, st))) break;
    k_cgs_init<View><<<grid, KT, 0, st>>>(A, S, b, x, r, rt, part, ticket, grid);
    psbx_count_launch(1 + long_launch(A));
    if ((rc = fetch())) break;
    if (hS->status == ST_DONE) break;
    if (hS->status == ST_BREAK) continue;
    rc = replay_until(gexec, st, (4 + 2 * long_launch(A)) * KGRAPH_ITERS, S, hS,
                      [](const KState &k) { return k.status == ST_RUN; });
    if (rc || hS->status == ST_DONE) break;
    // ST_BREAK (rho or sigma == 0): back to the restart
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
  if (!rc && e2 != cudaSuccess) rc = psbx_cuda_status(e2, "solve_cgs");
  return rc;
}

// CSR of A^T (0-based), entries of each column in ascending row order, from
// the matrix's own arrays (read back once per solve).
static int build_transpose(void *mat, int fmt, int n, int **tirp, int **tja, double **tval) {
  PsbxCtx &c = psbx_ctx();
  std::vector<int> rowptr(n + 1, 0), cols;
  std::vector<double> vals;
  auto get = [&](void *dst, const void *src, size_t bytes) -> int {
    if (!bytes) return SPGPU_SUCCESS;
    PSBX_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c.stream));
    return SPGPU_SUCCESS;
  };
  int rc = SPGPU_SUCCESS;
  if (fmt == PSBX_FMT_HLL) {
    HllDevice *m = (HllDevice *)mat;
    const int hk = m->hackSize, nh = (m->rows + hk - 1) / hk;
    std::vector<int> hko(nh + 1), irn(m->rows), ja(m->allocsize), perm;
    std::vector<double> val(m->allocsize);
    rc = get(hko.data(), m->hackOffs, sizeof(int) * (nh + 1));
    if (!rc) rc = get(irn.data(), m->rS, sizeof(int) * m->rows);
    if (!rc) rc = get(ja.data(), m->rP, sizeof(int) * (size_t)m->allocsize);
    if (!rc) rc = get(val.data(), m->cM, sizeof(double) * (size_t)m->allocsize);
    if (!rc && m->perm) {
      perm.resize(m->rows);
      rc = get(perm.data(), m->perm, sizeof(int) * m->rows);
    }
    if (!rc) PSBX_CK(cudaStreamSynchronize(c.stream));
    std::vector<int> srow(n);  // storage row of each matrix row
    for (int s = 0; s < m->rows; s++) srow[perm.empty() ? s : perm[s]] = s;
    for (int i = 0; i < n; i++) {
      const int s = srow[i], h = s / hk, l = s % hk;
      for (int j = 0; j < irn[s]; j++) {
        const size_t p = (size_t)hko[h] + (size_t)j * hk + l;
        cols.push_back(ja[p] - m->baseIndex);
        vals.push_back(val[p]);
      }
      rowptr[i + 1] = (int)cols.size();
    }
  } else if (fmt == PSBX_FMT_ELL) {
    EllDevice *m = (EllDevice *)mat;
    std::vector<int> irn(m->rows), ja((size_t)m->pitch * m->maxRowSize);
    std::vector<double> val((size_t)m->pitch * m->maxRowSize);
    rc = get(irn.data(), m->rS, sizeof(int) * m->rows);
    if (!rc) rc = get(ja.data(), m->rP, sizeof(int) * ja.size());
    if (!rc) rc = get(val.data(), m->cM, sizeof(double) * val.size());
    if (!rc) PSBX_CK(cudaStreamSynchronize(c.stream));
    for (int i = 0; i < n; i++) {
      for (int j = 0; j < irn[i]; j++) {
        const size_t p = (size_t)i + (size_t)j * m->pitch;
        cols.push_back(ja[p] - m->baseIndex);
        vals.push_back(val[p]);
      }
      rowptr[i + 1] = (int)cols.size();
    }
  } else {
    CsrDevice *m = (CsrDevice *)((psbx_d_Cmat *)mat)->mat;
    std::vector<int> irp(m->m + 1), ja(m->nz);
    std::vector<double> val(m->nz);
    rc = get(irp.data(), m->irp, sizeof(int) * (m->m + 1));
    if (!rc) rc = get(ja.data(), m->ja, sizeof(int) * (size_t)m->nz);
    if (!rc) rc = get(val.data(), m->val, sizeof(double) * (size_t)m->nz);
    if (!rc) PSBX_CK(cudaStreamSynchronize(c.stream));
    for (int i = 0; i < n; i++) {
      for (int k = irp[i] - m->baseIndex; k < irp[i + 1] - m->baseIndex; k++) {
        cols.push_back(ja[k] - m->baseIndex);
        vals.push_back(val[k]);
      }
      rowptr[i + 1] = (int)cols.size();
    }
  }
  if (rc) return rc;
  PSBX_CK(cudaStreamSynchronize(c.stream));
  // counting sort by column; rows are visited in ascending order, so each
  // column's entries come out in ascending row order
  const size_t nz = cols.size();
  std::vector<int> tp(n + 1, 0), tj(nz > 0 ? nz : 1), next;
  std::vector<double> tv(nz > 0 ? nz : 1);
  for (size_t k = 0; k < nz; k++) {
    if (cols[k] < 0 || cols[k] >= n) return SPGPU_UNSUPPORTED;  // BiCG needs a square matrix
    tp[cols[k] + 1]++;
  }
  for (int c2 = 0; c2 < n; c2++) tp[c2 + 1] += tp[c2];
  next.assign(tp.begin(), tp.end() - 1);
  for (int i = 0; i < n; i++)
    for (int k = rowptr[i]; k < rowptr[i + 1]; k++) {
      const int pos = next[cols[k]]++;
      tj[pos] = i;
      tv[pos] = vals[k];
    }
  PSBX_CK(psbx_malloc_async(tirp, sizeof(int) * (n + 1), c.stream));
  PSBX_CK(psbx_malloc_async(tja, sizeof(int) * tj.size(), c.stream));
  PSBX_CK(psbx_malloc_async(tval, sizeof(double) * tv.size(), c.stream));
  PSBX_CK(cudaMemcpyAsync(*tirp, tp.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, c.stream));
  PSBX_CK(cudaMemcpyAsync(*tja, tj.data(), sizeof(int) * tj.size(), cudaMemcpyHostToDevice, c.stream));
  PSBX_CK(cudaMemcpyAsync(*tval, tv.data(), sizeof(double) * tv.size(), cudaMemcpyHostToDevice, c.stream));
  PSBX_CK(cudaStreamSynchronize(c.stream));
  return SPGPU_SUCCESS;
}

// BiCG driver: transpose once, restart kernels on the host loop, then a graph
// of KGRAPH_ITERS x (p,pt | SpMV + (pt,q) | A^T pt | updates, stop test, top).
template <class View>
static int solve_bicg(const View &A, void *mat, int fmt, const double *dinv, const double *b, double *x, int n,
                      psbx_SolverOptions *opt) {
  PsbxCtx &c = psbx_ctx();
  cudaStream_t st = c.stream;
  int *tirp = nullptr, *tja = nullptr;
  double *tval = nullptr;
  int rc = build_transpose(mat, fmt, n, &tirp, &tja, &tval);
  if (rc) return rc;
  int grid = (n + KT - 1) / KT;
  if (grid > c.sms * 8) grid = c.sms * 8;
  if (grid < 1) grid = 1;
  const size_t nn = (size_t)(n > 0 ? n : 1);
  double *vec = nullptr, *part = nullptr;
  KState *S = nullptr;
  unsigned *ticket = nullptr;
  PSBX_CK(psbx_malloc_async(&vec, sizeof(double) * 8 * nn, st));
  PSBX_CK(psbx_malloc_async(&part, sizeof(double) * 2 * KLANES * (size_t)grid, st));
  PSBX_CK(psbx_malloc_async(&S, sizeof(KState), st));
  PSBX_CK(psbx_malloc_async(&ticket, sizeof(unsigned) * 8, st));
  PSBX_CK(cudaMemsetAsync(ticket, 0, sizeof(unsigned) * 8, st));
  PSBX_CK(cudaMemsetAsync(vec, 0, sizeof(double) * 8 * nn, st));
  KState *hS = (KState *)c.h_res;
  KState init;
  memset(&init, 0, sizeof(init));
  init.eps = opt->eps;
  init.itmax = opt->itmax;
  init.istop = opt->istop;
  init.status = ST_RUN;
  PSBX_CK(cudaMemcpyAsync(S, &init, sizeof(KState), cudaMemcpyHostToDevice, st));
  double *r = vec, *rt = vec + nn, *z = vec + 2 * nn, *zt = vec + 3 * nn, *p = vec + 4 * nn, *pt = vec + 5 * nn,
         *q = vec + 6 * nn, *qt = vec + 7 * nn;

  k_kry_setup<<<grid, KT, 0, st>>>(n, b, S, part, ticket, grid);
  psbx_count_launch();
  if (opt->istop == 1) {
    k_kry_normi<View><<<grid, KT, 0, st>>>(A, S, part, ticket, grid);
    psbx_count_launch();
  }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) rc = psbx_cuda_status(e, "BeginCapture");
  if (!rc) {
    for (int k = 0; k < KGRAPH_ITERS; k++) {
      k_bicg_p<<<grid, KT, 0, st>>>(S, n, z, zt, p, pt);
      psbx_long_rows(A, p, &S->status, st);
      k_bicg_spmv<View><<<grid, KT, 0, st>>>(A, S, p, pt, q, part, ticket, grid);
      k_spmv_t<<<grid, KT, 0, st>>>(S, n, tirp, tja, tval, pt, qt);
      k_bicg_update<<<grid, KT, 0, st>>>(S, n, p, q, qt, dinv, x, r, rt, z, zt, part, ticket, grid);
    }
    e = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "EndCapture");
  }
  if (!rc) {
    e = cudaGraphInstantiate(&gexec, graph, 0);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "GraphInstantiate");
  }
  auto fetch = [&]() -> int {
    PSBX_CK(cudaMemcpyAsync(hS, S, sizeof(KState), cudaMemcpyDeviceToHost, st));
    PSBX_CK(cudaStreamSynchronize(st));
    return SPGPU_SUCCESS;
  };
  if (!rc) rc = fetch();
  // restart loop of psb_dbicg.f90
  while (!rc) {
    if (hS->itx >= opt->itmax) break;
    if ((rc = psbx_long_rows(A, x, nullptr, st))) break;
    k_bicg_init<View><<<grid, KT, 0, st>>>(A, S, b, x, r, rt, part, ticket, grid);
    k_bicg_top<<<grid, KT, 0, st>>>(S, n, r, rt, dinv, z, zt, part, ticket, grid);
    psbx_count_launch(2 + long_launch(A));
    if ((rc = fetch())) break;
    if (hS->status == ST_DONE) break;
    if (hS->status == ST_BREAK) continue;
    rc = replay_until(gexec, st, (4 + long_launch(A)) * KGRAPH_ITERS, S, hS,
                      [](const KState &k) { return k.status == ST_RUN; });
    if (rc || hS->status == ST_DONE) break;
    // ST_BREAK (rho or sigma == 0): back to the restart
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
  cudaFreeAsync(tirp, st);
  cudaFreeAsync(tja, st);
  cudaFreeAsync(tval, st);
  cudaError_t e2 = cudaStreamSynchronize(st);
  if (!rc && e2 != cudaSuccess) rc = psbx_cuda_status(e2, "solve_bicg");
  return rc;
}

// BiCGSTAB(L) driver: the restart kernel on the host loop, then one graph
// per outer iteration (nl BiCG steps, the minimal-residual part, the stop
// test), replayed until the status changes.
template <class View>
static int solve_bicgstabl(const View &A, const double *dinv, const double *b, double *x, int n,
                           psbx_SolverOptions *opt) {
  PsbxCtx &c = psbx_ctx();
  cudaStream_t st = c.stream;
  const int nl = opt->irst, ld = nl + 1;
  int grid = (n + KT - 1) / KT;
  if (grid > c.sms * 8) grid = c.sms * 8;
  if (grid < 1) grid = 1;
  const size_t nn = (size_t)(n > 0 ? n : 1);
  double *vec = nullptr, *part = nullptr, *small = nullptr;
  KState *S = nullptr;
  LState *L = nullptr;
  unsigned *ticket = nullptr;
  // rt0, uh(0..nl), rh(0..nl)
  const size_t nv = 1 + 2 * (size_t)ld;
  PSBX_CK(psbx_malloc_async(&vec, sizeof(double) * nv * nn, st));
  PSBX_CK(psbx_malloc_async(&small, sizeof(double) * (4 * (size_t)ld + (size_t)ld * ld), st));
  PSBX_CK(psbx_malloc_async(&part, sizeof(double) * 2 * KLANES * (size_t)grid, st));
  PSBX_CK(psbx_malloc_async(&S, sizeof(KState), st));
  PSBX_CK(psbx_malloc_async(&L, sizeof(LState), st));
  PSBX_CK(psbx_malloc_async(&ticket, sizeof(unsigned) * 8, st));
  PSBX_CK(cudaMemsetAsync(ticket, 0, sizeof(unsigned) * 8, st));
  PSBX_CK(cudaMemsetAsync(vec, 0, sizeof(double) * nv * nn, st));
  PSBX_CK(cudaMemsetAsync(small, 0, sizeof(double) * (4 * (size_t)ld + (size_t)ld * ld), st));
  KState *hS = (KState *)c.h_res;
  KState init;
  memset(&init, 0, sizeof(init));
  init.eps = opt->eps;
  init.itmax = opt->itmax;
  init.istop = opt->istop;
  init.status = ST_RUN;
  PSBX_CK(cudaMemcpyAsync(S, &init, sizeof(KState), cudaMemcpyHostToDevice, st));
  LState hl;
  memset(&hl, 0, sizeof(hl));
  hl.gamma = small;
  hl.gamma1 = small + ld;
  hl.gamma2 = small + 2 * ld;
  hl.sigma = small + 3 * ld;
  hl.taum = small + 4 * ld;
  hl.nl = nl;
  PSBX_CK(cudaMemcpyAsync(L, &hl, sizeof(LState), cudaMemcpyHostToDevice, st));
  double *rt0 = vec;
  auto UH = [&](int k) { return vec + (1 + (size_t)k) * nn; };
  auto RH = [&](int k) { return vec + (1 + (size_t)ld + k) * nn; };
  const double *Lbeta = &L->beta, *Lalpha = &L->alpha;

  k_kry_setup<<<grid, KT, 0, st>>>(n, b, S, part, ticket, grid);
  psbx_count_launch();
  if (opt->istop == 1) {
    k_kry_normi<View><<<grid, KT, 0, st>>>(A, S, part, ticket, grid);
    psbx_count_launch();
  }
  int rc = SPGPU_SUCCESS, per_graph = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) rc = psbx_cuda_status(e, "BeginCapture");
  if (!rc) {
    auto spmv = [&](const double *in, double *out) {
      psbx_long_rows(A, in, &S->status, st);
      k_l_spmv<View><<<grid, KT, 0, st>>>(A, S, in, dinv, out);
      per_graph += 1 + long_launch(A);
    };
    auto axpby = [&](const double *pa, double ca, const double *xx, const double *pb, double cb, double *yy) {
      k_l_axpby<<<grid, KT, 0, st>>>(S, n, pa, ca, xx, pb, cb, yy);
      per_graph++;
    };
    auto dot = [&](int op, int i, int j, const double *a, const double *bb, const double *cc) {
      k_l_dot<<<grid, KT, 0, st>>>(S, L, op, i, j, n, a, bb, cc, part, ticket, grid);
      per_graph++;
    };
    k_l_top<<<1, 32, 0, st>>>(S, L);
    per_graph++;
    for (int j = 0; j < nl; j++) {
      dot(LOP_RHO, 0, j, RH(j), rt0, nullptr);
      for (int k = 0; k <= j; k++) axpby(nullptr, 1.0, RH(k), Lbeta, -1.0, UH(k));
      spmv(UH(j), UH(j + 1));
      dot(LOP_GAMMA, 0, j, UH(j + 1), rt0, nullptr);
      for (int k = 0; k <= j; k++) axpby(Lalpha, -1.0, UH(k + 1), nullptr, 1.0, RH(k));
      axpby(Lalpha, 1.0, UH(0), nullptr, 1.0, x);
      spmv(RH(j), RH(j + 1));
    }
    for (int j = 1; j <= nl; j++) {
      for (int i = 1; i <= j - 1; i++) {
        dot(LOP_TAU, i, j, RH(i), RH(j), nullptr);
        axpby(hl.taum + i + (size_t)j * ld, -1.0, RH(i), nullptr, 1.0, RH(j));
      }
      dot(LOP_SIGMA, 0, j, RH(j), nullptr, RH(0));
    }
    k_l_mr<<<1, 32, 0, st>>>(S, L);
    per_graph++;
    axpby(hl.gamma + 1, 1.0, RH(0), nullptr, 1.0, x);
    axpby(hl.gamma1 + nl, -1.0, RH(nl), nullptr, 1.0, RH(0));
    axpby(hl.gamma + nl, -1.0, UH(nl), nullptr, 1.0, UH(0));
    for (int j = 1; j <= nl - 1; j++) {
      axpby(hl.gamma + j, -1.0, UH(j), nullptr, 1.0, UH(0));
      axpby(hl.gamma2 + j, 1.0, RH(j), nullptr, 1.0, x);
      axpby(hl.gamma1 + j, -1.0, RH(j), nullptr, 1.0, RH(0));
    }
    k_l_check<<<grid, KT, 0, st>>>(S, n, x, RH(0), part, ticket, grid);
    per_graph++;
    e = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "EndCapture");
  }
  if (!rc) {
    e = cudaGraphInstantiate(&gexec, graph, 0);
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "GraphInstantiate");
  }
  auto fetch = [&]() -> int {
    PSBX_CK(cudaMemcpyAsync(hS, S, sizeof(KState), cudaMemcpyDeviceToHost, st));
    PSBX_CK(cudaStreamSynchronize(st));
    return SPGPU_SUCCESS;
  };
  if (!rc) rc = fetch();
  // restart loop of psb_dcgstabl.f90
  while (!rc) {
    if (hS->itx >= opt->itmax) break;
    if ((rc = psbx_long_rows(A, x, nullptr, st))) break;
    k_l_init<View><<<grid, KT, 0, st>>>(A, S, L, b, x, dinv, rt0, RH(0), UH(0), part, ticket, grid);
    psbx_count_launch(1 + long_launch(A));
    if ((rc = fetch())) break;
    if (hS->status == ST_DONE) break;
    rc = replay_until(gexec, st, per_graph, S, hS, [](const KState &k) { return k.status == ST_RUN; });
    if (rc || hS->status == ST_DONE) break;
    // ST_BREAK (rho or gamma(j) == 0): back to the restart
  }
  if (!rc) {
    opt->iter = hS->itx;
    opt->err = hS->errden == 0.0 ? hS->errnum : hS->errnum / hS->errden;
  }
  if (gexec) cudaGraphExecDestroy(gexec);
  if (graph) cudaGraphDestroy(graph);
  cudaFreeAsync(vec, st);
  cudaFreeAsync(small, st);
  cudaFreeAsync(part, st);
  cudaFreeAsync(S, st);
  cudaFreeAsync(L, st);
  cudaFreeAsync(ticket, st);
  cudaError_t e2 = cudaStreamSynchronize(st);
  if (!rc && e2 != cudaSuccess) rc = psbx_cuda_status(e2, "solve_bicgstabl");
  return rc;
}

template <class View>
static int run_method(int meth, const View &A, const double *dinv, const double *b, double *x, int n,
                      psbx_SolverOptions *opt) {
  if (meth == 2) return solve_fcg(A, dinv, b, x, n, opt);
  if (meth == 3) return solve_gmres(A, dinv, b, x, n, opt);
  if (meth == 4) return solve_cgs(A, dinv, b, x, n, opt);
  if (meth == 6) return solve_bicgstabl(A, dinv, b, x, n, opt);
  return solve(A, meth == 1, dinv, b, x, n, opt);
}

extern "C" int psbx_dkrylov(const char *method, void *mat, int fmt, void *dinv, void *b, void *x,
                            psbx_SolverOptions *opt) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  if (!method || !mat || !b || !x || !opt) return SPGPU_UNSUPPORTED;
  // 0 CG, 1 BICGSTAB, 2 FCG, 3 RGMRES, 4 CGS, 5 BICG, 6 BICGSTABL (psb_dkrylov.f90:179-210)
  int meth;
  if (!strcasecmp(method, "CG")) meth = 0;
  else if (!strcasecmp(method, "BICGSTAB")) meth = 1;
  else if (!strcasecmp(method, "FCG")) meth = 2;
  else if (!strcasecmp(method, "RGMRES") || !strcasecmp(method, "GMRES")) meth = 3;
  else if (!strcasecmp(method, "CGS")) meth = 4;
  else if (!strcasecmp(method, "BICG")) meth = 5;
  else if (!strcasecmp(method, "BICGSTABL")) meth = 6;
  else return SPGPU_UNSUPPORTED;  // other methods are outside this library
  if (opt->istop < 1 || opt->istop > 3) return SPGPU_UNSUPPORTED;  // psb_err_invalid_istop_
  // RGMRES: the reference accepts istop 1 and 2 (psb_drgmres.f90); istop 1
  // is not provided here, and irst must be positive (psb_err_invalid_irst_)
  if (meth == 3 && (opt->istop != 2 || opt->irst <= 0)) return SPGPU_UNSUPPORTED;
  if (meth == 6 && opt->irst <= 0) return SPGPU_UNSUPPORTED;  // psb_err_invalid_irst_
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
  if (meth == 5) {  // BiCG also needs the matrix's arrays, for its transpose
    const double *bp = (const double *)B->v_;
    double *xp = (double *)X->v_;
    if (fmt == PSBX_FMT_HLL) {
      HllDevice *m = (HllDevice *)mat;
      if (m->elemType != SPGPU_TYPE_DOUBLE) return SPGPU_UNSUPPORTED;
      const HllView v = hll_view(m);
      if (m->hackSize == 32 && v.nLong > 0) return solve_bicg(hll32w_view(v), mat, fmt, dv, bp, xp, n, opt);
      if (hll_short_rows(m)) return solve_bicg(hll32s_view(v), mat, fmt, dv, bp, xp, n, opt);
      if (m->hackSize == 32) return solve_bicg(hll32_view(v), mat, fmt, dv, bp, xp, n, opt);
      return solve_bicg(v, mat, fmt, dv, bp, xp, n, opt);
    }
    if (fmt == PSBX_FMT_ELL) return solve_bicg(ell_view((EllDevice *)mat), mat, fmt, dv, bp, xp, n, opt);
    if (fmt == PSBX_FMT_CSR)
      return solve_bicg(csr_view((CsrDevice *)((psbx_d_Cmat *)mat)->mat), mat, fmt, dv, bp, xp, n, opt);
    return SPGPU_UNSUPPORTED;
  }
  if (fmt == PSBX_FMT_HLL) {
    HllDevice *m = (HllDevice *)mat;
    if (m->elemType != SPGPU_TYPE_DOUBLE) return SPGPU_UNSUPPORTED;
    if (m->hackSize == 32) {
      const HllView v = hll_view(m);
      if (v.nLong > 0) return run_method(meth, hll32w_view(v), dv, (const double *)B->v_, (double *)X->v_, n, opt);
      if (hll_short_rows(m))
        return run_method(meth, hll32s_view(v), dv, (const double *)B->v_, (double *)X->v_, n, opt);
      return run_method(meth, hll32_view(v), dv, (const double *)B->v_, (double *)X->v_, n, opt);
    }
    return run_method(meth, hll_view(m), dv, (const double *)B->v_, (double *)X->v_, n, opt);
  }
  if (fmt == PSBX_FMT_ELL)
    return run_method(meth, ell_view((EllDevice *)mat), dv, (const double *)B->v_, (double *)X->v_, n, opt);
  if (fmt == PSBX_FMT_CSR)
    return run_method(meth, csr_view((CsrDevice *)((psbx_d_Cmat *)mat)->mat), dv, (const double *)B->v_,
                      (double *)X->v_, n, opt);
  return SPGPU_UNSUPPORTED;
}
