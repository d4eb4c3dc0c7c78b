// psbx_mixed.cu -- mixed-precision CG for one system: psbx_dmixed_cg.
//
// Solves A x = b to the FP64 tolerance ||b - A x||_2 <= eps ||b||_2 (the
// istop = 2 test of psb_d_krylov_conv_mod.f90:300-341) with the diagonal
// preconditioner, as psb_krylov('CG') does (krylov/psb_dcg.F90:218-295), but
// runs the iterations in FP32: the FP32 copy of the values (indices int32),
// FP32 vectors, every dot product accumulated in FP64 (a product of two
// floats is exact in FP64; the sums are compensated).  The FP64 parts are
// the residual r = b - A x, the solution x and the convergence test.
//
// The FP32 recursion is kept honest by residual replacement ("reliable
// updates": G. L. G. Sleijpen and H. A. van der Vorst, "Reliable updated
// residuals in hybrid Bi-CG methods", Computing 56, 1996; as used for mixed
// precision CG by M. A. Clark et al., Comput. Phys. Commun. 181, 2010).  The
// FP32 correction xh accumulates the steps; when the recursive residual has
// fallen by the factor delta since the last replacement (or below the
// tolerance), the correction is added to x in FP64, r = b - A x is formed in
// FP64, its FP32 rounding replaces the recursive residual, and the search
// direction is kept: beta = (r,z)_new / (r,z)_old.  A replacement whose true
// residual is more than MX_DRIFT times the recursive one (the FP32 recursion
// has lost track) restarts the direction instead (p = z).  Compared with a
// restart at every refinement, the Krylov space is not thrown away, so the
// inner iterations stay close to the FP64 CG's.
//
// Per inner iteration, three kernels (as the FP64 CG of psbx_krylov.cu):
//   p = z + beta p (z = d .* rh formed on the fly)
//   q = A p (FP32 product, two rows per thread: exact FP64 products added
//     in FP64, rounded once) and sigma = (p, q), alpha = rho / sigma
//   xh = alpha p + xh, rh = -alpha q + rh, z = d .* rh, rho' = (rh, z),
//     ||rh||^2, and the replacement test
// Every kernel returns at once when the status word is not RUN, so eight
// iterations are one CUDA graph replayed until the host sees a replacement
// request (then the replacement graph runs: fold, FP64 residual) or the end.
#include "psbx_internal.cuh"

#include <string.h>

enum { MX_RUN = 0, MX_DONE = 1, MX_REFRESH = 2, MX_BREAK = 3 };

struct MState {
  double rho, beta, alpha;
  double bn2, eps, delta;
  double rn2;    // ||rh||^2 after the last inner update
  double rmax;   // true ||r|| at the last replacement
  double rtrue;  // true ||b - A x|| at the last replacement
  int it, itmax, status, first, refreshes, restarts;
};

#define MT 256
#define MX_ITERS 8
#define MX_DRIFT 8.0

__device__ __forceinline__ bool mx_stopped(const MState *S) {
  return *((volatile const int *)&S->status) != MX_RUN;
}

// FP32 products of the row pair (s0, s0 + 1), s0 even, of a hack-32 matrix,
// both in one thread.  The two rows are adjacent in every column of their
// hack, so entry j of both is one float2 (values) and one int2 (indices):
// each load instruction of a warp moves 256 bytes, as the FP64 kernels' do,
// where one row per thread would move 128 (measured: 3.6 TB/s for one row
// per thread on the 7-point operator, against 6.25 TB/s for FP64).  Each
// row still adds its own entries in stored order, in FP64, from exact
// products, and rounds once.  Slots past a row's length (padding of the
// hack) may be loaded but are never added.
template <int U>
__device__ __forceinline__ void pair32(const HllViewF &A, int off, int n0, int n1, const float *__restrict__ x,
                                       float &y0, float &y1) {
  const float *vp = A.val + off;
  const int *jp = A.ja + off;
  const float *xb = x - A.base;
  const int n = max(n0, n1);
  double a0 = 0.0, a1 = 0.0;
  for (int j = 0; j < n; j += U) {
    int2 c[U];
    float2 v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const bool ok = j + u < n;
      c[u] = ok ? ld_stream((const int2 *)(jp + (j + u) * 32)) : make_int2(A.base, A.base);
      v[u] = ok ? ld_stream((const float2 *)(vp + (j + u) * 32)) : make_float2(0.0f, 0.0f);
    }
    float x0[U], x1[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      x0[u] = j + u < n0 ? ld_ro(xb + c[u].x) : 0.0f;
      x1[u] = j + u < n1 ? ld_ro(xb + c[u].y) : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (j + u < n0) a0 = radd(a0, rmul((double)v[u].x, (double)x0[u]));
      if (j + u < n1) a1 = radd(a1, rmul((double)v[u].y, (double)x1[u]));
    }
  }
  y0 = (float)a0;
  y1 = (float)a1;
}

__device__ __forceinline__ void exact_add(dd_t &acc, float a, float b) {
  dd_add_prod(acc, (double)a, (double)b);
}

template <int NS>
__device__ __forceinline__ void mx_publish(double *part, int grid, const dd_t (&v)[NS]) {
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NS; k++) {
      part[2 * ((size_t)k * grid + blockIdx.x)] = v[k].s;
      part[2 * ((size_t)k * grid + blockIdx.x) + 1] = v[k].c;
    }
  }
}

// ||b||_2 ; d32 = (float)dinv (1 when there is no preconditioner)
__global__ void __launch_bounds__(MT) k_mx_setup(int n, const double *__restrict__ b, const double *__restrict__ dinv,
                                                 float *__restrict__ d32, MState *S, double *__restrict__ part,
                                                 unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[64];
  dd_t s[1] = {{0.0, 0.0}};
  for (int i = blockIdx.x * MT + threadIdx.x; i < n; i += gridDim.x * MT) {
    const double v = b[i];
    dd_add_prod(s[0], v, v);
    d32[i] = dinv ? (float)dinv[i] : 1.0f;
  }
  block_sum_dd<1>(s, sm);
  mx_publish<1>(part, grid, s);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[1];
    final_sum_dd<1>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      S->bn2 = sqrt(dd_value(o[0]));
      *ticket = 0;
    }
  }
}

// x = x + xh (FP64) ; xh = 0
__global__ void __launch_bounds__(MT) k_mx_fold(int n, double *__restrict__ x, float *__restrict__ xh) {
  for (int i = blockIdx.x * MT + threadIdx.x; i < n; i += gridDim.x * MT) {
    x[i] = radd(x[i], (double)xh[i]);
    xh[i] = 0.0f;
  }
}

// Replacement: r = b - A x in FP64 ; rh = (float)r ; rho' = (rh, d.*rh) ;
// the true ||r|| decides: converged, continue with the kept direction, or
// restart the direction.
template <class View>
__global__ void __launch_bounds__(MT) k_mx_resid(View A, MState *S, const double *__restrict__ b,
                                                 const double *__restrict__ x, const float *__restrict__ d32,
                                                 float *__restrict__ rh, double *__restrict__ part,
                                                 unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[128];
  dd_t acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (int s = blockIdx.x * MT + threadIdx.x; s < A.rows; s += gridDim.x * MT) {
    const double ax = row_dot(A, s, x);
    const int i = out_row(A, s);
    const double r = radd(rmul(-1.0, ax), b[i]);
    const float rf = (float)r;
    const float zf = rmulf(ld_ro(d32 + i), rf);
    rh[i] = rf;
    exact_add(acc[0], rf, zf);
    dd_add_prod(acc[1], r, r);
  }
  block_sum_dd<2>(acc, sm);
  mx_publish<2>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[2];
    final_sum_dd<2>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      const double rhonew = dd_value(o[0]);
      const double rt = sqrt(dd_value(o[1]));
      const bool broke = S->status == MX_BREAK;
      S->rtrue = rt;
      S->refreshes += 1;
      const bool conv = S->bn2 == 0.0 ? rt <= S->eps : rt <= S->eps * S->bn2;
      if (conv || S->it >= S->itmax || rhonew == 0.0) {
        S->status = MX_DONE;
      } else {
        const bool restart = S->first || broke || S->rho == 0.0 || rt > MX_DRIFT * sqrt(S->rn2);
        if (restart) {
          if (!S->first) S->restarts += 1;
          S->first = 1;
        } else {
          S->beta = rhonew / S->rho;
        }
        S->rho = rhonew;
        S->rmax = rt;
        S->rn2 = rt * rt;
        S->status = MX_RUN;
      }
      *ticket = 0;
    }
  }
}

// The element-wise kernels take four entries per thread as one float4 per
// vector (256-byte-aligned workspace; the last n % 4 entries by the block's
// first threads one at a time).
__device__ __forceinline__ float4 ld4(const float *p, int k) { return ld_stream((const float4 *)p + k); }

// p = z (after a restart) or p = z + beta p, z = d .* rh
__device__ __forceinline__ float p_el(bool first, float beta, float d, float r, float p) {
  const float z = rmulf(d, r);
  return first ? z : raddf(z, rmulf(beta, p));
}
__global__ void __launch_bounds__(MT) k_mx_p(MState *S, int n, const float *__restrict__ d32,
                                             const float *__restrict__ rh, float *__restrict__ p) {
  if (mx_stopped(S)) return;
  const bool first = S->first != 0;
  const float beta = (float)S->beta;
  const int n4 = n >> 2;
  for (int k = blockIdx.x * MT + threadIdx.x; k < n4; k += gridDim.x * MT) {
    const float4 d = ld4(d32, k), r = ld4(rh, k), q = ((const float4 *)p)[k];
    ((float4 *)p)[k] = make_float4(p_el(first, beta, d.x, r.x, q.x), p_el(first, beta, d.y, r.y, q.y),
                                   p_el(first, beta, d.z, r.z, q.z), p_el(first, beta, d.w, r.w, q.w));
  }
  if (blockIdx.x == 0 && threadIdx.x < (n & 3)) {
    const int i = 4 * n4 + threadIdx.x;
    p[i] = p_el(first, beta, d32[i], rh[i], p[i]);
  }
}

// q = A p ; sigma = (p, q) ; alpha = rho / sigma   (hack size 32, row pairs)
// Capped at 64 registers (4 blocks of 256 per SM, no spills): uncapped, the
// prefetch of the next pair's header takes it to 80 (3 blocks per SM), and
// the 7-point 256^3 solve measured 323-331 ms that way against 289 ms capped.
template <int U>
__global__ void __launch_bounds__(MT, 4) k_mx_spmv(HllViewF A, MState *S, const float *__restrict__ p,
                                                float *__restrict__ q, double *__restrict__ part,
                                                unsigned *__restrict__ ticket, int grid) {
  __shared__ double sm[64];
  if (mx_stopped(S)) return;
  dd_t acc[1] = {{0.0, 0.0}};
  const int npair = (A.rows + 1) >> 1;
  const int step = gridDim.x * MT;
  // the next pair's row lengths and hack offset are loaded while the
  // current pair is summed (one dependent round trip less per pair)
  auto head = [&](int k, int &n0, int &n1, int &off) {
    if (k < npair) {
      const int s0 = 2 * k;
      n0 = ld_ro(A.irn + s0);
      n1 = s0 + 1 < A.rows ? ld_ro(A.irn + s0 + 1) : 0;
      off = ld_ro(A.hkoffs + (s0 >> 5)) + (s0 & 31);
    }
  };
  int k = blockIdx.x * MT + threadIdx.x;
  int n0 = 0, n1 = 0, off = 0;
  head(k, n0, n1, off);
  for (; k < npair; k += step) {
    const int s0 = 2 * k, s1 = s0 + 1;
    const bool has1 = s1 < A.rows;
    int m0 = 0, m1 = 0, moff = 0;
    head(k + step, m0, m1, moff);
    float t0, t1;
    pair32<U>(A, off, n0, n1, p, t0, t1);
    n0 = m0;
    n1 = m1;
    off = moff;
    if (A.perm) {
      const int i0 = ld_ro(A.perm + s0);
      q[i0] = t0;
      exact_add(acc[0], ld_ro(p + i0), t0);
      if (has1) {
        const int i1 = ld_ro(A.perm + s1);
        q[i1] = t1;
        exact_add(acc[0], ld_ro(p + i1), t1);
      }
    } else if (has1) {
      ((float2 *)q)[k] = make_float2(t0, t1);
      const float2 pp = ld_ro((const float2 *)p + k);
      exact_add(acc[0], pp.x, t0);
      exact_add(acc[0], pp.y, t1);
    } else {
      q[s0] = t0;
      exact_add(acc[0], ld_ro(p + s0), t0);
    }
  }
  block_sum_dd<1>(acc, sm);
  mx_publish<1>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[1];
    final_sum_dd<1>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      const double sigma = dd_value(o[0]);
      S->first = 0;
      if (sigma == 0.0) S->status = MX_BREAK;
      else S->alpha = S->rho / sigma;
      *ticket = 0;
    }
  }
}

// xh = alpha p + xh ; rh = -alpha q + rh ; rho' = (rh, d.*rh) ; ||rh||^2 ;
// replacement test
__device__ __forceinline__ void upd_el(float af, float maf, float p, float q, float d, float &xh, float &r,
                                       dd_t (&acc)[2]) {
  xh = raddf(rmulf(af, p), xh);
  r = raddf(rmulf(maf, q), r);
  const float z = rmulf(d, r);
  exact_add(acc[0], r, z);
  exact_add(acc[1], r, r);
}
__global__ void __launch_bounds__(MT) k_mx_update(MState *S, int n, const float *__restrict__ p,
                                                  const float *__restrict__ q, const float *__restrict__ d32,
                                                  float *__restrict__ xh, float *__restrict__ rh,
                                                  double *__restrict__ part, unsigned *__restrict__ ticket,
                                                  int grid) {
  __shared__ double sm[128];
  if (mx_stopped(S)) return;
  const float af = (float)S->alpha, maf = -af;
  dd_t acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  const int n4 = n >> 2;
  for (int k = blockIdx.x * MT + threadIdx.x; k < n4; k += gridDim.x * MT) {
    const float4 pp = ld4(p, k), qq = ld4(q, k), d = ld4(d32, k);
    float4 x = ((const float4 *)xh)[k], r = ((const float4 *)rh)[k];
    upd_el(af, maf, pp.x, qq.x, d.x, x.x, r.x, acc);
    upd_el(af, maf, pp.y, qq.y, d.y, x.y, r.y, acc);
    upd_el(af, maf, pp.z, qq.z, d.z, x.z, r.z, acc);
    upd_el(af, maf, pp.w, qq.w, d.w, x.w, r.w, acc);
    ((float4 *)xh)[k] = x;
    ((float4 *)rh)[k] = r;
  }
  if (blockIdx.x == 0 && threadIdx.x < (n & 3)) {
    const int i = 4 * n4 + threadIdx.x;
    float x = xh[i], r = rh[i];
    upd_el(af, maf, p[i], q[i], d32[i], x, r, acc);
    xh[i] = x;
    rh[i] = r;
  }
  block_sum_dd<2>(acc, sm);
  mx_publish<2>(part, grid, acc);
  if (psbx_last_block(ticket, gridDim.x)) {
    dd_t o[2];
    final_sum_dd<2>(part, grid, gridDim.x, o, sm);
    if (threadIdx.x == 0) {
      const double rhonew = dd_value(o[0]), rn2 = dd_value(o[1]);
      const double rn = sqrt(rn2);
      S->it += 1;
      S->rn2 = rn2;
      const double tol = S->bn2 == 0.0 ? S->eps : S->eps * S->bn2;
      if (rn <= tol || rn <= S->delta * S->rmax || S->it >= S->itmax || rhonew == 0.0) {
        S->status = MX_REFRESH;  // rho stays: the replacement forms beta from it
      } else {
        S->beta = rhonew / S->rho;
        S->rho = rhonew;
      }
      *ticket = 0;
    }
  }
}

template <class View>
static int mx_solve(const View &A64, const HllViewF &A32, bool shortRows, const double *dinv, const double *b,
                    double *x, int n, psbx_SolverOptions *opt, double delta, int *refreshes) {
  PsbxCtx &c = psbx_ctx();
  cudaStream_t st = c.stream;
  int grid = (n + MT - 1) / MT;
  if (grid > c.sms * 8) grid = c.sms * 8;
  if (grid < 1) grid = 1;
  const size_t nn = ((size_t)(n > 0 ? n : 1) + 63) / 64 * 64;  // 256-byte aligned vectors
  float *vec = nullptr;
  double *part = nullptr;
  MState *S = nullptr;
  unsigned *ticket = nullptr;
  PSBX_CK(psbx_malloc_async(&vec, sizeof(float) * 5 * nn, st));
  PSBX_CK(psbx_malloc_async(&part, sizeof(double) * 4 * (size_t)grid, st));
  PSBX_CK(psbx_malloc_async(&S, sizeof(MState), st));
  PSBX_CK(psbx_malloc_async(&ticket, sizeof(unsigned), st));
  PSBX_CK(cudaMemsetAsync(ticket, 0, sizeof(unsigned), st));
  PSBX_CK(cudaMemsetAsync(vec, 0, sizeof(float) * 5 * nn, st));
  float *rh = vec, *xh = vec + nn, *p = vec + 2 * nn, *q = vec + 3 * nn, *d32 = vec + 4 * nn;
  MState *hS = (MState *)c.h_res;
  MState init;
  memset(&init, 0, sizeof(init));
  init.eps = opt->eps;
  init.delta = delta;
  init.itmax = opt->itmax;
  init.first = 1;
  init.status = MX_RUN;
  PSBX_CK(cudaMemcpyAsync(S, &init, sizeof(MState), cudaMemcpyHostToDevice, st));
  k_mx_setup<<<grid, MT, 0, st>>>(n, b, dinv, d32, S, part, ticket, grid);
  PSBX_LAUNCH_CK("k_mx_setup");

  int rc = SPGPU_SUCCESS;
  cudaGraph_t gi = nullptr, gr = nullptr;
  cudaGraphExec_t ei = nullptr, er = nullptr;
  const int wide = A64.nLong > 0 ? 2 : 0;
  auto capture = [&](cudaGraph_t *g, cudaGraphExec_t *e, auto body) -> int {
    cudaError_t ce = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) return psbx_cuda_status(ce, "BeginCapture");
    body();
    ce = cudaStreamEndCapture(st, g);
    if (ce != cudaSuccess) return psbx_cuda_status(ce, "EndCapture");
    ce = cudaGraphInstantiate(e, *g, 0);
    if (ce != cudaSuccess) return psbx_cuda_status(ce, "GraphInstantiate");
    return SPGPU_SUCCESS;
  };
  // grids: the element-wise kernels take 4 entries per thread, the product
  // 2 rows per thread
  int gq = (n / 4 + MT - 1) / MT, gs = ((n + 1) / 2 + MT - 1) / MT;
  gq = gq < 1 ? 1 : (gq > grid ? grid : gq);
  gs = gs < 1 ? 1 : (gs > grid ? grid : gs);
  rc = capture(&gi, &ei, [&]() {
    for (int k = 0; k < MX_ITERS; k++) {
      k_mx_p<<<gq, MT, 0, st>>>(S, n, d32, rh, p);
      if (shortRows) k_mx_spmv<8><<<gs, MT, 0, st>>>(A32, S, p, q, part, ticket, gs);
      else k_mx_spmv<4><<<gs, MT, 0, st>>>(A32, S, p, q, part, ticket, gs);
      k_mx_update<<<gq, MT, 0, st>>>(S, n, p, q, d32, xh, rh, part, ticket, gq);
    }
  });
  if (!rc) rc = capture(&gr, &er, [&]() {
    k_mx_fold<<<grid, MT, 0, st>>>(n, x, xh);
    psbx_long_rows(A64, x, nullptr, st);
    k_mx_resid<View><<<grid, MT, 0, st>>>(A64, S, b, x, d32, rh, part, ticket, grid);
  });
  auto fetch = [&]() -> int {
    PSBX_CK(cudaMemcpyAsync(hS, S, sizeof(MState), cudaMemcpyDeviceToHost, st));
    PSBX_CK(cudaStreamSynchronize(st));
    return SPGPU_SUCCESS;
  };
  auto launch = [&](cudaGraphExec_t e, int kernels) -> int {
    cudaError_t ce = cudaGraphLaunch(e, st);
    if (ce != cudaSuccess) return psbx_cuda_status(ce, "GraphLaunch");
    psbx_count_launch(kernels);
    return SPGPU_SUCCESS;
  };
  if (!rc) rc = launch(er, 2 + wide);
  if (!rc) rc = fetch();
  while (!rc && hS->status != MX_DONE) {
    if (hS->status == MX_RUN) {
      // 1, 2, 4, then 8 replays between two reads of the state
      for (int batch = 1; !rc; batch = batch < 8 ? 2 * batch : 8) {
        for (int k = 0; k < batch && !rc; k++) rc = launch(ei, 3 * MX_ITERS);
        if (!rc) rc = fetch();
        if (rc || hS->status != MX_RUN) break;
      }
    }
    if (rc) break;
    if (hS->status == MX_REFRESH || hS->status == MX_BREAK) {
      if ((rc = launch(er, 2 + wide))) break;
      rc = fetch();
    }
  }
  if (!rc) {
    opt->iter = hS->it;
    opt->err = hS->bn2 == 0.0 ? hS->rtrue : hS->rtrue / hS->bn2;
    if (refreshes) *refreshes = hS->refreshes;
  }
  if (ei) cudaGraphExecDestroy(ei);
  if (er) cudaGraphExecDestroy(er);
  if (gi) cudaGraphDestroy(gi);
  if (gr) cudaGraphDestroy(gr);
  cudaFreeAsync(vec, st);
  cudaFreeAsync(part, st);
  cudaFreeAsync(S, st);
  cudaFreeAsync(ticket, st);
  cudaError_t e2 = cudaStreamSynchronize(st);
  if (!rc && e2 != cudaSuccess) rc = psbx_cuda_status(e2, "psbx_dmixed_cg");
  return rc;
}

extern "C" int psbx_dmixed_cg(void *mat, void *dinv, void *b, void *x, psbx_SolverOptions *opt, double delta,
                              int *refreshes) {
  HllDevice *m = (HllDevice *)mat;
  MultiVectDevice *B = (MultiVectDevice *)b, *X = (MultiVectDevice *)x, *D = (MultiVectDevice *)dinv;
  if (!m || !B || !X || !opt || m->elemType != SPGPU_TYPE_DOUBLE || m->hackSize != 32) return SPGPU_UNSUPPORTED;
  const int n = m->rows;
  if (B->size_ < n || X->size_ < n || (D && D->size_ < n) || B->elemType != SPGPU_TYPE_DOUBLE ||
      X->elemType != SPGPU_TYPE_DOUBLE || (D && D->elemType != SPGPU_TYPE_DOUBLE))
    return SPGPU_UNSUPPORTED;
  if (opt->istop != 2 || !(delta > 0.0 && delta < 1.0)) return SPGPU_UNSUPPORTED;
  if (opt->itmax <= 0) {
    opt->iter = 0;
    opt->err = 0.0;
    return SPGPU_SUCCESS;
  }
  if (!m->cM32) {
    int rc = psbx_hll_make_single(m);
    if (rc) return rc;
  }
  HllViewF A32;
  A32.val = m->cM32;
  A32.ja = m->rP;
  A32.irn = m->rS;
  A32.hkoffs = m->hackOffs;
  A32.perm = m->perm;
  A32.rows = m->rows;
  A32.hksz = 32;
  A32.base = m->baseIndex;
  const HllView v = hll_view(m);
  const double *dv = D ? (const double *)D->v_ : nullptr;
  const double *bp = (const double *)B->v_;
  double *xp = (double *)X->v_;
  // the FP32 product reads a row pair's entries in groups of 8 when no row
  // is longer than PSBX_SHORT_ROW (one group for the 7-point rows), else 4
  const bool shortRows = m->maxRowLen >= 0 && m->maxRowLen <= PSBX_SHORT_ROW;
  if (v.nLong > 0) return mx_solve(hll32w_view(v), A32, shortRows, dv, bp, xp, n, opt, delta, refreshes);
  if (hll_short_rows(m)) return mx_solve(hll32s_view(v), A32, true, dv, bp, xp, n, opt, delta, refreshes);
  return mx_solve(hll32_view(v), A32, shortRows, dv, bp, xp, n, opt, delta, refreshes);
}
