// psbx_batch.cu -- batched, mixed-precision CG engine: many independent SPD
// systems (each with K right-hand sides) solved together by one persistent
// grid, FP32 inner CG iterations with FP64-accumulated dot products inside
// an FP64 iterative-refinement loop, per-system convergence masks, CUDA-graph
// replays, and systems that join and leave between replays (the serving
// loop's continuous batching).
//
// Method per right-hand side (CG of krylov/psb_dcg.F90:218-295 with the
// diagonal preconditioner of prec/impl/psb_d_diagprec_impl.f90, used as the
// inner solver of iterative refinement):
//   r = b - A x                               (FP64 values, FP64 SpMV)
//   stop when ||r||_2 <= eps ||b||_2          (istop 2, FP64)
//   solve A d = r/||r|| by Jacobi-CG in FP32 until ||r_in||_2 <= tau,
//     tau = max(inner_tol, eps ||b|| / (2 ||r||)); values FP32, vectors
//     FP32, every dot product accumulated in FP64 (products of two FP32
//     numbers are exact in FP64)
//   x = x + ||r|| d                           (FP64)
// and the next inner loop keeps the search direction (residual replacement:
// the FP64 residual, rescaled, replaces the recursive one; p carries over
// with beta = rho_new / (rho_old * ratio), ratio = old scale / new scale, as
// the direction is in units of the old scale).  The direction restarts
// (p = z) on the first inner loop, after an inner breakdown, and when the
// true residual is more than DRIFT times the recursive one.  Compared with
// restarting every inner loop, the Krylov space is kept, and the inner
// iterations stay close to an FP64 CG's.
//
// Layout: each system is an HLL-32 matrix (FP64 values, FP32 copy, shared
// indices) with 1-based local columns, and K interleaved vectors
// v[row*K + j].  Work is cut in tiles of rows of one system (tile_plan);
// block b takes tiles b, b + grid, b + 2 grid, ... so the blocks in flight
// work on a window of consecutive tiles (whose gathered vectors share L2).  A tile's partial sums go to
// part[tile]; the block that completes the last tile of a system (per-system
// ticket) adds that system's partials in tile order -- fixed order, so the
// result does not depend on scheduling -- and advances the system's phase.
// Every kernel only touches systems in its own phase; a graph of ITERS x 6
// kernels is replayed and the host looks at the phases once per replay.
#include "psbx_internal.cuh"

#include <stdlib.h>
#include <string.h>
#include <vector>

namespace {

enum Phase { PH_IDLE = 0, PH_RESID = 1, PH_INIT = 2, PH_INNER = 3, PH_XUPD = 4, PH_DONE = 5 };
enum { BT = 256, ITERS = 8, MAXK = 8, LONG_ROW = 64 };
// Thread-per-row tile bounds (rows, stored entries): one right-hand side
// runs fastest with 4096 / 32K (7-point 111^3: 17.8 ms per solve against
// 19.7 with 2048 / 16K), eight with 2048 / 16K (their SpMV carries 8 sums
// per row: 534 against 635 us per launch on C4).
__host__ __device__ constexpr int tile_rows(int K) { return K == 1 ? 4096 : 2048; }
__host__ __device__ constexpr int tile_nnz(int K) { return K == 1 ? 32768 : 16384; }

struct BSys {                 // read-only for the kernels
  const double *val64;
  const float *val32;
  const int *ja, *irn, *hkoffs;
  const double *b;
  double *x, *r64;
  void *r32, *z, *p, *q, *d;  // inner vectors, of the engine's inner type (float, or double)
  const void *dinv;           // inverse diagonal, inner type
  int rows, sol0, tile0, ntiles;
};

// The inner iterations' values: the FP32 copy, or the FP64 values for an
// engine whose inner iterations run in FP64 (the batched FP64 comparison).
template <class TI> __device__ __forceinline__ const TI *inner_val(const BSys &S);
template <> __device__ __forceinline__ const float *inner_val<float>(const BSys &S) { return S.val32; }
template <> __device__ __forceinline__ const double *inner_val<double>(const BSys &S) { return S.val64; }

struct BState {               // written by the kernels
  int phase;
  unsigned ticket;
  int outer;
  int done_flag;
};

struct BSol {                 // one right-hand side
  double rho, sigma, alpha, beta;
  double bn2, rn, scale, tau, eps, inner_tol;
  double ratio;               // scale before the last refinement / scale after it
  double rrec;                // recursive residual (true units) when the inner loop stopped
  int it, it_total, itmax, outer_max;
  int active;                 // inner CG running for this rhs
  int done;                   // 0 running, 1 converged, 2 stopped (itmax / breakdown)
  int first;                  // bn2 not yet computed
  int restart;                // the next inner loop starts a new direction (p = z)
  int loop_it, loop_cap;      // iterations of the current inner loop, and its bound
};
// A refinement whose true residual is more than DRIFT times the inner loop's
// recursive one, or more than half the previous refinement's, restarts the
// search direction instead of keeping it.  An
// inner loop that continues a direction also stops after 4 times the
// iterations of the loop before it plus LOOP_SLACK: an FP32 recursion that
// has lost accuracy may never reach its reduction (measured: with
// inner_tol 1e-4, 14 of 128 anisotropic systems ran to itmax), and the
// refinement that follows restarts it.
#define DRIFT 8.0
#define LOOP_SLACK 64

struct BTile {
  int sys, row0, nrows, kind;  // kind 1: up to 8 long rows (tile_spmv)
};

struct BCtl {                 // read by every kernel at launch; lets the tile
  int ntiles, cap;            // table grow without re-capturing the graph
  const BTile *tiles;
  double *part;               // cap * 2*MAXK partial sums
  int *count;                 // systems in each phase (kept by the kernels)
};

struct Eng {
  int K = 1, max_sys = 0, max_tiles = 0, grid = 0;
  int fp64 = 0;               // inner iterations in FP64 (the batched FP64 comparison) instead of FP32
  BSys *d_sys = nullptr;
  BState *d_state = nullptr;
  BSol *d_sol = nullptr;
  BTile *d_tiles = nullptr;
  BCtl *d_ctl = nullptr;
  int *d_count = nullptr;     // [8] systems per phase
  double *d_part = nullptr;   // max_tiles * K * 2
  std::vector<BSys> h_sys;
  std::vector<BState> h_state;
  std::vector<int> used;      // slot in use
  std::vector<void *> owned;  // per slot: one allocation holding its vectors
  std::vector<std::vector<int>> plan;  // per slot: its matrix's tile plan
  cudaGraphExec_t gexec = nullptr;
  cudaGraph_t graph = nullptr;
  BState *h_state_pinned = nullptr;
  BSol *h_sol_pinned = nullptr;
  bool dirty = false;         // slots joined or left since the tile table was uploaded
  cudaEvent_t done_ev = nullptr;  // end of the last launch's state readback
  bool inflight = false;
  // pinned staging of the tables (no wait for the copies: the next upload
  // comes after a wait, which orders it after them)
  BTile *h_tiles_pinned = nullptr;
  int h_tiles_cap = 0;
  BSys *h_sys_pinned = nullptr;
  BCtl *h_ctl_pinned = nullptr;
  BSol *h_sol_init = nullptr;  // pinned, per slot: the initial BSol of an add
};

// --------------------------------------------------------------- helpers
// Occupancy targets (blocks of BT threads per SM).  The K = 1 kernels are
// latency-bound streams over short rows: the SpMV and the short vector
// kernels want every warp slot (8 blocks, <= 32 registers); the update keeps
// 4 rows of loads in flight per thread instead (4 blocks, no spills), which
// measured faster than 1 row per thread at 8 blocks.  The 8-rhs kernels carry
// 8 accumulators per row; their SpMV runs 4 blocks per SM even though that
// spills a few registers: on the 512 anisotropic systems 534 us, against
// 672 us at 2 blocks, 712 us at 3, 655 us at 3 blocks with 4 entries per
// load group, and 750-850 us when the 8 sums are formed as two halves of 4.
template <int K> struct Occ {
  static constexpr int blocks = K == 1 ? 8 : 2;
  static constexpr int spmv_blocks = K == 1 ? 8 : 4;
  static constexpr int update_blocks = K == 1 ? 4 : 2;
  static constexpr int resid_blocks = K == 1 ? 4 : 2;
};


// A kernel whose phase no system is in returns after one load (instead of
// walking the tile table); the finalisers move systems between phases and
// keep the counts.
// (one read by thread 0, shared with the block, so the block decides as one)
__device__ __forceinline__ bool phase_idle(const BCtl *ctl, int ph) {
  __shared__ int idle;
  if (threadIdx.x == 0) idle = *((volatile const int *)ctl->count + ph) == 0;
  __syncthreads();
  return idle;
}

__device__ __forceinline__ void move_phase(const BCtl *ctl, BState *st, int to) {
  atomicSub(ctl->count + st->phase, 1);
  atomicAdd(ctl->count + to, 1);
  st->phase = to;
}

struct RowRef {               // start of an HLL-32 row and its length
  int off, n;
};

__device__ __forceinline__ RowRef row_ref(const int *__restrict__ hkoffs, const int *__restrict__ irn, int r) {
  RowRef rr;
  rr.off = __ldg(hkoffs + (r >> 5)) + (r & 31);
  rr.n = __ldg(irn + r);
  return rr;
}

// The K values of one row of an interleaved vector (v[row*K + k]).  Rows of
// 8 values are 32-byte aligned (vector bases are 16-byte aligned), so they
// move as float4 / double2.
template <int K>
__device__ __forceinline__ void ld_row(const float *p, float (&v)[K]) {
  if constexpr (K % 4 == 0) {
#pragma unroll
    for (int q = 0; q < K / 4; q++) {
      const float4 t = reinterpret_cast<const float4 *>(p)[q];
      v[4 * q] = t.x, v[4 * q + 1] = t.y, v[4 * q + 2] = t.z, v[4 * q + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = p[k];
  }
}

template <int K>
__device__ __forceinline__ void ld_row_ro(const float *__restrict__ p, float (&v)[K]) {
  if constexpr (K % 4 == 0) {
#pragma unroll
    for (int q = 0; q < K / 4; q++) {
      const float4 t = __ldg(reinterpret_cast<const float4 *>(p) + q);
      v[4 * q] = t.x, v[4 * q + 1] = t.y, v[4 * q + 2] = t.z, v[4 * q + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = __ldg(p + k);
  }
}

template <int K>
__device__ __forceinline__ void st_row(float *p, const float (&v)[K]) {
  if constexpr (K % 4 == 0) {
#pragma unroll
    for (int q = 0; q < K / 4; q++)
      reinterpret_cast<float4 *>(p)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  } else {
#pragma unroll
    for (int k = 0; k < K; k++) p[k] = v[k];
  }
}

template <int K>
__device__ __forceinline__ void ld_row(const double *p, double (&v)[K]) {
  if constexpr (K % 2 == 0) {
#pragma unroll
    for (int q = 0; q < K / 2; q++) {
      const double2 t = reinterpret_cast<const double2 *>(p)[q];
      v[2 * q] = t.x, v[2 * q + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = p[k];
  }
}

template <int K>
__device__ __forceinline__ void ld_row_ro(const double *__restrict__ p, double (&v)[K]) {
  if constexpr (K % 2 == 0) {
#pragma unroll
    for (int q = 0; q < K / 2; q++) {
      const double2 t = __ldg(reinterpret_cast<const double2 *>(p) + q);
      v[2 * q] = t.x, v[2 * q + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = __ldg(p + k);
  }
}

template <int K>
__device__ __forceinline__ void st_row(double *p, const double (&v)[K]) {
  if constexpr (K % 2 == 0) {
#pragma unroll
    for (int q = 0; q < K / 2; q++) reinterpret_cast<double2 *>(p)[q] = make_double2(v[2 * q], v[2 * q + 1]);
  } else {
#pragma unroll
    for (int k = 0; k < K; k++) p[k] = v[k];
  }
}

// Row sums of one HLL-32 row for K interleaved vectors, entries in order.
template <class VT, class XT, int K>
__device__ __forceinline__ void row_multi(const VT *__restrict__ val, const int *__restrict__ ja, RowRef rr,
                                          const XT *__restrict__ x, double (&acc)[K]) {
  const VT *vp = val + rr.off;
  const int *jp = ja + rr.off;
  const int n = rr.n;
#pragma unroll
  for (int k = 0; k < K; k++) acc[k] = 0.0;
  constexpr int U = K == 1 ? 8 : 2;
  int j = 0;
  for (; j + U <= n; j += U) {
    int c[U];
    VT v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      c[u] = ld_stream(jp + (j + u) * 32) - 1;
      v[u] = ld_stream(vp + (j + u) * 32);
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      XT xv[K];
      ld_row_ro<K>(x + (size_t)c[u] * K, xv);
#pragma unroll
      for (int k = 0; k < K; k++) acc[k] = radd(acc[k], rmul((double)v[u], (double)xv[k]));
    }
  }
  if (j < n) {  // the tail as one predicated group: its loads overlap
    int c[U];
    VT v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const bool ok = j + u < n;
      c[u] = ok ? ld_stream(jp + (j + u) * 32) - 1 : 0;
      v[u] = ok ? ld_stream(vp + (j + u) * 32) : VT(0);
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (j + u < n) {
        XT xv[K];
        ld_row_ro<K>(x + (size_t)c[u] * K, xv);
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] = radd(acc[k], rmul((double)v[u], (double)xv[k]));
      }
    }
  }
}

// The rows of a long-row tile (up to 8 consecutive rows longer than
// LONG_ROW) summed by the whole block: thread t takes row t % 8 and its
// entries t/8, t/8 + 32, ... in order, W per round with their loads issued
// before the gathers, so one warp load reads entry j of 8 neighbouring rows
// -- 32 contiguous bytes of the hack's column-major layout -- for 4 columns
// (a warp on one row would touch a different 32-byte sector per lane).  The
// 32 partial sums of a row are added in column-phase order; thread i < nrows
// returns row i's sums.  Every thread of the block must call it.
static_assert(BT / 32 == 8, "a long-row tile holds BT/32 = 8 rows");
template <class VT, class XT, int K>
__device__ __forceinline__ bool rows_by_block(const BSys &S, const BTile &T, const VT *__restrict__ val,
                                              const XT *__restrict__ x, double (&out)[K]) {
  __shared__ double red[K * BT];
  const int i = threadIdx.x & 7, c0 = threadIdx.x >> 3;
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; k++) acc[k] = 0.0;
  if (i < T.nrows) {
    const RowRef rr = row_ref(S.hkoffs, S.irn, T.row0 + i);
    constexpr int W = K == 1 ? 8 : 2;
    for (int j0 = c0; j0 < rr.n; j0 += 32 * W) {
      int c[W];
      double v[W];
#pragma unroll
      for (int u = 0; u < W; u++) {
        const int j = j0 + 32 * u;
        const bool ok = j < rr.n;
        c[u] = ok ? ld_stream(S.ja + rr.off + j * 32) - 1 : 0;
        v[u] = ok ? (double)ld_stream(val + rr.off + j * 32) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < W; u++) {
        if (j0 + 32 * u < rr.n) {
          XT xv[K];
          ld_row_ro<K>(x + (size_t)c[u] * K, xv);
#pragma unroll
          for (int k = 0; k < K; k++) acc[k] = radd(acc[k], rmul(v[u], (double)xv[k]));
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < K; k++) red[k * BT + threadIdx.x] = acc[k];
  __syncthreads();
  const bool mine = threadIdx.x < T.nrows;
  if (mine) {
#pragma unroll
    for (int k = 0; k < K; k++) {
      double t = 0.0;
      for (int c = 0; c < BT / 8; c++) t = radd(t, red[k * BT + c * 8 + threadIdx.x]);
      out[k] = t;
    }
  }
  __syncthreads();  // red is reused by the next tile
  return mine;
}

// One long row summed by a whole warp (the 8-right-hand-side kernels, where
// the block-wide sums below cost registers): lane l takes entries l, l+32,
// ...; a fixed shuffle tree combines them; the result is valid in every lane.
template <class VT, class XT, int K>
__device__ __forceinline__ void row_multi_warp(const VT *__restrict__ val, const int *__restrict__ ja, RowRef rr,
                                               const XT *__restrict__ x, double (&acc)[K]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < K; k++) acc[k] = 0.0;
  // a lane's entries lane, lane+32, ... in order, W of them per round with
  // all their loads issued before the gathers
  constexpr int W = K == 1 ? 8 : 2;
  for (int j0 = lane; j0 < rr.n; j0 += 32 * W) {
    int c[W];
    double v[W];
#pragma unroll
    for (int u = 0; u < W; u++) {
      const int j = j0 + 32 * u;
      const bool ok = j < rr.n;
      c[u] = ok ? ld_stream(ja + rr.off + j * 32) - 1 : 0;
      v[u] = ok ? (double)ld_stream(val + rr.off + j * 32) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < W; u++) {
      if (j0 + 32 * u < rr.n) {
        XT xv[K];
        ld_row_ro<K>(x + (size_t)c[u] * K, xv);
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] = radd(acc[k], rmul(v[u], (double)xv[k]));
      }
    }
  }
#pragma unroll
  for (int k = 0; k < K; k++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] = radd(acc[k], __shfl_xor_sync(0xffffffffu, acc[k], o));
}

// Applies f(row, sums) to every row of a tile: thread-per-row tiles (kind 0)
// walk rows threadIdx.x, +BT, ... with the next row's offset and length
// loaded while the current row is summed; the rows of a long-row tile
// (kind 1) are summed by the whole block and f is called by thread i for row
// i (one right-hand side), or by a warp per row, f in lane 0 (8 of them).
template <class VT, class XT, int K, class F>
__device__ __forceinline__ void tile_spmv(const BSys &S, const BTile &T, const VT *__restrict__ val,
                                          const XT *__restrict__ x, F &&f) {
  if (T.kind == 1) {
    if constexpr (K == 1) {
      double a[K];
      if (rows_by_block<VT, XT, K>(S, T, val, x, a)) f(T.row0 + threadIdx.x, a);
    } else {
      for (int i = threadIdx.x >> 5; i < T.nrows; i += BT / 32) {
        const int r = T.row0 + i;
        double a[K];
        row_multi_warp<VT, XT, K>(val, S.ja, row_ref(S.hkoffs, S.irn, r), x, a);
        if ((threadIdx.x & 31) == 0) f(r, a);
      }
    }
    return;
  }
  int i = threadIdx.x;
  RowRef cur = {0, 0};
  if (i < T.nrows) cur = row_ref(S.hkoffs, S.irn, T.row0 + i);
  for (; i < T.nrows; i += BT) {
    RowRef nxt = {0, 0};
    if (i + BT < T.nrows) nxt = row_ref(S.hkoffs, S.irn, T.row0 + i + BT);
    double a[K];
    row_multi<VT, XT, K>(val, S.ja, cur, x, a);
    f(T.row0 + i, a);
    cur = nxt;
  }
}

// Block-reduce NS sums per rhs (K of each), publish the tile's partials,
// take the system's ticket; returns true in the block that finalises.
template <int K, int NS>
__device__ __forceinline__ bool tile_publish(double (&v)[NS][K], double *part, int tile, BState *st, int ntiles,
                                             double *smem /* >= 32*NS*K */) {
#pragma unroll
  for (int m = 0; m < NS; m++) {
#pragma unroll
    for (int k = 0; k < K; k++) {
      double t = v[m][k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t = radd(t, __shfl_down_sync(0xffffffffu, t, o));
      v[m][k] = t;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int m = 0; m < NS; m++)
#pragma unroll
      for (int k = 0; k < K; k++) smem[(m * K + k) * 32 + warp] = v[m][k];
  }
  __syncthreads();
  if (threadIdx.x < NS * K) {
    double s = 0.0;
    for (int w = 0; w < BT / 32; w++) s = radd(s, smem[threadIdx.x * 32 + w]);
    part[(size_t)tile * (2 * MAXK) + threadIdx.x] = s;
  }
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&st->ticket, 1u) == (unsigned)(ntiles - 1);
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// Totals of the system's tile partials for NV values (all threads of the
// finalising block): thread t adds tiles t, t+BT, ... in order, then a fixed
// shuffle tree and the warps in order.  The order depends only on the
// system's tile count, so a system's result does not depend on its company.
// Results in tot[0..NV).
template <int NV>
__device__ __forceinline__ void sys_totals(const double *part, int tile0, int ntiles, double *tot,
                                           double *scratch /* 32*NV */) {
  double v[NV];
#pragma unroll
  for (int m = 0; m < NV; m++) v[m] = 0.0;
  for (int t = threadIdx.x; t < ntiles; t += BT) {
    const double *pt = part + (size_t)(tile0 + t) * (2 * MAXK);
#pragma unroll
    for (int m = 0; m < NV; m++) v[m] = radd(v[m], __ldcg(pt + m));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < NV; m++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[m] = radd(v[m], __shfl_down_sync(0xffffffffu, v[m], o));
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int m = 0; m < NV; m++) scratch[m * 32 + warp] = v[m];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < BT / 32; w++) s = radd(s, scratch[threadIdx.x * 32 + w]);
    tot[threadIdx.x] = s;
  }
  __syncthreads();
}

// --------------------------------------------------------------- kernels
// PH_RESID: r = b - A x (FP64), ||r||^2 and (first time) ||b||^2 per rhs;
// stop test; next phase PH_INIT or PH_DONE.
template <int K>
__global__ void __launch_bounds__(BT, Occ<K>::resid_blocks) kb_resid(const BSys *__restrict__ sys, BState *state,
                                                                     BSol *sol, const BCtl *ctl) {
  __shared__ double sm[32 * 2 * MAXK];
  if (phase_idle(ctl, PH_RESID)) return;
  const BTile *__restrict__ tiles = ctl->tiles;
  double *part = ctl->part;
  const int ntiles = ctl->ntiles;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile T = tiles[t];
    BState *st = state + T.sys;
    if (st->phase != PH_RESID) continue;
    const BSys &S = sys[T.sys];
    double v[2][K];
#pragma unroll
    for (int k = 0; k < K; k++) v[0][k] = v[1][k] = 0.0;
    const double *__restrict__ b = S.b;
    double *__restrict__ r64 = S.r64;
    tile_spmv<double, double, K>(S, T, S.val64, S.x, [&](int r, const double (&ax)[K]) {
      double bb[K], rr[K];
      ld_row<K>(b + (size_t)r * K, bb);
#pragma unroll
      for (int k = 0; k < K; k++) {
        rr[k] = radd(bb[k], -ax[k]);
        v[0][k] = radd(v[0][k], rmul(rr[k], rr[k]));
        v[1][k] = radd(v[1][k], rmul(bb[k], bb[k]));
      }
      st_row<K>(r64 + (size_t)r * K, rr);
    });
    if (tile_publish<K, 2>(v, part, t, st, S.ntiles, sm)) {
      __shared__ double tot[2 * K];
      sys_totals<2 * K>(part, S.tile0, S.ntiles, tot, sm);
      if (threadIdx.x < K) {
        const int k = threadIdx.x;
        BSol *so = sol + S.sol0 + k;
        const double rr = tot[k];
        if (so->first) {
          so->bn2 = sqrt(tot[K + k]);
          so->first = 0;
        }
        if (so->done == 0) {
          so->rn = sqrt(rr);
          const double err = so->bn2 == 0.0 ? so->rn : so->rn / so->bn2;
          if (err <= so->eps) {
            so->done = 1;
          } else if (so->it_total >= so->itmax || st->outer >= so->outer_max) {
            so->done = 2;
          } else {
            if (so->scale > 0.0 && so->rn > 0.0) so->ratio = so->scale / so->rn;
            // restart the direction when the recursion has drifted from the
            // true residual, or when the last inner loop did not even halve
            // the true residual
            if (!(so->rn <= DRIFT * so->rrec) || !(so->rn <= 0.5 * so->scale)) so->restart = 1;
            so->scale = so->rn;
            so->tau = fmax(so->inner_tol, 0.5 * so->eps * (so->bn2 == 0.0 ? 1.0 : so->bn2) / so->rn);
          }
        }
        so->active = 0;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int all = 1;
        for (int k = 0; k < K; k++) all &= sol[S.sol0 + k].done != 0;
        move_phase(ctl, st, all ? PH_DONE : PH_INIT);
        st->done_flag = all;
        st->ticket = 0;
      }
    }
  }
}

// PH_INIT: r32 = r/scale, z = D r32, d = 0; rho = (r32, z).
template <int K, class TI>
__global__ void __launch_bounds__(BT, Occ<K>::blocks) kb_init(const BSys *__restrict__ sys, BState *state,
                                                              BSol *sol, const BCtl *ctl) {
  constexpr int RB = K == 1 ? 2 : 1;  // rows per thread whose loads are in flight together
  __shared__ double sm[32 * 2 * MAXK];
  if (phase_idle(ctl, PH_INIT)) return;
  const BTile *__restrict__ tiles = ctl->tiles;
  double *part = ctl->part;
  const int ntiles = ctl->ntiles;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile T = tiles[t];
    BState *st = state + T.sys;
    if (st->phase != PH_INIT) continue;
    const BSys &S = sys[T.sys];
    double inv[K];
    bool live[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      const BSol *so = sol + S.sol0 + k;
      live[k] = so->done == 0;
      inv[k] = live[k] ? 1.0 / so->scale : 0.0;
    }
    const double *__restrict__ r64 = S.r64;
    const TI *__restrict__ dinv = (const TI *)S.dinv;
    TI *__restrict__ r32 = (TI *)S.r32;
    TI *__restrict__ z = (TI *)S.z;
    TI *__restrict__ d = (TI *)S.d;
    double v[1][K];
#pragma unroll
    for (int k = 0; k < K; k++) v[0][k] = 0.0;
    for (int i0 = threadIdx.x; i0 < T.nrows; i0 += RB * BT) {
      double rv64[RB][K];
      TI dg[RB];
#pragma unroll
      for (int u = 0; u < RB; u++) {
        const int i = i0 + u * BT;
        const size_t r = (size_t)T.row0 + i;
        if (i < T.nrows) {
          dg[u] = dinv[r];
          ld_row<K>(r64 + r * K, rv64[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < RB; u++) {
        const int i = i0 + u * BT;
        if (i >= T.nrows) continue;
        const size_t r = (size_t)T.row0 + i;
        TI rv[K], zv[K], dz[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
          rv[k] = live[k] ? (TI)rmul(rv64[u][k], inv[k]) : TI(0);
          zv[k] = rmul(dg[u], rv[k]);
          dz[k] = TI(0);
          v[0][k] = radd(v[0][k], rmul((double)rv[k], (double)zv[k]));
        }
        st_row<K>(r32 + r * K, rv);
        st_row<K>(z + r * K, zv);
        st_row<K>(d + r * K, dz);
      }
    }
    if (tile_publish<K, 1>(v, part, t, st, S.ntiles, sm)) {
      __shared__ double tot[K];
      sys_totals<K>(part, S.tile0, S.ntiles, tot, sm);
      if (threadIdx.x < K) {
        BSol *so = sol + S.sol0 + threadIdx.x;
        if (so->done == 0) {
          const double rho = tot[threadIdx.x];
          if (so->restart || !(so->rho > 0.0) || !(so->ratio > 0.0)) {
            so->it = 1;  // p = z
            so->loop_cap = 0x7fffffff;
          } else {
            so->beta = rho / (so->rho * so->ratio);
            so->it = 2;  // p = z + beta p
            so->loop_cap = 4 * so->loop_it + LOOP_SLACK;
          }
          so->loop_it = 0;
          so->restart = 0;
          so->rho = rho;
          so->active = so->rho > 0.0 ? 1 : 0;
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        move_phase(ctl, st, PH_INNER);
        st->outer += 1;
        st->ticket = 0;
      }
    }
  }
}

// PH_INNER: p = z (it == 1) or p = z + beta p, for active rhs.
template <int K, class TI>
__global__ void __launch_bounds__(BT, Occ<K>::blocks) kb_p(const BSys *__restrict__ sys, const BState *state,
                                                           const BSol *sol, const BCtl *ctl) {
  constexpr int RB = K == 1 ? 4 : 1;
  if (phase_idle(ctl, PH_INNER)) return;
  const BTile *__restrict__ tiles = ctl->tiles;
  const int ntiles = ctl->ntiles;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile T = tiles[t];
    if (state[T.sys].phase != PH_INNER) continue;
    const BSys &S = sys[T.sys];
    TI beta[K];
    bool act[K], first[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      const BSol *so = sol + S.sol0 + k;
      act[k] = so->active;
      first[k] = so->it == 1;
      beta[k] = (TI)so->beta;
    }
    const TI *__restrict__ z = (const TI *)S.z;
    TI *__restrict__ p = (TI *)S.p;
    // p of a stopped rhs keeps its value; it is read only when some rhs
    // is past its first inner iteration or stopped
    bool any_act = false, need_p = false;
#pragma unroll
    for (int k = 0; k < K; k++) {
      any_act |= act[k];
      need_p |= !act[k] || !first[k];
    }
    if (!any_act) continue;
    for (int i0 = threadIdx.x; i0 < T.nrows; i0 += RB * BT) {
      TI zv[RB][K], pv[RB][K];
#pragma unroll
      for (int u = 0; u < RB; u++) {
        const int i = i0 + u * BT;
        const size_t o = ((size_t)T.row0 + i) * K;
#pragma unroll
        for (int k = 0; k < K; k++) pv[u][k] = TI(0);
        if (i < T.nrows) {
          ld_row<K>(z + o, zv[u]);
          if (need_p) ld_row<K>(p + o, pv[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < RB; u++) {
        const int i = i0 + u * BT;
        if (i >= T.nrows) continue;
        const size_t o = ((size_t)T.row0 + i) * K;
        TI pn[K];
#pragma unroll
        for (int k = 0; k < K; k++)
          pn[k] = !act[k] ? pv[u][k] : first[k] ? zv[u][k] : radd(zv[u][k], rmul(beta[k], pv[u][k]));
        st_row<K>(p + o, pn);
      }
    }
  }
}

// PH_INNER: q = A32 p ; sigma = (p, q) ; alpha = rho / sigma.
template <int K, class TI>
__global__ void __launch_bounds__(BT, Occ<K>::spmv_blocks) kb_spmv(const BSys *__restrict__ sys, BState *state,
                                                              BSol *sol, const BCtl *ctl) {
  __shared__ double sm[32 * 2 * MAXK];
  if (phase_idle(ctl, PH_INNER)) return;
  const BTile *__restrict__ tiles = ctl->tiles;
  double *part = ctl->part;
  const int ntiles = ctl->ntiles;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile T = tiles[t];
    BState *st = state + T.sys;
    if (st->phase != PH_INNER) continue;
    const BSys &S = sys[T.sys];
    double v[1][K];
#pragma unroll
    for (int k = 0; k < K; k++) v[0][k] = 0.0;
    const TI *__restrict__ p = (const TI *)S.p;
    TI *__restrict__ q = (TI *)S.q;
    tile_spmv<TI, TI, K>(S, T, inner_val<TI>(S), p, [&](int r, const double (&aq)[K]) {
      TI pv[K], qv[K];
      ld_row<K>(p + (size_t)r * K, pv);
#pragma unroll
      for (int k = 0; k < K; k++) {
        qv[k] = (TI)aq[k];
        v[0][k] = radd(v[0][k], rmul((double)pv[k], (double)qv[k]));
      }
      st_row<K>(q + (size_t)r * K, qv);
    });
    if (tile_publish<K, 1>(v, part, t, st, S.ntiles, sm)) {
      __shared__ double tot[K];
      sys_totals<K>(part, S.tile0, S.ntiles, tot, sm);
      if (threadIdx.x < K) {
        BSol *so = sol + S.sol0 + threadIdx.x;
        if (so->active) {
          so->sigma = tot[threadIdx.x];
          if (so->sigma > 0.0) {
            so->alpha = so->rho / so->sigma;
          } else {
            so->active = 0;  // breakdown of the inner solve: refine with what we have
            so->alpha = 0.0;
            so->restart = 1;
          }
        } else {
          so->alpha = 0.0;
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) st->ticket = 0;
    }
  }
}

// PH_INNER: d += alpha p ; r -= alpha q ; z = D r ; (r,z), (r,r) ; inner stop
// test per rhs ; all rhs stopped -> PH_XUPD.
template <int K, class TI>
__global__ void __launch_bounds__(BT, Occ<K>::update_blocks) kb_update(const BSys *__restrict__ sys, BState *state,
                                                                BSol *sol, const BCtl *ctl) {
  constexpr int RB = K == 1 ? 4 : 1;
  __shared__ double sm[32 * 2 * MAXK];
  if (phase_idle(ctl, PH_INNER)) return;
  const BTile *__restrict__ tiles = ctl->tiles;
  double *part = ctl->part;
  const int ntiles = ctl->ntiles;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile T = tiles[t];
    BState *st = state + T.sys;
    if (st->phase != PH_INNER) continue;
    const BSys &S = sys[T.sys];
    TI alpha[K];
    bool act[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      const BSol *so = sol + S.sol0 + k;
      act[k] = so->active;
      alpha[k] = (TI)so->alpha;
    }
    const TI *__restrict__ p = (const TI *)S.p;
    const TI *__restrict__ q = (const TI *)S.q;
    const TI *__restrict__ dinv = (const TI *)S.dinv;
    TI *__restrict__ d = (TI *)S.d;
    TI *__restrict__ r32 = (TI *)S.r32;
    TI *__restrict__ z = (TI *)S.z;
    double v[2][K];
#pragma unroll
    for (int k = 0; k < K; k++) v[0][k] = v[1][k] = 0.0;
    // a stopped rhs keeps d and r; its z is rewritten as D r, the value it
    // already holds
    bool any_act = false;
#pragma unroll
    for (int k = 0; k < K; k++) any_act |= act[k];
    for (int i0 = threadIdx.x; any_act && i0 < T.nrows; i0 += RB * BT) {
      TI dv[RB][K], pv[RB][K], rv[RB][K], qv[RB][K], dg[RB];
#pragma unroll
      for (int u = 0; u < RB; u++) {
        const int i = i0 + u * BT;
        const size_t o = ((size_t)T.row0 + i) * K;
        if (i < T.nrows) {
          dg[u] = dinv[T.row0 + i];
          ld_row<K>(d + o, dv[u]);
          ld_row<K>(p + o, pv[u]);
          ld_row<K>(r32 + o, rv[u]);
          ld_row<K>(q + o, qv[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < RB; u++) {
        const int i = i0 + u * BT;
        if (i >= T.nrows) continue;
        const size_t o = ((size_t)T.row0 + i) * K;
        TI dn[K], rn[K], zn[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
          dn[k] = act[k] ? radd(dv[u][k], rmul(alpha[k], pv[u][k])) : dv[u][k];
          rn[k] = act[k] ? radd(rv[u][k], -rmul(alpha[k], qv[u][k])) : rv[u][k];
          zn[k] = rmul(dg[u], rn[k]);
          if (act[k]) {
            v[0][k] = radd(v[0][k], rmul((double)rn[k], (double)zn[k]));
            v[1][k] = radd(v[1][k], rmul((double)rn[k], (double)rn[k]));
          }
        }
        st_row<K>(d + o, dn);
        st_row<K>(r32 + o, rn);
        st_row<K>(z + o, zn);
      }
    }
    if (tile_publish<K, 2>(v, part, t, st, S.ntiles, sm)) {
      __shared__ double tot[2 * K];
      sys_totals<2 * K>(part, S.tile0, S.ntiles, tot, sm);
      if (threadIdx.x < K) {
        const int k = threadIdx.x;
        BSol *so = sol + S.sol0 + k;
        if (so->active) {
          const double rz = tot[k];
          const double rr = tot[K + k];
          so->it_total += 1;
          so->loop_it += 1;
          if (sqrt(rr) <= so->tau || so->it_total >= so->itmax || rz <= 0.0 || so->loop_it >= so->loop_cap) {
            so->active = 0;
            so->rrec = sqrt(rr) * so->scale;  // rho stays: the next inner loop forms beta from it
            if (rz <= 0.0) so->restart = 1;
          } else {
            so->beta = rz / so->rho;
            so->rho = rz;
            so->it += 1;
          }
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int any = 0;
        for (int k = 0; k < K; k++) any |= sol[S.sol0 + k].active;
        if (!any) move_phase(ctl, st, PH_XUPD);
        st->ticket = 0;
      }
    }
  }
}

// PH_XUPD: x += scale * d (FP64) for rhs still running ; -> PH_RESID.
template <int K, class TI>
__global__ void __launch_bounds__(BT, Occ<K>::blocks) kb_xupd(const BSys *__restrict__ sys, BState *state,
                                                              const BSol *sol, const BCtl *ctl) {
  constexpr int RB = K == 1 ? 4 : 1;
  if (phase_idle(ctl, PH_XUPD)) return;
  const BTile *__restrict__ tiles = ctl->tiles;
  const int ntiles = ctl->ntiles;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile T = tiles[t];
    BState *st = state + T.sys;
    if (st->phase != PH_XUPD) continue;
    const BSys &S = sys[T.sys];
    double sc[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      const BSol *so = sol + S.sol0 + k;
      sc[k] = so->done == 0 ? so->scale : 0.0;
    }
    double *__restrict__ x = S.x;
    const TI *__restrict__ d = (const TI *)S.d;
    bool any = false;
#pragma unroll
    for (int k = 0; k < K; k++) any |= sc[k] != 0.0;
    for (int i0 = threadIdx.x; any && i0 < T.nrows; i0 += RB * BT) {
      double xv[RB][K];
      TI dv[RB][K];
#pragma unroll
      for (int u = 0; u < RB; u++) {
        const int i = i0 + u * BT;
        const size_t o = ((size_t)T.row0 + i) * K;
        if (i < T.nrows) {
          ld_row<K>(x + o, xv[u]);
          ld_row<K>(d + o, dv[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < RB; u++) {
        const int i = i0 + u * BT;
        if (i >= T.nrows) continue;
        const size_t o = ((size_t)T.row0 + i) * K;
        double xn[K];
#pragma unroll
        for (int k = 0; k < K; k++) xn[k] = sc[k] != 0.0 ? radd(xv[u][k], rmul(sc[k], (double)dv[u][k])) : xv[u][k];
        st_row<K>(x + o, xn);
      }
    }
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&st->ticket, 1u) == (unsigned)(S.ntiles - 1);
    __syncthreads();
    if (last && threadIdx.x == 0) {
      __threadfence();
      move_phase(ctl, st, PH_RESID);
      st->ticket = 0;
    }
  }
}

// A slot joins (phase PH_RESID) or leaves (PH_IDLE) between replays: fresh
// state, and the per-phase counts follow.  One thread.
__global__ void kb_set_phase(BState *state, int *count, int slot, int phase) {
  BState &b = state[slot];
  if (b.phase != PH_IDLE) atomicSub(count + b.phase, 1);
  b.phase = phase;
  b.ticket = 0;
  b.outer = 0;
  b.done_flag = 0;
  if (phase != PH_IDLE) atomicAdd(count + phase, 1);
}

template <class TI>
__global__ void kb_dinv(int n, const double *__restrict__ dinv, TI *__restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = dinv ? (TI)dinv[i] : TI(1);
}

// --------------------------------------------------------------- host side
template <int K, class TI>
static void capture_iters(Eng *e, cudaStream_t st) {
  for (int it = 0; it < ITERS; it++) {
    kb_xupd<K, TI><<<e->grid, BT, 0, st>>>(e->d_sys, e->d_state, e->d_sol, e->d_ctl);
    kb_resid<K><<<e->grid, BT, 0, st>>>(e->d_sys, e->d_state, e->d_sol, e->d_ctl);
    kb_init<K, TI><<<e->grid, BT, 0, st>>>(e->d_sys, e->d_state, e->d_sol, e->d_ctl);
    kb_p<K, TI><<<e->grid, BT, 0, st>>>(e->d_sys, e->d_state, e->d_sol, e->d_ctl);
    kb_spmv<K, TI><<<e->grid, BT, 0, st>>>(e->d_sys, e->d_state, e->d_sol, e->d_ctl);
    kb_update<K, TI><<<e->grid, BT, 0, st>>>(e->d_sys, e->d_state, e->d_sol, e->d_ctl);
  }
}

// Tile plan of one matrix (rows relative to the matrix), built once from its
// row lengths and kept on the matrix (the arrays' rewrite drops it): runs of
// up to BT/32 consecutive rows longer than LONG_ROW become long-row
// tiles; the rows between them are cut into thread-per-row tiles of at most
// tile_rows(K) rows and tile_nnz(K) stored entries -- whole passes of the block
// where the entry bound cuts -- so no thread carries a long serial chain
// (the head of a row-sorted power-law matrix, a long row among short ones).
// It depends on the matrix alone, so a system's tiles and the order of its
// partial sums do not depend on the other systems in the engine (the plan is
// rebuilt when an engine with another K adds the matrix).
static int tile_plan(HllDevice *m, int K) {
  const int n = m->rows;
  const int trows = tile_rows(K), tnnz = tile_nnz(K);
  std::vector<int> irn(n > 0 ? n : 1);
  if (n > 0) PSBX_CK(cudaMemcpy(irn.data(), m->rS, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost));
  std::vector<int> plan;
  for (int r = 0; r < n;) {
    int e = r;
    if (irn[r] > LONG_ROW) {
      while (e < n && e - r < BT / 32 && irn[e] > LONG_ROW) e++;
      plan.insert(plan.end(), {r, e - r, 1});
    } else {
      long long ent = 0;
      while (e < n && e - r < trows && irn[e] <= LONG_ROW && ent + irn[e] <= tnnz) ent += irn[e++];
      const bool entry_cut = e < n && e - r < trows && irn[e] <= LONG_ROW;
      if (entry_cut && e - r > BT) e = r + (e - r) / BT * BT;
      plan.insert(plan.end(), {r, e - r, 0});
    }
    r = e;
  }
  int *t = (int *)malloc(sizeof(int) * (plan.empty() ? 1 : plan.size()));
  if (!t) return SPGPU_OUTOFMEMORY;
  if (!plan.empty()) memcpy(t, plan.data(), sizeof(int) * plan.size());
  free(m->tplan);
  m->tplan = t;
  m->ntplan = (int)(plan.size() / 3);
  m->tplanK = K;
  return SPGPU_SUCCESS;
}

static int upload_tables(Eng *e, cudaStream_t st) {
  // rebuild the tile table from the slots in use
  std::vector<BTile> tiles;
  for (int s = 0; s < e->max_sys; s++) {
    if (!e->used[s]) continue;
    BSys &S = e->h_sys[s];
    S.tile0 = (int)tiles.size();
    const std::vector<int> &pl = e->plan[s];
    for (size_t k = 0; k + 2 < pl.size(); k += 3) {
      BTile T;
      T.sys = s;
      T.row0 = pl[k];
      T.nrows = pl[k + 1];
      T.kind = pl[k + 2];
      tiles.push_back(T);
    }
    S.ntiles = (int)tiles.size() - S.tile0;
  }
  if ((int)tiles.size() > e->max_tiles) {
    // grow the tile table and the partial sums (kernels read them via d_ctl)
    PSBX_CK(cudaStreamSynchronize(st));
    const int cap = (int)tiles.size() * 2;
    BTile *nt = nullptr;
    double *np_ = nullptr;
    PSBX_CK(cudaMalloc(&nt, sizeof(BTile) * cap));
    cudaError_t err = cudaMalloc(&np_, sizeof(double) * 2 * MAXK * (size_t)cap);
    if (err != cudaSuccess) {
      cudaFree(nt);
      return psbx_cuda_status(err, "psbx_batch tiles");
    }
    cudaFree(e->d_tiles);
    cudaFree(e->d_part);
    e->d_tiles = nt;
    e->d_part = np_;
    e->max_tiles = cap;
  }
  if ((int)tiles.size() > e->h_tiles_cap) {
    PSBX_CK(cudaStreamSynchronize(st));  // the old staging buffer may still be read
    cudaFreeHost(e->h_tiles_pinned);
    e->h_tiles_pinned = nullptr;
    e->h_tiles_cap = 0;
    const int cap = (int)tiles.size() * 2;
    PSBX_CK(cudaHostAlloc(&e->h_tiles_pinned, sizeof(BTile) * cap, 0));
    e->h_tiles_cap = cap;
  }
  BCtl &c = *e->h_ctl_pinned;
  memset(&c, 0, sizeof(c));
  c.ntiles = (int)tiles.size();
  c.cap = e->max_tiles;
  c.tiles = e->d_tiles;
  c.part = e->d_part;
  c.count = e->d_count;
  if (!tiles.empty()) {
    memcpy(e->h_tiles_pinned, tiles.data(), sizeof(BTile) * tiles.size());
    PSBX_CK(cudaMemcpyAsync(e->d_tiles, e->h_tiles_pinned, sizeof(BTile) * tiles.size(), cudaMemcpyHostToDevice, st));
  }
  memcpy(e->h_sys_pinned, e->h_sys.data(), sizeof(BSys) * e->max_sys);
  PSBX_CK(cudaMemcpyAsync(e->d_sys, e->h_sys_pinned, sizeof(BSys) * e->max_sys, cudaMemcpyHostToDevice, st));
  PSBX_CK(cudaMemcpyAsync(e->d_ctl, e->h_ctl_pinned, sizeof(BCtl), cudaMemcpyHostToDevice, st));
  return SPGPU_SUCCESS;
}

}  // namespace

extern "C" {

int psbx_batch_create(void **eng, int max_systems, int max_rows_total, int nrhs) {
  return psbx_batch_create_prec(eng, max_systems, max_rows_total, nrhs, 32);
}

int psbx_batch_create_prec(void **eng, int max_systems, int max_rows_total, int nrhs, int inner_bits) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  if (!eng || max_systems <= 0 || max_rows_total <= 0 || (nrhs != 1 && nrhs != 8)) return SPGPU_UNSUPPORTED;
  if (inner_bits != 32 && inner_bits != 64) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  Eng *e = new Eng();
  e->K = nrhs;
  e->fp64 = inner_bits == 64;
  e->max_sys = max_systems;
  e->max_tiles = max_rows_total / tile_rows(e->K) + max_systems + 1;
  e->grid = c.sms * 8;
  e->h_sys.assign(max_systems, BSys());
  e->h_state.assign(max_systems, BState());
  e->used.assign(max_systems, 0);
  e->owned.assign(max_systems, nullptr);
  e->plan.assign(max_systems, std::vector<int>());
  memset(e->h_sys.data(), 0, sizeof(BSys) * max_systems);
  memset(e->h_state.data(), 0, sizeof(BState) * max_systems);
  cudaError_t err = cudaSuccess;
  if (err == cudaSuccess) err = cudaMalloc(&e->d_sys, sizeof(BSys) * max_systems);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_state, sizeof(BState) * max_systems);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_sol, sizeof(BSol) * max_systems * nrhs);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_tiles, sizeof(BTile) * e->max_tiles);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_ctl, sizeof(BCtl));
  if (err == cudaSuccess) err = cudaMalloc(&e->d_count, sizeof(int) * 8);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->d_count, 0, sizeof(int) * 8, c.stream);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_part, sizeof(double) * 2 * MAXK * (size_t)e->max_tiles);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->done_ev, cudaEventDisableTiming);
  if (err == cudaSuccess) err = cudaHostAlloc(&e->h_sys_pinned, sizeof(BSys) * max_systems, 0);
  if (err == cudaSuccess) err = cudaHostAlloc(&e->h_ctl_pinned, sizeof(BCtl), 0);
  if (err == cudaSuccess) err = cudaHostAlloc(&e->h_sol_init, sizeof(BSol) * max_systems * nrhs, 0);
  if (err == cudaSuccess) err = cudaHostAlloc(&e->h_state_pinned, sizeof(BState) * max_systems, 0);
  if (err == cudaSuccess) err = cudaHostAlloc(&e->h_sol_pinned, sizeof(BSol) * max_systems * nrhs, 0);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->d_state, 0, sizeof(BState) * max_systems, c.stream);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->d_sol, 0, sizeof(BSol) * max_systems * nrhs, c.stream);
  if (err != cudaSuccess) {
    rc = psbx_cuda_status(err, "psbx_batch_create");
    psbx_batch_destroy(e);
    *eng = nullptr;
    return rc;
  }
  rc = upload_tables(e, c.stream);
  if (!rc) {
    err = cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess) {
      if (nrhs == 1) e->fp64 ? capture_iters<1, double>(e, c.stream) : capture_iters<1, float>(e, c.stream);
      else e->fp64 ? capture_iters<8, double>(e, c.stream) : capture_iters<8, float>(e, c.stream);
      err = cudaStreamEndCapture(c.stream, &e->graph);
    }
    if (err == cudaSuccess) err = cudaGraphInstantiate(&e->gexec, e->graph, 0);
    if (err != cudaSuccess) rc = psbx_cuda_status(err, "psbx_batch_create graph");
  }
  if (rc) {
    psbx_batch_destroy(e);
    *eng = nullptr;
    return rc;
  }
  *eng = e;
  return SPGPU_SUCCESS;
}

int psbx_batch_add(void *eng, void *hllMat, const double *d_b, double *d_x, const double *d_dinv, double eps,
                   double inner_tol, int itmax, int *slot) {
  Eng *e = (Eng *)eng;
  HllDevice *m = (HllDevice *)hllMat;
  if (!e || !m || !d_b || !d_x || !slot) return SPGPU_UNSUPPORTED;
  if (m->elemType != SPGPU_TYPE_DOUBLE || m->hackSize != 32 || m->perm || m->baseIndex != 1) {
    psbx_set_error("psbx_batch_add: the matrix must be an FP64 HLL of hack size 32, index base 1, "
                   "without a row permutation");
    return SPGPU_UNSUPPORTED;
  }
  // rows of 8 right-hand sides move as 16-byte vectors
  if (e->K > 1 && (((uintptr_t)d_b | (uintptr_t)d_x) & 15)) {
    psbx_set_error("psbx_batch_add: with several right-hand sides b and x must be 16-byte aligned");
    return SPGPU_UNSUPPORTED;
  }
  if (!m->cM32) {
    int rc = psbx_hll_make_single(m);
    if (rc) return rc;
  }
  int s = -1;
  for (int i = 0; i < e->max_sys; i++)
    if (!e->used[i]) {
      s = i;
      break;
    }
  if (s < 0) return SPGPU_OUTOFMEMORY;  // no free slot
  if (!m->tplan || m->tplanK != e->K) {
    int rc = tile_plan(m, e->K);
    if (rc) return rc;
  }
  PsbxCtx &c = psbx_ctx();
  const int K = e->K;
  const size_t n = (size_t)m->rows;
  // one allocation per slot: r64 (K n doubles), r32 z p q d (5 K n inner values), dinv (n inner values)
  const size_t ti = e->fp64 ? sizeof(double) : sizeof(float);
  const size_t bytes = sizeof(double) * K * n + ti * (5 * K + 1) * n + 256;
  char *buf = nullptr;
  cudaError_t err = psbx_malloc_async((void **)&buf, bytes, c.stream);
  if (err != cudaSuccess) return psbx_cuda_status(err, "psbx_batch_add");
  BSys S;
  memset(&S, 0, sizeof(S));
  S.val64 = (const double *)m->cM;
  S.val32 = m->cM32;
  S.ja = m->rP;
  S.irn = m->rS;
  S.hkoffs = m->hackOffs;
  S.b = d_b;
  S.x = d_x;
  S.r64 = (double *)buf;
  char *f = buf + sizeof(double) * K * n;
  S.r32 = f;
  S.z = f + ti * K * n;
  S.p = f + 2 * ti * K * n;
  S.q = f + 3 * ti * K * n;
  S.d = f + 4 * ti * K * n;
  char *dv = f + 5 * ti * K * n;
  S.dinv = dv;
  S.rows = (int)n;
  S.sol0 = s * K;
  e->plan[s].assign(m->tplan, m->tplan + 3 * (size_t)m->ntplan);
  if (e->fp64) kb_dinv<double><<<psbx_grid_for(n, 256), 256, 0, c.stream>>>((int)n, d_dinv, (double *)dv);
  else kb_dinv<float><<<psbx_grid_for(n, 256), 256, 0, c.stream>>>((int)n, d_dinv, (float *)dv);
  psbx_count_launch();
  std::vector<BSol> so(K);
  memset(so.data(), 0, sizeof(BSol) * K);
  for (int k = 0; k < K; k++) {
    so[k].eps = eps;
    so[k].inner_tol = inner_tol;
    so[k].itmax = itmax;
    so[k].outer_max = 64;
    so[k].first = 1;
    so[k].restart = 1;
  }
  e->h_sys[s] = S;
  e->used[s] = 1;
  e->owned[s] = buf;
  // from pinned memory: a pageable copy would wait for the replays in flight
  memcpy(e->h_sol_init + (size_t)s * K, so.data(), sizeof(BSol) * K);
  PSBX_CK(cudaMemcpyAsync(e->d_sol + (size_t)s * K, e->h_sol_init + (size_t)s * K, sizeof(BSol) * K,
                          cudaMemcpyHostToDevice, c.stream));
  kb_set_phase<<<1, 1, 0, c.stream>>>(e->d_state, e->d_count, s, PH_RESID);
  psbx_count_launch();
  e->dirty = true;  // the tile table is rebuilt once, before the next step
  // until the next step, poll reports the fresh state, not the slot's last occupant
  memset(&e->h_state_pinned[s], 0, sizeof(BState));
  e->h_state_pinned[s].phase = PH_RESID;
  memcpy(e->h_sol_pinned + (size_t)s * K, so.data(), sizeof(BSol) * K);
  *slot = s;
  return SPGPU_SUCCESS;
}

// Enqueues `replays` replays of the captured batch (ITERS iterations each)
// and the read-back of every slot's state, and returns at once; the host can
// prepare the next requests meanwhile.  psbx_batch_wait ends it.
int psbx_batch_launch(void *eng, int replays) {
  Eng *e = (Eng *)eng;
  if (!e || e->inflight) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  const int K = e->K;
  if (e->dirty) {
    int rc = upload_tables(e, c.stream);
    if (rc) return rc;
    e->dirty = false;
  }
  for (int r = 0; r < replays; r++) {
    cudaError_t err = cudaGraphLaunch(e->gexec, c.stream);
    if (err != cudaSuccess) return psbx_cuda_status(err, "psbx_batch_launch");
    psbx_count_launch(6 * ITERS);
  }
  PSBX_CK(cudaMemcpyAsync(e->h_state_pinned, e->d_state, sizeof(BState) * e->max_sys, cudaMemcpyDeviceToHost,
                          c.stream));
  PSBX_CK(cudaMemcpyAsync(e->h_sol_pinned, e->d_sol, sizeof(BSol) * e->max_sys * K, cudaMemcpyDeviceToHost,
                          c.stream));
  PSBX_CK(cudaEventRecord(e->done_ev, c.stream));
  e->inflight = true;
  return SPGPU_SUCCESS;
}

// Waits for the last launch; *n_running = slots still running.
int psbx_batch_wait(void *eng, int *n_running) {
  Eng *e = (Eng *)eng;
  if (!e) return SPGPU_UNSUPPORTED;
  if (e->inflight) {
    PSBX_CK(cudaEventSynchronize(e->done_ev));
    e->inflight = false;
  }
  int running = 0;
  for (int s = 0; s < e->max_sys; s++)
    if (e->used[s] && e->h_state_pinned[s].phase != PH_DONE) running++;
  if (n_running) *n_running = running;
  return SPGPU_SUCCESS;
}

// Runs `replays` replays of the captured batch (ITERS iterations each) and
// returns how many slots are still running in *n_running.
int psbx_batch_step(void *eng, int replays, int *n_running) {
  int rc = psbx_batch_launch(eng, replays);
  if (rc) return rc;
  return psbx_batch_wait(eng, n_running);
}

// Status of a slot as of the last step: *state 0 running, 1 all rhs
// converged, 2 finished with some rhs stopped (itmax / breakdown);
// iters[k] inner iterations, err[k] = ||b - A x||/||b|| at the last check.
int psbx_batch_poll(void *eng, int slot, int *state, int *outer, int *iters, double *err) {
  Eng *e = (Eng *)eng;
  if (!e || slot < 0 || slot >= e->max_sys || !e->used[slot]) return SPGPU_UNSUPPORTED;
  const BState &bs = e->h_state_pinned[slot];
  int st = 0;
  if (bs.phase == PH_DONE) {
    st = 1;
    for (int k = 0; k < e->K; k++)
      if (e->h_sol_pinned[slot * e->K + k].done != 1) st = 2;
  }
  if (state) *state = st;
  if (outer) *outer = bs.outer;
  for (int k = 0; k < e->K; k++) {
    const BSol &so = e->h_sol_pinned[slot * e->K + k];
    if (iters) iters[k] = so.it_total;
    if (err) err[k] = so.bn2 == 0.0 ? so.rn : so.rn / so.bn2;
  }
  return SPGPU_SUCCESS;
}

int psbx_batch_finished(void *eng, int *slots, int max, int *count) {
  Eng *e = (Eng *)eng;
  if (!e || !count || max < 0 || (max > 0 && !slots)) return SPGPU_UNSUPPORTED;
  int n = 0;
  for (int s = 0; s < e->max_sys; s++)
    if (e->used[s] && e->h_state_pinned[s].phase == PH_DONE) {
      if (n < max) slots[n] = s;
      n++;
    }
  *count = n;
  return SPGPU_SUCCESS;
}

int psbx_batch_remove(void *eng, int slot) {
  Eng *e = (Eng *)eng;
  if (!e || slot < 0 || slot >= e->max_sys || !e->used[slot]) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  kb_set_phase<<<1, 1, 0, c.stream>>>(e->d_state, e->d_count, slot, PH_IDLE);
  psbx_count_launch();
  cudaFreeAsync(e->owned[slot], c.stream);
  e->owned[slot] = nullptr;
  e->used[slot] = 0;
  memset(&e->h_sys[slot], 0, sizeof(BSys));
  e->dirty = true;  // its tiles leave the table before the next step (its phase is idle meanwhile)
  return SPGPU_SUCCESS;
}

int psbx_batch_destroy(void *eng) {
  Eng *e = (Eng *)eng;
  if (!e) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  cudaStreamSynchronize(c.stream);
  for (int s = 0; s < e->max_sys; s++)
    if (e->owned[s]) cudaFreeAsync(e->owned[s], c.stream);
  if (e->gexec) cudaGraphExecDestroy(e->gexec);
  if (e->graph) cudaGraphDestroy(e->graph);
  cudaFree(e->d_sys);
  cudaFree(e->d_state);
  cudaFree(e->d_sol);
  cudaFree(e->d_tiles);
  cudaFree(e->d_ctl);
  cudaFree(e->d_count);
  cudaFree(e->d_part);
  if (e->done_ev) cudaEventDestroy(e->done_ev);
  cudaFreeHost(e->h_tiles_pinned);
  cudaFreeHost(e->h_sys_pinned);
  cudaFreeHost(e->h_ctl_pinned);
  cudaFreeHost(e->h_sol_init);
  cudaFreeHost(e->h_state_pinned);
  cudaFreeHost(e->h_sol_pinned);
  cudaStreamSynchronize(c.stream);
  delete e;
  return SPGPU_SUCCESS;
}

}  // extern "C"
