// psbx_internal.cuh -- shared device objects, context and device helpers of
// libpsbx (B200 / sm_100a).  Not part of the public C-ABI (include/psbx.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <atomic>
#include <vector>

#include "../../include/psbx.h"

// ---------------------------------------------------------------------------
// Device objects.  The leading fields keep the names of the reference's C
// structs (cuda/vectordev.h:39-53, cuda/hlldev.h:36-66, cuda/elldev.h) so a
// maintainer can map one onto the other; the Fortran side never looks inside.
// ---------------------------------------------------------------------------
struct MultiVectDevice {
  int count_;      // number of vectors
  int size_;       // entries per vector
  int pitch_;      // entries between consecutive vectors
  void *v_;        // device data (pitch_*count_ elements)
  int elemType;    // SPGPU_TYPE_*
  int owns;        // 1 if v_ was allocated here (freed by freeMultiVecDevice)
};

struct HllDevice {
  void *cM;          // values, allocsize elements (FP64 or FP32 by elemType)
  int *rP;           // column indices, allocsize
  int *rS;           // row lengths (irn), rows
  int *diag;         // 1-based diagonal position (idiag), rows
  int *hackOffs;     // hackOffsLength+1 offsets
  int rows;
  int avgNzr;
  int hackOffsLength;
  int nzt;
  int hackSize;
  int allocsize;
  int baseIndex;
  // additions
  int elemType;
  int cols;
  float *cM32;       // optional FP32 copy of FP64 values (mixed precision)
  int *perm;         // optional storage-row -> matrix-row map (NULL: identity)
  int maxRowLen;     // longest stored row (-1: unknown)
  // hacks wider than longW (hack size 32 only): their row sums are formed
  // before each product (psbx_long_rows32: all products at once into wprod,
  // then a warp per hack adds them in order) and read back from lres by the
  // row kernels
  int *longHacks;    // hack ids, nLong of them
  int nLong;
  double *lres;      // rows entries (storage order), allocated when nLong > 0
  int longW;         // 0: default (PSBX_LONG_W or 4x the mean hack width); < 0: never
  int effW;          // the threshold the wide list was built with
  int *tplan;        // batch engine tile plan (host memory, 3 ints per tile), built on first use
  int ntplan;
  int tplanK;        // right-hand sides per row the plan was built for
  int *wideBase;     // nLong+1: offset of each wide hack's products in wprod
  int *wchunk;       // 2*nWChunks: (wide hack index, first entry column) per product block
  int nWChunks;
  double *wprod;     // products of the wide hacks, laid out as their values
  int wideSplit;     // 1 (default): tolerance mode -- wide hacks summed in column chunks, two
                     // threads per row allowed; 0: every row in stored order (exact)
  int tpr;           // standalone SpMV row mapping (hack size 32): 0 auto, 1 or 2 threads per
                     // row, -2 two rows per thread
  double *wpart;     // split mode: 32 row partials per product block (nWChunks x 32)
  unsigned *wticket; // split mode: per wide hack, product blocks done (kept at zero between calls)
  int *wcbase;       // nLong+1: first product block of each wide hack
  // host-buffer SpMV (psbx_hll_spmv_host): device staging vectors, and per
  // hack the smallest and largest column it holds (host arrays, built on
  // first use, dropped when the arrays are rewritten)
  double *hx, *hy;
  int *hcmin, *hcmax;
};

// Default width above which a hack of 32 rows takes the wide-hack path.
#define PSBX_LONG_W 64

struct EllDevice {
  void *cM;
  int *rP;
  int *diag;
  int *rS;
  int rows;
  int columns;
  int pitch;
  int cMPitch;
  int rPPitch;
  int maxRowSize;
  int avgRowSize;
  int allocsize;
  int baseIndex;
  int dataType;
};

struct CsrDevice {
  int m, n, nz;
  double *val;
  int *irp;
  int *ja;
  int baseIndex;     // 0 or 1 (d_CSRGDeviceSetMatIndexBase)
  int maxRowLen;     // computed at upload
  // work partition of the adaptive kernel (built at upload)
  int *rowBlocks;    // 2*nBlocks: start and end row of each row block
  int nBlocks;
  int *chunks;       // 6*nChunks: chunk records of rows longer than a tile
  int nChunks;
  double *chunkPart; // one partial sum per chunk
  unsigned *chunkTicket;  // one counter per long row (kept at zero between calls)
  int nLong;
  // triangular solve (d_spsvCSRGDevice): cuSPARSE descriptor settings kept
  // as the Fortran side sets them, and the solve's state, allocated by the
  // first solve
  int matType;       // 0 general, 3 triangular (cusparse_matrix_type_*)
  int fillMode;      // 0 lower, 1 upper (cusparse_fill_mode_*)
  int diagType;      // 0 non-unit, 1 unit (cusparse_diag_type_*)
  unsigned *svFlag;  // per row: generation of the solve that finished it
  unsigned *svCtl;   // [0] row ticket, [1] timeout flag
  unsigned svGen;    // generation of the last solve
};

// ---------------------------------------------------------------------------
// Context: one per process (the reference keeps one global SPGPU handle).
// ---------------------------------------------------------------------------
#define PSBX_MAX_PART 4096     // partial-sum slots (pairs) per reduction lane
#define PSBX_NLANES   8        // simultaneous reductions (vectors / dots)

struct PsbxCtx {
  bool init = false;
  int device = 0;
  int sms = 148;
  int maxThreadsPerMP = 2048;
  cudaStream_t defaultStream = nullptr;
  cudaStream_t stream = nullptr;
  cudaDeviceProp prop;
  double *d_part = nullptr;       // [PSBX_NLANES][PSBX_MAX_PART]
  unsigned *d_ticket = nullptr;   // [64] zero-initialised, reset by users
  double *d_res = nullptr;        // [64] reduction results
  double *h_res = nullptr;        // pinned [64]
  // Stream-ordered workspace of the solvers comes from this pool, which
  // keeps up to PSBX_POOL_KEEP bytes of freed memory mapped between calls:
  // with nothing kept, every solve remapped its workspace (1 GB for CG on
  // 16.8M rows), and calls of the same solve varied from 0.49 to 1.1 s.
  cudaMemPool_t pool = nullptr;
  // copy streams and events of the host-buffer SpMV (psbx_hll_spmv_host),
  // created on first use
  cudaStream_t h2d = nullptr, d2h = nullptr;
  std::vector<cudaEvent_t> xev;
};
#define PSBX_POOL_KEEP ((uint64_t)4 << 30)

PsbxCtx &psbx_ctx();             // lazily initialises on the current device
// cudaMallocAsync from the library's pool (freed with cudaFreeAsync)
template <class T>
static inline cudaError_t psbx_malloc_async(T **p, size_t bytes, cudaStream_t st) {
  return cudaMallocFromPoolAsync((void **)p, bytes, psbx_ctx().pool, st);
}
int psbx_ensure_init();          // 0 or error code
int psbx_cuda_status(cudaError_t e, const char *where);
void psbx_set_error(const char *msg);  // message for psbx_last_error, also printed
void psbx_count_launch(int n = 1);

#define PSBX_CK(call)                                                        \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) return psbx_cuda_status(e_, #call);               \
  } while (0)

#define PSBX_LAUNCH_CK(where)                                                \
  do {                                                                       \
    psbx_count_launch();                                                     \
    cudaError_t e_ = cudaGetLastError();                                     \
    if (e_ != cudaSuccess) return psbx_cuda_status(e_, where);               \
  } while (0)

static inline int psbx_grid_for(long long work, int threads, int perSM = 8) {
  PsbxCtx &c = psbx_ctx();
  long long need = (work + threads - 1) / threads;
  long long cap = (long long)c.sms * perSM;
  if (need < 1) need = 1;
  return (int)(need < cap ? need : cap);
}

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
// Rounded multiply and add with no contraction: the reference's loops are
// `acc = acc + v*x`, a rounded product then a rounded sum.
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float rmulf(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float raddf(float a, float b) { return __fadd_rn(a, b); }
// The same, overloaded, for kernels written once for double and float (an
// argument pair of mixed types does not resolve, which keeps mixed-precision
// arithmetic explicit).
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }

// Streaming (read-once) loads: evict-first in L1/L2 so gathered vectors stay.
template <class T>
__device__ __forceinline__ T ld_stream(const T *p) { return __ldcs(p); }
template <class T>
__device__ __forceinline__ T ld_ro(const T *p) { return __ldg(p); }

// Deterministic block sum of NV values (fixed shuffle tree, then warp 0).
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *smem /*[32*NV]*/) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] = radd(v[k], __shfl_down_sync(0xffffffffu, v[k], o));
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) smem[k * 32 + warp] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double t = lane < nw ? smem[k * 32 + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t = radd(t, __shfl_down_sync(0xffffffffu, t, o));
      v[k] = t;  // valid in thread 0
    }
  }
}

template <int NV>
__device__ __forceinline__ void block_max(double (&v)[NV], double *smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] = fmax(v[k], __shfl_down_sync(0xffffffffu, v[k], o));
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) smem[k * 32 + warp] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double t = lane < nw ? smem[k * 32 + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_down_sync(0xffffffffu, t, o));
      v[k] = t;
    }
  }
}

// ---------------------------------------------------------------------------
// Compensated dot products (Dot2 of Ogita, Rump and Oishi, SIAM J. Sci.
// Comput. 26(6), 2005): each product is split exactly into p + e with an
// FMA, running sums are kept as an unevaluated pair s + c (TwoSum), partial
// pairs merge with TwoSum.  The rounded result s + c is as accurate as a sum
// in twice the precision, so it almost never depends on the summation order:
// the device tree and the oracle's left-to-right loop give the same bits.
// ---------------------------------------------------------------------------
struct dd_t {
  double s, c;
};

__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
  s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}

__device__ __forceinline__ void dd_add_prod(dd_t &acc, double x, double y) {
  const double p = __dmul_rn(x, y);
  const double e = __fma_rn(x, y, -p);
  double s, t;
  two_sum(acc.s, p, s, t);
  acc.s = s;
  acc.c = __dadd_rn(acc.c, __dadd_rn(t, e));
}

__device__ __forceinline__ dd_t dd_merge(dd_t x, dd_t y) {
  dd_t r;
  double t;
  two_sum(x.s, y.s, r.s, t);
  r.c = __dadd_rn(t, __dadd_rn(x.c, y.c));
  return r;
}

__device__ __forceinline__ double dd_value(dd_t a) { return __dadd_rn(a.s, a.c); }

template <int NV>
__device__ __forceinline__ void block_sum_dd(dd_t (&v)[NV], double *smem /*[64*NV]*/) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      dd_t u;
      u.s = __shfl_down_sync(0xffffffffu, v[k].s, o);
      u.c = __shfl_down_sync(0xffffffffu, v[k].c, o);
      v[k] = dd_merge(v[k], u);
    }
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      smem[(k * 32 + warp) * 2] = v[k].s;
      smem[(k * 32 + warp) * 2 + 1] = v[k].c;
    }
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      dd_t t = {0.0, 0.0};
      if (lane < nw) {
        t.s = smem[(k * 32 + lane) * 2];
        t.c = smem[(k * 32 + lane) * 2 + 1];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        dd_t u;
        u.s = __shfl_down_sync(0xffffffffu, t.s, o);
        u.c = __shfl_down_sync(0xffffffffu, t.c, o);
        t = dd_merge(t, u);
      }
      v[k] = t;  // valid in thread 0
    }
  }
}

// Partial pairs of lane k, block b live at part[2*(k*stride + b)] (+1).
template <int NV>
__device__ __forceinline__ void final_sum_dd(const double *part, int stride, int n, dd_t (&out)[NV],
                                             double *smem) {
#pragma unroll
  for (int k = 0; k < NV; k++) {
    dd_t a = {0.0, 0.0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      dd_t u;
      u.s = __ldcg(part + 2 * ((size_t)k * stride + i));
      u.c = __ldcg(part + 2 * ((size_t)k * stride + i) + 1);
      a = dd_merge(a, u);
    }
    out[k] = a;
  }
  block_sum_dd<NV>(out, smem);
}

// Last-block-done: every block publishes its partials, then takes a ticket;
// the block that draws gridSize-1 sees all partials and finalises.  The
// finaliser resets the ticket for the next launch.
__device__ __forceinline__ bool psbx_last_block(unsigned *ticket, unsigned nblocks) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned t = atomicAdd(ticket, 1u);
    last = (t == nblocks - 1);
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// Sum of part[0..n) in a fixed order by one block (deterministic).
template <int NV>
__device__ __forceinline__ void final_sum(const double *part, int stride, int n,
                                          double (&out)[NV], double *smem) {
#pragma unroll
  for (int k = 0; k < NV; k++) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s = radd(s, __ldcg(part + k * stride + i));
    out[k] = s;
  }
  block_sum<NV>(out, smem);
}

template <int NV>
__device__ __forceinline__ void final_max(const double *part, int stride, int n,
                                          double (&out)[NV], double *smem) {
#pragma unroll
  for (int k = 0; k < NV; k++) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s = fmax(s, __ldcg(part + k * stride + i));
    out[k] = s;
  }
  block_max<NV>(out, smem);
}

// ---------------------------------------------------------------------------
// Matrix views used by the SpMV kernels and the fused Krylov kernels.
// row_dot() returns sum_j val(r,j)*x(ja(r,j)) in stored order (FP64).
// ---------------------------------------------------------------------------
struct HllView {
  const double *val;
  const int *ja;
  const int *irn;
  const int *hkoffs;
  const int *perm;   // storage row -> matrix row (NULL identity)
  int rows, hksz, base;
  const int *longHacks;  // hack size 32: hacks wider than longW
  const double *lres;    // their row sums, formed before the row kernel runs
  int nLong, longW;
  const int *wideBase;   // wide hack i's products start at wprod + wideBase[i]
  const int *wchunk;     // (wide hack index, first column) of each product block
  double *wprod;
  int nWChunks;
  int wideSplit;         // wide rows summed in column chunks (see psbx_hll_set_wide_split)
  double *wpart;
  unsigned *wticket;
  const int *wcbase;
};

struct HllViewF {  // FP32 values, FP32 x
  const float *val;
  const int *ja;
  const int *irn;
  const int *hkoffs;
  const int *perm;
  int rows, hksz, base;
};

struct EllView {
  const double *val;
  const int *ja;
  const int *irn;
  int rows, pitch, base;
};

struct EllViewF {  // FP32 values, FP32 x
  const float *val;
  const int *ja;
  const int *irn;
  int rows, pitch, base;
};

struct CsrView {
  const double *val;
  const int *ja;
  const int *irp;
  int rows, base;
};

// HLL with the reference's GPU hack size (32 = warp size,
// psb_d_cuda_cp_hlg_from_coo.F90:60): hack and lane come from shifts and the
// entry stride is a compile-time constant.
struct Hll32View : HllView {};
// Hack size 32 with wide hacks (nLong > 0): their rows' sums are read back
// from lres (a separate type, so the kernels of matrices without wide hacks
// carry no test for them).
struct Hll32WView : HllView {};
// Hack size 32, every row at most PSBX_SHORT_ROW entries (the 7-point
// operators): a row's entries are read as one predicated group, so all of its
// index and value loads are in flight at once instead of one after another.
struct Hll32SView : HllView {};
#define PSBX_SHORT_ROW 16

// Unrolled in-order accumulation over one row whose j-th entry sits at
// vp[j*stride] / jp[j*stride] (32-bit offsets: every format keeps its
// allocation below 2^31 entries, as psb_ipk_ does).  The U index and value
// loads of a group are issued before its U gathers, the gathers before the
// adds, so each thread keeps 2U streaming loads in flight.
template <class VT, class XT, int U, int STRIDE>
__device__ __forceinline__ double row_acc(const VT *__restrict__ vp, const int *__restrict__ jp, int stride, int n,
                                          const XT *__restrict__ xb) {
  const int st = STRIDE > 0 ? STRIDE : stride;
  double acc = 0.0;
  // full groups unpredicated (fewest registers), then the short tail.  (A
  // predicated last group was measured slower on B200: more registers cost
  // more occupancy than its extra loads in flight bring.)
  int j = 0;
  for (; j + U <= n; j += U) {
    int c[U];
    VT v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      c[u] = ld_stream(jp + (j + u) * st);
      v[u] = ld_stream(vp + (j + u) * st);
    }
    XT xv[U];
#pragma unroll
    for (int u = 0; u < U; u++) xv[u] = ld_ro(xb + c[u]);
#pragma unroll
    for (int u = 0; u < U; u++) acc = radd(acc, rmul((double)v[u], (double)xv[u]));
  }
  for (; j < n; j++) {
    const int c = ld_stream(jp + j * st);
    const VT v = ld_stream(vp + j * st);
    acc = radd(acc, rmul((double)v, (double)ld_ro(xb + c)));
  }
  return acc;
}

// row_acc with the tail as one predicated group of U: the loads of entries
// past the row's end are not issued and their terms are not added, so the
// sum (and its rounding) is the same as row_acc's.
template <class VT, class XT, int U, int STRIDE>
__device__ __forceinline__ double row_acc_p(const VT *__restrict__ vp, const int *__restrict__ jp, int stride, int n,
                                            const XT *__restrict__ xb, int base) {
  const int st = STRIDE > 0 ? STRIDE : stride;
  double acc = 0.0;
  int j = 0;
  for (; j + U <= n; j += U) {
    int c[U];
    VT v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      c[u] = ld_stream(jp + (j + u) * st);
      v[u] = ld_stream(vp + (j + u) * st);
    }
    XT xv[U];
#pragma unroll
    for (int u = 0; u < U; u++) xv[u] = ld_ro(xb + c[u]);
#pragma unroll
    for (int u = 0; u < U; u++) acc = radd(acc, rmul((double)v[u], (double)xv[u]));
  }
  if (j < n) {
    int c[U];
    VT v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const bool ok = j + u < n;
      c[u] = ok ? ld_stream(jp + (j + u) * st) : base;
      v[u] = ok ? ld_stream(vp + (j + u) * st) : VT(0);
    }
    XT xv[U];
#pragma unroll
    for (int u = 0; u < U; u++) xv[u] = j + u < n ? ld_ro(xb + c[u]) : XT(0);
#pragma unroll
    for (int u = 0; u < U; u++)
      if (j + u < n) acc = radd(acc, rmul((double)v[u], (double)xv[u]));
  }
  return acc;
}

__device__ __forceinline__ double row_dot(const Hll32SView &A, int s, const double *__restrict__ x) {
  const int off = ld_ro(A.hkoffs + (s >> 5)) + (s & 31);
  return row_acc_p<double, double, 8, 32>(A.val + off, A.ja + off, 32, ld_ro(A.irn + s), x - A.base, A.base);
}

__device__ __forceinline__ double row_dot(const Hll32View &A, int s, const double *__restrict__ x) {
  const int off = ld_ro(A.hkoffs + (s >> 5)) + (s & 31);
  return row_acc<double, double, 8, 32>(A.val + off, A.ja + off, 32, ld_ro(A.irn + s), x - A.base);
}

__device__ __forceinline__ double row_dot(const Hll32WView &A, int s, const double *__restrict__ x) {
  const int h0 = ld_ro(A.hkoffs + (s >> 5));
  // a row of a wide hack was summed (same order, same roundings) by the
  // long-row kernel launched just before with the same x
  if (((ld_ro(A.hkoffs + (s >> 5) + 1) - h0) >> 5) > A.longW) return __ldcg(A.lres + s);
  const int off = h0 + (s & 31);
  // the narrow rows of a skewed matrix are mostly short: their last group of
  // loads is issued at once (same sum, same bits)
  return row_acc_p<double, double, 8, 32>(A.val + off, A.ja + off, 32, ld_ro(A.irn + s), x - A.base, A.base);
}

__device__ __forceinline__ double row_dot(const HllView &A, int s, const double *__restrict__ x) {
  const int h = s / A.hksz;
  const int off = ld_ro(A.hkoffs + h) + (s - h * A.hksz);
  return row_acc<double, double, 8, 0>(A.val + off, A.ja + off, A.hksz, ld_ro(A.irn + s), x - A.base);
}

__device__ __forceinline__ double row_dot(const HllViewF &A, int s, const float *__restrict__ x) {
  const int h = s / A.hksz;
  const int off = ld_ro(A.hkoffs + h) + (s - h * A.hksz);
  if (A.hksz == 32)
    return row_acc<float, float, 8, 32>(A.val + off, A.ja + off, 32, ld_ro(A.irn + s), x - A.base);
  return row_acc<float, float, 8, 0>(A.val + off, A.ja + off, A.hksz, ld_ro(A.irn + s), x - A.base);
}

__device__ __forceinline__ double row_dot(const EllView &A, int r, const double *__restrict__ x) {
  return row_acc<double, double, 8, 0>(A.val + r, A.ja + r, A.pitch, ld_ro(A.irn + r), x - A.base);
}

__device__ __forceinline__ double row_dot(const EllViewF &A, int r, const float *__restrict__ x) {
  return row_acc<float, float, 8, 0>(A.val + r, A.ja + r, A.pitch, ld_ro(A.irn + r), x - A.base);
}

__device__ __forceinline__ double row_dot(const CsrView &A, int r, const double *__restrict__ x) {
  const int b = ld_ro(A.irp + r) - A.base, e = ld_ro(A.irp + r + 1) - A.base;
  return row_acc<double, double, 4, 1>(A.val + b, A.ja + b, 1, e - b, x - A.base);
}

// sum_j |val(r,j)| over the stored entries (psb_spnrmi, for istop = 1)
__device__ __forceinline__ double row_abs_sum(const HllView &A, int s);
__device__ __forceinline__ double row_abs_sum(const Hll32View &A, int s) {
  return row_abs_sum(static_cast<const HllView &>(A), s);
}
__device__ __forceinline__ double row_abs_sum(const Hll32SView &A, int s) {
  return row_abs_sum(static_cast<const HllView &>(A), s);
}
__device__ __forceinline__ double row_abs_sum(const Hll32WView &A, int s) {
  return row_abs_sum(static_cast<const HllView &>(A), s);
}
__device__ __forceinline__ double row_abs_sum(const HllView &A, int s) {
  const int h = s / A.hksz, ii = s - h * A.hksz;
  const size_t off = (size_t)A.hkoffs[h] + ii;
  double t = 0.0;
  for (int j = 0, n = A.irn[s]; j < n; j++) t = radd(t, fabs(A.val[off + (size_t)j * A.hksz]));
  return t;
}
__device__ __forceinline__ double row_abs_sum(const EllView &A, int r) {
  double t = 0.0;
  for (int j = 0, n = A.irn[r]; j < n; j++) t = radd(t, fabs(A.val[(size_t)r + (size_t)j * A.pitch]));
  return t;
}
__device__ __forceinline__ double row_abs_sum(const CsrView &A, int r) {
  double t = 0.0;
  for (int k = A.irp[r] - A.base; k < A.irp[r + 1] - A.base; k++) t = radd(t, fabs(A.val[k]));
  return t;
}

__device__ __forceinline__ int out_row(const HllView &A, int s) { return A.perm ? ld_ro(A.perm + s) : s; }
__device__ __forceinline__ int out_row(const Hll32View &A, int s) { return A.perm ? ld_ro(A.perm + s) : s; }
__device__ __forceinline__ int out_row(const Hll32WView &A, int s) { return A.perm ? ld_ro(A.perm + s) : s; }
__device__ __forceinline__ int out_row(const Hll32SView &A, int s) { return A.perm ? ld_ro(A.perm + s) : s; }
__device__ __forceinline__ int out_row(const HllViewF &A, int s) { return A.perm ? ld_ro(A.perm + s) : s; }
__device__ __forceinline__ int out_row(const EllView &, int r) { return r; }
__device__ __forceinline__ int out_row(const EllViewF &, int r) { return r; }
__device__ __forceinline__ int out_row(const CsrView &, int r) { return r; }

HllView hll_view(const HllDevice *m);
// Releases the iteration graphs (and workspaces) the Krylov driver keeps
// between calls; called when the context is torn down.
void psbx_krylov_cache_clear();
// Finds the wide hacks of a hack-32 matrix after its arrays are written.
int psbx_hll_index_long(HllDevice *m);
// Row sums of the wide hacks of a hack-32 matrix into lres (two launches), to
// be launched before any row kernel that reads them with the same x; status
// (nullable) makes the kernels return at once when *status != 0.
int psbx_long_rows32(const Hll32WView &A, const double *x, const int *status, cudaStream_t st);
static inline Hll32View hll32_view(const HllView &v) {
  Hll32View w;
  static_cast<HllView &>(w) = v;
  return w;
}
static inline Hll32WView hll32w_view(const HllView &v) {
  Hll32WView w;
  static_cast<HllView &>(w) = v;
  return w;
}
static inline Hll32SView hll32s_view(const HllView &v) {
  Hll32SView w;
  static_cast<HllView &>(w) = v;
  return w;
}
// A hack-32 matrix with no wide hacks whose rows all hold at most
// PSBX_SHORT_ROW entries runs the short-row kernels (Hll32SView).
static inline bool hll_short_rows(const HllDevice *m) {
  return m->hackSize == 32 && m->nLong == 0 && m->maxRowLen >= 0 && m->maxRowLen <= PSBX_SHORT_ROW;
}

template <class View>
static inline int psbx_long_rows(const View &, const double *, const int *, cudaStream_t) { return 0; }
static inline int psbx_long_rows(const Hll32WView &A, const double *x, const int *status, cudaStream_t st) {
  return psbx_long_rows32(A, x, status, st);
}
EllView ell_view(const EllDevice *m);
CsrView csr_view(const CsrDevice *m);

// Plain SpMV launchers (psbx_spmv.cu); y = alpha*A*x + beta*y on the stream.
int psbx_launch_hll_spmv(const HllDevice *m, double alpha, const double *x, double beta, double *y,
                         cudaStream_t st);
int psbx_launch_hll_spmv_f32(const HllDevice *m, float alpha, const float *x, float beta, float *y,
                             cudaStream_t st);
int psbx_launch_ell_spmv_f32(const EllDevice *m, float alpha, const float *x, float beta, float *y,
                             cudaStream_t st);
int psbx_launch_ell_spmv(const EllDevice *m, double alpha, const double *x, double beta, double *y,
                         cudaStream_t st);
int psbx_launch_csr_spmv(const CsrDevice *m, double alpha, const double *x, double beta, double *y,
                         cudaStream_t st);
int psbx_launch_scale(int n, double beta, double *y, cudaStream_t st);
