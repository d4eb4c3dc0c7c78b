// psbx_spmv.cu -- sparse matrix-vector kernels y = alpha*A*x + beta*y for
// the HLL, ELL and CSR device formats (sm_100a).
//
// Replaces cuda/spgpu/kernels/hell_spmv_base_template.cuh (spgpuDhellspmv),
// ell_spmv_base_template.cuh (spgpuDellspmv) and the cuSPARSE call of
// cuda/fcusparse_fct.h:108-124 (CSRG).
//
// HLL / ELL: one thread per row, a warp per 32 consecutive rows of a hack.
// Entry j of the 32 rows of a warp is one contiguous 256-byte run of values
// and 128-byte run of indices, so every value/index load instruction of the
// warp is fully coalesced; they are read with the streaming (evict-first)
// policy so that the gathered x stays cached.  Each row accumulates its
// stored entries in order with a rounded multiply and a rounded add, which
// is the reference's `acc = acc + val*x(ja)` (psb_d_hll_csmv.f90:345-360)
// bit for bit; padding slots are not read (rows stop at irn).
//
// CSR: a block takes a run of whole rows holding at most CSR_TILE entries
// (the row blocks are built at upload).  Its threads load the run's values
// and indices coalesced, form the products val*x(ja) and park them in shared
// memory; then one thread per row adds its products in stored order -- the
// same bits as the reference's row loop.  Rows longer than CSR_TILE are cut
// into CSR_TILE-entry chunks handled by extra blocks of the same launch;
// their chunk sums combine in a fixed order, which differs from the
// sequential sum only by rounding (checked against a tolerance).
#include "psbx_internal.cuh"

#include <algorithm>
#include <vector>

#define SPMV_T 256
#define CSR_TILE 2048
#define CSR_ROWS 256
static_assert(CSR_TILE % SPMV_T == 0, "a CSR row block is a whole number of passes of the block");

HllView hll_view(const HllDevice *m) {
  HllView v;
  v.val = (const double *)m->cM;
  v.ja = m->rP;
  v.irn = m->rS;
  v.hkoffs = m->hackOffs;
  v.perm = m->perm;
  v.rows = m->rows;
  v.hksz = m->hackSize;
  v.base = m->baseIndex;
  const bool wide = m->hackSize == 32 && m->nLong > 0;
  v.longHacks = wide ? m->longHacks : nullptr;
  v.lres = wide ? m->lres : nullptr;
  v.nLong = wide ? m->nLong : 0;
  v.longW = m->effW;  // the threshold the list was built with
  v.wideBase = wide ? m->wideBase : nullptr;
  v.wchunk = wide ? m->wchunk : nullptr;
  v.wprod = wide ? m->wprod : nullptr;
  v.nWChunks = wide ? m->nWChunks : 0;
  v.wideSplit = wide ? m->wideSplit : 0;
  v.wpart = wide ? m->wpart : nullptr;
  v.wticket = wide ? m->wticket : nullptr;
  v.wcbase = wide ? m->wcbase : nullptr;
  return v;
}

// --------------------------------------------------------------- wide hacks
// A hack whose width exceeds longW would hold its warp for width/8 rounds of
// two dependent memory latencies (the head of a row-sorted power-law matrix),
// far longer than the rest of the product.  Its row sums are formed before
// the row kernel in two launches:
//  k_hll_wprod -- every product val*x(ja) of the wide hacks, WP_COLS entries
//    of the hack's 32 rows per block, all blocks at once, stored in wprod in
//    the values' layout (entry j of row r of wide hack i at wideBase[i]+32j+r);
//  k_hll_wsum -- one warp per wide hack; lane r adds row r's products in
//    entry order from 0, the same roundings as the thread-per-row sum, so
//    results are unchanged bit for bit.  The products stream through a ring
//    of WS_NBUF shared-memory buffers that cp.async fills WS_NBUF-1 chunks
//    ahead, so only the additions are serial.
#define WP_COLS 64
#define WS_COLS 64
#define WS_NBUF 6
#define WS_WARPS 1
#define WS_SMEM (WS_WARPS * WS_NBUF * WS_COLS * 32 * (int)sizeof(double))

__global__ void __launch_bounds__(256) k_hll_wprod(Hll32WView A, const double *__restrict__ x, const int *status) {
  if (status && *((volatile const int *)status) != 0) return;
  const int i = A.wchunk[2 * blockIdx.x], c0 = A.wchunk[2 * blockIdx.x + 1];
  const int h = A.longHacks[i];
  const int off = A.hkoffs[h];
  const int r = threadIdx.x & 31;
  const int s = h * 32 + r;
  const int len = s < A.rows ? A.irn[s] : 0;
  const double *xb = x - A.base;
  double *pb = A.wprod + A.wideBase[i];
  constexpr int PER = WP_COLS * 32 / 256;  // entries per thread
  int c[PER];
  double v[PER];
#pragma unroll
  for (int u = 0; u < PER; u++) {
    const int j = c0 + (threadIdx.x >> 5) + 8 * u;
    const bool ok = j < len;
    const size_t p = (size_t)off + (size_t)j * 32 + r;
    c[u] = ok ? ld_stream(A.ja + p) : A.base;
    v[u] = ok ? ld_stream(A.val + p) : 0.0;
  }
#pragma unroll
  for (int u = 0; u < PER; u++) {
    const int j = c0 + (threadIdx.x >> 5) + 8 * u;
    if (j < len) pb[(size_t)j * 32 + r] = rmul(v[u], ld_ro(xb + c[u]));
  }
}

// (no memory clobber: the ring is read only after the wait below, which has one)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(32 * WS_WARPS) k_hll_wsum(Hll32WView A, double *__restrict__ lres,
                                                            const int *status) {
  if (status && *((volatile const int *)status) != 0) return;
  extern __shared__ __align__(16) double ring[];  // WS_WARPS rings of WS_NBUF chunks
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * WS_WARPS + w;
  if (i >= A.nLong) return;  // whole warps only; the block has no barrier
  const int h = A.longHacks[i];
  const int width = (A.hkoffs[h + 1] - A.hkoffs[h]) >> 5;
  const int s = h * 32 + lane;
  const int len = s < A.rows ? A.irn[s] : 0;
  const double *pb = A.wprod + A.wideBase[i];
  double *buf = ring + (size_t)w * WS_NBUF * WS_COLS * 32;
  const int nch = (width + WS_COLS - 1) / WS_COLS;
  // chunk c = columns [c*WS_COLS, min(width, (c+1)*WS_COLS)): one contiguous
  // run of 32 doubles per column, copied as 16-byte pieces (16 per column),
  // piece k by lane k % 32; each chunk is one commit group
  auto issue = [&](int c) {
    if (c < nch) {
      const double *src = pb + (size_t)c * WS_COLS * 32;
      double *dst = buf + (c % WS_NBUF) * WS_COLS * 32;
      const int npiece = min(WS_COLS, width - c * WS_COLS) * 16;
      for (int k = lane; k < npiece; k += 32) cp_async16(dst + 2 * k, src + 2 * k);
    }
  };
#pragma unroll
  for (int c = 0; c < WS_NBUF - 1; c++) {
    issue(c);
    cp_async_commit();
  }
  double acc = 0.0;
  for (int c = 0; c < nch; c++) {
    cp_async_wait<WS_NBUF - 2>();  // chunk c has landed (this lane's pieces)
    __syncwarp();                  // ... every lane's; and chunk c-1 is consumed
    const double *b = buf + (c % WS_NBUF) * WS_COLS * 32 + lane;
    const int n = min(WS_COLS, len - c * WS_COLS);
    const int cn = c + WS_NBUF - 1;  // issued now, into chunk c-1's buffer
    if (n == WS_COLS && (cn + 1) * WS_COLS <= width) {
      // a whole chunk to add and a whole chunk to fetch: the copies are
      // issued between the additions, in the cycles the add chain waits
      const double *src = pb + (size_t)cn * WS_COLS * 32 + 2 * lane;
      double *dst = buf + (cn % WS_NBUF) * WS_COLS * 32 + 2 * lane;
      double t[WS_COLS];
#pragma unroll
      for (int u = 0; u < WS_COLS; u++) t[u] = b[u * 32];
#pragma unroll
      for (int u = 0; u < WS_COLS; u++) {
        acc = radd(acc, t[u]);
        if (u & 1) cp_async16(dst + 64 * (u >> 1), src + 64 * (u >> 1));
      }
    } else {
      issue(cn);
      int j = 0;
      for (; j + 8 <= n; j += 8) {
        double t[8];
#pragma unroll
        for (int u = 0; u < 8; u++) t[u] = b[(j + u) * 32];
#pragma unroll
        for (int u = 0; u < 8; u++) acc = radd(acc, t[u]);
      }
      for (; j < n; j++) acc = radd(acc, b[j * 32]);
    }
    cp_async_commit();
  }
  if (s < A.rows) lres[s] = acc;
}

// Split mode (psbx_hll_set_wide_split): the product blocks of the ordered
// path (WP_COLS columns of one wide hack each, every block at once), but
// each block sums its products instead of storing them.  Warp w of the
// block takes columns c0 + w + 8u (u < WP_COLS/8) of each of the hack's 32
// rows (lane = row), all their loads in flight; the block adds its 8 warps'
// sums in warp order into one partial per row; the last block of the hack
// (ticket) adds the hack's partials in column order into the row sums.  No
// product makes a round trip through memory and no row has a long serial
// chain; the sum order is not the stored order, so the row sum agrees with
// the sequential one to rounding (|dy_i| <= len_i u sum_j |a_ij x_j|).
// Block b of the split wide-hack sum (256 threads).  True in warp 0 of the
// hack's last block, which then holds the sum of row s (its lane's row) in t.
__device__ __forceinline__ bool wide_split_chunk(const Hll32WView &A, const double *__restrict__ x, int b, double &t,
                                                 int &s) {
  __shared__ double red[8][32];
  __shared__ bool last;
  const int i = A.wchunk[2 * b], c0 = A.wchunk[2 * b + 1];
  const int h = A.longHacks[i];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t off = (size_t)A.hkoffs[h] + lane;
  s = h * 32 + lane;
  const int len = s < A.rows ? A.irn[s] : 0;
  const double *xb = x - A.base;
  constexpr int PER = WP_COLS / 8;
  int c[PER];
  double v[PER], xv[PER];
#pragma unroll
  for (int u = 0; u < PER; u++) {
    const int j = c0 + w + 8 * u;
    const bool ok = j < len;
    c[u] = ok ? ld_stream(A.ja + off + (size_t)j * 32) : A.base;
    v[u] = ok ? ld_stream(A.val + off + (size_t)j * 32) : 0.0;
  }
#pragma unroll
  for (int u = 0; u < PER; u++) xv[u] = c0 + w + 8 * u < len ? ld_ro(xb + c[u]) : 0.0;
  double acc = 0.0;
#pragma unroll
  for (int u = 0; u < PER; u++)
    if (c0 + w + 8 * u < len) acc = radd(acc, rmul(v[u], xv[u]));
  red[w][lane] = acc;
  __syncthreads();
  if (w == 0) {
    double r = red[0][lane];
#pragma unroll
    for (int k = 1; k < 8; k++) r = radd(r, red[k][lane]);
    A.wpart[(size_t)b * 32 + lane] = r;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(A.wticket + i, 1u) == (unsigned)(A.wcbase[i + 1] - A.wcbase[i] - 1);
  __syncthreads();
  if (!last || w != 0) return false;
  __threadfence();
  t = 0.0;
  for (int k = A.wcbase[i]; k < A.wcbase[i + 1]; k++) t = radd(t, __ldcg(A.wpart + (size_t)k * 32 + lane));
  if (lane == 0) A.wticket[i] = 0;
  return true;
}

__global__ void __launch_bounds__(256) k_hll_wide_split(Hll32WView A, const double *__restrict__ x,
                                                        double *__restrict__ lres, const int *status) {
  if (status && *((volatile const int *)status) != 0) return;
  double t;
  int s;
  if (wide_split_chunk(A, x, blockIdx.x, t, s) && s < A.rows) lres[s] = t;
}

int psbx_long_rows32(const Hll32WView &A, const double *x, const int *status, cudaStream_t st) {
  if (A.nLong <= 0) return SPGPU_SUCCESS;
  if (A.wideSplit) {
    k_hll_wide_split<<<A.nWChunks, 256, 0, st>>>(A, x, const_cast<double *>(A.lres), status);
    PSBX_LAUNCH_CK("k_hll_wide_split");
    return SPGPU_SUCCESS;
  }
  k_hll_wprod<<<A.nWChunks, 256, 0, st>>>(A, x, status);
  PSBX_LAUNCH_CK("k_hll_wprod");
  k_hll_wsum<<<(A.nLong + WS_WARPS - 1) / WS_WARPS, 32 * WS_WARPS, WS_SMEM, st>>>(A, const_cast<double *>(A.lres),
                                                                                 status);
  PSBX_LAUNCH_CK("k_hll_wsum");
  return SPGPU_SUCCESS;
}

// Lists the hacks wider than the wide threshold (hack size 32) from the
// offsets, with their product offsets and product blocks, and allocates the
// product and row-sum buffers; called whenever an HLL object's arrays are
// (re)written.  The default threshold is PSBX_LONG_W or four times the mean
// hack width, whichever is larger: a matrix whose hacks are all about
// equally wide keeps the thread-per-row sums (the extra product traffic
// would cost more than the chains it saves).
int psbx_hll_index_long(HllDevice *m) {
  free(m->tplan);  // the arrays changed: the batch engine's tile plan is redone
  m->tplan = nullptr;
  m->ntplan = 0;
  free(m->hcmin);  // and the host-buffer SpMV's column ranges
  free(m->hcmax);
  m->hcmin = m->hcmax = nullptr;
  cudaFree(m->longHacks);
  cudaFree(m->lres);
  cudaFree(m->wideBase);
  cudaFree(m->wchunk);
  cudaFree(m->wprod);
  cudaFree(m->wpart);
  cudaFree(m->wticket);
  cudaFree(m->wcbase);
  m->longHacks = nullptr;
  m->lres = nullptr;
  m->wideBase = nullptr;
  m->wchunk = nullptr;
  m->wprod = nullptr;
  m->wpart = nullptr;
  m->wticket = nullptr;
  m->wcbase = nullptr;
  m->nLong = 0;
  m->nWChunks = 0;
  if (m->hackSize != 32 || m->rows <= 0 || !m->hackOffs || m->longW < 0) return SPGPU_SUCCESS;
  const int nh = (m->rows + 31) / 32;
  PsbxCtx &c = psbx_ctx();
  std::vector<int> hk((size_t)nh + 1);
  PSBX_CK(cudaMemcpyAsync(hk.data(), m->hackOffs, sizeof(int) * ((size_t)nh + 1), cudaMemcpyDeviceToHost, c.stream));
  PSBX_CK(cudaStreamSynchronize(c.stream));
  int lw = m->longW;
  if (lw == 0) {
    const long long mean = ((long long)hk[nh] / 32 + nh - 1) / nh;
    lw = (int)std::max<long long>(PSBX_LONG_W, 4 * mean);
  }
  m->effW = lw;
  // widest first: their serial sums are the longest, so their warps start first
  std::vector<int> list;
  for (int h = 0; h < nh; h++)
    if (((hk[h + 1] - hk[h]) >> 5) > lw) list.push_back(h);
  std::stable_sort(list.begin(), list.end(), [&](int a, int b) { return hk[a + 1] - hk[a] > hk[b + 1] - hk[b]; });
  std::vector<int> wide, base(1, 0), chunks, cbase(1, 0);
  for (int h : list) {
    const int w = (hk[h + 1] - hk[h]) >> 5;
    for (int c0 = 0; c0 < w; c0 += WP_COLS) {
      chunks.push_back((int)wide.size());
      chunks.push_back(c0);
    }
    wide.push_back(h);
    base.push_back(base.back() + w * 32);
    cbase.push_back((int)(chunks.size() / 2));
  }
  if (wide.empty()) return SPGPU_SUCCESS;
  PSBX_CK(cudaMalloc(&m->longHacks, sizeof(int) * wide.size()));
  PSBX_CK(cudaMalloc(&m->lres, sizeof(double) * (size_t)m->rows));
  PSBX_CK(cudaMalloc(&m->wideBase, sizeof(int) * base.size()));
  PSBX_CK(cudaMalloc(&m->wchunk, sizeof(int) * chunks.size()));
  PSBX_CK(cudaMalloc(&m->wprod, sizeof(double) * (size_t)base.back()));
  PSBX_CK(cudaMalloc(&m->wpart, sizeof(double) * 32 * (chunks.size() / 2)));
  PSBX_CK(cudaMalloc(&m->wticket, sizeof(unsigned) * wide.size()));
  PSBX_CK(cudaMalloc(&m->wcbase, sizeof(int) * cbase.size()));
  PSBX_CK(cudaMemsetAsync(m->wticket, 0, sizeof(unsigned) * wide.size(), c.stream));
  PSBX_CK(cudaMemcpyAsync(m->wcbase, cbase.data(), sizeof(int) * cbase.size(), cudaMemcpyHostToDevice, c.stream));
  PSBX_CK(cudaMemcpyAsync(m->longHacks, wide.data(), sizeof(int) * wide.size(), cudaMemcpyHostToDevice, c.stream));
  PSBX_CK(cudaMemcpyAsync(m->wideBase, base.data(), sizeof(int) * base.size(), cudaMemcpyHostToDevice, c.stream));
  PSBX_CK(cudaMemcpyAsync(m->wchunk, chunks.data(), sizeof(int) * chunks.size(), cudaMemcpyHostToDevice, c.stream));
  PSBX_CK(cudaStreamSynchronize(c.stream));
  PSBX_CK(cudaFuncSetAttribute(k_hll_wsum, cudaFuncAttributeMaxDynamicSharedMemorySize, WS_SMEM));
  m->nLong = (int)wide.size();
  m->nWChunks = (int)(chunks.size() / 2);
  return SPGPU_SUCCESS;
}

EllView ell_view(const EllDevice *m) {
  EllView v;
  v.val = (const double *)m->cM;
  v.ja = m->rP;
  v.irn = m->rS;
  v.rows = m->rows;
  v.pitch = m->pitch;
  v.base = m->baseIndex;
  return v;
}

CsrView csr_view(const CsrDevice *m) {
  CsrView v;
  v.val = m->val;
  v.ja = m->ja;
  v.irp = m->irp;
  v.rows = m->m;
  v.base = m->baseIndex;
  return v;
}

// --------------------------------------------------------------- row kernels
// MODE 0: y = alpha*acc + beta*y ; MODE 1: beta == 0, y not read.
template <class View, int MODE>
__global__ void __launch_bounds__(SPMV_T) k_spmv_rows(View A, double alpha, const double *__restrict__ x,
                                                      double beta, double *__restrict__ y) {
  const int s = blockIdx.x * SPMV_T + threadIdx.x;
  if (s >= A.rows) return;
  const double acc = row_dot(A, s, x);
  const int r = out_row(A, s);
  const double t = rmul(alpha, acc);
  y[r] = MODE == 1 ? t : radd(t, rmul(beta, y[r]));
}

template <int MODE>
__global__ void __launch_bounds__(SPMV_T) k_hll_spmv_f32(HllViewF A, float alpha, const float *__restrict__ x,
                                                         float beta, float *__restrict__ y) {
  const int s = blockIdx.x * SPMV_T + threadIdx.x;
  if (s >= A.rows) return;
  const float acc = (float)row_dot(A, s, x);
  const int r = out_row(A, s);
  const float t = rmulf(alpha, acc);
  y[r] = MODE == 1 ? t : raddf(t, rmulf(beta, y[r]));
}

// Skewed matrices (hack size 32 with wide hacks: a row-sorted power-law
// matrix) are mostly rows of 1-4 entries, for which one row per thread is a
// chain of dependent round trips with little in flight.  Here a thread
// takes R adjacent rows of a hack -- entry j of two of them is one double2
// (values) and one int2 (indices), so a warp load moves 512 bytes -- and
// each row still adds its own entries in stored order (the same bits as
// k_spmv_rows).
#ifndef PSBX_HLL_R
#define PSBX_HLL_R 2
#endif
#ifndef PSBX_HLL_U
#define PSBX_HLL_U 4
#endif
template <int U, int R>
__device__ __forceinline__ void rgroup64(const HllView &A, int off, const int (&len)[R],
                                         const double *__restrict__ x, double (&acc)[R]) {
  static_assert(R % 2 == 0 && 32 % R == 0, "R adjacent rows of one hack, in pairs");
  const double *vp = A.val + off;
  const int *jp = A.ja + off;
  const double *xb = x - A.base;
  int n = 0;
#pragma unroll
  for (int r = 0; r < R; r++) {
    n = max(n, len[r]);
    acc[r] = 0.0;
  }
  for (int j = 0; j < n; j += U) {
    int2 c[U][R / 2];
    double2 v[U][R / 2];
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int q = 0; q < R / 2; q++) {
        const bool ok = j + u < n;
        c[u][q] = ok ? ld_stream((const int2 *)(jp + (j + u) * 32 + 2 * q)) : make_int2(A.base, A.base);
        v[u][q] = ok ? ld_stream((const double2 *)(vp + (j + u) * 32 + 2 * q)) : make_double2(0.0, 0.0);
      }
    double xv[U][R];
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int q = 0; q < R / 2; q++) {
        xv[u][2 * q] = j + u < len[2 * q] ? ld_ro(xb + c[u][q].x) : 0.0;
        xv[u][2 * q + 1] = j + u < len[2 * q + 1] ? ld_ro(xb + c[u][q].y) : 0.0;
      }
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int q = 0; q < R / 2; q++) {
        if (j + u < len[2 * q]) acc[2 * q] = radd(acc[2 * q], rmul(v[u][q].x, xv[u][2 * q]));
        if (j + u < len[2 * q + 1]) acc[2 * q + 1] = radd(acc[2 * q + 1], rmul(v[u][q].y, xv[u][2 * q + 1]));
      }
  }
}

template <int MODE>
__device__ __forceinline__ void put_row(int i, double alpha, double a, double beta, double *y) {
  const double t = rmul(alpha, a);
  y[i] = MODE == 1 ? t : radd(t, rmul(beta, y[i]));
}

// Rows of the narrow hacks, R per thread, from block `first` on; the rows
// of wide hacks come from lres (SPLIT 0) or are written by the wide blocks
// 0 .. first-1 of the same launch (SPLIT 1), which run the split sum and
// store y themselves: the long rows then overlap the short ones instead of
// running before them.
template <int MODE, int SPLIT>
__global__ void __launch_bounds__(SPMV_T) k_hll_rgroup(Hll32WView A, double alpha, const double *__restrict__ x,
                                                       double beta, double *__restrict__ y) {
  constexpr int R = PSBX_HLL_R;
  const int first = SPLIT ? A.nWChunks : 0;
  if (SPLIT && (int)blockIdx.x < first) {
    double t;
    int s;
    if (wide_split_chunk(A, x, blockIdx.x, t, s) && s < A.rows)
      put_row<MODE>(A.perm ? ld_ro(A.perm + s) : s, alpha, t, beta, y);
    return;
  }
  const int s0 = R * ((blockIdx.x - first) * SPMV_T + threadIdx.x);
  if (s0 >= A.rows) return;
  // the destinations are read with the offsets, not after the sums: one
  // round trip less per thread
  int dst[R];
#pragma unroll
  for (int r = 0; r < R; r++) dst[r] = A.perm && s0 + r < A.rows ? ld_ro(A.perm + s0 + r) : s0 + r;
  const int h0 = ld_ro(A.hkoffs + (s0 >> 5));
  double a[R];
  if (A.nLong > 0 && ((ld_ro(A.hkoffs + (s0 >> 5) + 1) - h0) >> 5) > A.longW) {
    if constexpr (SPLIT) {
      return;
    } else {
#pragma unroll
      for (int r = 0; r < R; r++) a[r] = s0 + r < A.rows ? __ldcg(A.lres + s0 + r) : 0.0;
    }
  } else {
    int len[R];
#pragma unroll
    for (int r = 0; r < R; r++) len[r] = s0 + r < A.rows ? ld_ro(A.irn + s0 + r) : 0;
    rgroup64<PSBX_HLL_U, R>(A, h0 + (s0 & 31), len, x, a);
  }
#pragma unroll
  for (int r = 0; r < R; r++)
    if (s0 + r < A.rows) put_row<MODE>(dst[r], alpha, a[r], beta, y);
}

// Two threads per row (the reference's two-thread HLL mode): lanes 2k and
// 2k+1 take the entries of row s at even and at odd positions, each adding
// its own in stored order, and the row sum is (even sum) + (odd sum) -- the
// tolerance mode only (|dy_i| <= len_i u sum_j |a_ij x_j|).  A warp holds 16
// rows of one hack, so the wide-hack test is the same for the whole warp.
template <int MODE, int SPLIT>
__global__ void __launch_bounds__(SPMV_T) k_hll_tpr2(Hll32WView A, double alpha, const double *__restrict__ x,
                                                     double beta, double *__restrict__ y) {
  const int first = SPLIT ? A.nWChunks : 0;
  if (SPLIT && (int)blockIdx.x < first) {
    double t;
    int s;
    if (wide_split_chunk(A, x, blockIdx.x, t, s) && s < A.rows)
      put_row<MODE>(A.perm ? ld_ro(A.perm + s) : s, alpha, t, beta, y);
    return;
  }
  const int g = (blockIdx.x - first) * SPMV_T + threadIdx.x;
  const int s = g >> 1, p = g & 1;
  if ((s & ~15) >= A.rows) return;  // the whole warp is past the last row
  const bool ok = s < A.rows;
  const int h0 = ld_ro(A.hkoffs + (s >> 5));
  const int dst = ok && p == 0 ? (A.perm ? ld_ro(A.perm + s) : s) : 0;
  if (A.nLong > 0 && ((ld_ro(A.hkoffs + (s >> 5) + 1) - h0) >> 5) > A.longW) {
    if constexpr (!SPLIT) {
      if (ok && p == 0) put_row<MODE>(dst, alpha, __ldcg(A.lres + s), beta, y);
    }
    return;
  }
  const int len = ok ? ld_ro(A.irn + s) : 0;
  const size_t off = (size_t)h0 + (s & 31);
  const double *xb = x - A.base;
  constexpr int U = 4;
  double acc = 0.0;
  for (int j = p; j < len; j += 2 * U) {
    int c[U];
    double v[U], xv[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const bool in = j + 2 * u < len;
      c[u] = in ? ld_stream(A.ja + off + (size_t)(j + 2 * u) * 32) : A.base;
      v[u] = in ? ld_stream(A.val + off + (size_t)(j + 2 * u) * 32) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; u++) xv[u] = j + 2 * u < len ? ld_ro(xb + c[u]) : 0.0;
#pragma unroll
    for (int u = 0; u < U; u++)
      if (j + 2 * u < len) acc = radd(acc, rmul(v[u], xv[u]));
  }
  const double odd = __shfl_xor_sync(0xffffffffu, acc, 1);
  if (ok && p == 0) put_row<MODE>(dst, alpha, radd(acc, odd), beta, y);
}

static int launch_tpr2(const Hll32WView &A, double alpha, const double *x, double beta, double *y,
                       cudaStream_t st) {
  if (A.rows <= 0) return SPGPU_SUCCESS;
  if (alpha == 0.0) return psbx_launch_scale(A.rows, beta, y, st);
  const int g = (int)(((long long)A.rows * 2 + SPMV_T - 1) / SPMV_T);
  if (A.nLong > 0 && A.wideSplit) {
    if (beta == 0.0)
      k_hll_tpr2<1, 1><<<A.nWChunks + g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
    else
      k_hll_tpr2<0, 1><<<A.nWChunks + g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
    PSBX_LAUNCH_CK("k_hll_tpr2");
    return SPGPU_SUCCESS;
  }
  int rc = psbx_long_rows32(A, x, nullptr, st);
  if (rc) return rc;
  if (beta == 0.0)
    k_hll_tpr2<1, 0><<<g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
  else
    k_hll_tpr2<0, 0><<<g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
  PSBX_LAUNCH_CK("k_hll_tpr2");
  return SPGPU_SUCCESS;
}

static int launch_rgroup(const Hll32WView &A, double alpha, const double *x, double beta, double *y,
                         cudaStream_t st) {
  static_assert(SPMV_T == 256, "the wide blocks of k_hll_rgroup run 256 threads");
  if (A.rows <= 0) return SPGPU_SUCCESS;
  if (alpha == 0.0) return psbx_launch_scale(A.rows, beta, y, st);
  const int g = ((A.rows + PSBX_HLL_R - 1) / PSBX_HLL_R + SPMV_T - 1) / SPMV_T;
  if (A.nLong > 0 && A.wideSplit) {
    if (beta == 0.0)
      k_hll_rgroup<1, 1><<<A.nWChunks + g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
    else
      k_hll_rgroup<0, 1><<<A.nWChunks + g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
    PSBX_LAUNCH_CK("k_hll_rgroup");
    return SPGPU_SUCCESS;
  }
  int rc = psbx_long_rows32(A, x, nullptr, st);
  if (rc) return rc;
  if (beta == 0.0)
    k_hll_rgroup<1, 0><<<g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
  else
    k_hll_rgroup<0, 0><<<g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
  PSBX_LAUNCH_CK("k_hll_rgroup");
  return SPGPU_SUCCESS;
}

template <class View>
static int launch_rows(const View &A, double alpha, const double *x, double beta, double *y, cudaStream_t st) {
  if (A.rows <= 0) return SPGPU_SUCCESS;
  if (alpha == 0.0) return psbx_launch_scale(A.rows, beta, y, st);
  int rc = psbx_long_rows(A, x, nullptr, st);
  if (rc) return rc;
  const int g = (A.rows + SPMV_T - 1) / SPMV_T;
  if (beta == 0.0)
    k_spmv_rows<View, 1><<<g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
  else
    k_spmv_rows<View, 0><<<g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
  PSBX_LAUNCH_CK("k_spmv_rows");
  return SPGPU_SUCCESS;
}

int psbx_launch_hll_spmv(const HllDevice *m, double alpha, const double *x, double beta, double *y,
                         cudaStream_t st) {
  if (m->elemType != SPGPU_TYPE_DOUBLE) return SPGPU_UNSUPPORTED;
  if (alpha == 0.0 && m->perm == nullptr) return psbx_launch_scale(m->rows, beta, y, st);
  if (m->hackSize == 32) {
    // row mapping: two threads per row only in the tolerance mode; two rows
    // per thread by default when there are wide hacks (skewed rows)
    const HllView v = hll_view(m);
    if (m->tpr == 2 && m->wideSplit) return launch_tpr2(hll32w_view(v), alpha, x, beta, y, st);
    if (m->tpr == -2 || m->tpr == 2 || (m->tpr == 0 && v.nLong > 0))
      return launch_rgroup(hll32w_view(v), alpha, x, beta, y, st);
    if (v.nLong > 0) return launch_rows(hll32w_view(v), alpha, x, beta, y, st);
    if (hll_short_rows(m)) return launch_rows(hll32s_view(v), alpha, x, beta, y, st);
    return launch_rows(hll32_view(v), alpha, x, beta, y, st);
  }
  return launch_rows(hll_view(m), alpha, x, beta, y, st);
}

// ------------------------------------------------- host-buffer SpMV
// y_host = alpha*A*x_host + beta*y_host with the copies overlapped with the
// product (psbx_hll_spmv_host).  The rows are cut into `chunks` blocks of
// whole hacks, x into blocks of the same size; x's blocks go up on one
// stream, in order, and row block k starts on the library stream once the
// block holding its largest column has arrived (from the per-hack column
// ranges, found once per matrix); its part of y goes down on a third stream
// as soon as it is done.  A banded matrix then costs about one copy of x
// up and one of y down running side by side, instead of copy, product and
// copy one after the other.  Each row is summed as by psbx_launch_hll_spmv
// (the same kernels over a row range), so the results are the same bits.

// Smallest and largest column of each hack (a warp per hack; rows of
// length 0 count for nothing: INT_MAX / INT_MIN).
__global__ void k_hll_colrange(HllView A, int nh, int *__restrict__ cmin, int *__restrict__ cmax) {
  const int h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (h >= nh) return;  // whole warps: blockDim is a multiple of 32
  const int s = h * 32 + lane;
  const int len = s < A.rows ? A.irn[s] : 0;
  const size_t off = (size_t)A.hkoffs[h] + lane;
  int lo = 0x7fffffff, hi = (int)0x80000000;
  for (int j = 0; j < len; j++) {
    const int c = A.ja[off + (size_t)j * 32];
    lo = min(lo, c);
    hi = max(hi, c);
  }
  lo = __reduce_min_sync(0xffffffffu, lo);
  hi = __reduce_max_sync(0xffffffffu, hi);
  if (lane == 0) {
    cmin[h] = lo;
    cmax[h] = hi;
  }
}

static int hll_colranges(HllDevice *m, cudaStream_t st) {
  if (m->hcmin) return SPGPU_SUCCESS;
  const int nh = (m->rows + 31) / 32;
  int *d = nullptr;
  PSBX_CK(cudaMalloc(&d, sizeof(int) * 2 * (size_t)nh));
  k_hll_colrange<<<(nh + 7) / 8, 256, 0, st>>>(hll_view(m), nh, d, d + nh);
  psbx_count_launch();
  cudaError_t e = cudaGetLastError();
  int *lo = (int *)malloc(sizeof(int) * (size_t)nh), *hi = (int *)malloc(sizeof(int) * (size_t)nh);
  if (e == cudaSuccess) e = cudaMemcpyAsync(lo, d, sizeof(int) * (size_t)nh, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hi, d + nh, sizeof(int) * (size_t)nh, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d);
  if (e != cudaSuccess) {
    free(lo);
    free(hi);
    return psbx_cuda_status(e, "hll column ranges");
  }
  m->hcmin = lo;
  m->hcmax = hi;
  return SPGPU_SUCCESS;
}

// rows [r0, r0 + nr) of a hack-32 matrix without wide hacks or permutation
static int launch_hll_rows_range(const HllDevice *m, int r0, int nr, double alpha, const double *x, double beta,
                                 double *y, cudaStream_t st) {
  HllView v = hll_view(m);
  v.irn += r0;
  v.hkoffs += r0 / 32;
  v.rows = nr;
  if (hll_short_rows(m)) return launch_rows(hll32s_view(v), alpha, x, beta, y + r0, st);
  return launch_rows(hll32_view(v), alpha, x, beta, y + r0, st);
}

extern "C" int psbx_hll_spmv_host(void *deviceMat, double alpha, const double *x, double beta, double *y,
                                  int chunks) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  HllDevice *m = (HllDevice *)deviceMat;
  if (!m || !x || !y || chunks < 0) return SPGPU_UNSUPPORTED;
  if (m->elemType != SPGPU_TYPE_DOUBLE) return SPGPU_UNSUPPORTED;
  const int n = m->rows, nc = m->cols;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  cudaStream_t st = c.stream;
  if (!m->hx) PSBX_CK(cudaMalloc(&m->hx, sizeof(double) * (size_t)(nc > 0 ? nc : 1)));
  if (!m->hy) PSBX_CK(cudaMalloc(&m->hy, sizeof(double) * (size_t)n));
  const size_t xb = sizeof(double) * (size_t)nc, yb = sizeof(double) * (size_t)n;
  const bool pipe = chunks != 1 && m->hackSize == 32 && m->nLong == 0 && !m->perm && alpha != 0.0;
  if (!pipe) {
    // one copy up, the product, one copy down, all on the library stream
    if (nc > 0) PSBX_CK(cudaMemcpyAsync(m->hx, x, xb, cudaMemcpyHostToDevice, st));
    if (beta != 0.0) PSBX_CK(cudaMemcpyAsync(m->hy, y, yb, cudaMemcpyHostToDevice, st));
    rc = psbx_launch_hll_spmv(m, alpha, m->hx, beta, m->hy, st);
    if (rc) return rc;
    PSBX_CK(cudaMemcpyAsync(y, m->hy, yb, cudaMemcpyDeviceToHost, st));
    PSBX_CK(cudaStreamSynchronize(st));
    return SPGPU_SUCCESS;
  }
  rc = hll_colranges(m, st);
  if (rc) return rc;
  const int nh = (n + 31) / 32;
  // 8 blocks by default: on the 27-point 200^3 operator (64 MB each way)
  // 1 / 2 / 4 / 8 / 16 / 32 / 64 blocks took 2.74 / 2.59 / 2.07 / 1.95 /
  // 2.03 / 2.20 / 2.44 ms -- each copy costs a fixed few microseconds
  int k = chunks == 0 ? 8 : chunks;
  if (k > nh) k = nh;
  const int hb = (nh + k - 1) / k;  // hacks per row block
  k = (nh + hb - 1) / hb;
  const int B = hb * 32;            // rows per block, and columns per block of x
  const int kx = nc > 0 ? (nc + B - 1) / B : 0;
  // y in page-locked host memory that the device can address (and beta = 0,
  // so y is only written): the row blocks store their part of y straight
  // into it over PCIe, in the other direction than x's copies, instead of
  // through a device copy and a copy down -- the two directions of the link
  // then carry the two vectors at the same time
  double *ydev = nullptr;
  if (beta == 0.0) {
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, y) == cudaSuccess && pa.type == cudaMemoryTypeHost && pa.devicePointer)
      ydev = (double *)pa.devicePointer;
    else
      cudaGetLastError();  // pageable memory: not an error, the copies are used
  }
  if (!c.h2d) PSBX_CK(cudaStreamCreateWithFlags(&c.h2d, cudaStreamNonBlocking));
  if (!c.d2h) PSBX_CK(cudaStreamCreateWithFlags(&c.d2h, cudaStreamNonBlocking));
  const size_t nev = (size_t)kx + 2 * (size_t)k + 1;
  while (c.xev.size() < nev) {
    cudaEvent_t e;
    PSBX_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    c.xev.push_back(e);
  }
  cudaEvent_t *ex = c.xev.data(), *ey = ex + kx, *ec = ey + k;  // x blocks, y blocks, row blocks
  cudaEvent_t e0 = c.xev[nev - 1];
  // the copies start after whatever the library stream still runs
  PSBX_CK(cudaEventRecord(e0, st));
  PSBX_CK(cudaStreamWaitEvent(c.h2d, e0, 0));
  PSBX_CK(cudaStreamWaitEvent(c.d2h, e0, 0));
  for (int b = 0; b < kx || b < k; b++) {
    if (b < kx) {
      const size_t c0 = (size_t)b * B, len = std::min((size_t)B, (size_t)nc - c0);
      PSBX_CK(cudaMemcpyAsync(m->hx + c0, x + c0, len * sizeof(double), cudaMemcpyHostToDevice, c.h2d));
      PSBX_CK(cudaEventRecord(ex[b], c.h2d));
    }
    if (b < k && beta != 0.0) {
      const size_t r0 = (size_t)b * B, len = std::min((size_t)B, (size_t)n - r0);
      PSBX_CK(cudaMemcpyAsync(m->hy + r0, y + r0, len * sizeof(double), cudaMemcpyHostToDevice, c.h2d));
      PSBX_CK(cudaEventRecord(ey[b], c.h2d));
    }
  }
  for (int b = 0; b < k; b++) {
    const int r0 = b * B, nr = std::min(B, n - r0);
    int hi = (int)0x80000000;
    for (int h = b * hb; h < std::min(nh, (b + 1) * hb); h++) hi = std::max(hi, m->hcmax[h]);
    if (kx > 0) {
      // the block of x holding the largest column, and at least x's block
      // b itself: its copy down may overwrite that host memory when x and y
      // are the same array
      int need = hi == (int)0x80000000 ? 0 : (hi - m->baseIndex) / B;
      need = std::max(need, b);
      need = need < 0 ? 0 : (need >= kx ? kx - 1 : need);
      PSBX_CK(cudaStreamWaitEvent(st, ex[need], 0));
    }
    if (beta != 0.0) PSBX_CK(cudaStreamWaitEvent(st, ey[b], 0));
    rc = launch_hll_rows_range(m, r0, nr, alpha, m->hx, beta, ydev ? ydev : m->hy, st);
    if (rc) return rc;
    if (ydev) continue;  // written in place
    PSBX_CK(cudaEventRecord(ec[b], st));
    PSBX_CK(cudaStreamWaitEvent(c.d2h, ec[b], 0));
    PSBX_CK(cudaMemcpyAsync(y + r0, m->hy + r0, (size_t)nr * sizeof(double), cudaMemcpyDeviceToHost, c.d2h));
  }
  // the library stream resumes after the last copy down; the call returns
  // with y on the host
  PSBX_CK(cudaEventRecord(e0, c.d2h));
  PSBX_CK(cudaStreamWaitEvent(st, e0, 0));
  PSBX_CK(cudaStreamSynchronize(c.d2h));
  PSBX_CK(cudaStreamSynchronize(st));
  return SPGPU_SUCCESS;
}

int psbx_launch_ell_spmv(const EllDevice *m, double alpha, const double *x, double beta, double *y,
                         cudaStream_t st) {
  if (m->dataType != SPGPU_TYPE_DOUBLE) return SPGPU_UNSUPPORTED;
  return launch_rows(ell_view(m), alpha, x, beta, y, st);
}

__global__ void k_f32_scale(int n, float beta, float *__restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = beta == 0.0f ? 0.0f : rmulf(beta, y[i]);
}

int psbx_launch_hll_spmv_f32(const HllDevice *m, float alpha, const float *x, float beta, float *y,
                             cudaStream_t st) {
  HllViewF A;
  A.val = m->elemType == SPGPU_TYPE_FLOAT ? (const float *)m->cM : m->cM32;
  if (!A.val) return SPGPU_UNSUPPORTED;
  A.ja = m->rP;
  A.irn = m->rS;
  A.hkoffs = m->hackOffs;
  A.perm = m->perm;
  A.rows = m->rows;
  A.hksz = m->hackSize;
  A.base = m->baseIndex;
  if (A.rows <= 0) return SPGPU_SUCCESS;
  if (alpha == 0.0f) {
    k_f32_scale<<<psbx_grid_for(A.rows, SPMV_T), SPMV_T, 0, st>>>(A.rows, beta, y);
    PSBX_LAUNCH_CK("k_f32_scale");
    return SPGPU_SUCCESS;
  }
  const int g = (A.rows + SPMV_T - 1) / SPMV_T;
  if (beta == 0.0f)
    k_hll_spmv_f32<1><<<g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
  else
    k_hll_spmv_f32<0><<<g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
  PSBX_LAUNCH_CK("k_hll_spmv_f32");
  return SPGPU_SUCCESS;
}

// FP32 ELL (spgpuSellspmv, ell_spmv_base_template.cuh with float values):
// the row sum is formed like the FP32 HLL one -- every product of two floats
// is exact in FP64, the products are added in FP64 in stored order and the
// sum is rounded to FP32 once -- then y = alpha*sum + beta*y in FP32.
template <int MODE>
__global__ void __launch_bounds__(SPMV_T) k_ell_spmv_f32(EllViewF A, float alpha, const float *__restrict__ x,
                                                         float beta, float *__restrict__ y) {
  const int r = blockIdx.x * SPMV_T + threadIdx.x;
  if (r >= A.rows) return;
  const float acc = (float)row_dot(A, r, x);
  const float t = rmulf(alpha, acc);
  y[r] = MODE == 1 ? t : raddf(t, rmulf(beta, y[r]));
}

int psbx_launch_ell_spmv_f32(const EllDevice *m, float alpha, const float *x, float beta, float *y,
                             cudaStream_t st) {
  if (m->dataType != SPGPU_TYPE_FLOAT) return SPGPU_UNSUPPORTED;
  EllViewF A;
  A.val = (const float *)m->cM;
  A.ja = m->rP;
  A.irn = m->rS;
  A.rows = m->rows;
  A.pitch = m->pitch;
  A.base = m->baseIndex;
  if (A.rows <= 0) return SPGPU_SUCCESS;
  if (alpha == 0.0f) {
    k_f32_scale<<<psbx_grid_for(A.rows, SPMV_T), SPMV_T, 0, st>>>(A.rows, beta, y);
    PSBX_LAUNCH_CK("k_f32_scale");
    return SPGPU_SUCCESS;
  }
  const int g = (A.rows + SPMV_T - 1) / SPMV_T;
  if (beta == 0.0f)
    k_ell_spmv_f32<1><<<g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
  else
    k_ell_spmv_f32<0><<<g, SPMV_T, 0, st>>>(A, alpha, x, beta, y);
  PSBX_LAUNCH_CK("k_ell_spmv_f32");
  return SPGPU_SUCCESS;
}

// --------------------------------------------------------------- CSR stream
// Block b holds rows rowBlocks[2b] .. rowBlocks[2b+1]-1; their entries (at
// most CSR_TILE) are contiguous in val/ja.
template <int MODE>
__device__ __forceinline__ void csr_stream_block(const CsrView &A, const int *__restrict__ rowBlocks, double alpha,
                                                 const double *__restrict__ x, double beta, double *__restrict__ y) {
  __shared__ double prod[CSR_TILE];
  const int r0 = rowBlocks[2 * blockIdx.x], r1 = rowBlocks[2 * blockIdx.x + 1];
  const int e0 = ld_ro(A.irp + r0) - A.base, e1 = ld_ro(A.irp + r1) - A.base;
  const int ne = e1 - e0;
  const double *xb = x - A.base;
  // all of a thread's index and value loads first, then its gathers (a block
  // holds at most CSR_TILE = CSR_U * SPMV_T entries)
  constexpr int CSR_U = CSR_TILE / SPMV_T;
  int c[CSR_U];
  double v[CSR_U];
#pragma unroll
  for (int u = 0; u < CSR_U; u++) {
    const int k = threadIdx.x + u * SPMV_T;
    c[u] = k < ne ? ld_stream(A.ja + e0 + k) : A.base;
    v[u] = k < ne ? ld_stream(A.val + e0 + k) : 0.0;
  }
#pragma unroll
  for (int u = 0; u < CSR_U; u++) {
    const int k = threadIdx.x + u * SPMV_T;
    if (k < ne) prod[k] = rmul(v[u], ld_ro(xb + c[u]));
  }
  __syncthreads();
  const int r = r0 + threadIdx.x;
  if (r < r1) {
    const int b = ld_ro(A.irp + r) - A.base - e0, e = ld_ro(A.irp + r + 1) - A.base - e0;
    double acc = 0.0;
    for (int k = b; k < e; k++) acc = radd(acc, prod[k]);
    const double t = rmul(alpha, acc);
    y[r] = MODE == 1 ? t : radd(t, rmul(beta, y[r]));
  }
}

// Chunks of rows longer than CSR_TILE entries run in the same launch as the
// row blocks (blocks nBlocks.. of the grid), so a skewed matrix does not wait
// for a second launch.  Chunk record (6 ints): row, first entry, end entry,
// index of the row's first chunk, chunks in the row, long-row ordinal.  A
// chunk block sums its entries (each thread in index order over a stride of
// the block, then a fixed shuffle tree), stores one partial, and the last
// chunk of the row to finish adds the row's partials in chunk order.
template <int MODE>
__device__ __forceinline__ void csr_chunk(const CsrView &A, const int *__restrict__ rec, double *__restrict__ part,
                                          unsigned *__restrict__ ticket, double alpha, const double *__restrict__ x,
                                          double beta, double *__restrict__ y) {
  __shared__ double sm[32];
  const int row = rec[0], e0 = rec[1], e1 = rec[2], first = rec[3], nch = rec[4], ord = rec[5];
  const double *xb = x - A.base;
  double acc[1] = {0.0};
  for (int k = e0 + threadIdx.x; k < e1; k += SPMV_T)
    acc[0] = radd(acc[0], rmul(ld_stream(A.val + k), ld_ro(xb + ld_stream(A.ja + k))));
  block_sum<1>(acc, sm);
  const int me = first + (e0 - (ld_ro(A.irp + row) - A.base)) / CSR_TILE;
  if (threadIdx.x == 0) part[me] = acc[0];
  if (psbx_last_block(ticket + ord, (unsigned)nch)) {
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int c = 0; c < nch; c++) s = radd(s, __ldcg(part + first + c));
      const double t = rmul(alpha, s);
      y[row] = MODE == 1 ? t : radd(t, rmul(beta, y[row]));
      ticket[ord] = 0;
    }
  }
}


// One launch: blocks [0, nBlocks) are row blocks, the rest long-row chunks.
template <int MODE>
__global__ void __launch_bounds__(SPMV_T) k_csr_adaptive(CsrView A, const int *__restrict__ rowBlocks, int nBlocks,
                                                         const int *__restrict__ chunks, double *__restrict__ part,
                                                         unsigned *__restrict__ ticket, double alpha,
                                                         const double *__restrict__ x, double beta,
                                                         double *__restrict__ y) {
  if ((int)blockIdx.x < nBlocks)
    csr_stream_block<MODE>(A, rowBlocks, alpha, x, beta, y);
  else
    csr_chunk<MODE>(A, chunks + 6 * (blockIdx.x - nBlocks), part, ticket, alpha, x, beta, y);
}

int psbx_launch_csr_spmv(const CsrDevice *m, double alpha, const double *x, double beta, double *y,
                         cudaStream_t st) {
  if (m->m <= 0) return SPGPU_SUCCESS;
  if (alpha == 0.0) return psbx_launch_scale(m->m, beta, y, st);
  CsrView A = csr_view(m);
  const int g = m->nBlocks + m->nChunks;
  if (g <= 0) return SPGPU_SUCCESS;
  if (beta == 0.0)
    k_csr_adaptive<1><<<g, SPMV_T, 0, st>>>(A, m->rowBlocks, m->nBlocks, m->chunks, m->chunkPart, m->chunkTicket,
                                            alpha, x, beta, y);
  else
    k_csr_adaptive<0><<<g, SPMV_T, 0, st>>>(A, m->rowBlocks, m->nBlocks, m->chunks, m->chunkPart, m->chunkTicket,
                                            alpha, x, beta, y);
  PSBX_LAUNCH_CK("k_csr_adaptive");
  return SPGPU_SUCCESS;
}

// Work partition for k_csr_adaptive (host side, from irp).  Greedy row
// blocks of <= CSR_TILE entries and <= CSR_ROWS rows; a row with more than
// CSR_TILE entries becomes ceil(len/CSR_TILE) chunk records.
void psbx_csr_partition(int m, const int *irp, std::vector<int> &rowBlocks, std::vector<int> &chunks, int *nLong) {
  rowBlocks.clear();
  chunks.clear();
  int nl = 0, nch = 0;
  int r = 0;
  while (r < m) {
    const int len = irp[r + 1] - irp[r];
    if (len > CSR_TILE) {
      const int k = (len + CSR_TILE - 1) / CSR_TILE;
      const int b = irp[r] - irp[0];
      for (int c = 0; c < k; c++) {
        const int e0 = b + c * CSR_TILE;
        const int e1 = e0 + CSR_TILE < b + len ? e0 + CSR_TILE : b + len;
        chunks.insert(chunks.end(), {r, e0, e1, nch, k, nl});
      }
      nch += k;
      nl++;
      r++;
      continue;
    }
    const int start = r;
    int cnt = 0;
    long long ent = 0;
    while (r < m && cnt < CSR_ROWS) {
      const int l = irp[r + 1] - irp[r];
      if (l > CSR_TILE || ent + l > CSR_TILE) break;
      ent += l;
      cnt++;
      r++;
    }
    rowBlocks.push_back(start);
    rowBlocks.push_back(r);
  }
  *nLong = nl;
}

#undef SPMV_T
