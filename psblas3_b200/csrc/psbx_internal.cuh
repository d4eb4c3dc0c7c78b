// psbx_internal.cuh -- shared device objects, context and device helpers of
// libpsbx (B200 / sm_100a).  Not part of the public C-ABI (include/psbx.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <atomic>

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
};

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
  // row blocks for the streaming kernel (built at upload)
  int *rowBlocks;    // nBlocks+1 row starts
  int nBlocks;
  int *longRows;     // rows handled by the warp-per-row kernel
  int nLong;
};

// ---------------------------------------------------------------------------
// Context: one per process (the reference keeps one global SPGPU handle).
// ---------------------------------------------------------------------------
#define PSBX_MAX_PART 4096     // partial-sum slots per reduction lane
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
};

PsbxCtx &psbx_ctx();             // lazily initialises on the current device
int psbx_ensure_init();          // 0 or error code
int psbx_cuda_status(cudaError_t e, const char *where);
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

struct CsrView {
  const double *val;
  const int *ja;
  const int *irp;
  int rows, base;
};

// Unrolled in-order accumulation over one row whose j-th entry sits at
// off + j*stride.  Loads of a group are issued before its adds.
template <class VT, class XT, int U>
__device__ __forceinline__ double row_acc_strided(const VT *__restrict__ val, const int *__restrict__ ja,
                                                  size_t off, size_t stride, int n,
                                                  const XT *__restrict__ xb) {
  double acc = 0.0;
  int j = 0;
  for (; j + U <= n; j += U) {
    int c[U];
    VT v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      c[u] = ld_stream(ja + off + (size_t)(j + u) * stride);
      v[u] = ld_stream(val + off + (size_t)(j + u) * stride);
    }
    XT xv[U];
#pragma unroll
    for (int u = 0; u < U; u++) xv[u] = ld_ro(xb + c[u]);
#pragma unroll
    for (int u = 0; u < U; u++) acc = radd(acc, rmul((double)v[u], (double)xv[u]));
  }
  for (; j < n; j++) {
    int c = ld_stream(ja + off + (size_t)j * stride);
    VT v = ld_stream(val + off + (size_t)j * stride);
    acc = radd(acc, rmul((double)v, (double)ld_ro(xb + c)));
  }
  return acc;
}

__device__ __forceinline__ double row_dot(const HllView &A, int s, const double *__restrict__ x) {
  const int h = s / A.hksz;
  const int ii = s - h * A.hksz;
  const size_t off = (size_t)ld_ro(A.hkoffs + h) + ii;
  const int n = ld_ro(A.irn + s);
  return row_acc_strided<double, double, 4>(A.val, A.ja, off, (size_t)A.hksz, n, x - A.base);
}

__device__ __forceinline__ double row_dot(const HllViewF &A, int s, const float *__restrict__ x) {
  const int h = s / A.hksz;
  const int ii = s - h * A.hksz;
  const size_t off = (size_t)ld_ro(A.hkoffs + h) + ii;
  const int n = ld_ro(A.irn + s);
  return row_acc_strided<float, float, 4>(A.val, A.ja, off, (size_t)A.hksz, n, x - A.base);
}

__device__ __forceinline__ double row_dot(const EllView &A, int r, const double *__restrict__ x) {
  const int n = ld_ro(A.irn + r);
  return row_acc_strided<double, double, 4>(A.val, A.ja, (size_t)r, (size_t)A.pitch, n, x - A.base);
}

__device__ __forceinline__ double row_dot(const CsrView &A, int r, const double *__restrict__ x) {
  const int b = ld_ro(A.irp + r) - A.base, e = ld_ro(A.irp + r + 1) - A.base;
  return row_acc_strided<double, double, 4>(A.val, A.ja, (size_t)b, 1, e - b, x - A.base);
}

// sum_j |val(r,j)| over the stored entries (psb_spnrmi, for istop = 1)
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
__device__ __forceinline__ int out_row(const HllViewF &A, int s) { return A.perm ? ld_ro(A.perm + s) : s; }
__device__ __forceinline__ int out_row(const EllView &, int r) { return r; }
__device__ __forceinline__ int out_row(const CsrView &, int r) { return r; }

HllView hll_view(const HllDevice *m);
EllView ell_view(const EllDevice *m);
CsrView csr_view(const CsrDevice *m);

// Plain SpMV launchers (psbx_spmv.cu); y = alpha*A*x + beta*y on the stream.
int psbx_launch_hll_spmv(const HllDevice *m, double alpha, const double *x, double beta, double *y,
                         cudaStream_t st);
int psbx_launch_hll_spmv_f32(const HllDevice *m, float alpha, const float *x, float beta, float *y,
                             cudaStream_t st);
int psbx_launch_ell_spmv(const EllDevice *m, double alpha, const double *x, double beta, double *y,
                         cudaStream_t st);
int psbx_launch_csr_spmv(const CsrDevice *m, double alpha, const double *x, double beta, double *y,
                         cudaStream_t st);
int psbx_launch_scale(int n, double beta, double *y, cudaStream_t st);
