// psbx_formats.cu -- HLL, ELL and CSR device matrix objects, their
// host<->device copies, the COO->HLL / COO->ELL device scatter kernels and
// the device-side CSR->HLL builder.
//
// Replaces cuda/hlldev.c:34-540, cuda/elldev.c, the CSRG glue of
// cuda/fcusparse_fct.h and cuda/CUDA/psi_cuda_CopyCooTo{Hlg,Elg}.cuh.
#include "psbx_internal.cuh"

#include <stdlib.h>
#include <string.h>
#include <vector>

void psbx_csr_partition(int m, const int *irp, std::vector<int> &rowBlocks, std::vector<int> &chunks, int *nLong);

static inline size_t vsize(int t) { return t == SPGPU_TYPE_FLOAT ? 4 : 8; }

static int dmalloc(void **p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return psbx_cuda_status(e, "cudaMalloc");
  }
  return SPGPU_SUCCESS;
}

static int h2d(void *d, const void *h, size_t bytes) {
  if (!bytes) return SPGPU_SUCCESS;
  if (!d || !h) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  PSBX_CK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, c.stream));
  return SPGPU_SUCCESS;
}

static int d2h(void *h, const void *d, size_t bytes) {
  if (!bytes) return SPGPU_SUCCESS;
  if (!d || !h) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  PSBX_CK(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, c.stream));
  return SPGPU_SUCCESS;
}

static int sync_stream() {
  PSBX_CK(cudaStreamSynchronize(psbx_ctx().stream));
  return SPGPU_SUCCESS;
}

// ============================================================== HLL objects
extern "C" {

int FallocHllDevice(void **deviceMat, unsigned hksize, unsigned rows, unsigned nzeros, unsigned allocsize,
                    unsigned elementType, unsigned firstIndex) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  if (!deviceMat || hksize == 0) return SPGPU_UNSUPPORTED;
  if (elementType != SPGPU_TYPE_DOUBLE && elementType != SPGPU_TYPE_FLOAT) return SPGPU_UNSUPPORTED;
  HllDevice *m = (HllDevice *)calloc(1, sizeof(HllDevice));
  m->hackSize = (int)hksize;
  m->rows = (int)rows;
  m->nzt = (int)nzeros;
  m->allocsize = (int)allocsize;
  m->avgNzr = rows ? (int)((nzeros + rows - 1) / rows) : 0;  // hlldev.c:45
  m->baseIndex = (int)firstIndex;
  m->hackOffsLength = (int)((rows + hksize - 1) / hksize);
  m->elemType = (int)elementType;
  m->cols = (int)rows;
  m->maxRowLen = -1;
  m->wideSplit = 1;  // tolerance mode by default; psbx_hll_set_wide_split(m, 0) for the exact sums
  rc = dmalloc((void **)&m->rP, sizeof(int) * (size_t)allocsize);
  if (!rc) rc = dmalloc((void **)&m->rS, sizeof(int) * (size_t)rows);
  if (!rc) rc = dmalloc((void **)&m->diag, sizeof(int) * (size_t)rows);
  if (!rc) rc = dmalloc((void **)&m->hackOffs, sizeof(int) * (size_t)(m->hackOffsLength + 1));
  if (!rc) rc = dmalloc(&m->cM, vsize(m->elemType) * (size_t)allocsize);
  if (rc) {
    cudaFree(m->rP); cudaFree(m->rS); cudaFree(m->diag); cudaFree(m->hackOffs); cudaFree(m->cM);
    free(m);
    *deviceMat = nullptr;
    return rc;
  }
  *deviceMat = m;
  return SPGPU_SUCCESS;
}

void freeHllDevice(void *deviceMat) {
  HllDevice *m = (HllDevice *)deviceMat;
  if (!m) return;
  cudaStreamSynchronize(psbx_ctx().stream);
  cudaFree(m->rP);
  cudaFree(m->rS);
  cudaFree(m->diag);
  cudaFree(m->hackOffs);
  cudaFree(m->cM);
  if (m->cM32) cudaFree(m->cM32);
  if (m->perm) cudaFree(m->perm);
  cudaFree(m->longHacks);
  cudaFree(m->lres);
  cudaFree(m->wideBase);
  cudaFree(m->wchunk);
  cudaFree(m->wprod);
  cudaFree(m->wpart);
  cudaFree(m->wticket);
  cudaFree(m->wcbase);
  cudaFree(m->hx);
  cudaFree(m->hy);
  free(m->hcmin);
  free(m->hcmax);
  free(m->tplan);
  free(m);
}

int getHllDeviceParams(void *deviceMat, int *hksize, int *rows, int *nzeros, int *allocsize, int *hackOffsLength,
                       int *firstIndex, int *avgnzr) {
  HllDevice *m = (HllDevice *)deviceMat;
  if (!m) return SPGPU_UNSUPPORTED;
  *hackOffsLength = m->hackOffsLength;
  *hksize = m->hackSize;
  *nzeros = m->nzt;
  *allocsize = m->allocsize;
  *rows = m->rows;
  *avgnzr = m->avgNzr;
  *firstIndex = m->baseIndex;
  return SPGPU_SUCCESS;
}

// cuda/hlldev.c:34-49: the parameter block FallocHllDevice is built from.
psbx_HllDeviceParams bldHllDeviceParams(unsigned hksize, unsigned rows, unsigned nzeros, unsigned allocsize,
                                        unsigned elementType, unsigned firstIndex) {
  psbx_HllDeviceParams p;
  p.elementType = elementType;
  p.hackSize = hksize;
  p.rows = rows;
  p.avgNzr = rows ? (nzeros + rows - 1) / rows : 0;
  p.nzt = nzeros;
  p.allocsize = allocsize;
  p.firstIndex = firstIndex;
  return p;
}

static int hll_copy(void *deviceMat, void *val, int *ja, int *hkoffs, int *irn, int *idiag, bool write, int type) {
  HllDevice *m = (HllDevice *)deviceMat;
  if (!m || m->elemType != type) return SPGPU_UNSUPPORTED;
  size_t as = (size_t)m->allocsize, nr = (size_t)m->rows, nh = (size_t)m->hackOffsLength + 1;
  int rc;
  if (write) {
    rc = h2d(m->cM, val, as * vsize(type));
    if (!rc) rc = h2d(m->rP, ja, as * sizeof(int));
    if (!rc) rc = h2d(m->rS, irn, nr * sizeof(int));
    if (!rc) rc = h2d(m->diag, idiag, nr * sizeof(int));
    if (!rc) rc = h2d(m->hackOffs, hkoffs, nh * sizeof(int));
    if (!rc && irn) {
      int mx = 0;
      for (size_t i = 0; i < nr; i++) mx = irn[i] > mx ? irn[i] : mx;
      m->maxRowLen = mx;
    }
    if (!rc) rc = psbx_hll_index_long(m);
  } else {
    rc = d2h(val, m->cM, as * vsize(type));
    if (!rc) rc = d2h(ja, m->rP, as * sizeof(int));
    if (!rc) rc = d2h(irn, m->rS, nr * sizeof(int));
    if (!rc) rc = d2h(idiag, m->diag, nr * sizeof(int));
    if (!rc) rc = d2h(hkoffs, m->hackOffs, nh * sizeof(int));
  }
  if (!rc) rc = sync_stream();
  return rc;
}

int writeHllDeviceDouble(void *deviceMat, double *val, int *ja, int *hkoffs, int *irn, int *idiag) {
  return hll_copy(deviceMat, val, ja, hkoffs, irn, idiag, true, SPGPU_TYPE_DOUBLE);
}
int readHllDeviceDouble(void *deviceMat, double *val, int *ja, int *hkoffs, int *irn, int *idiag) {
  return hll_copy(deviceMat, val, ja, hkoffs, irn, idiag, false, SPGPU_TYPE_DOUBLE);
}
int writeHllDeviceFloat(void *deviceMat, float *val, int *ja, int *hkoffs, int *irn, int *idiag) {
  return hll_copy(deviceMat, val, ja, hkoffs, irn, idiag, true, SPGPU_TYPE_FLOAT);
}
int readHllDeviceFloat(void *deviceMat, float *val, int *ja, int *hkoffs, int *irn, int *idiag) {
  return hll_copy(deviceMat, val, ja, hkoffs, irn, idiag, false, SPGPU_TYPE_FLOAT);
}

int spmvHllDeviceDouble(void *deviceMat, double alpha, void *deviceX, double beta, void *deviceY) {
  HllDevice *m = (HllDevice *)deviceMat;
  MultiVectDevice *x = (MultiVectDevice *)deviceX, *y = (MultiVectDevice *)deviceY;
  if (!m || !x || !y || y->size_ < m->rows) return SPGPU_UNSUPPORTED;
  if (x->elemType != SPGPU_TYPE_DOUBLE || y->elemType != SPGPU_TYPE_DOUBLE) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  for (int v = 0; v < y->count_ && v < x->count_; v++) {
    int rc = psbx_launch_hll_spmv(m, alpha, (const double *)x->v_ + (size_t)v * x->pitch_, beta,
                                  (double *)y->v_ + (size_t)v * y->pitch_, c.stream);
    if (rc) return rc;
  }
  return SPGPU_SUCCESS;
}

int spmvHllDeviceFloat(void *deviceMat, float alpha, void *deviceX, float beta, void *deviceY) {
  HllDevice *m = (HllDevice *)deviceMat;
  MultiVectDevice *x = (MultiVectDevice *)deviceX, *y = (MultiVectDevice *)deviceY;
  if (!m || !x || !y || y->size_ < m->rows) return SPGPU_UNSUPPORTED;
  if (x->elemType != SPGPU_TYPE_FLOAT || y->elemType != SPGPU_TYPE_FLOAT) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  for (int v = 0; v < y->count_ && v < x->count_; v++) {
    int rc = psbx_launch_hll_spmv_f32(m, alpha, (const float *)x->v_ + (size_t)v * x->pitch_, beta,
                                      (float *)y->v_ + (size_t)v * y->pitch_, c.stream);
    if (rc) return rc;
  }
  return SPGPU_SUCCESS;
}

int psbx_hll_spmv_raw(void *deviceMat, double alpha, const double *x, double beta, double *y) {
  HllDevice *m = (HllDevice *)deviceMat;
  if (!m) return SPGPU_UNSUPPORTED;
  return psbx_launch_hll_spmv(m, alpha, x, beta, y, psbx_ctx().stream);
}

}  // extern "C"

// ---------------------------------------------- COO -> HLL scatter (device)
// psi_cuda_CopyCooToHlg.cuh:28-68: one thread per row copies the row's COO
// run into the column-major hack slice; padding takes the column of the
// first entry of row 2 and value 0; idiag = 1-based diagonal position.
// Rows past nr in the last hack (not written by the reference) get the same
// padding so the whole allocation is defined.
template <class T>
__global__ void k_coo_to_hll(int nr, int hksz, int base, int nrpad, const int *__restrict__ rS,
                             const int *__restrict__ hackOffs, const int *__restrict__ idisp,
                             const int *__restrict__ cja, const T *__restrict__ cval, int jc,
                             int *__restrict__ idiag, int *__restrict__ rP, T *__restrict__ cM) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrpad) return;
  const int h = i / hksz, lane = i - h * hksz;
  const int nzm = (hackOffs[h + 1] - hackOffs[h]) / hksz;
  size_t ir = (size_t)hackOffs[h] + lane;
  int rsz = 0, idval = 0;
  if (i < nr) {
    rsz = rS[i];
    const int p0 = idisp[i];
    for (int k = 0; k < rsz; k++) {
      const int c = cja[p0 + k];
      cM[ir] = cval[p0 + k];
      if (c == i + base) idval = k + base;
      rP[ir] = c;
      ir += hksz;
    }
    idiag[i] = idval;
  }
  for (int k = rsz; k < nzm; k++) {
    rP[ir] = jc;
    cM[ir] = T(0);
    ir += hksz;
  }
}

template <class T>
static int coo_to_hll(int nr, int nza, int hacksz, int noffs, int isz, int *irn, int *hoffs, int *idisp, int *ja,
                      T *val, void *deviceMat, int type) {
  HllDevice *m = (HllDevice *)deviceMat;
  if (!m || m->elemType != type || m->rows != nr || m->hackSize != hacksz) return SPGPU_UNSUPPORTED;
  if (noffs != m->hackOffsLength || isz > m->allocsize) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  int *dIdisp = nullptr, *dJa = nullptr;
  T *dVal = nullptr;
  int rc = dmalloc((void **)&dIdisp, sizeof(int) * (size_t)(nr + 1));
  if (!rc) rc = dmalloc((void **)&dJa, sizeof(int) * (size_t)nza);
  if (!rc) rc = dmalloc((void **)&dVal, sizeof(T) * (size_t)nza);
  if (!rc) rc = h2d(dVal, val, sizeof(T) * (size_t)nza);
  if (!rc) rc = h2d(dJa, ja, sizeof(int) * (size_t)nza);
  if (!rc) rc = h2d(m->rS, irn, sizeof(int) * (size_t)nr);
  if (!rc) rc = h2d(m->hackOffs, hoffs, sizeof(int) * (size_t)(noffs + 1));
  if (!rc) rc = h2d(dIdisp, idisp, sizeof(int) * (size_t)(nr + 1));
  if (!rc && nr > 0) {
    // "pick one valid value" (psi_cuda_CopyCooToHlg.cuh:57-59): column of
    // entry idisp(2); guarded for one-row matrices.
    int jc = 1;
    if (nza > 0) jc = ja[(nr > 1 && idisp[1] < nza) ? idisp[1] : 0];
    const int nrpad = noffs * hacksz;
    const int TB = 256;
    k_coo_to_hll<T><<<(nrpad + TB - 1) / TB, TB, 0, c.stream>>>(nr, hacksz, m->baseIndex, nrpad, m->rS, m->hackOffs,
                                                               dIdisp, dJa, dVal, jc, m->diag, m->rP, (T *)m->cM);
    psbx_count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "k_coo_to_hll");
    int mx = 0;
    for (int i = 0; i < nr; i++) mx = irn[i] > mx ? irn[i] : mx;
    m->maxRowLen = mx;
  }
  if (!rc) rc = sync_stream();
  if (!rc && type == SPGPU_TYPE_DOUBLE) rc = psbx_hll_index_long(m);
  cudaFree(dIdisp);
  cudaFree(dJa);
  cudaFree(dVal);
  return rc;
}

extern "C" int psiCopyCooToHlgDouble(int nr, int nc, int nza, int hacksz, int noffs, int isz, int *irn, int *hoffs,
                                     int *idisp, int *ja, double *val, void *deviceMat) {
  (void)nc;
  return coo_to_hll<double>(nr, nza, hacksz, noffs, isz, irn, hoffs, idisp, ja, val, deviceMat, SPGPU_TYPE_DOUBLE);
}

extern "C" int psiCopyCooToHlgFloat(int nr, int nc, int nza, int hacksz, int noffs, int isz, int *irn, int *hoffs,
                                    int *idisp, int *ja, float *val, void *deviceMat) {
  (void)nc;
  return coo_to_hll<float>(nr, nza, hacksz, noffs, isz, irn, hoffs, idisp, ja, val, deviceMat, SPGPU_TYPE_FLOAT);
}

// ------------------------------------------------ CSR (device) -> HLL build
// Restates psi_d_convert_hll_from_coo.f90:31-122 / psi_d_xtr_ell_from_coo
// on the device: irn from irp, hack widths = max irn in the hack, hkoffs by
// an exclusive scan, then the column-major slices are filled (a warp per
// hack for hack size 32, k_hll_fill32; k_hll_fill otherwise).
// Padding is the CPU converter's: last stored column of the row (the hack's
// first stored column for an empty row), value 0; rows past nr in the last
// hack: column nr, value 0 (psi_d_convert_hll_from_coo.f90:94-96).
// With perm, storage row s of the layout holds matrix row perm[s].
__global__ void k_hll_widths(int nr, int hksz, const int *__restrict__ irp, const int *__restrict__ perm,
                             int *__restrict__ irn, int *__restrict__ width, int nhacks) {
  const int h = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (h >= nhacks) return;
  int mx = 0;
  for (int ii = lane; ii < hksz; ii += 32) {
    const int s = h * hksz + ii;
    if (s < nr) {
      const int r = perm ? perm[s] : s;
      const int len = irp[r + 1] - irp[r];
      irn[s] = len;
      mx = max(mx, len);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
  if (lane == 0) width[h] = mx;
}

// Hack offsets: exclusive scan of width[0..n) * hksz in 64-bit, in three
// launches (chunk sums | scan of the chunk sums | chunk scans), plus the
// widest hack.  SCAN_CHUNK = 256 threads x 16 hacks.
enum { SCAN_T = 256, SCAN_PER = 16, SCAN_CHUNK = SCAN_T * SCAN_PER };

__device__ __forceinline__ long long block_excl_scan(long long v, long long *sh /* [SCAN_T/32] */,
                                                     long long &block_total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  long long incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) sh[wid] = incl;
  __syncthreads();
  long long before = 0, tot = 0;
  for (int w = 0; w < SCAN_T / 32; w++) {
    if (w < wid) before += sh[w];
    tot += sh[w];
  }
  __syncthreads();
  block_total = tot;
  return before + incl - v;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_chunks(int n, int hksz, const int *__restrict__ width,
                                                        long long *__restrict__ csum, int *__restrict__ cmax) {
  __shared__ long long sh[SCAN_T / 32];
  const int i0 = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_PER;
  long long s = 0;
  int m = 0;
#pragma unroll
  for (int k = 0; k < SCAN_PER; k++) {
    const int w = i0 + k < n ? width[i0 + k] : 0;
    s += (long long)w * hksz;
    m = max(m, w);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
  long long tot;
  block_excl_scan(s, sh, tot);
  if (threadIdx.x == 0) csum[blockIdx.x] = tot;
  if ((threadIdx.x & 31) == 0) atomicMax(cmax + blockIdx.x, m);
}

// one block: exclusive scan of the nb chunk sums in place; total and widest
// hack into res[0], res[1]
__global__ void __launch_bounds__(SCAN_T) k_scan_top(int nb, long long *__restrict__ csum,
                                                     const int *__restrict__ cmax, long long *__restrict__ res) {
  __shared__ long long sh[SCAN_T / 32];
  __shared__ long long carry;
  __shared__ int mx;
  if (threadIdx.x == 0) {
    carry = 0;
    mx = 0;
  }
  __syncthreads();
  for (int b0 = 0; b0 < nb; b0 += SCAN_T) {
    const int b = b0 + threadIdx.x;
    const long long v = b < nb ? csum[b] : 0;
    if (b < nb) atomicMax(&mx, cmax[b]);
    long long tot;
    const long long ex = block_excl_scan(v, sh, tot);
    if (b < nb) csum[b] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    res[0] = carry;
    res[1] = mx;
  }
}

__global__ void __launch_bounds__(SCAN_T) k_scan_apply(int n, int hksz, const int *__restrict__ width,
                                                       const long long *__restrict__ csum, int *__restrict__ offs) {
  __shared__ long long sh[SCAN_T / 32];
  const int i0 = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_PER;
  long long w[SCAN_PER];
  long long s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_PER; k++) {
    w[k] = i0 + k < n ? (long long)width[i0 + k] * hksz : 0;
    s += w[k];
  }
  long long tot;
  long long run = csum[blockIdx.x] + block_excl_scan(s, sh, tot);
#pragma unroll
  for (int k = 0; k < SCAN_PER; k++) {
    if (i0 + k < n) offs[i0 + k] = (int)run;
    run += w[k];
    if (i0 + k == n - 1) offs[n] = (int)run;
  }
}

// HLL fill for hack size 32: one warp per hack, lane = row of the hack.  A
// lane reads its row's start and length once and writes entry j of its row
// at hkoffs + j*32 + lane (each j a coalesced 32-entry run); padding as
// psi_d_xtr_ell_from_coo.f90:53-60 (the row's last column, or the hack's
// first stored column for an empty row; ja = nr past the last row), idiag the
// 1-based position of the diagonal or 0.
__global__ void __launch_bounds__(256) k_hll_fill32(int nr, int base, const int *__restrict__ irp,
                                                    const int *__restrict__ cja, const double *__restrict__ cval,
                                                    const int *__restrict__ perm, const int *__restrict__ irn,
                                                    const int *__restrict__ hkoffs, int nhacks,
                                                    int *__restrict__ hja, double *__restrict__ hval,
                                                    int *__restrict__ idiag) {
  const int h = blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (h >= nhacks) return;
  const int off = hkoffs[h];
  const int width = (hkoffs[h + 1] - off) >> 5;
  const int s = h * 32 + lane;
  const bool valid = s < nr;
  const int r = valid ? (perm ? perm[s] : s) : 0;
  const int len = valid ? irn[s] : 0;
  const int p0 = valid ? irp[r] - base : 0;
  // first stored column of the hack, needed only when one of its rows is empty
  const unsigned full = __ballot_sync(0xffffffffu, valid && len > 0);
  const unsigned rows = __ballot_sync(0xffffffffu, valid);
  int first_col = nr;
  if (full != rows && full != 0u) {
    const int f = __ffs(full) - 1;
    const int c0 = len > 0 ? cja[p0] : 0;
    first_col = __shfl_sync(0xffffffffu, c0, f);
  }
  int diag = 0;
  const int last = len > 0 ? cja[p0 + len - 1] : first_col;
  for (int j = 0; j < width; j++) {
    int col;
    double v;
    if (!valid) {
      col = nr;
      v = 0.0;
    } else if (j < len) {
      col = cja[p0 + j];
      v = cval[p0 + j];
      if (col == r + base) diag = j + 1;
    } else {
      col = last;
      v = 0.0;
    }
    hja[(size_t)off + (size_t)j * 32 + lane] = col;
    hval[(size_t)off + (size_t)j * 32 + lane] = v;
  }
  if (valid) idiag[s] = diag;
}

__global__ void k_hll_fill(int nr, int hksz, int base, const int *__restrict__ irp, const int *__restrict__ cja,
                           const double *__restrict__ cval, const int *__restrict__ perm,
                           const int *__restrict__ irn, const int *__restrict__ hkoffs, int *__restrict__ hja,
                           double *__restrict__ hval, int *__restrict__ idiag) {
  const int h = blockIdx.x;
  const int off = hkoffs[h];
  const int width = (hkoffs[h + 1] - off) / hksz;
  if (width == 0) {
    for (int ii = threadIdx.x; ii < hksz; ii += blockDim.x) {
      const int s = h * hksz + ii;
      if (s < nr) idiag[s] = 0;
    }
    return;
  }
  // first stored column of the hack (jac(1) in psi_d_xtr_ell_from_coo.f90:57)
  __shared__ int first_col;
  if (threadIdx.x == 0) {
    int fc = nr;  // unused when every row of the hack is empty (width 0)
    for (int ii = 0; ii < hksz; ii++) {
      const int s = h * hksz + ii;
      if (s >= nr) break;
      const int r = perm ? perm[s] : s;
      if (irp[r + 1] > irp[r]) {
        fc = cja[irp[r] - base];
        break;
      }
    }
    first_col = fc;
  }
  __syncthreads();
  const long long total = (long long)width * hksz;
  for (long long e = threadIdx.x; e < total; e += blockDim.x) {
    const int j = (int)(e / hksz), ii = (int)(e - (long long)j * hksz);
    const int s = h * hksz + ii;
    int col;
    double v;
    if (s < nr) {
      const int r = perm ? perm[s] : s;
      const int len = irn[s];
      const int p0 = irp[r] - base;
      if (j < len) {
        col = cja[p0 + j];
        v = cval[p0 + j];
        if (col == r + base) idiag[s] = j + 1;
      } else {
        col = len > 0 ? cja[p0 + len - 1] : first_col;
        v = 0.0;
      }
    } else {
      col = nr;
      v = 0.0;
    }
    hja[(size_t)off + e] = col;
    hval[(size_t)off + e] = v;
  }
}

__global__ void k_zero_int(int n, int *__restrict__ p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = 0;
}

extern "C" int psbx_hll_from_csr_device(void **deviceMat, int rows, int cols, int nnz, const int *d_irp,
                                        const int *d_ja, const double *d_val, int hksz, const int *d_perm) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  if (!deviceMat || rows < 0 || hksz <= 0 || !d_irp) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  const int nh = (rows + hksz - 1) / hksz;
  int *width = nullptr, *irn = nullptr, *hk = nullptr, *cmax = nullptr;
  long long *dtot = nullptr, *csum = nullptr;
  const int nb = (nh + SCAN_CHUNK - 1) / SCAN_CHUNK;
  rc = dmalloc((void **)&width, sizeof(int) * (size_t)(nh + 1));
  if (!rc) rc = dmalloc((void **)&irn, sizeof(int) * (size_t)(rows + 1));
  if (!rc) rc = dmalloc((void **)&hk, sizeof(int) * (size_t)(nh + 1));
  if (!rc) rc = dmalloc((void **)&dtot, 2 * sizeof(long long));
  if (!rc) rc = dmalloc((void **)&csum, sizeof(long long) * (size_t)(nb > 0 ? nb : 1));
  if (!rc) rc = dmalloc((void **)&cmax, sizeof(int) * (size_t)(nb > 0 ? nb : 1));
  long long res[2] = {0, 0};
  if (!rc && nh > 0) {
    PSBX_CK(cudaMemsetAsync(cmax, 0, sizeof(int) * (size_t)nb, c.stream));
    k_hll_widths<<<(nh + 7) / 8, 256, 0, c.stream>>>(rows, hksz, d_irp, d_perm, irn, width, nh);
    k_scan_chunks<<<nb, SCAN_T, 0, c.stream>>>(nh, hksz, width, csum, cmax);
    k_scan_top<<<1, SCAN_T, 0, c.stream>>>(nb, csum, cmax, dtot);
    k_scan_apply<<<nb, SCAN_T, 0, c.stream>>>(nh, hksz, width, csum, hk);
    psbx_count_launch(4);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "hll widths/scan");
    if (!rc) rc = d2h(res, dtot, 2 * sizeof(long long));
    if (!rc) rc = sync_stream();
  }
  const long long total = res[0];
  if (!rc && total > 0x7fffffffLL) rc = SPGPU_UNSUPPORTED;  // int32 offsets, as psb_ipk_
  HllDevice *m = nullptr;
  if (!rc) rc = FallocHllDevice((void **)&m, (unsigned)hksz, (unsigned)rows, (unsigned)nnz, (unsigned)total,
                                SPGPU_TYPE_DOUBLE, 1);
  if (!rc) {
    m->cols = cols;
    // the builder's own buffers become the object's irn / hkoffs
    cudaFree(m->rS);
    cudaFree(m->hackOffs);
    m->rS = irn;
    m->hackOffs = hk;
    irn = nullptr;
    hk = nullptr;
    if (d_perm) {
      rc = dmalloc((void **)&m->perm, sizeof(int) * (size_t)rows);
      if (!rc) PSBX_CK(cudaMemcpyAsync(m->perm, d_perm, sizeof(int) * (size_t)rows, cudaMemcpyDeviceToDevice, c.stream));
    }
  }
  if (!rc && nh > 0) {
    if (hksz == 32) {
      k_hll_fill32<<<(nh + 7) / 8, 256, 0, c.stream>>>(rows, 1, d_irp, d_ja, d_val, m->perm, m->rS, m->hackOffs, nh,
                                                       m->rP, (double *)m->cM, m->diag);
      psbx_count_launch(1);
    } else {
      k_zero_int<<<psbx_grid_for(rows, 256), 256, 0, c.stream>>>(rows, m->diag);
      k_hll_fill<<<nh, 256, 0, c.stream>>>(rows, hksz, 1, d_irp, d_ja, d_val, m->perm, m->rS, m->hackOffs, m->rP,
                                          (double *)m->cM, m->diag);
      psbx_count_launch(2);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "k_hll_fill");
  }
  // longest row (the widest hack), for the solver's choice of kernels
  if (!rc && m) m->maxRowLen = (int)res[1];
  if (!rc && m) rc = psbx_hll_index_long(m);
  cudaFree(width);
  cudaFree(irn);
  cudaFree(hk);
  cudaFree(dtot);
  cudaFree(csum);
  cudaFree(cmax);
  if (rc) {
    if (m) freeHllDevice(m);
    *deviceMat = nullptr;
    return rc;
  }
  *deviceMat = m;
  return SPGPU_SUCCESS;
}

__global__ void k_d2f(size_t n, const double *__restrict__ a, float *__restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

extern "C" int psbx_hll_make_single(void *deviceMat) {
  HllDevice *m = (HllDevice *)deviceMat;
  if (!m || m->elemType != SPGPU_TYPE_DOUBLE) return SPGPU_UNSUPPORTED;
  if (m->cM32) return SPGPU_SUCCESS;
  int rc = dmalloc((void **)&m->cM32, sizeof(float) * (size_t)m->allocsize);
  if (rc) return rc;
  PsbxCtx &c = psbx_ctx();
  k_d2f<<<psbx_grid_for(m->allocsize, 256), 256, 0, c.stream>>>((size_t)m->allocsize, (const double *)m->cM, m->cM32);
  PSBX_LAUNCH_CK("k_d2f");
  return sync_stream();
}

// ============================================================== ELL objects
static int ell_pitch(int rows) { return ((rows + 31) / 32) * 32; }  // spgpu/ell.c:33-37

extern "C" {

int FallocEllDevice(void **deviceMat, unsigned rows, unsigned maxRowSize, unsigned nnzeros, unsigned columns,
                    unsigned elementType, unsigned firstIndex) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  if (!deviceMat) return SPGPU_UNSUPPORTED;
  if (elementType != SPGPU_TYPE_DOUBLE && elementType != SPGPU_TYPE_FLOAT) return SPGPU_UNSUPPORTED;
  EllDevice *m = (EllDevice *)calloc(1, sizeof(EllDevice));
  m->rows = (int)rows;
  m->cMPitch = ell_pitch((int)rows);
  m->rPPitch = m->cMPitch;
  m->pitch = m->cMPitch;
  m->maxRowSize = (int)maxRowSize;
  m->avgRowSize = rows ? (int)((nnzeros + rows - 1) / rows) : 0;
  m->allocsize = m->maxRowSize * m->pitch;
  m->columns = (int)columns;
  m->baseIndex = (int)firstIndex;
  m->dataType = (int)elementType;
  rc = dmalloc((void **)&m->rS, sizeof(int) * (size_t)rows);
  if (!rc) rc = dmalloc((void **)&m->diag, sizeof(int) * (size_t)rows);
  if (!rc) rc = dmalloc((void **)&m->rP, sizeof(int) * (size_t)m->allocsize);
  if (!rc) rc = dmalloc(&m->cM, vsize(m->dataType) * (size_t)m->allocsize);
  if (rc) {
    cudaFree(m->rS); cudaFree(m->diag); cudaFree(m->rP); cudaFree(m->cM);
    free(m);
    *deviceMat = nullptr;
    return rc;
  }
  *deviceMat = m;
  return SPGPU_SUCCESS;
}

void freeEllDevice(void *deviceMat) {
  EllDevice *m = (EllDevice *)deviceMat;
  if (!m) return;
  cudaStreamSynchronize(psbx_ctx().stream);
  cudaFree(m->rS);
  cudaFree(m->diag);
  cudaFree(m->rP);
  cudaFree(m->cM);
  free(m);
}

void zeroEllDevice(void *deviceMat) {
  EllDevice *m = (EllDevice *)deviceMat;
  if (!m) return;
  cudaMemsetAsync(m->cM, 0, vsize(m->dataType) * (size_t)m->allocsize, psbx_ctx().stream);
  cudaStreamSynchronize(psbx_ctx().stream);
}

int getEllDevicePitch(void *deviceMat) { return ((EllDevice *)deviceMat)->pitch; }
int getEllDeviceMaxRowSize(void *deviceMat) { return ((EllDevice *)deviceMat)->maxRowSize; }

static int ell_copy(void *deviceMat, void *val, int *ja, int ldj, int *irn, int *idiag, bool write, int type) {
  EllDevice *m = (EllDevice *)deviceMat;
  if (!m || m->dataType != type) return SPGPU_UNSUPPORTED;
  if (ldj != m->pitch) return SPGPU_UNSUPPORTED;  // host arrays must be pitch x maxRowSize
  size_t as = (size_t)m->allocsize, nr = (size_t)m->rows, es = vsize(type);
  int rc;
  if (write) {
    rc = h2d(m->cM, val, as * es);
    if (!rc) rc = h2d(m->rP, ja, as * 4);
    if (!rc) rc = h2d(m->rS, irn, nr * 4);
    if (!rc) rc = h2d(m->diag, idiag, nr * 4);
  } else {
    rc = d2h(val, m->cM, as * es);
    if (!rc) rc = d2h(ja, m->rP, as * 4);
    if (!rc) rc = d2h(irn, m->rS, nr * 4);
    if (!rc) rc = d2h(idiag, m->diag, nr * 4);
  }
  if (!rc) rc = sync_stream();
  return rc;
}

int writeEllDeviceDouble(void *deviceMat, double *val, int *ja, int ldj, int *irn, int *idiag) {
  return ell_copy(deviceMat, val, ja, ldj, irn, idiag, true, SPGPU_TYPE_DOUBLE);
}
int readEllDeviceDouble(void *deviceMat, double *val, int *ja, int ldj, int *irn, int *idiag) {
  return ell_copy(deviceMat, val, ja, ldj, irn, idiag, false, SPGPU_TYPE_DOUBLE);
}
int writeEllDeviceFloat(void *deviceMat, float *val, int *ja, int ldj, int *irn, int *idiag) {
  return ell_copy(deviceMat, val, ja, ldj, irn, idiag, true, SPGPU_TYPE_FLOAT);
}
int readEllDeviceFloat(void *deviceMat, float *val, int *ja, int ldj, int *irn, int *idiag) {
  return ell_copy(deviceMat, val, ja, ldj, irn, idiag, false, SPGPU_TYPE_FLOAT);
}

// cuda/elldev.c:36-64.  The pitch reported is the one FallocEllDevice uses
// (rows rounded up to 32), so psb_d_cuda_elg_to_gpu's comparison of the two
// (psb_d_cuda_elg_to_gpu.F90:65) holds and the object is not reallocated on
// every upload.
psbx_EllDeviceParams getEllDeviceParams(unsigned rows, unsigned maxRowSize, unsigned nnzeros, unsigned columns,
                                        unsigned elementType, unsigned firstIndex) {
  psbx_EllDeviceParams p;
  p.elementType = elementType;
  p.pitch = (unsigned)ell_pitch((int)rows);
  p.rows = rows;
  p.columns = columns;
  p.maxRowSize = maxRowSize;
  p.avgRowSize = rows ? (nnzeros + rows - 1) / rows : 0;
  p.firstIndex = firstIndex;
  return p;
}

// elldev_mod.F90:175-185 declares these; the reference's C glue defines
// neither and no Fortran routine calls them.  They exist so the module
// links: the library keeps no ELL timer, so the time is always 0.
void resetEllTimer(void) {}
double getEllTimer(void) { return 0.0; }

int spmvEllDeviceFloat(void *deviceMat, float alpha, void *deviceX, float beta, void *deviceY) {
  EllDevice *m = (EllDevice *)deviceMat;
  MultiVectDevice *x = (MultiVectDevice *)deviceX, *y = (MultiVectDevice *)deviceY;
  if (!m || !x || !y || y->size_ < m->rows) return SPGPU_UNSUPPORTED;
  if (x->elemType != SPGPU_TYPE_FLOAT || y->elemType != SPGPU_TYPE_FLOAT) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  for (int v = 0; v < y->count_ && v < x->count_; v++) {
    int rc = psbx_launch_ell_spmv_f32(m, alpha, (const float *)x->v_ + (size_t)v * x->pitch_, beta,
                                      (float *)y->v_ + (size_t)v * y->pitch_, c.stream);
    if (rc) return rc;
  }
  return SPGPU_SUCCESS;
}

int spmvEllDeviceDouble(void *deviceMat, double alpha, void *deviceX, double beta, void *deviceY) {
  EllDevice *m = (EllDevice *)deviceMat;
  MultiVectDevice *x = (MultiVectDevice *)deviceX, *y = (MultiVectDevice *)deviceY;
  if (!m || !x || !y || y->size_ < m->rows) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  for (int v = 0; v < y->count_ && v < x->count_; v++) {
    int rc = psbx_launch_ell_spmv(m, alpha, (const double *)x->v_ + (size_t)v * x->pitch_, beta,
                                  (double *)y->v_ + (size_t)v * y->pitch_, c.stream);
    if (rc) return rc;
  }
  return SPGPU_SUCCESS;
}

}  // extern "C"

// COO -> ELL scatter on the device (psi_cuda_CopyCooToElg.cuh): padding as
// the CPU converter (last column of the row; first COO column if empty).
template <class T>
__global__ void k_coo_to_ell(int nr, int nzm, int pitch, int base, const int *__restrict__ rS,
                             const int *__restrict__ idisp, const int *__restrict__ cja,
                             const T *__restrict__ cval, int *__restrict__ idiag, int *__restrict__ rP,
                             T *__restrict__ cM) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pitch) return;
  if (i >= nr) {
    for (int k = 0; k < nzm; k++) {
      rP[(size_t)k * pitch + i] = 1;
      cM[(size_t)k * pitch + i] = T(0);
    }
    return;
  }
  const int rsz = rS[i], p0 = idisp[i];
  int idval = 0, c = cja[0];
  for (int k = 0; k < rsz; k++) {
    c = cja[p0 + k];
    if (c == i + base) idval = k + base;
    rP[(size_t)k * pitch + i] = c;
    cM[(size_t)k * pitch + i] = cval[p0 + k];
  }
  for (int k = rsz; k < nzm; k++) {
    rP[(size_t)k * pitch + i] = c;
    cM[(size_t)k * pitch + i] = T(0);
  }
  idiag[i] = idval;
}

template <class T>
static int coo_to_ell(int nr, int nza, int nzm, int *irn, int *idisp, int *ja, T *val, void *deviceMat, int type) {
  EllDevice *m = (EllDevice *)deviceMat;
  if (!m || m->dataType != type || m->rows != nr || nzm > m->maxRowSize) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  int *dIdisp = nullptr, *dJa = nullptr;
  T *dVal = nullptr;
  int rc = dmalloc((void **)&dIdisp, sizeof(int) * (size_t)(nr + 1));
  if (!rc) rc = dmalloc((void **)&dJa, sizeof(int) * (size_t)(nza > 0 ? nza : 1));
  if (!rc) rc = dmalloc((void **)&dVal, sizeof(T) * (size_t)(nza > 0 ? nza : 1));
  if (!rc) rc = h2d(dVal, val, sizeof(T) * (size_t)nza);
  if (!rc) rc = h2d(dJa, ja, sizeof(int) * (size_t)nza);
  if (!rc) rc = h2d(m->rS, irn, sizeof(int) * (size_t)nr);
  if (!rc) rc = h2d(dIdisp, idisp, sizeof(int) * (size_t)(nr + 1));
  if (!rc && nza == 0) {
    int one = 1;
    rc = h2d(dJa, &one, sizeof(int));
  }
  if (!rc && m->pitch > 0) {
    k_coo_to_ell<T><<<(m->pitch + 255) / 256, 256, 0, c.stream>>>(nr, m->maxRowSize, m->pitch, m->baseIndex, m->rS,
                                                                  dIdisp, dJa, dVal, m->diag, m->rP, (T *)m->cM);
    psbx_count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = psbx_cuda_status(e, "k_coo_to_ell");
  }
  if (!rc) rc = sync_stream();
  cudaFree(dIdisp);
  cudaFree(dJa);
  cudaFree(dVal);
  return rc;
}

extern "C" int psiCopyCooToElgDouble(int nr, int nc, int nza, int hacksz, int ldv, int nzm, int *irn, int *idisp,
                                     int *ja, double *val, void *deviceMat) {
  (void)nc; (void)hacksz; (void)ldv;
  return coo_to_ell<double>(nr, nza, nzm, irn, idisp, ja, val, deviceMat, SPGPU_TYPE_DOUBLE);
}

extern "C" int psiCopyCooToElgFloat(int nr, int nc, int nza, int hacksz, int ldv, int nzm, int *irn, int *idisp,
                                    int *ja, float *val, void *deviceMat) {
  (void)nc; (void)hacksz; (void)ldv;
  return coo_to_ell<float>(nr, nza, nzm, irn, idisp, ja, val, deviceMat, SPGPU_TYPE_FLOAT);
}

// dev_csputEllDevice{Double,Float} (cuda/elldev.c:607-644, kernel
// ell_csput_base.cuh): overwrite the values of entries already present in
// the pattern.  Entry i of the update names row ia[i] (1-based) and column
// ja[i] (compared as stored); a binary search over the row's stored columns
// (assumed ascending, as the converters leave them) finds the slot and its
// value becomes val[i].  Entries whose column is not stored, or whose row is
// outside the matrix, change nothing.  ia, ja, val are device multivectors.
template <class T>
__global__ void k_ell_csput(int nnz, int rows, int pitch, const int *__restrict__ rS, const int *__restrict__ rP,
                            T *__restrict__ cM, const int *__restrict__ aI, const int *__restrict__ aJ,
                            const T *__restrict__ aVal) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
    const int row = aI[i] - 1;
    if (row < 0 || row >= rows) continue;
    const int col = aJ[i];
    int lo = 0, hi = rS[row] - 1;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1;
      const int c = rP[(size_t)mid * pitch + row];
      if (c == col) {
        cM[(size_t)mid * pitch + row] = aVal[i];
        break;
      }
      if (c < col) lo = mid + 1;
      else hi = mid - 1;
    }
  }
}

template <class T>
static int ell_csput(void *deviceMat, int nnz, void *ia, void *ja, void *val, int type) {
  EllDevice *m = (EllDevice *)deviceMat;
  MultiVectDevice *I = (MultiVectDevice *)ia, *J = (MultiVectDevice *)ja, *V = (MultiVectDevice *)val;
  if (nnz <= 0) return SPGPU_SUCCESS;
  if (!m || !I || !J || !V || m->dataType != type || V->elemType != type || I->elemType != SPGPU_TYPE_INT ||
      J->elemType != SPGPU_TYPE_INT || nnz > I->size_ || nnz > J->size_ || nnz > V->size_)
    return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  k_ell_csput<T><<<psbx_grid_for(nnz, 256), 256, 0, c.stream>>>(nnz, m->rows, m->pitch, m->rS, m->rP, (T *)m->cM,
                                                                 (const int *)I->v_, (const int *)J->v_,
                                                                 (const T *)V->v_);
  PSBX_LAUNCH_CK("k_ell_csput");
  return SPGPU_SUCCESS;
}

extern "C" int dev_csputEllDeviceDouble(void *deviceMat, int nnz, void *ia, void *ja, void *val) {
  return ell_csput<double>(deviceMat, nnz, ia, ja, val, SPGPU_TYPE_DOUBLE);
}
extern "C" int dev_csputEllDeviceFloat(void *deviceMat, int nnz, void *ia, void *ja, void *val) {
  return ell_csput<float>(deviceMat, nnz, ia, ja, val, SPGPU_TYPE_FLOAT);
}

// ============================================================== CSR objects
static CsrDevice *CM(psbx_d_Cmat *M) { return M ? (CsrDevice *)M->mat : nullptr; }

static void csr_free_arrays(CsrDevice *m) {
  if (m->svFlag) cudaFree(m->svFlag);
  if (m->svCtl) cudaFree(m->svCtl);
  m->svFlag = nullptr; m->svCtl = nullptr; m->svGen = 0;
  cudaFree(m->val);
  cudaFree(m->irp);
  cudaFree(m->ja);
  if (m->rowBlocks) cudaFree(m->rowBlocks);
  if (m->chunks) cudaFree(m->chunks);
  if (m->chunkPart) cudaFree(m->chunkPart);
  if (m->chunkTicket) cudaFree(m->chunkTicket);
  m->val = nullptr; m->irp = nullptr; m->ja = nullptr; m->rowBlocks = nullptr;
  m->chunks = nullptr; m->chunkPart = nullptr; m->chunkTicket = nullptr;
}

extern "C" {

int d_CSRGDeviceAlloc(psbx_d_Cmat *Mat, int nr, int nc, int nz) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  if (!Mat || nr < 0 || nz < 0) return SPGPU_UNSUPPORTED;
  if (Mat->mat) d_CSRGDeviceFree(Mat);
  CsrDevice *m = (CsrDevice *)calloc(1, sizeof(CsrDevice));
  m->m = nr;
  m->n = nc;
  m->nz = nz;
  m->baseIndex = 1;
  rc = dmalloc((void **)&m->irp, sizeof(int) * (size_t)(nr + 1));
  if (!rc) rc = dmalloc((void **)&m->ja, sizeof(int) * (size_t)nz);
  if (!rc) rc = dmalloc((void **)&m->val, sizeof(double) * (size_t)nz);
  if (rc) {
    csr_free_arrays(m);
    free(m);
    return rc;
  }
  Mat->mat = m;
  return SPGPU_SUCCESS;
}

int d_CSRGDeviceFree(psbx_d_Cmat *Mat) {
  CsrDevice *m = CM(Mat);
  if (!m) return SPGPU_SUCCESS;
  cudaStreamSynchronize(psbx_ctx().stream);
  csr_free_arrays(m);
  free(m);
  Mat->mat = nullptr;
  return SPGPU_SUCCESS;
}

int d_CSRGDeviceGetParms(psbx_d_Cmat *Mat, int *nr, int *nc, int *nz) {
  CsrDevice *m = CM(Mat);
  if (!m) return SPGPU_UNSUPPORTED;
  *nr = m->m;
  *nc = m->n;
  *nz = m->nz;
  return SPGPU_SUCCESS;
}

// Matrix type / fill mode / diag type only matter for the triangular solve
// (spsv), which is outside this library; accepted and ignored.
// The descriptor settings of cuda/fcusparse_fct.h (cusparseSetMat*); the
// fill mode and diagonal type select the triangle d_spsvCSRGDevice solves.
int d_CSRGDeviceSetMatType(psbx_d_Cmat *Mat, int type) {
  CsrDevice *m = CM(Mat);
  if (!m || type < 0 || type > 3) return SPGPU_UNSUPPORTED;
  m->matType = type;
  return SPGPU_SUCCESS;
}
int d_CSRGDeviceSetMatFillMode(psbx_d_Cmat *Mat, int type) {
  CsrDevice *m = CM(Mat);
  if (!m || (type != 0 && type != 1)) return SPGPU_UNSUPPORTED;
  m->fillMode = type;
  return SPGPU_SUCCESS;
}
int d_CSRGDeviceSetMatDiagType(psbx_d_Cmat *Mat, int type) {
  CsrDevice *m = CM(Mat);
  if (!m || (type != 0 && type != 1)) return SPGPU_UNSUPPORTED;
  m->diagType = type;
  return SPGPU_SUCCESS;
}
int d_CSRGDeviceSetMatIndexBase(psbx_d_Cmat *Mat, int type) {
  CsrDevice *m = CM(Mat);
  if (!m || (type != 0 && type != 1)) return SPGPU_UNSUPPORTED;
  m->baseIndex = type;
  return SPGPU_SUCCESS;
}

int d_CSRGHost2Device(psbx_d_Cmat *Mat, int m_, int n, int nz, int *irp, int *ja, double *val) {
  CsrDevice *m = CM(Mat);
  if (!m || m_ != m->m || nz > m->nz || !irp) return SPGPU_UNSUPPORTED;
  (void)n;
  int rc = h2d(m->irp, irp, sizeof(int) * (size_t)(m_ + 1));
  if (!rc) rc = h2d(m->ja, ja, sizeof(int) * (size_t)nz);
  if (!rc) rc = h2d(m->val, val, sizeof(double) * (size_t)nz);
  if (rc) return rc;
  // work partition of the adaptive kernel
  std::vector<int> blocks, chunks;
  int nl = 0;
  psbx_csr_partition(m_, irp, blocks, chunks, &nl);
  if (m->rowBlocks) cudaFree(m->rowBlocks);
  if (m->chunks) cudaFree(m->chunks);
  if (m->chunkPart) cudaFree(m->chunkPart);
  if (m->chunkTicket) cudaFree(m->chunkTicket);
  m->rowBlocks = nullptr;
  m->chunks = nullptr;
  m->chunkPart = nullptr;
  m->chunkTicket = nullptr;
  const int nb = (int)blocks.size() / 2, nc = (int)chunks.size() / 6;
  rc = dmalloc((void **)&m->rowBlocks, sizeof(int) * (blocks.size() + 2));
  if (!rc) rc = dmalloc((void **)&m->chunks, sizeof(int) * (chunks.size() + 6));
  if (!rc) rc = dmalloc((void **)&m->chunkPart, sizeof(double) * (size_t)(nc + 1));
  if (!rc) rc = dmalloc((void **)&m->chunkTicket, sizeof(unsigned) * (size_t)(nl + 1));
  if (!rc) rc = h2d(m->rowBlocks, blocks.data(), sizeof(int) * blocks.size());
  if (!rc) rc = h2d(m->chunks, chunks.data(), sizeof(int) * chunks.size());
  if (!rc) PSBX_CK(cudaMemsetAsync(m->chunkTicket, 0, sizeof(unsigned) * (size_t)(nl + 1), psbx_ctx().stream));
  m->nBlocks = nb;
  m->nChunks = nc;
  m->nLong = nl;
  int mx = 0;
  for (int i = 0; i < m_; i++) mx = irp[i + 1] - irp[i] > mx ? irp[i + 1] - irp[i] : mx;
  m->maxRowLen = mx;
  if (!rc) rc = sync_stream();
  return rc;
}

int d_CSRGDevice2Host(psbx_d_Cmat *Mat, int m_, int n, int nz, int *irp, int *ja, double *val) {
  CsrDevice *m = CM(Mat);
  if (!m || m_ != m->m || nz > m->nz) return SPGPU_UNSUPPORTED;
  (void)n;
  int rc = d2h(irp, m->irp, sizeof(int) * (size_t)(m_ + 1));
  if (!rc) rc = d2h(ja, m->ja, sizeof(int) * (size_t)nz);
  if (!rc) rc = d2h(val, m->val, sizeof(double) * (size_t)nz);
  if (!rc) rc = sync_stream();
  return rc;
}

int d_spmvCSRGDevice(psbx_d_Cmat *Mat, double alpha, void *deviceX, double beta, void *deviceY) {
  CsrDevice *m = CM(Mat);
  MultiVectDevice *x = (MultiVectDevice *)deviceX, *y = (MultiVectDevice *)deviceY;
  if (!m || !x || !y || y->size_ < m->m) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  for (int v = 0; v < y->count_ && v < x->count_; v++) {
    int rc = psbx_launch_csr_spmv(m, alpha, (const double *)x->v_ + (size_t)v * x->pitch_, beta,
                                  (double *)y->v_ + (size_t)v * y->pitch_, c.stream);
    if (rc) return rc;
  }
  return SPGPU_SUCCESS;
}

}  // extern "C"

// ------------------------------------------------------------ HLL autotune
// Builds the HLL form of a device CSR matrix for each candidate layout and
// keeps the one with the fastest SpMV (CUDA events on the library stream,
// 2 warm-up and 5 timed products with x = 0): hack size 32, 64 or 128 and,
// for hack size 32, the width above which a hack takes the wide path
// (summed by all blocks in 64-column chunks): 32, 64, 128, 256, 1024 or
// never, and the threads per row of the narrow hacks: two rows per thread,
// one, or two threads per row (entries of even and odd position).  The
// result is in the tolerance mode (the default); psbx_hll_set_wide_split(m,
// 0) afterwards gives the stored-order sums, the same bits for every layout.
static int cst(cudaError_t e, const char *where) { return e == cudaSuccess ? 0 : psbx_cuda_status(e, where); }

static int time_hll(HllDevice *m, const double *x, double *y, double *ms) {
  PsbxCtx &c = psbx_ctx();
  cudaEvent_t e0, e1;
  PSBX_CK(cudaEventCreate(&e0));
  PSBX_CK(cudaEventCreate(&e1));
  int rc = SPGPU_SUCCESS;
  for (int k = 0; k < 2 && !rc; k++) rc = psbx_launch_hll_spmv(m, 1.0, x, 0.0, y, c.stream);
  if (!rc) rc = cst(cudaEventRecord(e0, c.stream), "autotune");
  for (int k = 0; k < 5 && !rc; k++) rc = psbx_launch_hll_spmv(m, 1.0, x, 0.0, y, c.stream);
  if (!rc) rc = cst(cudaEventRecord(e1, c.stream), "autotune");
  if (!rc) rc = cst(cudaEventSynchronize(e1), "autotune");
  float t = 0.0f;
  if (!rc) rc = cst(cudaEventElapsedTime(&t, e0, e1), "autotune");
  *ms = t / 5.0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

extern "C" int psbx_hll_autotune_from_csr_device(void **deviceMat, int rows, int cols, int nnz, const int *d_irp,
                                                 const int *d_ja, const double *d_val, const int *d_perm,
                                                 int *hksz, int *wide_w, double *ms) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  if (!deviceMat || rows <= 0 || !d_irp) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  double *x = nullptr, *y = nullptr;
  rc = dmalloc((void **)&x, sizeof(double) * (size_t)(cols > rows ? cols : rows));
  if (!rc) rc = dmalloc((void **)&y, sizeof(double) * (size_t)rows);
  if (!rc) rc = cst(cudaMemsetAsync(x, 0, sizeof(double) * (size_t)(cols > rows ? cols : rows), c.stream),
                    "autotune");
  HllDevice *best = nullptr;
  double best_ms = 0.0;
  int best_w = 0;
  static const int hks[] = {32, 64, 128};
  static const int ws[] = {32, 64, 128, 256, 1024, -1};
  const int nws = (int)(sizeof(ws) / sizeof(ws[0]));
  static const int tps[] = {-2, 1, 2};
  const int ntps = (int)(sizeof(tps) / sizeof(tps[0]));
  int best_tp = 0;
  for (int hi = 0; hi < 3 && !rc; hi++) {
    HllDevice *m = nullptr;
    rc = psbx_hll_from_csr_device((void **)&m, rows, cols, nnz, d_irp, d_ja, d_val, hks[hi], d_perm);
    if (rc) break;
    const int nw = hks[hi] == 32 ? nws : 1;
    const int ntp = hks[hi] == 32 ? ntps : 1;
    int m_best_w = 0, m_best_tp = 0;
    double m_best = -1.0;
    for (int wi = 0; wi < nw && !rc; wi++) {
      if (hks[hi] == 32) {
        // thresholds at or above the longest row leave nothing to sum by blocks
        if (ws[wi] > 0 && m->maxRowLen >= 0 && ws[wi] >= m->maxRowLen && wi + 1 < nw) continue;
        m->longW = ws[wi];
        rc = psbx_hll_index_long(m);
        if (rc) break;
      }
      for (int ti = 0; ti < ntp && !rc; ti++) {
        m->tpr = hks[hi] == 32 ? tps[ti] : 0;
        double t = 0.0;
        rc = time_hll(m, x, y, &t);
        if (!rc && (m_best < 0.0 || t < m_best)) {
          m_best = t;
          m_best_w = hks[hi] == 32 ? ws[wi] : 0;
          m_best_tp = m->tpr;
        }
      }
    }
    if (!rc && (!best || m_best < best_ms)) {
      if (best) freeHllDevice(best);
      best = m;
      best_ms = m_best;
      best_w = m_best_w;
      best_tp = m_best_tp;
    } else {
      freeHllDevice(m);
    }
  }
  if (!rc && best && best->hackSize == 32) {
    best->longW = best_w;
    best->tpr = best_tp;
    rc = psbx_hll_index_long(best);
  }
  cudaFree(x);
  cudaFree(y);
  if (rc) {
    if (best) freeHllDevice(best);
    *deviceMat = nullptr;
    return rc;
  }
  *deviceMat = best;
  if (hksz) *hksz = best->hackSize;
  if (wide_w) *wide_w = best->hackSize == 32 ? best_w : 0;
  if (ms) *ms = best_ms;
  return SPGPU_SUCCESS;
}

// Sets the wide-hack threshold of a hack-32 HLL matrix (0: default, < 0:
// never) and rebuilds its wide-hack lists; in the exact mode the results are
// the same bits for every threshold.
extern "C" int psbx_hll_set_wide(void *deviceMat, int wide_w) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  HllDevice *m = (HllDevice *)deviceMat;
  if (!m) return SPGPU_UNSUPPORTED;
  if (m->hackSize != 32) return wide_w == 0 ? SPGPU_SUCCESS : SPGPU_UNSUPPORTED;
  m->longW = wide_w;
  return psbx_hll_index_long(m);
}

// Tolerance mode (1, the default: wide hacks summed split over 8 warps, two
// threads per row allowed) or exact mode (0: every row in stored order, the
// CPU csmv's bits).  See k_hll_wide_split.
extern "C" int psbx_hll_set_wide_split(void *deviceMat, int split) {
  HllDevice *m = (HllDevice *)deviceMat;
  if (!m || (split != 0 && split != 1)) return SPGPU_UNSUPPORTED;
  m->wideSplit = split;
  return SPGPU_SUCCESS;
}

// Row mapping of the standalone HLL SpMV (hack size 32): 0 auto, 1 or 2
// threads per row, -2 two rows per thread.  Other hack sizes take 0 or 1.
extern "C" int psbx_hll_set_threads_per_row(void *deviceMat, int tpr) {
  HllDevice *m = (HllDevice *)deviceMat;
  if (!m || (tpr != 0 && tpr != 1 && tpr != 2 && tpr != -2)) return SPGPU_UNSUPPORTED;
  if (m->hackSize != 32 && tpr != 0 && tpr != 1) return SPGPU_UNSUPPORTED;
  m->tpr = tpr;
  return SPGPU_SUCCESS;
}

extern "C" int psbx_hll_get_layout(void *deviceMat, int *hksz, int *wide_w, int *split, int *tpr) {
  const HllDevice *m = (const HllDevice *)deviceMat;
  if (!m) return SPGPU_UNSUPPORTED;
  if (hksz) *hksz = m->hackSize;
  if (wide_w) *wide_w = m->longW;
  if (split) *split = m->wideSplit;
  if (tpr) *tpr = m->tpr;
  return SPGPU_SUCCESS;
}
