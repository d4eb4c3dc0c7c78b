// psbx_trsv.cu -- triangular solve with a device CSR matrix,
// y = alpha * T^{-1} x, behind d_spsvCSRGDevice (cuda/fcusparse_fct.h:132-220,
// which calls cusparseSpSV; bound by cuda/d_cusparse_mod.F90 and called by
// psb_d_cuda_csrg_inner_vect_sv.F90:88 with beta == 0 and no transpose).
//
// T is the triangle the matrix's fill mode names (d_CSRGDeviceSetMatFillMode:
// 0 lower, 1 upper): entries on the other side of the diagonal are ignored;
// with diagonal type 1 (unit) the stored diagonal is ignored and taken as 1,
// with 0 (non-unit) row i is divided by its entry in column i.  Row i is
//   y(i) = (x(i) - sum_j a(i,j) y(j)) / a(i,i)
// with the sum over the row's triangle entries in stored order, a rounded
// multiply then a rounded add per entry, as the reference's CPU solve
// (base/serial/impl/psb_d_csr_impl.F90:890-940, inner_csrsv); alpha scales
// the solution afterwards (psb_d_csr_cssv, :862-873).  Beta is not used, as
// in cusparseSpSV.
//
// One launch, no analysis phase: a warp takes one row at a time from an
// atomic ticket, in dependency order (row t for lower, n-1-t for upper), so
// every row it waits for was taken by a warp that is already running; the
// lanes wait for the rows their entries read (a per-row flag holding the
// generation of the solve that finished it), form the products, and every
// lane adds them in stored order through shuffles.  A finished row publishes
// its value, then its flag with release order.  Every wait is bounded in
// time: past the bound the solve sets a timeout flag, every waiting warp
// stops waiting, and the call returns PSBX_TIMEOUT.
#include "psbx_internal.cuh"

#define TRSV_T 256
#define TRSV_WAIT_NS 2000000000ull  // 2 s for one row's dependencies

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__global__ void __launch_bounds__(TRSV_T) k_csr_trsv(int n, const int *__restrict__ irp, const int *__restrict__ ja,
                                                     const double *__restrict__ val, int base, int upper, int unit,
                                                     const double *x, double *y, unsigned *flag, unsigned *ctl,
                                                     unsigned gen) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(ctl, 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= (unsigned)n) return;
    const int i = upper ? n - 1 - (int)t : (int)t;
    const int b = irp[i] - base, e = irp[i + 1] - base;
    double acc = 0.0, d = 1.0;
    for (int k0 = b; k0 < e; k0 += 32) {
      const int k = k0 + lane;
      double p = 0.0;
      int use = 0;  // 1: a triangle entry; 2: the diagonal
      if (k < e) {
        const int c = ja[k] - base;
        if (c == i) {
          use = unit ? 0 : 2;
          if (!unit) d = val[k];
        } else if (upper ? c > i : c < i) {
          use = 1;
          if (c >= 0 && c < n) {
            if (ld_acquire_u32(flag + c) != gen) {
              const unsigned long long t0 = global_ns();
              while (ld_acquire_u32(flag + c) != gen) {
                if (*((volatile unsigned *)ctl + 1) != 0u) break;
                if (global_ns() - t0 > TRSV_WAIT_NS) {
                  atomicExch(ctl + 1, 1u);
                  break;
                }
                __nanosleep(32);
              }
            }
            p = rmul(val[k], __ldcg(y + c));
          }
        }
      }
      // the diagonal's value reaches every lane; the products are added in
      // stored order
      const unsigned dm = __ballot_sync(0xffffffffu, use == 2);
      if (dm) d = __shfl_sync(0xffffffffu, d, __ffs(dm) - 1);
      const unsigned um = __ballot_sync(0xffffffffu, use == 1);
      const int cnt = min(32, e - k0);
      for (int q = 0; q < cnt; q++) {
        const double pq = __shfl_sync(0xffffffffu, p, q);
        if (um & (1u << q)) acc = radd(acc, pq);
      }
    }
    if (lane == 0) {
      const double r = __dsub_rn(__ldcg(x + i), acc);
      __stcg(y + i, unit ? r : __ddiv_rn(r, d));
      st_release_u32(flag + i, gen);
    }
    __syncwarp();
  }
}

__global__ void k_trsv_scale(int n, double alpha, double *__restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = rmul(alpha, y[i]);
}

extern "C" {

// cuda/fcusparse_fct.h:465-471: nonzero until the first solve has set the
// matrix up for solving.
int d_CSRGIsNullSvBuffer(psbx_d_Cmat *Mat) {
  CsrDevice *m = Mat ? (CsrDevice *)Mat->mat : nullptr;
  if (!m) return 1;
  return m->svFlag == nullptr ? 1 : 0;
}

int d_spsvCSRGDevice(psbx_d_Cmat *Mat, double alpha, void *deviceX, double beta, void *deviceY) {
  (void)beta;
  CsrDevice *m = Mat ? (CsrDevice *)Mat->mat : nullptr;
  MultiVectDevice *x = (MultiVectDevice *)deviceX, *y = (MultiVectDevice *)deviceY;
  if (!m || !x || !y || x->elemType != SPGPU_TYPE_DOUBLE || y->elemType != SPGPU_TYPE_DOUBLE || x->size_ < m->m ||
      y->size_ < m->m || m->m != m->n)
    return SPGPU_UNSUPPORTED;
  const int n = m->m;
  if (n == 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  if (!m->svFlag) {
    PSBX_CK(cudaMalloc(&m->svFlag, sizeof(unsigned) * (size_t)n));
    PSBX_CK(cudaMalloc(&m->svCtl, sizeof(unsigned) * 2));
    PSBX_CK(cudaMemsetAsync(m->svFlag, 0, sizeof(unsigned) * (size_t)n, c.stream));
    m->svGen = 0;
  }
  if (++m->svGen == 0) {  // the generations wrapped: start the flags again
    PSBX_CK(cudaMemsetAsync(m->svFlag, 0, sizeof(unsigned) * (size_t)n, c.stream));
    m->svGen = 1;
  }
  PSBX_CK(cudaMemsetAsync(m->svCtl, 0, sizeof(unsigned) * 2, c.stream));
  const int blocksPerSM = c.maxThreadsPerMP / TRSV_T;
  const long long warps = (long long)n;
  long long g = (warps * 32 + TRSV_T - 1) / TRSV_T;
  const long long cap = (long long)c.sms * blocksPerSM;  // every block resident at once
  if (g > cap) g = cap;
  k_csr_trsv<<<(int)g, TRSV_T, 0, c.stream>>>(n, m->irp, m->ja, m->val, m->baseIndex, m->fillMode == 1,
                                               m->diagType == 1, (const double *)x->v_, (double *)y->v_,
                                               m->svFlag, m->svCtl, m->svGen);
  PSBX_LAUNCH_CK("k_csr_trsv");
  if (alpha != 1.0) {
    k_trsv_scale<<<psbx_grid_for(n, 256), 256, 0, c.stream>>>(n, alpha, (double *)y->v_);
    PSBX_LAUNCH_CK("k_trsv_scale");
  }
  unsigned timed_out = 0;
  PSBX_CK(cudaMemcpyAsync(&timed_out, m->svCtl + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, c.stream));
  PSBX_CK(cudaStreamSynchronize(c.stream));
  if (timed_out) {
    psbx_set_error("d_spsvCSRGDevice: a row waited past the bound for its dependencies");
    return PSBX_TIMEOUT;
  }
  return SPGPU_SUCCESS;
}

// base_cusparse_mod.F90:83-96 (cuda/fcusparse.c:44-70): the library needs
// no cuSPARSE handle; these succeed so that the Fortran initialisation runs.
int FcusparseCreate(void) { return psbx_ensure_init(); }
int FcusparseDestroy(void) { return SPGPU_SUCCESS; }

}  // extern "C"
