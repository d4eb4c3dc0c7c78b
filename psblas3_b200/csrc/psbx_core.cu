// psbx_core.cu -- process context, environment entry points and error
// handling.  Replaces cuda/cuda_util.c:220-440 and the SPGPU handle of
// cuda/spgpu/core.c:21-51 (one device, one stream per process).
#include "psbx_internal.cuh"

#include <stdlib.h>
#include <string.h>
#include <mutex>

static PsbxCtx g_ctx;
static std::atomic<uint64_t> g_launches{0};
static char g_last_error[512] = "";

void psbx_count_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

int psbx_cuda_status(cudaError_t e, const char *where) {
  snprintf(g_last_error, sizeof(g_last_error), "%s: %s", where, cudaGetErrorString(e));
  fprintf(stderr, "libpsbx: %s\n", g_last_error);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // clear the sticky-free allocation error
    return SPGPU_OUTOFMEMORY;
  }
  return SPGPU_UNSPECIFIED;
}

void psbx_set_error(const char *msg) {
  snprintf(g_last_error, sizeof(g_last_error), "%s", msg);
  fprintf(stderr, "libpsbx: %s\n", g_last_error);
}

static int ctx_create(int dev) {
  PsbxCtx &c = g_ctx;
  PSBX_CK(cudaSetDevice(dev));
  PSBX_CK(cudaGetDeviceProperties(&c.prop, dev));
  c.device = dev;
  c.sms = c.prop.multiProcessorCount;
  c.maxThreadsPerMP = c.prop.maxThreadsPerMultiProcessor;
  PSBX_CK(cudaStreamCreateWithFlags(&c.defaultStream, cudaStreamNonBlocking));
  c.stream = c.defaultStream;
  PSBX_CK(cudaMalloc(&c.d_part, sizeof(double) * 2 * PSBX_NLANES * PSBX_MAX_PART));
  PSBX_CK(cudaMalloc(&c.d_ticket, sizeof(unsigned) * 64));
  PSBX_CK(cudaMemset(c.d_ticket, 0, sizeof(unsigned) * 64));
  PSBX_CK(cudaMalloc(&c.d_res, sizeof(double) * 64));
  PSBX_CK(cudaHostAlloc(&c.h_res, sizeof(double) * 64, cudaHostAllocDefault));
  cudaMemPoolProps pp;
  memset(&pp, 0, sizeof(pp));
  pp.allocType = cudaMemAllocationTypePinned;
  pp.location.type = cudaMemLocationTypeDevice;
  pp.location.id = dev;
  PSBX_CK(cudaMemPoolCreate(&c.pool, &pp));
  uint64_t keep = PSBX_POOL_KEEP;
  PSBX_CK(cudaMemPoolSetAttribute(c.pool, cudaMemPoolAttrReleaseThreshold, &keep));
  c.init = true;
  return SPGPU_SUCCESS;
}

PsbxCtx &psbx_ctx() {
  if (!g_ctx.init) {
    int dev = 0;
    cudaGetDevice(&dev);
    ctx_create(dev);
  }
  return g_ctx;
}

int psbx_ensure_init() {
  if (g_ctx.init) return SPGPU_SUCCESS;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return psbx_cuda_status(e, "cudaGetDevice");
  return ctx_create(dev);
}

void psbx_noalloc_forget(void);

static void ctx_destroy() {
  psbx_noalloc_forget();
  PsbxCtx &c = g_ctx;
  if (!c.init) return;
  psbx_krylov_cache_clear();
  cudaStreamSynchronize(c.stream);
  cudaFree(c.d_part);
  cudaFree(c.d_ticket);
  cudaFree(c.d_res);
  cudaFreeHost(c.h_res);
  cudaStreamSynchronize(c.defaultStream);
  for (cudaEvent_t e : c.xev) cudaEventDestroy(e);
  if (c.h2d) cudaStreamDestroy(c.h2d);
  if (c.d2h) cudaStreamDestroy(c.d2h);
  if (c.pool) cudaMemPoolDestroy(c.pool);
  cudaStreamDestroy(c.defaultStream);
  c = PsbxCtx();
}

extern "C" {

uint64_t psbx_kernel_launches(void) { return g_launches.load(); }
const char *psbx_last_error(void) { return g_last_error; }

// cuda_util.c:220 -- select the device and create the handle.
int gpuInit(int dev) {
  if (g_ctx.init && g_ctx.device != dev) ctx_destroy();
  if (g_ctx.init) return SPGPU_SUCCESS;
  return ctx_create(dev);
}

void gpuClose(void) { ctx_destroy(); }

int setDevice(int dev) {
  cudaError_t e = cudaSetDevice(dev);
  return e == cudaSuccess ? SPGPU_SUCCESS : psbx_cuda_status(e, "cudaSetDevice");
}

int getDevice(void) {
  int d = -1;
  cudaGetDevice(&d);
  return d;
}

int getDeviceCount(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

static cudaDeviceProp &props() { return psbx_ctx().prop; }

int getDeviceHasUVA(void) { return props().unifiedAddressing; }
int DeviceHasUVA(void) { return props().unifiedAddressing; }
int getGPUMultiProcessors(void) { return props().multiProcessorCount; }
int getGPUMemoryBusWidth(void) { return props().memoryBusWidth; }
int getGPUMemoryClockRate(void) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMemoryClockRate, psbx_ctx().device);
  return v;
}
int getGPUWarpSize(void) { return props().warpSize; }
int getGPUMaxThreadsPerBlock(void) { return props().maxThreadsPerBlock; }
int getGPUMaxThreadsPerMP(void) { return props().maxThreadsPerMultiProcessor; }
int getGPUMaxRegistersPerBlock(void) { return props().regsPerBlock; }
void cpyGPUNameString(char *cstring) {
  strncpy(cstring, props().name, 255);
  cstring[255] = 0;
}

void cudaSync(void) {
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) psbx_cuda_status(e, "cudaSync");
}

// cuda_util.c:396 resets the device; here only this library's context is
// released (other users of the device are not affected).
void cudaReset(void) { ctx_destroy(); }

void *psb_cudaGetHandle(void) { return (void *)&psbx_ctx(); }
void psb_cudaCreateHandle(void) { psbx_ensure_init(); }
void psb_cudaDestroyHandle(void) { ctx_destroy(); }
void *psb_cudaGetStream(void) { return (void *)psbx_ctx().stream; }
void psb_cudaSetStream(void *stream) {
  PsbxCtx &c = psbx_ctx();
  c.stream = stream ? (cudaStream_t)stream : c.defaultStream;
}

// ---------------------------------------------------------------------------
// Plain device buffers: the "simple memory tools" of cuda/cuda_util.c:440-662
// (allocateInt/Float/Double, write*/read* whole, from an indexBase-based
// first entry, or m*n entries, free*), used by the Fortran vector types for
// their gather/scatter buffers (psb_d_cuda_vect_mod.F90:155-549).  Raw
// device pointers; copies run on the library stream and return when done.
// ---------------------------------------------------------------------------
static int buf_alloc(void **d, long long bytes) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  if (!d || bytes < 0) return SPGPU_UNSUPPORTED;
  cudaError_t e = cudaMalloc(d, bytes > 0 ? (size_t)bytes : 16);
  if (e != cudaSuccess) {
    *d = nullptr;
    return psbx_cuda_status(e, "allocate (device buffer)");
  }
  return SPGPU_SUCCESS;
}

static int buf_copy(void *dst, const void *src, long long bytes, cudaMemcpyKind kind) {
  if (bytes <= 0) return SPGPU_SUCCESS;
  if (!dst || !src) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  PSBX_CK(cudaMemcpyAsync(dst, src, (size_t)bytes, kind, c.stream));
  PSBX_CK(cudaStreamSynchronize(c.stream));
  return SPGPU_SUCCESS;
}

static void buf_free(void *d) {
  if (!d) return;
  if (g_ctx.init) cudaStreamSynchronize(g_ctx.stream);
  cudaFree(d);
}

// cudaHostRegister with the mapped flag, then the device alias of the host
// buffer (cuda_util.c:104-130).
static int map_host(void *buf, void **dp, long long bytes) {
  if (!buf || !dp || bytes <= 0) return SPGPU_UNSUPPORTED;
  PSBX_CK(cudaHostRegister(buf, (size_t)bytes, cudaHostRegisterMapped));
  PSBX_CK(cudaHostGetDevicePointer(dp, buf, 0));
  return SPGPU_SUCCESS;
}

#define PSBX_BUFFER_TOOLS(NAME, T)                                                                    \
  int allocate##NAME(void **d, int n) { return buf_alloc(d, (long long)n * sizeof(T)); }               \
  int allocateMulti##NAME(void **d, int m, int n) { return buf_alloc(d, (long long)m * n * sizeof(T)); } \
  int write##NAME(void *d, T *h, int n) {                                                               \
    return buf_copy(d, h, (long long)n * sizeof(T), cudaMemcpyHostToDevice);                           \
  }                                                                                                     \
  int read##NAME(void *d, T *h, int n) { return buf_copy(h, d, (long long)n * sizeof(T), cudaMemcpyDeviceToHost); } \
  int write##NAME##First(int first, void *d, T *h, int n, int IndexBase) {                              \
    if (!d) return SPGPU_UNSUPPORTED;                                                                   \
    return buf_copy((T *)d + (first - IndexBase), h, (long long)n * sizeof(T), cudaMemcpyHostToDevice); \
  }                                                                                                     \
  int read##NAME##First(int first, void *d, T *h, int n, int IndexBase) {                               \
    if (!d) return SPGPU_UNSUPPORTED;                                                                   \
    return buf_copy(h, (T *)d + (first - IndexBase), (long long)n * sizeof(T), cudaMemcpyDeviceToHost); \
  }                                                                                                     \
  int writeMulti##NAME(void *d, T *h, int m, int n) {                                                   \
    return buf_copy(d, h, (long long)m * n * sizeof(T), cudaMemcpyHostToDevice);                       \
  }                                                                                                     \
  int readMulti##NAME(void *d, T *h, int m, int n) {                                                    \
    return buf_copy(h, d, (long long)m * n * sizeof(T), cudaMemcpyDeviceToHost);                       \
  }                                                                                                     \
  void free##NAME(void *d) { buf_free(d); }                                                             \
  int registerMapped##NAME(void *buf, void **d_p, int n, T dummy) {                                     \
    (void)dummy;                                                                                        \
    return map_host(buf, d_p, (long long)n * sizeof(T));                                               \
  }

PSBX_BUFFER_TOOLS(Int, int)
PSBX_BUFFER_TOOLS(Float, float)
PSBX_BUFFER_TOOLS(Double, double)
#undef PSBX_BUFFER_TOOLS

// cuda/vectordev.c:145-148
int unregisterMapped(void *buf) {
  if (!buf) return SPGPU_UNSUPPORTED;
  PSBX_CK(cudaHostUnregister(buf));
  return SPGPU_SUCCESS;
}

int psbx_DefaultSolverOptions(psbx_SolverOptions *opt) {
  // cbind/krylov/psb_base_krylov_cbind_mod.f90:13-26 defaults
  if (!opt) return SPGPU_UNSUPPORTED;
  opt->iter = 0;
  opt->itmax = 1000;
  opt->itrace = 0;
  opt->irst = 10;
  opt->istop = 2;
  opt->eps = 1e-6;
  opt->err = 0.0;
  return SPGPU_SUCCESS;
}

}  // extern "C"
