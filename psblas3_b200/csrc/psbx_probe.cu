// Gather-rate probe: the bound of an SpMV whose column indices are spread
// over a vector larger than L1.  Every entry of a matrix costs one 8-byte
// read of x at its column; when the columns are random, each read is its own
// L2 sector request, and the rate at which L2 serves those requests -- not
// HBM bandwidth -- sets the floor on the SpMV time.  This kernel does only
// those reads (the matrix's own column stream, no values, no row sums, one
// double written per 8 entries), so its time is that floor for the matrix.
#include "psbx_internal.cuh"
#include "../../include/psbx_probe.h"

namespace {
constexpr int PT = 256;  // threads per block
constexpr int PU = 4;    // index pairs per thread

__global__ void __launch_bounds__(PT) k_probe_gather(const int2 *__restrict__ idx, long long npairs, int base,
                                                     const double *__restrict__ x, double *__restrict__ out) {
  const long long nt = (npairs + PU - 1) / PU;
  const long long t = (long long)blockIdx.x * PT + threadIdx.x;
  if (t >= nt) return;
  const double *xb = x - base;
  int2 c[PU];
#pragma unroll
  for (int u = 0; u < PU; u++) {
    const long long p = t + u * nt;
    c[u] = p < npairs ? ld_stream(idx + p) : make_int2(base, base);
  }
  double a = 0.0, b = 0.0;
#pragma unroll
  for (int u = 0; u < PU; u++) {
    a += ld_ro(xb + c[u].x);
    b += ld_ro(xb + c[u].y);
  }
  out[t] = a + b;
}
}  // namespace

extern "C" int psbx_probe_gather(const int *d_idx, long long n, int base, const double *d_x, double *d_out,
                                 int reps, double *best_ms) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  if (!d_idx || !d_x || !d_out || n < 2 || reps < 1 || ((uintptr_t)d_idx & 7)) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  const long long npairs = n / 2;
  const long long nt = (npairs + PU - 1) / PU;
  const unsigned grid = (unsigned)((nt + PT - 1) / PT);
  cudaEvent_t e0, e1;
  PSBX_CK(cudaEventCreate(&e0));
  PSBX_CK(cudaEventCreate(&e1));
  float best = -1.0f;
  for (int r = 0; r < reps + 2 && !rc; r++) {  // two untimed launches first
    cudaEventRecord(e0, c.stream);
    k_probe_gather<<<grid, PT, 0, c.stream>>>((const int2 *)d_idx, npairs, base, d_x, d_out);
    psbx_count_launch();
    cudaEventRecord(e1, c.stream);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
      rc = psbx_cuda_status(e, "k_probe_gather");
      break;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r >= 2 && (best < 0.0f || ms < best)) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!rc && best_ms) *best_ms = best;
  return rc;
}
