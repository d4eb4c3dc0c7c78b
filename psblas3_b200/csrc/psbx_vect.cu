// psbx_vect.cu -- dense multivector objects and the BLAS-1 kernels behind
// psb_geaxpby / psb_gedot / psb_genrm2 / psb_geamax / psb_geasum / mlt.
// Replaces cuda/vectordev.c, cuda/dvectordev.c:40-345 and the SPGPU kernels
// daxpby.cu, ddot.cu, dnrm2.cu, amax/asum, axy_base.cuh, dupd_xyz.cu,
// dxyzw.cu, scal/setscal/abs.
//
// Element-wise kernels use rounded multiplies and adds with no contraction,
// so their results equal the reference CPU loops (psi_daxpbyv and friends)
// bit for bit.  Reductions run on the device in a fixed order (per-thread
// grid-stride partials, a shuffle tree per block, one partial per block, the
// last block sums the partials), so a result depends only on n and the SM
// count -- unlike the reference, which copies per-block partials to the host
// and sums them there (ddot.cu:133-144).
#include "psbx_internal.cuh"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const int VT = 256;  // threads per block for streaming vector kernels

// ------------------------------------------------------------------ objects
static int vec_pitch(unsigned count, unsigned size, unsigned elem) {
  // cuda/vectordev.c:40-70: pitch = size for one vector, else rounded to 256 B
  size_t es = elem == SPGPU_TYPE_DOUBLE ? 8 : 4;
  if (elem == SPGPU_TYPE_COMPLEX_DOUBLE) es = 16;
  if (elem == SPGPU_TYPE_COMPLEX_FLOAT) es = 8;
  if (count <= 1) return (int)size;
  return (int)((((size_t)size * es + 255) / 256) * 256 / es);
}

static size_t elem_size(int t) {
  switch (t) {
    case SPGPU_TYPE_INT: return 4;
    case SPGPU_TYPE_FLOAT: return 4;
    case SPGPU_TYPE_DOUBLE: return 8;
    case SPGPU_TYPE_COMPLEX_FLOAT: return 8;
    case SPGPU_TYPE_COMPLEX_DOUBLE: return 16;
  }
  return 0;
}

extern "C" {

int FallocMultiVecDevice(void **deviceMultiVec, unsigned count, unsigned size, unsigned elementType) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  if (!deviceMultiVec || elem_size((int)elementType) == 0) return SPGPU_UNSUPPORTED;
  MultiVectDevice *v = (MultiVectDevice *)calloc(1, sizeof(MultiVectDevice));
  v->count_ = (int)count;
  v->size_ = (int)size;
  v->pitch_ = vec_pitch(count, size, elementType);
  v->elemType = (int)elementType;
  v->owns = 1;
  size_t bytes = (size_t)v->pitch_ * (count ? count : 1) * elem_size((int)elementType);
  if (bytes == 0) bytes = 256;
  cudaError_t e = cudaMalloc(&v->v_, bytes);
  if (e != cudaSuccess) {
    free(v);
    *deviceMultiVec = nullptr;
    return psbx_cuda_status(e, "FallocMultiVecDevice");
  }
  *deviceMultiVec = v;
  return SPGPU_SUCCESS;
}

int psbx_wrapMultiVecDevice(void **deviceVec, void *devPtr, unsigned size, unsigned elementType) {
  int rc = psbx_ensure_init();
  if (rc) return rc;
  if (!deviceVec || !devPtr || elem_size((int)elementType) == 0) return SPGPU_UNSUPPORTED;
  MultiVectDevice *v = (MultiVectDevice *)calloc(1, sizeof(MultiVectDevice));
  v->count_ = 1;
  v->size_ = (int)size;
  v->pitch_ = (int)size;
  v->v_ = devPtr;
  v->elemType = (int)elementType;
  v->owns = 0;
  *deviceVec = v;
  return SPGPU_SUCCESS;
}

void *psbx_multivec_data(void *deviceVec) { return deviceVec ? ((MultiVectDevice *)deviceVec)->v_ : nullptr; }

void freeMultiVecDevice(void *deviceVec) {
  MultiVectDevice *v = (MultiVectDevice *)deviceVec;
  if (!v) return;
  if (v->owns && v->v_) {
    cudaStreamSynchronize(psbx_ctx().stream);
    cudaFree(v->v_);
  }
  free(v);
}

int getMultiVecDeviceSize(void *deviceVec) { return ((MultiVectDevice *)deviceVec)->size_; }
int getMultiVecDeviceCount(void *deviceVec) { return ((MultiVectDevice *)deviceVec)->count_; }
int getMultiVecDevicePitch(void *deviceVec) { return ((MultiVectDevice *)deviceVec)->pitch_; }

static int vec_copy(void *deviceVec, void *host, bool h2d, int expect_type) {
  MultiVectDevice *v = (MultiVectDevice *)deviceVec;
  if (!v || !host) return SPGPU_UNSUPPORTED;
  if (v->elemType != expect_type) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  size_t bytes = (size_t)v->pitch_ * v->count_ * elem_size(v->elemType);
  if (bytes == 0) return SPGPU_SUCCESS;
  if (h2d)
    PSBX_CK(cudaMemcpyAsync(v->v_, host, bytes, cudaMemcpyHostToDevice, c.stream));
  else
    PSBX_CK(cudaMemcpyAsync(host, v->v_, bytes, cudaMemcpyDeviceToHost, c.stream));
  PSBX_CK(cudaStreamSynchronize(c.stream));
  return SPGPU_SUCCESS;
}

int writeMultiVecDeviceDouble(void *deviceVec, double *hostVec) {
  return vec_copy(deviceVec, hostVec, true, SPGPU_TYPE_DOUBLE);
}
int writeMultiVecDeviceDoubleR2(void *deviceVec, double *hostVec, int ld) {
  (void)ld;  // dvectordev.c:62-69 ignores ld as well
  return vec_copy(deviceVec, hostVec, true, SPGPU_TYPE_DOUBLE);
}
int readMultiVecDeviceDouble(void *deviceVec, double *hostVec) {
  return vec_copy(deviceVec, hostVec, false, SPGPU_TYPE_DOUBLE);
}
int readMultiVecDeviceDoubleR2(void *deviceVec, double *hostVec, int ld) {
  (void)ld;
  return vec_copy(deviceVec, hostVec, false, SPGPU_TYPE_DOUBLE);
}
int writeMultiVecDeviceFloat(void *deviceVec, float *hostVec) {
  return vec_copy(deviceVec, hostVec, true, SPGPU_TYPE_FLOAT);
}
int readMultiVecDeviceFloat(void *deviceVec, float *hostVec) {
  return vec_copy(deviceVec, hostVec, false, SPGPU_TYPE_FLOAT);
}

}  // extern "C"

// ------------------------------------------------------------------ kernels
// Written once for the element types of the vector families: double (the
// d type), float (the s type) and, for the index-vector operations, int.
template <class T>
__global__ void k_setscal(int first, int last, T val, T *__restrict__ x) {
  for (long long i = first + (long long)blockIdx.x * blockDim.x + threadIdx.x; i <= last;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = val;
}

template <class T>
__global__ void k_scal(long long n, T alpha, T *__restrict__ x) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] = rmul(alpha, x[i]);
}

// y = alpha*x + beta*y.  MODE 0: generic; 1: beta == 0 (y not read).
template <int MODE, class T>
__global__ void k_axpby(int n, T alpha, const T *__restrict__ x, T beta, T *__restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T ax = rmul(alpha, ld_stream(x + i));
    y[i] = MODE == 1 ? ax : radd(ax, rmul(beta, y[i]));
  }
}

// y = beta*y, for alpha == 0 (x not read); beta == 0 writes zeros.
template <class T>
__global__ void k_betay(int n, T beta, T *__restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = beta == T(0) ? T(0) : rmul(beta, y[i]);
}

template <class T>
__device__ __forceinline__ T axpby_el(T alpha, T x, T beta, T y) {
  if (alpha == T(0)) return beta == T(0) ? T(0) : rmul(beta, y);
  T ax = rmul(alpha, x);
  return beta == T(0) ? ax : radd(ax, rmul(beta, y));
}

template <class T>
__global__ void k_upd_xyz(int n, T a, T b, T g, T d, const T *__restrict__ x, T *__restrict__ y,
                          T *__restrict__ z) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T yy = axpby_el(a, a == T(0) ? T(0) : x[i], b, b == T(0) ? T(0) : y[i]);
    y[i] = yy;
    z[i] = axpby_el(g, yy, d, d == T(0) ? T(0) : z[i]);
  }
}

template <class T>
__global__ void k_xyzw(int n, T a, T b, T c, T d, T e, T f, const T *__restrict__ x, T *__restrict__ y,
                       T *__restrict__ z, T *__restrict__ w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T yy = radd(rmul(a, x[i]), rmul(b, y[i]));
    T zz = radd(rmul(c, yy), rmul(d, z[i]));
    T ww = radd(rmul(e, zz), rmul(f, w[i]));
    y[i] = yy;
    z[i] = zz;
    w[i] = ww;
  }
}

// z = alpha*(a.*b) + beta*z   (beta == 0: z not read)
template <class T>
__global__ void k_axybz(int n, T alpha, const T *__restrict__ a, const T *b, T beta, T *z) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T t = rmul(alpha, rmul(ld_stream(a + i), ld_stream(b + i)));
    z[i] = beta == T(0) ? t : radd(t, rmul(beta, z[i]));
  }
}

// buf[i] = v[idx[i] - base]
template <class T>
__global__ void k_gath(int n, const int *__restrict__ idx, int base, const T *__restrict__ v, T *__restrict__ buf) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) buf[i] = v[idx[i] - base];
}

__device__ __forceinline__ double scat_el(double beta, double v, double b) { return radd(rmul(beta, v), b); }
__device__ __forceinline__ float scat_el(float beta, float v, float b) { return radd(rmul(beta, v), b); }
__device__ __forceinline__ int scat_el(int beta, int v, int b) { return beta * v + b; }

// v[idx[i] - base] = beta * v[idx[i] - base] + buf[i]  (beta == 0: v not read)
template <class T>
__global__ void k_scat(int n, const int *__restrict__ idx, int base, const T *__restrict__ buf, T beta,
                       T *__restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int j = idx[i] - base;
    v[j] = beta == T(0) ? buf[i] : scat_el(beta, v[j], buf[i]);
  }
}

template <class T>
__global__ void k_abs(int n, T alpha, const T *__restrict__ a, T *__restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    b[i] = rmul(alpha, (T)fabs(a[i]));
}

enum { R_DOT = 0, R_NRM2 = 1, R_ASUM = 2, R_AMAX = 3 };

// One partial per block per vector (blockIdx.y), finalised by the last block.
// DOT and NRM2 accumulate compensated pairs (Dot2); ASUM is a plain sum;
// AMAX a max.  Partials of vector v, block b: part[2*(v*PSBX_MAX_PART + b)].
// The element type T is double or float; every value is converted to double
// as it is loaded (exact), so the FP32 reductions accumulate in FP64 and
// round to FP32 once, on the host.
template <int OP, class T>
__global__ void __launch_bounds__(256) k_reduce(int n, const T *__restrict__ x, int px,
                                                const T *__restrict__ y, int py,
                                                double *__restrict__ part, unsigned *__restrict__ ticket,
                                                double *__restrict__ res) {
  __shared__ double sm[64];
  const int v = blockIdx.y;
  const T *xv = x + (size_t)v * px;
  const T *yv = OP == R_DOT ? y + (size_t)v * py : xv;
  const int stride = gridDim.x * blockDim.x;
  double *pv = part + 2 * (size_t)v * PSBX_MAX_PART;
  if (OP == R_DOT || OP == R_NRM2) {
    dd_t acc[1] = {{0.0, 0.0}};
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n; i += 4 * stride) {
      const double a0 = (double)ld_stream(xv + i), a1 = (double)ld_stream(xv + i + stride);
      const double a2 = (double)ld_stream(xv + i + 2 * stride), a3 = (double)ld_stream(xv + i + 3 * stride);
      double b0 = a0, b1 = a1, b2 = a2, b3 = a3;
      if (OP == R_DOT) {
        b0 = (double)ld_stream(yv + i);
        b1 = (double)ld_stream(yv + i + stride);
        b2 = (double)ld_stream(yv + i + 2 * stride);
        b3 = (double)ld_stream(yv + i + 3 * stride);
      }
      dd_add_prod(acc[0], a0, b0);
      dd_add_prod(acc[0], a1, b1);
      dd_add_prod(acc[0], a2, b2);
      dd_add_prod(acc[0], a3, b3);
    }
    for (; i < n; i += stride) {
      const double a = (double)ld_stream(xv + i);
      dd_add_prod(acc[0], a, OP == R_DOT ? (double)ld_stream(yv + i) : a);
    }
    block_sum_dd<1>(acc, sm);
    if (threadIdx.x == 0) {
      pv[2 * blockIdx.x] = acc[0].s;
      pv[2 * blockIdx.x + 1] = acc[0].c;
    }
    if (psbx_last_block(ticket + v, gridDim.x)) {
      dd_t out[1];
      final_sum_dd<1>(pv, 0, gridDim.x, out, sm);
      if (threadIdx.x == 0) {
        const double t = dd_value(out[0]);
        res[v] = OP == R_NRM2 ? sqrt(t) : t;
        ticket[v] = 0;
      }
    }
    return;
  }
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double a = (double)ld_stream(xv + i);
    acc[0] = OP == R_ASUM ? radd(acc[0], fabs(a)) : fmax(acc[0], fabs(a));
  }
  if (OP == R_AMAX) block_max<1>(acc, sm);
  else block_sum<1>(acc, sm);
  if (threadIdx.x == 0) pv[2 * blockIdx.x] = acc[0];
  if (psbx_last_block(ticket + v, gridDim.x)) {
    double out[1];
    double s = 0.0, m = 0.0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
      const double t = __ldcg(pv + 2 * k);
      s = radd(s, t);
      m = fmax(m, t);
    }
    out[0] = OP == R_AMAX ? m : s;
    if (OP == R_AMAX) block_max<1>(out, sm);
    else block_sum<1>(out, sm);
    if (threadIdx.x == 0) {
      res[v] = out[0];
      ticket[v] = 0;
    }
  }
}

// ------------------------------------------------------------------ launchers
int psbx_launch_scale(int n, double beta, double *y, cudaStream_t st) {
  if (n <= 0) return SPGPU_SUCCESS;
  int g = psbx_grid_for(n, VT);
  k_betay<double><<<g, VT, 0, st>>>(n, beta, y);
  PSBX_LAUNCH_CK("k_betay");
  return SPGPU_SUCCESS;
}

static int launch_axpby(int n, double alpha, const double *x, double beta, double *y, cudaStream_t st) {
  if (n <= 0) return SPGPU_SUCCESS;
  int g = psbx_grid_for(n, VT);
  if (alpha == 0.0) {
    if (beta == 1.0) return SPGPU_SUCCESS;
    k_betay<double><<<g, VT, 0, st>>>(n, beta, y);
  } else if (beta == 0.0) {
    k_axpby<1, double><<<g, VT, 0, st>>>(n, alpha, x, beta, y);
  } else {
    k_axpby<0, double><<<g, VT, 0, st>>>(n, alpha, x, beta, y);
  }
  PSBX_LAUNCH_CK("k_axpby");
  return SPGPU_SUCCESS;
}

// Runs a reduction over count vectors; results land in c.d_res[0..count).
static int launch_reduce(int op, int n, const MultiVectDevice *a, const MultiVectDevice *b, int count,
                         cudaStream_t st, double *host_out) {
  PsbxCtx &c = psbx_ctx();
  for (int v0 = 0; v0 < count; v0 += PSBX_NLANES) {
    int nv = count - v0 < PSBX_NLANES ? count - v0 : PSBX_NLANES;
    int g = psbx_grid_for(n > 0 ? n : 1, VT * 4, 4);
    if (g > PSBX_MAX_PART) g = PSBX_MAX_PART;
    dim3 grid(g, nv);
    const double *xa = (const double *)a->v_ + (size_t)v0 * a->pitch_;
    const double *xb = b ? (const double *)b->v_ + (size_t)v0 * b->pitch_ : nullptr;
    switch (op) {
      case R_DOT: k_reduce<R_DOT, double><<<grid, VT, 0, st>>>(n, xa, a->pitch_, xb, b->pitch_, c.d_part, c.d_ticket, c.d_res); break;
      case R_NRM2: k_reduce<R_NRM2, double><<<grid, VT, 0, st>>>(n, xa, a->pitch_, nullptr, 0, c.d_part, c.d_ticket, c.d_res); break;
      case R_ASUM: k_reduce<R_ASUM, double><<<grid, VT, 0, st>>>(n, xa, a->pitch_, nullptr, 0, c.d_part, c.d_ticket, c.d_res); break;
      default: k_reduce<R_AMAX, double><<<grid, VT, 0, st>>>(n, xa, a->pitch_, nullptr, 0, c.d_part, c.d_ticket, c.d_res); break;
    }
    PSBX_LAUNCH_CK("k_reduce");
    PSBX_CK(cudaMemcpyAsync(c.h_res, c.d_res, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
    PSBX_CK(cudaStreamSynchronize(st));
    for (int k = 0; k < nv; k++) host_out[v0 + k] = c.h_res[k];
  }
  return SPGPU_SUCCESS;
}

static inline MultiVectDevice *MV(void *p) { return (MultiVectDevice *)p; }

extern "C" {

int setscalMultiVecDeviceDouble(double val, int first, int last, int indexBase, void *devVecX) {
  MultiVectDevice *x = MV(devVecX);
  if (!x) return SPGPU_UNSUPPORTED;
  int f = first - indexBase, l = last - indexBase;
  if (f < 0 || l >= x->pitch_ * x->count_) return SPGPU_UNSUPPORTED;
  if (l < f) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  int g = psbx_grid_for(l - f + 1, VT);
  k_setscal<double><<<g, VT, 0, c.stream>>>(f, l, val, (double *)x->v_);
  PSBX_LAUNCH_CK("k_setscal");
  return SPGPU_SUCCESS;
}

int scalMultiVecDeviceDouble(double alpha, void *devVecA) {
  MultiVectDevice *x = MV(devVecA);
  if (!x) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  long long n = (long long)x->pitch_ * x->count_;
  int g = psbx_grid_for(n, VT);
  k_scal<double><<<g, VT, 0, c.stream>>>(n, alpha, (double *)x->v_);
  PSBX_LAUNCH_CK("k_scal");
  return SPGPU_SUCCESS;
}

int nrm2MultiVecDeviceDouble(double *y_res, int n, void *devVecA) {
  MultiVectDevice *a = MV(devVecA);
  if (!a || !y_res || n > a->size_) return SPGPU_UNSUPPORTED;
  return launch_reduce(R_NRM2, n, a, nullptr, a->count_, psbx_ctx().stream, y_res);
}

int amaxMultiVecDeviceDouble(double *y_res, int n, void *devVecA) {
  MultiVectDevice *a = MV(devVecA);
  if (!a || !y_res || n > a->size_) return SPGPU_UNSUPPORTED;
  return launch_reduce(R_AMAX, n, a, nullptr, a->count_, psbx_ctx().stream, y_res);
}

int asumMultiVecDeviceDouble(double *y_res, int n, void *devVecA) {
  MultiVectDevice *a = MV(devVecA);
  if (!a || !y_res || n > a->size_) return SPGPU_UNSUPPORTED;
  return launch_reduce(R_ASUM, n, a, nullptr, a->count_, psbx_ctx().stream, y_res);
}

int dotMultiVecDeviceDouble(double *y_res, int n, void *devVecA, void *devVecB) {
  MultiVectDevice *a = MV(devVecA), *b = MV(devVecB);
  if (!a || !b || !y_res || n > a->size_ || n > b->size_ || a->count_ != b->count_) return SPGPU_UNSUPPORTED;
  return launch_reduce(R_DOT, n, a, b, a->count_, psbx_ctx().stream, y_res);
}

int axpbyMultiVecDeviceDouble(int n, double alpha, void *devVecX, double beta, void *devVecY) {
  MultiVectDevice *x = MV(devVecX), *y = MV(devVecY);
  if (!x || !y || n > y->size_ || n > x->size_) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  for (int j = 0; j < y->count_; j++) {
    int rc = launch_axpby(n, alpha, (const double *)x->v_ + (size_t)j * x->pitch_, beta,
                          (double *)y->v_ + (size_t)j * y->pitch_, c.stream);
    if (rc) return rc;
  }
  return SPGPU_SUCCESS;
}

int upd_xyzMultiVecDeviceDouble(int n, double alpha, double beta, double gamma, double delta, void *devVecX,
                                void *devVecY, void *devVecZ) {
  MultiVectDevice *x = MV(devVecX), *y = MV(devVecY), *z = MV(devVecZ);
  if (!x || !y || !z || n > y->size_ || n > x->size_ || n > z->size_) return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_upd_xyz<double><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, alpha, beta, gamma, delta, (const double *)x->v_,
                                                       (double *)y->v_, (double *)z->v_);
  PSBX_LAUNCH_CK("k_upd_xyz");
  return SPGPU_SUCCESS;
}

int xyzwMultiVecDeviceDouble(int n, double a, double b, double cc, double d, double e, double f, void *devVecX,
                             void *devVecY, void *devVecZ, void *devVecW) {
  MultiVectDevice *x = MV(devVecX), *y = MV(devVecY), *z = MV(devVecZ), *w = MV(devVecW);
  if (!x || !y || !z || !w || n > y->size_ || n > x->size_ || n > z->size_ || n > w->size_)
    return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_xyzw<double><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, a, b, cc, d, e, f, (const double *)x->v_,
                                                    (double *)y->v_, (double *)z->v_, (double *)w->v_);
  PSBX_LAUNCH_CK("k_xyzw");
  return SPGPU_SUCCESS;
}

int axyMultiVecDeviceDouble(int n, double alpha, void *devVecA, void *devVecB) {
  MultiVectDevice *a = MV(devVecA), *b = MV(devVecB);
  if (!a || !b || n > a->size_ || n > b->size_) return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_axybz<double><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, alpha, (const double *)a->v_, (const double *)b->v_,
                                                     0.0, (double *)b->v_);
  PSBX_LAUNCH_CK("k_axy");
  return SPGPU_SUCCESS;
}

int axybzMultiVecDeviceDouble(int n, double alpha, void *devVecA, void *devVecB, double beta, void *devVecZ) {
  MultiVectDevice *a = MV(devVecA), *b = MV(devVecB), *z = MV(devVecZ);
  if (!a || !b || !z || n > a->size_ || n > b->size_ || n > z->size_) return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_axybz<double><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, alpha, (const double *)a->v_, (const double *)b->v_,
                                                     beta, (double *)z->v_);
  PSBX_LAUNCH_CK("k_axybz");
  return SPGPU_SUCCESS;
}

int absMultiVecDeviceDouble2(int n, double alpha, void *devVecA, void *devVecB) {
  MultiVectDevice *a = MV(devVecA), *b = MV(devVecB);
  if (!a || !b || n > a->size_ || n > b->size_) return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_abs<double><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, alpha, (const double *)a->v_, (double *)b->v_);
  PSBX_LAUNCH_CK("k_abs");
  return SPGPU_SUCCESS;
}

int absMultiVecDeviceDouble(int n, double alpha, void *devVecA) {
  return absMultiVecDeviceDouble2(n, alpha, devVecA, devVecA);
}

// Gather / scatter through an index list: the two halves of a halo exchange
// (the send buffer is gathered from the owned entries, the received buffer
// is scattered into the halo entries).  vectorId selects one of the count
// vectors; first / hfirst are indexBase-based starts in idx / buf.
int igathMultiVecDeviceDouble(void *deviceVec, int vectorId, int n, int first, void *indexes, int hfirst,
                              void *host_values, int indexBase) {
  MultiVectDevice *x = MV(deviceVec);
  if (!x || (n > 0 && (!indexes || !host_values)) || vectorId < 0 || vectorId >= x->count_) return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  const int *idx = (const int *)indexes + (first - indexBase);
  double *buf = (double *)host_values + (hfirst - indexBase);
  const double *v = (const double *)x->v_ + (size_t)vectorId * x->pitch_;
  k_gath<double><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, idx, indexBase, v, buf);
  PSBX_LAUNCH_CK("k_gath");
  return SPGPU_SUCCESS;
}

int igathMultiVecDeviceDoubleVecIdx(void *deviceVec, int vectorId, int n, int first, void *deviceIdx, int hfirst,
                                    void *host_values, int indexBase) {
  MultiVectDevice *ix = MV(deviceIdx);
  if (!ix) return SPGPU_UNSUPPORTED;
  return igathMultiVecDeviceDouble(deviceVec, vectorId, n, first, ix->v_, hfirst, host_values, indexBase);
}

int iscatMultiVecDeviceDouble(void *deviceVec, int vectorId, int n, int first, void *indexes, int hfirst,
                              void *host_values, int indexBase, double beta) {
  MultiVectDevice *x = MV(deviceVec);
  if (!x || (n > 0 && (!indexes || !host_values)) || vectorId < 0 || vectorId >= x->count_) return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  const int *idx = (const int *)indexes + (first - indexBase);
  const double *buf = (const double *)host_values + (hfirst - indexBase);
  double *v = (double *)x->v_ + (size_t)vectorId * x->pitch_;
  k_scat<double><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, idx, indexBase, buf, beta, v);
  PSBX_LAUNCH_CK("k_scat");
  return SPGPU_SUCCESS;
}

int iscatMultiVecDeviceDoubleVecIdx(void *deviceVec, int vectorId, int n, int first, void *deviceIdx, int hfirst,
                                    void *host_values, int indexBase, double beta) {
  MultiVectDevice *ix = MV(deviceIdx);
  if (!ix) return SPGPU_UNSUPPORTED;
  return iscatMultiVecDeviceDouble(deviceVec, vectorId, n, first, ix->v_, hfirst, host_values, indexBase, beta);
}

// geinsMultiVecDeviceDouble (cuda/dvectordev.c:98-125): insert n values
// val[i] at the indexBase-based positions irl[i] of x, overwriting
// (dupl == INS_OVERWRITE, 0) or adding (INS_ADD, 1; any other code
// overwrites, as the reference); irl, val, x are device multivectors.
int geinsMultiVecDeviceDouble(int n, void *devMultiVecIrl, void *devMultiVecVal, int dupl, int indexBase,
                              void *devMultiVecX) {
  MultiVectDevice *irl = MV(devMultiVecIrl), *val = MV(devMultiVecVal), *x = MV(devMultiVecX);
  if (!irl || !val || !x || n > irl->size_ || n > val->size_) return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_scat<double><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, (const int *)irl->v_, indexBase,
                                                            (const double *)val->v_, dupl == 1 ? 1.0 : 0.0,
                                                            (double *)x->v_);
  PSBX_LAUNCH_CK("k_scat (geins)");
  return SPGPU_SUCCESS;
}

// ===================================================================== FP32
// cuda/svectordev.c / svectordev.h:40-80 (the psb_s_vect_cuda glue).  The
// element-wise operations round every FP32 multiply and add (no
// contraction), as the CPU loops of psi_s_serial_impl.F90 do.  dot and nrm2
// accumulate in FP64 -- the product of two floats is exact in FP64 -- with
// the compensated sum of the FP64 entries, and round to FP32 once; asum sums
// in FP64 and rounds once; amax is exact.  (The reference's SPGPU kernels
// sdot.cu / snrm2.cu / sasum.cu accumulate in FP32.)

int writeMultiVecDeviceFloatR2(void *deviceVec, float *hostVec, int ld) {
  (void)ld;  // svectordev.c:55-63 ignores ld as well
  return vec_copy(deviceVec, hostVec, true, SPGPU_TYPE_FLOAT);
}
int readMultiVecDeviceFloatR2(void *deviceVec, float *hostVec, int ld) {
  (void)ld;
  return vec_copy(deviceVec, hostVec, false, SPGPU_TYPE_FLOAT);
}

static inline bool is_f(const MultiVectDevice *v) { return v && v->elemType == SPGPU_TYPE_FLOAT; }
static inline bool is_i(const MultiVectDevice *v) { return v && v->elemType == SPGPU_TYPE_INT; }

int setscalMultiVecDeviceFloat(float val, int first, int last, int indexBase, void *devVecX) {
  MultiVectDevice *x = MV(devVecX);
  if (!is_f(x)) return SPGPU_UNSUPPORTED;
  int f = first - indexBase, l = last - indexBase;
  if (f < 0 || l >= x->pitch_ * x->count_) return SPGPU_UNSUPPORTED;
  if (l < f) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_setscal<float><<<psbx_grid_for(l - f + 1, VT), VT, 0, c.stream>>>(f, l, val, (float *)x->v_);
  PSBX_LAUNCH_CK("k_setscal<float>");
  return SPGPU_SUCCESS;
}

int scalMultiVecDeviceFloat(float alpha, void *devVecA) {
  MultiVectDevice *x = MV(devVecA);
  if (!is_f(x)) return SPGPU_UNSUPPORTED;
  PsbxCtx &c = psbx_ctx();
  long long n = (long long)x->pitch_ * x->count_;
  k_scal<float><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, alpha, (float *)x->v_);
  PSBX_LAUNCH_CK("k_scal<float>");
  return SPGPU_SUCCESS;
}

// Reductions of count FP32 vectors; each result rounded to FP32 on the host.
static int launch_reduce_f(int op, int n, const MultiVectDevice *a, const MultiVectDevice *b, float *out) {
  PsbxCtx &c = psbx_ctx();
  cudaStream_t st = c.stream;
  for (int v0 = 0; v0 < a->count_; v0 += PSBX_NLANES) {
    int nv = a->count_ - v0 < PSBX_NLANES ? a->count_ - v0 : PSBX_NLANES;
    int g = psbx_grid_for(n > 0 ? n : 1, VT * 4, 4);
    if (g > PSBX_MAX_PART) g = PSBX_MAX_PART;
    dim3 grid(g, nv);
    const float *xa = (const float *)a->v_ + (size_t)v0 * a->pitch_;
    const float *xb = b ? (const float *)b->v_ + (size_t)v0 * b->pitch_ : nullptr;
    switch (op) {
      case R_DOT: k_reduce<R_DOT, float><<<grid, VT, 0, st>>>(n, xa, a->pitch_, xb, b->pitch_, c.d_part, c.d_ticket, c.d_res); break;
      case R_NRM2: k_reduce<R_NRM2, float><<<grid, VT, 0, st>>>(n, xa, a->pitch_, nullptr, 0, c.d_part, c.d_ticket, c.d_res); break;
      case R_ASUM: k_reduce<R_ASUM, float><<<grid, VT, 0, st>>>(n, xa, a->pitch_, nullptr, 0, c.d_part, c.d_ticket, c.d_res); break;
      default: k_reduce<R_AMAX, float><<<grid, VT, 0, st>>>(n, xa, a->pitch_, nullptr, 0, c.d_part, c.d_ticket, c.d_res); break;
    }
    PSBX_LAUNCH_CK("k_reduce<float>");
    PSBX_CK(cudaMemcpyAsync(c.h_res, c.d_res, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
    PSBX_CK(cudaStreamSynchronize(st));
    for (int k = 0; k < nv; k++) out[v0 + k] = (float)c.h_res[k];
  }
  return SPGPU_SUCCESS;
}

int nrm2MultiVecDeviceFloat(float *y_res, int n, void *devVecA) {
  MultiVectDevice *a = MV(devVecA);
  if (!is_f(a) || !y_res || n > a->size_) return SPGPU_UNSUPPORTED;
  return launch_reduce_f(R_NRM2, n, a, nullptr, y_res);
}
int amaxMultiVecDeviceFloat(float *y_res, int n, void *devVecA) {
  MultiVectDevice *a = MV(devVecA);
  if (!is_f(a) || !y_res || n > a->size_) return SPGPU_UNSUPPORTED;
  return launch_reduce_f(R_AMAX, n, a, nullptr, y_res);
}
int asumMultiVecDeviceFloat(float *y_res, int n, void *devVecA) {
  MultiVectDevice *a = MV(devVecA);
  if (!is_f(a) || !y_res || n > a->size_) return SPGPU_UNSUPPORTED;
  return launch_reduce_f(R_ASUM, n, a, nullptr, y_res);
}
int dotMultiVecDeviceFloat(float *y_res, int n, void *devVecA, void *devVecB) {
  MultiVectDevice *a = MV(devVecA), *b = MV(devVecB);
  if (!is_f(a) || !is_f(b) || !y_res || n > a->size_ || n > b->size_ || a->count_ != b->count_)
    return SPGPU_UNSUPPORTED;
  return launch_reduce_f(R_DOT, n, a, b, y_res);
}

int axpbyMultiVecDeviceFloat(int n, float alpha, void *devVecX, float beta, void *devVecY) {
  MultiVectDevice *x = MV(devVecX), *y = MV(devVecY);
  if (!is_f(x) || !is_f(y) || n > y->size_ || n > x->size_) return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  const int g = psbx_grid_for(n, VT);
  for (int j = 0; j < y->count_; j++) {
    const float *xj = (const float *)x->v_ + (size_t)j * x->pitch_;
    float *yj = (float *)y->v_ + (size_t)j * y->pitch_;
    if (alpha == 0.0f) {
      if (beta == 1.0f) continue;
      k_betay<float><<<g, VT, 0, c.stream>>>(n, beta, yj);
    } else if (beta == 0.0f) {
      k_axpby<1, float><<<g, VT, 0, c.stream>>>(n, alpha, xj, beta, yj);
    } else {
      k_axpby<0, float><<<g, VT, 0, c.stream>>>(n, alpha, xj, beta, yj);
    }
    PSBX_LAUNCH_CK("k_axpby<float>");
  }
  return SPGPU_SUCCESS;
}

int upd_xyzMultiVecDeviceFloat(int n, float alpha, float beta, float gamma, float delta, void *devVecX,
                               void *devVecY, void *devVecZ) {
  MultiVectDevice *x = MV(devVecX), *y = MV(devVecY), *z = MV(devVecZ);
  if (!is_f(x) || !is_f(y) || !is_f(z) || n > y->size_ || n > x->size_ || n > z->size_) return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_upd_xyz<float><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, alpha, beta, gamma, delta, (const float *)x->v_,
                                                              (float *)y->v_, (float *)z->v_);
  PSBX_LAUNCH_CK("k_upd_xyz<float>");
  return SPGPU_SUCCESS;
}

int xyzwMultiVecDeviceFloat(int n, float a, float b, float cc, float d, float e, float f, void *devVecX,
                            void *devVecY, void *devVecZ, void *devVecW) {
  MultiVectDevice *x = MV(devVecX), *y = MV(devVecY), *z = MV(devVecZ), *w = MV(devVecW);
  if (!is_f(x) || !is_f(y) || !is_f(z) || !is_f(w) || n > y->size_ || n > x->size_ || n > z->size_ ||
      n > w->size_)
    return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_xyzw<float><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, a, b, cc, d, e, f, (const float *)x->v_,
                                                           (float *)y->v_, (float *)z->v_, (float *)w->v_);
  PSBX_LAUNCH_CK("k_xyzw<float>");
  return SPGPU_SUCCESS;
}

int axyMultiVecDeviceFloat(int n, float alpha, void *devVecA, void *devVecB) {
  MultiVectDevice *a = MV(devVecA), *b = MV(devVecB);
  if (!is_f(a) || !is_f(b) || n > a->size_ || n > b->size_) return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_axybz<float><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, alpha, (const float *)a->v_, (const float *)b->v_,
                                                            0.0f, (float *)b->v_);
  PSBX_LAUNCH_CK("k_axy<float>");
  return SPGPU_SUCCESS;
}

int axybzMultiVecDeviceFloat(int n, float alpha, void *devVecA, void *devVecB, float beta, void *devVecZ) {
  MultiVectDevice *a = MV(devVecA), *b = MV(devVecB), *z = MV(devVecZ);
  if (!is_f(a) || !is_f(b) || !is_f(z) || n > a->size_ || n > b->size_ || n > z->size_) return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_axybz<float><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, alpha, (const float *)a->v_, (const float *)b->v_,
                                                            beta, (float *)z->v_);
  PSBX_LAUNCH_CK("k_axybz<float>");
  return SPGPU_SUCCESS;
}

int absMultiVecDeviceFloat2(int n, float alpha, void *devVecA, void *devVecB) {
  MultiVectDevice *a = MV(devVecA), *b = MV(devVecB);
  if (!is_f(a) || !is_f(b) || n > a->size_ || n > b->size_) return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_abs<float><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, alpha, (const float *)a->v_, (float *)b->v_);
  PSBX_LAUNCH_CK("k_abs<float>");
  return SPGPU_SUCCESS;
}

int absMultiVecDeviceFloat(int n, float alpha, void *devVecA) {
  return absMultiVecDeviceFloat2(n, alpha, devVecA, devVecA);
}

}  // extern "C"

// Gather / scatter / insert of FP32 and integer vectors: the same index
// conventions as the FP64 ones above (psb_s_vectordev_mod.F90,
// psb_i_vectordev_mod.F90; cuda/svectordev.c:127-177, ivectordev.c:127-180).
template <class T>
static int gath_t(void *deviceVec, int vectorId, int n, int first, const void *indexes, int hfirst, void *buf_,
                  int indexBase, int type) {
  MultiVectDevice *x = MV(deviceVec);
  if (!x || x->elemType != type || (n > 0 && (!indexes || !buf_)) || vectorId < 0 || vectorId >= x->count_)
    return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  const int *idx = (const int *)indexes + (first - indexBase);
  T *buf = (T *)buf_ + (hfirst - indexBase);
  const T *v = (const T *)x->v_ + (size_t)vectorId * x->pitch_;
  k_gath<T><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, idx, indexBase, v, buf);
  PSBX_LAUNCH_CK("k_gath");
  return SPGPU_SUCCESS;
}

template <class T>
static int scat_t(void *deviceVec, int vectorId, int n, int first, const void *indexes, int hfirst,
                  const void *buf_, int indexBase, T beta, int type) {
  MultiVectDevice *x = MV(deviceVec);
  if (!x || x->elemType != type || (n > 0 && (!indexes || !buf_)) || vectorId < 0 || vectorId >= x->count_)
    return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  const int *idx = (const int *)indexes + (first - indexBase);
  const T *buf = (const T *)buf_ + (hfirst - indexBase);
  T *v = (T *)x->v_ + (size_t)vectorId * x->pitch_;
  k_scat<T><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, idx, indexBase, buf, beta, v);
  PSBX_LAUNCH_CK("k_scat");
  return SPGPU_SUCCESS;
}

template <class T>
static int geins_t(int n, void *devMultiVecIrl, void *devMultiVecVal, int dupl, int indexBase, void *devMultiVecX,
                   int type) {
  MultiVectDevice *irl = MV(devMultiVecIrl), *val = MV(devMultiVecVal), *x = MV(devMultiVecX);
  if (!irl || !val || !x || x->elemType != type || n > irl->size_ || n > val->size_) return SPGPU_UNSUPPORTED;
  if (n <= 0) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_scat<T><<<psbx_grid_for(n, VT), VT, 0, c.stream>>>(n, (const int *)irl->v_, indexBase, (const T *)val->v_,
                                                       dupl == 1 ? T(1) : T(0), (T *)x->v_);
  PSBX_LAUNCH_CK("k_scat (geins)");
  return SPGPU_SUCCESS;
}

extern "C" {

int igathMultiVecDeviceFloat(void *deviceVec, int vectorId, int n, int first, void *indexes, int hfirst,
                             void *host_values, int indexBase) {
  return gath_t<float>(deviceVec, vectorId, n, first, indexes, hfirst, host_values, indexBase, SPGPU_TYPE_FLOAT);
}
int igathMultiVecDeviceFloatVecIdx(void *deviceVec, int vectorId, int n, int first, void *deviceIdx, int hfirst,
                                   void *host_values, int indexBase) {
  MultiVectDevice *ix = MV(deviceIdx);
  if (!ix) return SPGPU_UNSUPPORTED;
  return gath_t<float>(deviceVec, vectorId, n, first, ix->v_, hfirst, host_values, indexBase, SPGPU_TYPE_FLOAT);
}
int iscatMultiVecDeviceFloat(void *deviceVec, int vectorId, int n, int first, void *indexes, int hfirst,
                             void *host_values, int indexBase, float beta) {
  return scat_t<float>(deviceVec, vectorId, n, first, indexes, hfirst, host_values, indexBase, beta,
                       SPGPU_TYPE_FLOAT);
}
int iscatMultiVecDeviceFloatVecIdx(void *deviceVec, int vectorId, int n, int first, void *deviceIdx, int hfirst,
                                   void *host_values, int indexBase, float beta) {
  MultiVectDevice *ix = MV(deviceIdx);
  if (!ix) return SPGPU_UNSUPPORTED;
  return scat_t<float>(deviceVec, vectorId, n, first, ix->v_, hfirst, host_values, indexBase, beta,
                       SPGPU_TYPE_FLOAT);
}
int geinsMultiVecDeviceFloat(int n, void *devMultiVecIrl, void *devMultiVecVal, int dupl, int indexBase,
                             void *devMultiVecX) {
  return geins_t<float>(n, devMultiVecIrl, devMultiVecVal, dupl, indexBase, devMultiVecX, SPGPU_TYPE_FLOAT);
}

// ===================================================================== int
// cuda/ivectordev.c (the psb_i_vect_cuda glue: index vectors of halo
// exchanges and of the ELL value updates).
int writeMultiVecDeviceInt(void *deviceVec, int *hostVec) {
  return vec_copy(deviceVec, hostVec, true, SPGPU_TYPE_INT);
}
int writeMultiVecDeviceIntR2(void *deviceVec, int *hostVec, int ld) {
  (void)ld;
  return vec_copy(deviceVec, hostVec, true, SPGPU_TYPE_INT);
}
int readMultiVecDeviceInt(void *deviceVec, int *hostVec) {
  return vec_copy(deviceVec, hostVec, false, SPGPU_TYPE_INT);
}
int readMultiVecDeviceIntR2(void *deviceVec, int *hostVec, int ld) {
  (void)ld;
  return vec_copy(deviceVec, hostVec, false, SPGPU_TYPE_INT);
}

int setscalMultiVecDeviceInt(int val, int first, int last, int indexBase, void *devVecX) {
  MultiVectDevice *x = MV(devVecX);
  if (!is_i(x)) return SPGPU_UNSUPPORTED;
  int f = first - indexBase, l = last - indexBase;
  if (f < 0 || l >= x->pitch_ * x->count_) return SPGPU_UNSUPPORTED;
  if (l < f) return SPGPU_SUCCESS;
  PsbxCtx &c = psbx_ctx();
  k_setscal<int><<<psbx_grid_for(l - f + 1, VT), VT, 0, c.stream>>>(f, l, val, (int *)x->v_);
  PSBX_LAUNCH_CK("k_setscal<int>");
  return SPGPU_SUCCESS;
}

int igathMultiVecDeviceInt(void *deviceVec, int vectorId, int n, int first, void *indexes, int hfirst,
                           void *host_values, int indexBase) {
  return gath_t<int>(deviceVec, vectorId, n, first, indexes, hfirst, host_values, indexBase, SPGPU_TYPE_INT);
}
int igathMultiVecDeviceIntVecIdx(void *deviceVec, int vectorId, int n, int first, void *deviceIdx, int hfirst,
                                 void *host_values, int indexBase) {
  MultiVectDevice *ix = MV(deviceIdx);
  if (!ix) return SPGPU_UNSUPPORTED;
  return gath_t<int>(deviceVec, vectorId, n, first, ix->v_, hfirst, host_values, indexBase, SPGPU_TYPE_INT);
}
int iscatMultiVecDeviceInt(void *deviceVec, int vectorId, int n, int first, void *indexes, int hfirst,
                           void *host_values, int indexBase, int beta) {
  return scat_t<int>(deviceVec, vectorId, n, first, indexes, hfirst, host_values, indexBase, beta, SPGPU_TYPE_INT);
}
int iscatMultiVecDeviceIntVecIdx(void *deviceVec, int vectorId, int n, int first, void *deviceIdx, int hfirst,
                                 void *host_values, int indexBase, int beta) {
  MultiVectDevice *ix = MV(deviceIdx);
  if (!ix) return SPGPU_UNSUPPORTED;
  return scat_t<int>(deviceVec, vectorId, n, first, ix->v_, hfirst, host_values, indexBase, beta, SPGPU_TYPE_INT);
}
int geinsMultiVecDeviceInt(int n, void *devMultiVecIrl, void *devMultiVecVal, int dupl, int indexBase,
                           void *devMultiVecX) {
  return geins_t<int>(n, devMultiVecIrl, devMultiVecVal, dupl, indexBase, devMultiVecX, SPGPU_TYPE_INT);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free dot products.
//
// dotMultiVecDeviceDouble keeps its per-block partial sums in scratch that
// the library allocates with cudaMalloc the first time it is used.  Some
// callers cannot let a library call cudaMalloc: code that owns every byte
// of device memory through its own pool or a fixed budget, and latency-
// critical loops where an allocation would synchronise the device.  For
// them psbx_dot_noalloc runs the same reduction kernel with its scratch in
// the file-scope device arrays below (512 KiB of partial pairs plus 8
// tickets, present on every GPU that loads the library until the process
// exits) and allocates nothing.
// ---------------------------------------------------------------------------
#define PSBX_NOALLOC_MAX_VECS PSBX_NLANES
#define PSBX_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double psbx_noalloc_part[2 * PSBX_NLANES * PSBX_MAX_PART];
static __device__ __align__(256) unsigned psbx_noalloc_ticket[PSBX_NLANES];

static double *g_na_part[PSBX_NOALLOC_MAX_DEVICES];
static unsigned *g_na_ticket[PSBX_NOALLOC_MAX_DEVICES];
static int g_na_sms[PSBX_NOALLOC_MAX_DEVICES];
static bool g_na_ready[PSBX_NOALLOC_MAX_DEVICES];

// Once per device, with that device current: the device addresses of the
// scratch arrays (in host code their names are host-side stand-ins, not
// device addresses), the SM count for the grid size, and the tickets set to
// zero.  After that every call leaves the tickets at zero itself: the last
// block of each vector's reduction resets its ticket (k_reduce).
static int noalloc_setup(int dev) {
  if (g_na_ready[dev]) return SPGPU_SUCCESS;
  cudaError_t e = cudaGetSymbolAddress((void **)&g_na_part[dev], psbx_noalloc_part);
  if (e != cudaSuccess) return psbx_cuda_status(e, "cudaGetSymbolAddress(psbx_noalloc_part)");
  e = cudaGetSymbolAddress((void **)&g_na_ticket[dev], psbx_noalloc_ticket);
  if (e != cudaSuccess) return psbx_cuda_status(e, "cudaGetSymbolAddress(psbx_noalloc_ticket)");
  e = cudaDeviceGetAttribute(&g_na_sms[dev], cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return psbx_cuda_status(e, "cudaDeviceGetAttribute");
  e = cudaMemset(g_na_ticket[dev], 0, sizeof(unsigned) * PSBX_NOALLOC_MAX_VECS);
  if (e != cudaSuccess) return psbx_cuda_status(e, "cudaMemset(ticket)");
  g_na_ready[dev] = true;
  return SPGPU_SUCCESS;
}

// Called when the library context is released (gpuClose, cudaReset,
// psb_cudaDestroyHandle): a context created afterwards may place the scratch
// arrays elsewhere, so the next call looks their addresses up again.
void psbx_noalloc_forget(void) {
  for (int d = 0; d < PSBX_NOALLOC_MAX_DEVICES; d++) g_na_ready[d] = false;
}

extern "C" int psbx_dot_noalloc(double *d_res, int n, int count, const double *x, const double *y, int pitch,
                                void *stream) {
  if (count < 1 || count > PSBX_NOALLOC_MAX_VECS) {
    psbx_set_error("psbx_dot_noalloc: count must be between 1 and 8 (the size of its fixed scratch)");
    return SPGPU_UNSUPPORTED;
  }
  if (n < 0 || !d_res || !x || !y || (count > 1 && pitch < n)) {
    psbx_set_error("psbx_dot_noalloc: invalid arguments");
    return SPGPU_UNSUPPORTED;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return psbx_cuda_status(e, "cudaGetDevice");
  if (dev < 0 || dev >= PSBX_NOALLOC_MAX_DEVICES) {
    psbx_set_error("psbx_dot_noalloc: device ordinal beyond 63");
    return SPGPU_UNSUPPORTED;
  }
  int rc = noalloc_setup(dev);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  long long blocks = ((long long)(n > 0 ? n : 1) + VT * 4 - 1) / (VT * 4);
  long long cap = (long long)g_na_sms[dev] * 4;
  int g = (int)(blocks < cap ? blocks : cap);
  if (g > PSBX_MAX_PART) g = PSBX_MAX_PART;
  if (g < 1) g = 1;
  const int px = count > 1 ? pitch : n;
  k_reduce<R_DOT, double><<<dim3(g, count), VT, 0, st>>>(n, x, px, y, px, g_na_part[dev], g_na_ticket[dev], d_res);
  PSBX_LAUNCH_CK("k_reduce (noalloc)");
  return SPGPU_SUCCESS;
}
