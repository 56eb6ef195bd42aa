// vec.cu - vector kernels and the scalar recurrences of PCG, with every
// reduction deterministic (fixed block order) and kept on the device: the
// Krylov scalars never travel to the host inside an iteration. This replaces
// the three host round trips per PCG iteration of the reference
// (float(cp.dot(...)) at src/gpu_fem/solver_v2.py:607,611,619).
#include "internal.cuh"
#include "reduce.cuh"

namespace topo {

static inline unsigned grid_for(long long n, int bs, unsigned cap = 4096) {
  long long b = (n + bs - 1) / bs;
  if (b < 1) b = 1;
  return (unsigned)(b > cap ? cap : b);
}

template <typename T>
__global__ void k_fill(long long n, T* x, T v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] = v;
}

void vfill(bool f64, long long n, void* x, double v, cudaStream_t s) {
  if (f64) k_fill<double><<<grid_for(n, 256), 256, 0, s>>>(n, (double*)x, v);
  else k_fill<float><<<grid_for(n, 256), 256, 0, s>>>(n, (float*)x, (float)v);
  TOPO_LAUNCH_CHECK();
}

void vcopy(bool f64, long long n, const void* a, void* b, cudaStream_t s) {
  TOPO_CUDA_CHECK(cudaMemcpyAsync(b, a, (size_t)n * (f64 ? 8 : 4), cudaMemcpyDeviceToDevice, s));
}

template <typename A, typename B>
__global__ void k_cast(long long n, const A* __restrict__ a, B* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (B)a[i];
}

void vcast(long long n, const void* src, bool src64, void* dst, bool dst64, cudaStream_t s) {
  const unsigned nb = grid_for(n, 256);
  if (src64 == dst64) {
    vcopy(src64, n, src, dst, s);
    return;
  }
  if (src64) k_cast<double, float><<<nb, 256, 0, s>>>(n, (const double*)src, (float*)dst);
  else k_cast<float, double><<<nb, 256, 0, s>>>(n, (const float*)src, (double*)dst);
  TOPO_LAUNCH_CHECK();
}

template <typename T>
__global__ void k_mask(long long n, T* x, const uint8_t* m) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (!m[i]) x[i] = 0;
}

void vmask(bool f64, long long n, void* x, const uint8_t* mask, cudaStream_t s) {
  if (f64) k_mask<double><<<grid_for(n, 256), 256, 0, s>>>(n, (double*)x, mask);
  else k_mask<float><<<grid_for(n, 256), 256, 0, s>>>(n, (float*)x, mask);
  TOPO_LAUNCH_CHECK();
}

// First Chebyshev step on the current residual (from x0 = 0 the residual is
// b itself: K 0 = 0, no operator application): d = c2 D^-1 r, x += ax d.
template <typename T>
__global__ void k_cheb_start(long long n, const T* __restrict__ b, T* __restrict__ r, const T* __restrict__ dinv,
                             T c2, T ax, T* __restrict__ x, T* __restrict__ d, int x_is_zero, const KrylovState* st) {
  if (st != nullptr && st->done) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    T ri;
    if (b != nullptr) {
      ri = b[i];
      r[i] = ri;
    } else {
      ri = r[i];
    }
    const T v = c2 * (dinv[i] * ri);
    d[i] = v;
    x[i] = (x_is_zero ? (T)0 : x[i]) + ax * v;
  }
}

void cheb_start(bool f64, long long n, const void* b, void* r, const void* dinv, double c2, double ax, void* x,
                void* d, bool x_is_zero, const KrylovState* st, cudaStream_t s) {
  if (f64)
    k_cheb_start<double><<<grid_for(n, 256), 256, 0, s>>>(n, (const double*)b, (double*)r, (const double*)dinv, c2,
                                                          ax, (double*)x, (double*)d, x_is_zero, st);
  else
    k_cheb_start<float><<<grid_for(n, 256), 256, 0, s>>>(n, (const float*)b, (float*)r, (const float*)dinv,
                                                         (float)c2, (float)ax, (float*)x, (float*)d, x_is_zero, st);
  TOPO_LAUNCH_CHECK();
}

// ------------------------------------------------------------------- dots
template <typename T>
__global__ void k_dot(long long n, const T* __restrict__ a, const T* __restrict__ b, double* out, RedWork red) {
  double v[1] = {0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[0] += (double)a[i] * (double)b[i];
  double tot[1];
  if (grid_sum<1>(v, red, tot) && threadIdx.x == 0) *out = tot[0];
}

void dot_to(bool f64, long long n, const void* a, const void* b, double* out, RedWork red, cudaStream_t s) {
  const unsigned nb = grid_for(n, kRedThreads, kRedBlocks);
  if (f64) k_dot<double><<<nb, kRedThreads, 0, s>>>(n, (const double*)a, (const double*)b, out, red);
  else k_dot<float><<<nb, kRedThreads, 0, s>>>(n, (const float*)a, (const float*)b, out, red);
  TOPO_LAUNCH_CHECK();
}

double dot_host(bool f64, long long n, const void* a, const void* b, RedWork red, double* dev_tmp, cudaStream_t s) {
  dot_to(f64, n, a, b, dev_tmp, red, s);
  double h = 0.0;
  TOPO_CUDA_CHECK(cudaMemcpyAsync(&h, dev_tmp, sizeof(double), cudaMemcpyDeviceToHost, s));
  TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
  return h;
}

// --------------------------------------------------------------------- PCG
__global__ void k_pcg_init(KrylovState* st, double tol) {
  st->tol2 = tol * tol * st->bb;
  st->done = 0;
  st->converged = 0;
  st->iters = 0;
}

void pcg_init(KrylovState* st, double tol, cudaStream_t s) {
  k_pcg_init<<<1, 1, 0, s>>>(st, tol);
  TOPO_LAUNCH_CHECK();
}

// x += alpha p ; r -= alpha Ap ; rr = r.r ; done when rr <= tol^2 b.b.
// The iterate x is FP64 whatever the working precision T of r, p, Ap, so an
// FP32 solve is not capped by the FP32 representation of x (reliable update).
template <typename T>
__global__ void k_pcg_xr(long long n, double* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                         const T* __restrict__ Ap, KrylovState* st, RedWork red) {
  if (st->done) return;
  const double alpha64 = st->alpha;
  const T alpha = (T)alpha64;
  double v[1] = {0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    x[i] += alpha64 * (double)p[i];
    const T ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    v[0] += (double)ri * (double)ri;
  }
  double tot[1];
  if (grid_sum<1>(v, red, tot) && threadIdx.x == 0) {
    st->rr = tot[0];
    if (tot[0] <= st->tol2) {
      st->done = 1;
      st->converged = 1;
    }
  }
}

void pcg_xr_update(bool f64, long long n, void* x, void* r, const void* p, const void* Ap, KrylovState* st,
                   RedWork red, cudaStream_t s) {
  const unsigned nb = grid_for(n, kRedThreads, kRedBlocks);
  if (f64)
    k_pcg_xr<double><<<nb, kRedThreads, 0, s>>>(n, (double*)x, (double*)r, (const double*)p, (const double*)Ap, st, red);
  else
    k_pcg_xr<float><<<nb, kRedThreads, 0, s>>>(n, (double*)x, (float*)r, (const float*)p, (const float*)Ap, st, red);
  TOPO_LAUNCH_CHECK();
}

// rz_new = r.z ; beta = rz_new / rz ; one more preconditioner application
template <typename T>
__global__ void k_pcg_rz(long long n, const T* __restrict__ r, const T* __restrict__ z, KrylovState* st,
                         RedWork red, int first) {
  if (st->done) return;
  double v[1] = {0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[0] += (double)r[i] * (double)z[i];
  double tot[1];
  if (grid_sum<1>(v, red, tot) && threadIdx.x == 0) {
    if (first) {
      st->beta = 0.0;
    } else {
      st->beta = tot[0] / st->rz;
    }
    st->rz = tot[0];
    st->iters += 1;
  }
}

void pcg_rz(bool f64, long long n, const void* r, const void* z, KrylovState* st, RedWork red, bool first,
            cudaStream_t s) {
  const unsigned nb = grid_for(n, kRedThreads, kRedBlocks);
  if (f64) k_pcg_rz<double><<<nb, kRedThreads, 0, s>>>(n, (const double*)r, (const double*)z, st, red, first);
  else k_pcg_rz<float><<<nb, kRedThreads, 0, s>>>(n, (const float*)r, (const float*)z, st, red, first);
  TOPO_LAUNCH_CHECK();
}

template <typename T>
__global__ void k_pcg_p(long long n, const T* __restrict__ z, T* __restrict__ p, const KrylovState* st, int first) {
  if (st->done) return;
  const T beta = first ? (T)0 : (T)st->beta;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = first ? z[i] : z[i] + beta * p[i];
}

void pcg_p_update(bool f64, long long n, const void* z, void* p, KrylovState* st, bool first, cudaStream_t s) {
  if (f64) k_pcg_p<double><<<grid_for(n, 256), 256, 0, s>>>(n, (const double*)z, (double*)p, st, first);
  else k_pcg_p<float><<<grid_for(n, 256), 256, 0, s>>>(n, (const float*)z, (float*)p, st, first);
  TOPO_LAUNCH_CHECK();
}

// x64 += a * z (z in the working precision)
template <typename T>
__global__ void k_axpy64(long long n, double a, const T* __restrict__ z, double* __restrict__ x) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] += a * (double)z[i];
}

void axpy_to64(bool f64, long long n, double a, const void* z, double* x, cudaStream_t s) {
  if (f64) k_axpy64<double><<<grid_for(n, 256), 256, 0, s>>>(n, a, (const double*)z, x);
  else k_axpy64<float><<<grid_for(n, 256), 256, 0, s>>>(n, a, (const float*)z, x);
  TOPO_LAUNCH_CHECK();
}

// y = a x + b y (host scalars)
template <typename T>
__global__ void k_axpby(long long n, T a, const T* __restrict__ x, T b, T* __restrict__ y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}

void axpby(bool f64, long long n, double a, const void* x, double b, void* y, cudaStream_t s) {
  if (f64) k_axpby<double><<<grid_for(n, 256), 256, 0, s>>>(n, a, (const double*)x, b, (double*)y);
  else k_axpby<float><<<grid_for(n, 256), 256, 0, s>>>(n, (float)a, (const float*)x, (float)b, (float*)y);
  TOPO_LAUNCH_CHECK();
}

// y = x * (*num / *den) with device scalars
template <typename T>
__global__ void k_scale_dev(long long n, const T* __restrict__ x, const double* num, const double* den, T* __restrict__ y) {
  const T f = (T)(*num / *den);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = f * x[i];
}

void scale_dev(bool f64, long long n, const void* x, const double* num, const double* den, void* y, cudaStream_t s) {
  if (f64) k_scale_dev<double><<<grid_for(n, 256), 256, 0, s>>>(n, (const double*)x, num, den, (double*)y);
  else k_scale_dev<float><<<grid_for(n, 256), 256, 0, s>>>(n, (const float*)x, num, den, (float*)y);
  TOPO_LAUNCH_CHECK();
}

}  // namespace topo
