// ctx.cu - the context object, multigrid setup, V-cycle, Krylov drivers and
// the extern "C" entry points declared in include/topo_b200.h.
//
// One PCG iteration (outer matvec + fused dot, x/r update, full V-cycle, r.z,
// p update) is recorded once per solve into a CUDA graph and replayed; every
// kernel in it returns at entry once the device-side convergence flag is set,
// so the host only polls that flag every few replays.
#include "internal.cuh"
#include "reduce.cuh"
#include "../../include/topo_b200.h"

#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace topo {

void level0_apply_bf16_input(const Grid& g, const void* u, const void* E, const uint8_t* mask, void* y,
                             cudaStream_t s);

static std::atomic<long long> g_launches{0};
void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

static std::mutex g_err_mu;
static std::string g_err;
void set_global_error(const std::string& m) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_err = m;
}
std::string global_error() {
  std::lock_guard<std::mutex> lk(g_err_mu);
  return g_err;
}

// Small helper kernels for the spectral estimates ---------------------------
// out = sum_i a_i b_i / dinv_i over entries with dinv_i != 0  (v^T D v)
template <typename T>
__global__ void k_dot_div(long long n, const T* __restrict__ a, const T* __restrict__ b, const T* __restrict__ dinv,
                          double* out, RedWork red) {
  double v[1] = {0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (dinv[i] != (T)0) v[0] += (double)a[i] * (double)b[i] / (double)dinv[i];
  double tot[1];
  if (grid_sum<1>(v, red, tot) && threadIdx.x == 0) *out = tot[0];
}

// y = dinv .* x
template <typename T>
__global__ void k_hadamard(long long n, const T* __restrict__ dinv, const T* __restrict__ x, T* __restrict__ y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = dinv[i] * x[i];
}

template <typename T>
__global__ void k_dinv_from_diag(long long n, const double* __restrict__ diag, const uint8_t* __restrict__ mask,
                                 T* __restrict__ dinv) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double d = diag[i];
    d = fabs(d) > 1e-12 ? d : 1.0;
    dinv[i] = mask[i] ? (T)(1.0 / d) : (T)0;
  }
}

// Start vector of the power iterations on the free DoFs: all ones (the
// reference's choice), or, for the Chebyshev-iteration smoother, a fixed
// pseudo-random vector (splitmix64 of the index, values of both signs) whose
// high-frequency content makes 10-20 steps reach the top of the spectrum.
__device__ __forceinline__ double hashed_unit(unsigned long long i) {
  unsigned long long z = i + 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z ^= z >> 31;
  const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);  // [0, 1)
  return (u < 0.5 ? -1.0 : 1.0) * (0.5 + u);
}

template <typename T>
__global__ void k_mask_to(long long n, const uint8_t* __restrict__ m, T* __restrict__ v, int random) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i] = m[i] ? (random ? (T)hashed_unit((unsigned long long)i) : (T)1) : (T)0;
}

template <typename T>
__global__ void k_gather_zero(long long n_full, T* __restrict__ x) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_full; i += (long long)gridDim.x * blockDim.x)
    x[i] = 0;
}

// Per-node free bits from the per-DoF mask: bit c set <=> DoF 3n+c is free.
__global__ void k_node_mask(long long nnodes, const uint8_t* __restrict__ mask, uint8_t* __restrict__ nmask) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nnodes; n += (long long)gridDim.x * blockDim.x)
    nmask[n] = (uint8_t)((mask[3 * n] ? 1 : 0) | (mask[3 * n + 1] ? 2 : 0) | (mask[3 * n + 2] ? 4 : 0));
}

__global__ void k_add_diag(int n, double* A, double eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) A[(long long)i * n + i] += eps;
}

__global__ void k_diag_sum(int n, const double* A, double* out) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += A[(long long)i * n + i];
  double a[1] = {v};
  block_sum<1>(a);
  if (threadIdx.x == 0) *out = a[0];
}

static unsigned gblocks(long long n, int bs = 256) {
  long long b = (n + bs - 1) / bs;
  return (unsigned)std::max<long long>(1, std::min<long long>(b, 4096));
}

// ---------------------------------------------------------------- context
struct Level {
  Grid g;
  Prec prec = Prec::F64;
  uint8_t* mask = nullptr;
  void* x = nullptr;     // iterate
  void* r = nullptr;     // residual
  void* d = nullptr;     // Chebyshev directions (ping-pong)
  void* d2 = nullptr;
  void* e = nullptr;     // prolongated coarse correction
  void* b = nullptr;     // right-hand side
  void* dinv = nullptr;  // Jacobi inverse diagonal
  double* S64 = nullptr;
  float* S32 = nullptr;
  __nv_bfloat16* S16 = nullptr;
  double lam = NAN;
  int degree = 2;
};

// One factorisation of the coarsest operator, with the stencil it is built from.
struct FactorSlot {
  double* S64c = nullptr;   // copy of the coarsest stencil the factor is built from
  CoarsestFactor f;
};

struct Coarsest {
  int n = 0;
  int band = 0;
  int* dof_index = nullptr;
  int* free_list = nullptr;
  CoarsestPlan plan;
  double* y = nullptr;      // 2n FP64: the forward and backward sweep vectors of the apply
  FactorSlot cur;           // the factor the V-cycle applies
  FactorSlot nxt;           // with coarse_lag: the factor being built in the background
  bool have = false;        // cur holds a factor
  bool bg_pending = false;  // nxt is being built on bg_stream
  cudaStream_t bg_stream = nullptr;
  cudaEvent_t ev_copy = nullptr, bg_done = nullptr;
  // set-up side stream: the coarse-level Jacobi diagonals, spectral bounds
  // and stencil copies run there while the coarsest factorisation runs
  cudaStream_t side = nullptr;
  cudaEvent_t ev_rap = nullptr, ev_side = nullptr;
  double* tmp = nullptr;   // FP64 Jacobi inverse of a coarse level when vectors are FP32
  double* scrA = nullptr;  // FP64 scratch vectors for the coarse power iterations
  double* scrB = nullptr;
  double* scrC = nullptr;
};

}  // namespace topo

using namespace topo;

struct topo_ctx {
  int device = 0;
  int mode = TOPO_MODE_FP64;
  bool vec64 = true;
  int n_levels = 1;
  int fine_degree = 2, coarse_degree = 2;
  double cheb_lower = 1.0 / 30.0;
  int cheb_form = 1;          // 0 reference recurrence, 1 Chebyshev iteration
  double lam_safety = 1.25;   // factor on the power-iteration lambda_max
  int dense_max = 16384;
  bool use_tc = true;         // BF16 level-0 operator on tcgen05 (TOPO_B200_NO_TC=1: CUDA cores)
  int cycle_gamma = 1;        // coarse corrections per level: 1 V-cycle, 2 W-cycle
  bool coarse_lag = false;    // V-cycle uses the previous setup's coarsest factor; the new one builds in the background
  std::vector<Level> L;
  Coarsest C;
  double* E64 = nullptr;
  float* E32 = nullptr;
  uint8_t* nmask0 = nullptr;  // level 0: per-node free bits, bit c = DoF 3n+c (read by the tensor-core K.u)
  double* diag0 = nullptr;
  double lam_Emax = NAN;
  bool problem_set = false;
  bool setup_done = false;
  // Krylov vectors (level 0, vector precision)
  void *kr = nullptr, *kz = nullptr, *kp = nullptr, *kAp = nullptr, *kt = nullptr;
  double *kx64 = nullptr, *kb64 = nullptr, *kr64 = nullptr;  // FP64 iterate, rhs, true residual
  void* Fvec = nullptr;
  // FGMRES basis (allocated on demand)
  std::vector<void*> fg_V, fg_Z;
  KrylovState* st = nullptr;
  // PCG iteration graph, kept across solves while its key (everything the
  // capture bakes in: Chebyshev bounds, options, buffer addresses) is unchanged
  cudaGraphExec_t pcg_exec = nullptr;
  long long pcg_exec_kernels = 0;
  std::vector<double> pcg_key;
  // block PCG workspace (FP64 columns R, Z, P, Q, Pn; allocated per block width)
  int blk_nv = 0;
  double* blk = nullptr;
  double* blk_part = nullptr;
  double* blk_G = nullptr;
  double* blk_Gh = nullptr;  // pinned host copy
  KrylovState* h_st = nullptr;  // pinned host mirror
  RedWork red{};
  double* dtmp = nullptr;       // 64 device doubles
  double* oc_state = nullptr;
  double* Hs = nullptr;
  FilterStencil fstencil;
  bool ke_registered = false;  // holds a reference on its device's KE
  cudaStream_t cs = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  cudaEvent_t ev_ph[6] = {};     // setup phase marks (timed)
  double setup_ms[5] = {0, 0, 0, 0, 0};
  std::vector<void*> allocs;
  long long bytes = 0;
  std::string err;

  template <typename T>
  T* alloc(long long count) {
    void* p = nullptr;
    const size_t sz = (size_t)std::max<long long>(count, 1) * sizeof(T);
    TOPO_CUDA_CHECK(cudaMalloc(&p, sz));
    TOPO_CUDA_CHECK(cudaMemset(p, 0, sz));
    allocs.push_back(p);
    bytes += (long long)sz;
    return (T*)p;
  }
  void* valloc(long long count) { return vec64 ? (void*)alloc<double>(count) : (void*)alloc<float>(count); }
  size_t vsize() const { return vec64 ? 8 : 4; }
};

namespace {

struct StreamGuard {
  topo_ctx* c;
  cudaStream_t user;
  StreamGuard(topo_ctx* ctx, void* stream) : c(ctx), user((cudaStream_t)stream) {
    TOPO_CUDA_CHECK(cudaSetDevice(c->device));
    TOPO_CUDA_CHECK(cudaEventRecord(c->ev_in, user));
    TOPO_CUDA_CHECK(cudaStreamWaitEvent(c->cs, c->ev_in, 0));
  }
  ~StreamGuard() {
    if (cudaEventRecord(c->ev_out, c->cs) == cudaSuccess) cudaStreamWaitEvent(user, c->ev_out, 0);
  }
};

int fail(topo_ctx* c, const std::exception& e) {
  if (c) c->err = e.what();
  set_global_error(e.what());
  return -1;
}

Prec outer_prec(const topo_ctx* c) { return c->vec64 ? Prec::F64 : Prec::F32; }
const void* outer_E(const topo_ctx* c) { return c->vec64 ? (const void*)c->E64 : (const void*)c->E32; }

// ----------------------------------------------------------- operators
void op_apply(topo_ctx* c, int l, Prec p, const void* u, void* y, Epi epi, const EpiArgs& ea, cudaStream_t s) {
  Level& Lv = c->L[l];
  if (l == 0) {
    const void* E = (p == Prec::F64) ? (const void*)c->E64 : (const void*)c->E32;
    if (p == Prec::BF16 && c->use_tc && level0_xs_supported(Lv.g))
      level0_apply_xs(false, Lv.g, u, E, c->nmask0, y, epi, ea, s);
    else level0_apply(p, Lv.g, u, E, Lv.mask, y, epi, ea, s);
  } else {
    const void* S = p == Prec::F64 ? (const void*)Lv.S64 : p == Prec::F32 ? (const void*)Lv.S32 : (const void*)Lv.S16;
    stencil_apply(p, c->vec64, Lv.g, S, u, Lv.mask, y, epi, ea, s);
  }
}

// Precision of the one update per V-cycle applied to a smooth vector (the
// prolongated correction): a BF16-input level uses its FP32 operator there.

Prec hi_prec(const Level& Lv) { return Lv.prec == Prec::BF16 ? Prec::F32 : Lv.prec; }

// Chebyshev-Jacobi smoothing on level l (reference: multigrid_v4.py:861-889)
// with a recursive residual: Lv.x and Lv.r are updated in place and the
// operator only ever multiplies a direction. from_zero: x = 0 and r = b.
// want_residual: also form the final residual r = b - K x (one more
// application, which replaces the reference's separate residual matvec).
void smooth(topo_ctx* c, int l, bool from_zero, bool want_residual, const KrylovState* st, cudaStream_t s) {
  Level& Lv = c->L[l];
  const double lam = (std::isfinite(Lv.lam) ? Lv.lam : 1.0) * c->lam_safety;
  const Cheb ch = make_cheb(lam, c->cheb_lower, Lv.degree, c->cheb_form);
  const long long n = Lv.g.ndof;
  cheb_start(c->vec64, n, from_zero ? Lv.b : nullptr, Lv.r, Lv.dinv, ch.c2[0], ch.ax[0], Lv.x, Lv.d, from_zero, st,
             s);
  void* dcur = Lv.d;
  void* dnext = Lv.d2;
  for (int j = 1; j < Lv.degree; ++j) {
    EpiArgs ea{};
    ea.dinv = Lv.dinv;
    ea.r = Lv.r;
    ea.x = Lv.x;
    ea.d_out = dnext;
    ea.s = ch.ax[j - 1];
    ea.c1 = ch.c1[j];
    ea.c2 = ch.c2[j];
    ea.ax = ch.ax[j];
    ea.st = const_cast<KrylovState*>(st);
    op_apply(c, l, Lv.prec, dcur, nullptr, Epi::ChebR, ea, s);
    std::swap(dcur, dnext);
  }
  if (want_residual) {
    EpiArgs ea{};
    ea.r = Lv.r;
    ea.s = ch.ax[Lv.degree - 1];
    ea.st = const_cast<KrylovState*>(st);
    op_apply(c, l, Lv.prec, dcur, nullptr, Epi::RUpd, ea, s);
  }
}

void coarsest_solve(topo_ctx* c, const KrylovState* st, cudaStream_t s) {
  const int l = c->n_levels - 1;
  Level& Lv = c->L[l];
  const long long n_full = Lv.g.ndof;
  if (c->vec64) k_gather_zero<double><<<gblocks(n_full), 256, 0, s>>>(n_full, (double*)Lv.x);
  else k_gather_zero<float><<<gblocks(n_full), 256, 0, s>>>(n_full, (float*)Lv.x);
  TOPO_LAUNCH_CHECK();
  if (c->C.n == 0) return;
  coarsest_apply(c->C.cur.f, c->vec64, Lv.b, c->C.y, Lv.x, st, s);
}

// One V-cycle (cycle_gamma 1, multigrid_v4.py:986-1008) or W-cycle
// (cycle_gamma 2, multigrid_v4.py:1010-1042) on level l: input Lv.b, output
// Lv.x. Each coarse correction restricts the recursive residual, recurses,
// adds e = P x_c and updates r -= K e, so the second correction of a W-cycle
// restricts b - K x without a separate residual product.
void vcycle(topo_ctx* c, int l, const KrylovState* st, cudaStream_t s) {
  Level& Lv = c->L[l];
  if (l == c->n_levels - 1) {
    if (c->n_levels == 1) smooth(c, 0, true, false, st, s);
    else coarsest_solve(c, st, s);
    return;
  }
  smooth(c, l, true, true, st, s);  // x = S b, r = b - K x
  Level& Lc = c->L[l + 1];
  for (int k = 0; k < c->cycle_gamma; ++k) {
    restrict_vec(c->vec64, Lv.g, Lc.g, Lv.r, Lc.mask, Lc.b, st, s);
    vcycle(c, l + 1, st, s);
    prolong_add(c->vec64, Lv.g, Lc.g, Lc.x, Lv.mask, Lv.x, Lv.e, st, s);  // x += e = P x_c
    EpiArgs ea{};
    ea.r = Lv.r;
    ea.s = 1.0;
    ea.st = const_cast<KrylovState*>(st);
    // r -= K e in FP32 even where the level's operator is BF16: the
    // post-smoother continues from this recursive residual, and BF16 here
    // raised the PCG iterations of the 1M-element cantilever from ~18 to ~95
    op_apply(c, l, hi_prec(Lv), Lv.e, nullptr, Epi::RUpd, ea, s);  // r -= K e
  }
  smooth(c, l, false, false, st, s);
}

void vcycle_apply(topo_ctx* c, const void* r, void* z, const KrylovState* st, cudaStream_t s) {
  Level& L0 = c->L[0];
  void* saved_b = L0.b;
  void* saved_x = L0.x;
  L0.b = const_cast<void*>(r);
  L0.x = z;
  vcycle(c, 0, st, s);
  L0.b = saved_b;
  L0.x = saved_x;
}

// ------------------------------------------------------- spectral bounds
// The power iterations keep their scalars on the device (dot products into
// dtmp, normalisations by kernels that read them) and read lambda back once
// at the end: no host round trip per iteration.

// y = x / sqrt(*s2) when *s2 > 0 (y keeps its value otherwise)
template <typename T>
__global__ void k_scale_rsqrt(long long n, const T* __restrict__ x, const double* s2, T* __restrict__ y) {
  const double q = *s2;
  if (!(q > 0.0)) return;
  const T f = (T)(1.0 / sqrt(q));
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = f * x[i];
}

// Keep the iteration's Rayleigh quotient parts (num, den) when its update
// norm is non-zero (the reference stops before a zero-norm update).
__global__ void k_commit_lambda(double* d) {
  if (d[2] > 0.0) {
    d[3] = d[1];
    d[4] = d[0];
  }
}

__global__ void k_set2(double* d, double a, double b) {
  d[3] = a;
  d[4] = b;
}

template <typename T>
static void scale_rsqrt(long long n, const void* x, const double* s2, void* y, cudaStream_t s) {
  k_scale_rsqrt<T><<<gblocks(n), 256, 0, s>>>(n, (const T*)x, s2, (T*)y);
  TOPO_LAUNCH_CHECK();
}

// lambda_max(D^-1 K) on level 0 by D-norm power iteration (multigrid_v4.py:273-295).
double lambda_fine(topo_ctx* c, cudaStream_t s) {
  Level& L0 = c->L[0];
  const long long n = L0.g.ndof;
  const bool f64 = c->vec64;
  void* v = L0.x;
  void* Kv = L0.r;
  void* Av = L0.d2;
  double* d = c->dtmp;  // d[0] v^T D v, d[1] v^T K v, d[2] |D^-1 K v|_D^2
  const int rnd = c->cheb_form == 1;
  if (f64) k_mask_to<double><<<gblocks(n), 256, 0, s>>>(n, L0.mask, (double*)v, rnd);
  else k_mask_to<float><<<gblocks(n), 256, 0, s>>>(n, L0.mask, (float*)v, rnd);
  TOPO_LAUNCH_CHECK();
  auto dotdiv = [&](const void* a, const void* b, double* out) {
    if (f64) k_dot_div<double><<<kRedBlocks, kRedThreads, 0, s>>>(n, (const double*)a, (const double*)b, (const double*)L0.dinv, out, c->red);
    else k_dot_div<float><<<kRedBlocks, kRedThreads, 0, s>>>(n, (const float*)a, (const float*)b, (const float*)L0.dinv, out, c->red);
    TOPO_LAUNCH_CHECK();
  };
  auto rs = [&](const void* x, const double* s2, void* y) {
    if (f64) scale_rsqrt<double>(n, x, s2, y, s);
    else scale_rsqrt<float>(n, x, s2, y, s);
  };
  dotdiv(v, v, d);
  rs(v, d, v);
  const Prec p = f64 ? Prec::F64 : Prec::F32;
  for (int it = 0; it < 20; ++it) {
    EpiArgs ea{};
    level0_apply(p, L0.g, v, f64 ? (const void*)c->E64 : (const void*)c->E32, L0.mask, Kv, Epi::Store, ea, s);
    dotdiv(v, v, d);
    dot_to(f64, n, v, Kv, d + 1, c->red, s);
    if (f64) k_hadamard<double><<<gblocks(n), 256, 0, s>>>(n, (const double*)L0.dinv, (const double*)Kv, (double*)Av);
    else k_hadamard<float><<<gblocks(n), 256, 0, s>>>(n, (const float*)L0.dinv, (const float*)Kv, (float*)Av);
    TOPO_LAUNCH_CHECK();
    dotdiv(Av, Av, d + 2);
    rs(Av, d + 2, v);
  }
  double h[2];
  TOPO_CUDA_CHECK(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
  TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
  return h[1] / std::max(h[0], 1e-300);
}

// Coarse level power iteration (multigrid_v4.py:298-314), FP64 stencil.
double lambda_coarse(topo_ctx* c, int l, double* dinv64, cudaStream_t s) {
  Level& Lv = c->L[l];
  const long long n = Lv.g.ndof;
  double* V = c->C.scrA;
  double* KV = c->C.scrB;
  double* AV = c->C.scrC;
  double* d = c->dtmp;  // d[0] v^T D v, d[1] v^T K v, d[2] |D^-1 K v|^2, d[3]/d[4] the kept quotient
  k_mask_to<double><<<gblocks(n), 256, 0, s>>>(n, Lv.mask, V, c->cheb_form == 1);
  TOPO_LAUNCH_CHECK();
  k_set2<<<1, 1, 0, s>>>(d, 1.0, 1.0);  // lambda 1 if the first update is zero
  TOPO_LAUNCH_CHECK();
  dot_to(true, n, V, V, d + 2, c->red, s);
  scale_rsqrt<double>(n, V, d + 2, V, s);
  for (int it = 0; it < 10; ++it) {
    EpiArgs ea{};
    stencil_apply(Prec::F64, true, Lv.g, Lv.S64, V, Lv.mask, KV, Epi::Store, ea, s);
    k_hadamard<double><<<gblocks(n), 256, 0, s>>>(n, dinv64, KV, AV);
    TOPO_LAUNCH_CHECK();
    dot_to(true, n, AV, AV, d + 2, c->red, s);
    dot_to(true, n, V, KV, d + 1, c->red, s);
    k_dot_div<double><<<kRedBlocks, kRedThreads, 0, s>>>(n, V, V, dinv64, d, c->red);
    TOPO_LAUNCH_CHECK();
    k_commit_lambda<<<1, 1, 0, s>>>(d);
    TOPO_LAUNCH_CHECK();
    scale_rsqrt<double>(n, AV, d + 2, V, s);
  }
  double h[2];
  TOPO_CUDA_CHECK(cudaMemcpyAsync(h, d + 3, sizeof(h), cudaMemcpyDeviceToHost, s));
  TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
  return std::max(h[0] / std::max(h[1], 1e-300), 1e-6);
}

// --------------------------------------------------------------- setup
void host_galerkin_q(const double* KE, double* Q) {
  static const int corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  for (int stu = 0; stu < 8; ++stu) {
    const int sv[3] = {stu >> 2, (stu >> 1) & 1, stu & 1};
    double P[8][8];
    for (int fn = 0; fn < 8; ++fn)
      for (int cn = 0; cn < 8; ++cn) {
        double w = 1.0;
        for (int d = 0; d < 3; ++d) {
          const double x = (sv[d] + corner[fn][d]) / 2.0;
          w *= corner[cn][d] ? x : 1.0 - x;
        }
        P[fn][cn] = w;
      }
    double* Qs = Q + stu * 576;
    for (int a = 0; a < 8; ++a)
      for (int cc = 0; cc < 3; ++cc)
        for (int b = 0; b < 8; ++b)
          for (int dd = 0; dd < 3; ++dd) {
            double acc = 0.0;
            for (int fn = 0; fn < 8; ++fn) {
              if (P[fn][a] == 0.0) continue;
              for (int fm = 0; fm < 8; ++fm) {
                if (P[fm][b] == 0.0) continue;
                acc += P[fn][a] * KE[(3 * fn + cc) * 24 + 3 * fm + dd] * P[fm][b];
              }
            }
            Qs[(3 * a + cc) * 24 + 3 * b + dd] = acc;
          }
  }
}

// ------------------------------------------------ coarsest factorisation
void* ctx_alloc_bytes(void* ctx, size_t bytes) {
  return static_cast<void*>(static_cast<topo_ctx*>(ctx)->alloc<char>((long long)bytes));
}

void alloc_slot(topo_ctx* c, FactorSlot& f) {
  f.S64c = c->alloc<double>(243LL * c->L[c->n_levels - 1].g.nnodes);
  coarsest_alloc(f.f, c->C.plan, c->C.band, c->vec64, ctx_alloc_bytes, c);
  f.f.d_free = c->C.free_list;
  f.f.kind = 0;
}

// Assembly (from the slot's stencil copy) and factorisation of one slot.
void slot_launch(topo_ctx* c, FactorSlot& f, cudaStream_t s) {
  const Level& Lc = c->L[c->n_levels - 1];
  coarsest_assemble(f.f, Lc.g, f.S64c, c->C.dof_index, s);
  coarsest_factor(f.f, s);
}

// After a slot's factorisation has run: read its pivot flag; on a
// non-positive pivot rebuild it from the stencil copy with eps*I added
// (multigrid_v4.py:778-811).
void slot_finish(topo_ctx* c, FactorSlot& f, cudaStream_t s) {
  const int st0 = coarsest_status(f.f, s);
  if (st0 < 0) throw std::runtime_error("coarsest-level Cholesky: a grid barrier wait timed out");
  if (st0 == 0) {
    f.f.kind = 1;
    return;
  }
  const Level& Lc = c->L[c->n_levels - 1];
  coarsest_assemble(f.f, Lc.g, f.S64c, c->C.dof_index, s);
  coarsest_regularise(f.f, c->dtmp, s);
  coarsest_factor(f.f, s);
  const int st1 = coarsest_status(f.f, s);
  if (st1 < 0) throw std::runtime_error("coarsest-level Cholesky: a grid barrier wait timed out");
  if (st1 > 0) throw std::runtime_error("coarsest-level Cholesky failed even after eps*I regularisation");
  f.f.kind = 2;
}

void coarse_wait_background(topo_ctx* c) {
  if (c->C.bg_pending) {
    TOPO_CUDA_CHECK(cudaEventSynchronize(c->C.bg_done));
    c->C.bg_pending = false;
  }
}

void do_setup(topo_ctx* c, const double* E, cudaStream_t s) {
  Level& L0 = c->L[0];
  const long long ne = L0.g.nelem;
  TOPO_CUDA_CHECK(cudaEventRecord(c->ev_ph[0], s));
  TOPO_CUDA_CHECK(cudaMemcpyAsync(c->E64, E, sizeof(double) * ne, cudaMemcpyDeviceToDevice, s));
  vcast(ne, c->E64, true, c->E32, false, s);
  // level-0 Jacobi diagonal (multigrid_v4.py:684-686)
  level0_diag(L0.g, c->E64, L0.mask, c->diag0, s);
  if (c->vec64) k_dinv_from_diag<double><<<gblocks(L0.g.ndof), 256, 0, s>>>(L0.g.ndof, c->diag0, L0.mask, (double*)L0.dinv);
  else k_dinv_from_diag<float><<<gblocks(L0.g.ndof), 256, 0, s>>>(L0.g.ndof, c->diag0, L0.mask, (float*)L0.dinv);
  TOPO_LAUNCH_CHECK();
  // re-estimate spectral bounds when max(E) moved by more than 10% (multigrid_v4.py:692-704)
  field_stats(ne, c->E64, c->dtmp + 8, c->red, s);
  double st4[4];
  TOPO_CUDA_CHECK(cudaMemcpyAsync(st4, c->dtmp + 8, sizeof(st4), cudaMemcpyDeviceToHost, s));
  TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
  if (!std::isfinite(st4[0]) || !std::isfinite(st4[1]) || !std::isfinite(st4[2]))
    throw std::invalid_argument("topo_gmg_setup: the moduli contain NaN or Inf");
  const double Emax = st4[2];
  const bool re = std::isnan(c->lam_Emax) || std::fabs(Emax - c->lam_Emax) / std::max(std::fabs(c->lam_Emax), 1e-12) > 0.10;
  if (re) {
    L0.lam = lambda_fine(c, s);
    c->lam_Emax = Emax;
  }
  TOPO_CUDA_CHECK(cudaEventRecord(c->ev_ph[1], s));
  // Galerkin operators of every coarse level first (each R.A.P reads the
  // level above), then the coarsest factorisation is queued on s and the
  // per-level Jacobi diagonals, spectral bounds and apply-precision stencil
  // copies run on the side stream meanwhile: the factorisation keeps at most
  // one CTA per SM busy on part of the GPU and only reads the coarsest
  // stencil.
  for (int l = 1; l < c->n_levels; ++l) {
    Level& Lv = c->L[l];
    if (l == 1) level1_assemble(c->L[0].g, Lv.g, c->E64, Lv.mask, Lv.S64, s);
    else rap(c->L[l - 1].g, Lv.g, c->L[l - 1].S64, Lv.mask, Lv.S64, s);
  }
  TOPO_CUDA_CHECK(cudaEventRecord(c->ev_ph[2], s));
  TOPO_CUDA_CHECK(cudaEventRecord(c->ev_ph[3], s));
  TOPO_CUDA_CHECK(cudaEventRecord(c->ev_ph[4], s));
  // the side stream starts from here, beside the factorisation queued next
  TOPO_CUDA_CHECK(cudaEventRecord(c->C.ev_rap, s));
  // coarsest: FP64 band Cholesky + diagonal-block inverses, with the
  // reference's eps*I retry (multigrid_v4.py:778-811)
  bool launched_cur = false;
  if (c->n_levels > 1 && c->C.n > 0) {
    Level& Lc = c->L[c->n_levels - 1];
    const size_t sb = sizeof(double) * 243 * Lc.g.nnodes;
    if (!c->coarse_lag || !c->C.have) {
      coarse_wait_background(c);
      TOPO_CUDA_CHECK(cudaMemcpyAsync(c->C.cur.S64c, Lc.S64, sb, cudaMemcpyDeviceToDevice, s));
      TOPO_CUDA_CHECK(cudaEventRecord(c->ev_ph[3], s));
      slot_launch(c, c->C.cur, s);
      TOPO_CUDA_CHECK(cudaEventRecord(c->ev_ph[4], s));
      launched_cur = true;
    } else {
      // The V-cycle keeps the previous setup's factor; this setup's factor
      // builds on the background stream and replaces it at the next setup.
      if (c->C.bg_pending) {
        TOPO_CUDA_CHECK(cudaEventSynchronize(c->C.bg_done));
        c->C.bg_pending = false;
        slot_finish(c, c->C.nxt, s);
        std::swap(c->C.cur, c->C.nxt);
      }
      if (!c->C.nxt.S64c) alloc_slot(c, c->C.nxt);
      TOPO_CUDA_CHECK(cudaMemcpyAsync(c->C.nxt.S64c, Lc.S64, sb, cudaMemcpyDeviceToDevice, s));
      TOPO_CUDA_CHECK(cudaEventRecord(c->C.ev_copy, s));
      TOPO_CUDA_CHECK(cudaStreamWaitEvent(c->C.bg_stream, c->C.ev_copy, 0));
      slot_launch(c, c->C.nxt, c->C.bg_stream);
      TOPO_CUDA_CHECK(cudaEventRecord(c->C.bg_done, c->C.bg_stream));
      c->C.bg_pending = true;
    }
  }
  {
    cudaStream_t t = c->C.side;
    TOPO_CUDA_CHECK(cudaStreamWaitEvent(t, c->C.ev_rap, 0));
    for (int l = 1; l < c->n_levels - 1; ++l) {
      Level& Lv = c->L[l];
      double* dinv64 = c->vec64 ? (double*)Lv.dinv : (double*)c->C.tmp;
      stencil_dinv(Lv.g, Lv.S64, Lv.mask, dinv64, c->vec64 ? nullptr : (float*)Lv.dinv, t);
      if (re || std::isnan(Lv.lam)) Lv.lam = lambda_coarse(c, l, dinv64, t);
      if (Lv.prec == Prec::F32 || Lv.prec == Prec::BF16)
        stencil_convert(Lv.g.nnodes, Lv.S64, Lv.S32, Lv.prec == Prec::BF16 ? Lv.S16 : nullptr, t);
    }
    TOPO_CUDA_CHECK(cudaEventRecord(c->C.ev_side, t));
    TOPO_CUDA_CHECK(cudaStreamWaitEvent(s, c->C.ev_side, 0));
  }
  if (launched_cur) {
    slot_finish(c, c->C.cur, s);
    c->C.have = true;
  }
  TOPO_CUDA_CHECK(cudaEventRecord(c->ev_ph[5], s));
  TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
  for (int p = 0; p < 5; ++p) {
    float ms = 0.f;
    TOPO_CUDA_CHECK(cudaEventElapsedTime(&ms, c->ev_ph[p], c->ev_ph[p + 1]));
    c->setup_ms[p] = ms;
  }
  c->setup_done = true;
}

// ----------------------------------------------------------------- PCG
void pcg_iteration(topo_ctx* c, cudaStream_t s) {
  Level& L0 = c->L[0];
  const long long n = L0.g.ndof;
  EpiArgs ea{};
  ea.st = c->st;
  ea.red = c->red;
  level0_apply(outer_prec(c), L0.g, c->kp, outer_E(c), L0.mask, c->kAp, Epi::StoreDot, ea, s);
  pcg_xr_update(c->vec64, n, c->kx64, c->kr, c->kp, c->kAp, c->st, c->red, s);
  vcycle_apply(c, c->kr, c->kz, c->st, s);
  pcg_rz(c->vec64, n, c->kr, c->kz, c->st, c->red, false, s);
  pcg_p_update(c->vec64, n, c->kz, c->kp, c->st, false, s);
}

std::vector<double> pcg_graph_key(const topo_ctx* c) {
  std::vector<double> k = {(double)c->cheb_form, c->lam_safety, c->cheb_lower, (double)c->use_tc,
                           (double)c->cycle_gamma,
                           (double)c->fine_degree, (double)c->coarse_degree,
                           (double)reinterpret_cast<uintptr_t>(c->C.cur.f.C), (double)reinterpret_cast<uintptr_t>(c->C.cur.f.W64),
                           (double)reinterpret_cast<uintptr_t>(c->C.y), (double)c->C.n, (double)c->C.cur.f.plan.nt};
  for (const Level& Lv : c->L) {
    k.push_back(std::isnan(Lv.lam) ? -1.0 : Lv.lam);  // NaN (no estimate) would never compare equal
    k.push_back((double)Lv.degree);
  }
  return k;
}

void read_state(topo_ctx* c, cudaStream_t s) {
  TOPO_CUDA_CHECK(cudaMemcpyAsync(c->h_st, c->st, sizeof(KrylovState), cudaMemcpyDeviceToHost, s));
  TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
}

// True residual r64 = b64 - K x64 with the FP64 operator, copied into the
// working-precision residual kr. Returns r.r (FP64).
double true_residual(topo_ctx* c, cudaStream_t s) {
  Level& L0 = c->L[0];
  EpiArgs ea{};
  ea.b = c->kb64;
  level0_apply(Prec::F64, L0.g, c->kx64, c->E64, L0.mask, c->kr64, Epi::Residual, ea, s);
  const double rr = dot_host(true, L0.g.ndof, c->kr64, c->kr64, c->red, c->dtmp, s);
  vcast(L0.g.ndof, c->kr64, true, c->kr, c->vec64, s);
  return rr;
}

__global__ void k_set_state(KrylovState* st, double bb, double tol2) {
  st->bb = bb;
  st->tol2 = tol2;
  st->done = 0;
  st->converged = 0;
  st->iters = 0;
}

// b, x: FP64 full-length vectors (x holds the initial guess).
int do_pcg(topo_ctx* c, const double* b, double* x, double tol, int maxiter, int* out_iters, double* out_relres,
           cudaStream_t s) {
  Level& L0 = c->L[0];
  const long long n = L0.g.ndof;
  const size_t vb = sizeof(double) * n;
  TOPO_CUDA_CHECK(cudaMemcpyAsync(c->kx64, x, vb, cudaMemcpyDeviceToDevice, s));
  TOPO_CUDA_CHECK(cudaMemcpyAsync(c->kb64, b, vb, cudaMemcpyDeviceToDevice, s));
  vmask(true, n, c->kx64, L0.mask, s);
  vmask(true, n, c->kb64, L0.mask, s);
  const double bb = dot_host(true, n, c->kb64, c->kb64, c->red, c->dtmp, s);
  if (!std::isfinite(bb)) throw std::invalid_argument("topo_pcg: the right-hand side contains NaN or Inf");
  const double tol2 = tol * tol * bb;
  double rr = true_residual(c, s);
  if (!std::isfinite(rr)) throw std::invalid_argument("topo_pcg: the initial guess contains NaN or Inf");
  int iters = 0;
  bool converged = rr <= tol2;  // up-front check (solver_v2.py:594-596)
  // one PCG iteration recorded as a CUDA graph on the context stream, reused
  // by later solves while nothing it captured has changed
  const std::vector<double> key = pcg_graph_key(c);
  if (c->pcg_exec && key != c->pcg_key) {
    cudaGraphExecDestroy(c->pcg_exec);
    c->pcg_exec = nullptr;
  }
  cudaGraphExec_t exec = c->pcg_exec;
  long long graph_kernels = c->pcg_exec_kernels;
  int refreshes = 0;
  while (!converged && iters < maxiter && refreshes < 8) {
    k_set_state<<<1, 1, 0, s>>>(c->st, bb, tol2);
    TOPO_LAUNCH_CHECK();
    vcycle_apply(c, c->kr, c->kz, nullptr, s);
    pcg_rz(c->vec64, n, c->kr, c->kz, c->st, c->red, true, s);
    pcg_p_update(c->vec64, n, c->kz, c->kp, c->st, true, s);
    iters += 1;
    if (exec == nullptr) {
      cudaGraph_t graph;
      const long long before = launch_count();
      TOPO_CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      pcg_iteration(c, s);
      TOPO_CUDA_CHECK(cudaStreamEndCapture(s, &graph));
      graph_kernels = launch_count() - before;  // recorded, not launched: counted per replay
      count_launches(-graph_kernels);
      TOPO_CUDA_CHECK(cudaGraphInstantiate(&exec, graph, 0));
      TOPO_CUDA_CHECK(cudaGraphDestroy(graph));
      c->pcg_exec = exec;
      c->pcg_exec_kernels = graph_kernels;
      c->pcg_key = key;
    }
    const int base = iters;  // V-cycles applied before this run of iterations
    int launched = 0;
    const int budget = maxiter - iters;
    bool done = false;
    while (launched < budget) {
      const int chunk = std::min(launched < 8 ? 2 : 4, budget - launched);
      for (int k = 0; k < chunk; ++k) {
        TOPO_CUDA_CHECK(cudaGraphLaunch(exec, s));
        count_launches(graph_kernels);
      }
      launched += chunk;
      read_state(c, s);
      if (c->h_st->done) {
        done = true;
        break;
      }
    }
    read_state(c, s);
    iters = base - 1 + c->h_st->iters;  // st->iters counted the first V-cycle too
    if (!done) break;
    if (c->vec64) {  // FP64: the recursive residual is the reference's test
      converged = true;
      break;
    }
    // FP32 working precision: confirm on the FP64 true residual; if it is not
    // yet below tol, continue from it (reliable update / iterative refinement)
    rr = true_residual(c, s);
    if (rr <= tol2) {
      converged = true;
      break;
    }
    ++refreshes;
  }
  rr = true_residual(c, s);
  if (xs_error_flag(s)) throw std::runtime_error("level-0 K.u: an mbarrier wait timed out");
  if (!std::isfinite(rr)) throw std::runtime_error("topo_pcg: the iteration produced NaN or Inf");
  TOPO_CUDA_CHECK(cudaMemcpyAsync(x, c->kx64, vb, cudaMemcpyDeviceToDevice, s));
  if (out_iters) *out_iters = iters;
  if (out_relres) *out_relres = bb > 0 ? std::sqrt(rr / bb) : 0.0;
  return converged ? 0 : 1;
}

// ---------------------------------------------------------------- FGMRES
// Right-preconditioned restarted flexible GMRES with modified Gram-Schmidt
// and Givens rotations (multigrid_v4.py:325-443). The Hessenberg factor is
// tiny and lives on the host; vectors and dots stay on the device; the
// iterate is FP64 and every restart starts from the FP64 true residual.
// ------------------------------------------------------------ block PCG
// Block preconditioned CG (O'Leary) for nv load cases on one density field,
// with the GMG V-cycle on every column and one multi-vector FP64 K.u per
// iteration; alpha = (P^T Q)^-1 (Z^T R), beta = (Z_old^T R_old)^-1 (Z^T R)
// on the host (nv x nv, Cholesky). A column whose relative residual reaches
// tol leaves the block (its X stays). Returns 0 when every column converged.
static bool small_chol_solve(int k, const double* A, const double* B, double* X) {
  // A (k x k SPD, stride 8), B (k x k, stride 8) -> X = A^-1 B
  double L[8][8] = {};
  for (int j = 0; j < k; ++j) {
    double d = A[j * 8 + j];
    for (int t = 0; t < j; ++t) d -= L[j][t] * L[j][t];
    if (!(d > 0.0) || !std::isfinite(d)) return false;
    L[j][j] = std::sqrt(d);
    for (int i = j + 1; i < k; ++i) {
      double v = A[i * 8 + j];
      for (int t = 0; t < j; ++t) v -= L[i][t] * L[j][t];
      L[i][j] = v / L[j][j];
    }
  }
  for (int col = 0; col < k; ++col) {
    double y[8];
    for (int i = 0; i < k; ++i) {
      double v = B[i * 8 + col];
      for (int t = 0; t < i; ++t) v -= L[i][t] * y[t];
      y[i] = v / L[i][i];
    }
    for (int i = k - 1; i >= 0; --i) {
      double v = y[i];
      for (int t = i + 1; t < k; ++t) v -= L[t][i] * X[t * 8 + col];
      X[i * 8 + col] = v / L[i][i];
    }
  }
  return true;
}

int do_block_pcg(topo_ctx* c, const double* B, double* X, int nv, double tol, int maxiter, int* out_iters,
                 double* out_relres, cudaStream_t s) {
  Level& L0 = c->L[0];
  const long long n = L0.g.ndof;
  if (c->blk_nv != nv) {
    c->blk = c->alloc<double>(5LL * nv * n);
    if (!c->blk_part) {
      c->blk_part = c->alloc<double>((long long)block_gram_partials());
      c->blk_G = c->alloc<double>(64);
      TOPO_CUDA_CHECK(cudaMallocHost(&c->blk_Gh, 64 * sizeof(double)));
    }
    c->blk_nv = nv;
  }
  double *R0 = c->blk, *Z0 = R0 + (long long)nv * n, *P0 = Z0 + (long long)nv * n, *Q0 = P0 + (long long)nv * n,
         *N0 = Q0 + (long long)nv * n;
  auto col = [&](double* base, int j) { return base + (long long)j * n; };
  auto gram = [&](double* const* A, int na, double* const* Bm, int nb, double* Gout) {
    block_gram(n, (const double* const*)A, na, (const double* const*)Bm, nb, c->blk_part, c->blk_G, s);
    TOPO_CUDA_CHECK(cudaMemcpyAsync(c->blk_Gh, c->blk_G, 64 * sizeof(double), cudaMemcpyDeviceToHost, s));
    TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
    std::memcpy(Gout, c->blk_Gh, 64 * sizeof(double));
  };
  auto precond = [&](const double* r, double* z) {
    if (c->vec64) {
      vcycle_apply(c, r, z, nullptr, s);
    } else {
      vcast(n, r, true, c->kr, false, s);
      vcycle_apply(c, c->kr, c->kz, nullptr, s);
      vcast(n, c->kz, false, z, true, s);
    }
  };
  std::vector<int> act;
  double* Xc[8];
  double* Rc[8];
  double* Zc[8];
  double* Pc[8];
  double* Qc[8];
  double* Nc[8];
  const double* Bc[8];
  for (int j = 0; j < nv; ++j) {
    Xc[j] = X + (long long)j * n;
    Bc[j] = B + (long long)j * n;
    Rc[j] = col(R0, j);
    Zc[j] = col(Z0, j);
    Pc[j] = col(P0, j);
    Qc[j] = col(Q0, j);
    Nc[j] = col(N0, j);
  }
  // masked right-hand sides and their norms (Z used as scratch)
  for (int j = 0; j < nv; ++j) {
    TOPO_CUDA_CHECK(cudaMemcpyAsync(Zc[j], Bc[j], sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    vmask(true, n, Zc[j], L0.mask, s);
  }
  double G[64], H[64], A8[64], Bm8[64];
  gram(Zc, nv, Zc, nv, G);
  double bnorm[8];
  for (int j = 0; j < nv; ++j) bnorm[j] = std::sqrt(std::max(G[j * 8 + j], 0.0));
  // R = mask(B) - A X
  level0_apply_block(L0.g, (const double* const*)Xc, c->E64, L0.mask, Qc, nv, s);
  {
    double I8[64] = {};
    for (int j = 0; j < 8; ++j) I8[j * 8 + j] = 1.0;
    block_combine(n, (const double* const*)Qc, nv, (const double* const*)Zc, Rc, nv, I8, -1.0, s);
  }
  gram(Rc, nv, Rc, nv, G);
  for (int j = 0; j < nv; ++j) {
    const double rel = bnorm[j] > 0 ? std::sqrt(std::max(G[j * 8 + j], 0.0)) / bnorm[j] : 0.0;
    out_relres[j] = rel;
    if (rel > tol) act.push_back(j);
  }
  int it = 0;
  auto pick = [&](double* const* all, double** out) {
    for (size_t a = 0; a < act.size(); ++a) out[a] = all[act[a]];
  };
  double *aR[8], *aZ[8], *aP[8], *aQ[8], *aN[8], *aX[8];
  double rz[64];
  if (!act.empty()) {
    pick(Rc, aR);
    pick(Zc, aZ);
    pick(Pc, aP);
    const int k = (int)act.size();
    for (int a = 0; a < k; ++a) {
      precond(aR[a], aZ[a]);
      TOPO_CUDA_CHECK(cudaMemcpyAsync(aP[a], aZ[a], sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    }
    gram(aZ, k, aR, k, rz);
    it = 1;
  }
  while (!act.empty() && it <= maxiter) {
    const int k = (int)act.size();
    pick(Rc, aR);
    pick(Zc, aZ);
    pick(Pc, aP);
    pick(Qc, aQ);
    pick(Nc, aN);
    pick(Xc, aX);
    level0_apply_block(L0.g, (const double* const*)aP, c->E64, L0.mask, aQ, k, s);
    gram(aP, k, aQ, k, G);  // P^T Q
    if (!small_chol_solve(k, G, rz, A8)) throw std::runtime_error("block PCG: P^T K P lost definiteness");
    block_combine(n, (const double* const*)aP, k, (const double* const*)aX, aX, k, A8, 1.0, s);
    block_combine(n, (const double* const*)aQ, k, (const double* const*)aR, aR, k, A8, -1.0, s);
    gram(aR, k, aR, k, G);
    std::vector<int> keep;
    for (int a = 0; a < k; ++a) {
      const int j = act[a];
      const double rel = std::sqrt(std::max(G[a * 8 + a], 0.0)) / bnorm[j];
      out_relres[j] = rel;
      if (rel > tol) keep.push_back(a);
    }
    if (keep.empty()) {
      act.clear();
      break;
    }
    if (it == maxiter) break;
    // deflate: restrict the old Z^T R to the surviving columns
    const int k2 = (int)keep.size();
    double rz_old[64] = {};
    for (int a = 0; a < k2; ++a)
      for (int b2 = 0; b2 < k2; ++b2) rz_old[a * 8 + b2] = rz[keep[a] * 8 + keep[b2]];
    std::vector<int> act2;
    for (int a : keep) act2.push_back(act[a]);
    act = act2;
    pick(Rc, aR);
    pick(Zc, aZ);
    pick(Pc, aP);
    pick(Nc, aN);
    for (int a = 0; a < k2; ++a) precond(aR[a], aZ[a]);
    gram(aZ, k2, aR, k2, H);  // Z^T R
    // P's surviving columns
    double* Pk[8];
    for (int a = 0; a < k2; ++a) Pk[a] = aP[a];
    if (!small_chol_solve(k2, rz_old, H, Bm8)) throw std::runtime_error("block PCG: Z^T R lost definiteness");
    block_combine(n, (const double* const*)Pk, k2, (const double* const*)aZ, aN, k2, Bm8, 1.0, s);
    // the new directions live in N: swap the column roles P <-> N
    for (int a = 0; a < k2; ++a) std::swap(Pc[act[a]], Nc[act[a]]);
    std::memcpy(rz, H, sizeof(rz));
    ++it;
  }
  *out_iters = it;
  return act.empty() ? 0 : 1;
}

int do_fgmres(topo_ctx* c, const double* b, double* x, double tol, int maxiter, int restart, int* out_iters,
              double* out_relres, cudaStream_t s) {
  Level& L0 = c->L[0];
  const long long n = L0.g.ndof;
  const bool f64 = c->vec64;
  const size_t vb = sizeof(double) * n;
  while ((int)c->fg_V.size() < restart + 1) c->fg_V.push_back(c->valloc(n));
  while ((int)c->fg_Z.size() < restart) c->fg_Z.push_back(c->valloc(n));
  TOPO_CUDA_CHECK(cudaMemcpyAsync(c->kx64, x, vb, cudaMemcpyDeviceToDevice, s));
  TOPO_CUDA_CHECK(cudaMemcpyAsync(c->kb64, b, vb, cudaMemcpyDeviceToDevice, s));
  vmask(true, n, c->kx64, L0.mask, s);
  vmask(true, n, c->kb64, L0.mask, s);
  const double bn = std::sqrt(dot_host(true, n, c->kb64, c->kb64, c->red, c->dtmp, s));
  int total = 0;
  bool converged = bn <= 1e-30;
  std::vector<double> H((restart + 1) * restart), cs(restart), sn(restart), g(restart + 1);
  auto Hij = [&](int i, int j) -> double& { return H[i * restart + j]; };
  while (!converged && total < maxiter) {
    const double beta = std::sqrt(true_residual(c, s));
    if (beta / bn <= tol) {
      converged = true;
      break;
    }
    axpby(f64, n, 1.0 / beta, c->kr, 0.0, c->fg_V[0], s);
    std::fill(H.begin(), H.end(), 0.0);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int jf = 0;
    const int inner = std::min(restart, maxiter - total);
    for (int j = 0; j < inner; ++j) {
      vcycle_apply(c, c->fg_V[j], c->fg_Z[j], nullptr, s);
      EpiArgs ea{};
      level0_apply(outer_prec(c), L0.g, c->fg_Z[j], outer_E(c), L0.mask, c->kt, Epi::Store, ea, s);
      for (int i = 0; i <= j; ++i) {
        Hij(i, j) = dot_host(f64, n, c->fg_V[i], c->kt, c->red, c->dtmp, s);
        axpby(f64, n, -Hij(i, j), c->fg_V[i], 1.0, c->kt, s);
      }
      const double hn = std::sqrt(dot_host(f64, n, c->kt, c->kt, c->red, c->dtmp, s));
      Hij(j + 1, j) = hn;
      if (hn > 1e-14) axpby(f64, n, 1.0 / hn, c->kt, 0.0, c->fg_V[j + 1], s);
      for (int i = 0; i < j; ++i) {
        const double t = cs[i] * Hij(i, j) + sn[i] * Hij(i + 1, j);
        Hij(i + 1, j) = -sn[i] * Hij(i, j) + cs[i] * Hij(i + 1, j);
        Hij(i, j) = t;
      }
      const double den = std::sqrt(Hij(j, j) * Hij(j, j) + Hij(j + 1, j) * Hij(j + 1, j));
      if (den < 1e-300) {
        cs[j] = 1.0;
        sn[j] = 0.0;
      } else {
        cs[j] = Hij(j, j) / den;
        sn[j] = Hij(j + 1, j) / den;
      }
      Hij(j, j) = cs[j] * Hij(j, j) + sn[j] * Hij(j + 1, j);
      Hij(j + 1, j) = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      ++total;
      jf = j + 1;
      if (std::fabs(g[j + 1]) / bn <= tol || hn <= 1e-14) {
        converged = true;
        break;
      }
    }
    // back substitution on the upper-triangular factor (with the reference's
    // fallback for a singular diagonal)
    std::vector<double> y(jf, 0.0);
    for (int i = jf - 1; i >= 0; --i) {
      double v = g[i];
      for (int k = i + 1; k < jf; ++k) v -= Hij(i, k) * y[k];
      y[i] = (Hij(i, i) != 0.0) ? v / Hij(i, i) : 0.0;
    }
    for (int i = 0; i < jf; ++i) axpy_to64(f64, n, y[i], c->fg_Z[i], c->kx64, s);
  }
  const double rr = true_residual(c, s);
  TOPO_CUDA_CHECK(cudaMemcpyAsync(x, c->kx64, vb, cudaMemcpyDeviceToDevice, s));
  if (out_iters) *out_iters = total;
  if (out_relres) *out_relres = bn > 0 ? std::sqrt(rr) / bn : 0.0;
  return converged ? 0 : 1;
}

}  // namespace

// ======================================================================
extern "C" {

// The element stiffness lives in constant memory (folded into the K.u
// instructions as operands) and in the tensor-core B tile, one copy per
// device shared by every context on it. The first live context of a device
// uploads it; later contexts must use the same KE to 1e-12 relative (a
// different one is refused, since it would silently change the operator of
// the others; one equal up to rounding uses the uploaded copy) and do not
// write it again while kernels of other contexts may be reading it.
namespace {
struct DeviceKE {
  std::vector<double> ke;
  int live = 0;
};
std::mutex g_ke_mu;
std::vector<DeviceKE> g_ke;
}  // namespace

static void register_ke(topo_ctx* c, const double* KE) {
  std::lock_guard<std::mutex> lk(g_ke_mu);
  if ((int)g_ke.size() <= c->device) g_ke.resize(c->device + 1);
  DeviceKE& d = g_ke[c->device];
  if (d.live > 0) {
    // the same stiffness up to rounding (one KE built by another code path
    // differs in the last bits) shares the uploaded copy
    double amax = 0.0, dmax = 0.0;
    for (int i = 0; i < 576; ++i) {
      amax = std::max(amax, std::fabs(d.ke[i]));
      dmax = std::max(dmax, std::fabs(d.ke[i] - KE[i]));
    }
    if (!(dmax <= 1e-12 * amax))
      throw std::invalid_argument(
          "topo_ctx_create: another live context on this device uses a different element stiffness KE "
          "(KE is held in constant memory shared by all contexts of a device)");
  } else {
    set_ke(KE);
    cc_set_ke(KE);
    set_ke_block(KE);
    std::vector<double> Q(8 * 576);
    host_galerkin_q(KE, Q.data());
    set_galerkin_q(Q.data());
    xs_prepare(KE);
    d.ke.assign(KE, KE + 576);
  }
  d.live += 1;
  c->ke_registered = true;
}

static void release_ke(topo_ctx* c) {
  if (!c->ke_registered) return;
  std::lock_guard<std::mutex> lk(g_ke_mu);
  if (c->device < (int)g_ke.size() && g_ke[c->device].live > 0) g_ke[c->device].live -= 1;
  c->ke_registered = false;
}

int topo_version(void) { return 100; }

int topo_ctx_create(int nelx, int nely, int nelz, int n_levels, int mode, int fine_degree, int coarse_degree,
                    double cheb_lower, int dense_max, const double* KE_host, topo_ctx** out) {
  topo_ctx* c = nullptr;
  try {
    if (!out || !KE_host) throw std::invalid_argument("topo_ctx_create: null pointer");
    if (nelx < 1 || nely < 1 || nelz < 1) throw std::invalid_argument("topo_ctx_create: grid dims must be >= 1");
    if (n_levels < 1 || n_levels > 12) throw std::invalid_argument("topo_ctx_create: n_levels must be in [1, 12]");
    if (mode < TOPO_MODE_FP64 || mode > TOPO_MODE_MIXED) throw std::invalid_argument("topo_ctx_create: bad mode");
    if (fine_degree < 1 || fine_degree > 15 || coarse_degree < 1 || coarse_degree > 15)
      throw std::invalid_argument("topo_ctx_create: Chebyshev degree must be in [1, 15]");
    c = new topo_ctx();
    TOPO_CUDA_CHECK(cudaGetDevice(&c->device));
    c->mode = mode;
    c->vec64 = (mode == TOPO_MODE_FP64);
    c->n_levels = n_levels;
    c->fine_degree = fine_degree;
    c->coarse_degree = coarse_degree;
    c->cheb_lower = cheb_lower;
    c->dense_max = dense_max;
    register_ke(c, KE_host);
    const char* no_tc = std::getenv("TOPO_B200_NO_TC");
    c->use_tc = !(no_tc && no_tc[0] == '1');
    TOPO_CUDA_CHECK(cudaStreamCreateWithFlags(&c->cs, cudaStreamNonBlocking));
    TOPO_CUDA_CHECK(cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming));
    TOPO_CUDA_CHECK(cudaEventCreateWithFlags(&c->ev_out, cudaEventDisableTiming));
    for (auto& e : c->ev_ph) TOPO_CUDA_CHECK(cudaEventCreate(&e));
    TOPO_CUDA_CHECK(cudaStreamCreateWithFlags(&c->C.bg_stream, cudaStreamNonBlocking));
    TOPO_CUDA_CHECK(cudaEventCreateWithFlags(&c->C.ev_copy, cudaEventDisableTiming));
    TOPO_CUDA_CHECK(cudaEventCreateWithFlags(&c->C.bg_done, cudaEventDisableTiming));
    TOPO_CUDA_CHECK(cudaStreamCreateWithFlags(&c->C.side, cudaStreamNonBlocking));
    TOPO_CUDA_CHECK(cudaEventCreateWithFlags(&c->C.ev_rap, cudaEventDisableTiming));
    TOPO_CUDA_CHECK(cudaEventCreateWithFlags(&c->C.ev_side, cudaEventDisableTiming));
    int nx = nelx, ny = nely, nz = nelz;
    for (int l = 0; l < n_levels; ++l) {
      Level Lv;
      Lv.g = make_grid(nx, ny, nz);
      if (c->vec64) Lv.prec = Prec::F64;
      else if (mode == TOPO_MODE_FP32) Lv.prec = Prec::F32;
      else Lv.prec = Prec::BF16;
      Lv.degree = (l == 0) ? fine_degree : coarse_degree;
      c->L.push_back(Lv);
      nx = std::max(1, nx / 2);
      ny = std::max(1, ny / 2);
      nz = std::max(1, nz / 2);
    }
    for (int l = 0; l < n_levels; ++l) {
      Level& Lv = c->L[l];
      const long long nd = Lv.g.ndof;
      Lv.mask = c->alloc<uint8_t>(nd + 16);  // the tensor-core K.u reads aligned 4-byte mask words
      Lv.x = c->valloc(nd);
      Lv.r = c->valloc(nd);
      Lv.d = c->valloc(nd);
      Lv.d2 = c->valloc(nd);
      Lv.e = c->valloc(nd);
      Lv.b = c->valloc(nd);
      Lv.dinv = c->valloc(nd);
      if (l >= 1) {
        Lv.S64 = c->alloc<double>(243LL * Lv.g.nnodes);
        if (l < n_levels - 1) {
          if (Lv.prec != Prec::F64) Lv.S32 = c->alloc<float>(27LL * 12 * Lv.g.nnodes);
          if (Lv.prec == Prec::BF16) Lv.S16 = c->alloc<__nv_bfloat16>(27LL * 12 * Lv.g.nnodes);
        }
      }
    }
    const Grid& g0 = c->L[0].g;
    c->E64 = c->alloc<double>(g0.nelem);
    c->E32 = c->alloc<float>(g0.nelem);
    c->nmask0 = c->alloc<uint8_t>(g0.nnodes + 16);
    c->diag0 = c->alloc<double>(g0.ndof);
    c->kr = c->valloc(g0.ndof);
    c->kz = c->valloc(g0.ndof);
    c->kp = c->valloc(g0.ndof);
    c->kAp = c->valloc(g0.ndof);
    c->kx64 = c->alloc<double>(g0.ndof);
    c->kb64 = c->alloc<double>(g0.ndof);
    c->kr64 = c->alloc<double>(g0.ndof);
    c->kt = c->valloc(g0.ndof);
    c->Fvec = c->alloc<double>(g0.ndof);
    c->st = c->alloc<KrylovState>(1);
    TOPO_CUDA_CHECK(cudaMallocHost((void**)&c->h_st, sizeof(KrylovState)));
    c->red.partials = c->alloc<double>(1 << 18);
    c->red.ticket = c->alloc<unsigned int>(1);
    c->dtmp = c->alloc<double>(64);
    c->oc_state = c->alloc<double>(16);
    c->Hs = c->alloc<double>(g0.nelem);
    c->fstencil.off = c->alloc<int>(3 * kMaxFilterOff);
    c->fstencil.w = c->alloc<double>(kMaxFilterOff);
    // largest coarse-level vector for FP64 scratch (used when vectors are FP32)
    long long maxc = 1;
    for (int l = 1; l < n_levels; ++l) maxc = std::max(maxc, c->L[l].g.ndof);
    c->C.tmp = c->alloc<double>(maxc);
    c->C.scrA = c->alloc<double>(maxc);
    c->C.scrB = c->alloc<double>(maxc);
    c->C.scrC = c->alloc<double>(maxc);
    *out = c;
    return 0;
  } catch (const std::exception& e) {
    set_global_error(e.what());
    if (c) topo_ctx_destroy(c);
    if (out) *out = nullptr;
    return -1;
  }
}

int topo_ctx_destroy(topo_ctx* c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  if (c->cs) cudaStreamSynchronize(c->cs);
  release_ke(c);
  for (void* p : c->allocs) cudaFree(p);
  if (c->h_st) cudaFreeHost(c->h_st);
  if (c->blk_Gh) cudaFreeHost(c->blk_Gh);
  if (c->pcg_exec) cudaGraphExecDestroy(c->pcg_exec);
  if (c->C.bg_pending && c->C.bg_done) cudaEventSynchronize(c->C.bg_done);
  if (c->C.ev_copy) cudaEventDestroy(c->C.ev_copy);
  if (c->C.bg_done) cudaEventDestroy(c->C.bg_done);
  if (c->C.bg_stream) cudaStreamDestroy(c->C.bg_stream);
  if (c->C.side) cudaStreamSynchronize(c->C.side);
  if (c->C.ev_rap) cudaEventDestroy(c->C.ev_rap);
  if (c->C.ev_side) cudaEventDestroy(c->C.ev_side);
  if (c->C.side) cudaStreamDestroy(c->C.side);
  if (c->ev_in) cudaEventDestroy(c->ev_in);
  if (c->ev_out) cudaEventDestroy(c->ev_out);
  for (auto& e : c->ev_ph)
    if (e) cudaEventDestroy(e);
  if (c->cs) cudaStreamDestroy(c->cs);
  delete c;
  return 0;
}

int topo_set_smoother(topo_ctx* c, int form, double lam_safety) {
  try {
    if (!c) throw std::invalid_argument("topo_set_smoother: null context");
    if (form != 0 && form != 1) throw std::invalid_argument("topo_set_smoother: form must be 0 or 1");
    if (!(lam_safety >= 1.0 && lam_safety <= 4.0)) throw std::invalid_argument("topo_set_smoother: lam_safety in [1, 4]");
    c->cheb_form = form;
    c->lam_safety = lam_safety;
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_last_error(topo_ctx* c, char* buf, int len) {
  const std::string m = c ? c->err : global_error();
  if (buf && len > 0) {
    const int k = std::min<int>(len - 1, (int)m.size());
    memcpy(buf, m.data(), k);
    buf[k] = 0;
  }
  return (int)m.size();
}

int topo_set_problem(topo_ctx* c, const uint8_t* free_mask, const double* F, void* stream) {
  try {
    if (!c || !free_mask || !F) throw std::invalid_argument("topo_set_problem: null pointer");
    StreamGuard sg(c, stream);
    cudaStream_t s = c->cs;
    Level& L0 = c->L[0];
    TOPO_CUDA_CHECK(cudaMemcpyAsync(L0.mask, free_mask, L0.g.ndof, cudaMemcpyDeviceToDevice, s));
    TOPO_CUDA_CHECK(cudaMemcpyAsync(c->Fvec, F, sizeof(double) * L0.g.ndof, cudaMemcpyDeviceToDevice, s));
    for (int l = 1; l < c->n_levels; ++l) inject_mask(c->L[l - 1].g, c->L[l].g, c->L[l - 1].mask, c->L[l].mask, s);
    k_node_mask<<<gblocks(L0.g.nnodes), 256, 0, s>>>(L0.g.nnodes, L0.mask, c->nmask0);
    TOPO_LAUNCH_CHECK();
    // coarsest compact numbering and band
    if (c->n_levels > 1) {
      Level& Lc = c->L[c->n_levels - 1];
      std::vector<uint8_t> m(Lc.g.ndof);
      TOPO_CUDA_CHECK(cudaMemcpyAsync(m.data(), Lc.mask, Lc.g.ndof, cudaMemcpyDeviceToHost, s));
      TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
      std::vector<int> idx(Lc.g.ndof, -1), fl;
      for (long long i = 0; i < Lc.g.ndof; ++i)
        if (m[i]) {
          idx[i] = (int)fl.size();
          fl.push_back((int)i);
        }
      const int n = (int)fl.size();
      if (n > c->dense_max)
        throw std::runtime_error("coarsest level has " + std::to_string(n) +
                                 " free DoFs, above dense_max; use more levels or raise dense_max");
      int band = 0;
      const Grid& g = Lc.g;
      for (long long I = 0; I < g.nnodes; ++I) {
        const int iz = (int)(I % g.NZ), iy = (int)((I / g.NZ) % g.NY), ix = (int)(I / ((long long)g.NZ * g.NY));
        for (int k = 0; k < 27; ++k) {
          const int jx = ix + k / 9 - 1, jy = iy + (k / 3) % 3 - 1, jz = iz + k % 3 - 1;
          if (jx < 0 || jx >= g.NX || jy < 0 || jy >= g.NY || jz < 0 || jz >= g.NZ) continue;
          const long long J = ((long long)jx * g.NY + jy) * g.NZ + jz;
          for (int cc = 0; cc < 3; ++cc)
            for (int dd = 0; dd < 3; ++dd) {
              const int a = idx[3 * I + cc], b = idx[3 * J + dd];
              if (a >= 0 && b >= 0) band = std::max(band, std::abs(a - b));
            }
        }
      }
      coarse_wait_background(c);
      c->C.have = false;
      CoarsestPlan plan = coarsest_plan(Lc.g, fl);
      if (c->C.n != n || c->C.band != band || c->C.cur.S64c == nullptr) {
        c->C.n = n;
        c->C.band = band;
        c->C.plan = plan;
        c->C.dof_index = c->alloc<int>(Lc.g.ndof);
        c->C.free_list = c->alloc<int>(std::max(n, 1));
        c->C.y = c->alloc<double>(2 * (size_t)std::max(n, 1));
        c->C.cur = FactorSlot();
        alloc_slot(c, c->C.cur);
        if (c->C.nxt.S64c) {
          c->C.nxt = FactorSlot();
          alloc_slot(c, c->C.nxt);
        }
      }
      TOPO_CUDA_CHECK(cudaMemcpyAsync(c->C.dof_index, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice, s));
      TOPO_CUDA_CHECK(cudaMemcpyAsync(c->C.free_list, fl.data(), sizeof(int) * std::max<size_t>(fl.size(), 1),
                                      cudaMemcpyHostToDevice, s));
      TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
    }
    c->problem_set = true;
    c->setup_done = false;
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_modulus(topo_ctx* c, const double* rho, double penal, double E0, double Emin, double* E, void* stream) {
  try {
    if (!c || !rho || !E) throw std::invalid_argument("topo_modulus: null pointer");
    StreamGuard sg(c, stream);
    modulus(c->L[0].g.nelem, rho, penal, E0, Emin, E, nullptr, c->cs);
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_matvec(topo_ctx* c, int dtype, const void* u, void* y, const void* E, void* stream) {
  try {
    if (!c || !u || !y || !E) throw std::invalid_argument("topo_matvec: null pointer");
    if (!c->problem_set) throw std::runtime_error("topo_matvec: call topo_set_problem first");
    StreamGuard sg(c, stream);
    if (xs_error_flag(c->cs, false))
      throw std::runtime_error("level-0 K.u: an mbarrier wait of an earlier launch timed out");
    Level& L0 = c->L[0];
    EpiArgs ea{};
    if (dtype == TOPO_F64) level0_apply(Prec::F64, L0.g, u, E, L0.mask, y, Epi::Store, ea, c->cs);
    else if (dtype == TOPO_F32) level0_apply(Prec::F32, L0.g, u, E, L0.mask, y, Epi::Store, ea, c->cs);
    else if (dtype == TOPO_BF16) {
      if (c->use_tc && level0_xs_supported(L0.g)) {
        level0_apply_xs(true, L0.g, u, E, c->nmask0, y, Epi::Store, ea, c->cs);
      } else {
        level0_apply_bf16_input(L0.g, u, E, L0.mask, y, c->cs);
      }
    }
    else throw std::invalid_argument("topo_matvec: bad dtype");
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_level0_apply(topo_ctx* c, int u_dtype, int epi, const void* u, const void* E, void* y, const void* b, void* r,
                      void* x, void* d_out, const void* dinv, double s, double c1, double c2, double ax,
                      void* stream) {
  try {
    if (!c || !u || !E) throw std::invalid_argument("topo_level0_apply: null pointer");
    if (!c->problem_set) throw std::runtime_error("topo_level0_apply: call topo_set_problem first");
    Epi ep;
    switch (epi) {
      case TOPO_EPI_STORE: ep = Epi::Store; if (!y) throw std::invalid_argument("topo_level0_apply: y is null"); break;
      case TOPO_EPI_RESIDUAL:
        ep = Epi::Residual;
        if (!y || !b) throw std::invalid_argument("topo_level0_apply: residual needs y and b");
        break;
      case TOPO_EPI_RUPD: ep = Epi::RUpd; if (!r) throw std::invalid_argument("topo_level0_apply: r is null"); break;
      case TOPO_EPI_CHEB:
        ep = Epi::ChebR;
        if (!r || !x || !d_out || !dinv) throw std::invalid_argument("topo_level0_apply: Chebyshev step needs r, x, d_out, dinv");
        if (d_out == u) throw std::invalid_argument("topo_level0_apply: d_out must differ from u");
        break;
      default: throw std::invalid_argument("topo_level0_apply: bad epilogue");
    }
    StreamGuard sg(c, stream);
    if (xs_error_flag(c->cs, false))
      throw std::runtime_error("level-0 K.u: an mbarrier wait of an earlier launch timed out");
    Level& L0 = c->L[0];
    EpiArgs ea{};
    ea.b = b;
    ea.r = r;
    ea.x = x;
    ea.d_out = d_out;
    ea.dinv = dinv;
    ea.s = s;
    ea.c1 = c1;
    ea.c2 = c2;
    ea.ax = ax;
    if (u_dtype == TOPO_F64) level0_apply(Prec::F64, L0.g, u, E, L0.mask, y, ep, ea, c->cs);
    else if (u_dtype == TOPO_F32) level0_apply(Prec::F32, L0.g, u, E, L0.mask, y, ep, ea, c->cs);
    else if (u_dtype == TOPO_BF16 || u_dtype == TOPO_BF16_F32IN) {
      const bool u16 = u_dtype == TOPO_BF16;
      if (c->use_tc && level0_xs_supported(L0.g)) {
        level0_apply_xs(u16, L0.g, u, E, c->nmask0, y, ep, ea, c->cs);
      } else if (!u16) {
        level0_apply(Prec::BF16, L0.g, u, E, L0.mask, y, ep, ea, c->cs);
      } else {
        if (ep != Epi::Store) throw std::runtime_error("topo_level0_apply: BF16-stored u on CUDA cores supports Store only");
        level0_apply_bf16_input(L0.g, u, E, L0.mask, y, c->cs);
      }
    } else {
      throw std::invalid_argument("topo_level0_apply: bad dtype");
    }
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_wait_status(topo_ctx* c, void* stream) {
  try {
    if (!c) throw std::invalid_argument("topo_wait_status: null context");
    StreamGuard sg(c, stream);
    if (xs_error_flag(c->cs, true)) throw std::runtime_error("level-0 K.u: an mbarrier wait timed out");
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_debug_bounds(int* tripped) {
  try {
    if (!tripped) throw std::invalid_argument("topo_debug_bounds: null pointer");
    const int t = bounds_flag_level0() | bounds_flag_xs() | bounds_flag_cc() | bounds_flag_coarse() |
                  bounds_flag_coarsest() | bounds_flag_design();
    *tripped = t ? 1 : 0;
#ifdef TOPO_DEBUG_BOUNDS
    return 0;
#else
    return 1;
#endif
  } catch (const std::exception& e) {
    return fail(nullptr, e);
  }
}

int topo_debug_tc_wait(int skip_first_arrival, int poll_limit) {
  xs_debug(skip_first_arrival, poll_limit);
  return 0;
}

int topo_diag(topo_ctx* c, const double* E, double* diag, void* stream) {
  try {
    if (!c || !E || !diag) throw std::invalid_argument("topo_diag: null pointer");
    if (!c->problem_set) throw std::runtime_error("topo_diag: call topo_set_problem first");
    StreamGuard sg(c, stream);
    level0_diag(c->L[0].g, E, c->L[0].mask, diag, c->cs);
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_gmg_setup(topo_ctx* c, const double* E, void* stream) {
  try {
    if (!c || !E) throw std::invalid_argument("topo_gmg_setup: null pointer");
    if (!c->problem_set) throw std::runtime_error("topo_gmg_setup: call topo_set_problem first");
    StreamGuard sg(c, stream);
    do_setup(c, E, c->cs);
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_gmg_apply(topo_ctx* c, const void* r, void* z, void* stream) {
  try {
    if (!c || !r || !z) throw std::invalid_argument("topo_gmg_apply: null pointer");
    if (!c->setup_done) throw std::runtime_error("topo_gmg_apply: call topo_gmg_setup first");
    StreamGuard sg(c, stream);
    if (xs_error_flag(c->cs, false))
      throw std::runtime_error("level-0 K.u: an mbarrier wait of an earlier launch timed out");
    vcycle_apply(c, r, z, nullptr, c->cs);
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_pcg(topo_ctx* c, const void* b, void* x, double tol, int maxiter, int* out_iters, double* out_relres,
             void* stream) {
  try {
    if (!c || !b || !x) throw std::invalid_argument("topo_pcg: null pointer");
    if (!c->setup_done) throw std::runtime_error("topo_pcg: call topo_gmg_setup first");
    if (maxiter < 1) throw std::invalid_argument("topo_pcg: maxiter must be >= 1");
    StreamGuard sg(c, stream);
    return do_pcg(c, (const double*)b, (double*)x, tol, maxiter, out_iters, out_relres, c->cs);
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_fgmres(topo_ctx* c, const void* b, void* x, double tol, int maxiter, int restart, int* out_iters,
                double* out_relres, void* stream) {
  try {
    if (!c || !b || !x) throw std::invalid_argument("topo_fgmres: null pointer");
    if (!c->setup_done) throw std::runtime_error("topo_fgmres: call topo_gmg_setup first");
    if (maxiter < 1 || restart < 1) throw std::invalid_argument("topo_fgmres: maxiter and restart must be >= 1");
    StreamGuard sg(c, stream);
    return do_fgmres(c, (const double*)b, (double*)x, tol, maxiter, restart, out_iters, out_relres, c->cs);
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_set_coarse_lag(topo_ctx* c, int on) {
  try {
    if (!c) throw std::invalid_argument("topo_set_coarse_lag: null context");
    c->coarse_lag = on != 0;
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_set_cycle(topo_ctx* c, int gamma) {
  try {
    if (!c) throw std::invalid_argument("topo_set_cycle: null context");
    if (gamma != 1 && gamma != 2) throw std::invalid_argument("topo_set_cycle: gamma must be 1 (V) or 2 (W)");
    c->cycle_gamma = gamma;
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_set_tc(topo_ctx* c, int on) {
  try {
    if (!c) throw std::invalid_argument("topo_set_tc: null context");
    c->use_tc = on != 0;
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_block_pcg(topo_ctx* c, const double* B, double* X, int nrhs, double tol, int maxiter, int* out_iters,
                   double* out_relres, void* stream) {
  try {
    if (!c || !B || !X || !out_iters || !out_relres) throw std::invalid_argument("topo_block_pcg: null pointer");
    if (!c->setup_done) throw std::runtime_error("topo_block_pcg: call topo_gmg_setup first");
    if (nrhs < 1 || nrhs > 8) throw std::invalid_argument("topo_block_pcg: nrhs must be 1..8");
    if (maxiter < 1) throw std::invalid_argument("topo_block_pcg: maxiter must be >= 1");
    StreamGuard sg(c, stream);
    return do_block_pcg(c, B, X, nrhs, tol, maxiter, out_iters, out_relres, c->cs);
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_sensitivity(topo_ctx* c, const void* u, int u_dtype, const double* rho, double penal, double E0,
                     double Emin, double* dc, void* stream) {
  try {
    if (!c || !u || !rho || !dc) throw std::invalid_argument("topo_sensitivity: null pointer");
    if (u_dtype != TOPO_F64 && u_dtype != TOPO_F32) throw std::invalid_argument("topo_sensitivity: bad dtype");
    StreamGuard sg(c, stream);
    sensitivity(c->L[0].g, u, nullptr, u_dtype == TOPO_F32, rho, penal, E0, Emin, dc, c->cs);
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_sensitivity_adjoint(topo_ctx* c, const void* u, const void* lam, int dtype, const double* rho,
                             double penal, double E0, double Emin, double* dc, void* stream) {
  try {
    if (!c || !u || !lam || !rho || !dc) throw std::invalid_argument("topo_sensitivity_adjoint: null pointer");
    if (dtype != TOPO_F64 && dtype != TOPO_F32) throw std::invalid_argument("topo_sensitivity_adjoint: bad dtype");
    StreamGuard sg(c, stream);
    sensitivity(c->L[0].g, u, lam, dtype == TOPO_F32, rho, penal, E0, Emin, dc, c->cs);
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_dot(topo_ctx* c, int dtype, const void* a, const void* b, long long n, double* out_host, void* stream) {
  try {
    if (!c || !a || !b || !out_host) throw std::invalid_argument("topo_dot: null pointer");
    if (dtype != TOPO_F64 && dtype != TOPO_F32) throw std::invalid_argument("topo_dot: bad dtype");
    StreamGuard sg(c, stream);
    *out_host = dot_host(dtype == TOPO_F64, n, a, b, c->red, c->dtmp, c->cs);
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_filter(topo_ctx* c, double rmin, const double* in, double* out, int transpose, void* stream) {
  try {
    if (!c || !in || !out) throw std::invalid_argument("topo_filter: null pointer");
    if (!(rmin > 0.0)) throw std::invalid_argument("topo_filter: rmin must be > 0");
    if (in == out) throw std::invalid_argument("topo_filter: in and out must differ");
    StreamGuard sg(c, stream);
    filter_apply(c->fstencil, c->L[0].g, rmin, in, out, transpose != 0, c->Hs, c->cs);
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_oc(topo_ctx* c, const double* rho, const double* dc, double volfrac, double move, double rho_min,
            double* out, int* out_evals, void* stream) {
  try {
    if (!c || !rho || !dc || !out) throw std::invalid_argument("topo_oc: null pointer");
    StreamGuard sg(c, stream);
    const int ev = oc_update(c->L[0].g.nelem, rho, dc, volfrac, move, rho_min, out, c->red, c->oc_state, c->cs);
    if (out_evals) *out_evals = ev;
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_oc_filtered(topo_ctx* c, const double* rho, const double* dc, const double* dv, const double* colsum,
                     double volfrac, double move, double rho_min, double* out, int* out_evals, void* stream) {
  try {
    if (!c || !rho || !dc || !dv || !colsum || !out) throw std::invalid_argument("topo_oc_filtered: null pointer");
    StreamGuard sg(c, stream);
    const int ev = oc_update_filtered(c->L[0].g.nelem, rho, dc, dv, colsum, volfrac, move, rho_min, out, c->red,
                                      c->oc_state, c->cs);
    if (out_evals) *out_evals = ev;
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_heaviside(topo_ctx* c, const double* rho_f, double beta, double eta, double* phys, double* dh,
                   void* stream) {
  try {
    if (!c || !rho_f || (!phys && !dh)) throw std::invalid_argument("topo_heaviside: null pointer");
    if (phys == rho_f || dh == rho_f) throw std::invalid_argument("topo_heaviside: outputs must not alias rho_f");
    StreamGuard sg(c, stream);
    heaviside_apply(c->L[0].g.nelem, rho_f, beta, eta, phys, dh, c->cs);
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_oc_projected(topo_ctx* c, double rmin, const double* rho, const double* dc, const double* dv, double beta,
                      double eta, double volfrac, double move, double rho_min, double* out, int* out_evals,
                      void* stream) {
  try {
    if (!c || !rho || !dc || !dv || !out) throw std::invalid_argument("topo_oc_projected: null pointer");
    if (!(rmin > 0.0)) throw std::invalid_argument("topo_oc_projected: rmin must be > 0");
    if (out == rho || out == dc || out == dv)
      throw std::invalid_argument("topo_oc_projected: out must not alias rho, dc or dv");
    StreamGuard sg(c, stream);
    const int ev = oc_update_projected(c->fstencil, c->L[0].g, rmin, rho, dc, dv, beta, eta, volfrac, move, rho_min, out, c->Hs,
                                       c->red, c->oc_state, c->cs);
    if (out_evals) *out_evals = ev;
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_field_stats(topo_ctx* c, const double* x, long long n, double* out_host, void* stream) {
  try {
    if (!c || !x || !out_host) throw std::invalid_argument("topo_field_stats: null pointer");
    StreamGuard sg(c, stream);
    field_stats(n, x, c->dtmp, c->red, c->cs);
    TOPO_CUDA_CHECK(cudaMemcpyAsync(out_host, c->dtmp, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->cs));
    TOPO_CUDA_CHECK(cudaStreamSynchronize(c->cs));
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_gmg_info(topo_ctx* c, long long* n_free, double* lambda_max, int* coarse_kind) {
  try {
    if (!c) throw std::invalid_argument("topo_gmg_info: null context");
    for (int l = 0; l < c->n_levels; ++l) {
      if (n_free) {
        std::vector<uint8_t> m(c->L[l].g.ndof);
        TOPO_CUDA_CHECK(cudaMemcpy(m.data(), c->L[l].mask, m.size(), cudaMemcpyDeviceToHost));
        long long k = 0;
        for (uint8_t v : m) k += v;
        n_free[l] = k;
      }
      if (lambda_max) lambda_max[l] = c->L[l].lam;
    }
    if (coarse_kind) *coarse_kind = c->C.cur.f.kind;
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_setup_phases(topo_ctx* c, double* ms) {
  try {
    if (!c || !ms) throw std::invalid_argument("topo_setup_phases: null pointer");
    for (int p = 0; p < 5; ++p) ms[p] = c->setup_ms[p];
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

int topo_gmg_level_operator(topo_ctx* c, int level, double* S_out, void* stream) {
  try {
    if (!c || !S_out) throw std::invalid_argument("topo_gmg_level_operator: null pointer");
    if (level < 1 || level >= c->n_levels) throw std::invalid_argument("topo_gmg_level_operator: bad level");
    if (!c->setup_done) throw std::runtime_error("topo_gmg_level_operator: call topo_gmg_setup first");
    StreamGuard sg(c, stream);
    const Level& Lv = c->L[level];
    TOPO_CUDA_CHECK(cudaMemcpyAsync(S_out, Lv.S64, sizeof(double) * 243 * Lv.g.nnodes, cudaMemcpyDeviceToDevice,
                                    c->cs));
    return 0;
  } catch (const std::exception& e) {
    return fail(c, e);
  }
}

long long topo_workspace_bytes(topo_ctx* c) { return c ? c->bytes : 0; }

long long topo_launch_count(void) { return launch_count(); }

}  // extern "C"
