// noalloc.cu - the bisection OC update without any device allocation.
//
// Some callers cannot let a library call cudaMalloc. One example is a host
// application whose device memory is owned by its own pool: a framework's
// caching allocator, or a Go/JVM runtime handing out pool pointers. A
// library allocating behind such a pool fragments it and breaks its
// accounting. Another is a latency-bound optimisation loop: cudaMalloc and
// cudaFree can synchronise the whole device. topo_oc_noalloc serves those
// callers. The caller passes the inputs and the output, and the only working
// memory is the file-scope array below, which every GPU that loads this
// library holds until process exit.
//
// The update itself is the one of topo_oc (src/topogpu/solver.py:94-117):
// lambda doubling from 1 while the candidate's mean volume exceeds volfrac,
// then up to 80 bisections stopping at |mean - volfrac| < 1e-8; the result is
// the last candidate evaluated. Element blocks here are fixed-size (2048 per
// CTA, one partial sum each), which is what bounds the problem size.
#include "internal.cuh"
#include "reduce.cuh"
#include "../../include/topo_b200.h"

#include <cmath>
#include <mutex>
#include <string>

namespace topo {
namespace noalloc {

constexpr int kThreads = 256;
constexpr int kPerThread = 8;
constexpr int kPerBlock = kThreads * kPerThread;                  // 2048 elements per CTA
constexpr int kMaxBlocks = 4096;                                  // one partial sum per CTA
constexpr long long kMaxElems = (long long)kMaxBlocks * kPerBlock; // 8,388,608 elements
constexpr int kStateOff = kMaxBlocks;                             // 16 slots of bisection state
constexpr int kTicketOff = kMaxBlocks + 16;                       // grid-reduction ticket
constexpr int kSlots = kMaxBlocks + 32;                           // 4128 doubles = 33,024 bytes

// The scratch of every topo_oc_noalloc call on this device: block partials,
// bisection state and the reduction ticket. Shared by all calls; it keeps the
// last call's contents, and k_init clears what must start at zero.
static __device__ __align__(256) double g_oc_scratch[kSlots];

enum Slot { LO = 0, HI, EVAL, MID, MEAN, PHASE, NBIS, DONE, EVALS };

__device__ __forceinline__ double candidate(double rho, double dc, double lam, double move, double rho_min) {
  const double dcs = fmin(dc, -1.0e-12);
  const double t = fmax(-dcs / fmax(lam, 1.0e-40), 0.0);
  const double v = rho * sqrt(t);
  return fmin(fmax(v, fmax(rho - move, rho_min)), fmin(rho + move, 1.0));
}

__global__ void k_init(double* scr) {
  double* st = scr + kStateOff;
  for (int i = 0; i < 16; ++i) st[i] = 0.0;
  st[HI] = 1.0;
  st[EVAL] = 1.0;
  *reinterpret_cast<unsigned int*>(scr + kTicketOff) = 0u;
}

__global__ void __launch_bounds__(kThreads) k_pass(long long n, const double* __restrict__ rho,
                                                  const double* __restrict__ dc, double volfrac, double move,
                                                  double rho_min, double* scr) {
  double* st = scr + kStateOff;
  if (st[DONE] != 0.0) return;
  const double lam = st[EVAL];
  double v[1] = {0.0};
  const long long base = (long long)blockIdx.x * kPerBlock + threadIdx.x;
#pragma unroll
  for (int k = 0; k < kPerThread; ++k) {
    const long long i = base + (long long)k * kThreads;
    if (i < n) v[0] += candidate(rho[i], dc[i], lam, move, rho_min);
  }
  RedWork red{scr, reinterpret_cast<unsigned int*>(scr + kTicketOff)};
  double tot[1];
  if (grid_sum<1>(v, red, tot) && threadIdx.x == 0) {
    const double mean = tot[0] / (double)n;
    st[MEAN] = mean;
    st[EVALS] += 1.0;
    if (st[PHASE] == 0.0) {
      if (mean > volfrac && st[HI] < 1.0e40) {
        st[LO] = st[HI];
        st[HI] = st[HI] * 2.0;
        st[EVAL] = st[HI];
      } else {
        st[PHASE] = 1.0;
        st[EVAL] = 0.5 * (st[LO] + st[HI]);
      }
    } else {
      const double mid = st[EVAL];
      if (mean > volfrac) st[LO] = mid;
      else st[HI] = mid;
      st[MID] = mid;
      st[NBIS] += 1.0;
      if (fabs(mean - volfrac) < 1.0e-8 || st[NBIS] >= 80.0) st[DONE] = 1.0;
      else st[EVAL] = 0.5 * (st[LO] + st[HI]);
    }
  }
}

__global__ void k_final(long long n, const double* __restrict__ rho, const double* __restrict__ dc, double move,
                        double rho_min, const double* scr, double* __restrict__ out) {
  const double lam = scr[kStateOff + MID];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = candidate(rho[i], dc[i], lam, move, rho_min);
}

// Device address of g_oc_scratch per device, looked up once per device with
// that device current (the symbol's host-side name is not a device address).
// The table is guarded by a mutex: two host threads making their first call
// on the same device at once would otherwise race on it.
constexpr int kMaxDevices = 64;
static double* g_scratch_ptr[kMaxDevices] = {};
static std::mutex g_scratch_mu;

static double* scratch_for_current_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) throw std::runtime_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("topo_oc_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (g_scratch_ptr[dev] == nullptr) {
    double* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_oc_scratch);
    if (e != cudaSuccess || p == nullptr)
      throw std::runtime_error(std::string("cudaGetSymbolAddress(g_oc_scratch): ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  return g_scratch_ptr[dev];
}

}  // namespace noalloc
}  // namespace topo

extern "C" int topo_oc_noalloc(const double* rho, const double* dc, long long n, double volfrac, double move,
                               double rho_min, double* out, int* out_evals, void* stream) {
  using namespace topo::noalloc;
  try {
    if (n < 1 || n > kMaxElems)
      throw std::invalid_argument("topo_oc_noalloc: n = " + std::to_string(n) + " is outside [1, " +
                                  std::to_string(kMaxElems) + "], the size its static scratch serves");
    if (!rho || !dc || !out) throw std::invalid_argument("topo_oc_noalloc: null pointer");
    if (out == rho || out == dc) throw std::invalid_argument("topo_oc_noalloc: out must not alias rho or dc");
    cudaStream_t s = (cudaStream_t)stream;
    double* scr = scratch_for_current_device();
    k_init<<<1, 1, 0, s>>>(scr);
    TOPO_LAUNCH_CHECK();
    const unsigned nb = (unsigned)((n + kPerBlock - 1) / kPerBlock);
    double h[16];
    int launched = 0;
    bool done = false;
    // at most 134 doublings (1 -> 2^133 > 1e40) and 80 bisections
    while (launched < 134 + 80 + 1) {
      const int chunk = launched < 16 ? 8 : 16;
      for (int k = 0; k < chunk; ++k, ++launched) {
        k_pass<<<nb, kThreads, 0, s>>>(n, rho, dc, volfrac, move, rho_min, scr);
        TOPO_LAUNCH_CHECK();
      }
      TOPO_CUDA_CHECK(cudaMemcpyAsync(h, scr + kStateOff, sizeof(h), cudaMemcpyDeviceToHost, s));
      TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
      if (h[DONE] != 0.0) {
        done = true;
        break;
      }
    }
    if (!done) throw std::runtime_error("topo_oc_noalloc: bisection did not terminate");
    k_final<<<(unsigned)std::min<long long>(4096, (n + 255) / 256), 256, 0, s>>>(n, rho, dc, move, rho_min, scr, out);
    TOPO_LAUNCH_CHECK();
    if (out_evals) *out_evals = (int)h[EVALS];
    return 0;
  } catch (const std::exception& e) {
    topo::set_global_error(e.what());
    return -1;
  }
}
