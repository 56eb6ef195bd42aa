// design.cu - density filter, OC updates and field statistics on the device.
//
// The OC bisection keeps its whole state (lambda bracket, phase, counters) in
// device memory: each pass evaluates one candidate's volume with a
// deterministic grid reduction and the last block advances the bisection, so
// the host only checks a "done" flag every few passes instead of reading a
// mean per step (the reference runs the loop in NumPy on the host,
// src/topogpu/solver.py:94-117).
#include "internal.cuh"
#include "reduce.cuh"

#include <cmath>
#include <functional>
#include <stdexcept>
#include <vector>

namespace topo {

// Offsets and weights of the linear-hat filter: every element at centre
// distance d <= rmin - 1e-10 with weight rmin - d, plus the element itself with
// weight rmin (pub_simp_solver.py:215-243; kd-tree query_pairs radius).
static void set_filter(FilterStencil& fs, double rmin, cudaStream_t s) {
  if (fs.rmin == rmin) return;
  const int R = (int)std::floor(rmin);
  std::vector<int> off;
  std::vector<double> w;
  for (int dx = -R; dx <= R; ++dx)
    for (int dy = -R; dy <= R; ++dy)
      for (int dz = -R; dz <= R; ++dz) {
        const double d = std::sqrt((double)(dx * dx + dy * dy + dz * dz));
        if (dx == 0 && dy == 0 && dz == 0) {
          off.insert(off.end(), {0, 0, 0});
          w.push_back(rmin);
        } else if (d <= rmin - 1e-10) {
          off.insert(off.end(), {dx, dy, dz});
          w.push_back(rmin - d);
        }
      }
  if ((int)w.size() > kMaxFilterOff) throw std::runtime_error("filter radius too large (rmin must be < 6)");
  TOPO_CUDA_CHECK(cudaMemcpyAsync(fs.off, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice, s));
  TOPO_CUDA_CHECK(cudaMemcpyAsync(fs.w, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice, s));
  TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
  fs.rmin = rmin;
  fs.n = (int)w.size();
}

__device__ __forceinline__ double row_weight_sum(const Grid& g, int ex, int ey, int ez, int noff,
                                                 const int* __restrict__ fo, const double* __restrict__ fw) {
  double hs = 0.0;
  for (int k = 0; k < noff; ++k) {
    const int x = ex + fo[3 * k], y = ey + fo[3 * k + 1], z = ez + fo[3 * k + 2];
    if (x >= 0 && x < g.nx && y >= 0 && y < g.ny && z >= 0 && z < g.nz) hs += fw[k];
  }
  return hs;
}

__global__ void k_filter_rowsum(Grid g, int noff, const int* __restrict__ fo, const double* __restrict__ fw,
                                double* __restrict__ Hs) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= g.nelem) return;
  const int ez = e % g.nz, ey = (e / g.nz) % g.ny, ex = e / ((long long)g.nz * g.ny);
  Hs[e] = row_weight_sum(g, ex, ey, ez, noff, fo, fw);
}

// out_i = sum_j (w_ij / Hs_i) in_j          (transpose = 0)
// out_j = sum_i (w_ij / Hs_i) in_i          (transpose = 1)
__global__ void k_filter(Grid g, int noff, const int* __restrict__ fo, const double* __restrict__ fw,
                         const double* __restrict__ in, double* __restrict__ out, const double* __restrict__ Hs,
                         int transpose) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= g.nelem) return;
  const int ez = e % g.nz, ey = (e / g.nz) % g.ny, ex = e / ((long long)g.nz * g.ny);
  double acc = 0.0;
  if (!transpose) {
    const double hs = Hs[e];
    for (int k = 0; k < noff; ++k) {
      const int x = ex + fo[3 * k], y = ey + fo[3 * k + 1], z = ez + fo[3 * k + 2];
      if (x < 0 || x >= g.nx || y < 0 || y >= g.ny || z < 0 || z >= g.nz) continue;
      const long long j = ((long long)x * g.ny + y) * g.nz + z;
      if (!topo_in_range(j, g.nelem)) continue;
      acc += (fw[k] / hs) * in[j];
    }
  } else {
    for (int k = 0; k < noff; ++k) {
      const int x = ex + fo[3 * k], y = ey + fo[3 * k + 1], z = ez + fo[3 * k + 2];
      if (x < 0 || x >= g.nx || y < 0 || y >= g.ny || z < 0 || z >= g.nz) continue;
      const long long i = ((long long)x * g.ny + y) * g.nz + z;
      if (!topo_in_range(i, g.nelem)) continue;
      acc += (fw[k] / Hs[i]) * in[i];
    }
  }
  out[e] = acc;
}

void filter_apply(FilterStencil& fs, const Grid& g, double rmin, const double* in, double* out, bool transpose,
                  double* Hs_work, cudaStream_t s) {
  set_filter(fs, rmin, s);
  const int bs = 256;
  const unsigned nb = (unsigned)((g.nelem + bs - 1) / bs);
  k_filter_rowsum<<<nb, bs, 0, s>>>(g, fs.n, fs.off, fs.w, Hs_work);
  TOPO_LAUNCH_CHECK();
  k_filter<<<nb, bs, 0, s>>>(g, fs.n, fs.off, fs.w, in, out, Hs_work, transpose ? 1 : 0);
  TOPO_LAUNCH_CHECK();
}

// ------------------------------------------------------------------- OC
// Device state of the bisection. Slots of a double[16] array:
enum OcSlot { OC_LO = 0, OC_HI, OC_EVAL, OC_MID, OC_MEAN, OC_PHASE, OC_NBIS, OC_DONE, OC_EVALS };

__device__ __forceinline__ double oc_candidate(double rho, double dc, double lam, double move, double rho_min) {
  const double dcs = fmin(dc, -1.0e-12);
  double t = -dcs / fmax(lam, 1.0e-40);
  t = fmax(t, 0.0);
  const double v = rho * sqrt(t);
  const double lo = fmax(rho - move, rho_min);
  const double hi = fmin(rho + move, 1.0);
  return fmin(fmax(v, lo), hi);
}

__global__ void k_oc_pass(long long n, const double* __restrict__ rho, const double* __restrict__ dc,
                          double volfrac, double move, double rho_min, double* st, RedWork red) {
  if (st[OC_DONE] != 0.0) return;
  const double lam = st[OC_EVAL];
  double v[1] = {0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[0] += oc_candidate(rho[i], dc[i], lam, move, rho_min);
  double tot[1];
  if (grid_sum<1>(v, red, tot) && threadIdx.x == 0) {
    const double mean = tot[0] / (double)n;
    st[OC_MEAN] = mean;
    st[OC_EVALS] += 1.0;
    if (st[OC_PHASE] == 0.0) {
      // lambda_hi doubling while the candidate volume is too large
      if (mean > volfrac && st[OC_HI] < 1.0e40) {
        st[OC_LO] = st[OC_HI];
        st[OC_HI] = st[OC_HI] * 2.0;
        st[OC_EVAL] = st[OC_HI];
      } else {
        st[OC_PHASE] = 1.0;
        st[OC_EVAL] = 0.5 * (st[OC_LO] + st[OC_HI]);
      }
    } else {
      const double mid = st[OC_EVAL];
      if (mean > volfrac) st[OC_LO] = mid;
      else st[OC_HI] = mid;
      st[OC_MID] = mid;
      st[OC_NBIS] += 1.0;
      if (fabs(mean - volfrac) < 1.0e-8 || st[OC_NBIS] >= 80.0) st[OC_DONE] = 1.0;
      else st[OC_EVAL] = 0.5 * (st[OC_LO] + st[OC_HI]);
    }
  }
}

__global__ void k_oc_final(long long n, const double* __restrict__ rho, const double* __restrict__ dc, double move,
                           double rho_min, const double* st, double* __restrict__ out) {
  const double lam = st[OC_MID];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = oc_candidate(rho[i], dc[i], lam, move, rho_min);
}

__global__ void k_oc_init(double* st) {
  for (int i = 0; i < 16; ++i) st[i] = 0.0;
  st[OC_LO] = 0.0;
  st[OC_HI] = 1.0;
  st[OC_EVAL] = 1.0;
}

static int run_until_done(const std::function<void()>& pass, const double* st, int max_passes, cudaStream_t s) {
  double h[16];
  int launched = 0;
  while (launched < max_passes) {
    const int chunk = launched < 16 ? 8 : 16;
    for (int k = 0; k < chunk && launched < max_passes; ++k, ++launched) pass();
    TOPO_CUDA_CHECK(cudaMemcpyAsync(h, st, sizeof(double) * 16, cudaMemcpyDeviceToHost, s));
    TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
    if (h[OC_DONE] != 0.0) return (int)h[OC_EVALS];
  }
  return -1;
}

int oc_update(long long n, const double* rho, const double* dc, double volfrac, double move, double rho_min,
              double* out, RedWork red, double* st, cudaStream_t s) {
  k_oc_init<<<1, 1, 0, s>>>(st);
  TOPO_LAUNCH_CHECK();
  const unsigned nb = (unsigned)std::min<long long>(kRedBlocks, (n + kRedThreads - 1) / kRedThreads);
  auto pass = [&]() {
    k_oc_pass<<<nb, kRedThreads, 0, s>>>(n, rho, dc, volfrac, move, rho_min, st, red);
    TOPO_LAUNCH_CHECK();
  };
  // at most 134 doublings (1 -> 2^133 > 1e40) and 80 bisections
  const int evals = run_until_done(pass, st, 134 + 80 + 1, s);
  if (evals < 0) throw std::runtime_error("OC bisection did not terminate");
  k_oc_final<<<nb, kRedThreads, 0, s>>>(n, rho, dc, move, rho_min, st, out);
  TOPO_LAUNCH_CHECK();
  return evals;
}

// ------------------------------------------------------- filtered-volume OC
enum OcfSlot { OF_L1 = 0, OF_L2, OF_LM, OF_LAST, OF_K, OF_DONE, OF_EVALS };

__device__ __forceinline__ double ocf_candidate(double rho, double dc, double dv, double lm, double move,
                                                double rho_min) {
  const double dcs = fmin(dc, -1e-12);
  const double dvs = fmax(dv, 1e-12);
  double rn = rho * sqrt(-dcs / (lm * dvs));
  rn = fmin(fmax(rn, rho - move), rho + move);
  rn = fmin(fmax(rn, rho_min), 1.0);
  return rn;
}

// Three bisection levels per pass: the 7 midpoints of the next three levels
// of the interval tree [l1, l2] are formed with the operations the
// sequential bisection would use (node q's children 2q+1 = left half, 2q+2 =
// right half, each midpoint 0.5 * (lo + hi) of that node's bounds), their
// volumes summed in one sweep over the elements (each by the same grid
// reduction as a single-candidate pass, so bit-identical), and the walk down
// the tree takes the sequential path: evaluation count, last multiplier and
// bounds are those of one level per pass.
__global__ void k_ocf_pass3(long long n, const double* __restrict__ rho, const double* __restrict__ dc,
                            const double* __restrict__ dv, const double* __restrict__ colsum, double volfrac,
                            double move, double rho_min, double* st, RedWork red) {
  if (st[OF_DONE] != 0.0) return;
  const double l1 = st[OF_L1], l2 = st[OF_L2];
  double c[7];
  c[0] = 0.5 * (l1 + l2);
  c[1] = 0.5 * (l1 + c[0]);
  c[2] = 0.5 * (c[0] + l2);
  c[3] = 0.5 * (l1 + c[1]);
  c[4] = 0.5 * (c[1] + c[0]);
  c[5] = 0.5 * (c[0] + c[2]);
  c[6] = 0.5 * (c[2] + l2);
  double v[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double r = rho[i], d = dc[i], w = dv[i], cs = colsum[i];
#pragma unroll
    for (int q = 0; q < 7; ++q) v[q] += ocf_candidate(r, d, w, c[q], move, rho_min) * cs;
  }
  double tot[7];
  if (grid_sum<7>(v, red, tot) && threadIdx.x == 0) {
    int q = 0;
    for (int level = 0; level < 3; ++level) {
      const double lm = c[q];
      st[OF_EVALS] += 1.0;
      const bool up = tot[q] / (double)n > volfrac;
      if (up) st[OF_L1] = lm;
      else st[OF_L2] = lm;
      st[OF_LAST] = lm;
      st[OF_K] += 1.0;
      if (st[OF_L2] - st[OF_L1] < 1e-9 || st[OF_K] >= 100.0) {
        st[OF_DONE] = 1.0;
        break;
      }
      st[OF_LM] = 0.5 * (st[OF_L1] + st[OF_L2]);
      q = 2 * q + (up ? 2 : 1);
    }
  }
}

__global__ void k_ocf_init(double* st) {
  for (int i = 0; i < 16; ++i) st[i] = 0.0;
  st[OF_L1] = 0.0;
  st[OF_L2] = 1e9;
  st[OF_LM] = 0.5 * (0.0 + 1e9);
}

__global__ void k_ocf_final(long long n, const double* __restrict__ rho, const double* __restrict__ dc,
                            const double* __restrict__ dv, double move, double rho_min, const double* st,
                            double* __restrict__ out) {
  const double lm = st[OF_LAST];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = ocf_candidate(rho[i], dc[i], dv[i], lm, move, rho_min);
}

int oc_update_filtered(long long n, const double* rho, const double* dc, const double* dv, const double* colsum,
                       double volfrac, double move, double rho_min, double* out, RedWork red, double* st,
                       cudaStream_t s) {
  k_ocf_init<<<1, 1, 0, s>>>(st);
  TOPO_LAUNCH_CHECK();
  const unsigned nb = (unsigned)std::min<long long>(kRedBlocks, (n + kRedThreads - 1) / kRedThreads);
  auto pass = [&]() {
    k_ocf_pass3<<<nb, kRedThreads, 0, s>>>(n, rho, dc, dv, colsum, volfrac, move, rho_min, st, red);
    TOPO_LAUNCH_CHECK();
  };
  // three levels per pass: 34 passes cover the 100-level cap
  double h[16];
  int launched = 0;
  while (true) {
    for (int k = 0; k < 8 && launched < 34; ++k, ++launched) pass();
    TOPO_CUDA_CHECK(cudaMemcpyAsync(h, st, sizeof(double) * 16, cudaMemcpyDeviceToHost, s));
    TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
    if (h[OF_DONE] != 0.0) break;
    if (launched >= 34) throw std::runtime_error("filtered OC bisection did not terminate");
  }
  k_ocf_final<<<nb, kRedThreads, 0, s>>>(n, rho, dc, dv, move, rho_min, st, out);
  TOPO_LAUNCH_CHECK();
  return (int)h[OF_EVALS];
}

// ------------------------------------------------- Heaviside projection
// Smoothed Heaviside of run_simp (pub_simp_solver.py:245-253):
//   h(x)  = (tanh(b e) + tanh(b (x - e))) / (tanh(b e) + tanh(b (1 - e)))
//   h'(x) = b (1 - tanh(b (x - e))^2) / (tanh(b e) + tanh(b (1 - e)))
// with the identity (h = x, h' = 1) unless b > 1e-6, the guard every run_simp
// call site applies (pub_simp_solver.py:331,348,366). The two tanh constants
// are computed on the host and passed in the kernel arguments.
struct Projection {
  double beta, eta, tbe, den;
  bool on;
};

static Projection make_projection(double beta, double eta) {
  Projection p{beta, eta, 0.0, 1.0, beta > 1e-6};
  if (p.on) {
    p.tbe = std::tanh(beta * eta);
    p.den = p.tbe + std::tanh(beta * (1.0 - eta));
  }
  return p;
}

__global__ void k_heaviside(long long n, const double* __restrict__ rho_f, Projection p, double* __restrict__ phys,
                            double* __restrict__ dh) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double x = rho_f[i];
    if (!p.on) {
      if (phys) phys[i] = x;
      if (dh) dh[i] = 1.0;
      continue;
    }
    const double t = tanh(p.beta * (x - p.eta));
    if (phys) phys[i] = (p.tbe + t) / p.den;
    if (dh) dh[i] = p.beta * (1.0 - t * t) / p.den;
  }
}

void heaviside_apply(long long n, const double* rho_f, double beta, double eta, double* phys, double* dh,
                     cudaStream_t s) {
  const Projection p = make_projection(beta, eta);
  if (n == 0) return;
  const unsigned nb = (unsigned)std::min<long long>(4 * kRedBlocks, (n + 255) / 256);
  k_heaviside<<<nb, 256, 0, s>>>(n, rho_f, p, phys, dh);
  TOPO_LAUNCH_CHECK();
}

// ------------------------------------------------- projected-volume OC
// run_simp's OC with Heaviside (pub_simp_solver.py:319-340): the volume of a
// candidate is sum_i h((H cand)_i) / n. The projection is nonlinear, so the
// colsum shortcut of the filtered OC does not apply; each bisection pass
// writes the candidate (k_ocp_cand) and then filters it at every element,
// projects and sums in one kernel (k_ocp_vol) whose last block advances the
// bisection exactly as k_ocf_pass does. The candidate buffer is the output
// array: once the bisection stops, k_ocp_cand skips, so the output holds the
// candidate of the last evaluated lambda, which is what the reference returns.
__global__ void k_ocp_cand(long long n, const double* __restrict__ rho, const double* __restrict__ dc,
                           const double* __restrict__ dv, double move, double rho_min, const double* st,
                           double* __restrict__ cand) {
  if (st[OF_DONE] != 0.0) return;
  const double lm = st[OF_LM];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    cand[i] = ocf_candidate(rho[i], dc[i], dv[i], lm, move, rho_min);
}

__global__ void k_ocp_vol(Grid g, int noff, const int* __restrict__ fo, const double* __restrict__ fw,
                          const double* __restrict__ cand, const double* __restrict__ Hs, Projection p,
                          double volfrac, double* st, RedWork red) {
  if (st[OF_DONE] != 0.0) return;
  const double lm = st[OF_LM];
  double v[1] = {0.0};
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < g.nelem;
       e += (long long)gridDim.x * blockDim.x) {
    const int ez = e % g.nz, ey = (e / g.nz) % g.ny, ex = e / ((long long)g.nz * g.ny);
    const double hs = Hs[e];
    double acc = 0.0;
    for (int k = 0; k < noff; ++k) {
      const int x = ex + fo[3 * k], y = ey + fo[3 * k + 1], z = ez + fo[3 * k + 2];
      if (x < 0 || x >= g.nx || y < 0 || y >= g.ny || z < 0 || z >= g.nz) continue;
      acc += (fw[k] / hs) * cand[((long long)x * g.ny + y) * g.nz + z];
    }
    v[0] += p.on ? (p.tbe + tanh(p.beta * (acc - p.eta))) / p.den : acc;
  }
  double tot[1];
  if (grid_sum<1>(v, red, tot) && threadIdx.x == 0) {
    st[OF_EVALS] += 1.0;
    if (tot[0] / (double)g.nelem > volfrac) st[OF_L1] = lm;
    else st[OF_L2] = lm;
    st[OF_LAST] = lm;
    st[OF_K] += 1.0;
    if (st[OF_L2] - st[OF_L1] < 1e-9 || st[OF_K] >= 100.0) st[OF_DONE] = 1.0;
    else st[OF_LM] = 0.5 * (st[OF_L1] + st[OF_L2]);
  }
}

int oc_update_projected(FilterStencil& fs, const Grid& g, double rmin, const double* rho, const double* dc, const double* dv,
                        double beta, double eta, double volfrac, double move, double rho_min, double* out,
                        double* Hs_work, RedWork red, double* st, cudaStream_t s) {
  const long long n = g.nelem;
  set_filter(fs, rmin, s);
  const Projection p = make_projection(beta, eta);
  const unsigned nb = (unsigned)std::min<long long>(kRedBlocks, (n + kRedThreads - 1) / kRedThreads);
  k_filter_rowsum<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(g, fs.n, fs.off, fs.w, Hs_work);
  TOPO_LAUNCH_CHECK();
  k_ocf_init<<<1, 1, 0, s>>>(st);
  TOPO_LAUNCH_CHECK();
  double h[16];
  int launched = 0;
  while (true) {
    for (int k = 0; k < 16 && launched < 100; ++k, ++launched) {
      k_ocp_cand<<<nb, kRedThreads, 0, s>>>(n, rho, dc, dv, move, rho_min, st, out);
      TOPO_LAUNCH_CHECK();
      k_ocp_vol<<<nb, kRedThreads, 0, s>>>(g, fs.n, fs.off, fs.w, out, Hs_work, p, volfrac, st, red);
      TOPO_LAUNCH_CHECK();
    }
    TOPO_CUDA_CHECK(cudaMemcpyAsync(h, st, sizeof(double) * 16, cudaMemcpyDeviceToHost, s));
    TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
    if (h[OF_DONE] != 0.0) break;
    if (launched >= 100) throw std::runtime_error("projected OC bisection did not terminate");
  }
  return (int)h[OF_EVALS];
}

// ------------------------------------------------------------ field stats
__global__ void k_stats(long long n, const double* __restrict__ x, double* out4, RedWork red) {
  double sum = 0.0, gray = 0.0, mn = INFINITY, mx = -INFINITY;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = x[i];
    sum += v;
    gray += v * (1.0 - v);
    mn = fmin(mn, v);
    mx = fmax(mx, v);
  }
  __shared__ double smn[32], smx[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  mn = warp_min(mn);
  mx = warp_max(mx);
  if (lane == 0) {
    smn[wid] = mn;
    smx[wid] = mx;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = blockDim.x >> 5;
    mn = warp_min(threadIdx.x < nw ? smn[threadIdx.x] : INFINITY);
    mx = warp_max(threadIdx.x < nw ? smx[threadIdx.x] : -INFINITY);
  }
  // min/max travel through the sum slots of a separate partial row
  double v[4] = {sum, gray, 0.0, 0.0};
  __shared__ bool s_last;
  block_sum<4>(v);
  const unsigned nb = gridDim.x;
  if (threadIdx.x == 0) {
    red.partials[(size_t)blockIdx.x * 4 + 0] = v[0];
    red.partials[(size_t)blockIdx.x * 4 + 1] = v[1];
    red.partials[(size_t)blockIdx.x * 4 + 2] = mn;
    red.partials[(size_t)blockIdx.x * 4 + 3] = mx;
    __threadfence();
    s_last = (atomicAdd(red.ticket, 1u) == nb - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x == 0) {
    double S = 0.0, G = 0.0, MN = INFINITY, MX = -INFINITY;
    for (unsigned b = 0; b < nb; ++b) {
      S += __ldcg(red.partials + (size_t)b * 4 + 0);
      G += __ldcg(red.partials + (size_t)b * 4 + 1);
      MN = fmin(MN, __ldcg(red.partials + (size_t)b * 4 + 2));
      MX = fmax(MX, __ldcg(red.partials + (size_t)b * 4 + 3));
    }
    out4[0] = S / (double)n;
    out4[1] = MN;
    out4[2] = MX;
    out4[3] = 4.0 * (G / (double)n);
    *red.ticket = 0u;
  }
}

void field_stats(long long n, const double* x, double* out4_dev, RedWork red, cudaStream_t s) {
  const unsigned nb = (unsigned)std::min<long long>(kRedBlocks, (n + kRedThreads - 1) / kRedThreads);
  k_stats<<<nb, kRedThreads, 0, s>>>(n, x, out4_dev, red);
  TOPO_LAUNCH_CHECK();
}

TOPO_BOUNDS_READER(bounds_flag_design)

}  // namespace topo
