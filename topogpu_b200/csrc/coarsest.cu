// coarsest.cu - direct FP64 solve of the coarsest multigrid level.
//
// The coarsest operator (free DoFs only, compact numbering in reference DoF
// order) couples x-planes only to their neighbours, so in plane blocks it is
// block tridiagonal and its Cholesky factor L is block bidiagonal: L_bb lower
// triangular and L_{b,b-1} dense. The setup
//   1. assembles the lower band (|i-j| <= band) into band storage,
//   2. factorises it with one persistent kernel: a right-looking band
//      Cholesky over 32-column panels, one grid barrier per panel (each CTA
//      factors the panel's diagonal block itself, solves the panel rows of
//      its trailing tiles and updates them; the factor goes to a separate
//      band array so no CTA reads a panel row another CTA has overwritten),
//   3. inverts every diagonal plane block, Di_b = L_bb^-1, and forms
//      M_b = Di_b L_{b,b-1} and N_b = Di_b^T L_{b+1,b}^T (FP64 arithmetic,
//      stored in the apply precision).
// The apply z = K^-1 r is then two sweeps over the plane blocks,
//   y_b = Di_b r_b - M_b y_{b-1},   z_b = Di_b^T y_b - N_b z_{b+1},
// run by one thread-block cluster (8 CTAs) with one cluster barrier per
// block: y and z stay in L2, each block step reads the previous block's
// values once into shared memory.
//
// Reference: the coarsest solve of GalerkinMatFreeGMG (src/gpu_fem/
// multigrid_v4.py:774-811, 969-984): dense Cholesky with an eps*I retry when a
// pivot is not positive. The factor here is the same (a band Cholesky creates
// no fill outside the band); only the storage and the apply differ.
#include "internal.cuh"
#include "reduce.cuh"

#include <algorithm>
#include <stdexcept>
#include <vector>

namespace topo {
namespace cst {

constexpr int CNB = 32;  // panel width

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }

// Band storage: row i holds columns i-band .. i at B[i*ldb + (j - i + band)];
// every access checks i - j <= band first (the band can be narrower than a
// 32-wide panel on small coarsest grids).
__device__ __forceinline__ long long bidx(long long i, long long j, int band, long long ldb) {
  return i * ldb + (j - i + band);
}

// --------------------------------------------------------------- assembly
__global__ void k_band_assemble(Grid g, const double* __restrict__ S, const int* __restrict__ dof_index, int band,
                                long long ldb, double* __restrict__ A) {
  const long long I = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (I >= g.nnodes) return;
  const int iz = (int)(I % g.NZ), iy = (int)((I / g.NZ) % g.NY), ix = (int)(I / ((long long)g.NZ * g.NY));
  for (int c = 0; c < 3; ++c) {
    const int row = dof_index[3 * I + c];
    if (row < 0) continue;
    for (int k = 0; k < 27; ++k) {
      const int jx = ix + k / 9 - 1, jy = iy + (k / 3) % 3 - 1, jz = iz + k % 3 - 1;
      if (jx < 0 || jx >= g.NX || jy < 0 || jy >= g.NY || jz < 0 || jz >= g.NZ) continue;
      const long long J = ((long long)jx * g.NY + jy) * g.NZ + jz;
      for (int d = 0; d < 3; ++d) {
        const int col = dof_index[3 * J + d];
        if (col < 0 || col > row || row - col > band) continue;
        A[bidx(row, col, band, ldb)] = S[(long long)(k * 9 + c * 3 + d) * g.nnodes + I];
      }
    }
  }
}

__global__ void k_band_add_diag(int n, int band, long long ldb, double* A, double eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) A[bidx(i, i, band, ldb)] += eps;
}

__global__ void k_band_diag_sum(int n, int band, long long ldb, const double* A, double* out) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += A[bidx(i, i, band, ldb)];
  double a[1] = {v};
  block_sum<1>(a);
  if (threadIdx.x == 0) *out = a[0];
}

// ------------------------------------------------------------ grid barrier
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Sense-counting barrier over all CTAs of a cooperative launch. Thread 0
// reads the generation, arrives, and the last arrival resets the count and
// bumps the generation; the others poll it with a bound (a timeout raises
// err and is reported to every thread of the CTA).
__device__ bool grid_barrier(unsigned* count, unsigned* gen, unsigned nblocks, int* err, int poll) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned g0 = ld_acquire(gen);
    __threadfence();
    if (atomicAdd(count, 1u) == nblocks - 1) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      int it = 0;
      while (ld_acquire(gen) == g0) {
        if (++it > poll) {
          ok = 0;
          atomicExch(err, 1);
          break;
        }
        __nanosleep(40);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ------------------------------------------------------ persistent Cholesky
// Shared memory of one CTA: the panel's diagonal block (factored in place by
// warp 0 into Ld and its reciprocal pivots), and the panel rows of the two
// row tiles of the trailing tile it updates (solved in place).
struct CholSmem {
  double W[CNB][CNB + 1];
  double Ld[CNB][CNB + 1];
  double invd[CNB];
  double Pi[CNB][CNB + 1];
  double Pj[CNB][CNB + 1];
  int bad;
};

__device__ __forceinline__ void tile_of(int t, int& ti, int& tj) {
  ti = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
  while (ti * (ti + 1) / 2 > t) --ti;
  tj = t - ti * (ti + 1) / 2;
}

// Solve rows [r0, r0+32) of the panel (columns k .. k+nb) against the
// factored diagonal block: X Ld^T = A_panel. Rows past `lim` or entries
// outside the band are zero. 32 threads, one row each.
__device__ __forceinline__ void panel_solve(const double* A, int band, long long ldb, int k, int nb, int r0, int lim,
                                            CholSmem& S, double (*P)[CNB + 1]) {
  const int t = threadIdx.x;
  if (t < CNB) {
    const int i = r0 + t;
    double x[CNB];
#pragma unroll
    for (int j = 0; j < CNB; ++j) x[j] = (i < lim && j < nb && i - (k + j) <= band) ? ldcg(A + bidx(i, k + j, band, ldb)) : 0.0;
#pragma unroll
    for (int j = 0; j < CNB; ++j) {
      x[j] *= S.invd[j];
#pragma unroll
      for (int q = j + 1; q < CNB; ++q) x[q] -= x[j] * S.Ld[q][j];
    }
#pragma unroll
    for (int j = 0; j < CNB; ++j) P[t][j] = x[j];
  }
}

__global__ void __launch_bounds__(256) k_band_chol(int n, int band, long long ldb, double* A, double* L, int* flag,
                                                   unsigned* bar_count, unsigned* bar_gen, int* err, int poll) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CholSmem& S = *reinterpret_cast<CholSmem*>(smem_raw);
  const int tid = threadIdx.x;
  for (int k = 0; k < n; k += CNB) {
    const int nb = min(CNB, n - k);
    // 1. the panel's diagonal block, factored by warp 0 (every CTA does the
    //    same arithmetic, so all agree); identity-padded past n
    for (int q = tid; q < CNB * CNB; q += blockDim.x) {
      const int i = q / CNB, j = q % CNB;
      S.W[i][j] = (i < nb && j < nb && j <= i) ? (i - j <= band ? ldcg(A + bidx(k + i, k + j, band, ldb)) : 0.0)
                                               : (i == j ? 1.0 : 0.0);
    }
    __syncthreads();
    if (tid < 32) {
      const int lane = tid;
      double wr[CNB];
#pragma unroll
      for (int t = 0; t < CNB; ++t) wr[t] = S.W[lane][t];
      bool bad = false;
#pragma unroll
      for (int j = 0; j < CNB; ++j) {
        const double d = __shfl_sync(0xffffffffu, wr[j], j);
        const bool ok = d > 0.0 && isfinite(d);
        const double dd = ok ? d : 1.0;
        const double rs = rsqrt(dd);
        const double lj = wr[j];
        if (lane == j) {
          bad |= !ok;
          S.Ld[j][j] = dd * rs;
          S.invd[j] = rs;
        } else {
          S.Ld[lane][j] = lane > j ? lj * rs : 0.0;
        }
        const double w = lj * (rs * rs);
#pragma unroll
        for (int t = j + 1; t < CNB; ++t) {
          const double ct = __shfl_sync(0xffffffffu, wr[j], t);
          if (t <= lane) wr[t] -= ct * w;
        }
      }
      bad = __any_sync(0xffffffffu, bad);
      if (lane == 0) S.bad = bad ? 1 : 0;
    }
    __syncthreads();
    if (blockIdx.x == 0) {
      for (int q = tid; q < CNB * CNB; q += blockDim.x) {
        const int i = q / CNB, j = q % CNB;
        if (i < nb && j <= i && i - j <= band) L[bidx(k + i, k + j, band, ldb)] = S.Ld[i][j];
      }
      if (tid == 0 && S.bad) *flag = 1;
    }
    // 2. trailing tiles of the band window: solve their panel rows, write
    //    the factor rows (owner of the diagonal tile), update
    const int base = k + nb;
    const int lim = min(n, base + band);
    const int nt = (lim - base + CNB - 1) / CNB;
    const int ntiles = lim > base ? nt * (nt + 1) / 2 : 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      int ti, tj;
      tile_of(t, ti, tj);
      const int i0 = base + CNB * ti, j0 = base + CNB * tj;
      if (i0 - (j0 + CNB - 1) > band) continue;  // whole tile outside the band (uniform)
      panel_solve(A, band, ldb, k, nb, i0, lim, S, S.Pi);
      if (tj != ti) {
        __syncthreads();
        if (tid >= 32 && tid < 64) {
          // second row tile by warp 1 (same code path, shifted thread index)
          const int tt = tid - 32;
          const int i = j0 + tt;
          double x[CNB];
#pragma unroll
          for (int j = 0; j < CNB; ++j)
            x[j] = (i < lim && j < nb && i - (k + j) <= band) ? ldcg(A + bidx(i, k + j, band, ldb)) : 0.0;
#pragma unroll
          for (int j = 0; j < CNB; ++j) {
            x[j] *= S.invd[j];
#pragma unroll
            for (int q = j + 1; q < CNB; ++q) x[q] -= x[j] * S.Ld[q][j];
          }
#pragma unroll
          for (int j = 0; j < CNB; ++j) S.Pj[tt][j] = x[j];
        }
      }
      __syncthreads();
      double(*Pj)[CNB + 1] = (tj == ti) ? S.Pi : S.Pj;
      if (tj == ti) {
        // owner of the diagonal tile writes the factor rows of this row tile
        for (int q = tid; q < CNB * CNB; q += blockDim.x) {
          const int r = q / CNB, j = q % CNB;
          const int i = i0 + r;
          if (i < lim && j < nb && i - (k + j) <= band) L[bidx(i, k + j, band, ldb)] = S.Pi[r][j];
        }
      }
      const int r = tid >> 3, c0 = (tid & 7) * 4;
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
      for (int q = 0; q < CNB; ++q) {
        const double li = S.Pi[r][q];
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m] = fma(li, Pj[c0 + m][q], acc[m]);
      }
      const int i = i0 + r;
      if (i < lim) {
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const int j = j0 + c0 + m;
          if (j < lim && j <= i && i - j <= band) A[bidx(i, j, band, ldb)] -= acc[m];
        }
      }
      __syncthreads();
    }
    if (!grid_barrier(bar_count, bar_gen, gridDim.x, err, poll)) return;
  }
}

}  // namespace cst
}  // namespace topo

namespace topo {
namespace cst {

// ------------------------------------------------------ block inverses
// Di_b = L_bb^-1 for every plane block: CTA (s, b) owns the 32 columns
// [32s, 32s+32) of block b and walks its 32-row sub-blocks I >= s:
//   R   = E - L[rows of I, cols 32s .. 32I) W[32s .. 32I, strip]
//   W_I = L_II^-1 R  (forward substitution, one thread per column)
// The strip's rows of W stay in shared memory (<= kMaxBlock rows).
constexpr int kMaxBlock = 512;  // largest plane block (3 (NY+1)(NZ+1) free DoFs)
struct InvSmem {
  double Wst[kMaxBlock][CNB + 1];
  double Lc[CNB][CNB + 1];
  double R[CNB][CNB + 1];
};

__global__ void __launch_bounds__(256) k_block_inverse(const int* __restrict__ boff, int band, long long ldb,
                                                       const double* __restrict__ L, const long long* __restrict__ dioff,
                                                       double* __restrict__ DI) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  InvSmem& S = *reinterpret_cast<InvSmem*>(smem_raw);
  const int b = blockIdx.y, s = blockIdx.x;
  const int o = boff[b], m = boff[b + 1] - o;
  const int c0 = CNB * s;
  if (c0 >= m) return;
  const int tid = threadIdx.x;
  const int nsub = (m + CNB - 1) / CNB;
  const int r = tid >> 3, cq = (tid & 7) * 4;
  for (int I = s; I < nsub; ++I) {
    const int i0 = CNB * I;
    // R = E - L[i0.., c0..i0) W[c0..i0, :]
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k0 = c0; k0 < i0; k0 += CNB) {
      __syncthreads();
      for (int q = tid; q < CNB * CNB; q += blockDim.x) {
        const int rr = q / CNB, kk = q % CNB;
        const long long gi = o + i0 + rr, gk = o + k0 + kk;
        S.Lc[rr][kk] = (i0 + rr < m && k0 + kk < i0 && gi - gk <= band) ? L[bidx(gi, gk, band, ldb)] : 0.0;
      }
      __syncthreads();
#pragma unroll 8
      for (int kk = 0; kk < CNB; ++kk) {
        const double l = S.Lc[r][kk];
        if (k0 + kk < i0) {
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[q] = fma(l, S.Wst[k0 + kk][cq + q], acc[q]);
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) S.R[r][cq + q] = ((i0 + r == c0 + cq + q) ? 1.0 : 0.0) - acc[q];
    // the diagonal sub-block L_II
    for (int q = tid; q < CNB * CNB; q += blockDim.x) {
      const int rr = q / CNB, kk = q % CNB;
      S.Lc[rr][kk] = (i0 + rr < m && i0 + kk < m && kk <= rr)
                         ? (rr - kk <= band ? L[bidx(o + i0 + rr, o + i0 + kk, band, ldb)] : 0.0)
                         : (rr == kk ? 1.0 : 0.0);
    }
    __syncthreads();
    if (tid < CNB) {
      const int c = tid;
      for (int rr = 0; rr < CNB; ++rr) {
        double v = S.R[rr][c];
        for (int q = 0; q < rr; ++q) v -= S.Lc[rr][q] * S.Wst[i0 + q][c];
        S.Wst[i0 + rr][c] = (i0 + rr < m) ? v / S.Lc[rr][rr] : 0.0;
      }
    }
    __syncthreads();
  }
  // write the strip: rows c0.. m-1 (entries above the diagonal are zero)
  double* D = DI + dioff[b];
  for (int q = tid; q < (m - c0) * CNB; q += blockDim.x) {
    const int rr = c0 + q / CNB, c = c0 + q % CNB;
    if (c < m) D[(long long)rr * m + c] = (c <= rr) ? S.Wst[rr][c - c0] : 0.0;
  }
  // and the zero upper part of these columns
  for (int q = tid; q < c0 * CNB; q += blockDim.x) {
    const int rr = q / CNB, c = c0 + q % CNB;
    if (c < m) D[(long long)rr * m + c] = 0.0;
  }
}

// L_{b,b-1} (dense, rows of block b x columns of block b-1) from band storage.
__global__ void k_extract_sub(const int* __restrict__ boff, int band, long long ldb, const double* __restrict__ L,
                              const long long* __restrict__ soff, double* __restrict__ Ls) {
  const int b = blockIdx.y + 1;
  const int o = boff[b], m = boff[b + 1] - o, op = boff[b - 1], mp = o - op;
  double* D = Ls + soff[b];
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (long long)m * mp;
       q += (long long)gridDim.x * blockDim.x) {
    const long long i = o + q / mp, j = op + q % mp;
    D[q] = (i - j <= band) ? L[bidx(i, j, band, ldb)] : 0.0;
  }
}

// Batched C_b = op(A_b) op(B_b) in FP64 with strided operands:
// A(i,k) = A[i*sai + k*sak], B(k,j) = B[k*sbk + j*sbj]; C row-major (m x n).
struct GemmJob {
  const double* A;
  const double* B;
  void* C;
  int m, n, kdim;
  int sai, sak, sbk, sbj;
};

template <typename TO>
__global__ void __launch_bounds__(256) k_gemm_batched(const GemmJob* __restrict__ jobs) {
  const GemmJob jb = jobs[blockIdx.z];
  const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
  if (i0 >= jb.m || j0 >= jb.n) return;
  __shared__ double As[32][33], Bs[32][33];
  const int tid = threadIdx.x, r = tid >> 3, cq = (tid & 7) * 4;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int k0 = 0; k0 < jb.kdim; k0 += 32) {
    __syncthreads();
    for (int q = tid; q < 1024; q += 256) {
      const int a = q / 32, bq = q % 32;
      As[a][bq] = (i0 + a < jb.m && k0 + bq < jb.kdim) ? jb.A[(long long)(i0 + a) * jb.sai + (long long)(k0 + bq) * jb.sak] : 0.0;
      Bs[a][bq] = (k0 + a < jb.kdim && j0 + bq < jb.n) ? jb.B[(long long)(k0 + a) * jb.sbk + (long long)(j0 + bq) * jb.sbj] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < 32; ++kk) {
      const double a = As[r][kk];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fma(a, Bs[kk][cq + q], acc[q]);
    }
  }
  TO* C = reinterpret_cast<TO*>(jb.C);
  if (i0 + r < jb.m) {
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (j0 + cq + q < jb.n) C[(long long)(i0 + r) * jb.n + j0 + cq + q] = (TO)acc[q];
  }
}

template <typename TO>
__global__ void k_convert_copy(long long n, const double* __restrict__ src, TO* __restrict__ dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (TO)src[i];
}

// --------------------------------------------------------------- apply
// One cluster of CL CTAs; block offsets, sizes and matrix offsets in a small
// device table. y (forward) and z (backward) live in global memory (L2),
// read with .cg loads after each cluster barrier (release/acquire at
// cluster scope orders the writes of every CTA of the cluster).
constexpr int CL = 8;
constexpr int AT = 256;

struct ApplyPlan {
  int nb;
  long long nfull;       // length of the full vectors rhs and x
  const int* boff;       // nb+1
  const int* link;       // link[b] = 1: block b couples to b-1
  const long long* dioff;  // Di_b, m_b x m_b
  const long long* moff;   // M_b, m_b x m_{b-1}
  const long long* noff;   // N_b, m_b x m_{b+1}
};

__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

template <typename T, typename TX>
__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(AT)
    k_coarsest_apply(int n, ApplyPlan P, const TX* __restrict__ DI, const TX* __restrict__ M, const TX* __restrict__ N,
                     const int* __restrict__ free_list, const T* __restrict__ rhs, double* __restrict__ y,
                     double* __restrict__ z, T* __restrict__ x, const KrylovState* st) {
  if (st != nullptr && st->done) return;
  __shared__ double vb[kMaxBlock];
  const int rank = (int)cluster_rank();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = rank * (AT / 32) + warp, nw = CL * (AT / 32);
  // 1. y_b = Di_b r_b for every block (one warp per row)
  for (int b = 0; b < P.nb; ++b) {
    const int o = P.boff[b], m = P.boff[b + 1] - o;
    const TX* D = DI + P.dioff[b];
    for (int i = gw; i < m; i += nw) {
      double acc = 0.0;
      for (int j = lane; j <= i; j += 32) {
        const int f = free_list[o + j];
        if (topo_in_range(f, P.nfull)) acc += (double)D[(long long)i * m + j] * (double)rhs[f];
      }
      acc = warp_sum(acc);
      if (lane == 0) y[o + i] = acc;
    }
  }
  cluster_sync();
  // 2. forward sweep: y_b -= M_b y_{b-1}
  for (int b = 1; b < P.nb; ++b) {
    const int o = P.boff[b], m = P.boff[b + 1] - o, op = P.boff[b - 1], mp = o - op;
    if (P.link[b]) {
      for (int j = threadIdx.x; j < mp; j += AT) vb[j] = __ldcg(y + op + j);
      __syncthreads();
      const TX* Mb = M + P.moff[b];
      for (int i = gw; i < m; i += nw) {
        double acc = 0.0;
        for (int j = lane; j < mp; j += 32) acc += (double)Mb[(long long)i * mp + j] * vb[j];
        acc = warp_sum(acc);
        if (lane == 0) y[o + i] = __ldcg(y + o + i) - acc;
      }
      __syncthreads();
    }
    cluster_sync();
  }
  // 3. z_b = Di_b^T y_b (one thread per column)
  for (int b = 0; b < P.nb; ++b) {
    const int o = P.boff[b], m = P.boff[b + 1] - o;
    const TX* D = DI + P.dioff[b];
    for (int j = rank * AT + threadIdx.x; j < m; j += CL * AT) {
      double acc = 0.0;
      for (int i = j; i < m; ++i) acc += (double)D[(long long)i * m + j] * __ldcg(y + o + i);
      z[o + j] = acc;
    }
  }
  cluster_sync();
  // 4. backward sweep: z_b -= N_b z_{b+1}
  for (int b = P.nb - 2; b >= 0; --b) {
    const int o = P.boff[b], m = P.boff[b + 1] - o, on = P.boff[b + 1], mn = P.boff[b + 2] - on;
    if (P.link[b + 1]) {
      for (int j = threadIdx.x; j < mn; j += AT) vb[j] = __ldcg(z + on + j);
      __syncthreads();
      const TX* Nb = N + P.noff[b];
      for (int i = gw; i < m; i += nw) {
        double acc = 0.0;
        for (int j = lane; j < mn; j += 32) acc += (double)Nb[(long long)i * mn + j] * vb[j];
        acc = warp_sum(acc);
        if (lane == 0) z[o + i] = __ldcg(z + o + i) - acc;
      }
      __syncthreads();
    }
    cluster_sync();
  }
  // 5. scatter
  for (int i = rank * AT + threadIdx.x; i < n; i += CL * AT) {
    const int f = free_list[i];
    if (topo_in_range(f, P.nfull)) x[f] = (T)__ldcg(z + i);
  }
}

}  // namespace cst

// ================================================================ host side
CoarsestPlan coarsest_plan(const Grid& g, const std::vector<int>& free_list) {
  CoarsestPlan p;
  p.n = (int)free_list.size();
  p.nfull = g.ndof;
  // plane of a compact DoF: node = dof/3, plane = node / (NY*NZ)
  const long long plane_nodes = (long long)g.NY * g.NZ;
  std::vector<int> plane_of(p.n);
  for (int i = 0; i < p.n; ++i) plane_of[i] = (int)((free_list[i] / 3) / plane_nodes);
  p.boff.push_back(0);
  p.link.push_back(0);
  for (int i = 1; i <= p.n; ++i) {
    if (i == p.n || plane_of[i] != plane_of[i - 1]) {
      p.boff.push_back(i);
      if (i < p.n) p.link.push_back(plane_of[i] == plane_of[i - 1] + 1 ? 1 : 0);
    }
  }
  p.nb = (int)p.boff.size() - 1;
  p.mmax = 0;
  long long di = 0, ms = 0, ns = 0;
  p.dioff.assign(p.nb, 0);
  p.moff.assign(p.nb, 0);
  p.noff.assign(p.nb, 0);
  for (int b = 0; b < p.nb; ++b) {
    const int m = p.boff[b + 1] - p.boff[b];
    p.mmax = std::max(p.mmax, m);
    p.dioff[b] = di;
    di += (long long)m * m;
    if (b > 0) {
      p.moff[b] = ms;
      ms += (long long)m * (p.boff[b] - p.boff[b - 1]);
    }
    if (b + 1 < p.nb) {
      p.noff[b] = ns;
      ns += (long long)m * (p.boff[b + 2] - p.boff[b + 1]);
    }
  }
  p.di_size = di;
  p.m_size = ms;
  p.n_size = ns;
  return p;
}

bool coarsest_supported(const CoarsestPlan& p) { return p.mmax <= cst::kMaxBlock; }

void coarsest_alloc(CoarsestFactor& f, const CoarsestPlan& p, int band, bool f64, void* (*alloc_bytes)(void*, size_t),
                    void* ctx) {
  auto A = [&](size_t bytes) { return alloc_bytes(ctx, bytes); };
  f.band = band;
  f.ldb = band + 1;
  f.f64 = f64;
  const size_t nb = (size_t)std::max(p.n, 1) * f.ldb;
  f.A = (double*)A(nb * sizeof(double));
  f.L = (double*)A(nb * sizeof(double));
  f.DI64 = (double*)A(std::max<long long>(p.di_size, 1) * sizeof(double));
  f.LS64 = (double*)A(std::max<long long>(p.m_size, 1) * sizeof(double));
  const size_t es = f64 ? sizeof(double) : sizeof(float);
  f.DI = A(std::max<long long>(p.di_size, 1) * es);
  f.M = A(std::max<long long>(p.m_size, 1) * es);
  f.N = A(std::max<long long>(p.n_size, 1) * es);
  f.flag = (int*)A(sizeof(int) * 4);
  f.bar = (unsigned*)A(sizeof(unsigned) * 4);
  f.err = f.flag + 1;
  // device copies of the plan
  f.d_boff = (int*)A(sizeof(int) * (p.nb + 1));
  f.d_link = (int*)A(sizeof(int) * std::max(p.nb, 1));
  f.d_dioff = (long long*)A(sizeof(long long) * std::max(p.nb, 1));
  f.d_moff = (long long*)A(sizeof(long long) * std::max(p.nb, 1));
  f.d_noff = (long long*)A(sizeof(long long) * std::max(p.nb, 1));
  f.d_jobs = A(sizeof(cst::GemmJob) * 2 * std::max(p.nb, 1));
  TOPO_CUDA_CHECK(cudaMemcpy(f.d_boff, p.boff.data(), sizeof(int) * (p.nb + 1), cudaMemcpyHostToDevice));
  TOPO_CUDA_CHECK(cudaMemcpy(f.d_link, p.link.data(), sizeof(int) * p.nb, cudaMemcpyHostToDevice));
  TOPO_CUDA_CHECK(cudaMemcpy(f.d_dioff, p.dioff.data(), sizeof(long long) * p.nb, cudaMemcpyHostToDevice));
  TOPO_CUDA_CHECK(cudaMemcpy(f.d_moff, p.moff.data(), sizeof(long long) * p.nb, cudaMemcpyHostToDevice));
  TOPO_CUDA_CHECK(cudaMemcpy(f.d_noff, p.noff.data(), sizeof(long long) * p.nb, cudaMemcpyHostToDevice));
  // GEMM jobs: M_b = Di_b L_{b,b-1} (b >= 1, linked), N_b = Di_b^T L_{b+1,b}^T
  std::vector<cst::GemmJob> jobs;
  for (int b = 0; b < p.nb; ++b) {
    const int m = p.boff[b + 1] - p.boff[b];
    if (b >= 1 && p.link[b]) {
      const int mp = p.boff[b] - p.boff[b - 1];
      cst::GemmJob j{};
      j.A = f.DI64 + p.dioff[b];
      j.B = f.LS64 + p.moff[b];
      j.C = (char*)f.M + p.moff[b] * es;
      j.m = m;
      j.n = mp;
      j.kdim = m;
      j.sai = m;
      j.sak = 1;
      j.sbk = mp;
      j.sbj = 1;
      jobs.push_back(j);
    }
    if (b + 1 < p.nb && p.link[b + 1]) {
      const int mn = p.boff[b + 2] - p.boff[b + 1];
      cst::GemmJob j{};
      j.A = f.DI64 + p.dioff[b];  // Di_b^T: A(i,k) = Di[k][i]
      j.B = f.LS64 + p.moff[b + 1];  // L_{b+1,b} is mn x m; its transpose: B(k,j) = L[j][k]
      j.C = (char*)f.N + p.noff[b] * es;
      j.m = m;
      j.n = mn;
      j.kdim = m;
      j.sai = 1;
      j.sak = m;
      j.sbk = 1;
      j.sbj = m;
      jobs.push_back(j);
    }
  }
  f.njobs = (int)jobs.size();
  if (!jobs.empty())
    TOPO_CUDA_CHECK(cudaMemcpy(f.d_jobs, jobs.data(), sizeof(cst::GemmJob) * jobs.size(), cudaMemcpyHostToDevice));
  // persistent factorisation: cooperative grid sized by co-residency
  int dev = 0, nsm = 0, per_sm = 0;
  TOPO_CUDA_CHECK(cudaGetDevice(&dev));
  TOPO_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  TOPO_CUDA_CHECK(cudaFuncSetAttribute(cst::k_band_chol, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(cst::CholSmem)));
  TOPO_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cst::k_band_chol, 256, sizeof(cst::CholSmem)));
  const int tiles_max = ((band + cst::CNB - 1) / cst::CNB) * ((band + cst::CNB - 1) / cst::CNB + 1) / 2;
  f.chol_grid = std::max(1, std::min(std::min(nsm * std::max(per_sm, 1), nsm), std::max(tiles_max, 1)));
  TOPO_CUDA_CHECK(cudaFuncSetAttribute(cst::k_block_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(cst::InvSmem)));
  f.plan = p;
}

void coarsest_assemble(CoarsestFactor& f, const Grid& g, const double* S, const int* dof_index, cudaStream_t s) {
  TOPO_CUDA_CHECK(cudaMemsetAsync(f.A, 0, sizeof(double) * (size_t)std::max(f.plan.n, 1) * f.ldb, s));
  const int bs = 128;
  cst::k_band_assemble<<<(unsigned)((g.nnodes + bs - 1) / bs), bs, 0, s>>>(g, S, dof_index, f.band, f.ldb, f.A);
  TOPO_LAUNCH_CHECK();
}

void coarsest_regularise(CoarsestFactor& f, double* dtmp, cudaStream_t s) {
  const int n = f.plan.n;
  cst::k_band_diag_sum<<<1, 256, 0, s>>>(n, f.band, f.ldb, f.A, dtmp);
  TOPO_LAUNCH_CHECK();
  double dsum = 0.0;
  TOPO_CUDA_CHECK(cudaMemcpyAsync(&dsum, dtmp, sizeof(double), cudaMemcpyDeviceToHost, s));
  TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
  const double eps = std::max(dsum / n * 1e-8, 1e-14);
  cst::k_band_add_diag<<<(n + 255) / 256, 256, 0, s>>>(n, f.band, f.ldb, f.A, eps);
  TOPO_LAUNCH_CHECK();
}

void coarsest_factor(CoarsestFactor& f, cudaStream_t s) {
  const CoarsestPlan& p = f.plan;
  const int n = p.n;
  if (n == 0) return;
  TOPO_CUDA_CHECK(cudaMemsetAsync(f.flag, 0, sizeof(int) * 4, s));
  TOPO_CUDA_CHECK(cudaMemsetAsync(f.bar, 0, sizeof(unsigned) * 4, s));
  TOPO_CUDA_CHECK(cudaMemsetAsync(f.L, 0, sizeof(double) * (size_t)n * f.ldb, s));
  {
    int nn = n, band = f.band;
    long long ldb = f.ldb;
    double* A = f.A;
    double* L = f.L;
    int* flag = f.flag;
    unsigned* cnt = f.bar;
    unsigned* gen = f.bar + 1;
    int* err = f.err;
    int poll = 1 << 22;
    void* args[] = {&nn, &band, &ldb, &A, &L, &flag, &cnt, &gen, &err, &poll};
    TOPO_CUDA_CHECK(cudaLaunchCooperativeKernel((const void*)cst::k_band_chol, dim3(f.chol_grid), dim3(256), args,
                                                sizeof(cst::CholSmem), s));
    count_launches(1);
  }
  const int strips = (p.mmax + cst::CNB - 1) / cst::CNB;
  cst::k_block_inverse<<<dim3(strips, p.nb), 256, sizeof(cst::InvSmem), s>>>(f.d_boff, f.band, f.ldb, f.L, f.d_dioff,
                                                                              f.DI64);
  TOPO_LAUNCH_CHECK();
  if (p.nb > 1) {
    cst::k_extract_sub<<<dim3(64, p.nb - 1), 256, 0, s>>>(f.d_boff, f.band, f.ldb, f.L, f.d_moff, f.LS64);
    TOPO_LAUNCH_CHECK();
  }
  if (f.njobs > 0) {
    const int t = (p.mmax + 31) / 32;
    if (f.f64) cst::k_gemm_batched<double><<<dim3(t, t, f.njobs), 256, 0, s>>>((const cst::GemmJob*)f.d_jobs);
    else cst::k_gemm_batched<float><<<dim3(t, t, f.njobs), 256, 0, s>>>((const cst::GemmJob*)f.d_jobs);
    TOPO_LAUNCH_CHECK();
  }
  if (f.f64) {
    TOPO_CUDA_CHECK(cudaMemcpyAsync(f.DI, f.DI64, sizeof(double) * p.di_size, cudaMemcpyDeviceToDevice, s));
  } else {
    cst::k_convert_copy<float><<<1024, 256, 0, s>>>(p.di_size, f.DI64, (float*)f.DI);
    TOPO_LAUNCH_CHECK();
  }
}

// Returns the non-positive-pivot flag (1) or a barrier timeout (< 0).
int coarsest_status(CoarsestFactor& f, cudaStream_t s) {
  int h[2] = {0, 0};
  TOPO_CUDA_CHECK(cudaMemcpyAsync(h, f.flag, sizeof(h), cudaMemcpyDeviceToHost, s));
  TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
  if (h[1]) return -1;
  return h[0] ? 1 : 0;
}

void coarsest_apply(const CoarsestFactor& f, bool vec64, const void* rhs, double* work, void* x, const KrylovState* st,
                    cudaStream_t s) {
  const CoarsestPlan& p = f.plan;
  if (p.n == 0) return;
  cst::ApplyPlan ap;
  ap.nb = p.nb;
  ap.nfull = p.nfull;
  ap.boff = f.d_boff;
  ap.link = f.d_link;
  ap.dioff = f.d_dioff;
  ap.moff = f.d_moff;
  ap.noff = f.d_noff;
  double* y = work;
  double* z = work + p.n;
  if (vec64) {
    cst::k_coarsest_apply<double, double><<<cst::CL, cst::AT, 0, s>>>(p.n, ap, (const double*)f.DI, (const double*)f.M,
                                                                      (const double*)f.N, f.d_free, (const double*)rhs,
                                                                      y, z, (double*)x, st);
  } else {
    cst::k_coarsest_apply<float, float><<<cst::CL, cst::AT, 0, s>>>(p.n, ap, (const float*)f.DI, (const float*)f.M,
                                                                    (const float*)f.N, f.d_free, (const float*)rhs, y, z,
                                                                    (float*)x, st);
  }
  TOPO_LAUNCH_CHECK();
}

TOPO_BOUNDS_READER(bounds_flag_coarsest)

}  // namespace topo
