// coarsest.cu - direct FP64 solve of the coarsest multigrid level.
//
// The coarsest operator (free DoFs only, compact numbering in reference DoF
// order) is banded: a DoF couples only to DoFs of its own and the two
// neighbouring x-planes, so |i-j| <= band with band about one x-plane of
// DoFs. The setup
//   1. assembles the lower band into band storage,
//   2. factorises it with one persistent kernel: a right-looking band
//      Cholesky over 32-column panels with one grid barrier per panel; the
//      CTA that updates the next panel's diagonal block factors it in one
//      warp's registers right away and publishes it (look-ahead), the others
//      fetch the panel rows of their trailing tiles, solve them in two warps
//      and update the tile; the factor goes to a separate band array so no
//      CTA reads a panel row another CTA has overwritten,
//   3. inverts the 32x32 diagonal blocks of L and forms W = L^-1 by forward
//      substitution in independent 16-column strips (W is dense lower
//      triangular; the band of L bounds each step's reads),
//   4. stores W (lower triangle) and W^T (strict upper triangle) in one
//      row-major matrix C in the apply precision.
// The apply z = K^-1 r = W^T (W r) is two bandwidth-bound passes over C, one
// warp per row, each reading a row contiguously.
//
// Reference: the coarsest solve of GalerkinMatFreeGMG (src/gpu_fem/
// multigrid_v4.py:774-811, 969-984): dense Cholesky with an eps*I retry when a
// pivot is not positive, and two triangular solves per application. The
// factor here is the same (a band Cholesky creates no fill outside the band);
// the triangular solves become products with the explicit inverse.
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

// Grid barrier over all CTAs of a cooperative launch on a monotonic counter:
// barrier number `epoch` (1, 2, ...) is passed once the counter reaches
// epoch * nblocks. Thread 0 arrives and polls with a bound (a timeout raises
// err and is reported to every thread of the CTA).
__device__ bool grid_barrier(unsigned* count, unsigned epoch, unsigned nblocks, int* err, int poll) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    const unsigned target = epoch * nblocks;
    if (atomicAdd(count, 1u) + 1u < target) {
      int it = 0;
      while (ld_acquire(count) < target) {
        if (++it > poll) {
          ok = 0;
          atomicExch(err, 1);
          break;
        }
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ------------------------------------------------------ persistent Cholesky
// Shared memory of one CTA: the panel's diagonal block (factored by warp 0
// into Ld and its reciprocal pivots) and the solved panel rows of the two row
// tiles of the trailing tile it updates.
struct CholSmem {
  double W[CNB][CNB + 1];
  double Ld[CNB][CNB + 1];
  double invd[CNB];
  double col[CNB];
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

// One pivot of the warp-register factor of a 32x32 diagonal block (lane =
// row). The pivot index is a template parameter so that every register index
// is a compile-time constant (the array stays in registers). Column J is
// broadcast through shared memory (one store per lane, broadcast reads);
// entries right of a lane's diagonal are updated too but never read.
template <int J>
__device__ __forceinline__ void chol_step(double (&wr)[CNB], int lane, CholSmem& S, bool& bad) {
  S.col[lane] = wr[J];
  __syncwarp();
  const double d = S.col[J];
  const bool ok = d > 0.0 && isfinite(d);
  const double dd = ok ? d : 1.0;
  const double rs = rsqrt(dd);
  const double lj = wr[J];
  if (lane == J) {
    bad |= !ok;
    S.Ld[J][J] = dd * rs;
    S.invd[J] = rs;
  } else {
    S.Ld[lane][J] = lane > J ? lj * rs : 0.0;
  }
  const double w = lj * (rs * rs);
#pragma unroll
  for (int t = J + 1; t < CNB; ++t) wr[t] = fma(-S.col[t], w, wr[t]);
  __syncwarp();
  if constexpr (J + 1 < CNB) chol_step<J + 1>(wr, lane, S, bad);
}

// Panel row i (columns k .. k+nb) into registers; zero past `lim` or outside
// the band.
__device__ __forceinline__ void panel_load(const double* A, int band, long long ldb, int k, int nb, int i, int lim,
                                           double (&x)[CNB]) {
#pragma unroll
  for (int j = 0; j < CNB; ++j)
    x[j] = (i < lim && j < nb && i - (k + j) <= band) ? ldcg(A + bidx(i, k + j, band, ldb)) : 0.0;
}

// x Ld^T = a for one row, column by column with the reciprocal pivots.
template <int J>
__device__ __forceinline__ void solve_step(double (&x)[CNB], const CholSmem& S) {
  x[J] *= S.invd[J];
#pragma unroll
  for (int q = J + 1; q < CNB; ++q) x[q] -= x[J] * S.Ld[q][J];
  if constexpr (J + 1 < CNB) solve_step<J + 1>(x, S);
}

// Warp 0 factors S.W into S.Ld and the reciprocal pivots S.invd; S.bad is
// set when a pivot was not positive (it is then taken as 1).
__device__ __forceinline__ void factor_block(CholSmem& S, int warp, int lane) {
  if (warp == 0) {
    double wr[CNB];
#pragma unroll
    for (int t = 0; t < CNB; ++t) wr[t] = S.W[lane][t];
    bool bad = false;
    chol_step<0>(wr, lane, S, bad);
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) S.bad = bad ? 1 : 0;
  }
}

// Warps: 0 factors diagonal blocks, 2 and 3 solve the panel rows of the two
// row tiles of each trailing tile (3 only for off-diagonal tiles), all 256
// threads update the tile (four outputs each). Look-ahead (band >= 32):
// tile 0 of panel k's trailing update, which CTA 0 owns, is panel k+1's
// diagonal block; CTA 0 keeps its updated values, factors them after its
// tiles and publishes the factor and pivots in Lnext (double-buffered by
// panel parity) before the barrier, so at panel k+1 the other CTAs load it
// instead of factoring, and the panel rows they prefetch meanwhile are the
// only load in front of their solves. Panel 0, and every panel when the
// band is narrower than a panel, is factored by every CTA from A.
__global__ void __launch_bounds__(256, 1) k_band_chol(int n, int band, long long ldb, double* A, double* L,
                                                      double* Lnext, int* flag, unsigned* bar_count, int* err,
                                                      int poll) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CholSmem& S = *reinterpret_cast<CholSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool solver = warp == 2 || warp == 3;
  const bool ahead = band >= CNB;
  constexpr int LN = CNB * (CNB + 1) + CNB;  // one published factor: Ld rows, then pivots
  for (int k = 0; k < n; k += CNB) {
    const int nb = min(CNB, n - k);
    const int base = k + nb;
    const int lim = min(n, base + band);
    const int nt = (lim - base + CNB - 1) / CNB;
    const int ntiles = lim > base ? nt * (nt + 1) / 2 : 0;
    const int par = (k / CNB) & 1;
    const bool own = ahead && k > 0;  // this panel's factor came from the look-ahead
    // 1. this panel's factored diagonal block and the first tile's panel rows
    if (!own) {
      for (int q = tid; q < CNB * CNB; q += blockDim.x) {
        const int i = q / CNB, j = q % CNB;
        S.W[i][j] = (i < nb && j < nb && j <= i) ? (i - j <= band ? ldcg(A + bidx(k + i, k + j, band, ldb)) : 0.0)
                                                 : (i == j ? 1.0 : 0.0);
      }
    } else if (blockIdx.x != 0) {
      const double* src = Lnext + par * LN;
      for (int q = tid; q < CNB * (CNB + 1); q += blockDim.x) (&S.Ld[0][0])[q] = ldcg(src + q);
      if (tid < CNB) S.invd[tid] = ldcg(src + CNB * (CNB + 1) + tid);
    }
    double x[CNB];
    const int r = tid >> 3, c0 = (tid & 7) * 4;  // this thread's four outputs of a trailing tile
    double a0[4] = {0.0, 0.0, 0.0, 0.0};        // their current values for the first tile
    if ((int)blockIdx.x < ntiles) {
      int ti, tj;
      tile_of(blockIdx.x, ti, tj);
      if (solver) panel_load(A, band, ldb, k, nb, (warp == 2 ? base + CNB * ti : base + CNB * tj) + lane, lim, x);
      const int i = base + CNB * ti + r;
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int j = base + CNB * tj + c0 + m;
        if (i < lim && j < lim && j <= i && i - j <= band) a0[m] = ldcg(A + bidx(i, j, band, ldb));
      }
    }
    __syncthreads();
    if (!own) {
      // every CTA does the same arithmetic, so all agree
      factor_block(S, warp, lane);
      __syncthreads();
      if (blockIdx.x == 0) {
        for (int q = tid; q < CNB * CNB; q += blockDim.x) {
          const int i = q / CNB, j = q % CNB;
          if (i < nb && j <= i && i - j <= band) L[bidx(k + i, k + j, band, ldb)] = S.Ld[i][j];
        }
        if (tid == 0 && S.bad) *flag = 1;
      }
    }
    // 2. trailing tiles of the band window
    const bool la = ahead && blockIdx.x == 0 && base < n;  // CTA 0 builds panel k+1's block in S.W
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      int ti, tj;
      tile_of(t, ti, tj);
      const int i0 = base + CNB * ti, j0 = base + CNB * tj;
      if (i0 - (j0 + CNB - 1) > band) continue;  // whole tile outside the band (uniform)
      if (warp == 2 || (warp == 3 && tj != ti)) {
        if (t != (int)blockIdx.x) panel_load(A, band, ldb, k, nb, (warp == 2 ? i0 : j0) + lane, lim, x);
        solve_step<0>(x, S);
        double(*P)[CNB + 1] = warp == 2 ? S.Pi : S.Pj;
#pragma unroll
        for (int j = 0; j < CNB; ++j) P[lane][j] = x[j];
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
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
      for (int q = 0; q < CNB; ++q) {
        const double li = S.Pi[r][q];
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m] = fma(li, Pj[c0 + m][q], acc[m]);
      }
      const int i = i0 + r;
      const bool blk = la && t == 0;  // tile 0 = panel k+1's diagonal block
      // all four loads before any store (the stores could alias them)
      double av[4];
      bool in[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int j = j0 + c0 + m;
        in[m] = i < lim && j < lim && j <= i && i - j <= band;
        const double cur = t == (int)blockIdx.x ? a0[m] : (in[m] ? ldcg(A + bidx(i, j, band, ldb)) : 0.0);
        av[m] = in[m] ? cur - acc[m] : 0.0;
      }
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        if (in[m]) A[bidx(i, j0 + c0 + m, band, ldb)] = av[m];
        // band >= 32: every entry of the block on or below the diagonal and
        // below row n is in the window; rows past n are identity-padded
        if (blk) S.W[r][c0 + m] = in[m] ? av[m] : ((i >= n && r == c0 + m) ? 1.0 : 0.0);
      }
      __syncthreads();
    }
    if (la) {
      // 3. look-ahead: factor panel k+1's block, publish it, write its L block
      factor_block(S, warp, lane);
      __syncthreads();
      const int nb1 = min(CNB, n - base);
      double* dst = Lnext + (par ^ 1) * LN;
      for (int q = tid; q < CNB * (CNB + 1); q += blockDim.x) dst[q] = (&S.Ld[0][0])[q];
      if (tid < CNB) dst[CNB * (CNB + 1) + tid] = S.invd[tid];
      for (int q = tid; q < CNB * CNB; q += blockDim.x) {
        const int i = q / CNB, j = q % CNB;
        if (i < nb1 && j <= i && i - j <= band) L[bidx(base + i, base + j, band, ldb)] = S.Ld[i][j];
      }
      if (tid == 0 && S.bad) *flag = 1;
    }
    if (!grid_barrier(bar_count, (unsigned)(k / CNB + 1), gridDim.x, err, poll)) return;
  }
}

// ------------------------------------------------------ inverse of L
// Dinv_I = L_II^-1 for every 32x32 diagonal block (identity past n): thread c
// forms column c by forward substitution.
__global__ void __launch_bounds__(CNB) k_diag_inverse(int n, int band, long long ldb, const double* __restrict__ L,
                                                      double* __restrict__ Dinv) {
  __shared__ double Ls[CNB][CNB + 1];
  __shared__ double X[CNB][CNB + 1];
  const int I = blockIdx.x, c = threadIdx.x;
  const long long r0 = (long long)I * CNB;
  for (int r = 0; r < CNB; ++r) {
    const long long i = r0 + r;
    Ls[r][c] = (i < n && c <= r && r - c <= band) ? L[bidx(i, r0 + c, band, ldb)] : (r == c ? 1.0 : 0.0);
  }
  __syncwarp();
  for (int r = 0; r < CNB; ++r) {
    double v = (r == c) ? 1.0 : 0.0;
    for (int q = c; q < r; ++q) v -= Ls[r][q] * X[q][c];
    X[r][c] = r >= c ? v / Ls[r][r] : 0.0;
  }
  __syncwarp();
  for (int r = 0; r < CNB; ++r) Dinv[(long long)I * CNB * CNB + r * CNB + c] = X[r][c];
}

// W = L^-1 by forward substitution, one strip of TWC columns per CTA. Every
// column of W is an independent forward substitution, so the strips need no
// communication: CTA J owns columns [TWC J, TWC J + TWC) and walks the
// 32-row blocks I from the one holding its first column to the last:
//   R    = E - sum_{k in [max(j0, 32I-band), 32I)} L[32I.., k] W[k, strip]
//   W_I  = Dinv_I R                    (E: the identity on these rows/columns)
// Every W read is of rows this CTA wrote in an earlier step (visible after
// __syncthreads). The strip of column 0 is the critical path, so strips are
// narrower than a row block. A step reads its L rows from L2 (all strips at
// block row I read the same rows) in 64-wide chunks, the next chunk
// prefetched into registers. Warp w takes the chunk columns k = w, w+8, ...;
// lane l keeps rows l%16 and l%16+16 of half the strip's columns (6 shared
// loads per 16 FMA, no bank conflicts); the 8 warp partials are summed
// through shared memory. The step's diagonal inverse is fetched at its start.
// W goes to W64 (lower part, FP64) and to the apply matrix (C64 or C32) as W
// in the lower triangle and W^T in the strict upper triangle, row stride ldc.
constexpr int TIT = 256, TKC = 64, TWC = 16;
struct TriSmem {
  double Ls[CNB][TKC + 1];
  double Wc[TKC][TWC];
  double red[TIT / 32][CNB][TWC + 1];
  double Rs[CNB][TWC + 1];
  double Ds[CNB][CNB + 1];
};

__global__ void __launch_bounds__(TIT) k_tri_inverse(int n, int band, long long ldb, const double* __restrict__ L,
                                                     const double* __restrict__ Dinv, double* W64, long long ldc,
                                                     double* C64, float* C32, int wave) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TriSmem& S = *reinterpret_cast<TriSmem*>(smem_raw);
  const int nT = (n + CNB - 1) / CNB;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  // Strip s takes about nT - s/2 steps. Blocks are placed on the SMs breadth
  // first (`wave` per pass), three per SM, so block b runs beside b +- wave:
  // the middle pass takes its strips in reverse order, which gives every SM
  // one long, one middle and one short strip instead of the first SMs the
  // three longest.
  int sidx = blockIdx.x;
  if (wave > 0 && (int)blockIdx.x >= wave && (int)blockIdx.x < 2 * wave) sidx = 3 * wave - 1 - (int)blockIdx.x;
  const int j0 = sidx * TWC;
  if (j0 >= n) return;  // uniform over the CTA
  constexpr int PL = CNB * TKC / TIT;  // L values fetched per thread per chunk
  constexpr int PW = TKC * TWC / TIT;  // W values fetched per thread per chunk
  constexpr int PO = CNB * TWC / TIT;  // outputs per thread per step
  static_assert(PL * TIT == CNB * TKC && PW * TIT == TKC * TWC && PO * TIT == CNB * TWC, "tile split");
  // lane mapping of the partial product: rows rl and rl+16, columns ch .. ch+TWC/2
  const int rl = lane & 15, ch = (lane >> 4) * (TWC / 2);
  double pl[PL], pw[PW];
  double dpre[CNB * CNB / TIT];
  for (int I = j0 / CNB; I < nT; ++I) {
    const int i0 = I * CNB;
    const int klo = max(j0, i0 - band);
#pragma unroll
    for (int m = 0; m < CNB * CNB / TIT; ++m) dpre[m] = Dinv[(long long)I * CNB * CNB + t + TIT * m];
    auto fetch = [&](int k0) {
#pragma unroll
      for (int m = 0; m < PL; ++m) {
        const int q = t + TIT * m;
        const int i = i0 + q / TKC, k = k0 + q % TKC;
        pl[m] = (i < n && k < i0 && i - k <= band) ? L[bidx(i, k, band, ldb)] : 0.0;
      }
#pragma unroll
      for (int m = 0; m < PW; ++m) {
        const int q = t + TIT * m;
        const int kw = k0 + q / TWC, cw = j0 + q % TWC;
        pw[m] = (kw < i0 && cw < n && cw <= kw) ? W64[(long long)kw * ldc + cw] : 0.0;
      }
    };
    double acc[TWC];
#pragma unroll
    for (int c = 0; c < TWC; ++c) acc[c] = 0.0;
    if (klo < i0) fetch(klo);
    for (int k0 = klo; k0 < i0; k0 += TKC) {
      __syncthreads();
#pragma unroll
      for (int m = 0; m < PL; ++m) {
        const int q = t + TIT * m;
        S.Ls[q / TKC][q % TKC] = pl[m];
      }
#pragma unroll
      for (int m = 0; m < PW; ++m) {
        const int q = t + TIT * m;
        S.Wc[q / TWC][q % TWC] = pw[m];
      }
      __syncthreads();
      if (k0 + TKC < i0) fetch(k0 + TKC);
#pragma unroll 4
      for (int m = 0; m < TKC / 8; ++m) {
        const int kk = warp + 8 * m;
        const double a0 = S.Ls[rl][kk], a1 = S.Ls[rl + 16][kk];
        const double2* wr = reinterpret_cast<const double2*>(&S.Wc[kk][ch]);
#pragma unroll
        for (int c2 = 0; c2 < TWC / 4; ++c2) {
          const double2 w = wr[c2];
          acc[2 * c2] = fma(a0, w.x, acc[2 * c2]);
          acc[2 * c2 + 1] = fma(a0, w.y, acc[2 * c2 + 1]);
          acc[TWC / 2 + 2 * c2] = fma(a1, w.x, acc[TWC / 2 + 2 * c2]);
          acc[TWC / 2 + 2 * c2 + 1] = fma(a1, w.y, acc[TWC / 2 + 2 * c2 + 1]);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < TWC / 2; ++c) {
      S.red[warp][rl][ch + c] = acc[c];
      S.red[warp][rl + 16][ch + c] = acc[TWC / 2 + c];
    }
#pragma unroll
    for (int m = 0; m < CNB * CNB / TIT; ++m) {
      const int q = t + TIT * m;
      S.Ds[q >> 5][q & 31] = dpre[m];
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PO; ++p) {
      const int q = t + TIT * p;
      const int r = q / TWC, c = q % TWC;
      double v = (i0 + r == j0 + c) ? 1.0 : 0.0;
#pragma unroll
      for (int w = 0; w < TIT / 32; ++w) v -= S.red[w][r][c];
      S.Rs[r][c] = v;
    }
    __syncthreads();
    double wv[PO];
#pragma unroll
    for (int p = 0; p < PO; ++p) {
      const int q = t + TIT * p;
      const int r = q / TWC, c = q % TWC;
      double v = 0.0;
      for (int m = 0; m <= r; ++m) v = fma(S.Ds[r][m], S.Rs[m][c], v);
      wv[p] = v;
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PO; ++p) {
      const int q = t + TIT * p;
      const int r = q / TWC, c = q % TWC;
      const int i = i0 + r, col = j0 + c;
      S.Rs[r][c] = wv[p];
      if (i < n && col < n && col <= i) {
        W64[(long long)i * ldc + col] = wv[p];
        if (C64 != nullptr && C64 != W64) C64[(long long)i * ldc + col] = wv[p];
        if (C32 != nullptr) C32[(long long)i * ldc + col] = (float)wv[p];
      }
    }
    __syncthreads();
    // transposed copy: rows j0 .. j0+TWC-1 of the upper triangle, columns i0 .. i0+31
    for (int q = t; q < TWC * CNB; q += TIT) {
      const int cr = j0 + q / CNB, ic = i0 + q % CNB;
      if (cr < n && ic < n && ic > cr) {
        const double v = S.Rs[q % CNB][q / CNB];
        if (C64 != nullptr) C64[(long long)cr * ldc + ic] = v;
        if (C32 != nullptr) C32[(long long)cr * ldc + ic] = (float)v;
      }
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------- apply
// z = W^T (W r) over C (W below and on the diagonal, W^T above): pass one
// y = W r_c (row i reads C[i][0..i]), pass two z_c = W^T y (row j reads
// C[j][j..n-1]). One warp per row, 16-byte loads (ldc is a multiple of 32
// elements, so every row starts 16-byte aligned), two loads in flight per
// lane, FP64 accumulation. The compact right-hand side is gathered once; both
// passes read the compact vectors (n doubles) through L1.
template <typename T>
__global__ void k_coarse_gather(int n, long long nfull, const int* __restrict__ free_list, const T* __restrict__ rhs,
                                double* __restrict__ rc, const KrylovState* st) {
  if (st != nullptr && st->done) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) {
    const int f = free_list[j];
    rc[j] = topo_in_range(f, nfull) ? (double)rhs[f] : 0.0;
  }
}

// Warp dot product sum_{j in [lo, hi)} Ci[j] v[j] of one row: 16-byte loads
// from a V-aligned start, four in flight per lane. Every load begins below
// hi <= n <= ldc at a multiple of V, and ldc is a multiple of 32, so none
// leaves the row's storage; entries outside [lo, hi) are not used.
template <typename TX>
__device__ __forceinline__ double row_dot(const TX* __restrict__ Ci, const double* __restrict__ v, int lo, int hi,
                                          int lane) {
  constexpr int V = 16 / sizeof(TX);
  constexpr int U = 4;
  double acc = 0.0;
  int j = (lo / V) * V + lane * V;
  for (; j + (U - 1) * 32 * V < hi; j += U * 32 * V) {
    TX w[U][V];
#pragma unroll
    for (int u = 0; u < U; ++u) *reinterpret_cast<uint4*>(w[u]) = __ldg(reinterpret_cast<const uint4*>(Ci + j + u * 32 * V));
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int q = 0; q < V; ++q) {
        const int jj = j + u * 32 * V + q;
        if (jj >= lo && jj < hi) acc += (double)w[u][q] * __ldg(v + jj);
      }
  }
  for (; j < hi; j += 32 * V) {
    TX w[V];
    *reinterpret_cast<uint4*>(w) = __ldg(reinterpret_cast<const uint4*>(Ci + j));
#pragma unroll
    for (int q = 0; q < V; ++q) {
      const int jj = j + q;
      if (jj >= lo && jj < hi) acc += (double)w[q] * __ldg(v + jj);
    }
  }
  return warp_sum(acc);
}

// pass one: y = W r_c (row i reads C[i][0..i])
template <typename TX>
__global__ void __launch_bounds__(256) k_coarse_lower(int n, long long ldc, const TX* __restrict__ C,
                                                      const double* __restrict__ rc, double* __restrict__ y,
                                                      const KrylovState* st) {
  if (st != nullptr && st->done) return;
  const int row = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (row >= n) return;
  const double acc = row_dot(C + (long long)row * ldc, rc, 0, row + 1, lane);
  if (lane == 0) y[row] = acc;
}

// pass two: z_c = W^T y (row j reads C[j][j..n-1]), scattered to the free DoFs
template <typename T, typename TX>
__global__ void __launch_bounds__(256) k_coarse_upper(int n, long long nfull, long long ldc, const TX* __restrict__ C,
                                                      const int* __restrict__ free_list,
                                                      const double* __restrict__ y, T* __restrict__ x,
                                                      const KrylovState* st) {
  if (st != nullptr && st->done) return;
  const int row = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (row >= n) return;
  const double acc = row_dot(C + (long long)row * ldc, y, row, n, lane);
  if (lane == 0) {
    const int f = free_list[row];
    if (topo_in_range(f, nfull)) x[f] = (T)acc;
  }
}

}  // namespace cst

// ================================================================ host side
CoarsestPlan coarsest_plan(const Grid& g, const std::vector<int>& free_list) {
  CoarsestPlan p;
  p.n = (int)free_list.size();
  p.nfull = g.ndof;
  p.nt = (p.n + cst::CNB - 1) / cst::CNB;
  return p;
}

void coarsest_alloc(CoarsestFactor& f, const CoarsestPlan& p, int band, bool f64, void* (*alloc_bytes)(void*, size_t),
                    void* ctx) {
  auto A = [&](size_t bytes) { return alloc_bytes(ctx, bytes); };
  f.band = band;
  f.ldb = band + 1;
  f.f64 = f64;
  const int n = std::max(p.n, 1);
  const size_t nbs = (size_t)n * f.ldb;
  f.A = (double*)A(nbs * sizeof(double));
  f.L = (double*)A(nbs * sizeof(double));
  f.Dinv = (double*)A((size_t)std::max(p.nt, 1) * cst::CNB * cst::CNB * sizeof(double));
  f.Lnext = (double*)A(2 * (size_t)(cst::CNB * (cst::CNB + 1) + cst::CNB) * sizeof(double));
  f.ldc = ((long long)n + 31) / 32 * 32;
  f.W64 = (double*)A((size_t)n * f.ldc * sizeof(double));
  f.C = f64 ? (void*)f.W64 : A((size_t)n * f.ldc * sizeof(float));
  f.flag = (int*)A(sizeof(int) * 4);
  f.bar = (unsigned*)A(sizeof(unsigned) * 4);
  f.err = f.flag + 1;
  // persistent factorisation: cooperative grid sized by co-residency
  int dev = 0, nsm = 0, per_sm = 0;
  TOPO_CUDA_CHECK(cudaGetDevice(&dev));
  TOPO_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  TOPO_CUDA_CHECK(cudaFuncSetAttribute(cst::k_band_chol, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(cst::CholSmem)));
  TOPO_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cst::k_band_chol, 256, sizeof(cst::CholSmem)));
  const int tiles_max = ((band + cst::CNB - 1) / cst::CNB) * ((band + cst::CNB - 1) / cst::CNB + 1) / 2;
  f.chol_grid = std::max(1, std::min(std::min(nsm * std::max(per_sm, 1), nsm), std::max(tiles_max, 1)));
  f.nsm = nsm;
  TOPO_CUDA_CHECK(cudaFuncSetAttribute(cst::k_tri_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(cst::TriSmem)));
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
    double* Ln = f.Lnext;
    int* flag = f.flag;
    unsigned* cnt = f.bar;
    int* err = f.err;
    int poll = 1 << 24;
    void* args[] = {&nn, &band, &ldb, &A, &L, &Ln, &flag, &cnt, &err, &poll};
    TOPO_CUDA_CHECK(cudaLaunchCooperativeKernel((const void*)cst::k_band_chol, dim3(f.chol_grid), dim3(256), args,
                                                sizeof(cst::CholSmem), s));
    count_launches(1);
  }
  cst::k_diag_inverse<<<p.nt, cst::CNB, 0, s>>>(n, f.band, f.ldb, f.L, f.Dinv);
  TOPO_LAUNCH_CHECK();
  cst::k_tri_inverse<<<(n + cst::TWC - 1) / cst::TWC, cst::TIT, sizeof(cst::TriSmem), s>>>(
      n, f.band, f.ldb, f.L, f.Dinv, f.W64, f.ldc, f.f64 ? f.W64 : nullptr, f.f64 ? nullptr : (float*)f.C,
      (n + cst::TWC - 1) / cst::TWC >= 3 * f.nsm ? f.nsm : 0);
  TOPO_LAUNCH_CHECK();
}

// Returns the non-positive-pivot flag (1) or a barrier timeout (< 0).
int coarsest_status(CoarsestFactor& f, cudaStream_t s) {
  int h[2] = {0, 0};
  TOPO_CUDA_CHECK(cudaMemcpyAsync(h, f.flag, sizeof(h), cudaMemcpyDeviceToHost, s));
  TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
  if (h[1]) return -1;
  return h[0] ? 1 : 0;
}

// work: 2n doubles (y, then the compact right-hand side).
void coarsest_apply(const CoarsestFactor& f, bool vec64, const void* rhs, double* work, void* x, const KrylovState* st,
                    cudaStream_t s) {
  const CoarsestPlan& p = f.plan;
  const int n = p.n;
  if (n == 0) return;
  const int wpb = 8;
  const unsigned nb = (unsigned)((n + wpb - 1) / wpb);
  const unsigned ng = (unsigned)((n + 255) / 256);
  double* y = work;
  double* rc = work + n;
  if (vec64) {
    if (!f.f64) throw std::runtime_error("coarsest apply: FP64 vectors need the FP64 inverse");
    cst::k_coarse_gather<double><<<ng, 256, 0, s>>>(n, p.nfull, f.d_free, (const double*)rhs, rc, st);
    TOPO_LAUNCH_CHECK();
    cst::k_coarse_lower<double><<<nb, 32 * wpb, 0, s>>>(n, f.ldc, (const double*)f.C, rc, y, st);
    TOPO_LAUNCH_CHECK();
    cst::k_coarse_upper<double, double><<<nb, 32 * wpb, 0, s>>>(n, p.nfull, f.ldc, (const double*)f.C, f.d_free, y,
                                                                (double*)x, st);
  } else {
    cst::k_coarse_gather<float><<<ng, 256, 0, s>>>(n, p.nfull, f.d_free, (const float*)rhs, rc, st);
    TOPO_LAUNCH_CHECK();
    if (f.f64) {
      cst::k_coarse_lower<double><<<nb, 32 * wpb, 0, s>>>(n, f.ldc, (const double*)f.C, rc, y, st);
      TOPO_LAUNCH_CHECK();
      cst::k_coarse_upper<float, double><<<nb, 32 * wpb, 0, s>>>(n, p.nfull, f.ldc, (const double*)f.C, f.d_free, y,
                                                                 (float*)x, st);
    } else {
      cst::k_coarse_lower<float><<<nb, 32 * wpb, 0, s>>>(n, f.ldc, (const float*)f.C, rc, y, st);
      TOPO_LAUNCH_CHECK();
      cst::k_coarse_upper<float, float><<<nb, 32 * wpb, 0, s>>>(n, p.nfull, f.ldc, (const float*)f.C, f.d_free, y,
                                                                (float*)x, st);
    }
  }
  TOPO_LAUNCH_CHECK();
}

TOPO_BOUNDS_READER(bounds_flag_coarsest)

}  // namespace topo
