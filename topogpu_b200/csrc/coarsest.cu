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
//   3. splits the rows into P diagonal blocks (boundaries on 32-row panels,
//      each block at least `band` rows, so L is block bidiagonal and block
//      q+1 reaches block q only through a band x band corner), inverts the
//      32x32 diagonal blocks of L and forms W_q = L_qq^-1 for every block by
//      forward substitution in independent 16-column strips (a strip is at
//      most m/32 steps long instead of n/32),
//   4. folds the corners through W_q into G_q = W_q Lc_q and
//      H_q = (Lc_{q+1} W_q[last band rows])^T (FP64 products),
//   5. stores per block W_q (lower triangle), W_q^T (strict upper triangle),
//      G_q and H_q in one row-major matrix in the apply precision.
// The apply z = K^-1 r runs the two triangular solves block by block: a
// lower pass y_q = W_q r_q - G_q y_{q-1}[tail] for q = 0 .. P-1 and an upper
// pass z_q = W_q^T y_q - H_q z_{q+1}[head] for q = P-1 .. 0, each a
// bandwidth-bound product, one warp per row. It reads the P diagonal blocks
// and their couplings (about n^2/P + 2 n band entries) instead of the n^2 of
// the dense W^T W.
//
// Reference: the coarsest solve of GalerkinMatFreeGMG (src/gpu_fem/
// multigrid_v4.py:774-811, 969-984): dense Cholesky with an eps*I retry when a
// pivot is not positive, and two triangular solves per application. The
// factor here is the same (a band Cholesky creates no fill outside the band);
// the triangular solves become products with the explicit inverses of the
// diagonal blocks.
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

// W_q = L_qq^-1 for every diagonal block q by forward substitution, one strip
// of TWC columns per CTA. Every column is an independent forward substitution
// inside its block, so the strips need no communication: a strip with first
// column j0 walks the 32-row blocks I from the one holding j0 to the end of
// its diagonal block:
//   R    = E - sum_{k in [max(j0, 32I-band), 32I)} L[32I.., k] W[k, strip]
//   W_I  = Dinv_I R                    (E: the identity on these rows/columns)
// Every W read is of rows this CTA wrote in an earlier step (visible after
// __syncthreads). A strip takes (block end - j0)/32 steps; CTA r takes strip
// r/P of block r%P, so the longest strips of all blocks start first. A step
// reads its L rows from L2 (all strips at block row I read the same rows) in
// 64-wide chunks, the next chunk prefetched into registers. Warp w takes the
// chunk columns k = w, w+8, ...; lane l keeps rows l%16 and l%16+16 of half
// the strip's columns (6 shared loads per 16 FMA, no bank conflicts); the 8
// warp partials are summed through shared memory. The step's diagonal inverse
// is fetched at its start. W_q goes to W64 (lower part, FP64) and to the
// apply matrix (C64 or C32) as W_q in the lower triangle and W_q^T in the
// strict upper triangle of the block's columns 0 .. m-1.
constexpr int TIT = 256, TKC = 64, TWC = 16;
struct TriSmem {
  double Ls[CNB][TKC + 1];
  double Wc[TKC][TWC];
  double red[TIT / 32][CNB][TWC + 1];
  double Rs[CNB][TWC + 1];
  double Ds[CNB][CNB + 1];
};

__global__ void __launch_bounds__(TIT) k_tri_inverse(int n, int band, long long ldb, const double* __restrict__ L,
                                                     const double* __restrict__ Dinv, CoarseBlocks bk, double* W64,
                                                     double* C64, float* C32) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TriSmem& S = *reinterpret_cast<TriSmem*>(smem_raw);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int blk = (int)blockIdx.x % bk.P;
  const int b0 = bk.b[blk], iend = bk.b[blk + 1];
  const int j0 = b0 + ((int)blockIdx.x / bk.P) * TWC;
  if (j0 >= iend) return;  // uniform over the CTA
  const int nT = (iend + CNB - 1) / CNB;
  const long long ld = bk.ld[blk];
  double* Wq = W64 + bk.off[blk];
  double* C64q = C64 != nullptr ? C64 + bk.off[blk] : nullptr;
  float* C32q = C32 != nullptr ? C32 + bk.off[blk] : nullptr;
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
        pw[m] = (kw < i0 && cw < iend && cw <= kw) ? Wq[(long long)(kw - b0) * ld + (cw - b0)] : 0.0;
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
      if (i < iend && col < iend && col <= i) {
        const long long a = (long long)(i - b0) * ld + (col - b0);
        Wq[a] = wv[p];
        if (C64q != nullptr && C64q != Wq) C64q[a] = wv[p];
        if (C32q != nullptr) C32q[a] = (float)wv[p];
      }
    }
    __syncthreads();
    // transposed copy: rows j0 .. j0+TWC-1 of the upper triangle, columns i0 .. i0+31
    for (int e = t; e < TWC * CNB; e += TIT) {
      const int cr = j0 + e / CNB, ic = i0 + e % CNB;
      if (cr < iend && ic < iend && ic > cr) {
        const double v = S.Rs[e % CNB][e / CNB];
        const long long a = (long long)(cr - b0) * ld + (ic - b0);
        if (C64q != nullptr) C64q[a] = v;
        if (C32q != nullptr) C32q[a] = (float)v;
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------- couplings between the blocks
// With the block-bidiagonal L (diagonal blocks L_qq, corners Lc_q = the rows
// b[q] .. b[q]+band-1 of L over the columns b[q]-band .. b[q]-1), the two
// triangular solves of K^-1 r become, block by block,
//   y_q = W_q r_q - G_q y_{q-1}[m_{q-1}-band ..],   G_q = W_q[:, 0:band] Lc_q
//   z_q = W_q^T y_q - H_q z_{q+1}[0 .. band),       H_q = (Lc_{q+1} W_q[m-band.., :])^T
// k_couplings forms G_q (q >= 1) and H_q (q < P-1) in FP64 from W64 and L:
// one CTA per 64 x 32 output tile, 16-wide l chunks staged in shared memory,
// each thread 2 rows x 4 columns. Lc_q[l][k] is non-zero for l <= k only and
// W_q is lower triangular, so a tile's l range is clipped to where both are.
constexpr int GTI = 64, GTK = 32, GTL = 16;
__global__ void __launch_bounds__(256) k_couplings(int band, long long ldb, const double* __restrict__ L,
                                                   CoarseBlocks bk, const double* W64, double* C64, float* C32) {
  __shared__ __align__(16) double As[GTL][GTI + 2];
  __shared__ __align__(16) double Bs[GTL][GTK + 2];
  const int q = (int)blockIdx.y >> 1, type = (int)blockIdx.y & 1;  // type 0: G_q, 1: H_q
  if (q >= bk.P || (type == 0 && q == 0) || (type == 1 && q == bk.P - 1)) return;
  const int m = bk.b[q + 1] - bk.b[q];
  const int nkt = (band + GTK - 1) / GTK;
  const int i0 = ((int)blockIdx.x / nkt) * GTI, k0 = ((int)blockIdx.x % nkt) * GTK;
  if (i0 >= m) return;
  const long long ld = bk.ld[q];
  const double* Wq = W64 + bk.off[q];
  // rows of L holding the corner: G_q uses block q's, H_q block q+1's
  const long long cb = type == 0 ? bk.b[q] : bk.b[q + 1];
  int lo, hi;
  if (type == 0) {  // l <= k and l <= i
    lo = 0;
    hi = min(band, min(k0 + GTK, i0 + GTI));
  } else {          // l >= k and m-band+l >= i
    lo = max(k0, i0 - (m - band));
    lo = max(lo, 0);
    hi = band;
  }
  const int t = threadIdx.x, tx = t & 7, ty = t >> 3;  // columns 4tx.., rows 2ty, 2ty+1
  double acc[2][4] = {};
  for (int l0 = lo; l0 < hi; l0 += GTL) {
    __syncthreads();
    // A(i, l): G: W_q[i][l]; H: W_q[m-band+l][i]
#pragma unroll
    for (int u = 0; u < GTI * GTL / 256; ++u) {
      const int e = t + 256 * u;
      int il, ll;
      if (type == 0) { ll = e % GTL; il = e / GTL; }   // l fastest: a row of W_q
      else { il = e % GTI; ll = e / GTI; }             // i fastest: a row of W_q
      const int i = i0 + il, l = l0 + ll;
      double v = 0.0;
      if (i < m && l < hi) {
        if (type == 0) { if (l <= i) v = Wq[(long long)i * ld + l]; }
        else { const int r = m - band + l; if (r >= i) v = Wq[(long long)r * ld + i]; }
      }
      As[ll][il] = v;
    }
    // B(l, k): G: Lc_q[l][k] = L[cb+l][cb-band+k]; H: Lc_{q+1}[k][l] = L[cb+k][cb-band+l]
#pragma unroll
    for (int u = 0; u < GTK * GTL / 256; ++u) {
      const int e = t + 256 * u;
      int kl, ll;
      if (type == 0) { kl = e % GTK; ll = e / GTK; }
      else { ll = e % GTL; kl = e / GTL; }
      const int k = k0 + kl, l = l0 + ll;
      double v = 0.0;
      if (k < band && l < hi) {
        if (type == 0) { if (l <= k) v = L[bidx(cb + l, cb - band + k, band, ldb)]; }
        else { if (k <= l) v = L[bidx(cb + k, cb - band + l, band, ldb)]; }
      }
      Bs[ll][kl] = v;
    }
    __syncthreads();
    const int lend = min(GTL, hi - l0);
    for (int ll = 0; ll < lend; ++ll) {
      const double2 a = *reinterpret_cast<const double2*>(&As[ll][2 * ty]);
      const double2 b01 = *reinterpret_cast<const double2*>(&Bs[ll][4 * tx]);
      const double2 b23 = *reinterpret_cast<const double2*>(&Bs[ll][4 * tx + 2]);
      const double b[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        acc[0][c] = fma(a.x, b[c], acc[0][c]);
        acc[1][c] = fma(a.y, b[c], acc[1][c]);
      }
    }
  }
  const int col0 = (type == 0 ? bk.gofs[q] : bk.hofs[q]) + k0 + 4 * tx;
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int i = i0 + 2 * ty + r;
    if (i >= m) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (k0 + 4 * tx + c >= band) continue;
      const long long a = bk.off[q] + (long long)i * ld + col0 + c;
      if (C64 != nullptr) C64[a] = acc[r][c];
      if (C32 != nullptr) C32[a] = (float)acc[r][c];
    }
  }
}

// --------------------------------------------------------------- apply
// z = K^-1 r block by block: the lower pass for q = 0 .. P-1 forms
// y_q = W_q r_q - G_q y_{q-1}[tail] (row i reads C_q[i][0..i] and G_q[i]), the
// upper pass for q = P-1 .. 0 forms z_q = W_q^T y_q - H_q z_{q+1}[head] (row i
// reads C_q[i][i..m-1] and H_q[i]) and scatters it to the free DoFs. Each row
// is split over RW warps (interleaved 32-lane chunks of 16-byte loads; row
// strides and segment starts are multiples of 32 elements, so every segment
// starts 16-byte aligned), FP64 accumulation, the RW partial sums added
// through shared memory. With four warps per row one block
// (about 4 band rows) is a single short wave, so the 2P dependent launches of
// an apply cost about 5 us each. The compact right-hand side is gathered
// once; both passes read the compact vectors through L1.
constexpr int RW = 4;  // warps per row

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

// One warp's share of sum_{j in [lo, hi)} Ci[j] v[j] over a row segment:
// chunks c = sub, sub+RW, ... of 32 lanes x one 16-byte load, four chunks in
// flight. Every load begins below hi at a multiple of V and every segment
// (W_q: m columns, G_q and H_q: band columns) is padded to a multiple of 32,
// so none leaves its segment; entries outside [lo, hi) are not used.
template <typename TX>
__device__ __forceinline__ double seg_dot(const TX* __restrict__ Ci, const double* __restrict__ v, int lo, int hi,
                                          int lane, int sub) {
  constexpr int V = 16 / sizeof(TX);
  constexpr int STEP = RW * 32 * V;
  constexpr int U = 4;
  double acc = 0.0;
  int j = (lo / V) * V + (sub * 32 + lane) * V;
  for (; j + (U - 1) * STEP < hi; j += U * STEP) {
    TX w[U][V];
#pragma unroll
    for (int u = 0; u < U; ++u) *reinterpret_cast<uint4*>(w[u]) = __ldg(reinterpret_cast<const uint4*>(Ci + j + u * STEP));
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int q = 0; q < V; ++q) {
        const int jj = j + u * STEP + q;
        if (jj >= lo && jj < hi) acc += (double)w[u][q] * __ldg(v + jj);
      }
  }
  for (; j < hi; j += STEP) {
    TX w[V];
    *reinterpret_cast<uint4*>(w) = __ldg(reinterpret_cast<const uint4*>(Ci + j));
#pragma unroll
    for (int q = 0; q < V; ++q) {
      const int jj = j + q;
      if (jj >= lo && jj < hi) acc += (double)w[q] * __ldg(v + jj);
    }
  }
  return acc;
}

// Sum of the RW warp partials of each row of the CTA (every thread calls it).
__device__ __forceinline__ double row_sum(double acc, int warp, int lane) {
  __shared__ double part[8];
  acc = warp_sum(acc);
  if (lane == 0) part[warp] = acc;
  __syncthreads();
  double t = 0.0;
  if (warp % RW == 0)
#pragma unroll
    for (int k = 0; k < RW; ++k) t += part[warp + k];
  return t;
}

// pass one, block q (rows b0 .. b0+m-1): y_q = W_q r_q - G_q y_{q-1}[m_{q-1}-band ..]
template <typename TX>
__global__ void __launch_bounds__(256) k_coarse_lower(int m, int b0, long long ld, int gofs, int band, int prev,
                                                      const TX* __restrict__ Cq, const double* __restrict__ rc,
                                                      double* y, const KrylovState* st) {
  if (st != nullptr && st->done) return;  // uniform over the grid
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = (int)blockIdx.x * (8 / RW) + warp / RW, sub = warp % RW;
  const bool live = row < m;
  double acc = 0.0;
  if (live) {
    const TX* Ci = Cq + (long long)row * ld;
    acc = seg_dot(Ci, rc + b0, 0, row + 1, lane, sub);
    if (prev) acc -= seg_dot(Ci + gofs, y + (b0 - band), 0, band, lane, sub);
  }
  acc = row_sum(acc, warp, lane);
  if (live && sub == 0 && lane == 0) y[b0 + row] = acc;
}

// pass two, block q: z_q = W_q^T y_q - H_q z_{q+1}[0 .. band), kept compact in
// z and scattered to the free DoFs of x
template <typename T, typename TX>
__global__ void __launch_bounds__(256) k_coarse_upper(int m, int b0, long long ld, int hofs, int band, int next,
                                                      long long nfull, const TX* __restrict__ Cq,
                                                      const int* __restrict__ free_list, const double* y, double* z,
                                                      T* __restrict__ x, const KrylovState* st) {
  if (st != nullptr && st->done) return;  // uniform over the grid
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = (int)blockIdx.x * (8 / RW) + warp / RW, sub = warp % RW;
  const bool live = row < m;
  double acc = 0.0;
  if (live) {
    const TX* Ci = Cq + (long long)row * ld;
    acc = seg_dot(Ci, y + b0, row, m, lane, sub);
    if (next) acc -= seg_dot(Ci + hofs, z + (b0 + m), 0, band, lane, sub);
  }
  acc = row_sum(acc, warp, lane);
  if (live && sub == 0 && lane == 0) {
    z[b0 + row] = acc;
    const int f = free_list[b0 + row];
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
  // diagonal blocks of W: at least max(4 band, 512) rows each (every block at
  // least `band` rows), boundaries on 32-row panels
  CoarseBlocks& bk = f.blk;
  int P = std::max(1, std::min(COARSE_MAXB, n / std::max(4 * band, 512)));
  for (;;) {
    bk.P = P;
    bk.b[0] = 0;
    for (int q = 1; q < P; ++q) bk.b[q] = (int)((long long)q * n / P / cst::CNB * cst::CNB);
    bk.b[P] = n;
    bool ok = true;
    for (int q = 0; q < P; ++q) ok = ok && bk.b[q + 1] - bk.b[q] >= std::max(band, 1);
    if (ok || P == 1) break;
    --P;
  }
  const long long bandp = ((long long)band + 31) / 32 * 32;
  long long off = 0;
  int maxm = 0;
  for (int q = 0; q < bk.P; ++q) {
    const int m = bk.b[q + 1] - bk.b[q];
    maxm = std::max(maxm, m);
    bk.gofs[q] = (m + 31) / 32 * 32;
    bk.hofs[q] = (int)(bk.gofs[q] + bandp);
    bk.ld[q] = bk.gofs[q] + (bk.P > 1 ? 2 * bandp : 0);
    bk.off[q] = off;
    off += (long long)m * bk.ld[q];
  }
  f.strips_per_block = (maxm + cst::TWC - 1) / cst::TWC;
  f.W64 = (double*)A((size_t)off * sizeof(double));
  f.C = f64 ? (void*)f.W64 : A((size_t)off * sizeof(float));
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
  const CoarseBlocks& bk = f.blk;
  double* C64 = f.f64 ? f.W64 : nullptr;
  float* C32 = f.f64 ? nullptr : (float*)f.C;
  cst::k_tri_inverse<<<(unsigned)(bk.P * f.strips_per_block), cst::TIT, sizeof(cst::TriSmem), s>>>(
      n, f.band, f.ldb, f.L, f.Dinv, bk, f.W64, C64, C32);
  TOPO_LAUNCH_CHECK();
  if (bk.P > 1) {
    int maxm = 0;
    for (int q = 0; q < bk.P; ++q) maxm = std::max(maxm, bk.b[q + 1] - bk.b[q]);
    const int nkt = (f.band + cst::GTK - 1) / cst::GTK;
    const dim3 grid((unsigned)(((maxm + cst::GTI - 1) / cst::GTI) * nkt), (unsigned)(2 * bk.P));
    cst::k_couplings<<<grid, 256, 0, s>>>(f.band, f.ldb, f.L, bk, f.W64, C64, C32);
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

// work: 2n doubles (y, then the compact right-hand side, overwritten by the
// compact solution in the second pass).
template <typename T, typename TX>
static void apply_blocks(const CoarsestFactor& f, const T* rhs, double* work, T* x, const KrylovState* st,
                         cudaStream_t s) {
  const CoarsestPlan& p = f.plan;
  const CoarseBlocks& bk = f.blk;
  const int n = p.n;
  constexpr int rpb = 8 / cst::RW;  // rows per 256-thread CTA
  double* y = work;
  double* rc = work + n;
  const TX* C = (const TX*)f.C;
  cst::k_coarse_gather<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, p.nfull, f.d_free, rhs, rc, st);
  TOPO_LAUNCH_CHECK();
  for (int q = 0; q < bk.P; ++q) {
    const int m = bk.b[q + 1] - bk.b[q];
    cst::k_coarse_lower<TX><<<(unsigned)((m + rpb - 1) / rpb), 256, 0, s>>>(
        m, bk.b[q], bk.ld[q], bk.gofs[q], f.band, (int)(q > 0), C + bk.off[q], rc, y, st);
    TOPO_LAUNCH_CHECK();
  }
  for (int q = bk.P - 1; q >= 0; --q) {
    const int m = bk.b[q + 1] - bk.b[q];
    cst::k_coarse_upper<T, TX><<<(unsigned)((m + rpb - 1) / rpb), 256, 0, s>>>(
        m, bk.b[q], bk.ld[q], bk.hofs[q], f.band, (int)(q < bk.P - 1), p.nfull, C + bk.off[q], f.d_free, y, rc, x,
        st);
    TOPO_LAUNCH_CHECK();
  }
}

void coarsest_apply(const CoarsestFactor& f, bool vec64, const void* rhs, double* work, void* x, const KrylovState* st,
                    cudaStream_t s) {
  if (f.plan.n == 0) return;
  if (vec64) {
    if (!f.f64) throw std::runtime_error("coarsest apply: FP64 vectors need the FP64 inverse");
    apply_blocks<double, double>(f, (const double*)rhs, work, (double*)x, st, s);
  } else if (f.f64) {
    apply_blocks<float, double>(f, (const float*)rhs, work, (float*)x, st, s);
  } else {
    apply_blocks<float, float>(f, (const float*)rhs, work, (float*)x, st, s);
  }
}

TOPO_BOUNDS_READER(bounds_flag_coarsest)

}  // namespace topo
