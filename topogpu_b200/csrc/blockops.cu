// blockops.cu - multi-vector kernels of the block PCG (several load cases on
// one density field).
//
//   * k_level0_block: Y_v = K(E) U_v for v < nv in one launch. A CTA stages
//     its brick of moduli once and reuses it for every vector (KE sits in
//     constant memory), so E is read once per launch instead of once per
//     load case.
//   * k_gram / k_gram_final: all nA x nB dot products A_i . B_j in one pass
//     over the vectors, with deterministic block partials.
//   * k_block_combine: Out_j = C_j + sign * sum_i In_i M[i][j], the column
//     updates X += P a, R -= Q a and P = Z + P b of block CG.
// Block vectors are FP64 and passed as device arrays of column pointers, so
// deflating converged columns only changes the pointer lists.
#include "internal.cuh"
#include "reduce.cuh"

#include <stdexcept>

namespace topo {

__device__ __forceinline__ int corner_id_b(int bx, int by, int bz) { return bz * 4 + (by ? (bx ? 2 : 3) : (bx ? 1 : 0)); }

__constant__ double cKEb[576];

void set_ke_block(const double* KE) { TOPO_CUDA_CHECK(cudaMemcpyToSymbol(cKEb, KE, sizeof(double) * 576)); }

constexpr int BZ = 32, BY = 4, BX = 2;
constexpr int BUZ = BZ + 2, BUY = BY + 2, BUX = BX + 2;
constexpr int BEZ = BZ + 1, BEY = BY + 1, BEX = BX + 1;
constexpr int MAXV = 16;

struct ColPtrs {
  const double* p[MAXV];
};
struct ColOut {
  double* p[MAXV];
};

__global__ void __launch_bounds__(BX * BY * BZ)
k_level0_block(Grid g, ColPtrs U, const double* __restrict__ E, const uint8_t* __restrict__ mask, ColOut Y, int nv) {
  __shared__ __align__(16) double us[BUX][BUY][BUZ][4];
  __shared__ double es[BEX][BEY][BEZ];
  const int z0 = blockIdx.x * BZ, y0 = blockIdx.y * BY, x0 = blockIdx.z * BX;
  const int tid = threadIdx.x + BZ * (threadIdx.y + BY * threadIdx.z);
  constexpr int NT = BX * BY * BZ;
  for (int idx = tid; idx < BEX * BEY * BEZ; idx += NT) {
    const int zz = idx % BEZ, yy = (idx / BEZ) % BEY, xx = idx / (BEZ * BEY);
    const int gx = x0 - 1 + xx, gy = y0 - 1 + yy, gz = z0 - 1 + zz;
    double v = 0;
    if (gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny && gz >= 0 && gz < g.nz)
      v = E[((long long)gx * g.ny + gy) * g.nz + gz];
    es[xx][yy][zz] = v;
  }
  const int tz = threadIdx.x, ty = threadIdx.y, tx = threadIdx.z;
  const int gx = x0 + tx, gy = y0 + ty, gz = z0 + tz;
  const bool inside = gx < g.NX && gy < g.NY && gz < g.NZ;
  const long long node = ((long long)gx * g.NY + gy) * g.NZ + gz;
  for (int v = 0; v < nv; ++v) {
    __syncthreads();  // previous vector's reads of us are done
    const double* u = U.p[v];
    for (int idx = tid; idx < BUX * BUY * BUZ * 3; idx += NT) {
      const int c = idx % 3, zz = (idx / 3) % BUZ, yy = (idx / (3 * BUZ)) % BUY, xx = idx / (3 * BUZ * BUY);
      const int ggx = x0 - 1 + xx, ggy = y0 - 1 + yy, ggz = z0 - 1 + zz;
      double val = 0;
      if (ggx >= 0 && ggx < g.NX && ggy >= 0 && ggy < g.NY && ggz >= 0 && ggz < g.NZ)
        val = u[3 * (((long long)ggx * g.NY + ggy) * g.NZ + ggz) + c];
      us[xx][yy][zz][c] = val;
    }
    __syncthreads();
    if (!inside) continue;
    double t[2][2][2][3];
#pragma unroll
    for (int o = 0; o < 8; ++o)
#pragma unroll
      for (int c = 0; c < 3; ++c) t[o >> 2][(o >> 1) & 1][o & 1][c] = 0;
#pragma unroll
    for (int dx = 0; dx < 3; ++dx)
#pragma unroll
      for (int dy = 0; dy < 3; ++dy)
#pragma unroll
        for (int dz = 0; dz < 3; ++dz) {
          const double* rec = &us[tx + dx][ty + dy][tz + dz][0];
          const double2 v01 = *reinterpret_cast<const double2*>(rec);
          const double uv[3] = {v01.x, v01.y, rec[2]};
#pragma unroll
          for (int ox = 0; ox < 2; ++ox)
#pragma unroll
            for (int oy = 0; oy < 2; ++oy)
#pragma unroll
              for (int oz = 0; oz < 2; ++oz) {
                const int mx = dx - ox, my = dy - oy, mz = dz - oz;
                if (mx < 0 || mx > 1 || my < 0 || my > 1 || mz < 0 || mz > 1) continue;
                const int a = corner_id_b(1 - ox, 1 - oy, 1 - oz);
                const int m = corner_id_b(mx, my, mz);
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                  for (int d = 0; d < 3; ++d) t[ox][oy][oz][c] += cKEb[(3 * a + c) * 24 + 3 * m + d] * uv[d];
              }
        }
    double acc[3] = {0, 0, 0};
#pragma unroll
    for (int ox = 0; ox < 2; ++ox)
#pragma unroll
      for (int oy = 0; oy < 2; ++oy)
#pragma unroll
        for (int oz = 0; oz < 2; ++oz) {
          const double Ee = es[tx + ox][ty + oy][tz + oz];
#pragma unroll
          for (int c = 0; c < 3; ++c) acc[c] += Ee * t[ox][oy][oz][c];
        }
    double* y = Y.p[v];
#pragma unroll
    for (int c = 0; c < 3; ++c) y[3 * node + c] = mask[3 * node + c] ? acc[c] : 0.0;
  }
}

void level0_apply_block(const Grid& g, const double* const* U, const double* E, const uint8_t* mask,
                        double* const* Y, int nv, cudaStream_t s) {
  if (nv < 1 || nv > MAXV) throw std::invalid_argument("level0_apply_block: 1..16 vectors");
  ColPtrs cu{};
  ColOut cy{};
  for (int v = 0; v < nv; ++v) {
    cu.p[v] = U[v];
    cy.p[v] = Y[v];
  }
  dim3 block(BZ, BY, BX), grid((g.NZ + BZ - 1) / BZ, (g.NY + BY - 1) / BY, (g.NX + BX - 1) / BX);
  k_level0_block<<<grid, block, 0, s>>>(g, cu, E, mask, cy, nv);
  TOPO_LAUNCH_CHECK();
}

// G[i][j] = A_i . B_j. Block b sums rows b, b + grid, ... and leaves its
// partials in part[b][i][j]; k_gram_final adds the partials in block order.
constexpr int GRAM_BLOCKS = 296, GRAM_THREADS = 256;
__global__ void __launch_bounds__(GRAM_THREADS) k_gram(long long n, ColPtrs A, int na, ColPtrs B, int nb,
                                                       double* __restrict__ part) {
  double acc[MAXV * MAXV / 4];  // na * nb <= 64 (block sizes up to 8)
#pragma unroll
  for (int q = 0; q < MAXV * MAXV / 4; ++q) acc[q] = 0.0;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
    double a[8], b[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      a[i] = i < na ? A.p[i][r] : 0.0;
      b[i] = i < nb ? B.p[i][r] : 0.0;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i * 8 + j] += a[i] * b[j];
  }
  __shared__ double red[GRAM_THREADS / 32][64];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 64; ++q) {
    const double v = warp_sum(acc[q]);
    if (lane == 0) red[warp][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < 64) {
    double s = 0.0;
    for (int w = 0; w < GRAM_THREADS / 32; ++w) s += red[w][threadIdx.x];
    part[(long long)blockIdx.x * 64 + threadIdx.x] = s;
  }
}

__global__ void k_gram_final(const double* __restrict__ part, int nblocks, double* __restrict__ G) {
  const int q = threadIdx.x;
  if (q >= 64) return;
  double s = 0.0;
  for (int b = 0; b < nblocks; ++b) s += part[(long long)b * 64 + q];
  G[q] = s;
}

// G (64 doubles, row-major 8 x 8, entry [i*8+j] = A_i . B_j) on the device.
void block_gram(long long n, const double* const* A, int na, const double* const* B, int nb, double* part,
                double* G, cudaStream_t s) {
  if (na < 1 || na > 8 || nb < 1 || nb > 8) throw std::invalid_argument("block_gram: 1..8 columns");
  ColPtrs ca{}, cb{};
  for (int i = 0; i < na; ++i) ca.p[i] = A[i];
  for (int j = 0; j < nb; ++j) cb.p[j] = B[j];
  k_gram<<<GRAM_BLOCKS, GRAM_THREADS, 0, s>>>(n, ca, na, cb, nb, part);
  TOPO_LAUNCH_CHECK();
  k_gram_final<<<1, 64, 0, s>>>(part, GRAM_BLOCKS, G);
  TOPO_LAUNCH_CHECK();
}

size_t block_gram_partials() { return (size_t)GRAM_BLOCKS * 64; }

struct Coef {
  double m[64];  // M[i][j] at i*8+j
};

// Out_j = C_j + sign * sum_i In_i M[i][j]; Out may alias C, not In.
__global__ void k_block_combine(long long n, ColPtrs In, int ni, ColPtrs Cc, ColOut Out, int no, Coef M, double sign) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
    double a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = i < ni ? In.p[i][r] : 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (j >= no) break;
      double v = 0.0;
#pragma unroll
      for (int i = 0; i < 8; ++i) v += a[i] * M.m[i * 8 + j];
      Out.p[j][r] = (Cc.p[j] != nullptr ? Cc.p[j][r] : 0.0) + sign * v;
    }
  }
}

void block_combine(long long n, const double* const* In, int ni, const double* const* Cc, double* const* Out, int no,
                   const double* M, double sign, cudaStream_t s) {
  if (ni < 1 || ni > 8 || no < 1 || no > 8) throw std::invalid_argument("block_combine: 1..8 columns");
  ColPtrs ci{}, cc{};
  ColOut co{};
  Coef m{};
  for (int i = 0; i < ni; ++i) ci.p[i] = In[i];
  for (int j = 0; j < no; ++j) {
    cc.p[j] = Cc ? Cc[j] : nullptr;
    co.p[j] = Out[j];
  }
  for (int q = 0; q < 64; ++q) m.m[q] = M[q];
  k_block_combine<<<kRedBlocks, 256, 0, s>>>(n, ci, ni, cc, co, no, m, sign);
  TOPO_LAUNCH_CHECK();
}

}  // namespace topo
