// coarse.cu - coarse multigrid levels on 27-point block stencils.
//
// Every coarse operator of the hierarchy is stored as a structured stencil:
// for node n and neighbour offset k = (dx+1)*9+(dy+1)*3+(dz+1), the 3x3 block
// coupling n to n+(dx,dy,dz) sits at S[(k*9 + c*3 + d) * nnodes + n]
// (coefficient-major, so consecutive threads read consecutive addresses).
// Rows and columns of fixed DoFs are zero. This replaces the reference's CSR
// matrices on compact free-DoF vectors (src/gpu_fem/multigrid_v4.py:132-270,
// 747-772) with no index arrays at all.
#include "internal.cuh"
#include "reduce.cuh"

#include <algorithm>
#include <stdexcept>
#include <vector>

namespace topo {

__constant__ double cQ[8 * 576];  // Q_stu = P24_stu^T KE P24_stu, stu = 4s+2t+u

void set_galerkin_q(const double* Q) { TOPO_CUDA_CHECK(cudaMemcpyToSymbol(cQ, Q, sizeof(double) * 8 * 576)); }

__host__ __device__ constexpr int corner_of(int bx, int by, int bz) {
  return bz * 4 + (by ? (bx ? 2 : 3) : (bx ? 1 : 0));
}

__device__ __forceinline__ void node_xyz(const Grid& g, long long n, int& ix, int& iy, int& iz) {
  iz = (int)(n % g.NZ);
  iy = (int)((n / g.NZ) % g.NY);
  ix = (int)(n / ((long long)g.NZ * g.NY));
}

// ------------------------------------------------------------ level-1 Galerkin
// Coarse element e contributes Kc_e = sum_stu E_f(2e+stu, clamped) Q_stu
// (multigrid_v4.py:182-203, 256). One thread per coarse node I gathers, for
// each neighbour J = I + delta, the 3x3 block sum over the coarse elements
// that contain both I and J.
__global__ void k_level1_assemble(Grid f, Grid c, const double* __restrict__ Ef, const uint8_t* __restrict__ mc,
                                  double* __restrict__ S) {
  const long long I = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (I >= c.nnodes) return;
  int ix, iy, iz;
  node_xyz(c, I, ix, iy, iz);
  for (int k = 0; k < 27; ++k) {
    const int dx = k / 9 - 1, dy = (k / 3) % 3 - 1, dz = k % 3 - 1;
    const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
    double B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const bool jin = jx >= 0 && jx < c.NX && jy >= 0 && jy < c.NY && jz >= 0 && jz < c.NZ;
    if (jin) {
      for (int ox = -1; ox <= 0; ++ox) {
        const int mx = dx - ox;
        if (mx < 0 || mx > 1) continue;
        const int ex = ix + ox;
        if (ex < 0 || ex >= c.nx) continue;
        for (int oy = -1; oy <= 0; ++oy) {
          const int my = dy - oy;
          if (my < 0 || my > 1) continue;
          const int ey = iy + oy;
          if (ey < 0 || ey >= c.ny) continue;
          for (int oz = -1; oz <= 0; ++oz) {
            const int mz = dz - oz;
            if (mz < 0 || mz > 1) continue;
            const int ez = iz + oz;
            if (ez < 0 || ez >= c.nz) continue;
            const int a = corner_of(-ox, -oy, -oz);
            const int m = corner_of(mx, my, mz);
            for (int stu = 0; stu < 8; ++stu) {
              const int s = stu >> 2, t = (stu >> 1) & 1, u = stu & 1;
              const int fx = min(2 * ex + s, f.nx - 1), fy = min(2 * ey + t, f.ny - 1), fz = min(2 * ez + u, f.nz - 1);
              const double Ee = Ef[((long long)fx * f.ny + fy) * f.nz + fz];
              const double* Q = cQ + stu * 576;
#pragma unroll
              for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                for (int dd = 0; dd < 3; ++dd) B[cc * 3 + dd] += Ee * Q[(3 * a + cc) * 24 + 3 * m + dd];
            }
          }
        }
      }
    }
    const long long J = jin ? (((long long)jx * c.NY + jy) * c.NZ + jz) : 0;
#pragma unroll
    for (int cc = 0; cc < 3; ++cc)
#pragma unroll
      for (int dd = 0; dd < 3; ++dd) {
        const bool keep = jin && mc[3 * I + cc] && mc[3 * J + dd];
        S[(long long)(k * 9 + cc * 3 + dd) * c.nnodes + I] = keep ? B[cc * 3 + dd] : 0.0;
      }
  }
}

void level1_assemble(const Grid& fine, const Grid& coarse, const double* E_f, const uint8_t* mask_c, double* S,
                     cudaStream_t s) {
  const int bs = 128;
  k_level1_assemble<<<(unsigned)((coarse.nnodes + bs - 1) / bs), bs, 0, s>>>(fine, coarse, E_f, mask_c, S);
  TOPO_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------- R.A.P
// K_c = P^T K_f P with the row-normalised trilinear P restricted to free DoFs
// (multigrid_v4.py:747-751). Block (I, J = I + d) of K_c is
//   sum_{i, j} P[i,I] P[j,J] K_f[i,j]
// over fine nodes i = 2I + s, j = 2J + t (s, t in {-1,0,1}^3) that are
// stencil neighbours (|j - i| <= 1 per dimension). Per dimension that leaves
// 7 (s, t) pairs for d = 0 and 3 for d = +-1. One thread per (I, d) keeps its
// 3x3 block in registers; threads of a warp share d (uniform loops) and take
// consecutive I.
struct PairList {
  int n;
  int s[7], t[7];
};

__host__ __device__ inline PairList rap_pairs(int d) {
  PairList p;
  p.n = 0;
  for (int s = -1; s <= 1; ++s)
    for (int t = -1; t <= 1; ++t) {
      const int gap = 2 * d + t - s;
      if (gap >= -1 && gap <= 1) {
        p.s[p.n] = s;
        p.t[p.n] = t;
        ++p.n;
      }
    }
  return p;
}

__global__ void __launch_bounds__(128) k_rap(Grid f, Grid c, const double* __restrict__ Sf, const uint8_t* __restrict__ mc,
                                             double* __restrict__ Sc) {
  // CTA b: neighbour offset kd = b % 27 (uniform per CTA) of coarse nodes
  // [128 (b / 27), +128); the 27 offsets of a node range are adjacent in
  // launch order, so they read that range's fine coefficients from L2
  const int kd = (int)(blockIdx.x % 27);
  const long long I = (long long)(blockIdx.x / 27) * blockDim.x + threadIdx.x;
  if (I >= c.nnodes) return;
  int Ix, Iy, Iz;
  node_xyz(c, I, Ix, Iy, Iz);
  const int dx = kd / 9 - 1, dy = (kd / 3) % 3 - 1, dz = kd % 3 - 1;
  const int Jx = Ix + dx, Jy = Iy + dy, Jz = Iz + dz;
  const bool jin = Jx >= 0 && Jx < c.NX && Jy >= 0 && Jy < c.NY && Jz >= 0 && Jz < c.NZ;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (jin) {
    const PairList px = rap_pairs(dx), py = rap_pairs(dy), pz = rap_pairs(dz);
    for (int a = 0; a < px.n; ++a) {
      const int ix = 2 * Ix + px.s[a], jx = 2 * Jx + px.t[a];
      if (ix < 0 || ix > f.nx || jx < 0 || jx > f.nx) continue;
      const double wx = prolong_w1(ix, Ix, c.nx) * prolong_w1(jx, Jx, c.nx);
      if (wx == 0.0) continue;
      for (int b = 0; b < py.n; ++b) {
        const int iy = 2 * Iy + py.s[b], jy = 2 * Jy + py.t[b];
        if (iy < 0 || iy > f.ny || jy < 0 || jy > f.ny) continue;
        const double wxy = wx * prolong_w1(iy, Iy, c.ny) * prolong_w1(jy, Jy, c.ny);
        if (wxy == 0.0) continue;
        for (int e = 0; e < pz.n; ++e) {
          const int iz = 2 * Iz + pz.s[e], jz = 2 * Jz + pz.t[e];
          if (iz < 0 || iz > f.nz || jz < 0 || jz > f.nz) continue;
          const double w = wxy * prolong_w1(iz, Iz, c.nz) * prolong_w1(jz, Jz, c.nz);
          if (w == 0.0) continue;
          const long long i = ((long long)ix * f.NY + iy) * f.NZ + iz;
          const int kt = (jx - ix + 1) * 9 + (jy - iy + 1) * 3 + (jz - iz + 1);
          const double* K = Sf + (long long)kt * 9 * f.nnodes + i;
#pragma unroll
          for (int q = 0; q < 9; ++q) acc[q] = fma(w, __ldg(K + (long long)q * f.nnodes), acc[q]);
        }
      }
    }
  }
  const long long J = jin ? (((long long)Jx * c.NY + Jy) * c.NZ + Jz) : 0;
#pragma unroll
  for (int cc = 0; cc < 3; ++cc)
#pragma unroll
    for (int dd = 0; dd < 3; ++dd) {
      const bool keep = jin && mc[3 * I + cc] && mc[3 * J + dd];
      Sc[(long long)(kd * 9 + cc * 3 + dd) * c.nnodes + I] = keep ? acc[cc * 3 + dd] : 0.0;
    }
}

void rap(const Grid& fine, const Grid& coarse, const double* S_f, const uint8_t* mask_c, double* S_c,
         cudaStream_t s) {
  const int bs = 128;
  k_rap<<<(unsigned)(27 * ((coarse.nnodes + bs - 1) / bs)), bs, 0, s>>>(fine, coarse, S_f, mask_c, S_c);
  TOPO_LAUNCH_CHECK();
}

// ------------------------------------------------------------- stencil apply
template <typename TC>
__device__ __forceinline__ float coef_f(const TC* p) {
  if constexpr (sizeof(TC) == 2) return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(p));
  else return (float)*p;
}

// Coefficients of block k of node n:
//  * FP64 (setup copy): S[(k*9 + q) * nnodes + n], q = c*3 + d;
//  * FP32 / BF16 (apply copies): packed per block, 12 slots (9 used) at
//    S[(k * nnodes + n) * 12 + q], so a block is three 16-byte (FP32) or
//    8-byte (BF16) vector loads and a warp reads 32 consecutive blocks.
constexpr int kPack = 12;

template <typename TC, typename T>
__device__ __forceinline__ void load_block(const TC* __restrict__ S, int k, long long n, long long nnodes, T (&s)[9]) {
  if constexpr (sizeof(TC) == 8) {
    const TC* Sk = S + (long long)(k * 9) * nnodes + n;
#pragma unroll
    for (int q = 0; q < 9; ++q) s[q] = (T)Sk[(long long)q * nnodes];
  } else if constexpr (sizeof(TC) == 4) {
    const float4* p = reinterpret_cast<const float4*>(S + ((long long)k * nnodes + n) * kPack);
    const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    s[0] = a.x; s[1] = a.y; s[2] = a.z; s[3] = a.w;
    s[4] = b.x; s[5] = b.y; s[6] = b.z; s[7] = b.w;
    s[8] = c.x;
  } else {
    const uint2* p = reinterpret_cast<const uint2*>(S + ((long long)k * nnodes + n) * kPack);
    const uint2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    const uint32_t w[6] = {a.x, a.y, b.x, b.y, c.x, c.y};
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const uint32_t h = (q & 1) ? (w[q >> 1] & 0xFFFF0000u) : (w[q >> 1] << 16);
      s[q] = (T)__uint_as_float(h);
    }
  }
}

// TC: stencil coefficient type; T: vector type; BF: round u to BF16.
template <typename TC, typename T, bool BF, Epi EPI>
__global__ void __launch_bounds__(128)
k_stencil(Grid g, const TC* __restrict__ S, const T* __restrict__ u, const uint8_t* __restrict__ mask,
          EpiDev<T> ep, const KrylovState* st) {
  if (st != nullptr && st->done) return;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= g.nnodes) return;
  int ix, iy, iz;
  node_xyz(g, n, ix, iy, iz);
  // clamped neighbour coordinates (out-of-grid couplings have zero
  // coefficients, so any in-grid value serves) and the nine row bases
  const int jxs[3] = {max(ix - 1, 0), ix, min(ix + 1, g.NX - 1)};
  const int jys[3] = {max(iy - 1, 0), iy, min(iy + 1, g.NY - 1)};
  const int jzs[3] = {max(iz - 1, 0), iz, min(iz + 1, g.NZ - 1)};
  long long rb[9];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) rb[a * 3 + b] = ((long long)jxs[a] * g.NY + jys[b]) * g.NZ;
  T a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    long long j = rb[k / 3] + jzs[k % 3];
    if (!topo_in_range(j, g.nnodes)) j = n;
    T uj[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      T v = u[3 * j + d];
      if constexpr (BF) v = __bfloat162float(__float2bfloat16_rn((float)v));
      uj[d] = v;
    }
    T s[9];
    load_block<TC, T>(S, k, n, g.nnodes, s);
    a0 += s[0] * uj[0] + s[1] * uj[1] + s[2] * uj[2];
    a1 += s[3] * uj[0] + s[4] * uj[1] + s[5] * uj[2];
    a2 += s[6] * uj[0] + s[7] * uj[1] + s[8] * uj[2];
  }
  const T acc[3] = {a0, a1, a2};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const long long i = 3 * n + c;
    if (!topo_in_range(i, g.ndof)) continue;
    epilogue_store<T, EPI>(ep, i, mask[i] != 0, acc[c], u[i]);
  }
}

template <typename TC, typename T, bool BF>
static void launch_stencil(const Grid& g, const void* S, const void* u, const uint8_t* mask, void* y, Epi epi,
                           const EpiArgs& ea, cudaStream_t s) {
  const int bs = 128;
  const unsigned nb = (unsigned)((g.nnodes + bs - 1) / bs);
  const TC* SS = (const TC*)S;
  const T* uu = (const T*)u;
  const EpiDev<T> ep = make_epi<T>(y, ea);
  switch (epi) {
    case Epi::Store:
      k_stencil<TC, T, BF, Epi::Store><<<nb, bs, 0, s>>>(g, SS, uu, mask, ep, ea.st);
      break;
    case Epi::Residual:
      k_stencil<TC, T, BF, Epi::Residual><<<nb, bs, 0, s>>>(g, SS, uu, mask, ep, ea.st);
      break;
    case Epi::ChebR:
      k_stencil<TC, T, BF, Epi::ChebR><<<nb, bs, 0, s>>>(g, SS, uu, mask, ep, ea.st);
      break;
    case Epi::RUpd:
      k_stencil<TC, T, BF, Epi::RUpd><<<nb, bs, 0, s>>>(g, SS, uu, mask, ep, ea.st);
      break;
    default:
      throw std::runtime_error("stencil_apply: unsupported epilogue");
  }
  TOPO_LAUNCH_CHECK();
}

void stencil_apply(Prec p, bool vec64, const Grid& g, const void* S, const void* u, const uint8_t* mask, void* y,
                   Epi epi, const EpiArgs& ea, cudaStream_t s) {
  if (vec64) {
    if (p != Prec::F64) throw std::runtime_error("stencil_apply: FP64 vectors need an FP64 stencil");
    launch_stencil<double, double, false>(g, S, u, mask, y, epi, ea, s);
  } else if (p == Prec::F32) {
    launch_stencil<float, float, false>(g, S, u, mask, y, epi, ea, s);
  } else if (p == Prec::BF16) {
    launch_stencil<__nv_bfloat16, float, true>(g, S, u, mask, y, epi, ea, s);
  } else {
    launch_stencil<double, float, false>(g, S, u, mask, y, epi, ea, s);
  }
}

// Jacobi inverse diagonal from the centre block (k = 13), with the
// reference's guard |d| <= 1e-12 -> 1 (multigrid_v4.py:269, 752).
__global__ void k_stencil_dinv(Grid g, const double* __restrict__ S, const uint8_t* __restrict__ mask,
                               double* __restrict__ d64, float* __restrict__ d32) {
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= g.nnodes) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double d = S[(long long)(13 * 9 + c * 3 + c) * g.nnodes + n];
    d = fabs(d) > 1e-12 ? d : 1.0;
    const double v = mask[3 * n + c] ? 1.0 / d : 0.0;
    if (d64) d64[3 * n + c] = v;
    if (d32) d32[3 * n + c] = (float)v;
  }
}

void stencil_dinv(const Grid& g, const double* S, const uint8_t* mask, double* dinv64, float* dinv32,
                  cudaStream_t s) {
  const int bs = 256;
  k_stencil_dinv<<<(unsigned)((g.nnodes + bs - 1) / bs), bs, 0, s>>>(g, S, mask, dinv64, dinv32);
  TOPO_LAUNCH_CHECK();
}

// FP64 setup stencil (coefficient-major) -> packed FP32 / BF16 apply copies.
__global__ void k_convert(long long nnodes, const double* __restrict__ S, float* __restrict__ S32,
                          __nv_bfloat16* __restrict__ S16) {
  const long long total = 27 * nnodes;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const long long k = t / nnodes, n = t - k * nnodes;
#pragma unroll
    for (int q = 0; q < kPack; ++q) {
      const double v = q < 9 ? S[(k * 9 + q) * nnodes + n] : 0.0;
      if (S32) S32[t * kPack + q] = (float)v;
      if (S16) S16[t * kPack + q] = __float2bfloat16_rn((float)v);
    }
  }
}

// nnodes: nodes of the level; the apply copies hold 27 * 12 * nnodes values.
void stencil_convert(long long nnodes, const double* S, float* S32, __nv_bfloat16* S16, cudaStream_t s) {
  k_convert<<<1184, 256, 0, s>>>(nnodes, S, S32, S16);
  TOPO_LAUNCH_CHECK();
}

// ----------------------------------------------------------------- transfers
// Coarse free set by injection, reproducing the reference's linear-index test
// (solver_v2.py:717-764): coarse node (I,J,K) reads fine node index
// 2I*(ny_f+1)*(nz_f+1) + 2J*(nz_f+1) + 2K; a DoF past the end is fixed.
__global__ void k_inject_mask(Grid f, Grid c, const uint8_t* __restrict__ mf, uint8_t* __restrict__ mc) {
  const long long I = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (I >= c.nnodes) return;
  int ix, iy, iz;
  node_xyz(c, I, ix, iy, iz);
  const long long fn = 2LL * ix * f.NY * f.NZ + 2LL * iy * f.NZ + 2LL * iz;
  for (int d = 0; d < 3; ++d) {
    const long long fd = 3 * fn + d;
    mc[3 * I + d] = (fd < f.ndof) ? mf[fd] : (uint8_t)0;
  }
}

void inject_mask(const Grid& fine, const Grid& coarse, const uint8_t* mf, uint8_t* mc, cudaStream_t s) {
  const int bs = 256;
  k_inject_mask<<<(unsigned)((coarse.nnodes + bs - 1) / bs), bs, 0, s>>>(fine, coarse, mf, mc);
  TOPO_LAUNCH_CHECK();
}

// r_c = mask_c * P^T r_f
template <typename T>
__global__ void k_restrict(Grid f, Grid c, const T* __restrict__ rf, const uint8_t* __restrict__ mc,
                           T* __restrict__ rc, const KrylovState* st) {
  if (st != nullptr && st->done) return;
  const long long I = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (I >= c.nnodes) return;
  int Ix, Iy, Iz;
  node_xyz(c, I, Ix, Iy, Iz);
  T a[3] = {0, 0, 0};
  for (int sx = -1; sx <= 1; ++sx) {
    const int ix = 2 * Ix + sx;
    if (ix < 0 || ix > f.nx) continue;
    const T wx = (T)prolong_w1(ix, Ix, c.nx);
    if (wx == (T)0) continue;
    for (int sy = -1; sy <= 1; ++sy) {
      const int iy = 2 * Iy + sy;
      if (iy < 0 || iy > f.ny) continue;
      const T wy = (T)prolong_w1(iy, Iy, c.ny);
      if (wy == (T)0) continue;
      for (int sz = -1; sz <= 1; ++sz) {
        const int iz = 2 * Iz + sz;
        if (iz < 0 || iz > f.nz) continue;
        const T wz = (T)prolong_w1(iz, Iz, c.nz);
        if (wz == (T)0) continue;
        const T w = wx * wy * wz;
        const long long i = ((long long)ix * f.NY + iy) * f.NZ + iz;
        if (!topo_in_range(i, f.nnodes)) continue;
        a[0] += w * rf[3 * i];
        a[1] += w * rf[3 * i + 1];
        a[2] += w * rf[3 * i + 2];
      }
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) rc[3 * I + d] = mc[3 * I + d] ? a[d] : (T)0;
}

void restrict_vec(bool vec64, const Grid& fine, const Grid& coarse, const void* rf, const uint8_t* mc, void* rc,
                  const KrylovState* st, cudaStream_t s) {
  const int bs = 128;
  const unsigned nb = (unsigned)((coarse.nnodes + bs - 1) / bs);
  if (vec64)
    k_restrict<double><<<nb, bs, 0, s>>>(fine, coarse, (const double*)rf, mc, (double*)rc, st);
  else
    k_restrict<float><<<nb, bs, 0, s>>>(fine, coarse, (const float*)rf, mc, (float*)rc, st);
  TOPO_LAUNCH_CHECK();
}

// x_f += mask_f * P e_c
template <typename T>
__global__ void k_prolong_add(Grid f, Grid c, const T* __restrict__ ec, const uint8_t* __restrict__ mf,
                              T* __restrict__ xf, T* __restrict__ e_out, const KrylovState* st) {
  if (st != nullptr && st->done) return;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= f.nnodes) return;
  int ix, iy, iz;
  node_xyz(f, i, ix, iy, iz);
  T a[3] = {0, 0, 0};
  const int px0 = ix >> 1, px1 = (ix & 1) ? px0 + 1 : px0;
  const int py0 = iy >> 1, py1 = (iy & 1) ? py0 + 1 : py0;
  const int pz0 = iz >> 1, pz1 = (iz & 1) ? pz0 + 1 : pz0;
  for (int Jx = px0; Jx <= min(px1, c.nx); ++Jx) {
    const T wx = (T)prolong_w1(ix, Jx, c.nx);
    for (int Jy = py0; Jy <= min(py1, c.ny); ++Jy) {
      const T wy = (T)prolong_w1(iy, Jy, c.ny);
      for (int Jz = pz0; Jz <= min(pz1, c.nz); ++Jz) {
        const T w = wx * wy * (T)prolong_w1(iz, Jz, c.nz);
        const long long J = ((long long)Jx * c.NY + Jy) * c.NZ + Jz;
        if (!topo_in_range(J, c.nnodes)) continue;
        a[0] += w * ec[3 * J];
        a[1] += w * ec[3 * J + 1];
        a[2] += w * ec[3 * J + 2];
      }
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const T v = mf[3 * i + d] ? a[d] : (T)0;
    xf[3 * i + d] += v;
    if (e_out) e_out[3 * i + d] = v;
  }
}

void prolong_add(bool vec64, const Grid& fine, const Grid& coarse, const void* ec, const uint8_t* mf, void* xf,
                 void* e_out, const KrylovState* st, cudaStream_t s) {
  const int bs = 128;
  const unsigned nb = (unsigned)((fine.nnodes + bs - 1) / bs);
  if (vec64)
    k_prolong_add<double><<<nb, bs, 0, s>>>(fine, coarse, (const double*)ec, mf, (double*)xf, (double*)e_out, st);
  else
    k_prolong_add<float><<<nb, bs, 0, s>>>(fine, coarse, (const float*)ec, mf, (float*)xf, (float*)e_out, st);
  TOPO_LAUNCH_CHECK();
}

TOPO_BOUNDS_READER(bounds_flag_coarse)

}  // namespace topo
