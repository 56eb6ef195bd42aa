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
// (multigrid_v4.py:747-751). One thread per coarse node I walks the fine nodes
// i of its support (weight P[i,I]), their 27 stencil neighbours j, and the
// coarse parents J of j, accumulating w_i * w_jJ * K_f[i,j] into block J-I.
__global__ void k_rap(Grid f, Grid c, const double* __restrict__ Sf, const uint8_t* __restrict__ mc,
                      double* __restrict__ Sc) {
  const long long I = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (I >= c.nnodes) return;
  int Ix, Iy, Iz;
  node_xyz(c, I, Ix, Iy, Iz);
  double acc[27 * 9];
  for (int q = 0; q < 27 * 9; ++q) acc[q] = 0.0;
  for (int sx = -1; sx <= 1; ++sx) {
    const int ix = 2 * Ix + sx;
    if (ix < 0 || ix > f.nx) continue;
    const double wx = prolong_w1(ix, Ix, c.nx);
    if (wx == 0.0) continue;
    for (int sy = -1; sy <= 1; ++sy) {
      const int iy = 2 * Iy + sy;
      if (iy < 0 || iy > f.ny) continue;
      const double wy = prolong_w1(iy, Iy, c.ny);
      if (wy == 0.0) continue;
      for (int sz = -1; sz <= 1; ++sz) {
        const int iz = 2 * Iz + sz;
        if (iz < 0 || iz > f.nz) continue;
        const double wz = prolong_w1(iz, Iz, c.nz);
        if (wz == 0.0) continue;
        const double wi = wx * wy * wz;
        const long long i = ((long long)ix * f.NY + iy) * f.NZ + iz;
        for (int kt = 0; kt < 27; ++kt) {
          const int jx = ix + kt / 9 - 1, jy = iy + (kt / 3) % 3 - 1, jz = iz + kt % 3 - 1;
          if (jx < 0 || jx > f.nx || jy < 0 || jy > f.ny || jz < 0 || jz > f.nz) continue;
          double K[9];
          bool any = false;
#pragma unroll
          for (int q = 0; q < 9; ++q) {
            K[q] = Sf[(long long)(kt * 9 + q) * f.nnodes + i];
            any |= (K[q] != 0.0);
          }
          if (!any) continue;
          const int px0 = jx >> 1, px1 = (jx & 1) ? px0 + 1 : px0;
          const int py0 = jy >> 1, py1 = (jy & 1) ? py0 + 1 : py0;
          const int pz0 = jz >> 1, pz1 = (jz & 1) ? pz0 + 1 : pz0;
          for (int Jx = px0; Jx <= px1; ++Jx) {
            if (Jx > c.nx) continue;
            const double vx = prolong_w1(jx, Jx, c.nx);
            if (vx == 0.0) continue;
            for (int Jy = py0; Jy <= py1; ++Jy) {
              if (Jy > c.ny) continue;
              const double vy = prolong_w1(jy, Jy, c.ny);
              if (vy == 0.0) continue;
              for (int Jz = pz0; Jz <= pz1; ++Jz) {
                if (Jz > c.nz) continue;
                const double vz = prolong_w1(jz, Jz, c.nz);
                if (vz == 0.0) continue;
                const double w = wi * vx * vy * vz;
                const int kd = (Jx - Ix + 1) * 9 + (Jy - Iy + 1) * 3 + (Jz - Iz + 1);
#pragma unroll
                for (int q = 0; q < 9; ++q) acc[kd * 9 + q] += w * K[q];
              }
            }
          }
        }
      }
    }
  }
  for (int k = 0; k < 27; ++k) {
    const int jx = Ix + k / 9 - 1, jy = Iy + (k / 3) % 3 - 1, jz = Iz + k % 3 - 1;
    const bool jin = jx >= 0 && jx < c.NX && jy >= 0 && jy < c.NY && jz >= 0 && jz < c.NZ;
    const long long J = jin ? (((long long)jx * c.NY + jy) * c.NZ + jz) : 0;
#pragma unroll
    for (int cc = 0; cc < 3; ++cc)
#pragma unroll
      for (int dd = 0; dd < 3; ++dd) {
        const bool keep = jin && mc[3 * I + cc] && mc[3 * J + dd];
        Sc[(long long)(k * 9 + cc * 3 + dd) * c.nnodes + I] = keep ? acc[k * 9 + cc * 3 + dd] : 0.0;
      }
  }
}

void rap(const Grid& fine, const Grid& coarse, const double* S_f, const uint8_t* mask_c, double* S_c,
         cudaStream_t s) {
  const int bs = 64;
  k_rap<<<(unsigned)((coarse.nnodes + bs - 1) / bs), bs, 0, s>>>(fine, coarse, S_f, mask_c, S_c);
  TOPO_LAUNCH_CHECK();
}

// ------------------------------------------------------------- stencil apply
template <typename TC>
__device__ __forceinline__ float coef_f(const TC* p) {
  if constexpr (sizeof(TC) == 2) return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(p));
  else return (float)*p;
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
    const long long j = rb[k / 3] + jzs[k % 3];
    T uj[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      T v = u[3 * j + d];
      if constexpr (BF) v = __bfloat162float(__float2bfloat16_rn((float)v));
      uj[d] = v;
    }
    const TC* Sk = S + (long long)(k * 9) * g.nnodes + n;
    T s[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      if constexpr (sizeof(TC) == 8) s[q] = (T)Sk[(long long)q * g.nnodes];
      else s[q] = (T)coef_f(Sk + (long long)q * g.nnodes);
    }
    a0 += s[0] * uj[0] + s[1] * uj[1] + s[2] * uj[2];
    a1 += s[3] * uj[0] + s[4] * uj[1] + s[5] * uj[2];
    a2 += s[6] * uj[0] + s[7] * uj[1] + s[8] * uj[2];
  }
  const T acc[3] = {a0, a1, a2};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const long long i = 3 * n + c;
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

__global__ void k_convert(long long n, const double* __restrict__ S, float* __restrict__ S32,
                          __nv_bfloat16* __restrict__ S16) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = S[i];
    if (S32) S32[i] = (float)v;
    if (S16) S16[i] = __float2bfloat16_rn((float)v);
  }
}

void stencil_convert(long long n, const double* S, float* S32, __nv_bfloat16* S16, cudaStream_t s) {
  k_convert<<<1184, 256, 0, s>>>(n, S, S32, S16);
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

// ------------------------------------------------------------ coarsest level
// Dense FP64 system over the free DoFs of the coarsest grid (dof_index maps a
// full-vector DoF to its compact row, -1 when fixed).
__global__ void k_dense_assemble(Grid g, const double* __restrict__ S, const int* __restrict__ dof_index, int n,
                                 double* __restrict__ A) {
  const long long I = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (I >= g.nnodes) return;
  int ix, iy, iz;
  node_xyz(g, I, ix, iy, iz);
  for (int c = 0; c < 3; ++c) {
    const int row = dof_index[3 * I + c];
    if (row < 0) continue;
    for (int k = 0; k < 27; ++k) {
      const int jx = ix + k / 9 - 1, jy = iy + (k / 3) % 3 - 1, jz = iz + k % 3 - 1;
      if (jx < 0 || jx >= g.NX || jy < 0 || jy >= g.NY || jz < 0 || jz >= g.NZ) continue;
      const long long J = ((long long)jx * g.NY + jy) * g.NZ + jz;
      for (int d = 0; d < 3; ++d) {
        const int col = dof_index[3 * J + d];
        if (col < 0) continue;
        A[(long long)row * n + col] = S[(long long)(k * 9 + c * 3 + d) * g.nnodes + I];
      }
    }
  }
}

void dense_assemble(const Grid& g, const double* S, const int* dof_index, int n, double* A, cudaStream_t s) {
  TOPO_CUDA_CHECK(cudaMemsetAsync(A, 0, sizeof(double) * (size_t)n * n, s));
  const int bs = 128;
  k_dense_assemble<<<(unsigned)((g.nnodes + bs - 1) / bs), bs, 0, s>>>(g, S, dof_index, n, A);
  TOPO_LAUNCH_CHECK();
}

// Banded right-looking Cholesky on dense row-major storage, panel width CNB.
// The band half-width `band` bounds every non-zero (|i-j| <= band), and the
// factor keeps the same band, so only that window is touched. The factored
// diagonal blocks go to a side array Dt (one CNB x CNB lower block per panel,
// identity-padded past n); the off-diagonal band of L overwrites A's lower
// part. A's diagonal blocks keep their updated, unfactored values and are not
// read as L afterwards.
constexpr int CNB = 32;

// One panel step. Every CTA factors the (k,k) block in one warp's registers
// (the same arithmetic in each, so all agree): per pivot j the trailing
// entries take W[i][c] -= W[c][j] (W[i][j] / d) while column j itself is only
// read, and its scaled values (sqrt(d) on the diagonal, W[i][j] * rsqrt(d)
// below) go to a separate output block L in shared memory. CTA 0
// stores L in Dt and raises `flag` on a non-positive or non-finite pivot (the
// pivot is then taken as 1). The block is identity-padded past n, so every
// loop below runs over the full 32 without predicates. Each thread then
// solves one panel row i in [k+nb, min(n, k+nb+band)), L_ik L_kk^T = A_ik,
// column by column with the reciprocal diagonal.
__global__ void __launch_bounds__(128) k_chol_step(int n, int k, int band, double* __restrict__ A,
                                                   double* __restrict__ Dt, int* __restrict__ flag) {
  __shared__ double W[CNB][CNB + 1];
  __shared__ double L[CNB][CNB + 1];
  __shared__ double invd[CNB];
  const int nb = min(CNB, n - k);
  const int tid = threadIdx.x;
  for (int q = tid; q < CNB * CNB; q += blockDim.x) {
    const int i = q / CNB, j = q % CNB;
    W[i][j] = (i < nb && j < nb && j <= i) ? A[(long long)(k + i) * n + k + j] : (i == j ? 1.0 : 0.0);
  }
  __syncthreads();
  // warp 0 factors with lane r holding row r of the block in registers
  // (wr[t] = W[r][t], t <= r). Per pivot j (fully unrolled, so register
  // indices are compile-time): every lane takes d = W[j][j] from lane j by a
  // shuffle and evaluates rsqrt(d) itself, its own multiplier W[r][j] / d is
  // local, and the column entries W[t][j] arrive by shuffles from lanes t and
  // are consumed at once: W[r][t] -= W[t][j] W[r][j] / d for j < t <= r. No
  // shared memory and no warp barrier on the pivot chain.
  bool bad = false;
  if (tid < 32) {
    const int lane = tid;
    double wr[CNB];
#pragma unroll
    for (int t = 0; t < CNB; ++t) wr[t] = W[lane][t];
#pragma unroll
    for (int j = 0; j < CNB; ++j) {
      const double d = __shfl_sync(0xffffffffu, wr[j], j);
      const bool ok = d > 0.0 && isfinite(d);
      const double dd = ok ? d : 1.0;
      const double rs = rsqrt(dd);
      const double lj = wr[j];
      if (lane == j) {
        bad |= !ok;
        L[j][j] = dd * rs;
        invd[j] = rs;
      } else {
        L[lane][j] = lane > j ? lj * rs : 0.0;
      }
      const double w = lj * (rs * rs);
#pragma unroll
      for (int t = j + 1; t < CNB; ++t) {
        const double ct = __shfl_sync(0xffffffffu, wr[j], t);
        if (t <= lane) wr[t] -= ct * w;
      }
    }
    bad = __any_sync(0xffffffffu, bad);
  }
  __syncthreads();
  if (blockIdx.x == 0) {
    double* D = Dt + (long long)(k / CNB) * CNB * CNB;
    for (int q = tid; q < CNB * CNB; q += blockDim.x) D[q] = (q % CNB <= q / CNB) ? L[q / CNB][q % CNB] : 0.0;
    if (tid == 0 && bad) *flag = 1;
  }
  const int i = k + nb + blockIdx.x * blockDim.x + tid;
  if (i >= n || i >= k + nb + band) return;
  double x[CNB];
  double* row = A + (long long)i * n + k;
#pragma unroll
  for (int j = 0; j < CNB; ++j) x[j] = (j < nb) ? row[j] : 0.0;
#pragma unroll
  for (int j = 0; j < CNB; ++j) {
    x[j] *= invd[j];
#pragma unroll
    for (int t = j + 1; t < CNB; ++t) x[t] -= x[j] * L[t][j];
  }
#pragma unroll
  for (int j = 0; j < CNB; ++j)
    if (j < nb) row[j] = x[j];
}

// Trailing update A[i][j] -= sum_t L[i][t] L[j][t] over the panel, for
// k+nb <= j <= i < k+nb+band and i-j <= band. One CTA per lower-triangular
// 32x32 tile (blockIdx.x enumerates them row by row), 256 threads, four
// outputs per thread.
__global__ void __launch_bounds__(256) k_chol_update(int n, int k, int band, double* __restrict__ A) {
  const int nb = min(CNB, n - k);
  const int base = k + nb;
  const int lim = min(n, base + band);
  // tile (ti, tj), tj <= ti, from the linear index
  int ti = (int)((sqrt(8.0 * blockIdx.x + 1.0) - 1.0) * 0.5);
  while ((ti + 1) * (ti + 2) / 2 <= (int)blockIdx.x) ++ti;
  while (ti * (ti + 1) / 2 > (int)blockIdx.x) --ti;
  const int tj = blockIdx.x - ti * (ti + 1) / 2;
  const int i0 = base + 32 * ti, j0 = base + 32 * tj;
  if (i0 - (j0 + 31) > band) return;  // whole tile outside the band
  __shared__ double Li[32][CNB + 1], Lj[32][CNB + 1];
  for (int q = threadIdx.x; q < 32 * CNB; q += 256) {
    const int r = q / CNB, t = q % CNB;
    Li[r][t] = (i0 + r < lim && t < nb) ? A[(long long)(i0 + r) * n + k + t] : 0.0;
    Lj[r][t] = (j0 + r < lim && t < nb) ? A[(long long)(j0 + r) * n + k + t] : 0.0;
  }
  __syncthreads();
  const int r = threadIdx.x >> 3, c0 = (threadIdx.x & 7) * 4;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
  for (int t = 0; t < CNB; ++t) {
    const double li = Li[r][t];
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = fma(li, Lj[c0 + q][t], acc[q]);
  }
  const int i = i0 + r;
  if (i >= lim) return;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int j = j0 + c0 + q;
    if (j < lim && j <= i && i - j <= band) A[(long long)i * n + j] -= acc[q];
  }
}

// Inverse of every factored diagonal block (identity-padded, so the last
// partial block inverts cleanly): thread j forms column j by forward
// substitution.
__global__ void k_block_tri_inv(const double* __restrict__ Dt, double* __restrict__ Di) {
  __shared__ double L[CNB][CNB + 1];
  __shared__ double X[CNB][CNB + 1];
  const long long base = (long long)blockIdx.x * CNB * CNB;
  for (int q = threadIdx.x; q < CNB * CNB; q += blockDim.x) L[q / CNB][q % CNB] = Dt[base + q];
  __syncthreads();
  const int j = threadIdx.x;
  for (int i = 0; i < CNB; ++i) {
    double v = (i == j) ? 1.0 : 0.0;
    for (int m = j; m < i; ++m) v -= L[i][m] * X[m][j];
    X[i][j] = v / L[i][i];
  }
  __syncthreads();
  for (int q = threadIdx.x; q < CNB * CNB; q += blockDim.x) Di[base + q] = X[q / CNB][q % CNB];
}

// W = L^-1 by forward substitution, one strip of TWC columns per CTA. Every
// column of W is an independent forward substitution, so the strips need no
// communication: CTA J owns columns [TWC J, TWC J + TWC) and walks the
// CNB-row blocks I from the one holding its first column to the last:
//   R    = E - sum_{k in [max(j0, 32I-band), 32I)} L[32I.., k] W[k, strip]
//   W_I  = Di_I R                    (E: the identity on these rows/columns)
// Every W read is of rows this CTA wrote in an earlier step (visible after
// __syncthreads). The strip of column 0 is the critical path (nT steps), so
// strips are narrower than a row block (16 columns; 32 and 8 measured
// slower): a step is mostly the latency of its L reads, which come from L2
// (all strips at block row I read the same L rows), in 64-wide chunks with
// the next chunk prefetched into registers.
// Warp w takes the chunk rows k = w, w+8, ...; lane r keeps row r of the
// 32 x TWC partial product and reads the W row as broadcast loads; the 8 warp
// partials are summed through shared memory.
// W goes to W64 (lower part, FP64) and to the apply matrices C64 / C32 as W
// in the lower triangle and W^T in the strict upper triangle, all with row
// stride ldc.
constexpr int TIT = 256, TKC = 64, TWC = 16;
struct TriSmem {
  double Ls[CNB][TKC + 1];
  double Wc[TKC][TWC];
  double red[TIT / 32][CNB][TWC + 1];
  double Rs[CNB][TWC + 1];
  double Ds[CNB][CNB + 1];
};
constexpr size_t TRI_SMEM = sizeof(TriSmem);

__global__ void __launch_bounds__(TIT) k_tri_inverse(int n, int band, const double* __restrict__ L,
                                                     const double* __restrict__ Di, double* W64, long long ldc,
                                                     double* C64, float* C32) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TriSmem& S = *reinterpret_cast<TriSmem*>(smem_raw);
  const int nT = (n + CNB - 1) / CNB;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int j0 = blockIdx.x * TWC;
  if (j0 >= n) return;  // uniform over the CTA
  constexpr int PL = CNB * TKC / TIT;  // L values fetched per thread per chunk
  constexpr int PW = TKC * TWC / TIT;  // W values fetched per thread per chunk
  constexpr int PO = CNB * TWC / TIT;  // outputs per thread per step
  static_assert(PL * TIT == CNB * TKC && PW * TIT == TKC * TWC && PO * TIT == CNB * TWC, "tile split");
  double pl[PL], pw[PW];
  for (int I = j0 / CNB; I < nT; ++I) {
    const int i0 = I * CNB;
    const int klo = max(j0, i0 - band);
    auto fetch = [&](int k0) {
#pragma unroll
      for (int m = 0; m < PL; ++m) {
        const int q = t + TIT * m;
        const int i = i0 + q / TKC, k = k0 + q % TKC;
        pl[m] = (i < n && k < i0) ? L[(long long)i * n + k] : 0.0;
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
        const double a = S.Ls[lane][kk];
        const double2* wr = reinterpret_cast<const double2*>(&S.Wc[kk][0]);
#pragma unroll
        for (int c2 = 0; c2 < TWC / 2; ++c2) {
          const double2 w = wr[c2];
          acc[2 * c2] = fma(a, w.x, acc[2 * c2]);
          acc[2 * c2 + 1] = fma(a, w.y, acc[2 * c2 + 1]);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < TWC; ++c) S.red[warp][lane][c] = acc[c];
    for (int q = t; q < CNB * CNB; q += TIT) S.Ds[q >> 5][q & 31] = Di[(long long)I * CNB * CNB + q];
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
    if (C64 != nullptr || C32 != nullptr) {
      for (int q = t; q < TWC * CNB; q += TIT) {
        const int cr = j0 + q / CNB, ic = i0 + q % CNB;
        if (cr < n && ic < n && ic > cr) {
          const double v = S.Rs[q % CNB][q / CNB];
          if (C64 != nullptr) C64[(long long)cr * ldc + ic] = v;
          if (C32 != nullptr) C32[(long long)cr * ldc + ic] = (float)v;
        }
      }
    }
    __syncthreads();
  }
}

void dense_cholesky_launch(int n, int band, double* A, double* Dt, int* flag, cudaStream_t s) {
  TOPO_CUDA_CHECK(cudaMemsetAsync(flag, 0, sizeof(int), s));
  for (int k = 0; k < n; k += CNB) {
    const int nb = std::min(CNB, n - k);
    const int rows = std::min(n - (k + nb), band);
    k_chol_step<<<std::max(1, (rows + 127) / 128), 128, 0, s>>>(n, k, band, A, Dt, flag);
    TOPO_LAUNCH_CHECK();
    if (rows > 0) {
      const int nt = (rows + 31) / 32;
      k_chol_update<<<nt * (nt + 1) / 2, 256, 0, s>>>(n, k, band, A);
      TOPO_LAUNCH_CHECK();
    }
  }
}

int dense_cholesky(int n, int band, double* A, double* Dt, int* flag, cudaStream_t s) {
  dense_cholesky_launch(n, band, A, Dt, flag, s);
  int h_flag = 0;
  TOPO_CUDA_CHECK(cudaMemcpyAsync(&h_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
  return h_flag ? 1 : 0;
}

void dense_inverse_factor(int n, int band, const double* A, const double* Dt, double* Di, double* W64, long long ldc,
                          double* C64, float* C32, cudaStream_t s) {
  const int nT = (n + CNB - 1) / CNB;
  k_block_tri_inv<<<nT, CNB, 0, s>>>(Dt, Di);
  TOPO_LAUNCH_CHECK();
  k_tri_inverse<<<(n + TWC - 1) / TWC, TIT, TRI_SMEM, s>>>(n, band, A, Di, W64, ldc, C64, C32);
  TOPO_LAUNCH_CHECK();
}

// Coarsest solve z = W^T (W r) = K^-1 r with W = L^-1, in two passes over the
// combined matrix C (W below and on the diagonal, W^T above): pass one
// y = W r_c (row i reads C[i][0..i]), pass two z_c = W^T y (row j reads
// C[j][j..n-1]). One warp per row, 16-byte loads (rows are padded to ldc, a
// multiple of 32 elements, so every row starts 16-byte aligned), two loads in
// flight per lane, FP64 accumulation. The compact right-hand side is gathered
// once (k_coarse_gather) and both passes read the compact vectors straight
// from global memory: they are n doubles, which every SM keeps in L1, so no
// block spends its first microseconds staging them.
template <typename T>
__global__ void k_coarse_gather(int n, const int* __restrict__ free_list, const T* __restrict__ rhs,
                                double* __restrict__ rc, const KrylovState* st) {
  if (st != nullptr && st->done) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) rc[j] = (double)rhs[free_list[j]];
}

template <typename TX>
__global__ void __launch_bounds__(256) k_coarse_lower(int n, long long ldc, const TX* __restrict__ C,
                                                      const double* __restrict__ rc, double* __restrict__ y,
                                                      const KrylovState* st) {
  if (st != nullptr && st->done) return;
  const int row = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (row >= n) return;
  constexpr int V = 16 / sizeof(TX);
  const TX* Ci = C + (long long)row * ldc;
  double acc = 0.0;
  int j = lane * V;
  for (; j + 32 * V <= row; j += 64 * V) {  // two 16-byte loads in flight
    TX v[V], w[V];
    *reinterpret_cast<uint4*>(v) = __ldg(reinterpret_cast<const uint4*>(Ci + j));
    const bool two = j + 32 * V <= row;
    if (two) *reinterpret_cast<uint4*>(w) = __ldg(reinterpret_cast<const uint4*>(Ci + j + 32 * V));
#pragma unroll
    for (int q = 0; q < V; ++q) acc += (double)v[q] * __ldg(rc + j + q);
    if (two) {
#pragma unroll
      for (int q = 0; q < V; ++q)
        if (j + 32 * V + q <= row) acc += (double)w[q] * __ldg(rc + j + 32 * V + q);
    }
  }
  for (; j <= row; j += 32 * V) {
    TX v[V];
    *reinterpret_cast<uint4*>(v) = __ldg(reinterpret_cast<const uint4*>(Ci + j));
#pragma unroll
    for (int q = 0; q < V; ++q)
      if (j + q <= row) acc += (double)v[q] * __ldg(rc + j + q);
  }
  acc = warp_sum(acc);
  if (lane == 0) y[row] = acc;
}

template <typename T, typename TX>
__global__ void __launch_bounds__(256) k_coarse_upper(int n, long long ldc, const TX* __restrict__ C,
                                                      const int* __restrict__ free_list,
                                                      const double* __restrict__ y, T* __restrict__ x,
                                                      const KrylovState* st) {
  if (st != nullptr && st->done) return;
  const int row = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (row >= n) return;
  constexpr int V = 16 / sizeof(TX);
  const TX* Cj = C + (long long)row * ldc;
  double acc = 0.0;
  int i = (row / V) * V + lane * V;
  for (; i + 32 * V < n; i += 64 * V) {  // two 16-byte loads in flight
    TX v[V], w[V];
    *reinterpret_cast<uint4*>(v) = __ldg(reinterpret_cast<const uint4*>(Cj + i));
    const bool two = i + 32 * V < n;
    if (two) *reinterpret_cast<uint4*>(w) = __ldg(reinterpret_cast<const uint4*>(Cj + i + 32 * V));
#pragma unroll
    for (int q = 0; q < V; ++q)
      if (i + q >= row) acc += (double)v[q] * __ldg(y + i + q);
    if (two) {
#pragma unroll
      for (int q = 0; q < V; ++q)
        if (i + 32 * V + q < n) acc += (double)w[q] * __ldg(y + i + 32 * V + q);
    }
  }
  for (; i < n; i += 32 * V) {
    TX v[V];
    *reinterpret_cast<uint4*>(v) = __ldg(reinterpret_cast<const uint4*>(Cj + i));
#pragma unroll
    for (int q = 0; q < V; ++q)
      if (i + q >= row && i + q < n) acc += (double)v[q] * __ldg(y + i + q);
  }
  acc = warp_sum(acc);
  if (lane == 0) x[free_list[row]] = (T)acc;
}

// The tri-inverse kernel stages column panels in shared memory beyond 48 KB.
void dense_apply_prepare(int n) {
  (void)n;
  TOPO_CUDA_CHECK(cudaFuncSetAttribute(k_tri_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRI_SMEM));
}

// work: 2n doubles (y, then the compact right-hand side).
void dense_apply(bool vec64, int n, long long ldc, const double* C64, const float* C32, const int* free_list,
                 const void* rhs, double* work, void* x, const KrylovState* st, cudaStream_t s) {
  const int wpb = 8;
  const unsigned nb = (unsigned)((n + wpb - 1) / wpb);
  double* y = work;
  double* rc = work + n;
  const unsigned ng = (unsigned)((n + 255) / 256);
  if (vec64) {
    k_coarse_gather<double><<<ng, 256, 0, s>>>(n, free_list, (const double*)rhs, rc, st);
    TOPO_LAUNCH_CHECK();
    k_coarse_lower<double><<<nb, 32 * wpb, 0, s>>>(n, ldc, C64, rc, y, st);
    TOPO_LAUNCH_CHECK();
    k_coarse_upper<double, double><<<nb, 32 * wpb, 0, s>>>(n, ldc, C64, free_list, y, (double*)x, st);
  } else {
    k_coarse_gather<float><<<ng, 256, 0, s>>>(n, free_list, (const float*)rhs, rc, st);
    TOPO_LAUNCH_CHECK();
    k_coarse_lower<float><<<nb, 32 * wpb, 0, s>>>(n, ldc, C32, rc, y, st);
    TOPO_LAUNCH_CHECK();
    k_coarse_upper<float, float><<<nb, 32 * wpb, 0, s>>>(n, ldc, C32, free_list, y, (float*)x, st);
  }
  TOPO_LAUNCH_CHECK();
}

}  // namespace topo
