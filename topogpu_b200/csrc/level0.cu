// level0.cu - level-0 (fine grid) matrix-free hex8 operator on CUDA cores,
// its diagonal, the SIMP modulus and the element-energy sensitivity.
//
// The operator is node-centric and owner-computes: one thread produces the
// three outputs of one node by summing E_e * KE[rows of the node, :] u_e over
// the (up to) eight elements around it. A thread block stages the nodal
// values of its brick plus a one-node halo, and the moduli of the elements
// touching the brick, in shared memory. Every output is written once by its
// owner: no atomics, deterministic results, no pre-zeroed output. KE lives in
// constant memory and every loop is unrolled, so the 576 multiply-adds per
// node take their KE factor as a constant-bank operand.
//
// Reference semantics: MatrixFreeKff.matvec (src/gpu_fem/solver_v2.py:1183-1223)
// and the fused kernels of src/gpu_fem/cuda_fused_matvec.py:41-246 (whose
// element-centric atomics this replaces).
#include "internal.cuh"
#include "reduce.cuh"

#include <stdexcept>

namespace topo {

__constant__ double cKE64[576];
__constant__ float cKE32[576];
__constant__ float cKEbf[576];  // KE rounded to BF16 (round-to-nearest-even), held as float

static inline float bf16_round_host(float x) {
  uint32_t b;
  memcpy(&b, &x, 4);
  b = (b + 0x7FFFu + ((b >> 16) & 1u)) & 0xFFFF0000u;
  float r;
  memcpy(&r, &b, 4);
  return r;
}

void set_ke(const double* KE) {
  float f[576], bf[576];
  for (int i = 0; i < 576; ++i) {
    f[i] = (float)KE[i];
    bf[i] = bf16_round_host(f[i]);
  }
  TOPO_CUDA_CHECK(cudaMemcpyToSymbol(cKE64, KE, sizeof(double) * 576));
  TOPO_CUDA_CHECK(cudaMemcpyToSymbol(cKE32, f, sizeof(float) * 576));
  TOPO_CUDA_CHECK(cudaMemcpyToSymbol(cKEbf, bf, sizeof(float) * 576));
}

// Local corner id of bit pattern (bx,by,bz) in the reference hex8 ordering
// (0,0,0)(1,0,0)(1,1,0)(0,1,0)(0,0,1)(1,0,1)(1,1,1)(0,1,1).
__host__ __device__ constexpr int corner_id(int bx, int by, int bz) {
  return bz * 4 + (by ? (bx ? 2 : 3) : (bx ? 1 : 0));
}

template <typename T, bool BF>
__device__ __forceinline__ T ke(int idx) {
  if constexpr (sizeof(T) == 8) return cKE64[idx];
  else if constexpr (BF) return cKEbf[idx];
  else return cKE32[idx];
}

// Read one value of u as TS (double stays double; float and bf16 become float).
template <typename TS, typename TU>
__device__ __forceinline__ TS load_as(const TU* p) {
  if constexpr (sizeof(TU) == 2) return (TS)__bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(p));
  else return (TS)(*p);
}

// Tile of owned nodes per block: 32 along z (one warp), 4 along y, 2 along x.
constexpr int TZ = 32, TY = 4, TX = 2;
constexpr int UZ = TZ + 2, UY = TY + 2, UX = TX + 2;  // node tile with halo
constexpr int EZ = TZ + 1, EY = TY + 1, EX = TX + 1;  // incident elements

// T  : accumulation / output type (double or float)
// TU : type of u in global memory (double, float or __nv_bfloat16)
// BF : round u and KE to BF16 before multiplying (FP32 accumulation)
template <typename T, typename TU, bool BF, Epi EPI>
__global__ void __launch_bounds__(TX * TY * TZ)
k_level0(Grid g, const TU* __restrict__ u, const T* __restrict__ E, const uint8_t* __restrict__ mask,
         EpiDev<T> ep, KrylovState* st, RedWork red) {
  if (st != nullptr && st->done) return;
  using TS = typename std::conditional<sizeof(T) == 8, double, float>::type;
  __shared__ __align__(16) TS us[UX][UY][UZ][4];
  __shared__ TS es[EX][EY][EZ];

  const int z0 = blockIdx.x * TZ, y0 = blockIdx.y * TY, x0 = blockIdx.z * TX;
  const int tid = threadIdx.x + TZ * (threadIdx.y + TY * threadIdx.z);
  constexpr int NT = TX * TY * TZ;

  // stage nodal values of the brick + halo (zero outside the grid). A node
  // column (xx, yy) is one contiguous z-run of 3*UZ values in global memory:
  // warp w copies columns w, w + 8, ... with its lanes along the run, so the
  // loads coalesce and the index arithmetic is one division by 3.
  {
    const int warp = tid >> 5, lane = tid & 31;
    for (int col = warp; col < UX * UY; col += NT / 32) {
      const int xx = col / UY, yy = col - UY * xx;
      const int gx = x0 - 1 + xx, gy = y0 - 1 + yy;
      const bool cin = gx >= 0 && gx < g.NX && gy >= 0 && gy < g.NY;
      const long long base = 3 * (((long long)gx * g.NY + gy) * g.NZ + (z0 - 1));
#pragma unroll
      for (int e = lane; e < 3 * UZ; e += 32) {
        const int zz = e / 3, c = e - 3 * zz;
        const int gz = z0 - 1 + zz;
        TS v = 0;
        if (cin && gz >= 0 && gz < g.NZ) {
          v = load_as<TS>(u + base + e);
          if constexpr (BF) v = __bfloat162float(__float2bfloat16_rn((float)v));
        }
        us[xx][yy][zz][c] = v;
      }
    }
    // moduli of the incident elements: element columns are contiguous z-runs too
    for (int col = warp; col < EX * EY; col += NT / 32) {
      const int xx = col / EY, yy = col - EY * xx;
      const int gx = x0 - 1 + xx, gy = y0 - 1 + yy;
      const bool cin = gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny;
      const long long base = ((long long)gx * g.ny + gy) * g.nz + (z0 - 1);
      for (int zz = lane; zz < EZ; zz += 32) {
        const int gz = z0 - 1 + zz;
        es[xx][yy][zz] = (cin && gz >= 0 && gz < g.nz) ? (TS)E[base + zz] : (TS)0;
      }
    }
  }
  __syncthreads();

  const int tz = threadIdx.x, ty = threadIdx.y, tx = threadIdx.z;
  const int gx = x0 + tx, gy = y0 + ty, gz = z0 + tz;
  const bool inside = gx < g.NX && gy < g.NY && gz < g.NZ;
  const long long node = ((long long)gx * g.NY + gy) * g.NZ + gz;

  TS acc0 = 0, acc1 = 0, acc2 = 0;
  if (inside) {
    // Neighbour-major order: each of the 27 neighbour records is read once
    // (one conflict-free vector load) and feeds the partial sums t[o] of
    // every element o that contains both it and this node; then
    // y = sum_o E_o t[o]. 576 multiply-adds, 27 shared-memory loads.
    TS t[2][2][2][3];
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
          const TS* rec = &us[tx + dx][ty + dy][tz + dz][0];
          TS uv[3];
          if constexpr (sizeof(TS) == 4) {
            const float4 v = *reinterpret_cast<const float4*>(rec);
            uv[0] = v.x;
            uv[1] = v.y;
            uv[2] = v.z;
          } else {
            const double2 v01 = *reinterpret_cast<const double2*>(rec);
            uv[0] = v01.x;
            uv[1] = v01.y;
            uv[2] = rec[2];
          }
#pragma unroll
          for (int ox = 0; ox < 2; ++ox)
#pragma unroll
            for (int oy = 0; oy < 2; ++oy)
#pragma unroll
              for (int oz = 0; oz < 2; ++oz) {
                const int mx = dx - ox, my = dy - oy, mz = dz - oz;  // neighbour's corner in element o
                if (mx < 0 || mx > 1 || my < 0 || my > 1 || mz < 0 || mz > 1) continue;
                const int a = corner_id(1 - ox, 1 - oy, 1 - oz);
                const int m = corner_id(mx, my, mz);
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                  for (int d = 0; d < 3; ++d)
                    t[ox][oy][oz][c] += ke<TS, BF>((3 * a + c) * 24 + 3 * m + d) * uv[d];
              }
        }
#pragma unroll
    for (int ox = 0; ox < 2; ++ox)
#pragma unroll
      for (int oy = 0; oy < 2; ++oy)
#pragma unroll
        for (int oz = 0; oz < 2; ++oz) {
          const TS Ee = es[tx + ox][ty + oy][tz + oz];
          acc0 += Ee * t[ox][oy][oz][0];
          acc1 += Ee * t[ox][oy][oz][1];
          acc2 += Ee * t[ox][oy][oz][2];
        }
  }

  const TS acc[3] = {acc0, acc1, acc2};
  if constexpr (EPI == Epi::StoreDot) {
    double part[1] = {0.0};
    if (inside) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const long long i = 3 * node + c;
        if (!topo_in_range(i, g.ndof)) continue;
        const T v = mask[i] ? (T)acc[c] : (T)0;
        ep.y[i] = v;
        part[0] += (double)load_as<TS>(u + i) * (double)v;
      }
    }
    double tot[1];
    if (grid_sum<1>(part, red, tot)) {
      if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
        st->pAp = tot[0];
        st->alpha = st->rz / tot[0];
      }
    }
    return;
  }
  if (!inside) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const long long i = 3 * node + c;
    if (!topo_in_range(i, g.ndof)) continue;
    epilogue_store<T, EPI>(ep, i, mask[i] != 0, (T)acc[c], load_as<T>(u + i));
  }
}

template <typename T, typename TU, bool BF>
static void launch_level0(const Grid& g, const void* u, const void* E, const uint8_t* mask, void* y,
                          Epi epi, const EpiArgs& ea, cudaStream_t s) {
  dim3 block(TZ, TY, TX);
  dim3 grid((g.NZ + TZ - 1) / TZ, (g.NY + TY - 1) / TY, (g.NX + TX - 1) / TX);
  const TU* uu = (const TU*)u;
  const T* EE = (const T*)E;
  const EpiDev<T> ep = make_epi<T>(y, ea);
  switch (epi) {
    case Epi::Store:
      k_level0<T, TU, BF, Epi::Store><<<grid, block, 0, s>>>(g, uu, EE, mask, ep, ea.st, ea.red);
      break;
    case Epi::Residual:
      k_level0<T, TU, BF, Epi::Residual><<<grid, block, 0, s>>>(g, uu, EE, mask, ep, ea.st, ea.red);
      break;
    case Epi::ChebR:
      k_level0<T, TU, BF, Epi::ChebR><<<grid, block, 0, s>>>(g, uu, EE, mask, ep, ea.st, ea.red);
      break;
    case Epi::StoreDot:
      k_level0<T, TU, BF, Epi::StoreDot><<<grid, block, 0, s>>>(g, uu, EE, mask, ep, ea.st, ea.red);
      break;
    case Epi::RUpd:
      k_level0<T, TU, BF, Epi::RUpd><<<grid, block, 0, s>>>(g, uu, EE, mask, ep, ea.st, ea.red);
      break;
  }
  TOPO_LAUNCH_CHECK();
}

void level0_apply(Prec p, const Grid& g, const void* u, const void* E, const uint8_t* mask, void* y, Epi epi,
                  const EpiArgs& ea, cudaStream_t s) {
  // FP64 / FP32: the x-streaming kernel (kmatvec_cc.cu) when its planes fit
  // in shared memory; the brick kernel below otherwise and for the BF16
  // emulation on CUDA cores.
  const bool al = ((uintptr_t)u & 15) == 0 && ((uintptr_t)E & 15) == 0;
  switch (p) {
    case Prec::F64:
      if (al && level0_cc_supported(g, true)) level0_apply_cc(true, g, u, E, mask, y, epi, ea, wait_error_flag(), s);
      else launch_level0<double, double, false>(g, u, E, mask, y, epi, ea, s);
      break;
    case Prec::F32:
      if (al && level0_cc_supported(g, false)) level0_apply_cc(false, g, u, E, mask, y, epi, ea, wait_error_flag(), s);
      else launch_level0<float, float, false>(g, u, E, mask, y, epi, ea, s);
      break;
    case Prec::BF16: launch_level0<float, float, true>(g, u, E, mask, y, epi, ea, s); break;
  }
}

// BF16-storage input variant used by the public matvec entry (u in bf16).
void level0_apply_bf16_input(const Grid& g, const void* u, const void* E, const uint8_t* mask, void* y,
                             cudaStream_t s) {
  EpiArgs ea{};
  launch_level0<float, __nv_bfloat16, true>(g, u, E, mask, y, Epi::Store, ea, s);
}

// ------------------------------------------------------------------ diagonal
__global__ void k_level0_diag(Grid g, const double* __restrict__ E, const uint8_t* __restrict__ mask,
                              double* __restrict__ diag) {
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= g.nnodes) return;
  const int iz = n % g.NZ, iy = (n / g.NZ) % g.NY, ix = n / ((long long)g.NZ * g.NY);
  double d[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int ox = 0; ox < 2; ++ox)
#pragma unroll
    for (int oy = 0; oy < 2; ++oy)
#pragma unroll
      for (int oz = 0; oz < 2; ++oz) {
        const int ex = ix - 1 + ox, ey = iy - 1 + oy, ez = iz - 1 + oz;
        if (ex < 0 || ex >= g.nx || ey < 0 || ey >= g.ny || ez < 0 || ez >= g.nz) continue;
        const double Ee = E[((long long)ex * g.ny + ey) * g.nz + ez];
        const int a = corner_id(1 - ox, 1 - oy, 1 - oz);
#pragma unroll
        for (int c = 0; c < 3; ++c) d[c] += Ee * cKE64[(3 * a + c) * 24 + 3 * a + c];
      }
#pragma unroll
  for (int c = 0; c < 3; ++c) diag[3 * n + c] = mask[3 * n + c] ? d[c] : 0.0;
}

void level0_diag(const Grid& g, const double* E, const uint8_t* mask, double* diag, cudaStream_t s) {
  const int bs = 256;
  k_level0_diag<<<(unsigned)((g.nnodes + bs - 1) / bs), bs, 0, s>>>(g, E, mask, diag);
  TOPO_LAUNCH_CHECK();
}

// ------------------------------------------------------------------ modulus
__global__ void k_modulus(long long n, const double* __restrict__ rho, double penal, double E0, double Emin,
                          double* __restrict__ E, float* __restrict__ E32) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double r = rho[i];
  const double rp = (penal == 3.0) ? r * r * r : pow(r, penal);
  const double e = Emin + (E0 - Emin) * rp;
  E[i] = e;
  if (E32) E32[i] = (float)e;
}

void modulus(long long n, const double* rho, double penal, double E0, double Emin, double* E, float* E32,
             cudaStream_t s) {
  const int bs = 256;
  k_modulus<<<(unsigned)((n + bs - 1) / bs), bs, 0, s>>>(n, rho, penal, E0, Emin, E, E32);
  TOPO_LAUNCH_CHECK();
}

// -------------------------------------------------------------- sensitivity
// dc_e = -p (E0-Emin) rho^(p-1) u_e^T KE u_e, FP64 arithmetic
// (src/gpu_fem/solver_v4.py:246-251).
template <typename TU>
__global__ void k_sensitivity(Grid g, const TU* __restrict__ u, const TU* __restrict__ v,
                              const double* __restrict__ rho, double penal, double E0, double Emin,
                              double* __restrict__ dc) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= g.nelem) return;
  const int ez = e % g.nz, ey = (e / g.nz) % g.ny, ex = e / ((long long)g.nz * g.ny);
  double ue[24], ve[24];
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const int bx = (m == 1 || m == 2 || m == 5 || m == 6);
    const int by = (m == 2 || m == 3 || m == 6 || m == 7);
    const int bz = (m >= 4);
    long long n = ((long long)(ex + bx) * g.NY + (ey + by)) * g.NZ + (ez + bz);
    if (!topo_in_range(n, g.nnodes)) n = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ue[3 * m + c] = (double)u[3 * n + c];
      ve[3 * m + c] = (v != nullptr) ? (double)v[3 * n + c] : ue[3 * m + c];
    }
  }
  // KE annihilates rigid translations, so the element means are removed
  // first: v_e^T KE u_e is unchanged and the contraction no longer cancels
  // the (large) translation part of the displacement in rounding.
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double mu = 0.0, mv = 0.0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      mu += ue[3 * m + c];
      mv += ve[3 * m + c];
    }
    mu *= 0.125;
    mv *= 0.125;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      ue[3 * m + c] -= mu;
      ve[3 * m + c] -= mv;
    }
  }
  // ce = v_e^T KE u_e (KE symmetric), v = u for compliance
  double ce = 0.0;
#pragma unroll
  for (int i = 0; i < 24; ++i) {
    double t = 0.0;
#pragma unroll
    for (int j = 0; j < 24; ++j) t += ue[j] * cKE64[j * 24 + i];
    ce += t * ve[i];
  }
  const double r = rho[e];
  const double rp = (penal == 3.0) ? r * r : pow(r, penal - 1.0);
  dc[e] = -penal * (E0 - Emin) * rp * ce;
}

void sensitivity(const Grid& g, const void* u, const void* v, bool u_f32, const double* rho, double penal,
                 double E0, double Emin, double* dc, cudaStream_t s) {
  const int bs = 128;
  const unsigned nb = (unsigned)((g.nelem + bs - 1) / bs);
  if (u_f32)
    k_sensitivity<float><<<nb, bs, 0, s>>>(g, (const float*)u, (const float*)v, rho, penal, E0, Emin, dc);
  else
    k_sensitivity<double><<<nb, bs, 0, s>>>(g, (const double*)u, (const double*)v, rho, penal, E0, Emin, dc);
  TOPO_LAUNCH_CHECK();
}

TOPO_BOUNDS_READER(bounds_flag_level0)

}  // namespace topo
