// kmatvec_tc.cu - level-0 hex8 K.u with BF16 inputs on the tcgen05 tensor
// cores (FP32 accumulation in tensor memory), for the mixed-precision smoother
// and the BF16 operator entry point.
//
// Per CTA: a patch of 16 x 16 elements in (x, y) and a chunk of z layers.
// For every element layer the contraction Y_e = KE u_e of 256 elements is
// four tcgen05.mma (M=128 elements, N=32 outputs, K=16 inputs each):
//   * the nodal values of two z planes sit in shared memory as BF16 records
//     (ux, uy, uz, 0) ordered x-fastest; an element's 32-entry input row is
//     four 16-byte chunks (node pairs along x at (dy, dz) = (0,0),(1,0),(0,1),
//     (1,1)); rows of one MMA tile are the 8 elements of one x parity along a
//     row (16 bytes apart) times 16 rows in y, so the tensor core reads its A
//     operand straight from the node tile through the shared-memory
//     descriptor - no gather. A second copy of the tile shifted by one node
//     serves the odd-x elements (16-byte alignment).
//   * KE (rows/columns permuted to that order, padded 24->32, rounded to
//     BF16) is the B operand.
// The epilogue turns element outputs into nodal sums without atomics: each
// thread owns the two elements of one x pair, adds the x-shared node in
// registers, gets the x- and y-neighbour shares by warp shuffles (one small
// shared-memory hand-off between warps) and carries the z+1 share to the
// next layer. Owned nodes are written once, z-contiguous.
//
// Reference semantics: FusedMatvec fused_matvec_bf16
// (src/gpu_fem/cuda_fused_matvec.py:112-246): BF16-rounded u and KE, FP32
// accumulation, then the scale by E_e.
#include "internal.cuh"
#include "reduce.cuh"

#include <stdexcept>

namespace topo {

namespace tc {

constexpr int PX = 16, PY = 16;       // elements per patch in x and y
constexpr int OWN = 15;               // owned nodes per patch per direction
constexpr int ZB = 4;                 // element layers per tensor-memory block
constexpr int ZC = 16;                // element layers per CTA
constexpr int RX = 16;                // node slots per row (x), 8 bytes each
constexpr int RY = 17;                // node rows per plane (y)
constexpr int NPL = ZB + 1;           // node planes per block
constexpr int ROW_B = RX * 8;         // 128 bytes
constexpr int PLANE_B = RX * RY * 8;  // 2176 bytes
constexpr int COPY_B = NPL * PLANE_B; // 10880 bytes
constexpr int NT = 128;
constexpr uint32_t TMEM_COLS = 256;   // ZB layers x 2 parity tiles x 32 columns
constexpr int NLEV = ZB + 1;          // output node levels staged per block

// shared-memory layout (bytes, from a 1024-aligned base; every region 16-aligned)
constexpr int al16(int x) { return (x + 15) & ~15; }
constexpr int OFF_B = 0;                                 // B operand: 32 x 32 bf16 = 2048
constexpr int OFF_A0 = 2048;                             // node copy, even x
constexpr int OFF_A1 = OFF_A0 + COPY_B;                  // node copy, odd x
constexpr int OFF_E = al16(OFF_A1 + COPY_B);             // E: ZB x 16 x 16 floats
constexpr int OFF_OUT = al16(OFF_E + ZB * PY * PX * 4);  // staged outputs
constexpr int OUT_FLOATS = OWN * OWN * NLEV * 3;
constexpr int OFF_XCH = al16(OFF_OUT + OUT_FLOATS * 4);  // warp hand-off: 4 x 8 x 12 floats
constexpr int OFF_BAR = al16(OFF_XCH + 4 * 8 * 12 * 4);  // ZB mbarriers (8-byte objects)
constexpr int OFF_TMEM = al16(OFF_BAR + ZB * 8);         // tensor-memory base address
static_assert(OFF_BAR % 8 == 0 && OFF_TMEM % 4 == 0, "barrier alignment");
constexpr int SMEM_BYTES = OFF_TMEM + 16 + 1024;  // + alignment slack
// 100 KB requested so that at most two CTAs share an SM (2 x 256 TMEM columns).
constexpr int SMEM_REQUEST = 100 * 1024;
static_assert(SMEM_BYTES <= SMEM_REQUEST, "shared memory budget");
static_assert(OFF_A0 % 16 == 0 && OFF_A1 % 16 == 0 && PLANE_B % 16 == 0, "descriptor alignment");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor, K-major, no swizzle (SM100 version 1).
__device__ __forceinline__ uint64_t make_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for tcgen05
  return d;
}

// Instruction descriptor: D f32, A bf16, B bf16, both K-major, N=32, M=128.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(IDESC), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after ~2^22 polls (far beyond any MMA latency) and
// reports it through the device error flag instead of spinning forever.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int it = 0; it < (1 << 22); ++it)
    if (mbar_try(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ uint2 pack_node(float a, float b, float c) {
  const __nv_bfloat162 lo = __floats2bfloat162_rn(a, b);
  const __nv_bfloat162 hi = __floats2bfloat162_rn(c, 0.0f);
  uint2 r;
  r.x = *reinterpret_cast<const uint32_t*>(&lo);
  r.y = *reinterpret_cast<const uint32_t*>(&hi);
  return r;
}

template <typename TU>
__device__ __forceinline__ float ldu(const TU* p) {
  if constexpr (sizeof(TU) == 2) return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(p));
  else return (float)*p;
}

// q(dx,dy,dz) = dx + 2 dy + 4 dz indexes the 8 corners; output column q*4+c.
template <typename TU, Epi EPI>
__global__ void __launch_bounds__(NT, 2)
k_level0_tc(Grid g, const TU* __restrict__ u, const float* __restrict__ E, const uint8_t* __restrict__ mask,
            const __nv_bfloat16* __restrict__ Bglob, EpiDev<float> ep, const KrylovState* st, int* errflag) {
  if (st != nullptr && st->done) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int x0 = -1 + OWN * (int)blockIdx.x, y0 = -1 + OWN * (int)blockIdx.y;
  const int zc0 = ZC * (int)blockIdx.z;
  const int zc1 = min(g.nz, zc0 + ZC);
  const int zs = max(0, zc0 - 1);  // one extra layer to seed the z carry

  float* es = reinterpret_cast<float*>(sm + OFF_E);
  float* outs = reinterpret_cast<float*>(sm + OFF_OUT);
  float* xch = reinterpret_cast<float*>(sm + OFF_XCH);
  const uint32_t bar0 = smem_u32(sm + OFF_BAR);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + OFF_TMEM);

  // B operand into its canonical K-major layout (precomputed on the host)
  for (int i = tid; i < 1024 / 8; i += NT)
    reinterpret_cast<uint4*>(sm + OFF_B)[i] = reinterpret_cast<const uint4*>(Bglob)[i];
  if (tid == 0)
    for (int l = 0; l < ZB; ++l) mbar_init(bar0 + 8 * l, 1);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;

  // thread <-> element pair: TMEM lane m = 32 warp + lane = 8 gy + r
  const int m = tid;
  const int gy = m >> 3, r = m & 7;
  float carry[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
  uint32_t phase = 0;
  bool ok = true;

  for (int zb = zs; zb < zc1 && ok; zb += ZB) {
    const int nb = min(ZB, zc1 - zb);
    // ---- stage node planes zb..zb+nb (BF16 records) and moduli ----------
    for (int idx = tid; idx < (nb + 1) * 17 * 17; idx += NT) {
      const int pz = idx % (nb + 1);
      const int col = idx / (nb + 1);
      const int xs = col % 17, ys = col / 17;
      const int gx = x0 + xs, gyy = y0 + ys, gz = zb + pz;
      float a = 0.f, b = 0.f, c = 0.f;
      if (gx >= 0 && gx < g.NX && gyy >= 0 && gyy < g.NY && gz < g.NZ) {
        const long long n = ((long long)gx * g.NY + gyy) * g.NZ + gz;
        a = ldu(u + 3 * n);
        b = ldu(u + 3 * n + 1);
        c = ldu(u + 3 * n + 2);
      }
      const uint2 rec = pack_node(a, b, c);
      if (ys < RY) {
        if (xs < RX) *reinterpret_cast<uint2*>(sm + OFF_A0 + pz * PLANE_B + ys * ROW_B + xs * 8) = rec;
        if (xs >= 1) *reinterpret_cast<uint2*>(sm + OFF_A1 + pz * PLANE_B + ys * ROW_B + (xs - 1) * 8) = rec;
      }
    }
    for (int idx = tid; idx < nb * PY * PX; idx += NT) {
      const int l = idx / (PY * PX), rem = idx % (PY * PX);
      const int ys = rem / PX, xs = rem % PX;
      const int ex = x0 + xs, ey = y0 + ys, ez = zb + l;
      float v = 0.f;
      if (ex >= 0 && ex < g.nx && ey >= 0 && ey < g.ny) v = E[((long long)ex * g.ny + ey) * g.nz + ez];
      es[idx] = v;
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    // ---- tensor cores: 2 parity tiles x 2 K halves per layer --------------
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(sm + OFF_A0), a1 = smem_u32(sm + OFF_A1), bb = smem_u32(sm + OFF_B);
      for (int l = 0; l < nb; ++l) {
#pragma unroll
        for (int p = 0; p < 2; ++p)
#pragma unroll
          for (int kh = 0; kh < 2; ++kh) {
            const uint32_t abase = (p ? a1 : a0) + (l + kh) * PLANE_B;
            mma_bf16(tbase + l * 64 + p * 32, make_desc(abase, ROW_B, ROW_B), make_desc(bb + kh * 256, 128, 512),
                     kh);
          }
        mma_commit(bar0 + 8 * l);
      }
    }
    // ---- epilogue: layer by layer ------------------------------------------
    for (int l = 0; l < nb; ++l) {
      const int z = zb + l;
      if (!mbar_wait(bar0 + 8 * l, phase)) {
        ok = false;
        if (tid == 0) atomicExch(errflag, 1);
      }
      tc_fence_after();
      float OA[32], OB[32];
      const uint32_t tl = tbase + ((uint32_t)(warp * 32) << 16) + l * 64;
      tmem_ld32(tl, OA);
      tmem_ld32(tl + 32, OB);
      tmem_wait_ld();
      const float EA = es[l * PY * PX + gy * PX + 2 * r];
      const float EB = es[l * PY * PX + gy * PX + 2 * r + 1];
      // S[node][dy][dz][c]: node 0 = x 2r+1 (shared by A and B), node 1 = x 2r+2
      float S[2][2][2][3];
#pragma unroll
      for (int dy = 0; dy < 2; ++dy)
#pragma unroll
        for (int dz = 0; dz < 2; ++dz)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int q0 = 0 + 2 * dy + 4 * dz, q1 = 1 + 2 * dy + 4 * dz;
            const float a_lo = EA * OA[q0 * 4 + c];  // A's corner at x 2r (dx=0)
            const float a_hi = EA * OA[q1 * 4 + c];  // A's corner at x 2r+1
            const float b_lo = EB * OB[q0 * 4 + c];  // B's corner at x 2r+1
            const float b_hi = EB * OB[q1 * 4 + c];  // B's corner at x 2r+2
            const float next_a_lo = __shfl_down_sync(0xffffffffu, a_lo, 1);  // lane+1's A corner at x 2r+2
            S[0][dy][dz][c] = a_hi + b_lo;
            S[1][dy][dz][c] = b_hi + next_a_lo;
          }
      // y: node row gy takes dy=0 from element row gy and dy=1 from row gy-1
      if (lane >= 24) {
        float* xo = xch + (warp * 8 + (lane - 24)) * 12;
#pragma unroll
        for (int nd = 0; nd < 2; ++nd)
#pragma unroll
          for (int dz = 0; dz < 2; ++dz)
#pragma unroll
            for (int c = 0; c < 3; ++c) xo[(nd * 2 + dz) * 3 + c] = S[nd][1][dz][c];
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
      float U[2][2][3];
#pragma unroll
      for (int nd = 0; nd < 2; ++nd)
#pragma unroll
        for (int dz = 0; dz < 2; ++dz)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            float prev = __shfl_up_sync(0xffffffffu, S[nd][1][dz][c], 8);
            if (lane < 8) prev = (warp > 0) ? xch[((warp - 1) * 8 + lane) * 12 + (nd * 2 + dz) * 3 + c] : 0.f;
            U[nd][dz][c] = S[nd][0][dz][c] + prev;
          }
      // z: level z = dz0 share of layer z + carried dz1 share of layer z-1
      const int lev = z - zb;  // staging slot of node level z
#pragma unroll
      for (int nd = 0; nd < 2; ++nd) {
        const int xr = 2 * r + 1 + nd;  // node x relative to x0
        const bool own = xr <= OWN && gy >= 1;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float v = U[nd][0][c] + carry[nd][c];
          carry[nd][c] = U[nd][1][c];
          if (own && z >= zc0) outs[(((gy - 1) * OWN + (xr - 1)) * NLEV + lev) * 3 + c] = v;
        }
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");  // xch reuse
    }
    // node level zc1 == nz comes from the carry alone
    const bool last_level = (zb + nb == zc1) && (zc1 == g.nz);
    if (last_level) {
#pragma unroll
      for (int nd = 0; nd < 2; ++nd) {
        const int xr = 2 * r + 1 + nd;
        if (xr <= OWN && gy >= 1)
#pragma unroll
          for (int c = 0; c < 3; ++c) outs[(((gy - 1) * OWN + (xr - 1)) * NLEV + nb) * 3 + c] = carry[nd][c];
      }
    }
    phase ^= 1u;
    tc_fence_before();
    __syncthreads();
    // ---- write owned nodes, z-contiguous --------------------------------
    const int zlo = max(zb, zc0);
    const int nlev_out = (zb + nb) - zlo + (last_level ? 1 : 0);
    if (nlev_out > 0) {
      const int per_node = nlev_out * 3;
      for (int idx = tid; idx < OWN * OWN * per_node; idx += NT) {
        const int on = idx / per_node, rem = idx % per_node;
        const int lv = rem / 3, c = rem % 3;
        const int xr = on % OWN + 1, yr = on / OWN + 1;
        const int gx = x0 + xr, gyy = y0 + yr, gz = zlo + lv;
        if (gx >= g.NX || gyy >= g.NY || gz >= g.NZ) continue;
        const long long i = 3 * (((long long)gx * g.NY + gyy) * g.NZ + gz) + c;
        const float acc = outs[(on * NLEV + (gz - zb)) * 3 + c];
        epilogue_store<float, EPI>(ep, i, mask[i] != 0, acc, ldu(u + i));
      }
    }
    __syncthreads();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TMEM_COLS));
}

}  // namespace tc

// B operand: KE rows/columns permuted to (corner q = dx+2dy+4dz, comp), padded
// to 32 x 32, rounded to BF16 and laid out as 8x8 core matrices
// (n-group stride 512 B, k-chunk stride 128 B).
static __nv_bfloat16* g_tcB = nullptr;
static int* g_tcErr = nullptr;

static inline uint16_t bf16_bits_rne(float f) {
  uint32_t b;
  memcpy(&b, &f, 4);
  b = (b + 0x7FFFu + ((b >> 16) & 1u)) >> 16;
  return (uint16_t)b;
}

void tc_prepare(const double* KE) {
  auto cid = [](int dx, int dy, int dz) { return dz * 4 + (dy ? (dx ? 2 : 3) : (dx ? 1 : 0)); };
  uint16_t h[1024];
  for (int n = 0; n < 32; ++n)
    for (int k = 0; k < 32; ++k) {
      const int q_out = n / 4, c_out = n % 4;
      const int kc = k / 8, dx_in = (k % 8) / 4, c_in = k % 4;
      const int dy_in = kc & 1, dz_in = kc >> 1;
      double v = 0.0;
      if (c_out < 3 && c_in < 3) {
        const int a = cid(q_out & 1, (q_out >> 1) & 1, q_out >> 2);
        const int b = cid(dx_in, dy_in, dz_in);
        v = KE[(3 * a + c_out) * 24 + 3 * b + c_in];
      }
      const int off = (n / 8) * 256 + (k / 8) * 64 + (n % 8) * 8 + (k % 8);
      h[off] = bf16_bits_rne((float)v);
    }
  if (!g_tcB) TOPO_CUDA_CHECK(cudaMalloc(&g_tcB, sizeof(h)));
  if (!g_tcErr) {
    TOPO_CUDA_CHECK(cudaMalloc(&g_tcErr, sizeof(int)));
    TOPO_CUDA_CHECK(cudaMemset(g_tcErr, 0, sizeof(int)));
  }
  TOPO_CUDA_CHECK(cudaMemcpy(g_tcB, h, sizeof(h), cudaMemcpyHostToDevice));
}

template <typename TU, Epi EPI>
static void launch_tc(const Grid& g, const void* u, const void* E, const uint8_t* mask, void* y, const EpiArgs& ea,
                      cudaStream_t s) {
  static bool attr_set = false;
  if (!attr_set) {
    TOPO_CUDA_CHECK(cudaFuncSetAttribute(tc::k_level0_tc<TU, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         tc::SMEM_REQUEST));
    attr_set = true;
  }
  dim3 grid((g.NX + tc::OWN - 1) / tc::OWN, (g.NY + tc::OWN - 1) / tc::OWN, (g.nz + tc::ZC - 1) / tc::ZC);
  const EpiDev<float> ep = make_epi<float>(y, ea);
  tc::k_level0_tc<TU, EPI><<<grid, tc::NT, tc::SMEM_REQUEST, s>>>(g, (const TU*)u, (const float*)E, mask, g_tcB, ep,
                                                                  ea.st, g_tcErr);
  TOPO_LAUNCH_CHECK();
}

// BF16-input K.u on the tensor cores. u_bf16: u stored as BF16 (else FP32,
// rounded when staged). Supports the Store, Residual, RUpd and ChebR epilogues.
void level0_apply_tc(bool u_bf16, const Grid& g, const void* u, const void* E, const uint8_t* mask, void* y, Epi epi,
                     const EpiArgs& ea, cudaStream_t s) {
  if (!g_tcB) throw std::runtime_error("tensor-core operator not prepared");
#define TOPO_TC_CASE(EP)                                                          \
  case Epi::EP:                                                                   \
    if (u_bf16) launch_tc<__nv_bfloat16, Epi::EP>(g, u, E, mask, y, ea, s);       \
    else launch_tc<float, Epi::EP>(g, u, E, mask, y, ea, s);                      \
    break;
  switch (epi) {
    TOPO_TC_CASE(Store)
    TOPO_TC_CASE(Residual)
    TOPO_TC_CASE(RUpd)
    TOPO_TC_CASE(ChebR)
    default:
      throw std::runtime_error("level0_apply_tc: unsupported epilogue");
  }
#undef TOPO_TC_CASE
}

// Returns and clears the device flag set when an mbarrier wait timed out.
int tc_error_flag(cudaStream_t s) {
  if (!g_tcErr) return 0;
  int h = 0;
  TOPO_CUDA_CHECK(cudaMemcpyAsync(&h, g_tcErr, sizeof(int), cudaMemcpyDeviceToHost, s));
  TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
  if (h) TOPO_CUDA_CHECK(cudaMemsetAsync(g_tcErr, 0, sizeof(int), s));
  return h;
}

}  // namespace topo
