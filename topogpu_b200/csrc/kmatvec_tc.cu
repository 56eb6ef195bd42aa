// kmatvec_tc.cu - level-0 hex8 K.u with BF16 inputs on the tcgen05 tensor
// cores (FP32 accumulation in tensor memory), for the mixed-precision smoother
// and the BF16 operator entry point.
//
// Work items: patches of 16 x 16 elements in (x, y) times z layers, walked by
// persistent CTAs (pipeline below). For every element layer the contraction Y_e = KE u_e of 256 elements is
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
constexpr int RX = 16;                // node slots per row (x), 8 bytes each
constexpr int RY = 17;                // node rows per plane (y)
constexpr int NPL = ZB + 1;           // node planes per block
constexpr int ROW_B = RX * 8;         // 128 bytes
constexpr int PLANE_B = RX * RY * 8;  // 2176 bytes
constexpr int COPY_B = NPL * PLANE_B; // 10880 bytes
constexpr int NLEV = ZB + 1;          // output node levels staged per block
constexpr int OUT_FLOATS = OWN * OWN * NLEV * 3;
constexpr int al16(int x) { return (x + 15) & ~15; }
static_assert(PLANE_B % 16 == 0, "descriptor alignment");

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

// ---------------------------------------------------------------------------
// Persistent warp-specialised pipeline. One CTA per SM walks a contiguous
// range of (column, z-layer) items, column = one 16x16-element patch, in
// blocks of ZB layers; four roles overlap successive blocks:
//   load   (warps 8-11): node planes -> BF16 records in a 3-stage ring
//   mma    (warp 12, one thread): 4 tcgen05.mma per layer into one of two
//          256-column TMEM buffers, commit -> tfull[tb] and empty[s]
//   reduce (warps 0-3 = TMEM lanes 0-127): TMEM -> E scaling -> nodal sums
//          (x pair in registers, y by shuffles, z by a carried share) ->
//          staged outputs (two buffers)
//   store  (warps 4-7): the epilogue (Store / Residual / RUpd / ChebR) on the
//          owned nodes of the block, z-contiguous
// Every wait is an mbarrier poll with an iteration limit; a timeout raises
// the device error flag and a CTA-wide abort so the other roles stop too.
constexpr int NSTAGE = 3;
constexpr int STAGE_B = 2 * COPY_B;
constexpr int OUT_B = al16(OUT_FLOATS * 4);
constexpr int NT2 = 416;
constexpr int W_STORE = 4, W_LOAD = 8, W_MMA = 12;
constexpr int P_B = 0;
constexpr int P_ST = 2048;
constexpr int P_OUT = al16(P_ST + NSTAGE * STAGE_B);
constexpr int P_XCH = al16(P_OUT + 2 * OUT_B);
constexpr int P_BAR = al16(P_XCH + 4 * 8 * 12 * 4);
constexpr int NBAR = 2 * NSTAGE + 8;  // full[3] empty[3] tfull[2] tempty[2] ofull[2] oempty[2]
constexpr int P_TMEM = al16(P_BAR + NBAR * 8);
constexpr int P_ABORT = P_TMEM + 4;
constexpr int SMEM2_BYTES = P_ABORT + 4 + 1024;
constexpr int SMEM2_REQUEST = 120 * 1024;  // one CTA per SM: it owns all 512 TMEM columns
constexpr uint32_t TMEM2_COLS = 512;
static_assert(SMEM2_BYTES <= SMEM2_REQUEST, "shared memory budget");
static_assert(P_ST % 16 == 0 && STAGE_B % 16 == 0 && COPY_B % 16 == 0, "descriptor alignment");
static_assert(P_BAR % 8 == 0, "barrier alignment");

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Bounded wait that also gives up when another role has aborted.
__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* errflag) {
  for (int it = 0; it < (1 << 22); ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 31) == 31 && *abort_flag) return false;
  }
  *abort_flag = 1;
  atomicExch(errflag, 1);
  return false;
}

// AND of a predicate over the 128 reduce threads (named barrier 1): their
// decision to stop must be uniform because they meet at that barrier.
__device__ __forceinline__ bool all_reduce_threads(bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, 1, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)pred)
      : "memory");
  return r != 0;
}

// The block sequence of one CTA: layer items [lo, hi) in column-major order
// (item = column * nz + z); per column a segment [z0, z1) processed from the
// seed layer max(0, z0 - 1) in blocks of ZB layers.
struct BlockSeq {
  int nz, lo, hi, c, c_hi, zb, z0, z1;
  __device__ void seg() {
    z0 = (c == lo / nz) ? lo - c * nz : 0;
    z1 = (c == c_hi) ? hi - c * nz : nz;
    zb = max(0, z0 - 1);
  }
  __device__ void init(int nz_, int lo_, int hi_) {
    nz = nz_, lo = lo_, hi = hi_;
    c = lo / nz;
    c_hi = (hi - 1) / nz;
    if (lo < hi) seg();
    else c = c_hi + 1;
  }
  __device__ bool valid() const { return lo < hi && c <= c_hi; }
  __device__ int nb() const { return min(ZB, z1 - zb); }
  __device__ bool first() const { return zb == max(0, z0 - 1); }
  __device__ void next() {
    zb += ZB;
    if (zb >= z1) {
      ++c;
      if (c <= c_hi) seg();
    }
  }
};

// q(dx,dy,dz) = dx + 2 dy + 4 dz indexes the 8 corners; output column q*4+c.
template <typename TU, Epi EPI>
__global__ void __launch_bounds__(NT2, 1)
k_level0_tc(Grid g, const TU* __restrict__ u, const float* __restrict__ E, const uint8_t* __restrict__ mask,
            const __nv_bfloat16* __restrict__ Bglob, EpiDev<float> ep, const KrylovState* st, int* errflag,
            int ncoly) {
  if (st != nullptr && st->done) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t bar_full = smem_u32(sm + P_BAR), bar_empty = bar_full + 8 * NSTAGE;
  const uint32_t bar_tfull = bar_empty + 8 * NSTAGE, bar_tempty = bar_tfull + 16;
  const uint32_t bar_ofull = bar_tempty + 16, bar_oempty = bar_ofull + 16;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + P_TMEM);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + P_ABORT);

  for (int i = tid; i < 1024 / 8; i += NT2)
    reinterpret_cast<uint4*>(sm + P_B)[i] = reinterpret_cast<const uint4*>(Bglob)[i];
  if (tid == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(bar_full + 8 * s, 128);
      mbar_init(bar_empty + 8 * s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(bar_tfull + 8 * b, 1);
      mbar_init(bar_tempty + 8 * b, 128);
      mbar_init(bar_ofull + 8 * b, 128);
      mbar_init(bar_oempty + 8 * b, 128);
    }
    *abort_flag = 0;
  }
  if (warp == W_MMA) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM2_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;

  const int ncol = ((g.NX + OWN - 1) / OWN) * ncoly;
  const long long T = (long long)ncol * g.nz;
  const int lo = (int)(T * blockIdx.x / gridDim.x), hi = (int)(T * (blockIdx.x + 1) / gridDim.x);
  BlockSeq q;
  q.init(g.nz, lo, hi);

  if (warp >= W_LOAD && warp < W_MMA) {
    // ------------------------------------------------------------ load
    const int pt = tid - 32 * W_LOAD;
    for (int k = 0; q.valid(); ++k, q.next()) {
      const int s = k % NSTAGE;
      if (!wait_bar(bar_empty + 8 * s, ((k / NSTAGE) & 1) ^ 1, abort_flag, errflag)) break;
      const int x0 = -1 + OWN * (q.c / ncoly), y0 = -1 + OWN * (q.c % ncoly);
      const int zb = q.zb, nb = q.nb();
      unsigned char* A0 = sm + P_ST + s * STAGE_B;
      unsigned char* A1 = A0 + COPY_B;
      for (int cidx = pt; cidx < 17 * 17; cidx += 128) {
        const int xs = cidx % 17, ys = cidx / 17;
        const int gx = x0 + xs, gyy = y0 + ys;
        const bool in = gx >= 0 && gx < g.NX && gyy >= 0 && gyy < g.NY;
        const long long n0 = ((long long)gx * g.NY + gyy) * g.NZ + zb;
        float v[ZB + 1][3];
#pragma unroll
        for (int pz = 0; pz <= ZB; ++pz)
#pragma unroll
          for (int c = 0; c < 3; ++c) v[pz][c] = (in && pz <= nb) ? ldu(u + 3 * (n0 + pz) + c) : 0.f;
#pragma unroll
        for (int pz = 0; pz <= ZB; ++pz) {
          const uint2 rec = pack_node(v[pz][0], v[pz][1], v[pz][2]);
          if (xs < RX) *reinterpret_cast<uint2*>(A0 + pz * PLANE_B + ys * ROW_B + xs * 8) = rec;
          if (xs >= 1) *reinterpret_cast<uint2*>(A1 + pz * PLANE_B + ys * ROW_B + (xs - 1) * 8) = rec;
        }
      }
      fence_async_smem();
      mbar_arrive(bar_full + 8 * s);
    }
  } else if (warp == W_MMA) {
    // ------------------------------------------------------------- mma
    if (lane == 0) {
      int last = -1;
      for (int k = 0; q.valid(); ++k, q.next()) {
        const int s = k % NSTAGE, tb = k & 1;
        if (!wait_bar(bar_full + 8 * s, (k / NSTAGE) & 1, abort_flag, errflag)) break;
        if (!wait_bar(bar_tempty + 8 * tb, ((k >> 1) & 1) ^ 1, abort_flag, errflag)) break;
        tc_fence_after();
        const uint32_t a0 = smem_u32(sm + P_ST + s * STAGE_B), a1 = a0 + COPY_B, bb = smem_u32(sm + P_B);
        const int nb = q.nb();
        for (int l = 0; l < nb; ++l)
#pragma unroll
          for (int p = 0; p < 2; ++p)
#pragma unroll
            for (int kh = 0; kh < 2; ++kh) {
              const uint32_t abase = (p ? a1 : a0) + (l + kh) * PLANE_B;
              mma_bf16(tbase + tb * 256 + l * 64 + p * 32, make_desc(abase, ROW_B, ROW_B),
                       make_desc(bb + kh * 256, 128, 512), kh);
            }
        mma_commit(bar_tfull + 8 * tb);
        mma_commit(bar_empty + 8 * s);
        last = k;
      }
      // never leave MMAs in flight behind an abort (bounded, ignores the abort flag)
      if (last >= 0) {
        const uint32_t b = bar_tfull + 8 * (last & 1), par = (last >> 1) & 1;
        for (int it = 0; it < (1 << 22) && !mbar_try(b, par); ++it) {
        }
      }
    }
  } else if (warp < W_STORE) {
    // ---------------------------------------------------------- reduce
    const int m = tid, gy = m >> 3, r = m & 7;
    float* xch = reinterpret_cast<float*>(sm + P_XCH);
    float carry[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    for (int k = 0; q.valid(); ++k, q.next()) {
      const int tb = k & 1, ob = k & 1;
      const int x0 = -1 + OWN * (q.c / ncoly), y0 = -1 + OWN * (q.c % ncoly);
      const int zb = q.zb, nb = q.nb(), z0 = q.z0, z1 = q.z1;
      if (q.first()) {
#pragma unroll
        for (int nd = 0; nd < 2; ++nd)
#pragma unroll
          for (int c = 0; c < 3; ++c) carry[nd][c] = 0.f;
      }
      // moduli of this thread's two elements, fetched before the wait
      float EA[ZB], EB[ZB];
      const int ex = x0 + 2 * r, ey = y0 + gy;
      const bool yin = ey >= 0 && ey < g.ny;
#pragma unroll
      for (int l = 0; l < ZB; ++l) {
        const long long e0 = ((long long)ex * g.ny + ey) * g.nz + zb + l;
        EA[l] = (l < nb && yin && ex >= 0 && ex < g.nx) ? E[e0] : 0.f;
        EB[l] = (l < nb && yin && ex + 1 >= 0 && ex + 1 < g.nx) ? E[e0 + (long long)g.ny * g.nz] : 0.f;
      }
      bool ok = wait_bar(bar_tfull + 8 * tb, (k >> 1) & 1, abort_flag, errflag);
      ok = ok && wait_bar(bar_oempty + 8 * ob, ((k >> 1) & 1) ^ 1, abort_flag, errflag);
      if (!all_reduce_threads(ok)) break;
      tc_fence_after();
      float* outs = reinterpret_cast<float*>(sm + P_OUT + ob * OUT_B);
#pragma unroll
      for (int l = 0; l < ZB; ++l) {
        if (l >= nb) break;
        const int z = zb + l;
        float OA[32], OB[32];
        const uint32_t tl = tbase + ((uint32_t)(warp * 32) << 16) + tb * 256 + l * 64;
        tmem_ld32(tl, OA);
        tmem_ld32(tl + 32, OB);
        tmem_wait_ld();
        // S[node][dy][dz][c]: node 0 = x 2r+1 (shared by A and B), node 1 = x 2r+2
        float S[2][2][2][3];
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
          for (int dz = 0; dz < 2; ++dz)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const int q0 = 0 + 2 * dy + 4 * dz, q1 = 1 + 2 * dy + 4 * dz;
              const float a_lo = EA[l] * OA[q0 * 4 + c];
              const float a_hi = EA[l] * OA[q1 * 4 + c];
              const float b_lo = EB[l] * OB[q0 * 4 + c];
              const float b_hi = EB[l] * OB[q1 * 4 + c];
              const float next_a_lo = __shfl_down_sync(0xffffffffu, a_lo, 1);
              S[0][dy][dz][c] = a_hi + b_lo;
              S[1][dy][dz][c] = b_hi + next_a_lo;
            }
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
        const int lev = z - zb;
#pragma unroll
        for (int nd = 0; nd < 2; ++nd) {
          const int xr = 2 * r + 1 + nd;
          const bool own = xr <= OWN && gy >= 1;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float v = U[nd][0][c] + carry[nd][c];
            carry[nd][c] = U[nd][1][c];
            if (own && z >= z0) outs[(((gy - 1) * OWN + (xr - 1)) * NLEV + lev) * 3 + c] = v;
          }
        }
        asm volatile("bar.sync 1, 128;" ::: "memory");  // xch reuse
      }
      tc_fence_before();
      mbar_arrive(bar_tempty + 8 * tb);
      if ((zb + nb == z1) && (z1 == g.nz)) {
#pragma unroll
        for (int nd = 0; nd < 2; ++nd) {
          const int xr = 2 * r + 1 + nd;
          if (xr <= OWN && gy >= 1)
#pragma unroll
            for (int c = 0; c < 3; ++c) outs[(((gy - 1) * OWN + (xr - 1)) * NLEV + nb) * 3 + c] = carry[nd][c];
        }
      }
      mbar_arrive(bar_ofull + 8 * ob);
    }
  } else {
    // ----------------------------------------------------------- store
    const int stid = tid - 32 * W_STORE;
    for (int k = 0; q.valid(); ++k, q.next()) {
      const int ob = k & 1;
      if (!wait_bar(bar_ofull + 8 * ob, (k >> 1) & 1, abort_flag, errflag)) break;
      const float* outs = reinterpret_cast<const float*>(sm + P_OUT + ob * OUT_B);
      const int x0 = -1 + OWN * (q.c / ncoly), y0 = -1 + OWN * (q.c % ncoly);
      const int zb = q.zb, nb = q.nb();
      const bool last_level = (zb + nb == q.z1) && (q.z1 == g.nz);
      const int zlo = max(zb, q.z0);
      const int nlev_out = (zb + nb) - zlo + (last_level ? 1 : 0);
      if (nlev_out > 0) {
        const int per_node = nlev_out * 3;
        const int total = OWN * OWN * per_node;
        for (int base = stid; base < total; base += 4 * 128) {
          long long ii[4];
          float acc[4], ui[4];
          bool val[4], fr[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int idx = base + 128 * j;
            val[j] = false;
            ii[j] = 0;
            acc[j] = 0.f;
            if (idx < total) {
              const int on = idx / per_node, rem = idx % per_node;
              const int lv = rem / 3, c = rem % 3;
              const int xr = on % OWN + 1, yr = on / OWN + 1;
              const int gx = x0 + xr, gyy = y0 + yr, gz = zlo + lv;
              if (gx < g.NX && gyy < g.NY && gz < g.NZ) {
                val[j] = true;
                ii[j] = 3 * (((long long)gx * g.NY + gyy) * g.NZ + gz) + c;
                acc[j] = outs[(on * NLEV + (gz - zb)) * 3 + c];
              }
            }
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            fr[j] = val[j] ? mask[ii[j]] != 0 : false;
            ui[j] = (EPI == Epi::ChebR && val[j]) ? ldu(u + ii[j]) : 0.f;
          }
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (val[j]) epilogue_store<float, EPI>(ep, ii[j], fr[j], acc[j], ui[j]);
        }
      }
      mbar_arrive(bar_oempty + 8 * ob);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == W_MMA)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TMEM2_COLS));
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
  static int nsm = 0;
  if (nsm == 0) {
    int dev = 0;
    TOPO_CUDA_CHECK(cudaGetDevice(&dev));
    TOPO_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    TOPO_CUDA_CHECK(cudaFuncSetAttribute(tc::k_level0_tc<TU, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         tc::SMEM2_REQUEST));
  }
  const int ncolx = (g.NX + tc::OWN - 1) / tc::OWN, ncoly = (g.NY + tc::OWN - 1) / tc::OWN;
  const long long items = (long long)ncolx * ncoly * g.nz;
  if (items >= (1LL << 31)) throw std::runtime_error("level0_apply_tc: grid too large");
  const int grid = (int)std::min<long long>(items, nsm);
  const EpiDev<float> ep = make_epi<float>(y, ea);
  tc::k_level0_tc<TU, EPI><<<grid, tc::NT2, tc::SMEM2_REQUEST, s>>>(g, (const TU*)u, (const float*)E, mask, g_tcB,
                                                                   ep, ea.st, g_tcErr, ncoly);
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
