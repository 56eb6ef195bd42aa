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

constexpr int OWN = 15;               // owned nodes per patch per direction
constexpr int ZB = 4;                 // element layers per tensor-memory block
constexpr int RX = 16;                // node slots per row (x), 8 bytes each
constexpr int RY = 17;                // node rows per plane (y)
constexpr int NPL = ZB + 1;           // node planes per block
constexpr int ROW_B = RX * 8;         // 128 bytes
constexpr int PLANE_B = RX * RY * 8;  // 2176 bytes
constexpr int COPY_B = NPL * PLANE_B; // 10880 bytes
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
//   load   (warps 12-14): node planes -> BF16 records, 2-stage ring
//   mma    (warp 15, one thread): 4 tcgen05.mma per layer into one of two
//          256-column TMEM buffers, commit -> tfull[tb] and empty[s]
//   reduce (warps 0-3 = TMEM lanes 0-127): TMEM -> E scaling -> sums over
//          the x pair (registers) and the y pair (shuffles inside a warp;
//          the row below a warp's first row goes to a small boundary
//          table) -> partial nodal values per layer and z side (dz = 0, 1)
//          into a double-buffered partial table. No barriers inside.
//   store  (warps 4-11): per owned DoF, level L = dz0 part of layer L +
//          dz1 part of layer L-1 (carried in registers across blocks), then
//          the epilogue (Store / Residual / RUpd / ChebR). The epilogue's
//          inputs (mask word, r, dinv, x, u or b) for the NEXT block are
//          prefetched into shared memory with cp.async while this block is
//          processed; each thread prefetches exactly the slots it consumes.
// Every wait is an mbarrier poll with an iteration limit; a timeout raises
// the device error flag and a CTA-wide abort so the other roles stop too.
constexpr int NSTAGE = 2;
constexpr int STAGE_B = 2 * COPY_B;
// 16 warps: each SM sub-partition holds 4, so 128 registers a thread fit
// the 16K registers of a sub-partition.
constexpr int NT2 = 512;
constexpr int W_STORE = 4, W_LOAD = 12, W_MMA = 15;
constexpr int NL_THREADS = 32 * (W_MMA - W_LOAD);
constexpr int NS_THREADS = 256;
constexpr int SLOT_COL = 12;                          // ZB levels x 3 components
constexpr int SLOTS = 2816;                           // >= 225 * 12, multiple of 256
constexpr int SLOTS_PER_THREAD = SLOTS / NS_THREADS;  // 11
constexpr int P_MAIN = ZB * 2 * 3 * OWN * OWN;        // [l][dz][c][yr-1][xr-1]
constexpr int P_BND = ZB * 2 * 3 * 3 * OWN;           // [l][dz][c][w][xr-1], node rows 4, 8, 12
constexpr int P_BUF_B = (P_MAIN + P_BND) * 4;
constexpr int N_IN = 5;                               // mask word + up to four vectors
constexpr int IN_BUF_B = N_IN * SLOTS * 4;
constexpr int P_B = 0;
constexpr int P_ST = 2048;
constexpr int P_P = al16(P_ST + NSTAGE * STAGE_B);
constexpr int P_IN = al16(P_P + 2 * P_BUF_B);
constexpr int P_BAR = al16(P_IN + 2 * IN_BUF_B);
constexpr int NBAR = 2 * NSTAGE + 8;  // full[2] empty[2] tfull[2] tempty[2] ofull[2] oempty[2]
constexpr int P_TMEM = al16(P_BAR + NBAR * 8);
constexpr int P_ABORT = P_TMEM + 4;
constexpr int SMEM2_REQUEST = P_ABORT + 4 + 1024;  // one CTA per SM: it owns all 512 TMEM columns
constexpr uint32_t TMEM2_COLS = 512;
static_assert(SMEM2_REQUEST <= 232448, "shared memory budget");
static_assert(SLOTS >= OWN * OWN * SLOT_COL && SLOTS % NS_THREADS == 0, "slot table");
static_assert(P_ST % 16 == 0 && STAGE_B % 16 == 0 && COPY_B % 16 == 0, "descriptor alignment");
static_assert(P_BAR % 8 == 0, "barrier alignment");

__device__ __forceinline__ int pidx(int l, int dz, int c, int yr1, int xr1) {
  return (((l * 2 + dz) * 3 + c) * OWN + yr1) * OWN + xr1;
}
__device__ __forceinline__ int bidx(int l, int dz, int c, int w, int xr1) {
  return P_MAIN + (((l * 2 + dz) * 3 + c) * 3 + w) * OWN + xr1;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src, uint32_t src_size) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(src_size) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
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

// AND of a predicate over the 128 reduce threads (named barrier 1), so that
// they stop together.
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
// seed layer max(0, z0 - 1) in blocks of ZB layers. Output levels of a
// block: [max(zb, z0), zb + nb), plus level nz after the last layer.
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
  __device__ int zlo() const { return max(zb, z0); }
  __device__ void next() {
    zb += ZB;
    if (zb >= z1) {
      ++c;
      if (c <= c_hi) seg();
    }
  }
};

// Epilogue on prefetched inputs (same arithmetic as epilogue_store).
template <Epi EPI>
__device__ __forceinline__ void epi_apply(const EpiDev<float>& e, long long i, bool fr, float acc, float a0, float a1,
                                          float a2, float a3) {
  if constexpr (EPI == Epi::Store) {
    e.y[i] = fr ? acc : 0.f;
  } else if constexpr (EPI == Epi::Residual) {
    e.y[i] = fr ? a0 - acc : 0.f;
  } else if constexpr (EPI == Epi::RUpd) {
    e.r[i] = fr ? a0 - e.s * acc : 0.f;
  } else if constexpr (EPI == Epi::ChebR) {
    if (fr) {
      const float rv = a0 - e.s * acc;
      e.r[i] = rv;
      const float dn = e.c1 * a3 + e.c2 * (a1 * rv);
      e.d_out[i] = dn;
      e.x[i] = a2 + e.ax * dn;
    } else {
      e.r[i] = 0.f;
      e.d_out[i] = 0.f;
    }
  }
}

template <Epi EPI>
__host__ __device__ constexpr int n_inputs() {
  return EPI == Epi::ChebR ? 4 : (EPI == Epi::Store ? 0 : 1);
}

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
      mbar_init(bar_full + 8 * s, NL_THREADS);
      mbar_init(bar_empty + 8 * s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(bar_tfull + 8 * b, 1);
      mbar_init(bar_tempty + 8 * b, 128);
      mbar_init(bar_ofull + 8 * b, 128);
      mbar_init(bar_oempty + 8 * b, NS_THREADS);
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
    // All node loads of a block are issued before the wait for the stage, so
    // they overlap with the previous block's MMA and with each other.
    const int pt = tid - 32 * W_LOAD;
    constexpr int NCOL = 17 * 17, CPT = (NCOL + NL_THREADS - 1) / NL_THREADS;
    for (int k = 0; q.valid(); ++k, q.next()) {
      const int s = k % NSTAGE;
      const int x0 = -1 + OWN * (q.c / ncoly), y0 = -1 + OWN * (q.c % ncoly);
      const int zb = q.zb, nb = q.nb();
      float v[CPT][ZB + 1][3];
#pragma unroll
      for (int t = 0; t < CPT; ++t) {
        const int cidx = pt + NL_THREADS * t;
        const int xs = cidx % 17, ys = cidx / 17;
        const int gx = x0 + xs, gyy = y0 + ys;
        const bool in = cidx < NCOL && gx >= 0 && gx < g.NX && gyy >= 0 && gyy < g.NY;
        const long long n0 = ((long long)gx * g.NY + gyy) * g.NZ + zb;
#pragma unroll
        for (int pz = 0; pz <= ZB; ++pz)
#pragma unroll
          for (int c = 0; c < 3; ++c) v[t][pz][c] = (in && pz <= nb) ? ldu(u + 3 * (n0 + pz) + c) : 0.f;
      }
      if (!wait_bar(bar_empty + 8 * s, ((k / NSTAGE) & 1) ^ 1, abort_flag, errflag)) break;
      unsigned char* A0 = sm + P_ST + s * STAGE_B;
      unsigned char* A1 = A0 + COPY_B;
#pragma unroll
      for (int t = 0; t < CPT; ++t) {
        const int cidx = pt + NL_THREADS * t;
        if (cidx >= NCOL) break;
        const int xs = cidx % 17, ys = cidx / 17;
#pragma unroll
        for (int pz = 0; pz <= ZB; ++pz) {
          const uint2 rec = pack_node(v[t][pz][0], v[t][pz][1], v[t][pz][2]);
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
    for (int k = 0; q.valid(); ++k, q.next()) {
      const int tb = k & 1, ob = k & 1;
      const int x0 = -1 + OWN * (q.c / ncoly), y0 = -1 + OWN * (q.c % ncoly);
      const int zb = q.zb, nb = q.nb();
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
      float* P = reinterpret_cast<float*>(sm + P_P + ob * P_BUF_B);
#pragma unroll
      for (int l = 0; l < ZB; ++l) {
        if (l >= nb) break;
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
        // node row gy: dy=0 share of element row gy + dy=1 share of row gy-1
#pragma unroll
        for (int nd = 0; nd < 2; ++nd) {
          const int xr = 2 * r + 1 + nd;
#pragma unroll
          for (int dz = 0; dz < 2; ++dz)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const float up = __shfl_up_sync(0xffffffffu, S[nd][1][dz][c], 8);
              const float v = S[nd][0][dz][c] + (lane >= 8 ? up : 0.f);
              if (xr <= OWN && gy >= 1) P[pidx(l, dz, c, gy - 1, xr - 1)] = v;
              if (xr <= OWN && lane >= 24 && warp < 3) P[bidx(l, dz, c, warp, xr - 1)] = S[nd][1][dz][c];
            }
        }
      }
      tc_fence_before();
      mbar_arrive(bar_tempty + 8 * tb);
      mbar_arrive(bar_ofull + 8 * ob);
    }
  } else {
    // ----------------------------------------------------------- store
    // Slot j of this thread is the fixed (column, position) pair
    // sidx = stid + 256 j -> column sidx / 12, position sidx % 12 = lv*3 + c,
    // so its geometry is computed once: K[j] = the DoF offset from the
    // block's first owned DoF, tag[j] = packed (x, y, lv, c, boundary row).
    const int stid = tid - 32 * W_STORE;
    constexpr int NIN = n_inputs<EPI>();
    constexpr bool U_IN = (EPI == Epi::ChebR) && sizeof(TU) == 4;
    const float* in_src[4] = {nullptr, nullptr, nullptr, nullptr};
    if constexpr (EPI == Epi::Residual) in_src[0] = ep.b;
    if constexpr (EPI == Epi::RUpd) in_src[0] = ep.r;
    if constexpr (EPI == Epi::ChebR) {
      in_src[0] = ep.r;
      in_src[1] = ep.dinv;
      in_src[2] = ep.x;
      in_src[3] = reinterpret_cast<const float*>(u);
    }
    const long long sx = 3LL * g.NZ * g.NY, sy = 3LL * g.NZ;
    int K[SLOTS_PER_THREAD];  // < 16 * 3 * NZ * NY + 12, well inside int range for any mesh that fits
    uint32_t tag[SLOTS_PER_THREAD];  // xr1 | yr1 << 4 | lv << 8 | c << 10 | bnd << 12, or ~0 when unused
#pragma unroll
    for (int j = 0; j < SLOTS_PER_THREAD; ++j) {
      const int sidx = stid + NS_THREADS * j;
      const int col = sidx / SLOT_COL, rem = sidx - SLOT_COL * col;
      const int xr1 = col % OWN, yr1 = col / OWN;
      const int lv = rem / 3, c = rem - 3 * lv;
      K[j] = (int)((xr1 + 1) * sx + (yr1 + 1) * sy + rem);
      tag[j] = col < OWN * OWN ? (uint32_t)(xr1 | (yr1 << 4) | (lv << 8) | (c << 10) | ((((yr1 + 1) & 3) == 0) << 12))
                               : 0xffffffffu;
    }
    struct BlkGeo {
      long long C;   // DoF index of (x0, y0, zlo), component 0
      int xlim, ylim, per_col, sd;
    };
    auto geo = [&](const BlockSeq& b) {
      BlkGeo r;
      const int x0 = -1 + OWN * (b.c / ncoly), y0 = -1 + OWN * (b.c % ncoly);
      const int zlo = b.zlo();
      r.C = x0 * sx + y0 * sy + 3LL * zlo;
      r.xlim = g.NX - 1 - x0;
      r.ylim = g.NY - 1 - y0;
      r.per_col = (b.zb + b.nb() - zlo) * 3;
      r.sd = zlo - b.zb;
      return r;
    };
    auto slot_ok = [&](uint32_t t, const BlkGeo& gb, int rem_pos) {
      return t != 0xffffffffu && rem_pos < gb.per_col && (int)(t & 15) + 1 <= gb.xlim &&
             (int)((t >> 4) & 15) + 1 <= gb.ylim;
    };
    auto prefetch = [&](const BlockSeq& b, int buf) {
      const BlkGeo gb = geo(b);
      const uint32_t base = smem_u32(sm + P_IN + buf * IN_BUF_B);
#pragma unroll
      for (int j = 0; j < SLOTS_PER_THREAD; ++j) {
        const int sidx = stid + NS_THREADS * j;
        const uint32_t t = tag[j];
        const int rem = (int)((t >> 8) & 3) * 3 + (int)((t >> 10) & 3);
        const bool val = slot_ok(t, gb, rem);
        const long long i = val ? gb.C + K[j] : 0;
        cp_async4(base + 4 * sidx, mask + (i & ~3LL), val ? 4u : 0u);
#pragma unroll
        for (int a = 0; a < 4; ++a)
          if (a < NIN && (a < 3 || U_IN)) cp_async4(base + 4 * ((a + 1) * SLOTS + sidx), in_src[a] + i, val ? 4u : 0u);
      }
      cp_async_commit();
    };
    BlockSeq pf = q;
    if (pf.valid()) prefetch(pf, 0);
    float carry[SLOTS_PER_THREAD];
#pragma unroll
    for (int j = 0; j < SLOTS_PER_THREAD; ++j) carry[j] = 0.f;
    for (int k = 0; q.valid(); ++k, q.next()) {
      const int ob = k & 1;
      pf.next();
      if (pf.valid()) prefetch(pf, (k + 1) & 1);
      else cp_async_commit();
      cp_async_wait<1>();
      if (!wait_bar(bar_ofull + 8 * ob, (k >> 1) & 1, abort_flag, errflag)) break;
      const float* P = reinterpret_cast<const float*>(sm + P_P + ob * P_BUF_B);
      const float* inb = reinterpret_cast<const float*>(sm + P_IN + ob * IN_BUF_B);
      const BlkGeo gb = geo(q);
      const int nb = q.nb();
      if (q.first()) {
#pragma unroll
        for (int j = 0; j < SLOTS_PER_THREAD; ++j) carry[j] = 0.f;
      }
      const bool last_level = (q.zb + nb == q.z1) && (q.z1 == g.nz);
#pragma unroll
      for (int j = 0; j < SLOTS_PER_THREAD; ++j) {
        const int sidx = stid + NS_THREADS * j;
        const uint32_t t = tag[j];
        if (t == 0xffffffffu) continue;
        const int xr1 = t & 15, yr1 = (t >> 4) & 15, lv = (t >> 8) & 3, c = (t >> 10) & 3;
        if (xr1 + 1 > gb.xlim || yr1 + 1 > gb.ylim) continue;
        const int off = yr1 * OWN + xr1;
        const int boff = P_MAIN + (((yr1 + 1) >> 2) - 1) * OWN + xr1;
        const bool bnd = (t >> 12) & 1;
        auto part = [&](int l, int dz) {
          const int lc = (l * 2 + dz) * 3 + c;
          float v = P[lc * (OWN * OWN) + off];
          if (bnd) v += P[lc * (3 * OWN) + boff];
          return v;
        };
        const int rem = lv * 3 + c;
        if (rem < gb.per_col) {
          const int l = lv + gb.sd;
          const float acc = part(l, 0) + (l >= 1 ? part(l - 1, 1) : carry[j]);
          const long long i = gb.C + K[j];
          const uint32_t mw = __float_as_uint(inb[sidx]);
          const bool fr = ((mw >> (8 * (int)(i & 3))) & 0xffu) != 0;
          const float a3 = U_IN ? inb[4 * SLOTS + sidx] : (EPI == Epi::ChebR ? ldu(u + i) : 0.f);
          epi_apply<EPI>(ep, i, fr, acc, inb[SLOTS + sidx], inb[2 * SLOTS + sidx], inb[3 * SLOTS + sidx], a3);
        }
        if (lv == 0) {
          // carry for level zb + nb: dz1 share of the last layer
          carry[j] = part(nb - 1, 1);
          if (last_level) {
            const long long i = gb.C + K[j] + 3LL * (g.nz - q.zlo());
            float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
            if constexpr (NIN >= 1) a0 = in_src[0][i];
            if constexpr (NIN >= 4) {
              a1 = in_src[1][i];
              a2 = in_src[2][i];
              a3 = ldu(u + i);
            }
            epi_apply<EPI>(ep, i, mask[i] != 0, carry[j], a0, a1, a2, a3);
          }
        }
      }
      mbar_arrive(bar_oempty + 8 * ob);
    }
    cp_async_wait<0>();
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
// rounded when staged). `mask` must stay readable 16 bytes past the last DoF
// (the store role prefetches aligned 4-byte mask words). Supports the Store, Residual, RUpd and ChebR epilogues.
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
