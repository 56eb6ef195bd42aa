// kmatvec_xs.cu - level-0 hex8 K.u with BF16 inputs on the tcgen05 tensor
// cores (FP32 accumulation in tensor memory), streaming along x.
//
// Memory order of every level-0 vector is z fastest (DoF 3*node+c, node
// (ix*NY+iy)*NZ+iz), so one x-plane of a window of consecutive y-rows is one
// contiguous range. The kernel is built around that:
//
//  * Work item = (window w, node plane P). A window is 16 element rows in y
//    (rows ey0 = 15w-1 .. 15w+14, one row of overlap with its neighbour) and
//    the full z extent; it owns the 15 node rows 15w .. 15w+14. A persistent
//    CTA takes a contiguous range of items (window-major) and walks the
//    planes of each window in x: element layer L needs node planes L and L+1
//    and completes node plane L (its dx=0 part plus the dx=1 part of layer
//    L-1, carried in registers). The first layer of a run only builds that
//    carry.
//  * Producer warp (one thread): per plane one cp.async.bulk (TMA, no
//    multicast) of the window's 17 node rows of u, per layer one of the 16
//    rows of E, and per output plane one of each epilogue input over the 15
//    owned rows plus the packed node mask, all into shared-memory rings
//    completed on mbarriers. Copies round their start down to 16 bytes; a
//    range ending inside the last 16 bytes of a vector gets its tail by plain
//    loads, so nothing outside a vector is read.
//  * Converter warps: raw u -> BF16 node records (ux, uy, uz, 0), two copies
//    per column: copy 0 puts node z at record z, copy 1 at record z-1. An
//    element (row c, z) then reads its four 16-byte chunks (the z-pair of
//    columns (dx, dy)) straight from a record plane: even z from copy 0, odd
//    z from copy 1, at byte 16*(z/2).
//  * MMA thread: per layer and parity, tiles of 128 rows = 16 window columns
//    (core matrices, stride = column stride) x 8 z-pairs; two
//    tcgen05.mma.kind::f16 (M=128, N=32, K=16) per tile: dx=0 chunks from
//    plane L, dx=1 chunks from plane L+1 (within one MMA the K step dy=0 ->
//    dy=1 is the next column, so LBO = SBO = column stride). KE (permuted,
//    padded 24->32, BF16) is the B operand. Results go to a ring of eight
//    64-column TMEM slots (both parities of one tile).
//  * Reduce warps 0-3 (TMEM lanes 0-127): lane = column c (4 per warp) x
//    z-pair (8). Each thread scales the outputs of its two elements (z = 2j,
//    2j+1) by E and forms nodal sums without atomics: z in registers and by
//    a shuffle of 1 (carried across tiles), y by a shuffle of 8 (plus a
//    small shared-memory hand-off between warps), x by the register carry.
//    Each thread then finishes its 2 (or 3) nodes of the owned plane with
//    the epilogue (Store / Residual / RUpd / ChebR) on the staged inputs.
//
// Every mbarrier wait is bounded; a timeout raises the device error flag
// and a CTA-wide abort, outstanding copies and MMAs are drained (again with
// bounded waits) and the tensor memory is freed before the CTA exits.
//
// Reference semantics: FusedMatvec fused_matvec_bf16
// (src/gpu_fem/cuda_fused_matvec.py:112-246): BF16-rounded u and KE, FP32
// accumulation, then the scale by E_e; MatrixFreeKff.matvec
// (src/gpu_fem/solver_v2.py:1183-1223) for the operator.
#include "internal.cuh"

#include <cstring>
#include <mutex>
#include <stdexcept>
#include <vector>

namespace topo {
namespace xs {

constexpr int WY = 16;          // element rows per window = core matrices per MMA tile
constexpr int OWNR = WY - 1;    // owned node rows per window
constexpr int NROW = WY + 1;    // staged node rows per plane
constexpr int NQMAX = 5;        // tiles per parity per layer (nz <= 80)
constexpr int TSLOT = 8;        // TMEM ring: 8 slots x 64 columns
constexpr int MAXRING = 6;
constexpr int NT = 320;         // 10 warps
constexpr int W_CONV = 4, W_MMA = 8, W_PROD = 9;
constexpr int RED_T = 128, CONV_T = 128;
constexpr int XB_FLOATS = 18;   // y hand-off per lane: up to 3 nodes x 2 dx x 3 comps

// mbarrier indices
constexpr int B_RAWF = 0, B_RAWE = 6, B_RECF = 12, B_RECE = 15, B_EF = 18, B_EE = 24, B_PF = 30, B_PE = 36,
              B_TF = 42, B_TE = 50, NBARS = 58;

template <typename TU>
struct Params {
  Grid g;
  int nwin, Lp, NQ;
  long long items;
  const TU* u;
  const float* E;
  const uint8_t* nmask;     // per node: bit c set <=> DoF 3n+c is free
  EpiDev<float> ep;
  const __nv_bfloat16* B;   // KE tile, 32 x 32 in core-matrix order
  int* err;
  const KrylovState* st;
  int nrec, nraw, ne, np;   // ring depths
  int off_rec, rec_slot, off_raw, raw_slot, off_e, e_slot, off_p, p_vec, p_slot, off_x, off_bar, off_misc;
  int poll;                 // mbarrier poll limit before giving up
  int skip;                 // test hook: the converters withhold their first arrival
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t make_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // tcgen05 descriptor version
  return d;
}

// D f32, A bf16, B bf16, both K-major, N = 32, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(IDESC), "r"(acc));
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
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

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

// AND of a predicate over the 128 reduce threads (named barrier 1); it also
// orders their shared-memory hand-off.
__device__ __forceinline__ bool red_all(bool pred) {
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

// Bounded mbarrier wait that also gives up once another role aborted.
__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* err, int poll) {
  for (int it = 0; it < poll; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 63) == 63 && *abort_flag) return false;
  }
  *abort_flag = 1;
  *(volatile int*)err = 1;  // mapped host memory: readable without a device sync
  __threadfence_system();
  return false;
}

// Step sequence of one CTA: items [lo, hi), item = w*NX + P. A run of
// items in one window covers planes [pa, pb]; it is processed as layers
// L = pa-1 (carry only) .. pb, and reads node planes pa-1 .. pb+1.
struct Seq {
  long long lo, hi;
  int NX;
  int w, pa, pb, L;
  bool ok;
  __device__ void start(long long it) {
    w = (int)(it / NX);
    pa = (int)(it - (long long)w * NX);
    const long long e = min(hi, (long long)(w + 1) * NX);
    pb = (int)(e - 1 - (long long)w * NX);
    L = pa - 1;
  }
  __device__ void init(long long lo_, long long hi_, int NX_) {
    lo = lo_;
    hi = hi_;
    NX = NX_;
    ok = lo < hi;
    if (ok) start(lo);
  }
  __device__ bool first() const { return L == pa - 1; }
  __device__ bool last() const { return L == pb; }
  __device__ int nplanes() const { return first() ? 2 : 1; }  // planes this step brings in
  __device__ void next() {
    if (L < pb) {
      ++L;
      return;
    }
    const long long nx = (long long)w * NX + pb + 1;
    if (nx >= hi) ok = false;
    else start(nx);
  }
};

// Stage global bytes [g0, g0+n) (base-relative offset off0 of a vector whose
// base is 16-byte aligned and whose length is vbytes) so that byte g0 lands
// at dst + (off0 % 16). Returns the bytes the bulk copy will deliver; bytes
// in the vector's last partial 16-byte word are copied here by plain loads.
__device__ __forceinline__ uint32_t stage_range(unsigned char* dst, const unsigned char* base, long long off0, long long n,
                                                long long vbytes) {
  if (n <= 0) return 0;
  const long long a = off0 & ~15LL;
  long long e = (off0 + n + 15) & ~15LL;
  const long long vfloor = vbytes & ~15LL;
  if (e > vfloor) {
    // tail inside the vector's last partial word: plain loads, then the bulk
    // copy stops at the last full word
    for (long long b = max(vfloor, a); b < off0 + n; ++b) dst[b - a] = base[b];
    e = vfloor;
  }
  return e > a ? (uint32_t)(e - a) : 0u;
}
__device__ __forceinline__ void issue_range(unsigned char* dst, const unsigned char* base, long long off0, uint32_t bytes,
                                            uint32_t bar) {
  if (bytes) bulk_g2s(smem_u32(dst), base + (off0 & ~15LL), bytes, bar);
}

template <Epi EPI>
__host__ __device__ constexpr int n_epi_vecs() {
  return EPI == Epi::ChebR ? 4 : (EPI == Epi::Store ? 0 : 1);
}

// q(dx,dy,dz) = dx + 2 dy + 4 dz indexes the corners; TMEM column q*4 + c.
template <typename TU, Epi EPI>
__global__ void __launch_bounds__(NT, 1) k_level0_xs(const Params<TU> P) {
  if (P.st != nullptr && P.st->done) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const Grid& g = P.g;
  const uint32_t bar0 = smem_u32(sm + P.off_bar);
  auto BAR = [&](int i) { return bar0 + 8u * (uint32_t)i; };
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + P.off_misc);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + P.off_misc + 4);
  constexpr int NV = n_epi_vecs<EPI>();

  // KE tile (B operand) at offset 0
  for (int i = tid; i < 2048 / 16; i += NT) reinterpret_cast<uint4*>(sm)[i] = reinterpret_cast<const uint4*>(P.B)[i];
  if (tid == 0) {
    for (int s = 0; s < MAXRING; ++s) {
      mbar_init(BAR(B_RAWF + s), 1);
      mbar_init(BAR(B_RAWE + s), CONV_T);
      mbar_init(BAR(B_EF + s), 1);
      mbar_init(BAR(B_EE + s), RED_T);
      mbar_init(BAR(B_PF + s), 1);
      mbar_init(BAR(B_PE + s), RED_T);
    }
    for (int s = 0; s < 3; ++s) {
      mbar_init(BAR(B_RECF + s), CONV_T);
      mbar_init(BAR(B_RECE + s), 1);
    }
    for (int s = 0; s < TSLOT; ++s) {
      mbar_init(BAR(B_TF + s), 1);
      mbar_init(BAR(B_TE + s), RED_T);
    }
    *abort_flag = 0;
  }
  if (warp == W_MMA) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;

  const int NX = g.NX, NY = g.NY, NZ = g.NZ;
  const long long lo = P.items * blockIdx.x / gridDim.x, hi = P.items * (blockIdx.x + 1) / gridDim.x;
  Seq q;
  q.init(lo, hi, NX);
  const int CS = 16 * P.Lp;           // record column stride (bytes)
  const int CPY = NROW * CS;          // record copy stride
  const int NREC = 2 * P.Lp;          // records per column and copy
  const int row3 = 3 * NZ;            // values per node row

  if (warp == W_PROD) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      long long kpl = 0, ks = 0, kp = 0;  // plane, step and epilogue-step counters
      bool ok = true;
      const unsigned char* ub = reinterpret_cast<const unsigned char*>(P.u);
      const long long ubytes = g.ndof * (long long)sizeof(TU);
      for (; q.ok && ok; q.next()) {
        const int ey0 = 15 * q.w - 1;
        for (int t = 0; t < q.nplanes() && ok; ++t, ++kpl) {
          const int Pl = q.L + (q.first() ? t : 1);
          const int s = (int)(kpl % P.nraw);
          ok = wait_bar(BAR(B_RAWE + s), (uint32_t)(((kpl / P.nraw) & 1) ^ 1), abort_flag, P.err, P.poll);
          if (!ok) break;
          unsigned char* dst = sm + P.off_raw + s * P.raw_slot;
          uint32_t bytes = 0;
          long long off0 = 0;
          if (Pl >= 0 && Pl < NX) {
            const int ra = max(ey0, 0), rb = min(ey0 + NROW, NY);
            off0 = (long long)row3 * ((long long)Pl * NY + ra) * (long long)sizeof(TU);
            bytes = stage_range(dst, ub, off0, (long long)(rb - ra) * row3 * (long long)sizeof(TU), ubytes);
          }
          mbar_arrive_tx(BAR(B_RAWF + s), bytes);
          issue_range(dst, ub, off0, bytes, BAR(B_RAWF + s));
        }
        if (!ok) break;
        {
          // moduli of layer L, window rows [ey0, ey0+16) within [0, ny)
          const int s = (int)(ks % P.ne);
          ok = wait_bar(BAR(B_EE + s), (uint32_t)(((ks / P.ne) & 1) ^ 1), abort_flag, P.err, P.poll);
          if (!ok) break;
          unsigned char* dst = sm + P.off_e + s * P.e_slot;
          uint32_t bytes = 0;
          long long off0 = 0;
          const unsigned char* eb = reinterpret_cast<const unsigned char*>(P.E);
          if (q.L >= 0 && q.L < g.nx) {
            const int ra = max(ey0, 0), rb = min(ey0 + WY, g.ny);
            off0 = 4LL * g.nz * ((long long)q.L * g.ny + ra);
            bytes = stage_range(dst, eb, off0, 4LL * (rb - ra) * g.nz, 4LL * g.nelem);
          }
          mbar_arrive_tx(BAR(B_EF + s), bytes);
          issue_range(dst, eb, off0, bytes, BAR(B_EF + s));
          ++ks;
        }
        if (!q.first()) {
          // epilogue inputs and node mask of output plane L, owned rows
          const int s = (int)(kp % P.np);
          ok = wait_bar(BAR(B_PE + s), (uint32_t)(((kp / P.np) & 1) ^ 1), abort_flag, P.err, P.poll);
          if (!ok) break;
          unsigned char* slot = sm + P.off_p + s * P.p_slot;
          const int oa = 15 * q.w, ob = min(15 * q.w + OWNR, NY);
          const long long n0 = (long long)NZ * ((long long)q.L * NY + oa);  // first owned node
          const long long nn = (long long)NZ * (ob - oa);
          const void* src[4] = {nullptr, nullptr, nullptr, nullptr};
          int esz[4] = {4, 4, 4, 4};
          if constexpr (EPI == Epi::Residual) src[0] = P.ep.b;
          if constexpr (EPI == Epi::RUpd) src[0] = P.ep.r;
          if constexpr (EPI == Epi::ChebR) {
            src[0] = P.ep.r;
            src[1] = P.ep.dinv;
            src[2] = P.ep.x;
            src[3] = P.u;
            esz[3] = (int)sizeof(TU);
          }
          uint32_t by[5] = {0, 0, 0, 0, 0};
          long long of[5] = {0, 0, 0, 0, 0};
          for (int v = 0; v < NV; ++v) {
            of[v] = 3 * n0 * esz[v];
            by[v] = stage_range(slot + v * P.p_vec, reinterpret_cast<const unsigned char*>(src[v]), of[v], 3 * nn * esz[v],
                                g.ndof * (long long)esz[v]);
          }
          of[4] = n0;
          by[4] = stage_range(slot + NV * P.p_vec, P.nmask, of[4], nn, g.nnodes);
          mbar_arrive_tx(BAR(B_PF + s), by[0] + by[1] + by[2] + by[3] + by[4]);
          for (int v = 0; v < NV; ++v)
            issue_range(slot + v * P.p_vec, reinterpret_cast<const unsigned char*>(src[v]), of[v], by[v], BAR(B_PF + s));
          issue_range(slot + NV * P.p_vec, P.nmask, of[4], by[4], BAR(B_PF + s));
          ++kp;
        }
      }
      if (!ok) {
        // drain: wait until the copies already issued have landed
        for (long long j = max(0LL, kpl - P.nraw); j < kpl; ++j)
          for (int it = 0; it < P.poll && !mbar_try(BAR(B_RAWF + (int)(j % P.nraw)), (uint32_t)((j / P.nraw) & 1)); ++it) {
          }
        for (long long j = max(0LL, ks - P.ne); j < ks; ++j)
          for (int it = 0; it < P.poll && !mbar_try(BAR(B_EF + (int)(j % P.ne)), (uint32_t)((j / P.ne) & 1)); ++it) {
          }
        for (long long j = max(0LL, kp - P.np); j < kp; ++j)
          for (int it = 0; it < P.poll && !mbar_try(BAR(B_PF + (int)(j % P.np)), (uint32_t)((j / P.np) & 1)); ++it) {
          }
      }
    }
  } else if (warp >= W_CONV && warp < W_MMA) {
    // ----------------------------------------------------------- converter
    const int ct = tid - 32 * W_CONV;
    long long kpl = 0;
    bool ok = true;
    for (; q.ok && ok; q.next()) {
      const int ey0 = 15 * q.w - 1;
      for (int t = 0; t < q.nplanes(); ++t, ++kpl) {
        const int Pl = q.L + (q.first() ? t : 1);
        const int s = (int)(kpl % P.nraw), r = (int)(kpl % P.nrec);
        ok = wait_bar(BAR(B_RAWF + s), (uint32_t)((kpl / P.nraw) & 1), abort_flag, P.err, P.poll) &&
             wait_bar(BAR(B_RECE + r), (uint32_t)(((kpl / P.nrec) & 1) ^ 1), abort_flag, P.err, P.poll);
        if (!ok) break;
        const unsigned char* raw = sm + P.off_raw + s * P.raw_slot;
        unsigned char* rec = sm + P.off_rec + r * P.rec_slot;
        const bool pv = Pl >= 0 && Pl < NX;
        const int ra = max(ey0, 0);
        const int delta =
            pv ? (int)(((long long)row3 * ((long long)Pl * NY + ra) * (long long)sizeof(TU)) & 15) : 0;
        for (int idx = ct; idx < NROW * (NREC + 1); idx += CONV_T) {
          const int rr = idx / (NREC + 1), z = idx - rr * (NREC + 1);
          const int R = ey0 + rr;
          float v0 = 0.f, v1 = 0.f, v2 = 0.f;
          if (pv && R >= 0 && R < NY && z < NZ) {
            const TU* src = reinterpret_cast<const TU*>(raw + delta) + (long long)(R - ra) * row3 + 3 * z;
            if constexpr (sizeof(TU) == 2) {
              v0 = __bfloat162float(src[0]);
              v1 = __bfloat162float(src[1]);
              v2 = __bfloat162float(src[2]);
            } else {
              v0 = src[0];
              v1 = src[1];
              v2 = src[2];
            }
          }
          const __nv_bfloat162 lo2 = __floats2bfloat162_rn(v0, v1);
          const __nv_bfloat162 hi2 = __floats2bfloat162_rn(v2, 0.0f);
          uint2 recv;
          recv.x = *reinterpret_cast<const uint32_t*>(&lo2);
          recv.y = *reinterpret_cast<const uint32_t*>(&hi2);
          if (z < NREC) *reinterpret_cast<uint2*>(rec + rr * CS + 8 * z) = recv;
          if (z >= 1) *reinterpret_cast<uint2*>(rec + CPY + rr * CS + 8 * (z - 1)) = recv;
        }
        fence_async_smem();
        mbar_arrive(BAR(B_RAWE + s));
        if (!(P.skip && kpl == 0)) mbar_arrive(BAR(B_RECF + r));
      }
    }
  } else if (warp == W_MMA) {
    // ----------------------------------------------------------------- MMA
    if (lane == 0) {
      long long kpl = 0, t = 0;
      long long last_commit = -1;
      bool ok = true;
      const uint32_t bB = smem_u32(sm);
      for (; q.ok && ok; q.next()) {
        const long long k0 = kpl + (q.first() ? 0 : -1);  // stream index of plane L
        if (q.first()) {
          ok = wait_bar(BAR(B_RECF + (int)(kpl % P.nrec)), (uint32_t)((kpl / P.nrec) & 1), abort_flag, P.err, P.poll);
          ++kpl;
          if (!ok) break;
        }
        ok = wait_bar(BAR(B_RECF + (int)(kpl % P.nrec)), (uint32_t)((kpl / P.nrec) & 1), abort_flag, P.err, P.poll);
        ++kpl;
        if (!ok) break;
        tc_fence_after();
        const uint32_t a0 = smem_u32(sm + P.off_rec + (int)(k0 % P.nrec) * P.rec_slot);
        const uint32_t a1 = smem_u32(sm + P.off_rec + (int)((k0 + 1) % P.nrec) * P.rec_slot);
        for (int qt = 0; qt < P.NQ && ok; ++qt, ++t) {
          const int ts = (int)(t % TSLOT);
          ok = wait_bar(BAR(B_TE + ts), (uint32_t)(((t / TSLOT) & 1) ^ 1), abort_flag, P.err, P.poll);
          if (!ok) break;
          tc_fence_after();
#pragma unroll
          for (int p = 0; p < 2; ++p) {
            const uint32_t d = tbase + ts * 64 + p * 32;
            const uint32_t off = p * CPY + 128 * qt;
            mma_bf16(d, make_desc(a0 + off, CS, CS), make_desc(bB, 128, 512), 0u);
            mma_bf16(d, make_desc(a1 + off, CS, CS), make_desc(bB + 256, 128, 512), 1u);
          }
          mma_commit(BAR(B_TF + ts));
          last_commit = t;
        }
        if (!ok) break;
        mma_commit(BAR(B_RECE + (int)(k0 % P.nrec)));
        if (q.last()) mma_commit(BAR(B_RECE + (int)((k0 + 1) % P.nrec)));
      }
      // never leave MMAs in flight (bounded; ignores the abort flag)
      if (last_commit >= 0) {
        const uint32_t b = BAR(B_TF + (int)(last_commit % TSLOT)), par = (uint32_t)((last_commit / TSLOT) & 1);
        for (int it = 0; it < P.poll && !mbar_try(b, par); ++it) {
        }
      }
    }
  } else {
    // -------------------------------------------------------------- reduce
    const int c = 4 * warp + (lane >> 3), zl = lane & 7;
    float* xb = reinterpret_cast<float*>(sm + P.off_x);  // [2][3 warps][8 lanes][XB_FLOATS]
    long long ks = 0, kp = 0, t = 0;
    int xbuf = 0;
    float carry[NQMAX][6];
    float carry_top[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < NQMAX; ++a)
#pragma unroll
      for (int b = 0; b < 6; ++b) carry[a][b] = 0.f;
    // node nz has a thread of its own unless the pairs end exactly at nz:
    // then the last pair's thread (tile NQ-1, zl 7) also finishes node nz
    const bool top_case = (NREC == g.nz);
    bool ok = true;
    for (; q.ok && ok; q.next()) {
      const int ey0 = 15 * q.w - 1;
      const int se = (int)(ks % P.ne);
      ok = wait_bar(BAR(B_EF + se), (uint32_t)((ks / P.ne) & 1), abort_flag, P.err, P.poll);
      const bool epi = !q.first();
      const int sp = (int)(kp % P.np);
      if (epi) ok = ok && wait_bar(BAR(B_PF + sp), (uint32_t)((kp / P.np) & 1), abort_flag, P.err, P.poll);
      const int ey = ey0 + c;
      const bool rowv = ey >= 0 && ey < g.ny && q.L >= 0 && q.L < g.nx;
      const int ra = max(ey0, 0);
      const float* Es = reinterpret_cast<const float*>(
          sm + P.off_e + se * P.e_slot +
          (rowv ? (int)((4LL * g.nz * ((long long)q.L * g.ny + ra)) & 15) : 0));
      const unsigned char* pslot = sm + P.off_p + sp * P.p_slot;
      const long long n0 = (long long)NZ * ((long long)q.L * NY + 15 * q.w);  // first owned node of plane L
      const bool own = epi && c >= 1 && ey < NY;
      const long long row_dof = 3LL * ((long long)q.L * NY + ey) * NZ;      // DoF of (L, node row ey, z = 0)
      const int lrow = (c - 1) * row3;                                       // owned-row offset in the staged inputs
      float zc[2][2][3];
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
          for (int cc = 0; cc < 3; ++cc) zc[a][b][cc] = 0.f;
#pragma unroll
      for (int qt = 0; qt < NQMAX; ++qt) {
        if (qt >= P.NQ) break;
        const int j = 8 * qt + zl;
        const int ts = (int)(t % TSLOT);
        ok = ok && wait_bar(BAR(B_TF + ts), (uint32_t)((t / TSLOT) & 1), abort_flag, P.err, P.poll);
        ++t;
        tc_fence_after();
        float A[32], Bv[32];
        const uint32_t ta = tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)(ts * 64);
        tmem_ld32(ta, A);
        tmem_ld32(ta + 32, Bv);
        tmem_wait_ld();
        tc_fence_before();
        mbar_arrive(BAR(B_TE + ts));
        const int za = 2 * j, zb = 2 * j + 1;
        const float Ea = (rowv && za < g.nz) ? Es[(ey - ra) * g.nz + za] : 0.f;
        const float Eb = (rowv && zb < g.nz) ? Es[(ey - ra) * g.nz + zb] : 0.f;
        const bool top = top_case && qt == P.NQ - 1;  // warp-uniform
        // N0/N1: nodes z = 2j, 2j+1; N2: the z = 2j+2 share for the next pair
        float N0[2][2][3], N1[2][2][3], N2[2][2][3];
#pragma unroll
        for (int dx = 0; dx < 2; ++dx)
#pragma unroll
          for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
              const int i0 = (dx + 2 * dy) * 4 + cc, i1 = (dx + 2 * dy + 4) * 4 + cc;
              const float n2 = Eb * Bv[i1];
              const float up = __shfl_up_sync(0xffffffffu, n2, 1);
              const float dn = __shfl_down_sync(0xffffffffu, n2, 7);
              N0[dx][dy][cc] = fmaf(Ea, A[i0], zl > 0 ? up : zc[dx][dy][cc]);
              N1[dx][dy][cc] = fmaf(Ea, A[i1], Eb * Bv[i0]);
              N2[dx][dy][cc] = n2;
              zc[dx][dy][cc] = dn;  // meaningful in the group's first lane, for the next tile
            }
        // y: node row c = dy0 shares of element row c + dy1 shares of row c-1
        float* xw = xb + ((xbuf * 3 + min(warp, 2)) * 8 + zl) * XB_FLOATS;
        if (warp < 3 && lane >= 24) {
#pragma unroll
          for (int dx = 0; dx < 2; ++dx)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
              xw[dx * 3 + cc] = N0[dx][1][cc];
              xw[6 + dx * 3 + cc] = N1[dx][1][cc];
              if (top) xw[12 + dx * 3 + cc] = N2[dx][1][cc];
            }
        }
        float Y0[2][3], Y1[2][3], Y2[2][3];
#pragma unroll
        for (int dx = 0; dx < 2; ++dx)
#pragma unroll
          for (int cc = 0; cc < 3; ++cc) {
            Y0[dx][cc] = __shfl_up_sync(0xffffffffu, N0[dx][1][cc], 8);
            Y1[dx][cc] = __shfl_up_sync(0xffffffffu, N1[dx][1][cc], 8);
            Y2[dx][cc] = top ? __shfl_up_sync(0xffffffffu, N2[dx][1][cc], 8) : 0.f;
          }
        ok = red_all(ok);  // also publishes the hand-off rows
        if (!ok) break;
        if (lane < 8) {
          if (warp >= 1) {
            const float* xr = xb + ((xbuf * 3 + warp - 1) * 8 + zl) * XB_FLOATS;
#pragma unroll
            for (int dx = 0; dx < 2; ++dx)
#pragma unroll
              for (int cc = 0; cc < 3; ++cc) {
                Y0[dx][cc] = xr[dx * 3 + cc];
                Y1[dx][cc] = xr[6 + dx * 3 + cc];
                if (top) Y2[dx][cc] = xr[12 + dx * 3 + cc];
              }
          } else {
#pragma unroll
            for (int dx = 0; dx < 2; ++dx)
#pragma unroll
              for (int cc = 0; cc < 3; ++cc) Y0[dx][cc] = Y1[dx][cc] = Y2[dx][cc] = 0.f;
          }
        }
        xbuf ^= 1;
        // x: plane L = dx0 part of layer L + dx1 part of layer L-1 (carry)
        float out[9];
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          out[cc] = N0[0][0][cc] + Y0[0][cc] + carry[qt][cc];
          out[3 + cc] = N1[0][0][cc] + Y1[0][cc] + carry[qt][3 + cc];
          carry[qt][cc] = N0[1][0][cc] + Y0[1][cc];
          carry[qt][3 + cc] = N1[1][0][cc] + Y1[1][cc];
          if (top) {
            out[6 + cc] = N2[0][0][cc] + Y2[0][cc] + carry_top[cc];
            carry_top[cc] = N2[1][0][cc] + Y2[1][cc];
          } else {
            out[6 + cc] = 0.f;
          }
        }
        if (own) {
          const int nnodes_here = (top && zl == 7) ? 3 : 2;
#pragma unroll
          for (int tn = 0; tn < 3; ++tn) {
            if (tn >= nnodes_here) break;
            const int z = 2 * j + tn;
            if (z > g.nz) break;
            const uint8_t mw = pslot[NV * P.p_vec + (int)(n0 & 15) + (c - 1) * NZ + z];
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
              const long long i = row_dof + 3 * z + cc;
              if (!topo_in_range(i, g.ndof)) continue;
              const int li = lrow + 3 * z + cc;
              const bool fr = (mw >> cc) & 1;
              const float acc = out[3 * tn + cc];
              if constexpr (EPI == Epi::Store) {
                P.ep.y[i] = fr ? acc : 0.f;
              } else if constexpr (EPI == Epi::Residual) {
                const float bv = reinterpret_cast<const float*>(pslot + (int)((12 * n0) & 15))[li];
                P.ep.y[i] = fr ? bv - acc : 0.f;
              } else if constexpr (EPI == Epi::RUpd) {
                const float rv = reinterpret_cast<const float*>(pslot + (int)((12 * n0) & 15))[li];
                P.ep.r[i] = fr ? rv - P.ep.s * acc : 0.f;
              } else if constexpr (EPI == Epi::ChebR) {
                const float r0 = reinterpret_cast<const float*>(pslot + (int)((12 * n0) & 15))[li];
                const float dv = reinterpret_cast<const float*>(pslot + P.p_vec + (int)((12 * n0) & 15))[li];
                const float xv = reinterpret_cast<const float*>(pslot + 2 * P.p_vec + (int)((12 * n0) & 15))[li];
                float uv;
                if constexpr (sizeof(TU) == 2)
                  uv = __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(pslot + 3 * P.p_vec + (int)((6 * n0) & 15))[li]);
                else
                  uv = reinterpret_cast<const float*>(pslot + 3 * P.p_vec + (int)((12 * n0) & 15))[li];
                if (fr) {
                  const float rv = r0 - P.ep.s * acc;
                  P.ep.r[i] = rv;
                  const float dn = P.ep.c1 * uv + P.ep.c2 * (dv * rv);
                  P.ep.d_out[i] = dn;
                  P.ep.x[i] = xv + P.ep.ax * dn;
                } else {
                  P.ep.r[i] = 0.f;
                  P.ep.d_out[i] = 0.f;
                }
              }
            }
          }
        }
      }
      if (!ok) break;
      // the staged E and epilogue inputs are read: hand the slots back to TMA
      fence_async_smem();
      mbar_arrive(BAR(B_EE + se));
      ++ks;
      if (epi) {
        mbar_arrive(BAR(B_PE + sp));
        ++kp;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == W_MMA) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(512));
}

}  // namespace xs
}  // namespace topo

namespace topo {

// ----------------------------------------------------------------- host side
// Everything the kernel needs beyond its arguments is held per device: the
// KE tile (B operand), the error flag, the SM count, and which kernel
// instances have had their shared-memory limit raised on that device. A
// context on device d only ever sees device d's entries.
namespace {
struct XsDevice {
  __nv_bfloat16* B = nullptr;
  int* err = nullptr;       // device alias of err_host
  int* err_host = nullptr;
  int nsm = 0;
  uint32_t attr_done = 0;  // bit per kernel instance
};
std::mutex g_xs_mu;
std::vector<XsDevice> g_xs;
int g_xs_skip = 0;         // test hook (topo_debug_tc_wait)
int g_xs_poll = 1 << 22;   // mbarrier poll limit

XsDevice& xs_device() {
  int dev = 0;
  TOPO_CUDA_CHECK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_xs_mu);
  if ((int)g_xs.size() <= dev) g_xs.resize(dev + 1);
  XsDevice& d = g_xs[dev];
  if (d.nsm == 0) TOPO_CUDA_CHECK(cudaDeviceGetAttribute(&d.nsm, cudaDevAttrMultiProcessorCount, dev));
  return d;
}

uint16_t bf16_bits_rne(float f) {
  uint32_t b;
  std::memcpy(&b, &f, 4);
  b = (b + 0x7FFFu + ((b >> 16) & 1u)) >> 16;
  return (uint16_t)b;
}

struct XsLayout {
  int nrec, nraw, ne, np;
  int off_rec, rec_slot, off_raw, raw_slot, off_e, e_slot, off_p, p_vec, p_slot, off_x, off_bar, off_misc;
  int total;
};

constexpr int kSmemMax = 232448 - 1024;  // opt-in limit minus the 1024-byte alignment slack
constexpr int kOneCtaPerSm = 120 * 1024;  // > half of the 228 KB an SM holds

int al128(long long x) { return (int)((x + 127) & ~127LL); }

bool xs_layout(const Grid& g, int Lp, int usz, int nvec, XsLayout& L) {
  const int rec_slot = 2 * xs::NROW * 16 * Lp;
  const int raw_slot = al128(3LL * g.NZ * xs::NROW * usz + 32);
  const int e_slot = al128(4LL * xs::WY * g.nz + 32);
  const int p_vec = al128(12LL * xs::OWNR * g.NZ + 32);  // FP32 vectors (a BF16 u takes half of its slot)
  const int p_slot = nvec * p_vec + al128((long long)xs::OWNR * g.NZ + 32);
  const int fixed = 2048 + al128(2 * 3 * 8 * xs::XB_FLOATS * 4) + al128(xs::NBARS * 8) + 128;
  // deepest rings that fit, preferring three record planes
  const int pref[][4] = {{3, 4, 4, 3}, {3, 3, 3, 2}, {3, 2, 2, 2}, {2, 2, 2, 2}};
  for (const auto& p : pref) {
    const int total = fixed + p[0] * rec_slot + p[1] * raw_slot + p[2] * e_slot + p[3] * p_slot;
    if (total <= kSmemMax) {
      L.nrec = p[0];
      L.nraw = p[1];
      L.ne = p[2];
      L.np = p[3];
      int o = 2048;
      L.off_rec = o;
      L.rec_slot = rec_slot;
      o += L.nrec * rec_slot;
      L.off_raw = o;
      L.raw_slot = raw_slot;
      o += L.nraw * raw_slot;
      L.off_e = o;
      L.e_slot = e_slot;
      o += L.ne * e_slot;
      L.off_p = o;
      L.p_vec = p_vec;
      L.p_slot = p_slot;
      o += L.np * p_slot;
      L.off_x = o;
      o += al128(2 * 3 * 8 * xs::XB_FLOATS * 4);
      L.off_bar = o;
      o += al128(xs::NBARS * 8);
      L.off_misc = o;
      o += 128;
      L.total = o;
      return true;
    }
  }
  return false;
}

template <typename TU, Epi EPI>
void launch_xs(const Grid& g, const void* u, const void* E, const uint8_t* nmask, void* y, const EpiArgs& ea,
               cudaStream_t s) {
  XsDevice& d = xs_device();
  if (!d.B) throw std::runtime_error("tensor-core operator not prepared on this device");
  const int NQ = (g.nz + 15) / 16, Lp = 8 * NQ;
  XsLayout L;
  if (NQ > xs::NQMAX || !xs_layout(g, Lp, (int)sizeof(TU), xs::n_epi_vecs<EPI>(), L))
    throw std::runtime_error("level0 tensor-core K.u: mesh not supported (nz must be <= 80)");
  constexpr int inst = (int)EPI * 2 + (sizeof(TU) == 2 ? 1 : 0);
  if (!(d.attr_done & (1u << inst))) {
    TOPO_CUDA_CHECK(
        cudaFuncSetAttribute(xs::k_level0_xs<TU, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemMax + 1024));
    std::lock_guard<std::mutex> lk(g_xs_mu);
    d.attr_done |= 1u << inst;
  }
  // Each CTA allocates all 512 tensor-memory columns, so no two may share an
  // SM: ask for more than half of the SM's shared memory even when the rings
  // need less (a second CTA would otherwise wait in tcgen05.alloc).
  const int smem = std::max(L.total + 1024, kOneCtaPerSm);
  xs::Params<TU> P;
  P.g = g;
  P.nwin = (g.NY + xs::OWNR - 1) / xs::OWNR;
  P.Lp = Lp;
  P.NQ = NQ;
  P.items = (long long)P.nwin * g.NX;
  P.u = (const TU*)u;
  P.E = (const float*)E;
  P.nmask = nmask;
  P.ep = make_epi<float>(y, ea);
  P.B = d.B;
  P.err = d.err;
  P.st = ea.st;
  P.nrec = L.nrec;
  P.nraw = L.nraw;
  P.ne = L.ne;
  P.np = L.np;
  P.off_rec = L.off_rec;
  P.rec_slot = L.rec_slot;
  P.off_raw = L.off_raw;
  P.raw_slot = L.raw_slot;
  P.off_e = L.off_e;
  P.e_slot = L.e_slot;
  P.off_p = L.off_p;
  P.p_vec = L.p_vec;
  P.p_slot = L.p_slot;
  P.off_x = L.off_x;
  P.off_bar = L.off_bar;
  P.off_misc = L.off_misc;
  P.poll = g_xs_poll;
  P.skip = g_xs_skip;
  const int grid = (int)std::min<long long>(P.items, d.nsm);
  xs::k_level0_xs<TU, EPI><<<grid, xs::NT, smem, s>>>(P);
  TOPO_LAUNCH_CHECK();
}
}  // namespace

bool level0_xs_supported(const Grid& g) { return g.nz <= 16 * xs::NQMAX; }

// B operand of the streaming kernel: row n = output (corner q = dx+2dy+4dz,
// component), column k = input (dx = k/16, dy = (k/8)%2, dz = (k%8)/4,
// component k%4); component 3 is padding. Laid out as 8x8 core matrices
// (N-group stride 512 B, K-chunk stride 128 B), rounded to BF16.
void xs_prepare(const double* KE) {
  auto cid = [](int dx, int dy, int dz) { return dz * 4 + (dy ? (dx ? 2 : 3) : (dx ? 1 : 0)); };
  uint16_t h[1024];
  for (int n = 0; n < 32; ++n)
    for (int k = 0; k < 32; ++k) {
      const int qo = n / 4, co = n % 4;
      const int dxi = k / 16, dyi = (k / 8) % 2, dzi = (k % 8) / 4, ci = k % 4;
      double v = 0.0;
      if (co < 3 && ci < 3) {
        const int a = cid(qo & 1, (qo >> 1) & 1, qo >> 2);
        const int b = cid(dxi, dyi, dzi);
        v = KE[(3 * a + co) * 24 + 3 * b + ci];
      }
      h[(n / 8) * 256 + (k / 8) * 64 + (n % 8) * 8 + (k % 8)] = bf16_bits_rne((float)v);
    }
  XsDevice& d = xs_device();
  if (!d.B) TOPO_CUDA_CHECK(cudaMalloc(&d.B, sizeof(h)));
  if (!d.err) {
    // Pinned, mapped host word: kernels store 1 through the device alias and
    // the host reads it without synchronising the stream.
    TOPO_CUDA_CHECK(cudaHostAlloc(&d.err_host, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable));
    *(volatile int*)d.err_host = 0;
    TOPO_CUDA_CHECK(cudaHostGetDevicePointer((void**)&d.err, d.err_host, 0));
  }
  TOPO_CUDA_CHECK(cudaMemcpy(d.B, h, sizeof(h), cudaMemcpyHostToDevice));
}

// BF16-input K.u streaming along x. u_bf16: u stored as BF16 (else FP32,
// rounded when staged). nmask: per-node free bits (bit c = DoF 3n+c). Every
// pointer must be 16-byte aligned. Epilogues: Store, Residual, RUpd, ChebR.
void level0_apply_xs(bool u_bf16, const Grid& g, const void* u, const void* E, const uint8_t* nmask, void* y, Epi epi,
                     const EpiArgs& ea, cudaStream_t s) {
  auto al = [](const void* p) { return p == nullptr || ((uintptr_t)p & 15) == 0; };
  if (!al(u) || !al(E) || !al(nmask) || !al(ea.b) || !al(ea.r) || !al(ea.dinv) || !al(ea.x))
    throw std::runtime_error("level0 tensor-core K.u: vectors must be 16-byte aligned");
#define TOPO_XS_CASE(EP)                                                     \
  case Epi::EP:                                                              \
    if (u_bf16) launch_xs<__nv_bfloat16, Epi::EP>(g, u, E, nmask, y, ea, s); \
    else launch_xs<float, Epi::EP>(g, u, E, nmask, y, ea, s);                \
    break;
  switch (epi) {
    TOPO_XS_CASE(Store)
    TOPO_XS_CASE(Residual)
    TOPO_XS_CASE(RUpd)
    TOPO_XS_CASE(ChebR)
    default:
      throw std::runtime_error("level0 tensor-core K.u: unsupported epilogue");
  }
#undef TOPO_XS_CASE
}

// Returns and clears this device's flag, set when an mbarrier wait timed out.
// sync: wait for the stream first, so launches already queued on it count;
// otherwise only launches that have finished are seen (no host stall).
int xs_error_flag(cudaStream_t s, bool sync) {
  XsDevice& d = xs_device();
  if (!d.err_host) return 0;
  if (sync) TOPO_CUDA_CHECK(cudaStreamSynchronize(s));
  volatile int* f = d.err_host;
  const int h = *f;
  if (h) *f = 0;
  return h;
}

// The device's wait-timeout flag shared by the streaming kernels (allocated
// when the device's KE tile is prepared, so never during a stream capture).
int* wait_error_flag() {
  XsDevice& d = xs_device();
  if (!d.err) throw std::runtime_error("streaming K.u: device not prepared");
  return d.err;
}

void xs_debug(int skip_first_arrival, int poll_limit) {
  std::lock_guard<std::mutex> lk(g_xs_mu);
  g_xs_skip = skip_first_arrival ? 1 : 0;
  g_xs_poll = poll_limit > 0 ? poll_limit : (1 << 22);
}

TOPO_BOUNDS_READER(bounds_flag_xs)

}  // namespace topo
