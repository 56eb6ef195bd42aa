// kmatvec_xs.cu - level-0 hex8 K.u with BF16 inputs on the tcgen05 tensor
// cores (FP32 accumulation in tensor memory), streaming along x.
//
// Memory order of every level-0 vector is z fastest (DoF 3*node+c, node
// (ix*NY+iy)*NZ+iz), so one x-plane of a window of consecutive y-rows is one
// contiguous range. The kernel is built around that:
//
//  * Work item = (window w, node plane x). A window owns the 16 node rows
//    16w .. 16w+15 and stages node rows 16w-1 .. 16w+16 and element rows
//    16w-1 .. 16w+15. A persistent CTA takes a contiguous range of items
//    (window-major) and walks the planes of each window in x: output plane
//    x reads node planes x-1, x, x+1 and element layers x-1, x, so every
//    plane is brought in once per run.
//  * Producer warp, two threads with streams of their own: per node plane
//    one cp.async.bulk (TMA, no multicast) of the window's 18 node rows of u,
//    and per element layer one of its 17 rows of E, into shared-memory rings
//    completed on mbarriers.
//    Copies round their start down to 16 bytes; a range ending inside the
//    last 16 bytes of a vector gets its tail by plain loads, so nothing
//    outside a vector is read.
//  * Converter warps: raw u -> BF16 node records (ux, uy, uz, 0), 8 bytes,
//    node z at record z+1 of its row (record 0 = node -1 = zero), so the
//    16-byte pair p holds nodes 2p-1, 2p.
//  * MMA thread: an MMA row is one node z-pair (nodes 2j, 2j+1) of one owned
//    row; a tile is 128 rows = 16 rows (core-matrix groups, stride = row
//    stride) x 8 z-pairs. Node n sits at local corner (ax, ay, az) of element
//    n - (ax, ay, az). For each xy-corner (ax, ay) four
//    tcgen05.mma.kind::f16 (M=128, N=16, K=16) accumulate into one 16-column
//    slice: K = (dy, two records, component) with the records of pair j (po
//    = 0) or j+1 (po = 1), i.e. nodes 2j-1 .. 2j+2 of the row y-ay+dy of
//    plane x-ax+dx; within one MMA the K step dy=0 -> dy=1 is the next row,
//    so LBO = SBO = row stride. The B tile holds KE so that output column
//    (t, az, c) receives the local output of node 2j+t, component c, of the
//    element below (az = 1) or at (az = 0) the node in z: both z-elements of
//    a node stay apart, in FP32, ready for their own E.
//  * Epilogue warps (two groups of four, alternate tiles; lane = node pair):
//    read the four slices, y(node) = sum over the 8 elements of
//    E_e * (K_e u_e)[node] with E from the staged layers, and finish the
//    node with the epilogue (Store / Residual / RUpd / ChebR), reading its
//    inputs straight from global memory.
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

constexpr int WY = 16;          // owned node rows per window = core-matrix groups of an MMA tile
constexpr int SROW = WY + 2;    // staged node rows
constexpr int EROW = WY + 1;    // staged element rows
constexpr int TSLOT = 8;        // TMEM ring: 8 slots x 64 columns
constexpr int NREC = 6, NRAW = 3, NE = 6;  // deepest rings: record planes, raw planes, E layers
constexpr int W_EPI = 8, W_CONV = 6;
constexpr int W_MMA = W_EPI + W_CONV, W_PROD = W_MMA + 1;
constexpr int NT = 32 * (W_PROD + 1);  // 16 warps
constexpr int EPI_T = 32 * W_EPI, CONV_T = 32 * W_CONV, GRP_T = 128;
constexpr int BTILE = 512;      // bytes of one B tile (16 x 16 BF16)
constexpr int NBT = 18;         // B tiles (16 x 16 each) of the ten MMAs of a tile

// mbarrier indices
constexpr int B_RAWF = 0, B_RAWE = B_RAWF + NRAW, B_RECF = B_RAWE + NRAW, B_RECE = B_RECF + NREC,
              B_EF = B_RECE + NREC, B_EE = B_EF + NE, B_TF = B_EE + NE, B_TE = B_TF + TSLOT,
              NBARS = B_TE + TSLOT;

template <typename TU>
struct Params {
  Grid g;
  int nwin, NQ;
  long long items;
  const TU* u;
  const float* E;
  const uint8_t* nmask;     // per node: bit c set <=> DoF 3n+c is free
  EpiDev<float> ep;
  const __nv_bfloat16* B;   // KE tiles in core-matrix order
  int* err;
  const KrylovState* st;
  int CS, nrecs;            // record row stride (bytes), records per row
  int nrec, nraw, ne;       // ring depths in use (<= NREC, NRAW, NE)
  int off_rec, rec_slot, off_raw, raw_slot, off_e, e_slot, off_bar, off_misc;
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

// D f32, A bf16, B bf16, both K-major, M = 128, N = 16 or 32.
__host__ __device__ constexpr uint32_t idesc_n(uint32_t n) { return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24); }

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
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

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

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

// Runs of one CTA: items [lo, hi), item = w*NX + x. A run is the output
// planes xa .. xb of one window; it reads node planes xa-1 .. xb+1 and
// element layers xa-1 .. xb.
struct Run {
  long long lo, hi, it;
  int NX;
  int w, xa, xb;
  __device__ void init(long long lo_, long long hi_, int NX_) {
    lo = lo_;
    hi = hi_;
    NX = NX_;
    it = lo;
  }
  __device__ bool next() {
    if (it >= hi) return false;
    w = (int)(it / NX);
    xa = (int)(it - (long long)w * NX);
    const long long e = min(hi, (long long)(w + 1) * NX);
    xb = (int)(e - 1 - (long long)w * NX);
    it = e;
    return true;
  }
};

// Stage global bytes [off0, off0+n) of a vector (16-byte aligned base,
// length vbytes) so that byte off0 lands at dst + (off0 % 16). Returns the
// bytes the bulk copy will deliver; bytes in the vector's last partial
// 16-byte word are copied here by plain loads.
__device__ __forceinline__ uint32_t stage_range(unsigned char* dst, const unsigned char* base, long long off0, long long n,
                                                long long vbytes) {
  if (n <= 0) return 0;
  const long long a = off0 & ~15LL;
  long long e = (off0 + n + 15) & ~15LL;
  const long long vfloor = vbytes & ~15LL;
  if (e > vfloor) {
    for (long long b = max(vfloor, a); b < off0 + n; ++b) dst[b - a] = base[b];
    e = vfloor;
  }
  return e > a ? (uint32_t)(e - a) : 0u;
}
__device__ __forceinline__ void issue_range(unsigned char* dst, const unsigned char* base, long long off0, uint32_t bytes,
                                            uint32_t bar) {
  if (bytes) bulk_g2s(smem_u32(dst), base + (off0 & ~15LL), bytes, bar);
}

template <typename TU>
__device__ __forceinline__ float to_f(TU v) {
  if constexpr (sizeof(TU) == 2) return __bfloat162float(v);
  else return v;
}

// Tile of 128 rows (16 owned rows x 8 z-pairs): D slices S0..S3 = corners
// (ax, ay) = (0,0), (1,0), (1,1), (0,1) at TMEM columns 64*slot + 0, 16, 32,
// 48; slice column (t, az, c) -> 6t + 3az + c. The A operand (plane x-ax+dx,
// row y-ay+dy) depends on the plane p in {x-1, x, x+1} and delta = dy-ay only,
// so nine operands cover the 16 (corner, dx, dy) products; each MMA writes
// the slices its operand feeds (adjacent by the slice order, except the
// (x+1, 0) operand, which feeds S0 and S3 in two MMAs; the B tiles between
// them are zero and unused).
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

  for (int i = tid; i < NBT * BTILE / 16; i += NT) reinterpret_cast<uint4*>(sm)[i] = reinterpret_cast<const uint4*>(P.B)[i];
  if (tid == 0) {
    for (int s = 0; s < NRAW; ++s) {
      mbar_init(BAR(B_RAWF + s), 1);
      mbar_init(BAR(B_RAWE + s), CONV_T);
    }
    for (int s = 0; s < NREC; ++s) {
      mbar_init(BAR(B_RECF + s), CONV_T);
      mbar_init(BAR(B_RECE + s), 1);
    }
    for (int s = 0; s < NE; ++s) {
      mbar_init(BAR(B_EF + s), 1);
      mbar_init(BAR(B_EE + s), EPI_T);
    }
    for (int s = 0; s < TSLOT; ++s) {
      mbar_init(BAR(B_TF + s), 1);
      mbar_init(BAR(B_TE + s), GRP_T);
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
  Run run;
  run.init(lo, hi, NX);
  const int CS = P.CS;
  const int row3 = 3 * NZ;

  if (warp == W_PROD) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      // node planes of u (raw, converted by the converter warps)
      long long kr = 0;
      bool ok = true;
      const unsigned char* ub = reinterpret_cast<const unsigned char*>(P.u);
      const long long ubytes = g.ndof * (long long)sizeof(TU);
      while (ok && run.next()) {
        const int ya = max(WY * run.w - 1, 0), yb = min(WY * run.w + WY + 1, NY);  // staged node rows
        const int nout = run.xb - run.xa + 1;
        for (int i = 0; i <= nout + 1 && ok; ++i) {
          const int Pl = run.xa - 1 + i;
          const int s = (int)(kr % P.nraw);
          ok = wait_bar(BAR(B_RAWE + s), (uint32_t)(((kr / P.nraw) & 1) ^ 1), abort_flag, P.err, P.poll);
          if (!ok) break;
          unsigned char* dst = sm + P.off_raw + s * P.raw_slot;
          uint32_t bytes = 0;
          long long off0 = 0;
          if (Pl >= 0 && Pl < NX && yb > ya) {
            off0 = (long long)row3 * ((long long)Pl * NY + ya) * (long long)sizeof(TU);
            bytes = stage_range(dst, ub, off0, (long long)(yb - ya) * row3 * (long long)sizeof(TU), ubytes);
          }
          mbar_arrive_tx(BAR(B_RAWF + s), bytes);
          issue_range(dst, ub, off0, bytes, BAR(B_RAWF + s));
          ++kr;
        }
      }
      if (!ok)  // drain: wait until the copies already issued have landed
        for (long long j = max(0LL, kr - (long long)P.nraw); j < kr; ++j)
          for (int it = 0; it < P.poll && !mbar_try(BAR(B_RAWF + (int)(j % P.nraw)), (uint32_t)((j / P.nraw) & 1)); ++it) {
          }
    }
    if (lane == 1) {
      // element layers of E (a stream of its own, so a full E ring never
      // holds back the next node plane)
      long long ke = 0;
      bool ok = true;
      const unsigned char* ebp = reinterpret_cast<const unsigned char*>(P.E);
      while (ok && run.next()) {
        const int ea = max(WY * run.w - 1, 0), eb = min(WY * run.w + WY, g.ny);  // staged element rows
        const int nout = run.xb - run.xa + 1;
        for (int i = 0; i <= nout && ok; ++i) {
          const int L = run.xa - 1 + i;
          const int s = (int)(ke % P.ne);
          ok = wait_bar(BAR(B_EE + s), (uint32_t)(((ke / P.ne) & 1) ^ 1), abort_flag, P.err, P.poll);
          if (!ok) break;
          unsigned char* dst = sm + P.off_e + s * P.e_slot;
          uint32_t bytes = 0;
          long long off0 = 0;
          if (L >= 0 && L < g.nx && eb > ea) {
            off0 = 4LL * g.nz * ((long long)L * g.ny + ea);
            bytes = stage_range(dst, ebp, off0, 4LL * (eb - ea) * g.nz, 4LL * g.nelem);
          }
          mbar_arrive_tx(BAR(B_EF + s), bytes);
          issue_range(dst, ebp, off0, bytes, BAR(B_EF + s));
          ++ke;
        }
      }
      if (!ok)
        for (long long j = max(0LL, ke - (long long)P.ne); j < ke; ++j)
          for (int it = 0; it < P.poll && !mbar_try(BAR(B_EF + (int)(j % P.ne)), (uint32_t)((j / P.ne) & 1)); ++it) {
          }
    }
  } else if (warp >= W_EPI && warp < W_MMA) {
    // ----------------------------------------------------------- converter
    const int ct = tid - 32 * W_EPI;
    long long kr = 0;
    bool ok = true;
    while (ok && run.next()) {
      const int y0 = WY * run.w - 1;  // node row of staged row 0
      const int ya = max(y0, 0);
      const int nout = run.xb - run.xa + 1;
      for (int i = 0; i <= nout + 1; ++i, ++kr) {
        const int Pl = run.xa - 1 + i;
        const int s = (int)(kr % P.nraw), r = (int)(kr % P.nrec);
        ok = wait_bar(BAR(B_RAWF + s), (uint32_t)((kr / P.nraw) & 1), abort_flag, P.err, P.poll) &&
             wait_bar(BAR(B_RECE + r), (uint32_t)(((kr / P.nrec) & 1) ^ 1), abort_flag, P.err, P.poll);
        if (!ok) break;
        const unsigned char* raw = sm + P.off_raw + s * P.raw_slot;
        unsigned char* rec = sm + P.off_rec + r * P.rec_slot;
        const bool pv = Pl >= 0 && Pl < NX;
        const int delta = pv ? (int)(((long long)row3 * ((long long)Pl * NY + ya) * (long long)sizeof(TU)) & 15) : 0;
        const TU* src0 = reinterpret_cast<const TU*>(raw + delta);
        // 16-byte pair pp of staged row rr holds nodes 2pp-1, 2pp; thread ct
        // walks (rr, pp) = divmod(ct + CONV_T k, npairs) incrementally
        const int npairs = P.nrecs >> 1;
        int rr = ct / npairs, pp = ct - rr * npairs;
        const int drr = CONV_T / npairs, dpp = CONV_T - drr * npairs;
        for (; rr < SROW; rr += drr, pp += dpp) {
          if (pp >= npairs) {
            pp -= npairs;
            ++rr;
            if (rr >= SROW) break;
          }
          const int y = y0 + rr;
          const bool rv = pv && y >= 0 && y < NY;
          float v[6];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int z = 2 * pp - 1 + h;
            const bool in = rv && z >= 0 && z < NZ;
            const TU* src = src0 + (long long)(y - ya) * row3 + 3 * z;
            v[3 * h] = in ? to_f(src[0]) : 0.f;
            v[3 * h + 1] = in ? to_f(src[1]) : 0.f;
            v[3 * h + 2] = in ? to_f(src[2]) : 0.f;
          }
          const __nv_bfloat162 w0 = __floats2bfloat162_rn(v[0], v[1]);
          const __nv_bfloat162 w1 = __floats2bfloat162_rn(v[2], 0.0f);
          const __nv_bfloat162 w2 = __floats2bfloat162_rn(v[3], v[4]);
          const __nv_bfloat162 w3 = __floats2bfloat162_rn(v[5], 0.0f);
          uint4 rec4;
          rec4.x = *reinterpret_cast<const uint32_t*>(&w0);
          rec4.y = *reinterpret_cast<const uint32_t*>(&w1);
          rec4.z = *reinterpret_cast<const uint32_t*>(&w2);
          rec4.w = *reinterpret_cast<const uint32_t*>(&w3);
          *reinterpret_cast<uint4*>(rec + rr * CS + 16 * pp) = rec4;
        }
        fence_async_smem();
        mbar_arrive(BAR(B_RAWE + s));
        if (!(P.skip && kr == 0)) mbar_arrive(BAR(B_RECF + r));
      }
    }
  } else if (warp == W_MMA) {
    // ----------------------------------------------------------------- MMA
    if (lane == 0) {
      long long kr = 0, t = 0, last_commit = -1;
      bool ok = true;
      const uint32_t bB = smem_u32(sm);
      const uint32_t rec0 = smem_u32(sm + P.off_rec);
      // B operand starting at tile i: address field + 32 i (512 B per tile)
      const uint64_t bd0 = make_desc(bB, 128, 256);
      auto bd = [&](int i) { return bd0 + (uint64_t)(i * (BTILE >> 4)); };
      while (ok && run.next()) {
        const int nout = run.xb - run.xa + 1;
        const long long k0 = kr;  // stream index of node plane xa-1
        for (int i = 0; i < 2 && ok; ++i)
          ok = wait_bar(BAR(B_RECF + (int)((k0 + i) % P.nrec)), (uint32_t)(((k0 + i) / P.nrec) & 1), abort_flag, P.err,
                        P.poll);
        for (int o = 0; o < nout && ok; ++o) {
          const long long kp = k0 + o;  // node plane x-1
          ok = wait_bar(BAR(B_RECF + (int)((kp + 2) % P.nrec)), (uint32_t)(((kp + 2) / P.nrec) & 1), abort_flag, P.err,
                        P.poll);
          if (!ok) break;
          tc_fence_after();
          // A descriptors of planes x-1, x, x+1 at row offset delta = -1, 0, 1
          // (K = two consecutive z-pairs, LBO 16 B); a tile adds 8 qt pairs
          // (+16 B each) to the address field
          uint64_t ab[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) ab[d] = make_desc(rec0 + (uint32_t)((kp + d) % P.nrec) * (uint32_t)P.rec_slot, 16, CS);
          const uint64_t cs16 = (uint64_t)(CS >> 4);
          auto ad = [&](int d, int dl) { return ab[d] + (uint64_t)dl * cs16; };
          for (int qt = 0; qt < P.NQ && ok; ++qt, ++t) {
            const int ts = (int)(t % TSLOT);
            ok = wait_bar(BAR(B_TE + ts), (uint32_t)(((t / TSLOT) & 1) ^ 1), abort_flag, P.err, P.poll);
            if (!ok) break;
            tc_fence_after();
            const uint32_t d0 = tbase + (uint32_t)(ts * 64);
            const uint64_t qa = (uint64_t)(8 * qt);
            // the nine (plane, delta) operands; slices S0..S3 = corners
            // (0,0), (1,0), (1,1), (0,1) at columns 0, 16, 32, 48
            mma_bf16(d0, ad(1, 1) + qa, bd(0), idesc_n(64), 0u);
            mma_bf16(d0, ad(1, 2) + qa, bd(4), idesc_n(32), 1u);
            mma_bf16(d0 + 32, ad(1, 0) + qa, bd(6), idesc_n(32), 1u);
            mma_bf16(d0, ad(2, 1) + qa, bd(8), idesc_n(16), 1u);
            mma_bf16(d0 + 48, ad(2, 1) + qa, bd(11), idesc_n(16), 1u);
            mma_bf16(d0 + 16, ad(0, 1) + qa, bd(12), idesc_n(32), 1u);
            mma_bf16(d0, ad(2, 2) + qa, bd(14), idesc_n(16), 1u);
            mma_bf16(d0 + 48, ad(2, 0) + qa, bd(15), idesc_n(16), 1u);
            mma_bf16(d0 + 16, ad(0, 2) + qa, bd(16), idesc_n(16), 1u);
            mma_bf16(d0 + 32, ad(0, 0) + qa, bd(17), idesc_n(16), 1u);
            mma_commit(BAR(B_TF + ts));
            last_commit = t;
          }
          if (!ok) break;
          mma_commit(BAR(B_RECE + (int)(kp % P.nrec)));  // plane x-1 is no longer read
        }
        if (!ok) break;
        mma_commit(BAR(B_RECE + (int)((k0 + nout) % P.nrec)));
        mma_commit(BAR(B_RECE + (int)((k0 + nout + 1) % P.nrec)));
        kr = k0 + nout + 2;
      }
      // never leave MMAs in flight (bounded; ignores the abort flag)
      if (last_commit >= 0) {
        const uint32_t b = BAR(B_TF + (int)(last_commit % TSLOT)), par = (uint32_t)((last_commit / TSLOT) & 1);
        for (int it = 0; it < P.poll && !mbar_try(b, par); ++it) {
        }
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int grp = warp >> 2, wq = warp & 3;
    const int m = 32 * wq + lane;
    const int gy = m >> 3, jj = m & 7;  // owned row of the window, z-pair within the tile
    long long ke = 0, t = 0;
    bool ok = true;
    while (ok && run.next()) {
      const int nout = run.xb - run.xa + 1;
      const long long k0 = ke;  // stream index of element layer xa-1
      const int ea = max(WY * run.w - 1, 0);
      const int y = WY * run.w + gy;
      const bool yv = y < NY;
      ok = wait_bar(BAR(B_EF + (int)(k0 % P.ne)), (uint32_t)((k0 / P.ne) & 1), abort_flag, P.err, P.poll);
      for (int o = 0; o < nout && ok; ++o) {
        const int x = run.xa + o;
        const long long kl = k0 + o;  // element layer x-1
        ok = wait_bar(BAR(B_EF + (int)((kl + 1) % P.ne)), (uint32_t)(((kl + 1) / P.ne) & 1), abort_flag, P.err, P.poll);
        if (!ok) break;
        const float* Es[2];
        bool lv[2];
#pragma unroll
        for (int ly = 0; ly < 2; ++ly) {
          const int L = x - 1 + ly;
          lv[ly] = L >= 0 && L < g.nx;
          Es[ly] = reinterpret_cast<const float*>(
              sm + P.off_e + (int)((kl + ly) % P.ne) * P.e_slot +
              (lv[ly] ? (int)((4LL * g.nz * ((long long)L * g.ny + ea)) & 15) : 0));
        }
        for (int qt = 0; qt < P.NQ; ++qt, ++t) {
          if ((int)(t & 1) != grp) continue;
          const int ts = (int)(t % TSLOT);
          const int j = 8 * qt + jj;
          const long long nd0 = ((long long)x * NY + y) * NZ + 2 * j;  // node (x, y, 2j)
          // inputs of the two nodes, fetched before the MMA wait
          bool nv[2];
          uint8_t mk[2];
          float in0[6], in1[6], in2[6], in3[6];
#pragma unroll
          for (int t2 = 0; t2 < 2; ++t2) {
            nv[t2] = yv && 2 * j + t2 < NZ;
            mk[t2] = nv[t2] && topo_in_range(nd0 + t2, g.nnodes) ? P.nmask[nd0 + t2] : (uint8_t)0;
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
              const long long i = 3 * (nd0 + t2) + cc;
              const bool iv = nv[t2] && topo_in_range(i, g.ndof);
              const int q = 3 * t2 + cc;
              in0[q] = in1[q] = in2[q] = in3[q] = 0.f;
              if constexpr (EPI == Epi::Residual) in0[q] = iv ? P.ep.b[i] : 0.f;
              if constexpr (EPI == Epi::RUpd) in0[q] = iv ? P.ep.r[i] : 0.f;
              if constexpr (EPI == Epi::ChebR) {
                in0[q] = iv ? P.ep.r[i] : 0.f;
                in1[q] = iv ? P.ep.dinv[i] : 0.f;
                in2[q] = iv ? P.ep.x[i] : 0.f;
                in3[q] = iv ? to_f(P.u[i]) : 0.f;
              }
            }
          }
          ok = wait_bar(BAR(B_TF + ts), (uint32_t)((t / TSLOT) & 1), abort_flag, P.err, P.poll);
          if (!ok) break;
          tc_fence_after();
          // E of the elements (x-ax, y-ay, 2j-1+k)
          float e[2][2][3];
#pragma unroll
          for (int ax = 0; ax < 2; ++ax)
#pragma unroll
            for (int ay = 0; ay < 2; ++ay)
#pragma unroll
              for (int k = 0; k < 3; ++k) {
                const int ey = y - ay, ez = 2 * j - 1 + k;
                const bool v = lv[1 - ax] && ey >= 0 && ey < g.ny && ez >= 0 && ez < g.nz;
                e[ax][ay][k] = v ? Es[1 - ax][(ey - ea) * g.nz + ez] : 0.f;
              }
          // nodal sums over the 8 elements, two xy-corner slices at a time
          // (slice a: corner ax = (a == 1 || a == 2), ay = a >> 1)
          float accs[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
          const uint32_t ta = tbase + ((uint32_t)(wq * 32) << 16) + (uint32_t)(ts * 64);
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            float D[2][16];
            tmem_ld16(ta + 32 * h, D[0]);
            tmem_ld16(ta + 32 * h + 16, D[1]);
            tmem_wait_ld();
            if (h == 1) {
              tc_fence_before();
              mbar_arrive(BAR(B_TE + ts));
            }
#pragma unroll
            for (int b = 0; b < 2; ++b) {
              const int a = 2 * h + b;
#pragma unroll
              for (int t2 = 0; t2 < 2; ++t2)
#pragma unroll
                for (int az = 0; az < 2; ++az)
#pragma unroll
                  for (int cc = 0; cc < 3; ++cc)
                    accs[3 * t2 + cc] = fmaf(e[(a == 1 || a == 2) ? 1 : 0][a >> 1][t2 - az + 1], D[b][6 * t2 + 3 * az + cc],
                                             accs[3 * t2 + cc]);
            }
          }
          for (int t2 = 0; t2 < 2; ++t2) {
            if (!nv[t2]) continue;
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
              const float acc = accs[3 * t2 + cc];
              const long long i = 3 * (nd0 + t2) + cc;
              if (!topo_in_range(i, g.ndof)) continue;
              const bool fr = (mk[t2] >> cc) & 1;
              const int q = 3 * t2 + cc;
              if constexpr (EPI == Epi::Store) {
                P.ep.y[i] = fr ? acc : 0.f;
              } else if constexpr (EPI == Epi::Residual) {
                P.ep.y[i] = fr ? in0[q] - acc : 0.f;
              } else if constexpr (EPI == Epi::RUpd) {
                P.ep.r[i] = fr ? in0[q] - P.ep.s * acc : 0.f;
              } else if constexpr (EPI == Epi::ChebR) {
                if (fr) {
                  const float rv = in0[q] - P.ep.s * acc;
                  P.ep.r[i] = rv;
                  const float dn = P.ep.c1 * in3[q] + P.ep.c2 * (in1[q] * rv);
                  P.ep.d_out[i] = dn;
                  P.ep.x[i] = in2[q] + P.ep.ax * dn;
                } else {
                  P.ep.r[i] = 0.f;
                  P.ep.d_out[i] = 0.f;
                }
              }
            }
          }
        }
        if (!ok) break;
        mbar_arrive(BAR(B_EE + (int)(kl % P.ne)));  // layer x-1 is no longer read
      }
      if (!ok) break;
      mbar_arrive(BAR(B_EE + (int)((k0 + nout) % P.ne)));
      ke = k0 + nout + 1;
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
// KE tiles (B operand), the error flag, the SM count, and which kernel
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
  int NQ, nrecs, CS, nrec, nraw, ne;
  int off_rec, rec_slot, off_raw, raw_slot, off_e, e_slot, off_bar, off_misc;
  int total;
};

constexpr int kSmemMax = 232448 - 1024;  // opt-in limit minus the 1024-byte alignment slack
constexpr int kOneCtaPerSm = 120 * 1024;  // > half of the 228 KB an SM holds

int al128(long long x) { return (int)((x + 127) & ~127LL); }

// Tiles per plane, record rows and the deepest rings that fit (at least 4
// record planes, 2 raw planes, 3 element layers); false if none fits.
bool xs_layout(const Grid& g, int usz, XsLayout& L) {
  L.NQ = (g.NZ + 15) / 16;  // z-pairs (2j < NZ) in tiles of 8
  L.nrecs = 16 * L.NQ + 2;  // nodes -1 .. 16 NQ
  L.CS = 8 * L.nrecs;
  L.rec_slot = al128((long long)xs::SROW * L.CS);
  L.raw_slot = al128(3LL * g.NZ * xs::SROW * usz + 32);
  L.e_slot = al128(4LL * xs::EROW * g.nz + 32);
  const int pref[][3] = {{xs::NREC, xs::NRAW, xs::NE}, {5, 3, 5}, {5, 2, 4}, {4, 2, 4}, {4, 2, 3}};
  for (const auto& q : pref) {
    int o = xs::NBT * xs::BTILE;
    L.nrec = q[0];
    L.nraw = q[1];
    L.ne = q[2];
    L.off_rec = o;
    o += L.nrec * L.rec_slot;
    L.off_raw = o;
    o += L.nraw * L.raw_slot;
    L.off_e = o;
    o += L.ne * L.e_slot;
    L.off_bar = o;
    o += al128(xs::NBARS * 8);
    L.off_misc = o;
    o += 128;
    L.total = o;
    if (L.total <= kSmemMax) return true;
  }
  return false;
}

template <typename TU, Epi EPI>
void launch_xs(const Grid& g, const void* u, const void* E, const uint8_t* nmask, void* y, const EpiArgs& ea,
               cudaStream_t s) {
  XsDevice& d = xs_device();
  if (!d.B) throw std::runtime_error("tensor-core operator not prepared on this device");
  XsLayout L;
  if (!xs_layout(g, (int)sizeof(TU), L))
    throw std::runtime_error("level0 tensor-core K.u: mesh not supported (z extent too large for shared memory)");
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
  P.nwin = (g.NY + xs::WY - 1) / xs::WY;
  P.NQ = L.NQ;
  P.items = (long long)P.nwin * g.NX;
  P.u = (const TU*)u;
  P.E = (const float*)E;
  P.nmask = nmask;
  P.ep = make_epi<float>(y, ea);
  P.B = d.B;
  P.err = d.err;
  P.st = ea.st;
  P.CS = L.CS;
  P.nrecs = L.nrecs;
  P.nrec = L.nrec;
  P.nraw = L.nraw;
  P.ne = L.ne;
  P.off_rec = L.off_rec;
  P.rec_slot = L.rec_slot;
  P.off_raw = L.off_raw;
  P.raw_slot = L.raw_slot;
  P.off_e = L.off_e;
  P.e_slot = L.e_slot;
  P.off_bar = L.off_bar;
  P.off_misc = L.off_misc;
  P.poll = g_xs_poll;
  P.skip = g_xs_skip;
  const int grid = (int)std::min<long long>(P.items, d.nsm);
  xs::k_level0_xs<TU, EPI><<<grid, xs::NT, smem, s>>>(P);
  TOPO_LAUNCH_CHECK();
}
}  // namespace

bool level0_xs_supported(const Grid& g) {
  XsLayout L;
  return xs_layout(g, 4, L);
}

// B operand: 18 tiles of 16 x 16 BF16 in the order the ten MMAs read
// them. Tile T(ax, ay, dx, dy): input k = (pair po = k/8, record rr = (k/4)%2,
// component k%4) is node 2j-1+r (r = 2po + rr) of row y-ay+dy of plane
// x-ax+dx; output n = (t = n/6, az = (n%6)/3, c = n%3) is component c of node
// z = 2j+t as local corner (ax, ay, az) of element (x-ax, y-ay, z-az), whose
// input node has local dz = r-1-t+az. Entries outside 0 <= dz <= 1,
// components 3 and outputs 12..15 are zero, and so are the two padding
// tiles. Core-matrix order: N-group stride 256 B, K-chunk stride 128 B.
void xs_prepare(const double* KE) {
  auto cid = [](int dx, int dy, int dz) { return dz * 4 + (dy ? (dx ? 2 : 3) : (dx ? 1 : 0)); };
  // (ax, ay, dx, dy) per tile; ax = -1 marks a zero tile
  static const int T[xs::NBT][4] = {
      {0, 0, 0, 0}, {1, 0, 1, 0}, {1, 1, 1, 1}, {0, 1, 0, 1},   // plane x, delta 0 -> S0..S3
      {0, 0, 0, 1}, {1, 0, 1, 1},                               // plane x, delta +1 -> S0, S1
      {1, 1, 1, 0}, {0, 1, 0, 0},                               // plane x, delta -1 -> S2, S3
      {0, 0, 1, 0}, {-1, 0, 0, 0}, {-1, 0, 0, 0}, {0, 1, 1, 1}, // plane x+1, delta 0 -> S0, -, -, S3
      {1, 0, 0, 0}, {1, 1, 0, 1},                               // plane x-1, delta 0 -> S1, S2
      {0, 0, 1, 1},                                             // plane x+1, delta +1 -> S0
      {0, 1, 1, 0},                                             // plane x+1, delta -1 -> S3
      {1, 0, 0, 1},                                             // plane x-1, delta +1 -> S1
      {1, 1, 0, 0}};                                            // plane x-1, delta -1 -> S2
  uint16_t h[xs::NBT * 256];
  for (int b = 0; b < xs::NBT; ++b) {
    const int ax = T[b][0], ay = T[b][1], dx = T[b][2], dy = T[b][3];
    for (int n = 0; n < 16; ++n)
      for (int k = 0; k < 16; ++k) {
        const int po = k / 8, rr = (k / 4) % 2, ci = k % 4;
        const int t = n / 6, az = (n % 6) / 3, co = n % 3;
        const int dz = 2 * po + rr - 1 - t + az;
        double v = 0.0;
        if (ax >= 0 && n < 12 && ci < 3 && dz >= 0 && dz <= 1)
          v = KE[(3 * cid(ax, ay, az) + co) * 24 + 3 * cid(dx, dy, dz) + ci];
        h[b * 256 + (n / 8) * 128 + (k / 8) * 64 + (n % 8) * 8 + (k % 8)] = bf16_bits_rne((float)v);
      }
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
