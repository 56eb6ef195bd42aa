// kmatvec_cc.cu - level-0 hex8 K.u on the CUDA cores (FP32 or FP64),
// streaming along x with TMA-staged node planes.
//
// Same work decomposition as the tensor-core kernel: a persistent CTA takes
// a contiguous range of (window, node plane) items; a window owns R
// consecutive node rows in y and the full z extent; output plane P needs the
// node planes P-1, P, P+1 of the window's rows plus one halo row on each
// side, and the element layers P-1 and P. Each plane range is one contiguous
// run of u, so a producer thread stages planes (and element layers of E)
// with cp.async.bulk into shared-memory rings completed on mbarriers, and
// the compute warps read them in place: one thread per owned node, 27
// neighbour records, 576 multiply-adds with KE as constant-bank operands
// (partial sums per incident element, then the E scaling).
//
// Out-of-mesh couplings need no predicates on u: every element outside the
// mesh gets E = 0 (the E reads are predicated), and every node value read
// from shared memory is finite (the rings are zeroed at start; a slot only
// ever holds staged u), so their products vanish exactly.
//
// Reference semantics: MatrixFreeKff.matvec (src/gpu_fem/solver_v2.py:1183-1223).
#include "internal.cuh"
#include "reduce.cuh"

#include <cstring>
#include <mutex>
#include <stdexcept>
#include <vector>

namespace topo {

namespace cc {

// KE in this file's own constant bank (the library is built without
// relocatable device code, so constants cannot be shared across files; the
// per-device upload is cc_set_ke, called with the other KE copies).
__constant__ double cKE64[576];
__constant__ float cKE32[576];

constexpr int NCW = 8;            // compute warps
constexpr int NT = 32 * (NCW + 1);
constexpr int W_PROD = NCW;
constexpr int MAXR = 6;
// mbarrier indices: raw full / empty, E full / empty
constexpr int B_RF = 0, B_RE = 6, B_EF = 12, B_EE = 18, NBARS = 24;

template <typename T>
struct Params {
  Grid g;
  int nwin, R;              // windows and owned node rows per window
  long long items;
  const T* u;
  const T* E;
  const uint8_t* mask;
  EpiDev<T> ep;
  KrylovState* st;
  RedWork red;
  int* err;
  int nraw, ne;
  int off_raw, raw_slot, raw_pad, off_e, e_slot, off_bar;
  int poll;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
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

// AND of a predicate over the compute threads (named barrier 1).
__device__ __forceinline__ bool comp_all(bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(32 * NCW)
      : "memory");
  return r != 0;
}

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

// Stage global bytes [off0, off0+n) of a vector (16-byte aligned base,
// vbytes long) into dst so that byte off0 lands at dst + (off0 % 16); bytes
// in the vector's last partial 16-byte word by plain loads. Returns the bulk
// bytes to issue.
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

// Items [lo, hi), item = w*NX + P. A run of one window covers output planes
// [pa, pb]; it reads node planes pa-1 .. pb+1 and element layers pa-1 .. pb.
struct Seq {
  long long lo, hi;
  int NX, w, pa, pb, P;
  bool ok;
  __device__ void start(long long it) {
    w = (int)(it / NX);
    pa = (int)(it - (long long)w * NX);
    pb = (int)(min(hi, (long long)(w + 1) * NX) - 1 - (long long)w * NX);
    P = pa;
  }
  __device__ void init(long long lo_, long long hi_, int NX_) {
    lo = lo_;
    hi = hi_;
    NX = NX_;
    ok = lo < hi;
    if (ok) start(lo);
  }
  __device__ bool first() const { return P == pa; }
  __device__ bool last() const { return P == pb; }
  __device__ void next() {
    if (P < pb) {
      ++P;
      return;
    }
    const long long nx = (long long)w * NX + pb + 1;
    if (nx >= hi) ok = false;
    else start(nx);
  }
};

template <typename T>
__device__ __forceinline__ T ke(int idx) {
  if constexpr (sizeof(T) == 8) return cKE64[idx];
  else return cKE32[idx];
}

__host__ __device__ constexpr int corner(int bx, int by, int bz) { return bz * 4 + (by ? (bx ? 2 : 3) : (bx ? 1 : 0)); }

template <typename T, Epi EPI>
__global__ void __launch_bounds__(NT) k_level0_cc(const Params<T> P) {
  if (P.st != nullptr && P.st->done) return;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const Grid& g = P.g;
  const uint32_t bar0 = smem_u32(sm + P.off_bar);
  auto BAR = [&](int i) { return bar0 + 8u * (uint32_t)i; };
  volatile int* abort_flag = &s_abort;
  double part = 0.0;  // StoreDot: this thread's share of u . K u
  // zero the rings once (stale slots then only ever hold finite values)
  for (int i = tid; i < P.off_bar / 16; i += NT) reinterpret_cast<uint4*>(sm)[i] = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    for (int s = 0; s < MAXR; ++s) {
      mbar_init(BAR(B_RF + s), 1);
      mbar_init(BAR(B_RE + s), 32 * NCW);
      mbar_init(BAR(B_EF + s), 1);
      mbar_init(BAR(B_EE + s), 32 * NCW);
    }
    s_abort = 0;
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  fence_async_smem();
  __syncthreads();

  const int NX = g.NX, NY = g.NY, NZ = g.NZ, row3 = 3 * NZ;
  const long long lo = P.items * blockIdx.x / gridDim.x, hi = P.items * (blockIdx.x + 1) / gridDim.x;
  Seq q;
  q.init(lo, hi, NX);
  const int R = P.R;

  if (warp == W_PROD) {
    if (lane == 0) {
      long long kpl = 0, kel = 0;
      bool ok = true;
      const unsigned char* ub = reinterpret_cast<const unsigned char*>(P.u);
      const unsigned char* eb = reinterpret_cast<const unsigned char*>(P.E);
      const long long ubytes = g.ndof * (long long)sizeof(T), ebytes = g.nelem * (long long)sizeof(T);
      for (; q.ok && ok; q.next()) {
        const int oy0 = R * q.w;
        // node planes: P-1, P, P+1 on a run's first step, else P+1
        for (int t = q.first() ? -1 : 1; t <= 1 && ok; ++t, ++kpl) {
          const int Pl = q.P + t;
          const int s = (int)(kpl % P.nraw);
          ok = wait_bar(BAR(B_RE + s), (uint32_t)(((kpl / P.nraw) & 1) ^ 1), abort_flag, P.err, P.poll);
          if (!ok) break;
          // staged rows land at slot + raw_pad (16-byte aligned); the pad
          // leaves room for local row 0 when the window starts at row 0
          unsigned char* dst = sm + P.off_raw + s * P.raw_slot + P.raw_pad;
          uint32_t bytes = 0;
          long long off0 = 0;
          if (Pl >= 0 && Pl < NX) {
            const int ra = max(oy0 - 1, 0), rb = min(oy0 + R + 1, NY);
            off0 = (long long)row3 * ((long long)Pl * NY + ra) * (long long)sizeof(T);
            bytes = stage_range(dst, ub, off0, (long long)(rb - ra) * row3 * (long long)sizeof(T), ubytes);
          }
          mbar_arrive_tx(BAR(B_RF + s), bytes);
          if (bytes) bulk_g2s(smem_u32(dst), ub + (off0 & ~15LL), bytes, BAR(B_RF + s));
        }
        if (!ok) break;
        // element layers: P-1, P on a run's first step, else P
        for (int t = q.first() ? -1 : 0; t <= 0 && ok; ++t, ++kel) {
          const int L = q.P + t;
          const int s = (int)(kel % P.ne);
          ok = wait_bar(BAR(B_EE + s), (uint32_t)(((kel / P.ne) & 1) ^ 1), abort_flag, P.err, P.poll);
          if (!ok) break;
          unsigned char* dst = sm + P.off_e + s * P.e_slot;
          uint32_t bytes = 0;
          long long off0 = 0;
          if (L >= 0 && L < g.nx) {
            const int ra = max(oy0 - 1, 0), rb = min(oy0 + R, g.ny);
            off0 = (long long)g.nz * ((long long)L * g.ny + ra) * (long long)sizeof(T);
            bytes = stage_range(dst, eb, off0, (long long)(rb - ra) * g.nz * (long long)sizeof(T), ebytes);
          }
          mbar_arrive_tx(BAR(B_EF + s), bytes);
          if (bytes) bulk_g2s(smem_u32(dst), eb + (off0 & ~15LL), bytes, BAR(B_EF + s));
        }
      }
      if (!ok) {
        for (long long j = max(0LL, kpl - P.nraw); j < kpl; ++j)
          for (int it = 0; it < P.poll && !mbar_try(BAR(B_RF + (int)(j % P.nraw)), (uint32_t)((j / P.nraw) & 1)); ++it) {
          }
        for (long long j = max(0LL, kel - P.ne); j < kel; ++j)
          for (int it = 0; it < P.poll && !mbar_try(BAR(B_EF + (int)(j % P.ne)), (uint32_t)((j / P.ne) & 1)); ++it) {
          }
      }
    }
  } else {
    // ------------------------------------------------------------ compute
    long long kpl = 0, kel = 0;
    bool ok = true;
    for (; q.ok; q.next()) {
      const int oy0 = R * q.w;
      // planes P-1, P, P+1 are stream entries kpl-? : on a run's first step
      // this step brings in three, else one (the two older are still held)
      const long long kP1 = q.first() ? kpl + 2 : kpl;  // stream index of plane P+1
      if (q.first()) {
        ok = ok && wait_bar(BAR(B_RF + (int)(kpl % P.nraw)), (uint32_t)((kpl / P.nraw) & 1), abort_flag, P.err, P.poll);
        ok = ok && wait_bar(BAR(B_RF + (int)((kpl + 1) % P.nraw)), (uint32_t)(((kpl + 1) / P.nraw) & 1), abort_flag,
                            P.err, P.poll);
      }
      ok = ok && wait_bar(BAR(B_RF + (int)(kP1 % P.nraw)), (uint32_t)((kP1 / P.nraw) & 1), abort_flag, P.err, P.poll);
      const long long kL = q.first() ? kel + 1 : kel;  // stream index of layer P
      if (q.first())
        ok = ok && wait_bar(BAR(B_EF + (int)(kel % P.ne)), (uint32_t)((kel / P.ne) & 1), abort_flag, P.err, P.poll);
      ok = ok && wait_bar(BAR(B_EF + (int)(kL % P.ne)), (uint32_t)((kL / P.ne) & 1), abort_flag, P.err, P.poll);
      if (!comp_all(ok)) break;
      // views: planes P-1, P, P+1 (slots of stream kP1-2 .. kP1), layers P-1, P
      const T* pl[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const long long k = kP1 - 2 + d;
        const int Pl = q.P - 1 + d;
        const int ra = max(oy0 - 1, 0);
        const int delta = (Pl >= 0 && Pl < NX) ? (int)(((long long)row3 * ((long long)Pl * NY + ra) * (long long)sizeof(T)) & 15) : 0;
        // the first staged row (ra) is local row ra - (oy0 - 1) (0 or 1)
        pl[d] = reinterpret_cast<const T*>(sm + P.off_raw + (int)(k % P.nraw) * P.raw_slot + P.raw_pad + delta) -
                (long long)(ra - (oy0 - 1)) * row3;
      }
      const T* el[2];
      bool lv[2];
#pragma unroll
      for (int d = 0; d < 2; ++d) {
        const long long k = kL - 1 + d;
        const int L = q.P - 1 + d;
        lv[d] = L >= 0 && L < g.nx;
        const int ra = max(oy0 - 1, 0);
        const int delta = lv[d] ? (int)(((long long)g.nz * ((long long)L * g.ny + ra) * (long long)sizeof(T)) & 15) : 0;
        // element row e_local = element row - (oy0 - 1)
        el[d] = reinterpret_cast<const T*>(sm + P.off_e + (int)(k % P.ne) * P.e_slot + delta) -
                (long long)(ra - (oy0 - 1)) * g.nz;
      }
      const int nown = min(R, NY - oy0) * NZ;
      for (int nl = tid; nl < nown; nl += 32 * NCW) {
        const int r = nl / NZ, z = nl - r * NZ;  // owned row r: node row oy0 + r, local row r + 1
        // moduli of the eight incident elements (ox, oy, oz) in {0,1}^3:
        // element (P-1+ox, oy0+r-1+oy, z-1+oz)
        T Ee[2][2][2];
#pragma unroll
        for (int ox = 0; ox < 2; ++ox)
#pragma unroll
          for (int oy = 0; oy < 2; ++oy)
#pragma unroll
            for (int oz = 0; oz < 2; ++oz) {
              const int ey = oy0 + r - 1 + oy, ez = z - 1 + oz;
              const bool v = lv[ox] && ey >= 0 && ey < g.ny && ez >= 0 && ez < g.nz;
              Ee[ox][oy][oz] = v ? el[ox][(r + oy) * g.nz + ez] : (T)0;
            }
        T t[2][2][2][3];
#pragma unroll
        for (int o = 0; o < 8; ++o)
#pragma unroll
          for (int c = 0; c < 3; ++c) t[o >> 2][(o >> 1) & 1][o & 1][c] = 0;
#pragma unroll
        for (int dx = 0; dx < 3; ++dx)
#pragma unroll
          for (int dy = 0; dy < 3; ++dy) {
            const T* rowp = pl[dx] + (long long)(r + dy) * row3 + 3 * z;
#pragma unroll
            for (int dz = 0; dz < 3; ++dz) {
              const T u0 = rowp[3 * (dz - 1)], u1 = rowp[3 * (dz - 1) + 1], u2 = rowp[3 * (dz - 1) + 2];
              const T uv[3] = {u0, u1, u2};
#pragma unroll
              for (int ox = 0; ox < 2; ++ox)
#pragma unroll
                for (int oy = 0; oy < 2; ++oy)
#pragma unroll
                  for (int oz = 0; oz < 2; ++oz) {
                    const int mx = dx - ox, my = dy - oy, mz = dz - oz;
                    if (mx < 0 || mx > 1 || my < 0 || my > 1 || mz < 0 || mz > 1) continue;
                    const int a = corner(1 - ox, 1 - oy, 1 - oz);
                    const int m = corner(mx, my, mz);
#pragma unroll
                    for (int c = 0; c < 3; ++c)
#pragma unroll
                      for (int d = 0; d < 3; ++d) t[ox][oy][oz][c] += ke<T>((3 * a + c) * 24 + 3 * m + d) * uv[d];
                  }
            }
          }
        T acc[3] = {0, 0, 0};
#pragma unroll
        for (int ox = 0; ox < 2; ++ox)
#pragma unroll
          for (int oy = 0; oy < 2; ++oy)
#pragma unroll
            for (int oz = 0; oz < 2; ++oz)
#pragma unroll
              for (int c = 0; c < 3; ++c) acc[c] += Ee[ox][oy][oz] * t[ox][oy][oz][c];
        const long long node = ((long long)q.P * NY + oy0 + r) * NZ + z;
        const T* uc = pl[1] + (long long)(r + 1) * row3 + 3 * z;  // this node's own u
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const long long i = 3 * node + c;
          if (!topo_in_range(i, g.ndof)) continue;
          const bool fr = P.mask[i] != 0;
          if constexpr (EPI == Epi::StoreDot) {
            const T v = fr ? acc[c] : (T)0;
            P.ep.y[i] = v;
            part += (double)uc[c] * (double)v;
          } else {
            epilogue_store<T, EPI>(P.ep, i, fr, acc[c], uc[c]);
          }
        }
      }
      // release plane P-1 (and at a run's end P and P+1), layer P-1 (and P)
      fence_async_smem();
      mbar_arrive(BAR(B_RE + (int)((kP1 - 2) % P.nraw)));
      if (q.last()) {
        mbar_arrive(BAR(B_RE + (int)((kP1 - 1) % P.nraw)));
        mbar_arrive(BAR(B_RE + (int)(kP1 % P.nraw)));
      }
      mbar_arrive(BAR(B_EE + (int)((kL - 1) % P.ne)));
      if (q.last()) mbar_arrive(BAR(B_EE + (int)(kL % P.ne)));
      kpl = kP1 + 1;
      kel = kL + 1;
    }
  }
  __syncthreads();
  if constexpr (EPI == Epi::StoreDot) {
    // deterministic grid reduction over all CTAs (the producer warp adds 0)
    double v[1] = {part};
    double tot[1];
    if (grid_sum<1>(v, P.red, tot) && tid == 0) {
      P.st->pAp = tot[0];
      P.st->alpha = P.st->rz / tot[0];
    }
  }
}

}  // namespace cc
}  // namespace topo

namespace topo {
namespace {
struct CcDevice {
  int nsm = 0;
  uint32_t attr_done = 0;
};
std::mutex g_cc_mu;
std::vector<CcDevice> g_cc;

CcDevice& cc_device() {
  int dev = 0;
  TOPO_CUDA_CHECK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_cc_mu);
  if ((int)g_cc.size() <= dev) g_cc.resize(dev + 1);
  CcDevice& d = g_cc[dev];
  if (d.nsm == 0) TOPO_CUDA_CHECK(cudaDeviceGetAttribute(&d.nsm, cudaDevAttrMultiProcessorCount, dev));
  return d;
}

// the opt-in limit covers static and dynamic shared memory together; the
// kernel's static part (abort flag, reduction scratch) stays under 2 KB
constexpr int kCcSmemMax = 232448 - 2048;
int al128(long long x) { return (int)((x + 127) & ~127LL); }

struct CcLayout {
  int nwin, R, nraw, ne, off_raw, raw_slot, raw_pad, off_e, e_slot, off_bar, total;
};

bool cc_layout(const Grid& g, int s, CcLayout& L) {
  L.nwin = (g.NY + 15) / 16;
  L.R = (g.NY + L.nwin - 1) / L.nwin;
  const long long row = 3LL * g.NZ * s;
  L.raw_pad = al128(row + 64);
  L.raw_slot = al128(L.raw_pad + (L.R + 2) * row + 64);
  L.e_slot = al128((long long)(L.R + 1) * g.nz * s + 64);
  const int pref[][2] = {{5, 4}, {4, 3}};
  for (const auto& p : pref) {
    L.nraw = p[0];
    L.ne = p[1];
    L.off_raw = 128;  // room for the reads just before slot 0
    L.off_e = L.off_raw + L.nraw * L.raw_slot;
    L.off_bar = L.off_e + L.ne * L.e_slot;
    L.total = L.off_bar + al128(cc::NBARS * 8);
    if (L.total <= kCcSmemMax) return true;
  }
  return false;
}

template <typename T, Epi EPI>
void launch_cc(const Grid& g, const void* u, const void* E, const uint8_t* mask, void* y, const EpiArgs& ea,
               int* err, cudaStream_t s) {
  CcDevice& d = cc_device();
  CcLayout L;
  if (!cc_layout(g, (int)sizeof(T), L)) throw std::runtime_error("level0 K.u: mesh too large for the streaming kernel");
  constexpr int inst = (int)EPI * 2 + (sizeof(T) == 8 ? 1 : 0);
  if (!(d.attr_done & (1u << inst))) {
    TOPO_CUDA_CHECK(cudaFuncSetAttribute(cc::k_level0_cc<T, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, kCcSmemMax));
    std::lock_guard<std::mutex> lk(g_cc_mu);
    d.attr_done |= 1u << inst;
  }
  cc::Params<T> P;
  P.g = g;
  P.nwin = L.nwin;
  P.R = L.R;
  P.items = (long long)L.nwin * g.NX;
  P.u = (const T*)u;
  P.E = (const T*)E;
  P.mask = mask;
  P.ep = make_epi<T>(y, ea);
  P.st = ea.st;
  P.red = ea.red;
  P.err = err;
  P.nraw = L.nraw;
  P.ne = L.ne;
  P.off_raw = L.off_raw;
  P.raw_slot = L.raw_slot;
  P.raw_pad = L.raw_pad;
  P.off_e = L.off_e;
  P.e_slot = L.e_slot;
  P.off_bar = L.off_bar;
  P.poll = 1 << 22;
  const int per_sm = L.total <= kCcSmemMax / 2 - 1024 ? 2 : 1;
  const long long grid = std::min<long long>(P.items, (long long)d.nsm * per_sm);
  cc::k_level0_cc<T, EPI><<<(unsigned)grid, cc::NT, L.total, s>>>(P);
  TOPO_LAUNCH_CHECK();
}
}  // namespace

void cc_set_ke(const double* KE) {
  float f[576];
  for (int i = 0; i < 576; ++i) f[i] = (float)KE[i];
  TOPO_CUDA_CHECK(cudaMemcpyToSymbol(cc::cKE64, KE, sizeof(double) * 576));
  TOPO_CUDA_CHECK(cudaMemcpyToSymbol(cc::cKE32, f, sizeof(float) * 576));
}

bool level0_cc_supported(const Grid& g, bool f64) {
  CcLayout L;
  return cc_layout(g, f64 ? 8 : 4, L);
}

// FP32 / FP64 K.u streaming along x; every pointer 16-byte aligned. err:
// device flag raised when a bounded wait runs out.
void level0_apply_cc(bool f64, const Grid& g, const void* u, const void* E, const uint8_t* mask, void* y, Epi epi,
                     const EpiArgs& ea, int* err, cudaStream_t s) {
  auto al = [](const void* p) { return p == nullptr || ((uintptr_t)p & 15) == 0; };
  if (!al(u) || !al(E)) throw std::runtime_error("level0 K.u: u and E must be 16-byte aligned");
#define TOPO_CC_CASE(EP)                                             \
  case Epi::EP:                                                      \
    if (f64) launch_cc<double, Epi::EP>(g, u, E, mask, y, ea, err, s); \
    else launch_cc<float, Epi::EP>(g, u, E, mask, y, ea, err, s);      \
    break;
  switch (epi) {
    TOPO_CC_CASE(Store)
    TOPO_CC_CASE(Residual)
    TOPO_CC_CASE(ChebR)
    TOPO_CC_CASE(StoreDot)
    TOPO_CC_CASE(RUpd)
  }
#undef TOPO_CC_CASE
}

TOPO_BOUNDS_READER(bounds_flag_cc)

}  // namespace topo
