// internal.cuh - types and launchers shared by the translation units of
// libtopo_b200.so. Nothing here is part of the public C ABI.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

namespace topo {

// Structured hex grid of one multigrid level: element counts and derived node
// counts. Node (ix,iy,iz) -> (ix*NY+iy)*NZ+iz, DoF = 3*node+c.
struct Grid {
  int nx, ny, nz;        // elements
  int NX, NY, NZ;        // nodes = elements + 1
  long long nnodes;
  long long ndof;
  long long nelem;
};

inline Grid make_grid(int nx, int ny, int nz) {
  Grid g;
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.NX = nx + 1; g.NY = ny + 1; g.NZ = nz + 1;
  g.nnodes = (long long)g.NX * g.NY * g.NZ;
  g.ndof = 3 * g.nnodes;
  g.nelem = (long long)nx * ny * nz;
  return g;
}

// 1-D weight of coarse node I in the row-normalised trilinear prolongation of
// fine node i (fine grid has nf elements, coarse nc). Even i takes its single
// parent i/2 with weight 1; odd i takes parents i>>1 and (i>>1)+1 with weight
// 1/2 each, and when (i>>1)+1 lies beyond the coarse grid the row is rescaled
// so it still sums to one. The 3-D weight is the product over dimensions.
__host__ __device__ inline double prolong_w1(int i, int I, int nc) {
  if ((i & 1) == 0) return (I == (i >> 1)) ? 1.0 : 0.0;
  const int lo = i >> 1, hi = lo + 1;
  const bool hi_ok = hi <= nc;
  if (I == lo) return hi_ok ? 0.5 : 1.0;
  if (I == hi && hi_ok) return 0.5;
  return 0.0;
}

// Chebyshev-Jacobi smoothing on [lower*lam, lam], written for a recursive
// residual. Step j (0-based) forms d_j = c1[j] d_{j-1} + c2[j] D^-1 r_j,
// moves x by ax[j] d_j and, before step j+1, updates r -= ax[j] K d_j.
//  form 0 ("reference"): the recurrence of the reference smoother
//    (multigrid_v4.py:861-889): d_0 = z unscaled, x += alpha_0 d_0;
//    d_j = alpha_j (z + gamma_j d_{j-1}), alpha_j = 1/(sigma - delta^2 alpha_{j-1}/4).
//  form 1 ("chebyshev"): first-kind Chebyshev iteration (Saad, Iterative
//    Methods, Alg. 12.1): d_0 = z/theta; d_j = rho_j rho_{j-1} d_{j-1} + (2 rho_j/delta) z,
//    rho_j = 1/(2 theta/delta - rho_{j-1}).
// The recursive residual is algebraically the reference's r = b - K x but
// applies the operator only to increments, which keeps BF16/FP32 operators
// accurate.
struct Cheb {
  int degree;
  double c1[16], c2[16], ax[16];
};

inline Cheb make_cheb(double lam_max, double lower_frac, int degree, int form) {
  Cheb c;
  c.degree = degree;
  const double lam_min = lower_frac * lam_max;
  const double theta = 0.5 * (lam_max + lam_min);
  const double delta = 0.5 * (lam_max - lam_min);
  if (form == 0) {
    double a = 2.0 / (lam_max + lam_min);
    c.c1[0] = 0.0;
    c.c2[0] = 1.0;
    c.ax[0] = a;
    for (int j = 1; j < degree && j < 16; ++j) {
      const double an = 1.0 / (theta - delta * delta * a * 0.25);
      c.c1[j] = an * delta * delta * a * 0.25;
      c.c2[j] = an;
      c.ax[j] = 1.0;
      a = an;
    }
  } else {
    const double sig = theta / delta;
    double rho = 1.0 / sig;
    c.c1[0] = 0.0;
    c.c2[0] = 1.0 / theta;
    c.ax[0] = 1.0;
    for (int j = 1; j < degree && j < 16; ++j) {
      const double rn = 1.0 / (2.0 * sig - rho);
      c.c1[j] = rn * rho;
      c.c2[j] = 2.0 * rn / delta;
      c.ax[j] = 1.0;
      rho = rn;
    }
  }
  return c;
}

// Scalar state shared by the kernels of one Krylov solve (device memory).
struct KrylovState {
  double bb;        // b.b
  double tol2;      // tol^2 * b.b
  double rr;        // r.r (recursive)
  double rz;        // r.z
  double rz_new;
  double pAp;
  double alpha;
  double beta;
  double scratch[8];
  int done;         // 1 once converged: every iteration kernel returns at entry
  int iters;        // preconditioner applications
  int converged;
  int pad;
};

// Deterministic two-stage reductions: each block writes NS partial sums to
// partials[block*8 + s]; the last block to finish (ticket counter) adds them in
// block order and runs the finaliser.
constexpr int kRedBlocks = 592;   // 4 x 148 SMs
constexpr int kRedThreads = 256;
constexpr int kRedSlots = 8;

struct RedWork {
  double* partials;   // kRedBlocks * kRedSlots
  unsigned int* ticket;
};

// ---------------------------------------------------------------- launchers
// level-0 operator (level0.cu)
enum class Prec : int { F64 = 0, F32 = 1, BF16 = 2 };
void set_ke(const double* KE_host);
void set_galerkin_q(const double* Q_host);  // 8 x 576

// Epilogue kinds of the level-0 / stencil operators (u is the operator input).
// Fixed DoFs are masked in every epilogue.
enum class Epi : int {
  Store = 0,      // y = Au
  Residual = 1,   // y = b - Au
  ChebR = 2,      // Chebyshev step on a recursive residual, u = previous direction:
                  //   r -= s Au ; d_out = c1 u + c2 D^-1 r ; x += ax d_out
  StoreDot = 3,   // y = Au and sum u.y -> st->pAp; alpha = rz / pAp
  RUpd = 4,       // r -= s Au  (residual update by an increment u)
};

struct EpiArgs {
  const void* b;      // rhs (Residual)
  const void* dinv;   // Jacobi inverse diagonal (ChebR)
  void* r;            // residual updated in place (ChebR, RUpd)
  void* x;            // iterate updated in place (ChebR)
  void* d_out;        // new direction (ChebR)
  double s, c1, c2, ax;
  KrylovState* st;    // done flag / dot results (may be null)
  RedWork red;
};

// Typed view of EpiArgs handed to the operator kernels.
template <typename T>
struct EpiDev {
  T* y;
  const T* b;
  const T* dinv;
  T* r;
  T* x;
  T* d_out;
  T s, c1, c2, ax;
};

template <typename T>
inline EpiDev<T> make_epi(void* y, const EpiArgs& ea) {
  EpiDev<T> e;
  e.y = (T*)y;
  e.b = (const T*)ea.b;
  e.dinv = (const T*)ea.dinv;
  e.r = (T*)ea.r;
  e.x = (T*)ea.x;
  e.d_out = (T*)ea.d_out;
  e.s = (T)ea.s;
  e.c1 = (T)ea.c1;
  e.c2 = (T)ea.c2;
  e.ax = (T)ea.ax;
  return e;
}

// Per-DoF epilogue of an operator kernel: acc = (K u)_i, ui = u_i.
template <typename T, Epi EPI>
__device__ __forceinline__ void epilogue_store(const EpiDev<T>& e, long long i, bool free_dof, T acc, T ui) {
  if constexpr (EPI == Epi::Store) {
    e.y[i] = free_dof ? acc : (T)0;
  } else if constexpr (EPI == Epi::Residual) {
    e.y[i] = free_dof ? (T)(e.b[i] - acc) : (T)0;
  } else if constexpr (EPI == Epi::RUpd) {
    e.r[i] = free_dof ? (T)(e.r[i] - e.s * acc) : (T)0;
  } else if constexpr (EPI == Epi::ChebR) {
    if (free_dof) {
      const T rv = e.r[i] - e.s * acc;
      e.r[i] = rv;
      const T dn = e.c1 * ui + e.c2 * (e.dinv[i] * rv);
      e.d_out[i] = dn;
      e.x[i] += e.ax * dn;
    } else {
      e.r[i] = (T)0;
      e.d_out[i] = (T)0;
    }
  }
}

void level0_apply(Prec p, const Grid& g, const void* u, const void* E, const uint8_t* mask, void* y,
                  Epi epi, const EpiArgs& ea, cudaStream_t s);
void level0_diag(const Grid& g, const double* E, const uint8_t* mask, double* diag, cudaStream_t s);
// tensor-core BF16-input operator streaming along x (kmatvec_xs.cu); the
// KE tile and the error flag are per device
void xs_prepare(const double* KE_host);
bool level0_xs_supported(const Grid& g);
// nmask: per-node free bits (bit c = DoF 3n+c free)
void level0_apply_xs(bool u_bf16, const Grid& g, const void* u, const void* E, const uint8_t* nmask, void* y, Epi epi,
                     const EpiArgs& ea, cudaStream_t s);
int xs_error_flag(cudaStream_t s, bool sync = true);
int* wait_error_flag();
// FP32 / FP64 level-0 K.u on the CUDA cores streaming along x (kmatvec_cc.cu)
void cc_set_ke(const double* KE_host);
bool level0_cc_supported(const Grid& g, bool f64);
void level0_apply_cc(bool f64, const Grid& g, const void* u, const void* E, const uint8_t* mask, void* y, Epi epi,
                     const EpiArgs& ea, int* err, cudaStream_t s);
void xs_debug(int skip_first_arrival, int poll_limit);
void modulus(long long n, const double* rho, double penal, double E0, double Emin, double* E,
             float* E32, cudaStream_t s);
// dc_e = -penal (E0-Emin) rho_e^(penal-1) v_e^T KE u_e (v = u when null)
void sensitivity(const Grid& g, const void* u, const void* v, bool u_f32, const double* rho, double penal,
                 double E0, double Emin, double* dc, cudaStream_t s);

// coarse levels (coarse.cu): 27-point block stencils S[k*9 + c*3 + d][node]
void level1_assemble(const Grid& fine, const Grid& coarse, const double* E_f, const uint8_t* mask_c,
                     double* S, cudaStream_t s);
void rap(const Grid& fine, const Grid& coarse, const double* S_f, const uint8_t* mask_c, double* S_c,
         cudaStream_t s);
void stencil_apply(Prec p, bool vec64, const Grid& g, const void* S, const void* u, const uint8_t* mask,
                   void* y, Epi epi, const EpiArgs& ea, cudaStream_t s);
void stencil_dinv(const Grid& g, const double* S, const uint8_t* mask, double* dinv64, float* dinv32,
                  cudaStream_t s);
// FP64 coefficient-major stencil -> packed FP32 / BF16 apply copies (27*12 values per node)
void stencil_convert(long long nnodes, const double* S, float* S32, __nv_bfloat16* S16, cudaStream_t s);
void inject_mask(const Grid& fine, const Grid& coarse, const uint8_t* mf, uint8_t* mc, cudaStream_t s);
void restrict_vec(bool vec64, const Grid& fine, const Grid& coarse, const void* rf, const uint8_t* mc,
                  void* rc, const KrylovState* st, cudaStream_t s);
// x_f += e = mask_f * P e_c ; e is also written to e_out when not null
void prolong_add(bool vec64, const Grid& fine, const Grid& coarse, const void* ec, const uint8_t* mf,
                 void* xf, void* e_out, const KrylovState* st, cudaStream_t s);
// coarsest level (coarsest.cu): band Cholesky of the free-DoF operator and
// the inverses of its diagonal blocks. Compact DoF i -> full DoF free[i].
struct CoarsestPlan {
  int n = 0;                                // free DoFs (compact rows)
  int nt = 0;                               // 32-row blocks
  long long nfull = 0;                      // DoFs of the full coarsest-level vectors
};
// Diagonal blocks of the coarsest factor: rows b[q] .. b[q+1]-1 (boundaries
// multiples of 32, every block at least `band` rows, so L couples block q+1
// to block q only through the band x band corner L[b[q+1]+k][b[q+1]-band+l],
// l >= k). Block q of the apply matrix starts at element off[q], row stride
// ld[q]: columns 0 .. m-1 hold W_q = L_qq^-1 (lower) and W_q^T (strict upper),
// columns gofs .. gofs+band-1 G_q = W_q Lc_q, columns hofs .. hofs+band-1
// H_q = (Lc_{q+1} W_q[m-band .. m-1, :])^T.
constexpr int COARSE_MAXB = 8;
struct CoarseBlocks {
  int P = 1;
  int b[COARSE_MAXB + 1] = {};
  long long off[COARSE_MAXB] = {};
  long long ld[COARSE_MAXB] = {};
  int gofs[COARSE_MAXB] = {};
  int hofs[COARSE_MAXB] = {};
};
struct CoarsestFactor {
  CoarsestPlan plan;
  int band = 0;
  long long ldb = 0;
  bool f64 = true;                          // apply matrix and vectors in FP64 (else FP32)
  double *A = nullptr, *L = nullptr;        // band storage (n x (band+1)): operator, factor
  double* Dinv = nullptr;                   // inverses of the 32x32 diagonal blocks of L
  double* Lnext = nullptr;                  // look-ahead: the next panel's factored block (two slots)
  CoarseBlocks blk;                         // diagonal blocks of W and the apply matrix
  double* W64 = nullptr;                    // per block: W_q (lower), in FP64 also W_q^T, G_q, H_q
  void* C = nullptr;                        // apply matrix in the apply precision (W64 itself in FP64)
  int* flag = nullptr;                      // [0] non-positive pivot, [1] barrier timeout
  int* err = nullptr;
  unsigned* bar = nullptr;
  int chol_grid = 1;
  int strips_per_block = 0;                 // 16-column W strips of the largest block
  const int* d_free = nullptr;
  int kind = 0;                             // 0 none, 1 Cholesky, 2 Cholesky of K + eps I
};
CoarsestPlan coarsest_plan(const Grid& g, const std::vector<int>& free_list);
void coarsest_alloc(CoarsestFactor& f, const CoarsestPlan& p, int band, bool f64, void* (*alloc_bytes)(void*, size_t),
                    void* ctx);
void coarsest_assemble(CoarsestFactor& f, const Grid& g, const double* S, const int* dof_index, cudaStream_t s);
void coarsest_regularise(CoarsestFactor& f, double* dtmp, cudaStream_t s);
void coarsest_factor(CoarsestFactor& f, cudaStream_t s);
int coarsest_status(CoarsestFactor& f, cudaStream_t s);
void coarsest_apply(const CoarsestFactor& f, bool vec64, const void* rhs, double* work, void* x, const KrylovState* st,
                    cudaStream_t s);

// block PCG kernels (blockops.cu): FP64 column blocks as pointer lists
void set_ke_block(const double* KE_host);
void level0_apply_block(const Grid& g, const double* const* U, const double* E, const uint8_t* mask,
                        double* const* Y, int nv, cudaStream_t s);
size_t block_gram_partials();
// G[i*8+j] = A_i . B_j (device, 64 doubles); part: block_gram_partials() doubles
void block_gram(long long n, const double* const* A, int na, const double* const* B, int nb, double* part,
                double* G, cudaStream_t s);
// Out_j = C_j + sign * sum_i In_i M[i*8+j] (C may be null, Out may alias C)
void block_combine(long long n, const double* const* In, int ni, const double* const* Cc, double* const* Out, int no,
                   const double* M, double sign, cudaStream_t s);

// vectors and reductions (vec.cu)
void vfill(bool f64, long long n, void* x, double v, cudaStream_t s);
void vcopy(bool f64, long long n, const void* a, void* b, cudaStream_t s);
void vcast(long long n, const void* src, bool src64, void* dst, bool dst64, cudaStream_t s);
void vmask(bool f64, long long n, void* x, const uint8_t* mask, cudaStream_t s);
// First Chebyshev step on residual r (copied from b first when b is not
// null): d = c2 D^-1 r ; x = (x_is_zero ? 0 : x) + ax d
void cheb_start(bool f64, long long n, const void* b, void* r, const void* dinv, double c2, double ax, void* x,
                void* d, bool x_is_zero, const KrylovState* st, cudaStream_t s);
// out = sum a_i b_i (fp64 accumulate) to a device double
void dot_to(bool f64, long long n, const void* a, const void* b, double* out, RedWork red,
            cudaStream_t s);
double dot_host(bool f64, long long n, const void* a, const void* b, RedWork red, double* dev_tmp,
                cudaStream_t s);
// PCG pieces
void pcg_init(KrylovState* st, double tol, cudaStream_t s);    // bb, rr already set by dot_to
void pcg_xr_update(bool f64, long long n, void* x, void* r, const void* p, const void* Ap,
                   KrylovState* st, RedWork red, cudaStream_t s);
void pcg_rz(bool f64, long long n, const void* r, const void* z, KrylovState* st, RedWork red,
            bool first, cudaStream_t s);
void pcg_p_update(bool f64, long long n, const void* z, void* p, KrylovState* st, bool first,
                  cudaStream_t s);
void axpby(bool f64, long long n, double a, const void* x, double b, void* y, cudaStream_t s);
void axpy_to64(bool f64, long long n, double a, const void* z, double* x, cudaStream_t s);
void scale_dev(bool f64, long long n, const void* x, const double* num, const double* den, void* y,
               cudaStream_t s);

// design (design.cu)
// Offsets and weights of the linear-hat density filter for one radius, in
// device memory owned by a context (so contexts with different radii, or on
// different devices, never share it).
constexpr int kMaxFilterOff = 1331;  // (2*5+1)^3: rmin < 6
struct FilterStencil {
  double rmin = -1.0;
  int n = 0;
  int* off = nullptr;    // 3 * kMaxFilterOff
  double* w = nullptr;   // kMaxFilterOff
};
void filter_apply(FilterStencil& fs, const Grid& g, double rmin, const double* in, double* out, bool transpose,
                  double* Hs_work, cudaStream_t s);
int oc_update(long long n, const double* rho, const double* dc, double volfrac, double move,
              double rho_min, double* out, RedWork red, double* state, cudaStream_t s);
int oc_update_filtered(long long n, const double* rho, const double* dc, const double* dv,
                       const double* colsum, double volfrac, double move, double rho_min, double* out,
                       RedWork red, double* state, cudaStream_t s);
void heaviside_apply(long long n, const double* rho_f, double beta, double eta, double* phys, double* dh,
                     cudaStream_t s);
int oc_update_projected(FilterStencil& fs, const Grid& g, double rmin, const double* rho, const double* dc, const double* dv,
                        double beta, double eta, double volfrac, double move, double rho_min, double* out,
                        double* Hs_work, RedWork red, double* st, cudaStream_t s);
void field_stats(long long n, const double* x, double* out4_dev, RedWork red, cudaStream_t s);

// error plumbing
void set_global_error(const std::string& msg);
std::string global_error();

// Kernel-launch accounting (reported by topo_launch_count): every launch site
// counts one; a replayed CUDA graph counts its kernel nodes.
void count_launches(long long n);
long long launch_count();

}  // namespace topo

#define TOPO_CUDA_CHECK(expr)                                                     \
  do {                                                                            \
    cudaError_t _e = (expr);                                                      \
    if (_e != cudaSuccess) {                                                      \
      throw std::runtime_error(std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    }                                                                             \
  } while (0)

#define TOPO_LAUNCH_CHECK()      \
  do {                           \
    topo::count_launches(1);     \
    TOPO_CUDA_CHECK(cudaGetLastError()); \
  } while (0)

// ------------------------------------------------ index range-check build
// Built with -DTOPO_DEBUG_BOUNDS (python -m topogpu_b200.build
// --debug-bounds -> libtopo_b200_dbg.so), every checked gather/scatter index
// is tested before the access; an index out of range skips the access and
// raises a device flag (one per translation unit) that topo_debug_bounds
// reads back as a status. No trap, no assert. In the normal build the check
// is the constant true and compiles away.
#ifdef TOPO_DEBUG_BOUNDS
static __device__ int g_topo_bounds_flag;
__device__ __forceinline__ bool topo_in_range(long long i, long long n) {
  if (i >= 0 && i < n) return true;
  atomicExch(&g_topo_bounds_flag, 1);
  return false;
}
#define TOPO_BOUNDS_READER(name)                                                   \
  int name() {                                                                     \
    int h = 0;                                                                     \
    TOPO_CUDA_CHECK(cudaMemcpyFromSymbol(&h, g_topo_bounds_flag, sizeof(int)));  \
    if (h) {                                                                       \
      const int z = 0;                                                             \
      TOPO_CUDA_CHECK(cudaMemcpyToSymbol(g_topo_bounds_flag, &z, sizeof(int)));  \
    }                                                                              \
    return h;                                                                      \
  }
#else
__device__ __forceinline__ constexpr bool topo_in_range(long long, long long) { return true; }
#define TOPO_BOUNDS_READER(name) \
  int name() { return 0; }
#endif

namespace topo {
// per translation unit: read and clear its range-check flag (0 in the normal build)
int bounds_flag_level0();
int bounds_flag_xs();
int bounds_flag_cc();
int bounds_flag_coarse();
int bounds_flag_coarsest();
int bounds_flag_design();
}  // namespace topo
