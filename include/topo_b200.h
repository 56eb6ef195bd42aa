/*
 * topo_b200.h - C ABI of the B200 SolverV4 state solve and design update.
 *
 * Every entry point takes plain device pointers (caller-owned, contiguous),
 * sizes and an explicit cudaStream_t (passed as void*), and returns an int:
 *   0  success
 *  >0  completed but a cap was hit (e.g. Krylov did not converge)
 *  <0  error (bad argument, CUDA error, device-side bounds flag, wait timeout);
 *      topo_last_error() describes it.
 * The library owns only the workspaces inside a context. A context is bound to
 * the CUDA device that was current when it was created; contexts are not
 * thread-safe (one per host thread).
 *
 * Layout (identical to TopoGPU's): node (ix,iy,iz) of a nelx x nely x nelz hex
 * grid has id (ix*(nely+1)+iy)*(nelz+1)+iz, DoF = 3*id+comp; element (ex,ey,ez)
 * has id (ex*nely+ey)*nelz+ez. Vectors are full length (all DoFs); fixed DoFs
 * are held at zero by a per-DoF free mask instead of being compacted away.
 *
 * The reference interface each entry replaces is cited per function
 * (paths inside the TopoGPU project).
 */
#ifndef TOPO_B200_H
#define TOPO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct topo_ctx topo_ctx;

/* Arithmetic of a vector or operator. TOPO_BF16_F32IN: BF16 operator whose
 * input u is stored FP32 and rounded to BF16 when staged (the smoother's form). */
enum { TOPO_F64 = 0, TOPO_F32 = 1, TOPO_BF16 = 2, TOPO_BF16_F32IN = 3 };

/* Epilogues of the level-0 operator (topo_level0_apply). */
enum { TOPO_EPI_STORE = 0, TOPO_EPI_RESIDUAL = 1, TOPO_EPI_CHEB = 2, TOPO_EPI_RUPD = 4 };

/* Precision schedule of the state solve.
 *  FP64  : FP64 outer PCG, FP64 operators on every level.
 *  FP32  : FP32 outer PCG, FP32 operators on levels 0..L-2 ("plain FP32").
 *  MIXED : FP32 outer PCG with true-residual refresh, BF16-input/FP32-accumulate
 *          operators on levels 0..L-2.
 * In every mode the coarsest level is factorised by FP64 Cholesky. */
enum { TOPO_MODE_FP64 = 0, TOPO_MODE_FP32 = 1, TOPO_MODE_MIXED = 2 };

/* Library version (major*10000 + minor*100 + patch). */
int topo_version(void);

/* Create a context for one structured hex8 grid and GMG hierarchy.
 * Replaces SolverV4.__init__ + _ensure_matfree_components
 * (src/gpu_fem/solver_v4.py:38-145) and GalerkinMatFreeGMG.__init__
 * (src/gpu_fem/multigrid_v4.py:455-574).
 *  KE_host        24x24 FP64 unit stiffness, row-major, host memory
 *                 (KE_UNIT_3D, src/gpu_fem/pub_simp_solver.py:157-186)
 *  n_levels       multigrid levels including the fine level (>=1)
 *  fine_degree    Chebyshev degree on level 0 (gmg_fine_degree)
 *  coarse_degree  Chebyshev degree on levels 1..L-2 (gmg_smooth_iters)
 *  cheb_lower     lambda_min / lambda_max of the Chebyshev window (1/30)
 *  dense_max      largest coarsest system factorised by dense Cholesky;
 *                 larger ones use the fixed 80-step Jacobi-PCG
 *                 (dense_chol_max / coarse_pcg_iters, multigrid_v4.py:471-472) */
int topo_ctx_create(int nelx, int nely, int nelz, int n_levels, int mode, int fine_degree,
                    int coarse_degree, double cheb_lower, int dense_max, const double* KE_host,
                    topo_ctx** out);
int topo_ctx_destroy(topo_ctx* ctx);

/* Smoother variant (takes effect at the next V-cycle).
 *  form 0: the reference's recurrence (multigrid_v4.py:861-889: first
 *          direction unscaled) - reproduces the reference V-cycle;
 *  form 1: first-kind Chebyshev iteration (Saad, Alg. 12.1) [default].
 *  lam_safety: factor applied to the power-iteration estimate of
 *          lambda_max(D^-1 K) (reference: 1.0; default 1.25, because 20 power
 *          steps underestimate it and Chebyshev amplifies modes above it).
 * Both forms run on a recursive residual with the coarse correction updated
 * by the level's FP32 (or FP64) operator. */
int topo_set_smoother(topo_ctx* ctx, int form, double lam_safety);

/* Multigrid cycle: gamma 1 = V-cycle (default; multigrid_v4.py:986-1008),
 * gamma 2 = W-cycle, two coarse corrections per level (multigrid_v4.py:
 * 1010-1042, GalerkinMatFreeGMG(cycle_type="w"), SolverV4(gmg_cycle_type)).
 * Takes effect at the next preconditioner application. */
int topo_set_cycle(topo_ctx* ctx, int gamma);

/* Copy the last error message of this context (or of the library, if ctx is
 * NULL) into buf. Returns the message length. */
int topo_last_error(topo_ctx* ctx, char* buf, int len);

/* Free mask (uint8 per DoF, 1 = free) and load vector F (FP64, all DoFs).
 * Replaces the free/F upload of GPUFEMSolver._upload_cupy (src/gpu_fem/fem_gpu.py:361-379). */
int topo_set_problem(topo_ctx* ctx, const uint8_t* free_mask, const double* F, void* stream);

/* E_e = Emin + (E0-Emin) rho^penal for every element (src/gpu_fem/solver_v4.py:168). */
int topo_modulus(topo_ctx* ctx, const double* rho, double penal, double E0, double Emin, double* E,
                 void* stream);

/* Level-0 matrix-free y = K(E) u on full-length vectors, fixed DoFs of y set
 * to zero and fixed DoFs of u assumed zero.
 * Replaces MatrixFreeKff.matvec (src/gpu_fem/solver_v2.py:1183-1223) and
 * FusedMatvec.matvec/matvec_full (src/gpu_fem/cuda_fused_matvec.py:336-384).
 *  dtype TOPO_F64: u,y,E double.  TOPO_F32: u,y,E float.
 *  TOPO_BF16: u bf16 (uint16 bit patterns), y float, E float; products of
 *  BF16-rounded u and KE accumulated in FP32 on the tensor cores. */
int topo_matvec(topo_ctx* ctx, int dtype, const void* u, void* y, const void* E, void* stream);

/* Level-0 operator with its fused epilogue: the building block of the
 * smoother, exposed so each form can be checked on its own.
 *  u_dtype TOPO_F64: FP64 CUDA cores; u, E and the epilogue vectors double.
 *          TOPO_F32: FP32 CUDA cores; everything float.
 *          TOPO_BF16 / TOPO_BF16_F32IN: tensor cores, u bf16 / float, E and
 *          the epilogue vectors float.
 *  epi TOPO_EPI_STORE    y = K u
 *      TOPO_EPI_RESIDUAL y = b - K u
 *      TOPO_EPI_RUPD     r = r - s K u
 *      TOPO_EPI_CHEB     r = r - s K u; d_out = c1 u + c2 dinv r; x = x + ax d_out
 * Fixed DoFs of y, r and d_out are set to zero (x keeps them). u and d_out
 * must differ; r and x are updated in place. Every vector 16-byte aligned.
 * Replaces one step of the fused smoother _chebyshev_steps / _smooth_fine
 * (src/gpu_fem/multigrid_v4.py:861-932) over FusedMatvec.matvec
 * (src/gpu_fem/cuda_fused_matvec.py:336-370). */
int topo_level0_apply(topo_ctx* ctx, int u_dtype, int epi, const void* u, const void* E, void* y, const void* b,
                      void* r, void* x, void* d_out, const void* dinv, double s, double c1, double c2, double ax,
                      void* stream);

/* Bounded waits (no reference counterpart). Every mbarrier wait of the
 * streaming level-0 kernels gives up after a poll limit, raises a per-device
 * flag in mapped host memory, drains its copies in flight and exits. The
 * asynchronous entries (topo_matvec, topo_level0_apply, topo_gmg_apply)
 * report a flag raised by an earlier launch that has finished, before they
 * launch; topo_pcg / topo_solve and topo_wait_status synchronise and report
 * it at once. The flag is cleared when reported. */

/* Synchronises the context's stream (stream != NULL: that stream) and
 * returns nonzero, with the message in topo_last_error, when a wait of a
 * level-0 kernel launched before it timed out. */
int topo_wait_status(topo_ctx* ctx, void* stream);

/* Test hook for the bounded waits: with skip_first_arrival != 0 the
 * tensor-core K.u's converter warps withhold their first arrival, so its
 * MMA role's wait runs out after poll_limit polls (<= 0: the default limit)
 * and the kernel raises the flag. Applies to later launches in this
 * process. */
int topo_debug_tc_wait(int skip_first_arrival, int poll_limit);

/* Index range checks (no reference counterpart). In the library built with
 * -DTOPO_DEBUG_BOUNDS (libtopo_b200_dbg.so: python -m topogpu_b200.build
 * --debug-bounds) every checked gather/scatter index of the kernels is
 * tested before the access; an out-of-range index skips the access and
 * raises a device flag. *tripped receives 1 when a check failed since the
 * last call (the flags are then cleared), else 0; synchronises the device.
 * Returns 0 in that build and 1 (checks not compiled, *tripped = 0) in the
 * normal one. */
int topo_debug_bounds(int* tripped);

/* diag(K(E)) on all DoFs (zero at fixed DoFs).
 * Replaces MatrixFreeKff.extract_diagonal (src/gpu_fem/solver_v2.py:1229-1252). */
int topo_diag(topo_ctx* ctx, const double* E, double* diag, void* stream);

/* Build the hierarchy for moduli E (FP64, device): level-0 Jacobi diagonal,
 * Chebyshev spectral bounds, level-1 Galerkin operator, R.A.P on deeper levels,
 * coarsest Cholesky.  Replaces GalerkinMatFreeGMG.setup (multigrid_v4.py:657-813). */
int topo_gmg_setup(topo_ctx* ctx, const double* E, void* stream);

/* One V-cycle z = M r on full-length vectors in the context's vector precision
 * (double for TOPO_MODE_FP64, float otherwise).
 * Replaces GalerkinMatFreeGMG.apply (multigrid_v4.py:834-844, 986-1008). */
int topo_gmg_apply(topo_ctx* ctx, const void* r, void* z, void* stream);

/* Preconditioned CG on K(E) x = b with the V-cycle, E from the last
 * topo_gmg_setup. b and x are full-length FP64 vectors in every mode; x holds
 * the initial guess on entry (zero it for a cold start). The iterate stays
 * FP64; r, z, p and K p use the mode's working precision, and in the FP32 and
 * MIXED modes convergence is confirmed on the FP64 true residual b - K x
 * (the solve continues from it when the recursive residual was optimistic).
 * Convergence: ||r|| <= tol ||b|| (checked before the first V-cycle too).
 * out_iters counts V-cycle applications, out_relres the final true
 * ||b - K x|| / ||b||. Returns 1 if maxiter was reached.
 * Replaces _cupy_pcg (src/gpu_fem/solver_v2.py:552-624). */
int topo_pcg(topo_ctx* ctx, const void* b, void* x, double tol, int maxiter, int* out_iters,
             double* out_relres, void* stream);

/* Flexible GMRES(restart) with the V-cycle as right preconditioner, same
 * conventions as topo_pcg (FP64 b and x; each restart begins from the FP64
 * true residual). Replaces _cupy_fgmres (multigrid_v4.py:325-443). */
int topo_fgmres(topo_ctx* ctx, const void* b, void* x, double tol, int maxiter, int restart,
                int* out_iters, double* out_relres, void* stream);

/* Lagged coarsest factor (on != 0): from the second topo_gmg_setup on, the
 * V-cycle applies the coarsest factor of the previous setup while the factor
 * of the current operator is built on a background stream (it replaces the
 * old one at the next setup). The preconditioner stays symmetric positive
 * definite; Krylov solves still converge to their tolerance. Off by default;
 * the reference refactorises synchronously (multigrid_v4.py:774-811). */
int topo_set_coarse_lag(topo_ctx* ctx, int on);

/* BF16 level-0 operator on the tensor cores (on != 0, the default) or on the
 * CUDA cores (same BF16 inputs and FP32 accumulation, another summation
 * order); a tuning switch with no reference counterpart. */
int topo_set_tc(topo_ctx* ctx, int on);

/* Block PCG for nrhs load cases (1..8) on the current hierarchy: B and X are
 * nrhs full-length FP64 vectors stored one after another (X holds the
 * initial guesses and receives the solutions). One multi-vector FP64 K.u per
 * iteration (moduli staged once for all columns), the GMG V-cycle on every
 * column, alpha/beta from nrhs x nrhs Gram matrices; columns leave the block
 * once ||r_j|| <= tol ||mask b_j||. out_relres receives nrhs values.
 * Returns 0 (all converged), 1 (maxiter reached) or < 0. The reference solves
 * one load case per PCG (_cupy_pcg, src/gpu_fem/solver_v2.py:552-624); this
 * replaces nrhs of those calls. */
int topo_block_pcg(topo_ctx* ctx, const double* B, double* X, int nrhs, double tol, int maxiter,
                   int* out_iters, double* out_relres, void* stream);

/* Element-energy sensitivity dc_e = -penal (E0-Emin) rho_e^(penal-1) u_e^T KE u_e
 * with u in u_dtype (TOPO_F64 or TOPO_F32), FP64 arithmetic.
 * Replaces src/gpu_fem/solver_v4.py:246-251. */
int topo_sensitivity(topo_ctx* ctx, const void* u, int u_dtype, const double* rho, double penal,
                     double E0, double Emin, double* dc, void* stream);

/* Adjoint sensitivity of a linear functional J = L^T u with K(rho) u = F:
 * with lam from K lam = L (a second GMG-PCG solve on the same hierarchy),
 * dJ/drho_e = -penal (E0-Emin) rho_e^(penal-1) lam_e^T KE u_e, written to dc.
 * lam = u gives the compliance sensitivity. u and lam share `dtype`
 * (TOPO_F64 or TOPO_F32). The reference differentiates only compliance
 * (src/gpu_fem/solver_v4.py:244-251); this is the non-self-adjoint form of
 * the same element contraction. */
int topo_sensitivity_adjoint(topo_ctx* ctx, const void* u, const void* lam, int dtype, const double* rho,
                             double penal, double E0, double Emin, double* dc, void* stream);

/* FP64 dot product sum_i a_i b_i (a,b in dtype TOPO_F64 or TOPO_F32); the
 * result is written to *out_host (synchronises the stream). Used for the
 * compliance F.u (src/gpu_fem/solver_v4.py:244). */
int topo_dot(topo_ctx* ctx, int dtype, const void* a, const void* b, long long n, double* out_host,
             void* stream);

/* Linear-hat density filter out = H in (transpose=0) or H^T in (transpose=1),
 * rows normalised by their weight sums; neighbours at centre distance
 * <= rmin-1e-10. Replaces _build_density_filter + H.dot / H.T.dot
 * (src/gpu_fem/pub_simp_solver.py:215-243, 347-371). */
int topo_filter(topo_ctx* ctx, double rmin, const double* in, double* out, int transpose,
                void* stream);

/* Bisection OC update of the public GPU path (src/topogpu/solver.py:94-117):
 * lambda doubling then <=80 bisections with |mean-volfrac|<1e-8 early exit;
 * out = the last candidate evaluated. out_evals (host, may be NULL) receives
 * the number of candidate evaluations. */
int topo_oc(topo_ctx* ctx, const double* rho, const double* dc, double volfrac, double move,
            double rho_min, double* out, int* out_evals, void* stream);

/* Filtered-volume OC of run_simp (src/gpu_fem/pub_simp_solver.py:319-340),
 * no Heaviside: l1=0, l2=1e9, <=100 bisections until l2-l1<1e-9; the volume
 * of a candidate is sum(H cand)/n, evaluated as cand . colsum where
 * colsum = H^T 1 (passed in dv_colsum together with the sensitivity dv). */
int topo_oc_filtered(topo_ctx* ctx, const double* rho, const double* dc, const double* dv,
                     const double* colsum, double volfrac, double move, double rho_min, double* out,
                     int* out_evals, void* stream);

/* Smoothed Heaviside projection of run_simp (src/gpu_fem/pub_simp_solver.py:
 * 245-253) over the ctx's n_elem elements: phys = h(rho_f), dh = h'(rho_f)
 * (either output may be NULL, not both); the identity (phys = rho_f, dh = 1)
 * unless beta > 1e-6, the guard of every run_simp call site (331, 348, 366). */
int topo_heaviside(topo_ctx* ctx, const double* rho_f, double beta, double eta, double* phys,
                   double* dh, void* stream);

/* Projected-volume OC of run_simp with use_heaviside (src/gpu_fem/
 * pub_simp_solver.py:319-340): l1=0, l2=1e9, <=100 bisections until
 * l2-l1<1e-9; the volume of a candidate is sum(h(H cand))/n with H the
 * linear-hat filter of radius rmin. out must not alias rho, dc or dv; it is
 * the candidate of the last evaluated lambda. */
int topo_oc_projected(topo_ctx* ctx, double rmin, const double* rho, const double* dc,
                      const double* dv, double beta, double eta, double volfrac, double move,
                      double rho_min, double* out, int* out_evals, void* stream);

/* Bisection OC update that allocates no device memory: the same update as
 * topo_oc, without a context. This entry point has no counterpart in the
 * reference. It is for callers that cannot let a library call cudaMalloc:
 * an application whose device memory belongs to its own pool (a framework
 * caching allocator, a Go/JVM runtime), or a latency-bound loop that cannot
 * afford the device-wide synchronisation cudaMalloc/cudaFree may cause.
 * rho, dc, out: n FP64 values in device memory owned by the caller; out
 * must not alias rho or dc (the kernels take all three as non-aliasing
 * pointers; a call with out == rho or out == dc is rejected).
 * Limit: 1 <= n <= 8,388,608 elements; larger n is rejected with an error.
 * Working memory is a 33,024-byte static device array inside the library,
 * held by every GPU that loads it until the process exits and shared by all
 * calls: calls that overlap on the GPU (on different streams or threads)
 * race and must be serialised by the caller. The first call on a device
 * looks up that array's device address (with that device current), so make
 * it before any stream capture. Synchronises `stream` while it polls the
 * bisection's convergence flag. out_evals (host, may be NULL) receives the
 * number of candidate evaluations. */
int topo_oc_noalloc(const double* rho, const double* dc, long long n, double volfrac, double move,
                    double rho_min, double* out, int* out_evals, void* stream);

/* Summary statistics of an element field (FP64): mean, min, max and
 * grayness 4 mean(x(1-x)) written to out_host[4] (synchronises the stream).
 * Replaces the history fields of src/topogpu/solver.py:120-121, 228-240. */
int topo_field_stats(topo_ctx* ctx, const double* x, long long n, double* out_host, void* stream);

/* Diagnostics of the last setup: per level n_free, lambda_max, and the
 * coarsest solve kind (0 none, 1 dense Cholesky, 2 regularised Cholesky,
 * 3 iterative). Arrays have n_levels entries. */
int topo_gmg_info(topo_ctx* ctx, long long* n_free, double* lambda_max, int* coarse_kind);
/* Device time (ms) of the phases of the last topo_gmg_setup: ms[0] fine
 * diagonal and lambda_max check, ms[1] coarse stencils (level-1 Galerkin,
 * R.A.P), ms[2] copy of the coarsest stencil, ms[3] coarsest factorisation
 * (assembly, banded Cholesky, inverses of its diagonal blocks and their
 * couplings, one graph; the coarse levels' Jacobi diagonals, lambda and
 * stencil conversions run beside it on a second stream; 0 when it runs in
 * the background under topo_set_coarse_lag), ms[4] the join of that stream,
 * pivot check and eps*I retry. Diagnostic of GalerkinMatFreeGMG.setup
 * (src/gpu_fem/multigrid_v4.py:657-811), which the reference times only as a
 * whole in SolverV4.last_timing (solver_v4.py:231-267). */
int topo_setup_phases(topo_ctx* ctx, double* ms);

/* Copy the FP64 operator of coarse level `level` (1..n_levels-1) from the
 * last setup into S_out (device, 243*nnodes_level doubles): the 3x3 block
 * coupling node n to neighbour n+(dx,dy,dz) is at
 * S_out[(k*9 + c*3 + d)*nnodes + n], k = (dx+1)*9+(dy+1)*3+(dz+1); rows and
 * columns of fixed DoFs are zero. The free-free part equals the reference's
 * level operator: K1 of assemble_level1_galerkin (multigrid_v4.py:248-270)
 * and R K P of multigrid_v4.py:747-751. */
int topo_gmg_level_operator(topo_ctx* ctx, int level, double* S_out, void* stream);

/* Device bytes held by the context's workspaces. */
long long topo_workspace_bytes(topo_ctx* ctx);

/* Kernels launched by this library since it was loaded (a replayed CUDA
 * graph counts each of its kernels). Diagnostic; no reference counterpart. */
long long topo_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* TOPO_B200_H */
