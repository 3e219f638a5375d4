/*
 * lhl_gpu.h -- C ABI of liblhl_gpu.so, the sm_100a (B200) implementation of
 * LHLFactorization.jl's hot path: the ELMHES reduction J = Z H Z^-1 (Z = D P L) and the
 * per-shift chain lhl_shift! -> Hessenberg LU -> lhl_ldiv! -> lhl_refine!.
 *
 * Every entry point takes plain pointers and sizes.  Matrix / vector arguments named d*
 * are DEVICE pointers owned by the caller (a Julia CuArray, a torch tensor, cudaMalloc);
 * the workspace and shift objects own their device scratch.  All work is enqueued on the
 * given stream (a cudaStream_t passed as void*; NULL = the legacy default stream).
 * Arguments are validated on the host before anything is launched.  Return value: 0 or
 * one of the LHL_ERR_* codes.  Matrices are column-major FP64 with a leading dimension;
 * pivot and permutation vectors are int64 with 1-based values, exactly as the reference
 * stores them.  One workspace / shift object must not serve concurrent calls (the
 * reference's rule, docs/src/release_notes.md:53-54, src/LHLFactorization.jl:81-82).
 *
 * "F:" below is src/LHLFactorization.jl of the reference.
 */
#ifndef LHL_GPU_H
#define LHL_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    LHL_OK = 0,
    LHL_ERR_ARG = 1,      /* ArgumentError in the reference (F:167-169, F:2463-2473, F:3084-3085) */
    LHL_ERR_DIM = 2,      /* DimensionMismatch (F:2071, F:3056-3057) */
    LHL_ERR_CUDA = 3,     /* a CUDA runtime call failed */
    LHL_ERR_TIMEOUT = 4,  /* a bounded grid-barrier wait expired inside a persistent kernel */
    LHL_ERR_ALLOC = 5     /* device allocation failed */
};

enum {
    LHL_PREC_FP64 = 0,    /* plain form: FP64 throughout, the reference's operation order */
    LHL_PREC_MIXED = 1    /* mixed form: FP32 reduction (FP64-accumulated column updates), FP64
                             balancing, shifts, solves, residuals and refinement */
};

typedef struct lhl_ws_s* lhl_ws_t;       /* LHLWorkspace{Float64} (F:144-178) */
typedef struct lhl_shift_s* lhl_shift_t; /* a batch of LHLShift{Float64} (F:84-116) */

/* Device views of a workspace's reduction (all device pointers, owned by the workspace). */
typedef struct {
    int64_t n;
    double* factors;  /* n x n, ld n: H in triu(factors,-1), multipliers below (F:127-129) */
    double* Ht;       /* n x n, ld n: Ht[j,i] = H[i,j] for i <= j+1, zero elsewhere (F:2005) */
    int64_t* ipiv;    /* n-2 pivots, 1-based (F:478) */
    int64_t* perm;    /* P as a vector, 1-based (F:376-384) */
    int64_t* iperm;   /* its inverse (F:385-387) */
    double* scale;    /* balancing D (powers of two) (F:299-340) */
    double* iscale;   /* 1 ./ scale */
} lhl_ws_view;

/* Device views of a shift batch: shift s occupies Gt + s*ldg*n, swap + s*n, ... */
typedef struct {
    int64_t n, nshifts, ldg;
    double* Gt;       /* LU of sigma I + tau H transposed (F:70-73), ldg = n + 4 rows, pad zero */
    uint8_t* swap;    /* interchanges (F:2540) */
    double* rdiag;    /* 1 / pivots (F:2590) */
    int32_t* info;    /* first zero pivot, 0 if none (F:2450) */
    double* sigma;
    double* tau;
    int64_t po;         /* complex shifts: rows per plane of the planar Gt */
    int32_t is_complex; /* 1: LHLShift{ComplexF64} on a real reduction */
} lhl_shift_view;

/* ---- workspace ------------------------------------------------------------------ */
/* LHLWorkspace{Float64}(n) (F:164-178).  precision: LHL_PREC_*.  With LHL_PREC_MIXED,
 * lhl_reduce computes the factors in FP32 (stored widened to FP64 in the same layout), for
 * use with lhl_refine_tol; every other entry point is unchanged.  Orders: n <= 16384 in
 * both forms, else LHL_ERR_DIM. */
int lhl_ws_create(int64_t n, int precision, lhl_ws_t* ws);
int lhl_ws_destroy(lhl_ws_t ws);
int lhl_ws_get_view(lhl_ws_t ws, lhl_ws_view* view);
/* Waits for the stream and reports a device-side error recorded by the last reduction
 * (LHL_ERR_TIMEOUT from a bounded barrier wait), then clears it. */
int lhl_ws_check(lhl_ws_t ws, void* stream);
/* Wall time (ns) of the last reduction by phase, measured on the device: [0] balancing,
 * [1] pivot + GEMV phases, [2] row phases, [3] panel-end interchanges / TRSM, [4] panel-end
 * GEMMs, [5] CTA 0's total grid-barrier wait, [6] CTA 0's per-step table builds, [7] the
 * whole persistent kernel.  Waits for the stream. */
int lhl_ws_phase_ns(lhl_ws_t ws, uint64_t* out8, void* stream);
/* Finer device timers of the last reduction, per sub-phase of one CTA (16 slots). */
int lhl_ws_probe_ns(lhl_ws_t ws, uint64_t* out16, void* stream);
/* Profiling hook: on = 1 makes the reductions of this workspace record the timers that
 * lhl_ws_phase_ns and lhl_ws_probe_ns read (off by default: the timer reads and their
 * accumulation lengthen CTA 0's per-step path; with them off both read zeros). */
int lhl_ws_set_probes(lhl_ws_t ws, int on);
/* Test hook for the mixed form (LHL_PREC_MIXED): which FP32 reduction kernel later reductions
 * use.  0 (default): by the order -- rows held on chip while they fit (the eager kernel, rank-1
 * row updates every step), else the panel-delayed kernel (rows in global memory, rank-16 row
 * updates once per panel); 1: the eager kernel at every order; 2: the panel-delayed kernel at
 * every order.  Both give a similarity J = Z H Z^-1 to FP32 accuracy; their roundings differ. */
int lhl_ws_set_mixed_kernel(lhl_ws_t ws, int which);
/* Launch shape of the shift LU for shifts on this workspace (no counterpart in the reference,
 * which runs one code path per element type, F:2476-2492): 0 (default) picks it by the order;
 * v >= 1 selects shape v of the real (real_variant) or complex (complex_variant) kernel, as
 * lhl_shift_variant_shape describes it.  Every shape gives the same bits; only the time differs,
 * which is what the host-side tuner (lhl_gpu/tune.py) measures.  A shape whose threads x
 * elements per thread is below the order is LHL_ERR_ARG. */
int lhl_ws_set_shift_variant(lhl_ws_t ws, int real_variant, int complex_variant);
/* Shape `variant` (1-based) of the real (is_complex = 0) or complex shift LU kernel: threads per
 * CTA and pending-row elements per thread (it serves orders n <= threads x per_thread).
 * LHL_ERR_ARG past the last shape. */
int lhl_shift_variant_shape(int is_complex, int variant, int* threads, int* per_thread);
/* Test hook: the wall-time limit of every grid-barrier wait of this workspace's kernels. */
int lhl_ws_set_barrier_limit_ns(lhl_ws_t ws, uint64_t limit_ns);

/* lhl_reduce!(ws, J, balance) (F:355-390): balance, reduce (unblocked below n = 500,
 * blocked with nb = 16 panels otherwise, F:398-402), fill Ht, build perm / iperm.
 * dJ (n x n, leading dimension ldj) is not modified. */
int lhl_reduce(lhl_ws_t ws, const double* dJ, int64_t ldj, int balance, void* stream);

/* Loads a saved reduction into a workspace of the same order and precision, in place of
 * lhl_reduce: device-to-device copies of the arrays of lhl_ws_view (dfactors and dHt n x n,
 * ld n; dipiv n-2; dperm, diperm, dscale, discale n), then, for the mixed form, the inverses
 * of L's diagonal blocks that its solves use.  With the arrays of an earlier lhl_reduce, the
 * workspace then shifts and solves exactly as it did.  No counterpart in the reference, whose
 * workspaces live only in a Julia session. */
int lhl_ws_import(lhl_ws_t ws, const double* dfactors, const double* dHt, const int64_t* dipiv, const int64_t* dperm,
                  const int64_t* diperm, const double* dscale, const double* discale, void* stream);

/* lhl_ldiv!(x, sh, ws) with a complex x on a real shift object (F:3052-3074: eltype(x) differs
 * from the shift's, the generic path): x n x nrhs interleaved complex (ld ldx complex elements),
 * in place.  A real shift is real-linear, so the real and imaginary parts are solved as two real
 * right-hand sides of the same shift slot.  A complex shift object takes the plain lhl_ldiv. */
int lhl_ldiv_complex_rhs(lhl_shift_t sh, lhl_ws_t ws, double* dX, int64_t ldx, int64_t nrhs, int64_t rhs_per_shift,
                         void* stream);

/* ---- element type Float32 (LHLWorkspace{Float32}, F:703-705) ------------------------
 * lhl_ws_create_f32 makes a workspace whose element type is Float32.  Its arrays keep FP64
 * storage holding float values, so every view, shift object and solve entry point of this
 * header applies unchanged:
 *   - J is rounded to float on the way in (lhl_reduce) or taken as float (lhl_reduce_f32);
 *   - the plain form reduces in float arithmetic as the reference does: balancing
 *     (F:299-340) and, below n = 1024 (_lhl_block_min(Float32), F:703-705), the unblocked
 *     ELMHES (F:466-678), from there the blocked form (F:765-1006), with T = Float32; the
 *     mixed form runs the mixed reduction and rounds its factors and Ht to float;
 *   - the shift LU (lhl_shift, lhl_shift_batched) runs in float arithmetic with sigma and tau
 *     rounded to float, as LHLShift{Float32} does (F:2529-2594 with T = Float32);
 *   - complex shifts (LHLShift{ComplexF32}, a shift object from lhl_shift_create_complex):
 *     sigma and tau rounded to ComplexF32, the LU in FP64 arithmetic on the float Ht;
 *   - solves take FP64 vectors (lhl_ldiv) or float ones (lhl_ldiv_f32, widened, solved in
 *     FP64 with the float factors, rounded back; ComplexF32 vectors, interleaved, for a
 *     complex shift object). */
int lhl_ws_create_f32(int64_t n, int precision, lhl_ws_t* ws);
/* lhl_reduce!(ws, J, balance) with J Float32 (dJ n x n, ld ldj, float).  On a Float64
 * workspace the float values are taken exactly, as the reference converts them. */
int lhl_reduce_f32(lhl_ws_t ws, const float* dJ, int64_t ldj, int balance, void* stream);
/* lhl_ldiv!(x, sh, ws) for float right-hand sides (dX n x nrhs, ld ldx, float; for a complex
 * shift object interleaved ComplexF32, ld ldx complex elements), in place.  The widened copy
 * lives in a workspace buffer, allocated by the first call that needs it. */
int lhl_ldiv_f32(lhl_shift_t sh, lhl_ws_t ws, float* dX, int64_t ldx, int64_t nrhs, int64_t rhs_per_shift,
                 void* stream);

/* ---- element type ComplexF64 (LHLWorkspace{ComplexF64}, test/core_tests.jl:241-249) -----
 * lhl_ws_create_c128 makes a workspace for a complex J (FP64 form only; n <= 8192, else
 * LHL_ERR_DIM).  Its factors and Ht (lhl_ws_view) are n x n interleaved complex (re, im
 * pairs, ld n), scale / iscale real; lhl_ws_import takes arrays of that layout.  Replaces
 * lhl_reduce!(ws, J, balance) for complex T (F:355-390; balancing F:299-340 and the pivot
 * search F:470-477 on the modulus |z|; the unblocked ELMHES with the generic sweep F:466-538
 * at every n, the path the reference takes below n = 768).  Its shifts are complex: only a
 * shift object made by lhl_shift_create_complex serves it (LHL_ERR_ARG otherwise, F:2463-2465),
 * through lhl_shift_complex / lhl_shift_batched_complex (real sigma, tau are converted).
 * lhl_ldiv, lhl_applyZ, lhl_applyZinv, lhl_refine, lhl_refine_tol, lhl_refine_gmres and
 * lhl_residual_norms take interleaved complex vectors and, for the refinements, a complex dJ
 * (n x n interleaved, ld ldj complex elements); the solve is applyZinv!, the planar Hessenberg
 * solve, applyZ! (F:3111-3121).  lhl_reduce and lhl_reduce_f32 on it are LHL_ERR_ARG. */
int lhl_ws_create_c128(int64_t n, lhl_ws_t* ws);
/* lhl_reduce!(ws, J, balance) for a complex J (dJ n x n interleaved complex, ld ldj complex
 * elements); a workspace not made by lhl_ws_create_c128 is LHL_ERR_ARG. */
int lhl_reduce_c128(lhl_ws_t ws, const double* dJ, int64_t ldj, int balance, void* stream);

/* ---- element type ComplexF32 (LHLWorkspace{ComplexF32}) ------------------------------
 * lhl_ws_create_c64 makes a complex-J workspace whose element type is ComplexF32: the arrays
 * of lhl_ws_create_c128, holding ComplexF32 values.  J is rounded to ComplexF32 on the way in
 * (lhl_reduce_c128) or taken as ComplexF32 (lhl_reduce_c64, interleaved complex64, ld ldj
 * complex elements); the reduction runs as for ComplexF64 (FP64 arithmetic on the float
 * values) and its factors and Ht are rounded to ComplexF32; shifts are rounded to ComplexF32;
 * solves take ComplexF64 vectors (lhl_ldiv) or ComplexF32 ones (lhl_ldiv_f32).  Not the
 * reference's single-precision rounding, which is not restated. */
int lhl_ws_create_c64(int64_t n, lhl_ws_t* ws);
int lhl_reduce_c64(lhl_ws_t ws, const float* dJ, int64_t ldj, int balance, void* stream);

/* ---- shifts --------------------------------------------------------------------- */
/* A batch of nshifts LHLShift{Float64}(n) objects (F:107-116). */
int lhl_shift_create(int64_t n, int64_t nshifts, lhl_shift_t* sh);
int lhl_shift_destroy(lhl_shift_t sh);
int lhl_shift_get_view(lhl_shift_t sh, lhl_shift_view* view);

/* lhl_shift!(sh, ws, sigma, tau) for shifts s0..s0+count-1 of the batch, with the
 * shifts given as device arrays (F:2456-2594).  One launch; info per shift in the view. */
int lhl_shift_batched(lhl_shift_t sh, lhl_ws_t ws, int64_t s0, int64_t count, const double* dsigma,
                      const double* dtau, void* stream);
/* lhl_shift!(ws, sigma, tau) for one shift slot with host scalars. */
int lhl_shift(lhl_shift_t sh, lhl_ws_t ws, int64_t slot, double sigma, double tau, void* stream);

/* ---- complex shifts on a real reduction (LHLShift{ComplexF64} on LHLWorkspace{Float64}) ----
 * LHLShift{Complex{T}}(n) (F:107-116, F:180-191): nshifts slots whose Gt is planar, (2 po) x n
 * per slot with real parts in rows 1..n and imaginary parts in rows po+1..po+n (po in the
 * view); rdiag, sigma and tau hold interleaved (re, im) pairs.  lhl_ldiv, lhl_refine,
 * lhl_refine_tol and lhl_residual_norms given such a shift take interleaved complex dX / dB /
 * dR (CuArray{ComplexF64} memory; leading dimensions counted in complex elements), and the
 * solve is the reference's complex-on-real one (F:3080-3110). */
int lhl_shift_create_complex(int64_t n, int64_t nshifts, lhl_shift_t* sh);
/* LHLShift{Float32} / LHLShift{ComplexF32}: shift objects for the single-precision workspaces
 * (lhl_ws_create_f32, lhl_ws_create_c64).  An LHLShift{TG} serves an LHLWorkspace{T} only for
 * TG = T or Complex{real(T)} (F:2461-2465): a single-precision shift object on a double-precision
 * workspace, or the other way round, makes the shift calls return LHL_ERR_ARG. */
int lhl_shift_create_f32(int64_t n, int64_t nshifts, lhl_shift_t* sh);
int lhl_shift_create_complex64(int64_t n, int64_t nshifts, lhl_shift_t* sh);
/* lhl_shift!(sh, ws, sigma, tau) with complex sigma, tau (F:2456-2594 with TG = ComplexF64).
 * A shift object made by lhl_shift_create takes only real shifts: LHL_ERR_ARG otherwise
 * (F:2466-2472).  A real shift on a complex object is converted. */
int lhl_shift_complex(lhl_shift_t sh, lhl_ws_t ws, int64_t slot, double sigma_re, double sigma_im, double tau_re,
                      double tau_im, void* stream);
/* Batched complex shifts: dsigma, dtau are count interleaved complex values on the device. */
int lhl_shift_batched_complex(lhl_shift_t sh, lhl_ws_t ws, int64_t s0, int64_t count, const double* dsigma,
                              const double* dtau, void* stream);

/* ---- solves --------------------------------------------------------------------- */
/* lhl_ldiv!(x, sh, ws) (F:3052-3068) for nrhs columns of dX (n x nrhs, leading dimension
 * ldx), in place.  Column j is solved with shift slot j / rhs_per_shift. */
int lhl_ldiv(lhl_shift_t sh, lhl_ws_t ws, double* dX, int64_t ldx, int64_t nrhs, int64_t rhs_per_shift,
             void* stream);

/* lhl_refine!(x, A, b, sh, ws, steps) (F:3144-3157) with A = sigma_s I + tau_s J applied
 * from J (dJ, n x n, ld ldj): r = b - A x, ldiv(r), x += r, `steps` times per column.
 * dR (n x nrhs, ld ldx) is caller scratch for the residual. */
int lhl_refine(lhl_shift_t sh, lhl_ws_t ws, const double* dJ, int64_t ldj, const double* dB, int64_t ldb,
               double* dX, int64_t ldx, double* dR, int64_t nrhs, int64_t rhs_per_shift, int steps,
               void* stream);

/* lhl_refine! driven by a tolerance instead of a step count: up to max_steps refinement
 * steps; a column whose relative residual ||b - A x||_2 / ||b||_2 is already <= tol is left
 * alone (its solve and update are skipped on the device, no host round trip).  On return
 * dres (nrhs) holds every column's final relative residual.  This is how the mixed form
 * (LHL_PREC_MIXED workspace) reaches FP64 accuracy from its FP32 factors.  The reference's
 * lhl_refine! (F:3144-3157) takes a fixed step count; with max_steps = steps and tol = 0 this
 * performs the same updates. */
int lhl_refine_tol(lhl_shift_t sh, lhl_ws_t ws, const double* dJ, int64_t ldj, const double* dB, int64_t ldb,
                   double* dX, int64_t ldx, double* dR, double* dres, int64_t nrhs, int64_t rhs_per_shift, double tol,
                   int max_steps, void* stream);

/* Refinement by GMRES-IR, for where lhl_refine!'s fixed-point iteration (F:3144-3157)
 * contracts slowly (the mixed form near a shift where sigma I + tau J is close to singular).
 * Starting from the solution in dX, each cycle computes r = b - A x for every column whose
 * relative residual is above tol, then up to `restart` steps of GMRES on A d = r
 * left-preconditioned by the shift's factorisation (each step one lhl_ldiv and one product
 * with A), stopping a column's cycle once its estimated residual is below 0.1 tol, and
 * x += d.  At most max_cycles cycles; columns at or below tol are left alone, and so is a
 * column whose residual did not at least halve over its last cycle (it is at the accuracy this
 * preconditioner and FP64 allow for that shift; its last iterate stays).  On return dres holds
 * every column's final relative residual, as for lhl_refine_tol.
 * host_check = 1: the host reads which columns still refine after each cycle (a stream
 * synchronisation) and stops once none does; 0: max_cycles cycles are launched without a host
 * round trip (finished columns skip their work), which a CUDA graph can capture.
 * 1 <= restart <= 32.  The Krylov basis, nrhs (restart + 1) n doubles, is kept in the
 * workspace: allocated by the first call that needs it, reused after.  With a complex shift
 * batch, dX / dB / dR are interleaved complex (as for lhl_refine_tol) and GMRES runs on the
 * realified system: each interleaved column is a real vector of 2n, the real inner product is
 * Re<v, w>, and the basis takes 2n doubles per vector. */
int lhl_refine_gmres(lhl_shift_t sh, lhl_ws_t ws, const double* dJ, int64_t ldj, const double* dB, int64_t ldb,
                     double* dX, int64_t ldx, double* dR, double* dres, int64_t nrhs, int64_t rhs_per_shift,
                     double tol, int max_cycles, int restart, int host_check, void* stream);

/* lhl_refine!(x, A, b, sh, ws, steps) (F:3144-3157) with the caller's system matrix A, as the
 * reference takes it (dA, n x n, ld lda; its tests pass Matrix(W)): r = b - A x, ldiv by shift
 * slot `slot` of sh, x += r, for every one of the nrhs columns.  A need not be sigma I + tau J:
 * the refinement converges to A^-1 b wherever the slot's factorisation is close enough to A
 * (a mass matrix M other than a multiple of I in W = J - M / gamma, say).  Tolerance, dres and
 * the step count as for lhl_refine_tol (tol = 0: exactly max_steps steps, the reference's
 * lhl_refine!); the _gmres form refines as lhl_refine_gmres.  With a complex shift object A,
 * dB, dX and dR are interleaved complex. */
int lhl_refine_system(lhl_shift_t sh, lhl_ws_t ws, int64_t slot, const double* dA, int64_t lda, const double* dB,
                      int64_t ldb, double* dX, int64_t ldx, double* dR, double* dres, int64_t nrhs, double tol,
                      int max_steps, void* stream);
int lhl_refine_system_gmres(lhl_shift_t sh, lhl_ws_t ws, int64_t slot, const double* dA, int64_t lda,
                            const double* dB, int64_t ldb, double* dX, int64_t ldx, double* dR, double* dres,
                            int64_t nrhs, double tol, int max_cycles, int restart, int host_check, void* stream);

/* Relative residuals ||b - (sigma I + tau J) x||_2 / ||b||_2 per column into dres (nrhs). */
int lhl_residual_norms(lhl_shift_t sh, const double* dJ, int64_t ldj, const double* dB, int64_t ldb,
                       const double* dX, int64_t ldx, double* dR, double* dres, int64_t nrhs,
                       int64_t rhs_per_shift, void* stream);

/* applyZ!(x, ws) / applyZinv!(x, ws) (F:2069-2126) on nrhs columns. */
int lhl_applyZ(lhl_ws_t ws, double* dX, int64_t ldx, int64_t nrhs, void* stream);
int lhl_applyZinv(lhl_ws_t ws, double* dX, int64_t ldx, int64_t nrhs, void* stream);

/* ---- batches of independent matrices of uneven order -------------------------------- */
/* Many Jacobians J_m (order n_m <= 499: the reference's unblocked path) with S shifts each,
 * in one launch per phase.  Packed column-major storage:
 *   J_m, factors_m, Ht_m at sum_{l<m} n_l^2 (leading dimension n_m);
 *   ipiv/perm/iperm/scale/iscale of matrix m at sum_{l<m} n_l;
 *   shift s of matrix m: Gt at sum_{l<m} S (n_l+4) n_l + s (n_m+4) n_m (leading dimension
 *   n_m+4), swap and rdiag at S sum_{l<m} n_l + s n_m, info/sigma/tau at m S + s;
 *   right-hand side r of shift s of matrix m (lhl_solve_batched): column s R + r of the
 *   n_m x (S R) block at S R sum_{l<m} n_l.
 * Results per matrix are those of lhl_reduce (bit-identical) and lhl_shift. */
typedef struct lhl_batch_s* lhl_batch_t;
typedef struct {
    int64_t count, shifts, total_n, total_nn, total_g;
    double* factors;
    double* Ht;
    int64_t* ipiv;
    int64_t* perm;
    int64_t* iperm;
    double* scale;
    double* iscale;
    double* Gt;
    uint8_t* swap;
    double* rdiag;
    int32_t* info;
    double* sigma;
    double* tau;
} lhl_batch_view;
int lhl_batch_create(int64_t count, const int64_t* ns, int64_t shifts_per_matrix, lhl_batch_t* batch);
int lhl_batch_destroy(lhl_batch_t batch);
int lhl_batch_get_view(lhl_batch_t batch, lhl_batch_view* view);
/* lhl_reduce!(ws_m, J_m, balance) for every m: one CTA per matrix (F:355-390, F:466-501). */
int lhl_reduce_batched(lhl_batch_t batch, const double* dJ, int balance, void* stream);
/* lhl_shift! of all count x S shifts (dsigma, dtau: count S values, matrix-major): one CTA per shift. */
int lhl_shift_batched_all(lhl_batch_t batch, const double* dsigma, const double* dtau, void* stream);
/* x = W^-1 b for every right-hand side (lhl_ldiv!, F:3052-3068), then lhl_refine! (F:3144-3157)
 * with W = sigma I + tau J_m from the caller's dJ until ||b - W x|| / ||b|| <= tol or max_steps
 * refinement steps: one CTA per right-hand side, everything on chip, one launch.  dres
 * (count S R, optional) receives every final relative residual. */
int lhl_solve_batched(lhl_batch_t batch, const double* dJ, const double* dB, double* dX, int64_t rhs_per_shift,
                      double tol, int max_steps, double* dres, void* stream);

/* ---- reduction without device allocation ------------------------------------------ */
/* No counterpart in the reference (which allocates its workspace in Julia).  For callers
 * that cannot call cudaMalloc -- a host that owns a fixed device-memory budget, a Julia
 * session whose CUDA.jl pool must stay the only allocator, code that must not trigger an
 * allocation's device synchronization: the same reduction as lhl_reduce, with every input
 * and output passed in (dJ n x n ld ldj; dfactors and dHt n x n with leading dimension n;
 * dipiv n-2; dperm, diperm, dscale, discale n) and the scratch held in a fixed static device
 * array of the library (about 2.5 MB, present on every GPU that loads it until exit).
 * n <= LHL_NOALLOC_NMAX, else LHL_ERR_DIM.  The first call on a device resolves the array's
 * device address (make it before any stream capture).  All calls share the array: calls
 * whose work overlaps on the GPU race.  dJ must not overlap dfactors or dHt (LHL_ERR_ARG).
 * Allocates nothing. */
#define LHL_NOALLOC_NMAX 1024
int lhl_reduce_noalloc(int64_t n, const double* dJ, int64_t ldj, int balance, double* dfactors, double* dHt,
                       int64_t* dipiv, int64_t* dperm, int64_t* diperm, double* dscale, double* discale,
                       void* stream);
/* Waits for the stream, then reports a device-side error that the last lhl_reduce_noalloc on
 * the current device recorded in the static array (LHL_ERR_TIMEOUT from a bounded wait) and
 * clears it; LHL_OK otherwise.  The counterpart of lhl_ws_check for the allocation-free call:
 * without it a reduction cut short by a wait limit would look successful.  The next
 * lhl_reduce_noalloc clears the word, so check before it.  Allocates nothing. */
int lhl_reduce_noalloc_check(void* stream);
/* Test hook: the wall-time limit of every bounded wait of later lhl_reduce_noalloc calls in
 * this process (0 restores the default of 2 s). */
int lhl_reduce_noalloc_set_barrier_limit_ns(uint64_t limit_ns);

/* Library build identification (for loaders that check they bound the right .so). */
const char* lhl_version(void);

#ifdef __cplusplus
}
#endif

#endif /* LHL_GPU_H */
