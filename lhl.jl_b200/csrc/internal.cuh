// internal.cuh -- argument blocks and launchers shared by the .cu files of liblhl_gpu.
#pragma once
#include <cuda.h>
#include <string.h>

#include "common.cuh"

namespace lhl {

// Launch settings that belong to a device.  A kernel's dynamic shared-memory opt-in is an
// attribute of the function in one device's context, and SM counts and occupancy are per
// device, so a process that drives several GPUs (a Julia session switching devices, one
// host thread per GPU) needs them on every device it launches on.  The launchers keep one
// entry per device ordinal, filled the first time that device is current.
constexpr int MAX_DEVICES = 64;

inline cudaError_t current_device(int* dev)
{
    cudaError_t e = cudaGetDevice(dev);
    if (e == cudaSuccess && (*dev < 0 || *dev >= MAX_DEVICES)) e = cudaErrorInvalidDevice;
    return e;
}

// Opts fn in to `bytes` of dynamic shared memory on the current device, unless it already
// holds at least that much there (set[dev] keeps the largest size set on device dev).
inline cudaError_t opt_in_smem(const void* fn, size_t bytes, size_t (&set)[MAX_DEVICES])
{
    int dev = 0;
    cudaError_t e = current_device(&dev);
    if (e != cudaSuccess || bytes <= set[dev]) return e;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) set[dev] = bytes;
    return e;
}

// Device buffers of one reduction (see reduce.cu).
struct RedArgs {
    int n;
    int nb;
    double* A;        // n x n, ld n (factors in place)
    int64_t* ipiv;    // n-2
    double* B0;       // n x (nb+1): pre-panel copies of the panel columns
    double* part;     // GEMV partials, Pmax x n
    double* tab;      // per-step table
    double* cand_v;   // per-CTA pivot candidates: |value|, row, signed value
    int* cand_i;
    double* cand_s;
    double* buf2;     // unblocked path: second matrix buffer (n x n)
    double* tsnap;    // blocked path: rows 1..k0 of the panel columns before the top GEMM
    double* scale;    // balancing D
    double* iscale;
    double* bsum;     // balancing: 2n sums
    double* bfac;     // balancing: per-sweep factors (n)
    int* bflag;       // balancing: [0] scaled-in-sweep flag
    unsigned int* bar;
    int* err;
    unsigned long long limit_ns;
    unsigned long long* ptimes;  // per-phase wall time (ns) accumulated by CTA 0, 8 slots
    int use_tma;                 // GEMV through TMA tiles (needs an even n >= 64)
};

// One solve launch (see solve.cu).
struct LdivArgs {
    int n;
    const double* F;      // factors, ld ldf
    int ldf;
    const int64_t* perm;
    const int64_t* iperm;
    const double* scale;
    const double* iscale;
    const double* Gt;     // shift batch base
    int ldg;
    const uint8_t* swp;
    const double* rdiag;
    double* X;
    int ldx;
    int rhs_per_shift;
    int mode;             // 0 ldiv, 1 applyZinv, 2 applyZ
    const double* done;   // optional: column c is skipped when done[c] <= tol
    double tol;
    double* Y;            // ldiv scratch: n x ycap (the workspace's)
    int ycap;
    int nshifts;          // shift slots in the batch at Gt (for the tensor map over all of them)
    const double* uinv;   // mixed form: inverses of U's 32 x 32 diagonal blocks per shift, or null
    const double* linv;   // mixed form: inverses of L's 64 x 64 diagonal blocks, or null
    int cplx;             // complex shift: Gt planar (po rows per plane), rdiag and X interleaved complex
    int po;
    int* zflags;          // ldiv scratch: ready flags of the blocked forward substitution
    int nzflags;
    int* tail;            // ldiv scratch: the complex solve's few-groups plan and barrier counters (64 ints)
    int* err;             // bounded-wait status (the workspace's error word)
    unsigned long long limit_ns;
    int cj;               // complex reduction (LHLWorkspace{ComplexF64}): F interleaved complex (cplxj.cu)
};

// Many independent matrices of uneven order (lhl_reduce_batched, batch.cu): matrix m has order
// n[m] <= 512 and S shifts; its arrays start at the prefix offsets below.
struct BatchDesc {
    int count, S;
    const int* n;
    const int64_t* off2;  // sum of n^2 over earlier matrices: J, factors, Ht
    const int64_t* off1;  // sum of n: ipiv, perm, iperm, scale, iscale; x S for swap, rdiag
    const int64_t* offg;  // sum of S (n + 4) n: Gt
    double* F;
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
};
constexpr int BATCH_NMAX = 499;  // the reference reduces n < 500 unblocked (F:398-402)

// One L sweep over a tile of right-hand sides (see solve.cu).
struct ZArgs {
    int n;
    const double* F;
    int ldf;
    const int64_t* perm;
    const double* scale;
    const double* iscale;
    const double* src;
    int lds;
    double* dst;
    int ldd;
    int m;       // right-hand sides
    int gather;  // zinv: read x[perm[i]] * iscale[perm[i]]
    int* flags;  // zinv: per (row block, tile) ready flags, cleared before each launch
    int nflags;
    const double* done;  // optional: a tile whose columns all have done[c] <= tol is skipped
    double tol;
    const double* linv;  // zinv, mixed form: inverses of L's 64 x 64 diagonal blocks
    int cplx;            // gather source / scatter destination interleaved complex (column c: part
                         // c & 1 of complex column c >> 1)
    int* err;
    unsigned long long limit_ns;
};

// Mixed-precision reduction (see reduce_mixed.cu).
struct MixArgs {
    int n, rpc, ldr;        // order, rows per CTA, row pitch (floats)
    double* A;              // balanced J in, factors out (n x n, ld n)
    int64_t* ipiv;
    int64_t* perm;          // out: perm and iperm (1-based), from the final row labels
    int64_t* iperm;
    unsigned long long* hdr;  // 2 x grid: per CTA and step parity, value << 32 | step << 16 | row
    unsigned long long* cval;  // 2 x n column values by physical row (tagged words); the panel-delayed
                               // kernel's pivot-row exchange follows (8 MIX_LAZY_LM words)
    unsigned long long* crow;  // 2 x grid x ldr candidate rows (tagged words)
    float* grows;           // n x ldr rows when they do not fit in shared memory
    int* err;
    unsigned long long limit_ns;
    unsigned long long* ptimes;
    int ring;               // panel-delayed form: rows in flight per thread in the panel update (set at launch)
};

struct MixPlan {
    int rpc, grid, ldr, smem_rows, ok;
    size_t smem;
};

constexpr size_t MIX_SMEM_MAX = 227 * 1024 - 4096;  // dynamic part; the kernel's static shared arrays use 2.4 KB
constexpr size_t MIX_SMEM_TOTAL = 227 * 1024;       // dynamic + static shared memory per CTA
void mixed_plan(int n, int sms, MixPlan* pl);
cudaError_t launch_reduce_mixed(MixArgs a, const MixPlan& pl, cudaStream_t st);
// Rows in global memory (pl.smem_rows == 0): the panel-delayed form (reduce_lazy.cu), whose
// candidate rows need MIX_LAZY_RING slots of grid x ldr exchange words instead of 2.
constexpr int MIX_LAZY_RING = 18;
// each ring slot holds, per CTA, its candidate row (ldr words) and the row's multipliers of the
// panel so far (MIX_LAZY_LM words)
constexpr int MIX_LAZY_LM = 16;
cudaError_t launch_reduce_mixed_lazy(MixArgs a, const MixPlan& pl, cudaStream_t st);
// whether the panel-delayed kernel's shared memory fits for row pitch ldr (n up to about 10400)
bool lazy_fits(int ldr);
// after it: Ht, plus the deferred right updates of the rows above each panel (factors and Ht)
cudaError_t launch_lazy_finish(int n, double* F, double* Ht, cudaStream_t st);

cudaError_t launch_reduce(RedArgs a, int balance, int mode, cudaStream_t st);
cudaError_t launch_unblocked_assemble(int n, double* A, const double* B2, const int64_t* ipiv, cudaStream_t st);
// LHLWorkspace{Float32}, n < 1024: balancing and the unblocked reduction in float over the
// buffers A32 / B32 (n x n floats each), then the factors widened into F
cudaError_t launch_reduce_f32(RedArgs a, int balance, float* A32, float* B32, cudaStream_t st);
cudaError_t launch_unblocked_assemble_f32(int n, double* F, const float* A32, const float* B32, const int64_t* ipiv,
                                          cudaStream_t st);
// from n = 1024 the blocked float form: A32 n x n floats, B0 and pre n x 17 floats, w n floats;
// the factors are widened into a.A
cudaError_t launch_reduce_f32_blocked(RedArgs a, int balance, float* A32, float* B0, float* w, float* pre,
                                     cudaStream_t st);
cudaError_t launch_ht_perm(int n, const double* A, double* Ht, const int64_t* ipiv, int64_t* perm, int64_t* iperm,
                           cudaStream_t st);
cudaError_t launch_ht_fill(int n, const double* A, double* Ht, cudaStream_t st);
cudaError_t launch_fill_ones(double* a, double* b, int n, cudaStream_t st);
cudaError_t launch_set_pair(double* a, double* b, double va, double vb, cudaStream_t st);
size_t stepTabBytes();
// 2-D tensor map of a column-major FP64 array (rows x cols, leading dimension ld, even) in
// boxes of box_r x box_c, for TMA loads (reduce.cu).
bool make_tmap_2d(void* tmap, const double* base, int rows, int cols, int ld, int box_r, int box_c);
int reduce_grid_size();

// f32 = 1: the elimination in float arithmetic (LHLWorkspace{Float32}); Ht holds float values
// variant > 0: launch shape `variant` of the table in shift.cu (shift_shape), else by order
cudaError_t launch_shift_lu(int n, const double* Ht, int ldh, const double* sig, const double* tau, int s0, int count,
                            double* Gt, int ldg, uint8_t* swp, double* rd, int32_t* info, cudaStream_t st,
                            int f32 = 0, int variant = 0);
// launch shape `variant` (1-based) of the real / complex shift LU: threads T, elements per thread
// E (and rows in flight D for the real one); 0 when there is no such variant
int shift_shape(int variant, int* T, int* E, int* D);
int shift_shape_cplx(int variant, int* T, int* E);

cudaError_t launch_ldiv(const LdivArgs& a, int nrhs, cudaStream_t st);
cudaError_t launch_linv(int n, const double* F, int ldf, double* linv, cudaStream_t st);
// batches of independent matrices (batch.cu, shift.cu, solve.cu)
cudaError_t launch_reduce_batch(const BatchDesc& d, const double* J, int balance, cudaStream_t st);
cudaError_t launch_shift_lu_batch(const BatchDesc& d, const double* sig, const double* tau, cudaStream_t st);
cudaError_t launch_solve_batch(const BatchDesc& d, const double* J, const double* B, double* X, int R,
                               const double* sig, const double* tau, double tol, int max_steps, double* res,
                               cudaStream_t st);
// complex shifts on a real reduction (complex.cu)
// ht_complex = 1: Ht of a complex reduction (interleaved complex, ld ldh complex elements)
cudaError_t launch_shift_lu_cplx(int n, const double* Ht, int ldh, const double* sig, const double* tau, int s0,
                                 int count, double* Gt, int ldg, int po, uint8_t* swp, double* rd, int32_t* info,
                                 cudaStream_t st, int ht_complex = 0, int variant = 0);
cudaError_t launch_hess_cplx(int n, const double* Gt, int ldg, int po, const uint8_t* swp, const double* rd,
                             double* Y, int ldy, int col0, int count, int rhs_per_shift, const double* done,
                             double tol, cudaStream_t st);
// the same solve for groups of right-hand sides of one shift per CTA (rhs_per_shift >= 2)
// tail (64 ints of scratch), err and limit_ns: the few-groups path of refinement steps (done
// given); null tail: the multi-vector kernel alone
cudaError_t launch_hess_cplx_mrhs(int n, const double* Gt, int ldg, int po, const uint8_t* swp, const double* rd,
                                  double* Y, int ldy, int col0, int count, int rhs_per_shift, const double* done,
                                  double tol, cudaStream_t st, int* tail = nullptr, int* err = nullptr,
                                  unsigned long long limit_ns = 0);
cudaError_t launch_residual_cplx(int n, const double* J, int ldj, const double* B, int ldb, const double* X, int ldx,
                                 double* R, int ldr, int nrhs, int rhs_per_shift, const double* sig, const double* tau,
                                 cudaStream_t st, const double* done = nullptr, double tol = 0.0);
cudaError_t launch_real_to_cplx(const double* re, double* out, int count, cudaStream_t st);
cudaError_t launch_uinv(int n, const double* Gt, int ldg, const double* rd, int s0, int count, double* uinv,
                        cudaStream_t st);
cudaError_t launch_residual(int n, const double* J, int ldj, const double* B, int ldb, const double* X, int ldx,
                            double* R, int ldr, int nrhs, int rhs_per_shift, const double* sig, const double* tau,
                            cudaStream_t st, const double* done = nullptr, double tol = 0.0);
cudaError_t launch_axpy_cols(int n, double* X, int ldx, const double* R, int ldr, int nrhs, cudaStream_t st,
                             const double* done = nullptr, double tol = 0.0);
cudaError_t launch_relres(int n, const double* R, int ldr, const double* B, int ldb, double* out, int nrhs,
                          cudaStream_t st);

// perm from ipiv and its inverse (reduce.cu)
cudaError_t launch_perm(int n, const int64_t* ipiv, int64_t* perm, int64_t* iperm, cudaStream_t st);

// Complex J, LHLWorkspace{ComplexF64} (cplxj.cu).  A, B, Ht: n x n interleaved complex, ld n.
struct CjArgs {
    int n;
    double* A;        // J in (balanced in place), factors out
    double* B;        // second step buffer
    double* Ht;
    int64_t* ipiv;
    int64_t* perm;
    int64_t* iperm;
    double* scale;
    double* iscale;
    double* bsum;     // 2n
    double* bfac;     // n
    int* bflag;
    double* cand_v;   // per-CTA pivot candidates (cj_grid_size(n) of them)
    int* cand_i;
    unsigned int* bar;
    int* err;
    unsigned long long limit_ns;
};
constexpr int CJ_NMAX = 8192;
int cj_grid_size(int n);
cudaError_t launch_reduce_cj(CjArgs a, int balance, cudaStream_t st);
cudaError_t launch_ldiv_cj(const LdivArgs& a, int nrhs, cudaStream_t st);
cudaError_t launch_residual_cj(int n, const double* J, int ldj, const double* B, int ldb, const double* X, int ldx,
                               double* R, int ldr, int nrhs, int rhs_per_shift, const double* sig, const double* tau,
                               cudaStream_t st, const double* done = nullptr, double tol = 0.0);

// Float32 workspaces (f32.cu): column-major block conversions
cudaError_t launch_f32_to_f64(const float* src, int lds, double* dst, int ldd, int rows, int cols, cudaStream_t st);
cudaError_t launch_round_f32(const double* src, int lds, double* dst, int ldd, int rows, int cols, cudaStream_t st);
cudaError_t launch_f64_to_f32(const double* src, int lds, float* dst, int ldd, int rows, int cols, cudaStream_t st);
// interleaved complex columns (ld ldx complex elements) <-> real column pairs (re, im; ld n)
cudaError_t launch_split_complex(const double* X, int ldx, double* R, int n, int cols, cudaStream_t st);
cudaError_t launch_join_complex(const double* R, int n, double* X, int ldx, int cols, cudaStream_t st);

// GMRES-IR (gmres.cu)
size_t gm_state_doubles(int m);
cudaError_t launch_gm_mark(const double* res, double* prev, double* act, double tol, int first, int nrhs,
                           cudaStream_t st);
cudaError_t launch_gm_begin(int n, int m, const double* R, int ldr, double* V, double* S, double* act,
                            const double* res, double tol, int nrhs, cudaStream_t st);
cudaError_t launch_gm_arnoldi(int n, int m, int j, double* R, int ldr, double* V, double* S, double* act, int nrhs,
                              cudaStream_t st);
cudaError_t launch_gm_update(int n, int m, double* X, int ldx, const double* V, const double* S, int nrhs,
                             cudaStream_t st);

}  // namespace lhl
