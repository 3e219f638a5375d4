// api.cu -- the C ABI of liblhl_gpu.so (declared in include/lhl_gpu.h): argument checks
// on the host, device buffers of the workspace and shift objects, stream-ordered launches.
#include <stdlib.h>
#include <string.h>

#include <new>

#include "internal.cuh"

struct lhl_ws_s {
    int64_t n;
    int precision;
    int grid;
    double *F, *Ht, *scale, *iscale, *B0, *part, *tab, *cand_v, *cand_s, *buf2, *tsnap, *bsum, *bfac;
    int64_t *ipiv, *perm, *iperm;
    int *cand_i, *bflag, *err;
    unsigned int* bar;
    unsigned long long limit_ns;
    unsigned long long* ptimes;
    double* linv;  // mixed form: inverses of L's 64 x 64 diagonal blocks
    double* ybuf;  // ldiv scratch: n x ycap right-hand sides
    int ycap;
    int* zflags;   // ldiv scratch: ready flags, ceil(n/64) x ceil(ycap/4)
    int nzflags;
    int* tailw;    // ldiv scratch: the complex solve's few-groups plan and barrier counters (64 ints)
    // mixed form (LHL_PREC_MIXED) only
    lhl::MixPlan mplan;
    unsigned long long *mhdr, *mcval, *mcrow;
    float* mgrows;
    // lhl_refine_gmres: Krylov bases, per-column state and activity, host copy of dres
    double *gmV, *gmS, *gmA, *gmH, *gmP;
    size_t gmV_cap, gmS_cap, gmA_cap, gmH_cap, gmP_cap;
    int probes;  // device timers in the reduction kernels (lhl_ws_set_probes)
    int f32;     // LHLWorkspace{Float32}: float values in the FP64 arrays, float shift arithmetic
    double* f32x;  // lhl_ldiv_f32: widened right-hand sides (grow-only)
    float* f32a;   // LHLWorkspace{Float32}, n >= 1024: the blocked float reduction's matrix and scratch
    size_t f32x_cap;
    int cj;        // LHLWorkspace{ComplexF64}: F, Ht, buf2 interleaved complex (cplxj.cu)
    int mix_kernel;  // mixed form: 0 by the plan (rows on chip: eager, else panel-delayed), 1 eager, 2 panel-delayed
    int shift_variant[2];  // launch shape of the real / complex shift LU (0: by order; lhl_ws_set_shift_variant)
};

struct lhl_shift_s {
    int64_t n, nshifts, ldg;
    double *Gt, *rdiag, *sigma, *tau;
    double* uinv;  // mixed form: inverses of U's 32 x 32 diagonal blocks (n / 32 blocks per shift)
    int cplx;      // complex shifts: Gt planar (2 po rows), rdiag / sigma / tau interleaved complex
    int64_t po;
    uint8_t* swap;
    int32_t* info;
    int cj;        // the slots were last loaded from a complex reduction: residuals take a complex J
    int single;    // element type Float32 / ComplexF32: serves Float32 and ComplexF32 workspaces only
};

struct lhl_batch_s {
    int64_t count, S, total_n, total_nn, total_g;
    int64_t* ns_host;
    int *d_n;
    int64_t *d_off2, *d_off1, *d_offg;
    double *F, *Ht, *scale, *iscale, *Gt, *rdiag, *sigma, *tau;
    int64_t *ipiv, *perm, *iperm;
    uint8_t* swap;
    int32_t* info;
};

static int cuda_status(cudaError_t e) { return e == cudaSuccess ? LHL_OK : LHL_ERR_CUDA; }

template <class T>
static cudaError_t dalloc(T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc((void**)p, count * sizeof(T));
}

static void ws_free(lhl_ws_t w)
{
    if (!w) return;
    void* ptrs[] = {w->F, w->Ht, w->scale, w->iscale, w->B0, w->part, w->tab, w->cand_v, w->cand_s, w->buf2, w->tsnap,
                    w->bsum, w->bfac, w->ipiv, w->perm, w->iperm, w->cand_i, w->bflag, w->err, w->bar,
                    w->ptimes, w->mhdr, w->mcval, w->mcrow, w->mgrows, w->ybuf, w->zflags, w->tailw, w->linv, w->gmV, w->gmS, w->gmA, w->f32x, w->gmP, w->f32a};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (w->gmH) cudaFreeHost(w->gmH);
    delete w;
}

extern "C" {

const char* lhl_version(void) { return "lhl_gpu 0.1 sm_100a"; }

int lhl_ws_create(int64_t n, int precision, lhl_ws_t* out)
{
    if (!out) return LHL_ERR_ARG;
    *out = nullptr;
    if (n < 0 || n > 16384) return LHL_ERR_DIM;
    if (precision != LHL_PREC_FP64 && precision != LHL_PREC_MIXED) return LHL_ERR_ARG;
    lhl_ws_t w = new (std::nothrow) lhl_ws_s();
    if (!w) return LHL_ERR_ALLOC;
    memset(w, 0, sizeof(*w));
    w->n = n;
    w->precision = precision;
    w->grid = lhl::reduce_grid_size();
    w->limit_ns = 2000000000ull;  // 2 s per barrier wait
    const size_t nn = (size_t)n * (size_t)n;
    const size_t Pmax = (size_t)((n + 63) / 64);
    cudaError_t e = cudaSuccess;
#define A_(p, cnt) if (e == cudaSuccess) e = dalloc(&w->p, (cnt))
    A_(F, nn);
    A_(Ht, nn);
    A_(scale, n);
    A_(iscale, n);
    A_(B0, (size_t)n * 17);
    A_(part, Pmax * n);
    A_(tab, (lhl::stepTabBytes() + 7) / 8);
    A_(cand_v, w->grid > 0 ? w->grid : 1);
    A_(cand_s, w->grid > 0 ? w->grid : 1);
    A_(cand_i, w->grid > 0 ? w->grid : 1);
    A_(buf2, n < 1024 ? nn : 1);  // unblocked path: second buffer (FP64 n < 500; float n < 1024: two)
    A_(tsnap, (size_t)n * 17);
    A_(bsum, 2 * (size_t)n);
    A_(bfac, n);
    A_(ipiv, n > 2 ? n - 2 : 1);
    A_(perm, n);
    A_(iperm, n);
    A_(bflag, 4);
    A_(err, 4);
    A_(bar, 4);
    A_(ptimes, 24);
    w->ycap = 256;
    A_(ybuf, (size_t)n * w->ycap);
    w->nzflags = (int)(((n + 63) / 64) * ((w->ycap + 3) / 4));
    A_(zflags, (size_t)w->nzflags);
    A_(tailw, 64);
    if (precision == LHL_PREC_MIXED && n >= 3) {
        int dev = 0, sms = 0;
        if (e == cudaSuccess) e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) {
            lhl::mixed_plan((int)n, sms, &w->mplan);
            // rows that do not fit on chip need the panel-delayed kernel's shared memory
            if (w->mplan.ok && !w->mplan.smem_rows && !lhl::lazy_fits(w->mplan.ldr)) w->mplan.ok = 0;
            if (!w->mplan.ok) {
                ws_free(w);
                return LHL_ERR_DIM;
            }
        }
        const size_t ldr = (size_t)w->mplan.ldr, g = (size_t)w->mplan.grid;
        A_(mhdr, 2 * g);
        A_(mcval, 2 * (size_t)n + 8 * lhl::MIX_LAZY_LM);  // + the panel-delayed kernel's pivot-row exchange
        // the panel-delayed kernel's ring of candidate rows and global rows are allocated at every
        // order (a test hook can select that kernel where rows would fit on chip)
        A_(mcrow, (size_t)lhl::MIX_LAZY_RING * g * (ldr + lhl::MIX_LAZY_LM));
        A_(mgrows, (size_t)n * ldr);
        A_(linv, (size_t)((n + 63) / 64) * 64 * 64);
    }
#undef A_
    if (e == cudaSuccess) e = cudaMemset(w->err, 0, 4 * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(w->ptimes, 0, 24 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(w->Ht, 0, (nn ? nn : 1) * sizeof(double));
    if (e != cudaSuccess) {
        ws_free(w);
        return e == cudaErrorMemoryAllocation ? LHL_ERR_ALLOC : LHL_ERR_CUDA;
    }
    *out = w;
    return LHL_OK;
}

int lhl_ws_create_f32(int64_t n, int precision, lhl_ws_t* out)
{
    int rc = lhl_ws_create(n, precision, out);
    if (rc != LHL_OK) return rc;
    (*out)->f32 = 1;
    if (n >= 1024 && precision == LHL_PREC_FP64) {
        const size_t cnt = (size_t)n * (size_t)n + 40 * (size_t)n;
        if (cudaMalloc((void**)&(*out)->f32a, cnt * sizeof(float)) != cudaSuccess) {
            (*out)->f32a = nullptr;
            lhl_ws_destroy(*out);
            *out = nullptr;
            return LHL_ERR_ALLOC;
        }
    }
    return LHL_OK;
}

int lhl_ws_create_c128(int64_t n, lhl_ws_t* out)
{
    if (!out) return LHL_ERR_ARG;
    *out = nullptr;
    if (n < 0 || n > lhl::CJ_NMAX) return LHL_ERR_DIM;
    lhl_ws_t w = new (std::nothrow) lhl_ws_s();
    if (!w) return LHL_ERR_ALLOC;
    memset(w, 0, sizeof(*w));
    w->n = n;
    w->precision = LHL_PREC_FP64;
    w->cj = 1;
    w->grid = lhl::cj_grid_size((int)n);
    w->limit_ns = 2000000000ull;
    const size_t nn = (size_t)n * (size_t)n;
    cudaError_t e = cudaSuccess;
#define A_(p, cnt) if (e == cudaSuccess) e = dalloc(&w->p, (cnt))
    A_(F, 2 * nn);
    A_(Ht, 2 * nn);
    A_(buf2, 2 * nn);
    A_(scale, n);
    A_(iscale, n);
    A_(bsum, 2 * (size_t)n);
    A_(bfac, n);
    A_(ipiv, n > 2 ? n - 2 : 1);
    A_(perm, n);
    A_(iperm, n);
    A_(cand_v, w->grid);
    A_(cand_i, w->grid);
    A_(bflag, 4);
    A_(err, 4);
    A_(bar, 4);
    A_(ptimes, 24);
    w->ycap = 256;
    A_(ybuf, (size_t)n * w->ycap);
#undef A_
    if (e == cudaSuccess) e = cudaMemset(w->err, 0, 4 * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(w->ptimes, 0, 24 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(w->Ht, 0, (nn ? 2 * nn : 1) * sizeof(double));
    if (e != cudaSuccess) {
        ws_free(w);
        return e == cudaErrorMemoryAllocation ? LHL_ERR_ALLOC : LHL_ERR_CUDA;
    }
    *out = w;
    return LHL_OK;
}

int lhl_ws_destroy(lhl_ws_t ws)
{
    if (!ws) return LHL_ERR_ARG;
    ws_free(ws);
    return LHL_OK;
}

int lhl_ws_get_view(lhl_ws_t ws, lhl_ws_view* v)
{
    if (!ws || !v) return LHL_ERR_ARG;
    v->n = ws->n;
    v->factors = ws->F;
    v->Ht = ws->Ht;
    v->ipiv = ws->ipiv;
    v->perm = ws->perm;
    v->iperm = ws->iperm;
    v->scale = ws->scale;
    v->iscale = ws->iscale;
    return LHL_OK;
}

int lhl_ws_set_barrier_limit_ns(lhl_ws_t ws, uint64_t limit_ns)
{
    if (!ws || limit_ns == 0) return LHL_ERR_ARG;
    ws->limit_ns = limit_ns;
    return LHL_OK;
}

int lhl_ws_check(lhl_ws_t ws, void* stream)
{
    if (!ws) return LHL_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return LHL_ERR_CUDA;
    int err = 0;
    e = cudaMemcpy(&err, ws->err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return LHL_ERR_CUDA;
    if (err) cudaMemset(ws->err, 0, sizeof(int));
    return err ? err : LHL_OK;
}

int lhl_ws_phase_ns(lhl_ws_t ws, uint64_t* out8, void* stream)
{
    if (!ws || !out8) return LHL_ERR_ARG;
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaMemcpy(out8, ws->ptimes, 8 * sizeof(uint64_t), cudaMemcpyDeviceToHost);
    return cuda_status(e);
}

int lhl_ws_probe_ns(lhl_ws_t ws, uint64_t* out16, void* stream)
{
    if (!ws || !out16) return LHL_ERR_ARG;
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaMemcpy(out16, ws->ptimes + 8, 16 * sizeof(uint64_t), cudaMemcpyDeviceToHost);
    return cuda_status(e);
}

int lhl_ws_set_mixed_kernel(lhl_ws_t ws, int which)
{
    if (!ws) return LHL_ERR_ARG;
    if (which < 0 || which > 2) return LHL_ERR_ARG;
    ws->mix_kernel = which;
    return LHL_OK;
}

int lhl_ws_set_shift_variant(lhl_ws_t ws, int real_variant, int complex_variant)
{
    if (!ws) return LHL_ERR_ARG;
    int T, E, D;
    if (real_variant < 0 || (real_variant > 0 && (!lhl::shift_shape(real_variant, &T, &E, &D) || T * E < ws->n)))
        return LHL_ERR_ARG;
    if (complex_variant < 0 ||
        (complex_variant > 0 && (!lhl::shift_shape_cplx(complex_variant, &T, &E) || T * E < ws->n)))
        return LHL_ERR_ARG;
    ws->shift_variant[0] = real_variant;
    ws->shift_variant[1] = complex_variant;
    return LHL_OK;
}

int lhl_shift_variant_shape(int is_complex, int variant, int* threads, int* per_thread)
{
    if (!threads || !per_thread) return LHL_ERR_ARG;
    int T, E, D;
    const int ok = is_complex ? lhl::shift_shape_cplx(variant, &T, &E) : lhl::shift_shape(variant, &T, &E, &D);
    if (!ok) return LHL_ERR_ARG;
    *threads = T;
    *per_thread = E;
    return LHL_OK;
}

int lhl_ws_set_probes(lhl_ws_t ws, int on)
{
    if (!ws) return LHL_ERR_ARG;
    ws->probes = on ? 1 : 0;
    return LHL_OK;
}

// The reduction of the matrix already copied into ws->F (the entry points below load it).
static int reduce_loaded(lhl_ws_t ws, int balance, cudaStream_t st);

// Float32 workspace: the reduction's factors and Ht rounded to float values, in place (the
// FP64 and mixed reductions; below n = 1024 the plain form already reduces in float)
static int round_reduction_f32(lhl_ws_t ws, cudaStream_t st)
{
    const int n = (int)ws->n;
    if (ws->precision != LHL_PREC_MIXED && (n < 1024 || ws->f32a)) return LHL_OK;
    cudaError_t e = lhl::launch_round_f32(ws->F, n, ws->F, n, n, n, st);
    if (e == cudaSuccess) e = lhl::launch_round_f32(ws->Ht, n, ws->Ht, n, n, n, st);
    return cuda_status(e);
}

int lhl_reduce(lhl_ws_t ws, const double* dJ, int64_t ldj, int balance, void* stream)
{
    if (!ws || (!dJ && ws->n > 0)) return LHL_ERR_ARG;
    if (ws->cj) return LHL_ERR_ARG;  // a complex workspace takes a complex J (lhl_reduce_c128)
    const int64_t n = ws->n;
    if (ldj < n || ldj < 1) return LHL_ERR_DIM;
    if (n == 0) return LHL_OK;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = ws->f32 ? lhl::launch_round_f32(dJ, (int)ldj, ws->F, (int)n, (int)n, (int)n, st)  // J -> Float32
                            : cudaMemcpy2DAsync(ws->F, n * sizeof(double), dJ, ldj * sizeof(double), n * sizeof(double),
                                                n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return LHL_ERR_CUDA;
    int rc = reduce_loaded(ws, balance, st);
    if (rc == LHL_OK && ws->f32) rc = round_reduction_f32(ws, st);
    return rc;
}

int lhl_reduce_f32(lhl_ws_t ws, const float* dJ, int64_t ldj, int balance, void* stream)
{
    if (!ws || (!dJ && ws->n > 0)) return LHL_ERR_ARG;
    if (ws->cj) return LHL_ERR_ARG;
    const int64_t n = ws->n;
    if (ldj < n || ldj < 1) return LHL_ERR_DIM;
    if (n == 0) return LHL_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (lhl::launch_f32_to_f64(dJ, (int)ldj, ws->F, (int)n, (int)n, (int)n, st) != cudaSuccess) return LHL_ERR_CUDA;
    int rc = reduce_loaded(ws, balance, st);
    if (rc == LHL_OK && ws->f32) rc = round_reduction_f32(ws, st);
    return rc;
}

static int reduce_cj_loaded(lhl_ws_t ws, int balance, cudaStream_t st);

int lhl_reduce_c128(lhl_ws_t ws, const double* dJ, int64_t ldj, int balance, void* stream)
{
    if (!ws || (!dJ && ws->n > 0)) return LHL_ERR_ARG;
    if (!ws->cj) return LHL_ERR_ARG;  // a complex J needs a workspace made by lhl_ws_create_c128
    const int64_t n = ws->n;
    if (ldj < n || ldj < 1) return LHL_ERR_DIM;
    if (n == 0) return LHL_OK;
    cudaStream_t st = (cudaStream_t)stream;
    // LHLWorkspace{ComplexF32}: J rounded to ComplexF32 on the way in
    cudaError_t e = ws->f32 ? lhl::launch_round_f32(dJ, (int)(2 * ldj), ws->F, (int)(2 * n), (int)(2 * n), (int)n, st)
                            : cudaMemcpy2DAsync(ws->F, n * 2 * sizeof(double), dJ, ldj * 2 * sizeof(double),
                                                n * 2 * sizeof(double), n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return LHL_ERR_CUDA;
    return reduce_cj_loaded(ws, balance, st);
}

int lhl_ws_create_c64(int64_t n, lhl_ws_t* out)
{
    const int rc = lhl_ws_create_c128(n, out);
    if (rc == LHL_OK) (*out)->f32 = 1;
    return rc;
}

int lhl_reduce_c64(lhl_ws_t ws, const float* dJ, int64_t ldj, int balance, void* stream)
{
    if (!ws || (!dJ && ws->n > 0)) return LHL_ERR_ARG;
    if (!ws->cj) return LHL_ERR_ARG;
    const int64_t n = ws->n;
    if (ldj < n || ldj < 1) return LHL_ERR_DIM;
    if (n == 0) return LHL_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (lhl::launch_f32_to_f64(dJ, (int)(2 * ldj), ws->F, (int)(2 * n), (int)(2 * n), (int)n, st) != cudaSuccess)
        return LHL_ERR_CUDA;
    return reduce_cj_loaded(ws, balance, st);
}

// The reduction of the complex J already in ws->F; on a ComplexF32 workspace the factors and Ht
// are rounded to ComplexF32 values afterwards.
static int reduce_cj_loaded(lhl_ws_t ws, int balance, cudaStream_t st)
{
    const int64_t n = ws->n;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMemsetAsync(ws->bar, 0, sizeof(unsigned int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws->err, 0, sizeof(int), st);
    if (e == cudaSuccess && !balance) e = lhl::launch_fill_ones(ws->scale, ws->iscale, (int)n, st);
    if (e != cudaSuccess) return LHL_ERR_CUDA;
    lhl::CjArgs a;
    memset(&a, 0, sizeof(a));
    a.n = (int)n;
    a.A = ws->F;
    a.B = ws->buf2;
    a.Ht = ws->Ht;
    a.ipiv = ws->ipiv;
    a.perm = ws->perm;
    a.iperm = ws->iperm;
    a.scale = ws->scale;
    a.iscale = ws->iscale;
    a.bsum = ws->bsum;
    a.bfac = ws->bfac;
    a.bflag = ws->bflag;
    a.cand_v = ws->cand_v;
    a.cand_i = ws->cand_i;
    a.bar = ws->bar;
    a.err = ws->err;
    a.limit_ns = ws->limit_ns;
    e = lhl::launch_reduce_cj(a, balance ? 1 : 0, st);
    if (e == cudaSuccess && ws->f32) {
        e = lhl::launch_round_f32(ws->F, (int)(2 * n), ws->F, (int)(2 * n), (int)(2 * n), (int)n, st);
        if (e == cudaSuccess) e = lhl::launch_round_f32(ws->Ht, (int)(2 * n), ws->Ht, (int)(2 * n), (int)(2 * n), (int)n, st);
    }
    return cuda_status(e);
}

static int reduce_loaded(lhl_ws_t ws, int balance, cudaStream_t st)
{
    const int64_t n = ws->n;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMemsetAsync(ws->bar, 0, sizeof(unsigned int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws->err, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws->ptimes, 0, 24 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return LHL_ERR_CUDA;
    lhl::RedArgs a;
    memset(&a, 0, sizeof(a));
    a.n = (int)n;
    a.nb = 16;
    a.A = ws->F;
    a.ipiv = ws->ipiv;
    a.B0 = ws->B0;
    a.part = ws->part;
    a.tab = ws->tab;
    a.cand_v = ws->cand_v;
    a.cand_s = ws->cand_s;
    a.cand_i = ws->cand_i;
    a.buf2 = ws->buf2;
    a.tsnap = ws->tsnap;
    a.scale = ws->scale;
    a.iscale = ws->iscale;
    a.bsum = ws->bsum;
    a.bfac = ws->bfac;
    a.bflag = ws->bflag;
    a.bar = ws->bar;
    a.err = ws->err;
    a.limit_ns = ws->limit_ns;
    a.ptimes = ws->probes ? ws->ptimes : nullptr;
    a.use_tma = (n % 2 == 0) ? 1 : 0;
    if (ws->precision == LHL_PREC_MIXED && n >= 3) {
        // balancing (FP64, the plain kernel's balance-only mode), then the FP32 reduction
        if (!balance) e = lhl::launch_fill_ones(ws->scale, ws->iscale, (int)n, st);
        // exchange words are tagged with their step: clear the previous reduction's
        if (e == cudaSuccess)
            e = cudaMemsetAsync(ws->mhdr, 0, 2 * (size_t)ws->mplan.grid * sizeof(unsigned long long), st);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(ws->mcval, 0, (2 * (size_t)n + 8 * lhl::MIX_LAZY_LM) * sizeof(unsigned long long), st);
        const bool lazy = ws->mix_kernel == 2 || (ws->mix_kernel == 0 && !ws->mplan.smem_rows);
        const size_t ring = lazy ? lhl::MIX_LAZY_RING : 2;
        if (e == cudaSuccess)
            e = cudaMemsetAsync(ws->mcrow, 0,
                                ring * (size_t)ws->mplan.grid * (ws->mplan.ldr + lhl::MIX_LAZY_LM) *
                                    sizeof(unsigned long long), st);
        if (e == cudaSuccess) e = lhl::launch_reduce(a, balance ? 1 : 0, 0, st);
        if (e != cudaSuccess) return LHL_ERR_CUDA;
        lhl::MixArgs m;
        memset(&m, 0, sizeof(m));
        m.n = (int)n;
        m.A = ws->F;
        m.ipiv = ws->ipiv;
        m.perm = ws->perm;
        m.iperm = ws->iperm;
        m.hdr = ws->mhdr;
        m.cval = ws->mcval;
        m.crow = ws->mcrow;
        m.grows = ws->mgrows;
        m.err = ws->err;
        m.limit_ns = ws->limit_ns;
        m.ptimes = ws->probes ? ws->ptimes : nullptr;
        // rows on chip: the eager kernel; rows in global memory: the panel-delayed one
        if (lazy) {
            lhl::MixPlan pl = ws->mplan;
            pl.smem_rows = 0;
            e = lhl::launch_reduce_mixed_lazy(m, pl, st);  // writes perm / iperm too
        } else {
            e = lhl::launch_reduce_mixed(m, ws->mplan, st);  // rows on chip where they fit
        }
        if (e == cudaSuccess) e = lhl::launch_linv((int)n, ws->F, (int)n, ws->linv, st);
        if (e != cudaSuccess) return LHL_ERR_CUDA;
        if (lazy) return cuda_status(lhl::launch_lazy_finish((int)n, ws->F, ws->Ht, st));
        return cuda_status(lhl::launch_ht_fill((int)n, ws->F, ws->Ht, st));
    }
    if (ws->f32 && n >= 1024 && ws->f32a) {
        // LHLWorkspace{Float32} from its blocked threshold: the reference's blocked Float32 form
        if (!balance) e = lhl::launch_fill_ones(ws->scale, ws->iscale, (int)n, st);
        float* A32 = ws->f32a;
        float* B0 = A32 + (size_t)n * n;
        if (e == cudaSuccess)
            e = lhl::launch_reduce_f32_blocked(a, balance ? 1 : 0, A32, B0, B0 + 17 * (size_t)n, B0 + 18 * (size_t)n, st);
        if (e == cudaSuccess) e = lhl::launch_ht_perm((int)n, ws->F, ws->Ht, ws->ipiv, ws->perm, ws->iperm, st);
        return cuda_status(e);
    }
    if (ws->f32 && n < 1024) {
        // LHLWorkspace{Float32} below its blocked threshold: the reference's Float32 arithmetic
        if (!balance) e = lhl::launch_fill_ones(ws->scale, ws->iscale, (int)n, st);
        float* A32 = (float*)ws->buf2;
        if (e == cudaSuccess) e = lhl::launch_reduce_f32(a, balance ? 1 : 0, A32, A32 + (size_t)n * n, st);
        if (e == cudaSuccess)
            e = lhl::launch_unblocked_assemble_f32((int)n, ws->F, A32, A32 + (size_t)n * n, ws->ipiv, st);
        if (e == cudaSuccess) e = lhl::launch_ht_perm((int)n, ws->F, ws->Ht, ws->ipiv, ws->perm, ws->iperm, st);
        return cuda_status(e);
    }
    const int mode = n <= 2 ? 0 : (n < 500 ? 1 : 2);
    if (!balance) {
        // scale = iscale = 1
        e = lhl::launch_fill_ones(ws->scale, ws->iscale, (int)n, st);
        if (e != cudaSuccess) return LHL_ERR_CUDA;
    }
    e = lhl::launch_reduce(a, balance ? 1 : 0, mode, st);
    if (e != cudaSuccess) return LHL_ERR_CUDA;
    if (mode == 1) {
        e = lhl::launch_unblocked_assemble((int)n, ws->F, ws->buf2, ws->ipiv, st);
        if (e != cudaSuccess) return LHL_ERR_CUDA;
    }
    e = lhl::launch_ht_perm((int)n, ws->F, ws->Ht, ws->ipiv, ws->perm, ws->iperm, st);
    return cuda_status(e);
}

int lhl_ws_import(lhl_ws_t ws, const double* dfactors, const double* dHt, const int64_t* dipiv, const int64_t* dperm,
                  const int64_t* diperm, const double* dscale, const double* discale, void* stream)
{
    if (!ws) return LHL_ERR_ARG;
    const int64_t n = ws->n;
    if (n == 0) return LHL_OK;
    if (!dfactors || !dHt || !dperm || !diperm || !dscale || !discale || (n > 2 && !dipiv)) return LHL_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nn = (size_t)n * (size_t)n * (ws->cj ? 2 : 1);  // complex reduction: interleaved pairs
    cudaError_t e = cudaMemcpyAsync(ws->F, dfactors, nn * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ws->Ht, dHt, nn * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && n > 2)
        e = cudaMemcpyAsync(ws->ipiv, dipiv, (size_t)(n - 2) * sizeof(int64_t), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ws->perm, dperm, (size_t)n * sizeof(int64_t), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ws->iperm, diperm, (size_t)n * sizeof(int64_t), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ws->scale, dscale, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ws->iscale, discale, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && ws->precision == LHL_PREC_MIXED && n >= 3)
        e = lhl::launch_linv((int)n, ws->F, (int)n, ws->linv, st);
    return cuda_status(e);
}

static int shift_create(int64_t n, int64_t nshifts, int cplx, lhl_shift_t* out)
{
    if (!out) return LHL_ERR_ARG;
    *out = nullptr;
    if (n < 0 || n > 16384 || nshifts < 1) return LHL_ERR_DIM;
    if (cplx && n > 8192) return LHL_ERR_DIM;
    lhl_shift_t s = new (std::nothrow) lhl_shift_s();
    if (!s) return LHL_ERR_ALLOC;
    memset(s, 0, sizeof(*s));
    s->n = n;
    s->nshifts = nshifts;
    s->cplx = cplx;
    s->po = (n + 4) + ((n + 4) & 1);   // rows per plane, even (16-byte aligned planes)
    s->ldg = cplx ? 2 * s->po : n + 4;
    const int P = cplx ? 2 : 1;
    const size_t gsz = (size_t)s->ldg * (size_t)n * (size_t)nshifts;
    cudaError_t e = dalloc(&s->Gt, gsz);
    if (e == cudaSuccess) e = dalloc(&s->rdiag, (size_t)P * n * nshifts);
    if (e == cudaSuccess) e = dalloc(&s->sigma, (size_t)P * nshifts);
    if (e == cudaSuccess) e = dalloc(&s->tau, (size_t)P * nshifts);
    if (e == cudaSuccess) e = dalloc(&s->swap, (size_t)n * nshifts);
    if (e == cudaSuccess) e = dalloc(&s->info, nshifts);
    if (e == cudaSuccess) e = dalloc(&s->uinv, cplx ? 1 : (size_t)((n + 31) / 32) * 32 * 32 * (size_t)nshifts);
    if (e == cudaSuccess) e = cudaMemset(s->Gt, 0, (gsz ? gsz : 1) * sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(s->info, 0, nshifts * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemset(s->sigma, 0, (size_t)P * nshifts * sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(s->tau, 0, (size_t)P * nshifts * sizeof(double));
    if (e != cudaSuccess) {
        lhl_shift_destroy(s);
        return e == cudaErrorMemoryAllocation ? LHL_ERR_ALLOC : LHL_ERR_CUDA;
    }
    *out = s;
    return LHL_OK;
}

int lhl_shift_create(int64_t n, int64_t nshifts, lhl_shift_t* out) { return shift_create(n, nshifts, 0, out); }

int lhl_shift_create_complex(int64_t n, int64_t nshifts, lhl_shift_t* out)
{
    return shift_create(n, nshifts, 1, out);
}

// LHLShift{Float32} and LHLShift{ComplexF32}: the shift objects of single-precision workspaces
int lhl_shift_create_f32(int64_t n, int64_t nshifts, lhl_shift_t* out)
{
    const int rc = shift_create(n, nshifts, 0, out);
    if (rc == LHL_OK) (*out)->single = 1;
    return rc;
}

int lhl_shift_create_complex64(int64_t n, int64_t nshifts, lhl_shift_t* out)
{
    const int rc = shift_create(n, nshifts, 1, out);
    if (rc == LHL_OK) (*out)->single = 1;
    return rc;
}

int lhl_shift_destroy(lhl_shift_t s)
{
    if (!s) return LHL_ERR_ARG;
    void* ptrs[] = {s->Gt, s->rdiag, s->sigma, s->tau, s->swap, s->info, s->uinv};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete s;
    return LHL_OK;
}

int lhl_shift_get_view(lhl_shift_t s, lhl_shift_view* v)
{
    if (!s || !v) return LHL_ERR_ARG;
    v->n = s->n;
    v->nshifts = s->nshifts;
    v->ldg = s->ldg;
    v->Gt = s->Gt;
    v->swap = s->swap;
    v->rdiag = s->rdiag;
    v->info = s->info;
    v->sigma = s->sigma;
    v->tau = s->tau;
    v->po = s->po;
    v->is_complex = s->cplx;
    return LHL_OK;
}

static int shift_run(lhl_shift_t sh, lhl_ws_t ws, int64_t s0, int64_t count, cudaStream_t st)
{
    cudaError_t e;
    sh->cj = ws->cj;
    if (sh->cplx) {
        // LHLShift{ComplexF32} on a Float32 workspace: sigma and tau rounded to ComplexF32 as the
        // reference stores them; the LU itself runs in FP64 on the float Ht
        if (ws->f32) {
            e = lhl::launch_round_f32(sh->sigma + 2 * s0, (int)(2 * count), sh->sigma + 2 * s0, (int)(2 * count),
                                      (int)(2 * count), 1, st);
            if (e == cudaSuccess)
                e = lhl::launch_round_f32(sh->tau + 2 * s0, (int)(2 * count), sh->tau + 2 * s0, (int)(2 * count),
                                          (int)(2 * count), 1, st);
            if (e != cudaSuccess) return LHL_ERR_CUDA;
        }
        e = lhl::launch_shift_lu_cplx((int)ws->n, ws->Ht, (int)ws->n, sh->sigma + 2 * s0, sh->tau + 2 * s0, (int)s0,
                                      (int)count, sh->Gt, (int)sh->ldg, (int)sh->po, sh->swap, sh->rdiag, sh->info, st,
                                      ws->cj, ws->shift_variant[1]);
        return cuda_status(e);
    }
    e = lhl::launch_shift_lu((int)ws->n, ws->Ht, (int)ws->n, sh->sigma + s0, sh->tau + s0, (int)s0, (int)count,
                             sh->Gt, (int)sh->ldg, sh->swap, sh->rdiag, sh->info, st, ws->f32, ws->shift_variant[0]);
    if (e == cudaSuccess && ws->precision == LHL_PREC_MIXED)
        e = lhl::launch_uinv((int)ws->n, sh->Gt, (int)sh->ldg, sh->rdiag, (int)s0, (int)count, sh->uinv, st);
    return cuda_status(e);
}

static int shift_args(lhl_shift_t sh, lhl_ws_t ws, int64_t s0, int64_t count)
{
    if (!sh || !ws) return LHL_ERR_ARG;
    if (ws->cj && !sh->cplx) return LHL_ERR_ARG;  // an LHLShift{Float64} cannot serve a ComplexF64 workspace (F:2463-2465)
    // an LHLShift{TG} serves an LHLWorkspace{T} for TG = T or Complex{real(T)} only (F:2461-2465)
    if (sh->single != (ws->f32 ? 1 : 0)) return LHL_ERR_ARG;
    if (sh->n != ws->n) return LHL_ERR_DIM;
    if (s0 < 0 || count < 0 || s0 + count > sh->nshifts) return LHL_ERR_DIM;
    return LHL_OK;
}

int lhl_shift_batched(lhl_shift_t sh, lhl_ws_t ws, int64_t s0, int64_t count, const double* dsigma,
                      const double* dtau, void* stream)
{
    int rc = shift_args(sh, ws, s0, count);
    if (rc != LHL_OK) return rc;
    if (count == 0 || ws->n == 0) return LHL_OK;
    if (!dsigma || !dtau) return LHL_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    if (sh->cplx) {  // real shifts on a complex LHLShift: converted (F:2474-2475)
        e = lhl::launch_real_to_cplx(dsigma, sh->sigma + 2 * s0, (int)count, st);
        if (e == cudaSuccess) e = lhl::launch_real_to_cplx(dtau, sh->tau + 2 * s0, (int)count, st);
    } else {
        if (dsigma != sh->sigma + s0)
            e = cudaMemcpyAsync(sh->sigma + s0, dsigma, count * sizeof(double), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess && dtau != sh->tau + s0)
            e = cudaMemcpyAsync(sh->tau + s0, dtau, count * sizeof(double), cudaMemcpyDeviceToDevice, st);
    }
    if (e != cudaSuccess) return LHL_ERR_CUDA;
    return shift_run(sh, ws, s0, count, st);
}

int lhl_shift_batched_complex(lhl_shift_t sh, lhl_ws_t ws, int64_t s0, int64_t count, const double* dsigma,
                              const double* dtau, void* stream)
{
    int rc = shift_args(sh, ws, s0, count);
    if (rc != LHL_OK) return rc;
    if (!sh->cplx) return LHL_ERR_ARG;  // complex shifts need a complex LHLShift (F:2466-2472)
    if (count == 0 || ws->n == 0) return LHL_OK;
    if (!dsigma || !dtau) return LHL_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    if (dsigma != sh->sigma + 2 * s0)
        e = cudaMemcpyAsync(sh->sigma + 2 * s0, dsigma, 2 * count * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && dtau != sh->tau + 2 * s0)
        e = cudaMemcpyAsync(sh->tau + 2 * s0, dtau, 2 * count * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return LHL_ERR_CUDA;
    return shift_run(sh, ws, s0, count, st);
}

int lhl_shift_complex(lhl_shift_t sh, lhl_ws_t ws, int64_t slot, double sigma_re, double sigma_im, double tau_re,
                      double tau_im, void* stream)
{
    int rc = shift_args(sh, ws, slot, 1);
    if (rc != LHL_OK) return rc;
    if (!sh->cplx) {
        if (sigma_im != 0.0 || tau_im != 0.0) return LHL_ERR_ARG;  // F:2466-2472
        return lhl_shift(sh, ws, slot, sigma_re, tau_re, stream);
    }
    if (ws->n == 0) return LHL_OK;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = lhl::launch_set_pair(sh->sigma + 2 * slot, sh->sigma + 2 * slot + 1, sigma_re, sigma_im, st);
    if (e == cudaSuccess) e = lhl::launch_set_pair(sh->tau + 2 * slot, sh->tau + 2 * slot + 1, tau_re, tau_im, st);
    if (e != cudaSuccess) return LHL_ERR_CUDA;
    return shift_run(sh, ws, slot, 1, st);
}

int lhl_shift(lhl_shift_t sh, lhl_ws_t ws, int64_t slot, double sigma, double tau, void* stream)
{
    int rc = shift_args(sh, ws, slot, 1);
    if (rc != LHL_OK) return rc;
    if (sh->cplx) return lhl_shift_complex(sh, ws, slot, sigma, 0.0, tau, 0.0, stream);
    if (ws->n == 0) return LHL_OK;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = lhl::launch_set_pair(sh->sigma + slot, sh->tau + slot, sigma, tau, st);
    if (e != cudaSuccess) return LHL_ERR_CUDA;
    return shift_run(sh, ws, slot, 1, st);
}

// Complex shifts with many right-hand sides: the solve scratch Y (n x ycap real columns) grows
// so that one pass of the solve kernels covers every right-hand side (each complex one is two
// real columns), up to 1 GiB; the multi-right-hand-side Hessenberg solve then has every
// shift's group of vectors in one launch.  Grow-only; a failed allocation keeps the old buffer
// (the solve then runs in chunks of it).  cudaFree waits for work in flight on the old one.
static void ws_grow_y(lhl_ws_t ws, lhl_shift_t sh, int64_t nrhs)
{
    if (!sh || !sh->cplx || ws->cj || ws->n <= 0) return;
    const int64_t want = 2 * nrhs;
    if (want <= ws->ycap) return;
    const int64_t cap_max = (int64_t)((1ull << 30) / (8ull * (uint64_t)ws->n));
    const int64_t cap = want < cap_max ? want : cap_max;
    if (cap <= ws->ycap) return;
    const int64_t nflags = ((ws->n + 63) / 64) * ((cap + 3) / 4);
    double* y = nullptr;
    int* f = nullptr;
    if (cudaMalloc((void**)&y, (size_t)ws->n * (size_t)cap * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    if (cudaMalloc((void**)&f, (size_t)nflags * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(y);
        return;
    }
    cudaFree(ws->ybuf);
    cudaFree(ws->zflags);
    ws->ybuf = y;
    ws->zflags = f;
    ws->ycap = (int)cap;
    ws->nzflags = (int)nflags;
}

static int ldiv_common(lhl_shift_t sh, lhl_ws_t ws, double* dX, int64_t ldx, int64_t nrhs, int64_t rps, int mode,
                       cudaStream_t st)
{
    const int64_t n = ws->n;
    if (nrhs < 0) return LHL_ERR_DIM;
    if (nrhs == 0 || n == 0) return LHL_OK;
    if (!dX) return LHL_ERR_ARG;
    if (ldx < n) return LHL_ERR_DIM;
    if (n > 8192) return LHL_ERR_DIM;
    if (ws->cj && sh && !sh->cplx) return LHL_ERR_ARG;
    if (mode == 0) ws_grow_y(ws, sh, nrhs);
    lhl::LdivArgs a;
    memset(&a, 0, sizeof(a));
    a.n = (int)n;
    a.cj = ws->cj;
    a.F = ws->F;
    a.ldf = (int)n;
    a.perm = ws->perm;
    a.iperm = ws->iperm;
    a.scale = ws->scale;
    a.iscale = ws->iscale;
    a.X = dX;
    a.ldx = (int)ldx;
    a.mode = mode;
    a.rhs_per_shift = 1;
    a.Y = ws->ybuf;
    a.ycap = ws->ycap;
    a.linv = ws->linv;  // null for the plain form
    a.zflags = ws->zflags;
    a.nzflags = ws->nzflags;
    a.tail = ws->tailw;
    a.err = ws->err;
    a.limit_ns = ws->limit_ns;
    if (sh) {
        a.Gt = sh->Gt;
        a.ldg = (int)sh->ldg;
        a.swp = sh->swap;
        a.rdiag = sh->rdiag;
        a.rhs_per_shift = (int)rps;
        a.nshifts = (int)sh->nshifts;
        a.uinv = (ws->precision == LHL_PREC_MIXED && !sh->cplx) ? sh->uinv : nullptr;
        a.cplx = sh->cplx;
        a.po = (int)sh->po;
    }
    return cuda_status(lhl::launch_ldiv(a, (int)nrhs, st));
}

int lhl_ldiv(lhl_shift_t sh, lhl_ws_t ws, double* dX, int64_t ldx, int64_t nrhs, int64_t rhs_per_shift, void* stream)
{
    if (!sh || !ws) return LHL_ERR_ARG;
    if (sh->n != ws->n) return LHL_ERR_DIM;
    if (rhs_per_shift < 1) return LHL_ERR_ARG;
    if (nrhs > 0 && (nrhs + rhs_per_shift - 1) / rhs_per_shift > sh->nshifts) return LHL_ERR_DIM;
    return ldiv_common(sh, ws, dX, ldx, nrhs, rhs_per_shift, 0, (cudaStream_t)stream);
}

int lhl_ldiv_complex_rhs(lhl_shift_t sh, lhl_ws_t ws, double* dX, int64_t ldx, int64_t nrhs, int64_t rhs_per_shift,
                         void* stream)
{
    if (!sh || !ws) return LHL_ERR_ARG;
    if (sh->cplx) return lhl_ldiv(sh, ws, dX, ldx, nrhs, rhs_per_shift, stream);  // a complex shift: as always
    if (sh->n != ws->n) return LHL_ERR_DIM;
    if (ws->cj) return LHL_ERR_ARG;  // a complex J takes complex shift objects only
    if (rhs_per_shift < 1) return LHL_ERR_ARG;
    if (nrhs < 0) return LHL_ERR_DIM;
    if (nrhs > 0 && (nrhs + rhs_per_shift - 1) / rhs_per_shift > sh->nshifts) return LHL_ERR_DIM;
    const int64_t n = ws->n;
    if (nrhs == 0 || n == 0) return LHL_OK;
    if (!dX) return LHL_ERR_ARG;
    if (ldx < n) return LHL_ERR_DIM;
    cudaStream_t st = (cudaStream_t)stream;
    // a real shift is real-linear: the real and imaginary parts solve as two real columns
    const size_t need = 2 * (size_t)n * (size_t)nrhs;
    if (ws->f32x_cap < need || !ws->f32x) {
        if (ws->f32x) cudaFree(ws->f32x);
        ws->f32x = nullptr;
        ws->f32x_cap = 0;
        if (cudaMalloc((void**)&ws->f32x, need * sizeof(double)) != cudaSuccess) return LHL_ERR_ALLOC;
        ws->f32x_cap = need;
    }
    if (lhl::launch_split_complex(dX, (int)ldx, ws->f32x, (int)n, (int)nrhs, st) != cudaSuccess) return LHL_ERR_CUDA;
    const int rc = ldiv_common(sh, ws, ws->f32x, n, 2 * nrhs, 2 * rhs_per_shift, 0, st);
    if (rc != LHL_OK) return rc;
    return cuda_status(lhl::launch_join_complex(ws->f32x, (int)n, dX, (int)ldx, (int)nrhs, st));
}

int lhl_ldiv_f32(lhl_shift_t sh, lhl_ws_t ws, float* dX, int64_t ldx, int64_t nrhs, int64_t rhs_per_shift,
                 void* stream)
{
    if (!sh || !ws) return LHL_ERR_ARG;
    if (sh->n != ws->n) return LHL_ERR_DIM;
    if (rhs_per_shift < 1) return LHL_ERR_ARG;
    if (nrhs < 0) return LHL_ERR_DIM;
    if (nrhs > 0 && (nrhs + rhs_per_shift - 1) / rhs_per_shift > sh->nshifts) return LHL_ERR_DIM;
    const int64_t n = ws->n;
    if (nrhs == 0 || n == 0) return LHL_OK;
    if (!dX) return LHL_ERR_ARG;
    if (ldx < n) return LHL_ERR_DIM;
    cudaStream_t st = (cudaStream_t)stream;
    // a complex shift takes ComplexF32 vectors: interleaved, 2n floats per column, ld 2 ldx
    const int P = sh->cplx ? 2 : 1;
    const size_t need = (size_t)P * (size_t)n * (size_t)nrhs;
    if (ws->f32x_cap < need || !ws->f32x) {
        if (ws->f32x) cudaFree(ws->f32x);
        ws->f32x = nullptr;
        ws->f32x_cap = 0;
        if (cudaMalloc((void**)&ws->f32x, need * sizeof(double)) != cudaSuccess) return LHL_ERR_ALLOC;
        ws->f32x_cap = need;
    }
    if (lhl::launch_f32_to_f64(dX, (int)(P * ldx), ws->f32x, (int)(P * n), (int)(P * n), (int)nrhs, st) !=
        cudaSuccess)
        return LHL_ERR_CUDA;
    const int rc = ldiv_common(sh, ws, ws->f32x, n, nrhs, rhs_per_shift, 0, st);
    if (rc != LHL_OK) return rc;
    return cuda_status(
        lhl::launch_f64_to_f32(ws->f32x, (int)(P * n), dX, (int)(P * ldx), (int)(P * n), (int)nrhs, st));
}

int lhl_applyZ(lhl_ws_t ws, double* dX, int64_t ldx, int64_t nrhs, void* stream)
{
    if (!ws) return LHL_ERR_ARG;
    return ldiv_common(nullptr, ws, dX, ldx, nrhs, 1, 2, (cudaStream_t)stream);
}

int lhl_applyZinv(lhl_ws_t ws, double* dX, int64_t ldx, int64_t nrhs, void* stream)
{
    if (!ws) return LHL_ERR_ARG;
    return ldiv_common(nullptr, ws, dX, ldx, nrhs, 1, 1, (cudaStream_t)stream);
}

// residual, norms and update for real or complex (interleaved) right-hand sides
static cudaError_t resid_any(lhl_shift_t sh, int64_t n, const double* dJ, int64_t ldj, const double* dB, int64_t ldb,
                             const double* dX, int64_t ldx, double* dR, int64_t ldr, int64_t nrhs, int64_t rps,
                             cudaStream_t st, const double* done, double tol)
{
    if (sh->cplx && sh->cj)  // complex J (the slots came from a complex reduction)
        return lhl::launch_residual_cj((int)n, dJ, (int)ldj, dB, (int)ldb, dX, (int)ldx, dR, (int)ldr, (int)nrhs,
                                       (int)rps, sh->sigma, sh->tau, st, done, tol);
    if (sh->cplx)
        return lhl::launch_residual_cplx((int)n, dJ, (int)ldj, dB, (int)ldb, dX, (int)ldx, dR, (int)ldr, (int)nrhs,
                                         (int)rps, sh->sigma, sh->tau, st, done, tol);
    return lhl::launch_residual((int)n, dJ, (int)ldj, dB, (int)ldb, dX, (int)ldx, dR, (int)ldr, (int)nrhs, (int)rps,
                                sh->sigma, sh->tau, st, done, tol);
}

static cudaError_t relres_any(lhl_shift_t sh, int64_t n, const double* dR, int64_t ldr, const double* dB,
                              int64_t ldb, double* dres, int64_t nrhs, cudaStream_t st)
{
    const int P = sh->cplx ? 2 : 1;  // an interleaved complex column is a real vector of 2n
    return lhl::launch_relres((int)(P * n), dR, (int)(P * ldr), dB, (int)(P * ldb), dres, (int)nrhs, st);
}

static cudaError_t axpy_any(lhl_shift_t sh, int64_t n, double* dX, int64_t ldx, const double* dR, int64_t ldr,
                            int64_t nrhs, cudaStream_t st, const double* done, double tol)
{
    const int P = sh->cplx ? 2 : 1;
    return lhl::launch_axpy_cols((int)(P * n), dX, (int)(P * ldx), dR, (int)(P * ldr), (int)nrhs, st, done, tol);
}

int lhl_refine(lhl_shift_t sh, lhl_ws_t ws, const double* dJ, int64_t ldj, const double* dB, int64_t ldb, double* dX,
               int64_t ldx, double* dR, int64_t nrhs, int64_t rhs_per_shift, int steps, void* stream)
{
    if (!sh || !ws) return LHL_ERR_ARG;
    if (ws->cj && !sh->cplx) return LHL_ERR_ARG;
    const int64_t n = ws->n;
    if (sh->n != n) return LHL_ERR_DIM;
    if (rhs_per_shift < 1 || steps < 0) return LHL_ERR_ARG;
    if (nrhs < 0) return LHL_ERR_DIM;
    if (nrhs == 0 || n == 0 || steps == 0) return LHL_OK;
    if (!dJ || !dB || !dX || !dR) return LHL_ERR_ARG;
    if (ldj < n || ldb < n || ldx < n) return LHL_ERR_DIM;
    if ((nrhs + rhs_per_shift - 1) / rhs_per_shift > sh->nshifts) return LHL_ERR_DIM;
    cudaStream_t st = (cudaStream_t)stream;
    for (int s = 0; s < steps; ++s) {
        cudaError_t e = resid_any(sh, n, dJ, ldj, dB, ldb, dX, ldx, dR, ldx, nrhs, rhs_per_shift, st, nullptr, 0.0);
        if (e != cudaSuccess) return LHL_ERR_CUDA;
        int rc = ldiv_common(sh, ws, dR, ldx, nrhs, rhs_per_shift, 0, st);
        if (rc != LHL_OK) return rc;
        e = axpy_any(sh, n, dX, ldx, dR, ldx, nrhs, st, nullptr, 0.0);
        if (e != cudaSuccess) return LHL_ERR_CUDA;
    }
    return LHL_OK;
}

// lhl_ldiv's arguments for the refinement loops: R in place, columns with done[c] <= tol skipped
static lhl::LdivArgs refine_ldiv_args(lhl_shift_t sh, lhl_ws_t ws, double* dR, int64_t ldr, int64_t rps,
                                      const double* done, double tol, int64_t nrhs)
{
    ws_grow_y(ws, sh, nrhs);
    lhl::LdivArgs a;
    memset(&a, 0, sizeof(a));
    a.n = (int)ws->n;
    a.cj = ws->cj;
    a.F = ws->F;
    a.ldf = (int)ws->n;
    a.perm = ws->perm;
    a.iperm = ws->iperm;
    a.scale = ws->scale;
    a.iscale = ws->iscale;
    a.X = dR;
    a.ldx = (int)ldr;
    a.mode = 0;
    a.Gt = sh->Gt;
    a.ldg = (int)sh->ldg;
    a.swp = sh->swap;
    a.rdiag = sh->rdiag;
    a.rhs_per_shift = (int)rps;
    a.nshifts = (int)sh->nshifts;
    a.uinv = (ws->precision == LHL_PREC_MIXED && !sh->cplx) ? sh->uinv : nullptr;
    a.cplx = sh->cplx;
    a.po = (int)sh->po;
    a.linv = ws->linv;
    a.done = done;
    a.tol = tol;
    a.Y = ws->ybuf;
    a.ycap = ws->ycap;
    a.zflags = ws->zflags;
    a.nzflags = ws->nzflags;
    a.tail = ws->tailw;
    a.err = ws->err;
    a.limit_ns = ws->limit_ns;
    return a;
}

static int refine_args_check(lhl_shift_t sh, lhl_ws_t ws, const double* dJ, int64_t ldj, const double* dB,
                             int64_t ldb, const double* dX, int64_t ldx, const double* dR, const double* dres,
                             int64_t nrhs, int64_t rhs_per_shift, double tol, bool bad_count)
{
    if (!sh || !ws) return LHL_ERR_ARG;
    if (ws->cj && !sh->cplx) return LHL_ERR_ARG;
    const int64_t n = ws->n;
    if (sh->n != n) return LHL_ERR_DIM;
    if (rhs_per_shift < 1 || bad_count || !(tol >= 0.0)) return LHL_ERR_ARG;
    if (nrhs < 0) return LHL_ERR_DIM;
    if (nrhs == 0 || n == 0) return LHL_OK;
    if (!dJ || !dB || !dX || !dR || !dres) return LHL_ERR_ARG;
    if (ldj < n || ldb < n || ldx < n) return LHL_ERR_DIM;
    if ((nrhs + rhs_per_shift - 1) / rhs_per_shift > sh->nshifts) return LHL_ERR_DIM;
    if (n > 8192) return LHL_ERR_DIM;
    return LHL_OK;
}

int lhl_refine_tol(lhl_shift_t sh, lhl_ws_t ws, const double* dJ, int64_t ldj, const double* dB, int64_t ldb,
                   double* dX, int64_t ldx, double* dR, double* dres, int64_t nrhs, int64_t rhs_per_shift, double tol,
                   int max_steps, void* stream)
{
    const int chk =
        refine_args_check(sh, ws, dJ, ldj, dB, ldb, dX, ldx, dR, dres, nrhs, rhs_per_shift, tol, max_steps < 0);
    if (chk != LHL_OK || nrhs == 0 || ws->n == 0) return chk;
    const int64_t n = ws->n;
    cudaStream_t st = (cudaStream_t)stream;
    for (int s = 0; s <= max_steps; ++s) {
        // step 0 computes every residual; later steps only those of unconverged columns
        cudaError_t e = resid_any(sh, n, dJ, ldj, dB, ldb, dX, ldx, dR, ldx, nrhs, rhs_per_shift, st,
                                  s > 0 ? dres : nullptr, tol);
        if (e == cudaSuccess) e = relres_any(sh, n, dR, ldx, dB, ldb, dres, nrhs, st);
        if (e != cudaSuccess) return LHL_ERR_CUDA;
        if (s == max_steps) break;
        e = lhl::launch_ldiv(refine_ldiv_args(sh, ws, dR, ldx, rhs_per_shift, dres, tol, nrhs), (int)nrhs, st);
        if (e == cudaSuccess) e = axpy_any(sh, n, dX, ldx, dR, ldx, nrhs, st, dres, tol);
        if (e != cudaSuccess) return LHL_ERR_CUDA;
    }
    return LHL_OK;
}

// grow-only device buffer of the workspace
static cudaError_t ws_grow(double** p, size_t* cap, size_t need)
{
    if (*cap >= need && *p) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc((void**)p, need * sizeof(double));
    if (e == cudaSuccess) *cap = need;
    return e;
}

int lhl_refine_gmres(lhl_shift_t sh, lhl_ws_t ws, const double* dJ, int64_t ldj, const double* dB, int64_t ldb,
                     double* dX, int64_t ldx, double* dR, double* dres, int64_t nrhs, int64_t rhs_per_shift,
                     double tol, int max_cycles, int restart, int host_check, void* stream)
{
    const int chk = refine_args_check(sh, ws, dJ, ldj, dB, ldb, dX, ldx, dR, dres, nrhs, rhs_per_shift, tol,
                                      max_cycles < 0 || restart < 1 || restart > 32);
    if (chk != LHL_OK || nrhs == 0 || ws->n == 0) return chk;
    // Complex shifts: GMRES on the realified system.  An interleaved complex column of n
    // entries is a real vector of 2n; the product with W and the preconditioner are real-linear
    // maps of it, and the real inner product is Re<v, w>.  The Arnoldi kernels run on 2n reals.
    const int P = sh->cplx ? 2 : 1;
    const int n = (int)ws->n, ne = P * n, m = restart, nr = (int)nrhs;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = ws_grow(&ws->gmV, &ws->gmV_cap, (size_t)nr * (m + 1) * ne);
    if (e == cudaSuccess) e = ws_grow(&ws->gmS, &ws->gmS_cap, (size_t)nr * lhl::gm_state_doubles(m));
    if (e == cudaSuccess) e = ws_grow(&ws->gmA, &ws->gmA_cap, (size_t)nr);
    if (e == cudaSuccess) e = ws_grow(&ws->gmP, &ws->gmP_cap, (size_t)nr);
    if (e == cudaSuccess && host_check && (ws->gmH_cap < (size_t)nr || !ws->gmH)) {
        if (ws->gmH) cudaFreeHost(ws->gmH);
        ws->gmH = nullptr;
        ws->gmH_cap = 0;
        e = cudaHostAlloc((void**)&ws->gmH, (size_t)nr * sizeof(double), cudaHostAllocDefault);
        if (e == cudaSuccess) ws->gmH_cap = (size_t)nr;
    }
    if (e != cudaSuccess) return LHL_ERR_ALLOC;
    const int ldv = (m + 1) * n;  // in (complex) elements: column c's vector i at gmV + P (c ldv + i n)
    for (int cyc = 0; cyc <= max_cycles; ++cyc) {
        e = resid_any(sh, n, dJ, ldj, dB, ldb, dX, ldx, dR, ldx, nrhs, rhs_per_shift, st, cyc > 0 ? dres : nullptr,
                      tol);
        if (e == cudaSuccess) e = relres_any(sh, n, dR, ldx, dB, ldb, dres, nrhs, st);
        if (e != cudaSuccess) return LHL_ERR_CUDA;
        if (cyc == max_cycles) break;
        // the columns that take this cycle: above tol and not stagnated
        e = lhl::launch_gm_mark(dres, ws->gmP, ws->gmA, tol, cyc == 0, nr, st);
        if (e != cudaSuccess) return LHL_ERR_CUDA;
        if (host_check) {
            e = cudaMemcpyAsync(ws->gmH, ws->gmA, (size_t)nr * sizeof(double), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return LHL_ERR_CUDA;
            bool none = true;
            for (int c = 0; c < nr && none; ++c) none = !(ws->gmH[c] > 0.5);
            if (none) break;
        }
        // z = W~^-1 r for those columns, then the cycle's Arnoldi steps
        e = lhl::launch_ldiv(refine_ldiv_args(sh, ws, dR, ldx, rhs_per_shift, ws->gmA, 0.5, nr), nr, st);
        if (e == cudaSuccess)
            e = lhl::launch_gm_begin(ne, m, dR, (int)(P * ldx), ws->gmV, ws->gmS, ws->gmA, dres, tol, nr, st);
        for (int j = 0; j < m && e == cudaSuccess; ++j) {
            e = resid_any(sh, n, dJ, ldj, nullptr, 0, ws->gmV + (size_t)P * j * n, ldv, dR, ldx, nrhs,
                          rhs_per_shift, st, ws->gmA, 0.5);
            if (e == cudaSuccess)
                e = lhl::launch_ldiv(refine_ldiv_args(sh, ws, dR, ldx, rhs_per_shift, ws->gmA, 0.5, nr), nr, st);
            if (e == cudaSuccess)
                e = lhl::launch_gm_arnoldi(ne, m, j, dR, (int)(P * ldx), ws->gmV, ws->gmS, ws->gmA, nr, st);
        }
        if (e == cudaSuccess) e = lhl::launch_gm_update(ne, m, dX, (int)(P * ldx), ws->gmV, ws->gmS, nr, st);
        if (e != cudaSuccess) return LHL_ERR_CUDA;
    }
    return LHL_OK;
}

// (sigma, tau) = (0, 1) as real values and as interleaved complex pairs: a shift view with these
// makes the residual kernels apply the caller's system matrix A itself, r = b - A x.
__device__ double g_system_shift[4] = {0.0, 0.0, 1.0, 0.0};

// One slot of a shift object as a shift batch of its own whose residuals take a system matrix:
// the slot's factorisation (Gt, swap, rdiag, U block inverses) and (sigma, tau) = (0, 1).  A
// complex shift's system matrix is complex (the complex-J residual).
static int system_view(lhl_shift_t sh, int64_t slot, lhl_shift_s* v)
{
    if (!sh) return LHL_ERR_ARG;
    if (slot < 0 || slot >= sh->nshifts) return LHL_ERR_DIM;
    void* u = nullptr;
    if (cudaGetSymbolAddress(&u, g_system_shift) != cudaSuccess) return LHL_ERR_CUDA;
    *v = *sh;
    const size_t n = (size_t)sh->n;
    const size_t P = sh->cplx ? 2 : 1;
    v->Gt = sh->Gt + (size_t)slot * (size_t)sh->ldg * n;
    v->swap = sh->swap + (size_t)slot * n;
    v->rdiag = sh->rdiag + (size_t)slot * P * n;
    if (!sh->cplx) v->uinv = sh->uinv + (size_t)slot * ((n + 31) / 32) * 32 * 32;
    v->info = sh->info + slot;
    v->sigma = (double*)u;
    v->tau = (double*)u + 2;
    v->nshifts = 1;
    v->cj = sh->cplx;
    return LHL_OK;
}

int lhl_refine_system(lhl_shift_t sh, lhl_ws_t ws, int64_t slot, const double* dA, int64_t lda, const double* dB,
                      int64_t ldb, double* dX, int64_t ldx, double* dR, double* dres, int64_t nrhs, double tol,
                      int max_steps, void* stream)
{
    lhl_shift_s v;
    const int rc = system_view(sh, slot, &v);
    if (rc != LHL_OK) return rc;
    return lhl_refine_tol(&v, ws, dA, lda, dB, ldb, dX, ldx, dR, dres, nrhs, nrhs > 0 ? nrhs : 1, tol, max_steps,
                          stream);
}

int lhl_refine_system_gmres(lhl_shift_t sh, lhl_ws_t ws, int64_t slot, const double* dA, int64_t lda,
                            const double* dB, int64_t ldb, double* dX, int64_t ldx, double* dR, double* dres,
                            int64_t nrhs, double tol, int max_cycles, int restart, int host_check, void* stream)
{
    lhl_shift_s v;
    const int rc = system_view(sh, slot, &v);
    if (rc != LHL_OK) return rc;
    return lhl_refine_gmres(&v, ws, dA, lda, dB, ldb, dX, ldx, dR, dres, nrhs, nrhs > 0 ? nrhs : 1, tol, max_cycles,
                            restart, host_check, stream);
}

int lhl_residual_norms(lhl_shift_t sh, const double* dJ, int64_t ldj, const double* dB, int64_t ldb,
                       const double* dX, int64_t ldx, double* dR, double* dres, int64_t nrhs, int64_t rhs_per_shift,
                       void* stream)
{
    if (!sh) return LHL_ERR_ARG;
    const int64_t n = sh->n;
    if (rhs_per_shift < 1) return LHL_ERR_ARG;
    if (nrhs < 0) return LHL_ERR_DIM;
    if (nrhs == 0 || n == 0) return LHL_OK;
    if (!dJ || !dB || !dX || !dR || !dres) return LHL_ERR_ARG;
    if (ldj < n || ldb < n || ldx < n) return LHL_ERR_DIM;
    if ((nrhs + rhs_per_shift - 1) / rhs_per_shift > sh->nshifts) return LHL_ERR_DIM;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = resid_any(sh, n, dJ, ldj, dB, ldb, dX, ldx, dR, ldx, nrhs, rhs_per_shift, st, nullptr, 0.0);
    if (e != cudaSuccess) return LHL_ERR_CUDA;
    return cuda_status(relres_any(sh, n, dR, ldx, dB, ldb, dres, nrhs, st));
}


// ---- batches of independent matrices of uneven order ----
static lhl::BatchDesc batch_desc(lhl_batch_t b)
{
    lhl::BatchDesc d;
    d.count = (int)b->count;
    d.S = (int)b->S;
    d.n = b->d_n;
    d.off2 = b->d_off2;
    d.off1 = b->d_off1;
    d.offg = b->d_offg;
    d.F = b->F;
    d.Ht = b->Ht;
    d.ipiv = b->ipiv;
    d.perm = b->perm;
    d.iperm = b->iperm;
    d.scale = b->scale;
    d.iscale = b->iscale;
    d.Gt = b->Gt;
    d.swap = b->swap;
    d.rdiag = b->rdiag;
    d.info = b->info;
    return d;
}

int lhl_batch_destroy(lhl_batch_t b)
{
    if (!b) return LHL_ERR_ARG;
    void* ptrs[] = {b->d_n, b->d_off2, b->d_off1, b->d_offg, b->F, b->Ht, b->scale, b->iscale, b->Gt, b->rdiag,
                    b->sigma, b->tau, b->ipiv, b->perm, b->iperm, b->swap, b->info};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    free(b->ns_host);
    delete b;
    return LHL_OK;
}

int lhl_batch_create(int64_t count, const int64_t* ns, int64_t shifts_per_matrix, lhl_batch_t* out)
{
    if (!out || !ns) return LHL_ERR_ARG;
    *out = nullptr;
    if (count < 1 || shifts_per_matrix < 1 || count * shifts_per_matrix > (1ll << 30)) return LHL_ERR_DIM;
    for (int64_t m = 0; m < count; ++m)
        if (ns[m] < 1 || ns[m] > lhl::BATCH_NMAX) return LHL_ERR_DIM;
    lhl_batch_t b = new (std::nothrow) lhl_batch_s();
    if (!b) return LHL_ERR_ALLOC;
    memset(b, 0, sizeof(*b));
    b->count = count;
    b->S = shifts_per_matrix;
    b->ns_host = (int64_t*)malloc(count * sizeof(int64_t));
    int* hn = (int*)malloc(count * sizeof(int));
    int64_t* h2 = (int64_t*)malloc(count * sizeof(int64_t));
    int64_t* h1 = (int64_t*)malloc(count * sizeof(int64_t));
    int64_t* hg = (int64_t*)malloc(count * sizeof(int64_t));
    if (!b->ns_host || !hn || !h2 || !h1 || !hg) {
        free(hn); free(h2); free(h1); free(hg);
        lhl_batch_destroy(b);
        return LHL_ERR_ALLOC;
    }
    int64_t o2 = 0, o1 = 0, og = 0;
    for (int64_t m = 0; m < count; ++m) {
        const int64_t n = ns[m];
        b->ns_host[m] = n;
        hn[m] = (int)n;
        h2[m] = o2;
        h1[m] = o1;
        hg[m] = og;
        o2 += n * n;
        o1 += n;
        og += b->S * (n + 4) * n;
    }
    b->total_nn = o2;
    b->total_n = o1;
    b->total_g = og;
    const int64_t S = b->S;
    cudaError_t e = cudaSuccess;
#define A_(p, cnt) if (e == cudaSuccess) e = dalloc(&b->p, (size_t)(cnt))
    A_(d_n, count);
    A_(d_off2, count);
    A_(d_off1, count);
    A_(d_offg, count);
    A_(F, o2);
    A_(Ht, o2);
    A_(scale, o1);
    A_(iscale, o1);
    A_(ipiv, o1);
    A_(perm, o1);
    A_(iperm, o1);
    A_(Gt, og);
    A_(rdiag, S * o1);
    A_(swap, S * o1);
    A_(info, S * count);
    A_(sigma, S * count);
    A_(tau, S * count);
#undef A_
    if (e == cudaSuccess) e = cudaMemcpy(b->d_n, hn, count * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_off2, h2, count * sizeof(int64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_off1, h1, count * sizeof(int64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_offg, hg, count * sizeof(int64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(b->Gt, 0, (og ? og : 1) * sizeof(double));
    free(hn); free(h2); free(h1); free(hg);
    if (e != cudaSuccess) {
        lhl_batch_destroy(b);
        return e == cudaErrorMemoryAllocation ? LHL_ERR_ALLOC : LHL_ERR_CUDA;
    }
    *out = b;
    return LHL_OK;
}

int lhl_batch_get_view(lhl_batch_t b, lhl_batch_view* v)
{
    if (!b || !v) return LHL_ERR_ARG;
    v->count = b->count;
    v->shifts = b->S;
    v->total_n = b->total_n;
    v->total_nn = b->total_nn;
    v->total_g = b->total_g;
    v->factors = b->F;
    v->Ht = b->Ht;
    v->ipiv = b->ipiv;
    v->perm = b->perm;
    v->iperm = b->iperm;
    v->scale = b->scale;
    v->iscale = b->iscale;
    v->Gt = b->Gt;
    v->swap = b->swap;
    v->rdiag = b->rdiag;
    v->info = b->info;
    v->sigma = b->sigma;
    v->tau = b->tau;
    return LHL_OK;
}

int lhl_reduce_batched(lhl_batch_t b, const double* dJ, int balance, void* stream)
{
    if (!b || !dJ) return LHL_ERR_ARG;
    return cuda_status(lhl::launch_reduce_batch(batch_desc(b), dJ, balance ? 1 : 0, (cudaStream_t)stream));
}

int lhl_shift_batched_all(lhl_batch_t b, const double* dsigma, const double* dtau, void* stream)
{
    if (!b || !dsigma || !dtau) return LHL_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t cnt = (size_t)b->S * b->count;
    cudaError_t e = cudaSuccess;
    if (dsigma != b->sigma) e = cudaMemcpyAsync(b->sigma, dsigma, cnt * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && dtau != b->tau)
        e = cudaMemcpyAsync(b->tau, dtau, cnt * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = lhl::launch_shift_lu_batch(batch_desc(b), b->sigma, b->tau, st);
    return cuda_status(e);
}

int lhl_solve_batched(lhl_batch_t b, const double* dJ, const double* dB, double* dX, int64_t rhs_per_shift, double tol,
                      int max_steps, double* dres, void* stream)
{
    if (!b || !dJ || !dB || !dX) return LHL_ERR_ARG;
    if (rhs_per_shift < 1 || max_steps < 0 || !(tol >= 0.0)) return LHL_ERR_ARG;
    if (b->count * b->S * rhs_per_shift > (1ll << 31) - 1) return LHL_ERR_DIM;
    return cuda_status(lhl::launch_solve_batch(batch_desc(b), dJ, dB, dX, (int)rhs_per_shift, b->sigma, b->tau, tol,
                                               max_steps, dres, (cudaStream_t)stream));
}

}  // extern "C"
