// reduce.cu -- lhl_reduce! on sm_100a: balancing (F:299-340), the unblocked ELMHES
// reduction (n < 500, F:466-678) and the blocked delayed-update reduction (n >= 500,
// F:765-1006 with its helpers), Ht fill (F:2005-2061) and perm / iperm (F:376-387).
//
// Plain FP64 form: every element of H and L is produced by the same sequence of IEEE
// operations as the reference's Float64 path on x86-64 (fused multiply-add exactly where
// the reference calls llvm.fmuladd), so pivots, H and L are bit-identical to a faithful
// CPU restatement.  Summation orders are the reference's own: 64-column GEMV groups with
// four-column passes, group sums added in order, per-element fma chains in the panel-end
// products.  Parallelism comes from rows, columns and column groups, never from
// reassociating a sum.
//
// Both reductions are single cooperative launches: one CTA per SM, phases separated by
// a grid barrier whose wait is bounded (common.cuh).  The matrix stays in HBM/L2,
// column-major with leading dimension n.
#include "internal.cuh"

#include <cudaTypedefs.h>

namespace lhl {

constexpr int RT = 256;        // threads per CTA of the reduction kernels
constexpr int RW = RT / 32;    // warps per CTA
constexpr int NBMAX = 16;      // panel width nb (F:706)
constexpr int GEMV_GROUP = 64; // _LHL_GEMV_GROUP (F:1451)
constexpr int PMAX = 256;      // column groups (n <= 16384)
constexpr int T64_SLOTS = 5;   // 64x64 FP64 tiles in flight per CTA in the GEMV phase
constexpr int TILE64_BYTES = 64 * 64 * 8;
constexpr int PBOX_G = 32;     // groups per TMA box of GEMV partials (phase B)
constexpr int PBOX_BYTES = RT * PBOX_G * 8;
constexpr int PBOX_SLOTS = 2;
// A TMA wait gives up after the workspace's wall-time limit, but never sooner than this: a copy
// in flight completes in microseconds, so a short limit (the tests of the timeout path use 1 ns)
// still ends the kernel at a grid barrier with no copy in flight into its shared memory.
constexpr unsigned long long TMA_WAIT_FLOOR_NS = 100000000ull;
__device__ __forceinline__ unsigned long long tma_wait_ns(const RedArgs& a)
{
    return a.limit_ns > TMA_WAIT_FLOOR_NS ? a.limit_ns : TMA_WAIT_FLOOR_NS;
}


// ---------------------------------------------------------------------------------
// Per-step table written by one warp in phase A and read by every CTA in phase B.
// ---------------------------------------------------------------------------------
struct StepTab {
    int p, pulled, nov, skip;
    double piv;
    double R1[NBMAX + 2], RP[NBMAX + 2], PJ[NBMAX + 2], VJ[NBMAX + 2], CX[NBMAX + 2];
    double OV[2 * NBMAX + 4];
    int OR[2 * NBMAX + 4];
};

// Phase timers: CTA 0, thread 0 adds the wall time since the last mark to slot `slot`.
__device__ __forceinline__ void tmark(const RedArgs& a, int slot, uint64_t& last)
{
    if (blockIdx.x == 0 && threadIdx.x == 0 && a.ptimes) {
        const uint64_t t = globaltimer_ns();
        a.ptimes[slot] += t - last;
        last = t;
    }
}

// Finer probe: thread 0 of CTA `cta` adds the time since `last` into slot 8 + slot.
__device__ __forceinline__ void tprobe(const RedArgs& a, int cta, int slot, uint64_t& last)
{
    if (blockIdx.x == cta && threadIdx.x == 0 && a.ptimes) {
        const uint64_t t = globaltimer_ns();
        a.ptimes[8 + slot] += t - last;
        last = t;
    }
}

__device__ __forceinline__ void combine_candidates(const RedArgs& a, int* s_p, double* s_red, int* s_redi)
{
    // every CTA reads all CTA candidates and reduces them (first max, F:1038-1051)
    const int t = threadIdx.x;
    double v = 0.0;
    int vi = 0;
    for (int c = t; c < (int)gridDim.x; c += RT) {
        const int ci = ((volatile int*)a.cand_i)[c];
        const double cv = ((volatile double*)a.cand_v)[c];
        argmax_combine(v, vi, cv, ci);
    }
    warp_argmax(v, vi);
    if ((t & 31) == 0) {
        s_red[t >> 5] = v;
        s_redi[t >> 5] = vi;
    }
    __syncthreads();
    if (t == 0) {
        double bv = 0.0;
        int bi = 0;
        for (int w = 0; w < RW; ++w) argmax_combine(bv, bi, s_red[w], s_redi[w]);
        *s_p = bi;
    }
    __syncthreads();
}

// CTA-local first-max over this thread's candidate, published to cand[blockIdx.x].
__device__ __forceinline__ void publish_candidate(const RedArgs& a, double v, int vi, double* s_red, int* s_redi)
{
    warp_argmax(v, vi);
    const int t = threadIdx.x;
    if ((t & 31) == 0) {
        s_red[t >> 5] = v;
        s_redi[t >> 5] = vi;
    }
    __syncthreads();
    if (t == 0) {
        double bv = 0.0;
        int bi = 0;
        for (int w = 0; w < RW; ++w) argmax_combine(bv, bi, s_red[w], s_redi[w]);
        a.cand_v[blockIdx.x] = bv;
        a.cand_i[blockIdx.x] = bi;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------------
// Balancing (F:299-340).  Per sweep: (1) every index's column and row 1-norm (without
// the diagonal), each one summed sequentially in the reference's order by one thread;
// (2) CTA 0 walks i = 1..n in order taking the reference's decision, RT indices at a
// time: the first index of the chunk that scales is applied, the sums of the indices
// still to come are patched for it (its row and column entries change by the factor),
// and the walk resumes after it; (3) all CTAs apply the sweep's power-of-two factors to A
// (exact).  The decision of an index after an in-sweep scaling therefore reads a patched
// sum, which differs from a fresh sequential sum by rounding only.
// ---------------------------------------------------------------------------------
__device__ bool balance_phase(const RedArgs& a, GridBarrier& gb)
{
    const int n = a.n;
    double* A = a.A;
    const int gt = blockIdx.x * RT + threadIdx.x;
    const int gsz = gridDim.x * RT;
    for (int i = gt; i < n; i += gsz) {
        a.scale[i] = 1.0;
        a.iscale[i] = 1.0;
    }
    __shared__ int s_first;
    __shared__ double s_f;
    for (int sweep = 0; sweep < 20; ++sweep) {
        // (1) sums, sequential per index in the reference's order, loads in batches
        for (int i = 1 + gt; i <= n; i += gsz) {
            double c = 0.0, r = 0.0;
            int j = 1;
            for (; j + 7 <= n; j += 8) {
                double vc[8], vr[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    vc[u] = M1(A, n, j + u, i);
                    vr[u] = M1(A, n, i, j + u);
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    if (j + u == i) continue;
                    c += fabs(vc[u]);
                    r += fabs(vr[u]);
                }
            }
            for (; j <= n; ++j) {
                if (j == i) continue;
                c += fabs(M1(A, n, j, i));
                r += fabs(M1(A, n, i, j));
            }
            a.bsum[i - 1] = c;
            a.bsum[n + i - 1] = r;
            a.bfac[i - 1] = 1.0;
        }
        if (gt == 0) a.bflag[0] = 0;
        if (!gb.sync()) return false;
        // (2) the ordered decision walk, CTA 0
        if (blockIdx.x == 0) {
            int base = 1;
            while (base <= n) {
                if (threadIdx.x == 0) s_first = 0x7fffffff;
                __syncthreads();
                const int i = base + threadIdx.x;
                double f = 1.0;
                if (i <= n && balance_decide(a.bsum[i - 1], a.bsum[n + i - 1], f)) atomicMin(&s_first, i);
                __syncthreads();
                const int si = s_first;
                if (si == 0x7fffffff) {
                    base += RT;
                    continue;
                }
                if (i == si) {
                    s_f = f;
                    a.bflag[0] = 1;
                }
                __syncthreads();
                const double fs = s_f;
                // patch the sums of m > si: row si's entry in column m is divided by fs,
                // column si's entry in row m multiplied (indices > si are unscaled so far)
                // (four indices per thread at a time, every load issued before the stores)
                for (int m0 = si + 1 + threadIdx.x; m0 <= n; m0 += 4 * RT) {
                    double vr[4], vc[4], br[4], bc[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int m = m0 + u * RT;
                        if (m <= n) {
                            vr[u] = fabs(M1(A, n, si, m));
                            vc[u] = fabs(M1(A, n, m, si));
                            br[u] = a.bsum[m - 1];
                            bc[u] = a.bsum[n + m - 1];
                        }
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int m = m0 + u * RT;
                        if (m <= n) {
                            a.bsum[m - 1] = (br[u] - vr[u]) + vr[u] / fs;
                            a.bsum[n + m - 1] = (bc[u] - vc[u]) + vc[u] * fs;
                        }
                    }
                }
                if (threadIdx.x == 0) {
                    a.bfac[si - 1] = fs;
                    a.scale[si - 1] *= fs;
                    a.iscale[si - 1] /= fs;
                }
                __syncthreads();
                base = si + 1;
            }
        }
        if (!gb.sync()) return false;
        const int scaled = ((volatile int*)a.bflag)[0];
        if (!scaled) break;
        // (3) apply: A[i,j] <- A[i,j] / fac[i] * fac[j] (powers of two, exact)
        for (size_t e = gt; e < (size_t)n * n; e += gsz) {
            const int i = (int)(e % n), j = (int)(e / n);
            const double fi = a.bfac[i], fj = a.bfac[j];
            if (fi != 1.0 || fj != 1.0) A[e] = (A[e] / fi) * fj;
        }
        if (!gb.sync()) return false;
    }
    return true;
}

// ---------------------------------------------------------------------------------
// Unblocked reduction (F:466-501), per-row semantics of the row-block kernel (F:547-678)
// for n >= 8 and of the paired sweep (F:508-538) below.  Step k reads the matrix of step
// k-1 (buffer (k-1)&1, rows and columns k+1 <-> p swapped on the fly) and writes buffer
// k&1, one thread per row, so a step needs one grid barrier (the pivot search).  Column
// j's final values land in buffer j&1 at step j; later interchanges reach them in the
// final assembly.
// ---------------------------------------------------------------------------------
template <typename T>
__device__ bool unblocked_phase(const RedArgs& a, GridBarrier& gb, T* A0, T* A1)
{
    const int n = a.n;
    T* buf[2] = {A0, A1};
    __shared__ T s_l[4096 / sizeof(T)];  // n < 512 (FP64) or n < 1024 (float)
    __shared__ double s_red[RW];
    __shared__ int s_redi[RW];
    __shared__ int s_p;
    const int gt = blockIdx.x * RT + threadIdx.x;
    // this thread's row: rows by warps spread over the CTAs (global warp w = local warp * grid +
    // CTA holds rows 32 w + 1 .. 32 w + 32), so that many SMs stream the matrix each step
    const int i = 32 * ((threadIdx.x >> 5) * (int)gridDim.x + (int)blockIdx.x) + (threadIdx.x & 31) + 1;
    const bool generic = n < 8;

    // candidates for column 1
    {
        double v = 0.0;
        int vi = 0;
        if (i >= 2 && i <= n) { v = fabs((double)M1(A0, n, i, 1)); vi = i; }
        publish_candidate(a, v, vi, s_red, s_redi);
    }
    if (!gb.sync()) return false;
    for (int k = 1; k <= n - 2; ++k) {
        const T* R = buf[(k - 1) & 1];
        T* W = buf[k & 1];
        combine_candidates(a, &s_p, s_red, s_redi);
        const int p = (s_p >= k + 1 && s_p <= n) ? s_p : k + 1;
        if (gt == 0) a.ipiv[k - 1] = p;
        auto sw = [&](int r) { return r == k + 1 ? p : (r == p ? k + 1 : r); };
        const T piv = M1(R, n, p, k);
        // multipliers l_j = A'[j,k] / piv, j = k+2..n, into shared memory
        for (int j = k + 2 + threadIdx.x; j <= n; j += RT)
            s_l[j - 1] = (piv != (T)0) ? M1(R, n, sw(j), k) / piv : M1(R, n, sw(j), k);
        __syncthreads();
        double cand = 0.0;
        int candi = 0;
        if (i <= n) {
            const int si = sw(i);
            // column k
            T ck = M1(R, n, si, k);
            if (piv != (T)0 && i >= k + 2) ck = s_l[i - 1];
            M1(W, n, i, k) = ck;
            // column k+1 (swapped with p), left update by pk = A'[k+1,k+1]
            T ck1 = M1(R, n, si, p);
            if (piv == (T)0) {
                // step skipped (F:488): rows/columns still carry the interchange
                for (int j = k + 2; j <= n; ++j) M1(W, n, i, j) = M1(R, n, si, sw(j));
                M1(W, n, i, k + 1) = ck1;
            } else {
                const T pk = M1(R, n, p, p);
                const T li = (i >= k + 2) ? s_l[i - 1] : (T)0;
                if (pk != (T)0 && i >= k + 2) ck1 = dsub(ck1, dmul(li, pk));
                if (!generic) {
                    T s = 0;
                    const bool low = i >= k + 2;
                    int j = k + 2;
                    // sixteen columns at a time: every load of the block is issued before its
                    // stores (a store to W could otherwise hold back the next load from R)
                    for (; j + 15 <= n; j += 16) {
                        T v[16], pr[16];
#pragma unroll
                        for (int u = 0; u < 16; ++u) {
                            const int sj = sw(j + u);
                            v[u] = M1(R, n, si, sj);
                            pr[u] = low ? M1(R, n, p, sj) : (T)0;
                        }
#pragma unroll
                        for (int u = 0; u < 16; ++u) {
                            T x = v[u];
                            if (low) x = dfma(li, -pr[u], x);
                            M1(W, n, i, j + u) = x;
                            s = dfma(s_l[j + u - 1], x, s);
                        }
                    }
                    for (; j <= n; ++j) {
                        const int sj = sw(j);
                        T v = M1(R, n, si, sj);
                        if (low) v = dfma(li, -M1(R, n, p, sj), v);
                        M1(W, n, i, j) = v;
                        s = dfma(s_l[j - 1], v, s);
                    }
                    ck1 = dadd(ck1, s);
                } else {
                    int j = k + 2;
                    while (j + 1 <= n) {
                        T v0 = M1(R, n, si, sw(j)), v1 = M1(R, n, si, sw(j + 1));
                        if (i >= k + 2) {
                            v0 = dsub(v0, dmul(li, M1(R, n, p, sw(j))));
                            v1 = dsub(v1, dmul(li, M1(R, n, p, sw(j + 1))));
                        }
                        M1(W, n, i, j) = v0;
                        M1(W, n, i, j + 1) = v1;
                        ck1 = dadd(ck1, dadd(dmul(s_l[j - 1], v0), dmul(s_l[j], v1)));
                        j += 2;
                    }
                    if (j <= n) {
                        T v0 = M1(R, n, si, sw(j));
                        if (i >= k + 2) v0 = dsub(v0, dmul(li, M1(R, n, p, sw(j))));
                        M1(W, n, i, j) = v0;
                        ck1 = dadd(ck1, dmul(s_l[j - 1], v0));
                    }
                }
                M1(W, n, i, k + 1) = ck1;
            }
            if (i >= k + 2) { cand = fabs((double)ck1); candi = i; }
        }
        publish_candidate(a, cand, candi, s_red, s_redi);
        if (!gb.sync()) return false;
    }
    return true;
}

// Final assembly of the unblocked result into a.A: column j from buffer j&1 (columns
// n-1, n from the last step's buffer), with the interchanges of steps j+1..n-2 applied
// (the reference applies them as they happen, F:480-485).  One CTA per column.
template <typename T>
__global__ void __launch_bounds__(RT) unblocked_assemble_kernel(int n, double* out, const T* A, const T* B2,
                                                                const int64_t* ipiv)
{
    const int j = blockIdx.x + 1;
    if (j > n) return;
    const T* src;
    int from;
    if (j <= n - 2) {
        src = (j & 1) ? B2 : A;
        from = j + 1;
    } else {
        const int kl = n - 2;  // last step
        src = (kl >= 1 && (kl & 1)) ? B2 : A;
        from = n - 1;
    }
    __shared__ T col[4096 / sizeof(T)];
    for (int i = threadIdx.x; i < n; i += RT) col[i] = src[(size_t)(j - 1) * n + i];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = from; k <= n - 2; ++k) {
            const int p = (int)ipiv[k - 1];
            if (p > k + 1 && p <= n) {
                const T t = col[k];
                col[k] = col[p - 1];
                col[p - 1] = t;
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += RT) out[(size_t)(j - 1) * n + i] = (double)col[i];
}

// ---------------------------------------------------------------------------------
// LHLWorkspace{Float32} below _lhl_block_min(Float32) = 1024 (F:703-705): J rounded to
// float, balancing in float (F:299-340 with Tr = Float32) and the unblocked ELMHES in float
// with the row-block kernel's per-row fma order (F:547-678; the paired sweep F:508-538 below
// n = 8), so pivots, factors, Ht and scale are the reference's Float32 results.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ bool balance_decide_f32(float c, float r, float& f)
{
    if (c == 0.0f || r == 0.0f) return false;
    f = 1.0f;
    const float s = __fadd_rn(c, r);
    int guard = 0;  // never reached by finite norms; ends the loops on an infinite one
    while (c < __fdiv_rn(r, 2.0f) && guard < 4200) {
        c = __fmul_rn(c, 2.0f);
        r = __fdiv_rn(r, 2.0f);
        f = __fmul_rn(f, 2.0f);
        ++guard;
    }
    while (c >= __fmul_rn(2.0f, r) && guard < 8400) {
        c = __fdiv_rn(c, 2.0f);
        r = __fmul_rn(r, 2.0f);
        f = __fdiv_rn(f, 2.0f);
        ++guard;
    }
    return __fadd_rn(c, r) < __fmul_rn(0.95f, s);
}

// Column and row 1-norms of index i without the diagonal, summed in j order, of the matrix
// as the reference holds it when its sweep reaches i: the sweep's starting matrix with the
// factors of the indices scaled so far in the sweep (row j divided by fac[j], column j
// multiplied, the same single operations the reference applies); fac == nullptr: none yet.
__device__ __forceinline__ void bal_sums_f32(const float* A, int n, int i, const double* fac, float& c, float& r)
{
    c = 0.0f;
    r = 0.0f;
    int j = 1;
    for (; j + 7 <= n; j += 8) {
        float vc[8], vr[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            vc[u] = M1(A, n, j + u, i);
            vr[u] = M1(A, n, i, j + u);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (j + u == i) continue;
            const float fc = fac ? __fdiv_rn(vc[u], (float)fac[j + u - 1]) : vc[u];
            const float fr = fac ? __fmul_rn(vr[u], (float)fac[j + u - 1]) : vr[u];
            c = __fadd_rn(c, fabsf(fc));
            r = __fadd_rn(r, fabsf(fr));
        }
    }
    for (; j <= n; ++j) {
        if (j == i) continue;
        const float vc = M1(A, n, j, i), vr = M1(A, n, i, j);
        c = __fadd_rn(c, fabsf(fac ? __fdiv_rn(vc, (float)fac[j - 1]) : vc));
        r = __fadd_rn(r, fabsf(fac ? __fmul_rn(vr, (float)fac[j - 1]) : vr));
    }
}

// Balancing in float.  Per sweep: (1) every index's sums from the sweep's starting matrix,
// one thread per index; (2) CTA 0 walks i = 1..n in order, RT indices at a time, and takes
// the first index of the chunk that scales; once an index has scaled in the sweep, every
// later chunk sums afresh with the sweep's factors so far (bal_sums_f32), so each decision
// reads exactly the reference's sums; (3) all CTAs apply the sweep's factors to A in the
// reference's order per element (row i divided when i is reached, column j multiplied when
// j is: (a / f_i) f_j for i <= j, (a f_j) / f_i otherwise).
__device__ bool balance_phase_f32(const RedArgs& a, float* A, GridBarrier& gb)
{
    const int n = a.n;
    const int gt = blockIdx.x * RT + threadIdx.x;
    const int gsz = gridDim.x * RT;
    for (int i = gt; i < n; i += gsz) {
        a.scale[i] = 1.0;
        a.iscale[i] = 1.0;
    }
    __shared__ int s_first;
    for (int sweep = 0; sweep < 20; ++sweep) {
        for (int i = 1 + gt; i <= n; i += gsz) {
            float c, r;
            bal_sums_f32(A, n, i, nullptr, c, r);
            a.bsum[i - 1] = c;
            a.bsum[n + i - 1] = r;
            a.bfac[i - 1] = 1.0;
        }
        if (gt == 0) a.bflag[0] = 0;
        if (!gb.sync()) return false;
        if (blockIdx.x == 0) {
            bool fresh = false;  // an index has scaled in this sweep: sum afresh
            int base = 1;
            __syncthreads();
            while (base <= n) {
                if (threadIdx.x == 0) s_first = 0x7fffffff;
                __syncthreads();
                const int i = base + threadIdx.x;
                float f = 1.0f;
                if (i <= n) {
                    float c, r;
                    if (fresh) {
                        bal_sums_f32(A, n, i, a.bfac, c, r);
                    } else {
                        c = (float)a.bsum[i - 1];
                        r = (float)a.bsum[n + i - 1];
                    }
                    if (balance_decide_f32(c, r, f)) atomicMin(&s_first, i);
                }
                __syncthreads();
                const int si = s_first;
                if (si == 0x7fffffff) {
                    base += RT;
                    continue;
                }
                if (i == si) {
                    a.bfac[si - 1] = f;
                    a.bflag[0] = 1;
                    a.scale[si - 1] = __fmul_rn((float)a.scale[si - 1], f);
                    a.iscale[si - 1] = __fdiv_rn((float)a.iscale[si - 1], f);
                }
                __syncthreads();
                fresh = true;
                base = si + 1;
            }
        }
        if (!gb.sync()) return false;
        const int scaled = ((volatile int*)a.bflag)[0];
        if (!scaled) break;
        for (size_t e = gt; e < (size_t)n * n; e += gsz) {
            const int i = (int)(e % n), j = (int)(e / n);
            const float fi = (float)a.bfac[i], fj = (float)a.bfac[j];
            if (fi != 1.0f || fj != 1.0f)
                A[e] = i <= j ? __fmul_rn(__fdiv_rn(A[e], fi), fj) : __fdiv_rn(__fmul_rn(A[e], fj), fi);
        }
        if (!gb.sync()) return false;
    }
    return true;
}

// ---------------------------------------------------------------------------------
// The blocked Float32 form (n >= 1024): the reference's pointer path (F:765-1006 and its
// helpers) with T = Float32.  Its vector width only spreads rows over lanes, so every element
// sees the operations of the Float64 path in the same order: per step the pivot, the step
// table (the rows k+1 and p of the panel columns, the pulled column's values and corrections,
// F:1088-1132), the multipliers, the GEMV over the trailing columns in 64-column groups of
// four-column passes with the group sums added in order (F:1451-1553), the row kernel (row and
// column interchange, the pulled column, left and right transforms inside the panel,
// F:1166-1296) and the correction of w by the panel's interchanges and left transforms; at the
// panel end the row interchanges, the TRSM through the explicit (M^-1 - I) (F:1944-1955), the
// rank-16 GEMM as fused multiply-add chains, the top rows' panel part and their fma chain
// over the trailing columns (F:1588-1672); after the last panel the deferred interchanges.
// Not tuned: one thread per row walks its row of the trailing block in each step's GEMV.
// ---------------------------------------------------------------------------------
constexpr int FB = 16;  // panel width (F:706)
struct F32Tab {
    int p, skip, pulled, nov;
    float piv;
    float R1[FB + 2], RP[FB + 2], PJ[FB + 2], OV[2 * FB + 4], CX[FB + 1];
    int OR[2 * FB + 4];
};
struct F32Chain {
    float LW[FB + 2], LQ[FB + 2], XS[FB + 1];
    int LR[FB + 2];
    int nq;
};

// One 64-column group's part of row i's GEMV (F:1496-1553): multipliers l_j = A[j,k] (already
// divided by the pivot); column psub is read from `sub`.
__device__ __forceinline__ float f32_gemv_group(const float* A, int n, int k, int i, int c0, int c1, int psub,
                                                const float* sub)
{
    auto col = [&](int j) -> float { return j == psub ? sub[i - 1] : M1(A, n, i, j); };
    float out;
    int j = c0;
    if (j + 3 <= c1) {
        const float l1 = M1(A, n, j, k), l2 = M1(A, n, j + 1, k), l3 = M1(A, n, j + 2, k), l4 = M1(A, n, j + 3, k);
        out = dadd(dadd(dmul(l1, col(j)), dmul(l2, col(j + 1))), dadd(dmul(l3, col(j + 2)), dmul(l4, col(j + 3))));
        j += 4;
    } else {
        out = dmul(M1(A, n, j, k), col(j));
        j += 1;
    }
    for (; j + 3 <= c1; j += 4) {
        const float l1 = M1(A, n, j, k), l2 = M1(A, n, j + 1, k), l3 = M1(A, n, j + 2, k), l4 = M1(A, n, j + 3, k);
        out = dadd(out, dadd(dadd(dmul(l1, col(j)), dmul(l2, col(j + 1))), dadd(dmul(l3, col(j + 2)), dmul(l4, col(j + 3)))));
    }
    for (; j <= c1; ++j) {
        const float lj = M1(A, n, j, k);
        if (lj != 0.0f) out = dadd(out, dmul(lj, col(j)));
    }
    return out;
}

// The interchange of a step whose pivot is zero (the generic step swaps, F:857-890), CTA 0 alone.
__device__ void f32_step_swaps(float* A, int n, float* B0, const int64_t* ipiv, int k0, int kb, int k, int p)
{
    const int t = threadIdx.x;
    if (t == 0)
        for (int j = k0; j <= kb + 1; ++j) {
            if (j == k) continue;
            const float x = M1(A, n, k + 1, j);
            M1(A, n, k + 1, j) = M1(A, n, p, j);
            M1(A, n, p, j) = x;
        }
    __syncthreads();
    if (p <= kb + 1) {
        for (int i = 1 + t; i <= n; i += RT) {
            float x = M1(A, n, i, k + 1);
            M1(A, n, i, k + 1) = M1(A, n, i, p);
            M1(A, n, i, p) = x;
            x = M1(B0, n, i, k + 1 - k0);
            M1(B0, n, i, k + 1 - k0) = M1(B0, n, i, p - k0);
            M1(B0, n, i, p - k0) = x;
        }
        __syncthreads();
        return;
    }
    for (int i = 1 + t; i <= n; i += RT) {
        const float x = M1(A, n, i, p);
        M1(A, n, i, p) = M1(B0, n, i, k + 1 - k0);
        M1(B0, n, i, k + 1 - k0) = x;
        M1(A, n, i, k + 1) = x;
    }
    __syncthreads();
    if (t == 0)
        for (int kk = k0; kk <= k; ++kk) {
            const int q = (int)ipiv[kk - 1];
            if (q != kk + 1) {
                const float x = M1(A, n, kk + 1, k + 1);
                M1(A, n, kk + 1, k + 1) = M1(A, n, q, k + 1);
                M1(A, n, q, k + 1) = x;
            }
        }
    __syncthreads();
    for (int kk = k0; kk <= k - 1; ++kk) {
        const float x = M1(A, n, kk + 1, k + 1);
        if (x != 0.0f)
            for (int i = kk + 2 + t; i <= n; i += RT) M1(A, n, i, k + 1) = dsub(M1(A, n, i, k + 1), dmul(M1(A, n, i, kk), x));
        __syncthreads();
    }
}

// The step table (thread 0 of every CTA, from the matrix as the previous step left it; no
// writes): F:1060-1132 of the pointer path.  Column k's rows k+1 and p are exchanged later by
// their owners, so every CTA reads the same values here.
__device__ void f32_step_table(const RedArgs& a, const float* A, int n, F32Tab& T, int k0, int kb, int k, int p)
{
    T.p = p;
    for (int j = k0; j <= kb + 1; ++j) {
        T.R1[j - k0] = M1(A, n, k + 1, j);
        T.RP[j - k0] = M1(A, n, p, j);
    }
    const float piv = T.RP[k - k0];  // A[k+1, k] after the exchange
    T.piv = piv;
    T.pulled = p > kb + 1;
    T.skip = piv == 0.0f;
    T.nov = 0;
    if (T.skip) return;
    if (T.pulled) {  // pulled_tables (F:1088-1132)
        const int m = k - k0 + 1;
        for (int kk = k0; kk <= k; ++kk) {
            T.OV[kk - k0] = M1(A, n, kk + 1, p);
            T.OR[kk - k0] = kk + 1;
        }
        int nov = m;
        for (int kk = k0; kk <= k; ++kk) {
            const int q = kk == k ? p : (int)a.ipiv[kk - 1];  // step k's entry may not be visible yet
            if (q == kk + 1) continue;
            int sl = -1;
            for (int r = 0; r < nov; ++r)
                if (T.OR[r] == q) { sl = r; break; }
            if (sl < 0) {
                sl = nov++;
                T.OV[sl] = M1(A, n, q, p);
                T.OR[sl] = q;
            }
            const float x = T.OV[kk - k0];
            T.OV[kk - k0] = T.OV[sl];
            T.OV[sl] = x;
        }
        for (int kk = k0; kk <= k - 1; ++kk) {
            const float x = T.OV[kk - k0];
            T.CX[kk - k0] = x;
            if (x == 0.0f) continue;
            for (int i = kk + 2; i <= k + 1; ++i) {
                const float aik = (i == k + 1) ? T.RP[kk - k0] : M1(A, n, i, kk);
                T.OV[i - k0 - 1] = dsub(T.OV[i - k0 - 1], dmul(aik, x));
            }
        }
        T.nov = nov;
    }
    for (int j = k + 1; j <= kb + 1; ++j) T.PJ[j - k - 1] = T.RP[j - k0];
    if (T.pulled) {
        T.PJ[0] = T.OV[k - k0];
    } else if (p != k + 1) {
        T.PJ[0] = T.RP[p - k0];
        T.PJ[p - k - 1] = T.RP[k + 1 - k0];
    }
}

// blocked float reduction over A (n x n floats, ld n), after balancing; scratch: B0 (n x 17),
// w (n), pre (n x 17), the step table in global memory
__device__ bool f32_blocked(const RedArgs& a, GridBarrier& gb, float* A, float* B0, float* w, float* pre)
{
    const int n = a.n;
    __shared__ double s_red[RW];
    __shared__ int s_redi[RW];
    __shared__ F32Tab T;
    __shared__ F32Chain C;
    __shared__ float Pm[FB][FB];
    __shared__ float Bs[FB];
    __shared__ int s_p;
    const int t = threadIdx.x;
    const int gt = blockIdx.x * RT + t, gsz = gridDim.x * RT;
    const int i = 32 * ((t >> 5) * (int)gridDim.x + (int)blockIdx.x) + (t & 31) + 1;  // this thread's row
    {
        double v = 0.0;
        int vi = 0;
        if (i >= 2 && i <= n) { v = fabs((double)M1(A, n, i, 1)); vi = i; }
        publish_candidate(a, v, vi, s_red, s_redi);
    }
    if (!gb.sync()) return false;
    for (int k0 = 1; k0 <= n - 2; k0 += FB) {
        const int kb = k0 + FB - 1 < n - 2 ? k0 + FB - 1 : n - 2;
        const int np = kb + 1 - k0;
        for (size_t e = gt; e < (size_t)n * np; e += gsz) {
            const int r = (int)(e % n) + 1, jj = (int)(e / n) + 1;
            M1(B0, n, r, jj) = M1(A, n, r, k0 + jj);
        }
        if (!gb.sync()) return false;
        for (int k = k0; k <= kb; ++k) {
            // the pivot: first maximum of |A[k+1:n, k]| (F:1038-1051), then the step table
            combine_candidates(a, &s_p, s_red, s_redi);
            const int p = (s_p >= k + 1 && s_p <= n) ? s_p : k + 1;
            if (gt == 0) a.ipiv[k - 1] = p;
            if (t == 0) f32_step_table(a, A, n, T, k0, kb, k, p);
            __syncthreads();
            if (T.skip) {
                // a zero pivot: the interchange alone (F:1054-1057, generic step swaps), CTA 0
                if (!gb.sync()) return false;
                if (blockIdx.x == 0 && p != k + 1) {
                    if (t == 0) {
                        const float x = M1(A, n, k + 1, k);
                        M1(A, n, k + 1, k) = M1(A, n, p, k);
                        M1(A, n, p, k) = x;
                    }
                    __syncthreads();
                    f32_step_swaps(A, n, B0, a.ipiv, k0, kb, k, p);
                }
                if (!gb.sync()) return false;
            }
            if (!T.skip) {
                const float piv = T.piv;
                // column k's exchange of rows k+1 and p, and the multipliers (F:1058,
                // F:1506-1509) of every row below k+1; every CTA has read its table first
                if (!gb.sync()) return false;
                if (i == k + 1) M1(A, n, k + 1, k) = piv;
                if (i >= k + 2 && i <= n) M1(A, n, i, k) = __fdiv_rn(i == p ? T.R1[k - k0] : M1(A, n, i, k), piv);
                if (!gb.sync()) return false;
                const bool trailing = kb + 2 <= n;
                float wi = 0.0f;
                if (i >= 1 && i <= n) {
                    // GEMV of this row over the trailing columns, groups of 64 added in order
                    if (trailing && i >= k0 + 1) {
                        const float* sub = T.pulled ? B0 + (size_t)(k - k0) * n : nullptr;
                        const int psub = T.pulled ? p : 0;
                        for (int ga = kb + 2; ga <= n; ga += 64) {
                            const int gb2 = ga + 63 < n ? ga + 63 : n;
                            const float part = f32_gemv_group(A, n, k, i, ga, gb2, psub, sub);
                            wi = ga == kb + 2 ? part : dadd(wi, part);
                        }
                        w[i - 1] = wi;
                    }
                    // the row kernel (F:1166-1296): interchange (every row), pulled column,
                    // left transforms (rows below k+1), right transforms (rows below k0)
                    if (p != k + 1) {
                        if (i == k + 1)
                            for (int j = k0; j <= kb + 1; ++j) if (j != k) M1(A, n, k + 1, j) = T.RP[j - k0];
                        if (i == p)
                            for (int j = k0; j <= kb + 1; ++j) if (j != k) M1(A, n, p, j) = T.R1[j - k0];
                        if (p <= kb + 1) {
                            float x = M1(A, n, i, k + 1);
                            M1(A, n, i, k + 1) = M1(A, n, i, p);
                            M1(A, n, i, p) = x;
                            x = M1(B0, n, i, k + 1 - k0);
                            M1(B0, n, i, k + 1 - k0) = M1(B0, n, i, p - k0);
                            M1(B0, n, i, p - k0) = x;
                        } else {
                            const float x = M1(A, n, i, p);
                            M1(A, n, i, p) = M1(B0, n, i, k + 1 - k0);
                            M1(B0, n, i, k + 1 - k0) = x;
                            M1(A, n, i, k + 1) = x;
                        }
                    }
                    if (T.pulled) {
                        for (int r = 0; r < T.nov; ++r)
                            if (T.OR[r] == i) M1(A, n, i, k + 1) = T.OV[r];
                        if (i >= k + 2)
                            for (int kk = k0; kk <= k - 1; ++kk) {
                                const float x = T.CX[kk - k0];
                                if (x != 0.0f) M1(A, n, i, k + 1) = dsub(M1(A, n, i, k + 1), dmul(M1(A, n, i, kk), x));
                            }
                    }
                    if (i >= k + 2)
                        for (int j = k + 1; j <= kb + 1; ++j) {
                            const float pj = T.PJ[j - k - 1];
                            if (pj != 0.0f) M1(A, n, i, j) = dsub(M1(A, n, i, j), dmul(M1(A, n, i, k), pj));
                        }
                    if (i >= k0 + 1)
                        for (int j = k + 2; j <= kb + 1; ++j) {
                            const float vj = M1(A, n, j, k);
                            if (vj != 0.0f) M1(A, n, i, k + 1) = dadd(M1(A, n, i, k + 1), dmul(vj, M1(A, n, i, j)));
                        }
                }
                if (!gb.sync()) return false;
                if (trailing) {
                    // the correction of w by the panel's interchanges and left transforms, on
                    // rows k0+1..k+1 and the swap partners beyond (every CTA, thread 0)
                    if (t == 0) {
                        for (int r = k0 + 1; r <= k + 1; ++r) C.LW[r - k0 - 1] = w[r - 1];
                        int nq = 0;
                        for (int kk = k0; kk <= k; ++kk) {
                            const int q = kk == k ? p : (int)a.ipiv[kk - 1];
                            if (q == kk + 1) continue;
                            if (q <= k + 1) {
                                const float x = C.LW[kk - k0];
                                C.LW[kk - k0] = C.LW[q - k0 - 1];
                                C.LW[q - k0 - 1] = x;
                            } else {
                                int sl = -1;
                                for (int r = 0; r < nq; ++r)
                                    if (C.LR[r] == q) { sl = r; break; }
                                if (sl < 0) { sl = nq++; C.LQ[sl] = w[q - 1]; C.LR[sl] = q; }
                                const float x = C.LW[kk - k0];
                                C.LW[kk - k0] = C.LQ[sl];
                                C.LQ[sl] = x;
                            }
                        }
                        C.nq = nq;
                        for (int kk = k0; kk <= k; ++kk) {
                            const float x = C.LW[kk - k0];
                            C.XS[kk - k0] = x;
                            if (x == 0.0f) continue;
                            for (int r = kk + 2; r <= k; ++r) C.LW[r - k0 - 1] = dsub(C.LW[r - k0 - 1], dmul(M1(A, n, r, kk), x));
                            if (kk + 2 <= k + 1) C.LW[k - k0] = dsub(C.LW[k - k0], dmul(T.RP[kk - k0], x));
                        }
                    }
                    __syncthreads();
                    if (i >= k0 + 1 && i <= n) {
                        if (i <= k + 1) {
                            M1(A, n, i, k + 1) = dadd(M1(A, n, i, k + 1), C.LW[i - k0 - 1]);
                        } else {
                            for (int r = 0; r < C.nq; ++r)
                                if (C.LR[r] == i) wi = C.LQ[r];
                            for (int kk = k0; kk <= k; ++kk) {
                                const float x = C.XS[kk - k0];
                                if (x != 0.0f) wi = dsub(wi, dmul(M1(A, n, i, kk), x));
                            }
                            M1(A, n, i, k + 1) = dadd(M1(A, n, i, k + 1), wi);
                        }
                    }
                    __syncthreads();  // C is rewritten next step
                }
            }
            // the next step's candidates: column k+1, rows k+2..n
            double v = 0.0;
            int vi = 0;
            if (i >= k + 2 && i <= n) { v = fabs((double)M1(A, n, i, k + 1)); vi = i; }
            publish_candidate(a, v, vi, s_red, s_redi);
            if (!gb.sync()) return false;
        }
        const int nbp = kb - k0 + 1;
        if (kb + 2 <= n) {
            // P = M^-1 - I, M[r,s] = A[k0+r, k0+s-1] for r > s (F:1944-1955), in every CTA
            if (t == 0)
                for (int q = 1; q <= nbp; ++q) {
                    for (int r = 1; r <= q; ++r) Pm[r - 1][q - 1] = 0.0f;
                    for (int r = q + 1; r <= nbp; ++r) {
                        float acc = -M1(A, n, k0 + r, k0 + q - 1);
                        for (int s2 = q + 1; s2 <= r - 1; ++s2) acc = dsub(acc, dmul(M1(A, n, k0 + r, k0 + s2 - 1), Pm[s2 - 1][q - 1]));
                        Pm[r - 1][q - 1] = acc;
                    }
                }
            __syncthreads();
            for (int c = kb + 2 + (int)blockIdx.x; c <= n; c += gridDim.x) {
                if (t == 0) {
                    for (int k = k0; k <= kb; ++k) {
                        const int q = (int)a.ipiv[k - 1];
                        if (q != k + 1) {
                            const float x = M1(A, n, k + 1, c);
                            M1(A, n, k + 1, c) = M1(A, n, q, c);
                            M1(A, n, q, c) = x;
                        }
                    }
                    if (nbp >= 2) {
                        for (int s2 = 1; s2 <= nbp; ++s2) Bs[s2 - 1] = M1(A, n, k0 + s2, c);
                        for (int r = 1; r <= nbp; ++r) {
                            float v = M1(A, n, k0 + r, c);
                            for (int s2 = 1; s2 <= nbp; ++s2) v = dfma(Pm[r - 1][s2 - 1], Bs[s2 - 1], v);
                            M1(A, n, k0 + r, c) = v;
                        }
                    }
                }
                __syncthreads();
                for (int r = kb + 2 + t; r <= n; r += RT) {
                    float v = M1(A, n, r, c);
                    for (int kk = 1; kk <= nbp; ++kk) v = dfma(-M1(A, n, r, k0 + kk - 1), M1(A, n, k0 + kk, c), v);
                    M1(A, n, r, c) = v;
                }
                __syncthreads();
            }
        }
        // the top rows' snapshot of the panel columns (rows 1..k0)
        for (size_t e = gt; e < (size_t)k0 * nbp; e += gsz) {
            const int r = (int)(e % k0) + 1, c = k0 + 1 + (int)(e / k0);
            pre[(size_t)(c - k0 - 1) * k0 + r - 1] = M1(A, n, r, c);
        }
        if (!gb.sync()) return false;
        // top rows: panel part, then one fma chain over the trailing columns (F:1635-1672)
        for (size_t e = gt; e < (size_t)k0 * nbp; e += gsz) {
            const int r = (int)(e % k0) + 1, c = k0 + 1 + (int)(e / k0);
            float v = M1(A, n, r, c);
            for (int j = c + 1; j <= kb + 1; ++j) {
                const float vj = M1(A, n, j, c - 1);
                if (vj != 0.0f) v = dadd(v, dmul(vj, pre[(size_t)(j - k0 - 1) * k0 + r - 1]));
            }
            for (int j = kb + 2; j <= n; ++j) v = dfma(M1(A, n, r, j), M1(A, n, j, c - 1), v);
            M1(A, n, r, c) = v;
        }
        if (!gb.sync()) return false;
    }
    // the interchanges deferred on the multipliers (F:1383-1393)
    for (int c = 1 + gt; c <= n - 2; c += gsz) {
        const int kbc = ((c - 1) / FB + 1) * FB < n - 2 ? ((c - 1) / FB + 1) * FB : n - 2;
        for (int k = kbc + 1; k <= n - 2; ++k) {
            const int q = (int)a.ipiv[k - 1];
            if (q != k + 1) {
                const float x = M1(A, n, k + 1, c);
                M1(A, n, k + 1, c) = M1(A, n, q, c);
                M1(A, n, q, c) = x;
            }
        }
    }
    return true;
}

__global__ void __launch_bounds__(RT, 1) reduce_f32_blocked_kernel(RedArgs a, int balance, float* A32, float* B0,
                                                                    float* w, float* pre)
{
    GridBarrier gb{a.bar, a.err, a.limit_ns, 0, nullptr};
    const int n = a.n;
    const int gt = blockIdx.x * RT + threadIdx.x;
    for (size_t e = gt; e < (size_t)n * n; e += (size_t)gridDim.x * RT) A32[e] = (float)a.A[e];
    if (!gb.sync()) return;
    if (balance && !balance_phase_f32(a, A32, gb)) return;
    if (!f32_blocked(a, gb, A32, B0, w, pre)) return;
    if (!gb.sync()) return;
    for (size_t e = gt; e < (size_t)n * n; e += (size_t)gridDim.x * RT) a.A[e] = (double)A32[e];  // widened
}

// One cooperative launch: J (float values in a.A) into A32, balancing, the unblocked
// reduction over the float buffers A32 / B32 (assembled into a.A by unblocked_assemble_kernel).
__global__ void __launch_bounds__(RT, 1) reduce_f32_kernel(RedArgs a, int balance, float* A32, float* B32)
{
    GridBarrier gb{a.bar, a.err, a.limit_ns, 0, nullptr};
    const int n = a.n;
    const int gt = blockIdx.x * RT + threadIdx.x;
    for (size_t e = gt; e < (size_t)n * n; e += (size_t)gridDim.x * RT) A32[e] = (float)a.A[e];
    if (!gb.sync()) return;
    if (balance && !balance_phase_f32(a, A32, gb)) return;
    unblocked_phase<float>(a, gb, A32, B32);
}

// ---------------------------------------------------------------------------------
// Blocked reduction (the reference's Float64 pointer path), nb = 16.
// ---------------------------------------------------------------------------------
struct PanelSh {
    StepTab tab;                       // this step's table (built by warp 0 of every CTA)
    double LW[NBMAX + 2], XS[NBMAX + 2];
    double VAL[2 * NBMAX + 2];         // values at the special slots (see slot_map)
    double Pm[NBMAX][NBMAX];
    int srow[2 * NBMAX + 2];  // rows touched by the panel's interchanges
    int ssrc[2 * NBMAX + 2];  // source slot of each after all interchanges
    int nsr;
    double red[RW];
    int redi[RW];
    double reds[RW];                   // signed values of the warps' candidates
    double tri[NBMAX + 1][NBMAX + 1];  // A[k0+1+r, k0+c] (r > c): the panel's multipliers, final rows
    int slist[2 * NBMAX + 2];          // swap partners beyond row k+1, first-occurrence order
    int slot[NBMAX + 1];               // step kk's swap partner slot (-1: no interchange)
    int nsl;
    int ipv[NBMAX + 1];                // pivots of the panel's steps so far
};

// sum of the GEMV partials of row i in group order (F:1558-1583); loads issued in batches
__device__ __forceinline__ double partial_sum(const RedArgs& a, int P, int i)
{
    const double* pp = a.part + (i - 1);
    const size_t st = (size_t)a.n;
    double s = pp[0];
    int g = 1;
    for (; g + 15 < P; g += 16) {
        double v[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) v[u] = pp[(size_t)(g + u) * st];
#pragma unroll
        for (int u = 0; u < 16; ++u) s = dadd(s, v[u]);
    }
    for (; g + 3 < P; g += 4) {
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = pp[(size_t)(g + u) * st];
#pragma unroll
        for (int u = 0; u < 4; ++u) s = dadd(s, v[u]);
    }
    for (; g < P; ++g) s = dadd(s, pp[(size_t)g * st]);
    return s;
}

// Every warp reads all CTA candidates and reduces them (first max, F:1038-1051); returns p
// and the signed pivot value A[p, k] published with it.
__device__ __forceinline__ int warp_combine(const RedArgs& a, double& pivs)
{
    const int lane = threadIdx.x & 31;
    double v = 0.0, sv = 0.0;
    int vi = 0;
    for (int c = lane; c < (int)gridDim.x; c += 32) {
        const int ci = ((volatile int*)a.cand_i)[c];
        const double cv = ((volatile double*)a.cand_v)[c];
        const double cs = ((volatile double*)a.cand_s)[c];
        if (ci != 0 && (vi == 0 || cv > v || (cv == v && ci < vi))) { v = cv; vi = ci; sv = cs; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double b = __shfl_xor_sync(0xffffffffu, v, o);
        const int ib = __shfl_xor_sync(0xffffffffu, vi, o);
        const double sb = __shfl_xor_sync(0xffffffffu, sv, o);
        if (ib != 0 && (vi == 0 || b > v || (b == v && ib < vi))) { v = b; vi = ib; sv = sb; }
    }
    // lane 0's result for every lane: with NaN candidates the comparison is no total order, and
    // the butterfly could leave lanes with different winners (and the threads of a CTA with
    // different branches around its barriers); lane 0 computes the same in every warp and CTA
    vi = __shfl_sync(0xffffffffu, vi, 0);
    sv = __shfl_sync(0xffffffffu, sv, 0);
    pivs = sv;
    return vi;
}

// CTA-local first-max candidate (|value|, row, signed value) published to slot blockIdx.x.
__device__ __forceinline__ void publish_cand(const RedArgs& a, double v, int vi, double sv, PanelSh& S)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double b = __shfl_xor_sync(0xffffffffu, v, o);
        const int ib = __shfl_xor_sync(0xffffffffu, vi, o);
        const double sb = __shfl_xor_sync(0xffffffffu, sv, o);
        if (ib != 0 && (vi == 0 || b > v || (b == v && ib < vi))) { v = b; vi = ib; sv = sb; }
    }
    const int t = threadIdx.x;
    if ((t & 31) == 0) {
        S.red[t >> 5] = v;
        S.redi[t >> 5] = vi;
        S.reds[t >> 5] = sv;
    }
    __syncthreads();
    if (t == 0) {
        double bv = 0.0, bs = 0.0;
        int bi = 0;
        for (int w = 0; w < RW; ++w) {
            const int ib = S.redi[w];
            if (ib != 0 && (bi == 0 || S.red[w] > bv || (S.red[w] == bv && ib < bi))) {
                bv = S.red[w];
                bi = ib;
                bs = S.reds[w];
            }
        }
        a.cand_v[blockIdx.x] = bv;
        a.cand_i[blockIdx.x] = bi;
        a.cand_s[blockIdx.x] = bs;
    }
    __syncthreads();
}

// Slot map of step k (one warp).  Slots 0..m-1 are rows k0+1..k+1; slots m.. are the swap
// partners beyond row k+1 of steps k0..k in first-occurrence order.  slot[kk-k0] is the
// slot step kk's row kk+1 exchanges with (-1: no interchange).  Both the pulled column's
// table (F:1104-1124) and the correction's special sums (F:1236-1259) move on these slots.
__device__ __forceinline__ void slot_map(PanelSh& S, int k0, int k, int p)
{
    const int lane = threadIdx.x & 31;
    const int m = k - k0 + 1;
    const bool act = lane < m;
    const int q = act ? ((lane == m - 1) ? p : S.ipv[lane]) : 0;
    const bool partner = act && q > k + 1;
    const unsigned am = __ballot_sync(0xffffffffu, act);
    const unsigned same = __match_any_sync(0xffffffffu, partner ? q : -1 - lane);
    const int first = __ffs(same & am) - 1;                     // first lane with this q
    const bool isfirst = partner && first == lane;
    const unsigned fm = __ballot_sync(0xffffffffu, isfirst);
    const int idx_first = __popc(fm & ((1u << lane) - 1u));   // partner index if first
    const int idx = __shfl_sync(0xffffffffu, idx_first, partner ? first : lane);
    if (isfirst) S.slist[idx_first] = q;
    if (act) S.slot[lane] = (q == k0 + lane + 1) ? -1 : (q <= k + 1 ? q - k0 - 1 : m + idx);
    if (lane == 0) S.nsl = __popc(fm);
    __syncwarp();
}

// Apply the interchanges of steps k0..k to a slot vector (one lane; shared memory only).
__device__ __forceinline__ void slot_swaps(PanelSh& S, double* V, int k0, int k)
{
    for (int kk = 0; kk <= k - k0; ++kk) {
        const int s = S.slot[kk];
        if (s < 0) continue;
        const double t = V[kk];
        V[kk] = V[s];
        V[s] = t;
    }
}

// Phase A step table, warp 0 of every CTA (F:952-980; pulled tables F:1088-1132).
// r1 / vsrc were prefetched before the pivot was known.
__device__ void step_table(const RedArgs& a, PanelSh& S, int k0, int kb, int k, int p, double piv, double r1,
                           double vsrc)
{
    const int n = a.n;
    const double* A = a.A;
    const int lane = threadIdx.x & 31;
    StepTab& T = S.tab;
    const int w = kb + 2 - k0;  // panel columns k0..kb+1
    const int m = k - k0 + 1;
    const int pulled = p > kb + 1;
    slot_map(S, k0, k, p);
    // one batch of loads: row p of the panel, and the pulled column at the slot rows
    const double rp = (lane < w) ? M1(A, n, p, k0 + lane) : 0.0;
    double ov = 0.0;
    if (pulled) {
        if (lane < m) ov = M1(A, n, k0 + 1 + lane, p);
        else if (lane < m + S.nsl) ov = M1(A, n, S.slist[lane - m], p);
    }
    if (lane < w) {
        T.R1[lane] = r1;
        T.RP[lane] = rp;
    }
    {
        const int j = k + 2 + lane;
        const double r1k = __shfl_sync(0xffffffffu, r1, k - k0);  // A[k+1, k], the pre-swap row k+1
        if (j <= kb + 1) T.VJ[j - k0] = ((j == p) ? r1k : vsrc) / piv;
    }
    if (pulled) {
        S.VAL[lane] = ov;
        __syncwarp();
        if (lane == 0) slot_swaps(S, S.VAL, k0, k);
        __syncwarp();
        // catch-up of rows k0+1..k+1 by the left transforms k0..k-1, lanes = rows
        double o = (lane < m) ? S.VAL[lane] : 0.0;
        const int row = k0 + 1 + lane;
        for (int kk = k0; kk <= k - 1; ++kk) {
            const double x = __shfl_sync(0xffffffffu, o, kk - k0);
            if (lane == 0) T.CX[kk - k0] = x;
            if (x != 0.0 && lane < m && row >= kk + 2) {
                const double aik = (row == k + 1) ? T.RP[kk - k0] : S.tri[lane][kk - k0];
                o = dsub(o, dmul(aik, x));
            }
        }
        if (lane < m) S.VAL[lane] = o;
        __syncwarp();
        if (lane < m + S.nsl) T.OV[lane] = S.VAL[lane];
    }
    __syncwarp();
    if (lane == 0) {
        T.p = p;
        T.piv = piv;
        T.pulled = pulled;
        T.skip = 0;
        T.nov = pulled ? m + S.nsl : 0;
        for (int j = k + 1; j <= kb + 1; ++j) T.PJ[j - k - 1] = T.RP[j - k0];
        if (pulled) T.PJ[0] = T.OV[k - k0];
        else if (p != k + 1) {
            T.PJ[0] = T.RP[p - k0];
            T.PJ[p - k - 1] = T.RP[k + 1 - k0];
        }
    }
    // row k+1 is final after this step: its multipliers (pre-swap row p) join the triangle
    if (lane < m - 1) S.tri[m - 1][lane] = T.RP[lane];
    if (lane == 0) S.ipv[m - 1] = p;
    __syncwarp();
}

// GEMV partials of phase A (F:1496-1553): task = (group g, 32-row tile), lane = row.
__device__ void gemv_tasks(const RedArgs& a, int k0, int kb, int k, int p, double piv)
{
    const int n = a.n;
    const double* A = a.A;
    const int c0 = kb + 2;
    const int P = (n - c0 + 1 + GEMV_GROUP - 1) / GEMV_GROUP;
    const int ntiles = (n - k0 + 31) / 32;
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (RW - 1) + (threadIdx.x >> 5) - 1;  // warps 1..RW-1 of every CTA
    const int nw = gridDim.x * (RW - 1);
    const bool pulled = p > kb + 1;
    const double* sub = a.B0 + (size_t)(k - k0) * n;  // pre-panel copy of column k+1
    const int ntask = P * ntiles;
    for (int task = gw; task < ntask; task += nw) {
        const int g = task / ntiles, tile = task % ntiles;
        const int ga = c0 + g * GEMV_GROUP;
        const int gb = min(ga + GEMV_GROUP - 1, n);
        // multipliers of the group's columns: lane m holds columns ga+m and ga+32+m
        double l0 = 0.0, l1 = 0.0;
        {
            const int j0 = ga + lane, j1 = ga + 32 + lane;
            if (j0 <= gb) l0 = ((j0 == p) ? M1(A, n, k + 1, k) : M1(A, n, j0, k)) / piv;
            if (j1 <= gb) l1 = ((j1 == p) ? M1(A, n, k + 1, k) : M1(A, n, j1, k)) / piv;
        }
        const int i = k0 + 1 + tile * 32 + lane;
        const bool act = i <= n;
        const int ii = act ? i : n;
        auto COL = [&](int j) -> const double* { return (pulled && j == p) ? sub : A + (size_t)(j - 1) * n; };
        // the reference's group order: the first four-column pass assigns, later passes add,
        // single tail columns add l*a (skipped when l == 0; a group of <= 3 columns assigns
        // its first); operands are fetched 16 columns at a time
        const int w = gb - ga + 1;
        const int nquad = w >> 2;
        double acc = 0.0;
        bool have = false;
        for (int b0 = 0; b0 < w; b0 += 16) {
            double av[16], lv[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) av[u] = (b0 + u < w) ? COL(ga + b0 + u)[ii - 1] : 0.0;
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int m = b0 + u;
                const double v0 = __shfl_sync(0xffffffffu, l0, m & 31);
                const double v1 = __shfl_sync(0xffffffffu, l1, m & 31);
                lv[u] = m < 32 ? v0 : v1;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (((b0 >> 2) + q) < nquad) {
                    const double quad = dadd(dadd(dmul(lv[4 * q], av[4 * q]), dmul(lv[4 * q + 1], av[4 * q + 1])),
                                             dadd(dmul(lv[4 * q + 2], av[4 * q + 2]), dmul(lv[4 * q + 3], av[4 * q + 3])));
                    acc = have ? dadd(acc, quad) : quad;
                    have = true;
                }
            }
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int off = b0 + u;
                if (off >= 4 * nquad && off < w) {
                    if (!have) {
                        acc = dmul(lv[u], av[u]);
                        have = true;
                    } else if (lv[u] != 0.0) {
                        acc = dadd(acc, dmul(lv[u], av[u]));
                    }
                }
            }
        }
        if (act) a.part[(size_t)g * n + (i - 1)] = acc;
    }
}

// GEMV partials of phase A through TMA: the trailing block is streamed in 64x64 FP64
// tiles (64 rows x one 64-column group), T64_SLOTS tiles in flight per CTA, completion on
// one mbarrier per slot.  Two warps consume a tile (32 rows each); the arithmetic per row
// is the reference's group order (F:1496-1553), read from shared memory.  The pulled
// column (p > kb+1) is taken from its pre-panel copy in B0, as the reference reads it
// from pSub (F:1492).  Warp 0 only joins the per-round CTA barriers.
__device__ void gemv_tma64(const RedArgs& a, const void* tmA, uint64_t* bars, double* tiles, int k0, int kb, int k,
                         int p, double piv, uint32_t& ph)
{
    const int n = a.n;
    const double* A = a.A;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int P = (n - kb - 1 + GEMV_GROUP - 1) / GEMV_GROUP;
    const int r0t = k0 / 64;  // first 64-row tile holding 0-based row k0 (= row k0+1)
    const int RTn = (n + 63) / 64 - r0t;
    const int ntask = RTn * P;
    const int G = gridDim.x, bid = blockIdx.x;
    const int cnt = (ntask > bid) ? (ntask - bid - 1) / G + 1 : 0;
    const bool pulled = p > kb + 1;
    const double* sub = a.B0 + (size_t)(k - k0) * n;
    for (int base = 0; base < cnt; base += T64_SLOTS) {
        const int nr = min(T64_SLOTS, cnt - base);
        if (threadIdx.x == 32) {
            fence_proxy_async_global();
            fence_proxy_async_shared();
            for (int s = 0; s < nr; ++s) {
                const int t = bid + (base + s) * G;
                const int g = t / RTn, rt = r0t + t % RTn;
                mbar_expect_tx(&bars[s], TILE64_BYTES);
                tma_load_2d(tiles + (size_t)s * 4096, tmA, rt * 64, kb + 1 + 64 * g, &bars[s]);
            }
        }
        if (warp >= 1) {
            for (int u = warp - 1; u < 2 * nr; u += RW - 1) {
                const int s = u >> 1, half = u & 1;
                const int t = bid + (base + s) * G;
                const int g = t / RTn, rt = r0t + t % RTn;
                const int ga = kb + 2 + 64 * g;
                const int gb = min(ga + 63, n);
                const int w = gb - ga + 1;
                double l0 = 0.0, l1 = 0.0;
                {
                    const int j0 = ga + lane, j1 = ga + 32 + lane;
                    if (j0 <= gb) l0 = ((j0 == p) ? M1(A, n, k + 1, k) : M1(A, n, j0, k)) / piv;
                    if (j1 <= gb) l1 = ((j1 == p) ? M1(A, n, k + 1, k) : M1(A, n, j1, k)) / piv;
                }
                const int r = half * 32 + lane;       // row within the tile
                const int i = rt * 64 + r + 1;         // 1-based row
                const bool act = i >= k0 + 1 && i <= n;
                const bool psub = pulled && p >= ga && p <= gb;
                const double bval = (psub && act) ? sub[i - 1] : 0.0;
                if (!mbar_wait_ns(&bars[s], (ph >> s) & 1u, tma_wait_ns(a))) atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
                const double* tl = tiles + (size_t)s * 4096 + r;
                auto TV = [&](int j) -> double { return (psub && j == p) ? bval : tl[(j - ga) * 64]; };
                auto LV = [&](int j) -> double {
                    const int m = j - ga;
                    const double v0 = __shfl_sync(0xffffffffu, l0, m & 31);
                    const double v1 = __shfl_sync(0xffffffffu, l1, m & 31);
                    return m < 32 ? v0 : v1;
                };
                const int nquad = w >> 2;
                double acc = 0.0;
                bool have = false;
                for (int q = 0; q < nquad; ++q) {
                    const int j = ga + 4 * q;
                    const double q1 = LV(j), q2 = LV(j + 1), q3 = LV(j + 2), q4 = LV(j + 3);
                    const double quad = dadd(dadd(dmul(q1, TV(j)), dmul(q2, TV(j + 1))),
                                             dadd(dmul(q3, TV(j + 2)), dmul(q4, TV(j + 3))));
                    acc = have ? dadd(acc, quad) : quad;
                    have = true;
                }
                for (int j = ga + 4 * nquad; j <= gb; ++j) {
                    const double lj = LV(j);
                    if (!have) {
                        acc = dmul(lj, TV(j));
                        have = true;
                    } else if (lj != 0.0) {
                        acc = dadd(acc, dmul(lj, TV(j)));
                    }
                }
                if (act) a.part[(size_t)g * n + (i - 1)] = acc;
            }
        }
        __syncthreads();
        ph ^= (1u << nr) - 1u;
    }
}

// The correction triangle of phase B, warp 0 of every CTA with rows to finish (F:1232-1269):
// the GEMV sums at the special slots, the interchanges of steps k0..k on them, then the
// x's: LW (rows k0+1..k+1), VAL[m..] (the partners' values), XS.
__device__ void correction_triangle(const RedArgs& a, PanelSh& S, int k0, int k, int P)
{
    const int lane = threadIdx.x & 31;
    const int m = k - k0 + 1;
    const int ns = m + S.nsl;
    for (int idx = lane; idx < ns; idx += 32) {
        const int row = (idx < m) ? k0 + 1 + idx : S.slist[idx - m];
        S.VAL[idx] = partial_sum(a, P, row);
    }
    __syncwarp();
    if (lane == 0) slot_swaps(S, S.VAL, k0, k);
    __syncwarp();
    // x triangle: lanes hold rows k0+1+lane, sequential over kk
    double lw = (lane < m) ? S.VAL[lane] : 0.0;
    const int row = k0 + 1 + lane;
    for (int kk = k0; kk <= k; ++kk) {
        const double x = __shfl_sync(0xffffffffu, lw, kk - k0);
        if (lane == 0) S.XS[kk - k0] = x;
        if (x != 0.0 && lane < m) {
            if (row >= kk + 2 && row <= k) lw = dsub(lw, dmul(S.tri[lane][kk - k0], x));
            else if (row == k + 1 && kk + 2 <= k + 1) lw = dsub(lw, dmul(S.tab.RP[kk - k0], x));
        }
    }
    if (lane < m) S.LW[lane] = lw;
    __syncwarp();
}

// Phase B row work for row i in k0+1..n (F:1166-1296); returns |A[i,k+1]| candidate.
template <int NB>
__device__ void panel_row(const RedArgs& a, const PanelSh& S, int k0, int kb, int k, int P, int i, double wsum,
                          double& cand, int& candi, double& cands)
{
    // The row's panel values stay in registers: every access to v[] below has a compile-time
    // index; the columns at run-time positions (k, k+1, p) are selected by predicates.
    const int n = a.n;
    double* A = a.A;
    const StepTab& T = S.tab;
    const int p = T.p;
    const int w = kb + 1 - k0 + 1;  // columns k0..kb+1
    double v[NB + 2];
#pragma unroll
    for (int c = 0; c < NB + 2; ++c) v[c] = (c < w) ? M1(A, n, i, k0 + c) : 0.0;
    const int ck = k - k0, ck1 = k + 1 - k0;
    auto GET = [&](int idx) -> double {
        double r = 0.0;
#pragma unroll
        for (int c = 0; c < NB + 2; ++c)
            if (c == idx) r = v[c];
        return r;
    };
    double x1 = GET(ck1);  // column k+1
    if (T.skip) {
        if (i >= k + 2) { cand = fabs(x1); candi = i; cands = x1; }
        return;
    }
    const double piv = T.piv;
    // (1) interchange: rows k+1 <-> p on the panel columns, then columns k+1 <-> p
    if (p != k + 1) {
        if (i == k + 1) {
#pragma unroll
            for (int c = 0; c < NB + 2; ++c) if (c < w) v[c] = T.RP[c];
        } else if (i == p) {
#pragma unroll
            for (int c = 0; c < NB + 2; ++c) if (c < w) v[c] = T.R1[c];
        }
        x1 = GET(ck1);
        if (p <= kb + 1) {
            const int cp = p - k0;
            const double t = x1;
            x1 = GET(cp);
#pragma unroll
            for (int c = 0; c < NB + 2; ++c)
                if (c == cp) v[c] = t;
            double* b1 = a.B0 + (size_t)(k - k0) * n + (i - 1);
            double* bp = a.B0 + (size_t)(p - k0 - 1) * n + (i - 1);
            const double tb = *b1;
            *b1 = *bp;
            *bp = tb;
        } else {
            double* ap = A + (size_t)(p - 1) * n + (i - 1);
            double* b1 = a.B0 + (size_t)(k - k0) * n + (i - 1);
            const double t = *ap;
            *ap = *b1;
            *b1 = t;
            x1 = t;
        }
    }
    // (2) the pulled column's tables and catch-up (F:1193-1205)
    if (T.pulled) {
        int sl = -1;
        if (i >= k0 + 1 && i <= k + 1) sl = i - k0 - 1;
        else
            for (int r = 0; r < S.nsl; ++r)
                if (S.slist[r] == i) sl = k - k0 + 1 + r;
        if (sl >= 0) x1 = T.OV[sl];
        if (i >= k + 2) {
#pragma unroll
            for (int c = 0; c < NB; ++c) {
                if (c < ck) {
                    const double x = T.CX[c];
                    if (x != 0.0) x1 = dsub(x1, dmul(v[c], x));
                }
            }
        }
    }
    // scale the multiplier (F:968-970, F:1503-1505)
    double xk = GET(ck);
    if (i >= k + 2) xk = xk / piv;
    // (3) left update of the panel columns (F:1206-1213)
    if (i >= k + 2) {
#pragma unroll
        for (int c = 1; c < NB + 2; ++c) {
            if (c >= ck1 && c < w) {
                const double pj = T.PJ[c - ck1];
                if (pj != 0.0) {
                    if (c == ck1) x1 = dsub(x1, dmul(xk, pj));
                    else v[c] = dsub(v[c], dmul(xk, pj));
                }
            }
        }
    }
    // (4) right update from the panel columns (F:1214-1221)
#pragma unroll
    for (int c = 2; c < NB + 2; ++c) {
        if (c >= ck1 + 1 && c < w) {
            const double vj = T.VJ[c];
            if (vj != 0.0) x1 = dadd(x1, dmul(vj, v[c]));
        }
    }
    // (5) the GEMV part with its correction (F:1222-1293)
    if (i <= k + 1) {
        x1 = dadd(x1, S.LW[i - k0 - 1]);
    } else {
        int r = -1;
        for (int q = 0; q < S.nsl; ++q)
            if (S.slist[q] == i) r = q;
        double wv = (r >= 0) ? S.VAL[k - k0 + 1 + r] : wsum;
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            if (c <= ck) {
                const double x = S.XS[c];
                if (x != 0.0) wv = dsub(wv, dmul(c == ck ? xk : v[c], x));
            }
        }
        x1 = dadd(x1, wv);
        cand = fabs(x1);
        candi = i;
        cands = x1;
    }
    const bool swapped_row = p != k + 1 && (i == k + 1 || i == p);
#pragma unroll
    for (int c = 0; c < NB + 2; ++c) {
        if (c < w && (c >= ck || swapped_row)) {
            const double val = (c == ck) ? xk : ((c == ck1) ? x1 : v[c]);
            M1(A, n, i, k0 + c) = val;
        }
    }
}

// Panel-end interchange map: rows touched by steps k0..kb and, for each, the row whose
// pre-sweep value it receives after the whole sequence (F:1344-1379, F:1395-1415).
__device__ void build_swap_map(const RedArgs& a, PanelSh& S, int k0, int kb)
{
    // warp 0 replays the panel's interchanges on the list of rows they touch: entry q (in
    // order of first appearance) lives in lane q % 32, slot q / 32, as (row, row whose value
    // it ends with); a lookup is one ballot per slot
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int row0 = 0, row1 = 0, val0 = 0, val1 = 0;
        int nsr = 0;
        auto find = [&](int r) -> int {
            const unsigned m0 = __ballot_sync(0xffffffffu, lane < nsr && row0 == r);
            const unsigned m1 = __ballot_sync(0xffffffffu, lane + 32 < nsr && row1 == r);
            if (m0) return __ffs(m0) - 1;
            if (m1) return 32 + __ffs(m1) - 1;
            const int q = nsr++;
            if (q < 32) {
                if (lane == q) { row0 = r; val0 = r; }
            } else if (lane == q - 32) {
                row1 = r;
                val1 = r;
            }
            return q;
        };
        for (int k = k0; k <= kb; ++k) {
            const int p = S.ipv[k - k0];
            if (p <= k + 1 || p > a.n) continue;
            const int s1 = find(k + 1), s2 = find(p);
            const int v1 = __shfl_sync(0xffffffffu, s1 < 32 ? val0 : val1, s1 & 31);
            const int v2 = __shfl_sync(0xffffffffu, s2 < 32 ? val0 : val1, s2 & 31);
            if (lane == (s1 & 31)) {
                if (s1 < 32) val0 = v2;
                else val1 = v2;
            }
            if (lane == (s2 & 31)) {
                if (s2 < 32) val0 = v1;
                else val1 = v1;
            }
        }
        if (lane < nsr) {
            S.srow[lane] = row0;
            S.ssrc[lane] = val0;
        }
        if (lane + 32 < nsr) {
            S.srow[lane + 32] = row1;
            S.ssrc[lane + 32] = val1;
        }
        if (lane == 0) S.nsr = nsr;
    }
    __syncthreads();
}

// P = M^-1 - I of the panel's multipliers (F:1944-1955), into shared memory.
__device__ void build_trsm_inverse(const RedArgs& a, PanelSh& S, int k0, int kb)
{
    const int nbp = kb - k0 + 1;   // S.tri[r-1][s-1] = M[r,s] = A[k0+r, k0+s-1], r > s
    const int q = threadIdx.x + 1;  // column q of P, kept in registers while it is built
    if (threadIdx.x < nbp) {
        double pc[NBMAX];
#pragma unroll
        for (int r = 1; r <= NBMAX; ++r) {
            double acc = 0.0;
            if (r <= nbp && r > q) {
                acc = -S.tri[r - 1][q - 1];
#pragma unroll
                for (int s = 2; s <= NBMAX - 1; ++s)
                    if (s >= q + 1 && s <= r - 1) acc = dsub(acc, dmul(S.tri[r - 1][s - 1], pc[s - 1]));
            }
            pc[r - 1] = acc;
            if (r <= nbp) S.Pm[r - 1][q - 1] = acc;
        }
    }
    __syncthreads();
}

// Apply the panel's interchanges to column c (rows in the swap map); for a trailing
// column also the TRSM on rows k0+1..kb+1 (F:1933-2001).
__device__ void column_end(const RedArgs& a, const PanelSh& S, int k0, int kb, int c, bool trsm)
{
    const int n = a.n;
    double* col = a.A + (size_t)(c - 1) * n;
    const int nsr = S.nsr;
    double old[2 * NBMAX + 2];
#pragma unroll
    for (int q = 0; q < 2 * NBMAX + 2; ++q)
        if (q < nsr) old[q] = col[S.ssrc[q] - 1];
#pragma unroll
    for (int q = 0; q < 2 * NBMAX + 2; ++q)
        if (q < nsr) col[S.srow[q] - 1] = old[q];
    if (!trsm) return;
    const int nbp = kb - k0 + 1;
    if (nbp < 2) return;
    double B[NBMAX];
#pragma unroll
    for (int s = 0; s < NBMAX; ++s) B[s] = (s < nbp) ? col[k0 + s] : 0.0;
#pragma unroll
    for (int r = 0; r < NBMAX; ++r) {
        if (r < nbp) {
            double v = B[r];
#pragma unroll
            for (int s = 0; s < NBMAX; ++s)
                if (s < nbp) v = dfma(S.Pm[r][s], B[s], v);
            col[k0 + r] = v;
        }
    }
}

template <int NB>
__device__ bool blocked_phase(const RedArgs& a, GridBarrier& gb, PanelSh& S, uint64_t& last, const void* tmA,
                              const void* tmP, uint64_t* bars, double* tiles)
{
    uint32_t ph = 0;  // per-slot mbarrier phase parity (identical in every thread)
    const int n = a.n;
    const int nb = NB;
    double* A = a.A;
    const int gt = blockIdx.x * RT + threadIdx.x;
    const int gsz = gridDim.x * RT;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    // setup: candidates of column 1, B0 of the first panel
    {
        double v = 0.0, sv = 0.0;
        int vi = 0;
        for (int i = 2 + gt; i <= n; i += gsz) {
            const double x = M1(A, n, i, 1);
            if (vi == 0 || fabs(x) > v) { v = fabs(x); vi = i; sv = x; }
        }
        publish_cand(a, v, vi, sv, S);
        const int kb = min(nb, n - 2);
        for (size_t e = gt; e < (size_t)n * (kb + 1 - 1); e += gsz) {
            const int i = (int)(e % n), c = (int)(e / n);
            a.B0[(size_t)c * n + i] = A[(size_t)(c + 1) * n + i];
        }
    }
    if (!gb.sync()) return false;

    for (int k0 = 1; k0 <= n - 2; k0 += nb) {
        const int kb = min(k0 + nb - 1, n - 2);
        const int P = (n - kb - 1 + GEMV_GROUP - 1) / GEMV_GROUP;
        for (int k = k0; k <= kb; ++k) {
            // ---- phase A: pivot (every warp), step table (warp 0 of every CTA), GEMV ----
            uint64_t pa = globaltimer_ns();
            double r1 = 0.0, vsrc = 0.0;
            if (warp == 0) {  // prefetch what the table needs before the pivot is known
                if (lane < kb + 2 - k0) r1 = M1(A, n, k + 1, k0 + lane);
                if (k + 2 + lane <= kb + 1) vsrc = M1(A, n, k + 2 + lane, k);
            }
            double piv = 0.0;
            int p = warp_combine(a, piv);
            if (p < k + 1 || p > n) {  // no candidate (a zero column): no interchange
                p = k + 1;
                piv = M1(A, n, k + 1, k);
            }
            tprobe(a, 0, 5, pa);
            if (warp == 0) {
                if (blockIdx.x == 0 && lane == 0) a.ipiv[k - 1] = p;
                if (piv != 0.0) {
                    step_table(a, S, k0, kb, k, p, piv, r1, vsrc);
                } else {
                    if (lane == 0) {
                        S.tab.skip = 1;
                        S.tab.p = p;
                        S.tab.piv = piv;
                        S.tab.pulled = 0;
                        S.tab.nov = 0;
                        S.ipv[k - k0] = p;
                    }
                    if (lane < k - k0) S.tri[k - k0][lane] = r1;  // p == k+1: row k+1 is final as is
                    __syncwarp();
                }
                tprobe(a, 0, 6, pa);
            } else if (!a.use_tma) {
                uint64_t pg = globaltimer_ns();
                if (piv != 0.0) gemv_tasks(a, k0, kb, k, p, piv);
                tprobe(a, 1, 7, pg);
            }
            if (a.use_tma && piv != 0.0) {
                uint64_t pg = globaltimer_ns();
                gemv_tma64(a, tmA, bars, tiles, k0, kb, k, p, piv, ph);
                tprobe(a, 1, 7, pg);
            }
            if (!gb.sync()) return false;
            tprobe(a, 0, 8, pa);
            tmark(a, 1, last);
            // ---- phase B: rows ----
            uint64_t pb = globaltimer_ns();
            const bool skip = S.tab.skip != 0;
            const int i = 1 + gt;  // this thread's row
            const bool cta_rows = (blockIdx.x + 1) * RT >= k0 + 1 && blockIdx.x * RT + 1 <= n;
            tprobe(a, (n - 1) / RT, 0, pb);
            double wsum = 0.0;
            if (a.use_tma && !skip && cta_rows && threadIdx.x == 32) {
                // this CTA's rows of the GEMV partials, PBOX_G groups per box
                fence_proxy_async_global();
                fence_proxy_async_shared();
                for (int s = 0; s < PBOX_SLOTS && s * PBOX_G < P; ++s) {
                    mbar_expect_tx(&bars[s], PBOX_BYTES);
                    tma_load_2d(tiles + (size_t)s * RT * PBOX_G, tmP, blockIdx.x * RT, s * PBOX_G, &bars[s]);
                }
            }
            if (warp == 0 && !skip && cta_rows) correction_triangle(a, S, k0, k, P);
            if (!skip && i >= k + 2 && i <= n) {
                if (a.use_tma) {
                    // sum from the staged partials, in group order; boxes beyond PBOX_SLOTS
                    // (n > 4096) are read from global memory
                    double sacc = 0.0;
                    const int r = threadIdx.x;
                    for (int s = 0; s < PBOX_SLOTS && s * PBOX_G < P; ++s) {
                        if (!mbar_wait_ns(&bars[s], (ph >> s) & 1u, tma_wait_ns(a))) atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
                        const double* pb = tiles + (size_t)s * RT * PBOX_G;
                        const int gend = min(P - s * PBOX_G, PBOX_G);
                        for (int gg = 0; gg < gend; ++gg) {
                            const double x = pb[gg * RT + r];
                            sacc = (s == 0 && gg == 0) ? x : dadd(sacc, x);
                        }
                    }
                    for (int g = PBOX_SLOTS * PBOX_G; g < P; ++g) sacc = dadd(sacc, a.part[(size_t)g * n + (i - 1)]);
                    wsum = sacc;
                } else {
                    wsum = partial_sum(a, P, i);
                }
            }
            __syncthreads();
            if (a.use_tma && !skip && cta_rows) {
                const int ns = min(PBOX_SLOTS, (P + PBOX_G - 1) / PBOX_G);
                ph ^= (1u << ns) - 1u;
            }
            tprobe(a, (n - 1) / RT, 1, pb);
            double cand = 0.0, cands = 0.0;
            int candi = 0;
            if (i >= k0 + 1 && i <= n) {
                panel_row<NB>(a, S, k0, kb, k, P, i, wsum, cand, candi, cands);
            } else if (i <= k0 && !skip && p != k + 1) {
                // top rows: the column part of the interchange (F:1135-1161)
                if (p <= kb + 1) {
                    double* x1 = A + (size_t)k * n + (i - 1);
                    double* xp = A + (size_t)(p - 1) * n + (i - 1);
                    double t = *x1; *x1 = *xp; *xp = t;
                    double* b1 = a.B0 + (size_t)(k - k0) * n + (i - 1);
                    double* bp = a.B0 + (size_t)(p - k0 - 1) * n + (i - 1);
                    t = *b1; *b1 = *bp; *bp = t;
                } else {
                    double* ap = A + (size_t)(p - 1) * n + (i - 1);
                    double* b1 = a.B0 + (size_t)(k - k0) * n + (i - 1);
                    const double t = *ap;
                    *ap = *b1;
                    *b1 = t;
                    A[(size_t)k * n + (i - 1)] = t;
                }
            }
            tprobe(a, (n - 1) / RT, 2, pb);
            publish_cand(a, cand, candi, cands, S);
            tprobe(a, (n - 1) / RT, 3, pb);
            if (!gb.sync()) return false;
            tprobe(a, (n - 1) / RT, 4, pb);
            tmark(a, 2, last);
        }
        // ---- panel end E1: interchange map, TRSM inverse, column sweeps ----
        build_swap_map(a, S, k0, kb);
        build_trsm_inverse(a, S, k0, kb);
        // columns spread over every CTA (column c on CTA c mod grid) for memory parallelism
        for (int c = 1 + (int)blockIdx.x + (int)gridDim.x * (int)threadIdx.x; c <= n; c += gsz) {
            if (c >= kb + 2) column_end(a, S, k0, kb, c, true);
            else if (c < k0) column_end(a, S, k0, kb, c, false);
        }
        {
            const int nbp = kb - k0 + 1;
            for (size_t e = gt; e < (size_t)k0 * nbp; e += gsz) {
                const int i = (int)(e % k0), c = (int)(e / k0);
                a.tsnap[(size_t)c * n + i] = A[(size_t)(k0 + c) * n + i];
            }
        }
        if (!gb.sync()) return false;
        tmark(a, 3, last);
        // ---- panel end E2: trailing GEMM, top GEMM, next panel's B0 ----
        {
            const int nbp = kb - k0 + 1;
            const int k0n = kb + 1;
            const int kbn = min(k0n + nb - 1, n - 2);
            const bool more = k0n <= n - 2;
            const int m = n - kb - 1;                    // trailing size
            const int tiles = (m + 31) / 32;
            const int ntr = tiles * tiles;               // 32x32 trailing tiles
            const int ntop = ((k0 + 31) / 32) * ((nbp + 3) / 4);
            const int gw = blockIdx.x * RW + warp, nw = gridDim.x * RW;
            for (int task = gw; task < ntr + ntop; task += nw) {
                if (task < ntr) {
                    const int ti = task % tiles, tj = task / tiles;
                    const int i = kb + 2 + ti * 32 + lane;
                    const bool act = i <= n;
                    double Lr[NBMAX];
#pragma unroll
                    for (int s = 0; s < NBMAX; ++s) Lr[s] = (act && s < nbp) ? -M1(A, n, i, k0 + s) : 0.0;
                    const int cend = min(kb + 2 + tj * 32 + 31, n);
                    // 16 columns per round: their U rows (lane s holds U[s]) and this lane's
                    // elements are all requested before the first chain starts
                    for (int cb = kb + 2 + tj * 32; cb <= cend; cb += 16) {
                        const int ncol = min(16, cend - cb + 1);
                        double uc[16], vc[16];
#pragma unroll
                        for (int u = 0; u < 16; ++u) {
                            const int c = cb + u;
                            uc[u] = (u < ncol && lane < nbp) ? A[(size_t)(c - 1) * n + k0 + lane] : 0.0;  // rows k0+1..kb+1
                            vc[u] = (u < ncol && act) ? M1(A, n, i, c) : 0.0;
                        }
#pragma unroll
                        for (int u = 0; u < 16; ++u) {
                            if (u < ncol) {
                                const int c = cb + u;
                                double v = vc[u];
#pragma unroll
                                for (int s = 0; s < NBMAX; ++s) {
                                    const double us = __shfl_sync(0xffffffffu, uc[u], s);  // all lanes
                                    if (s < nbp) v = dfma(Lr[s], us, v);
                                }
                                if (act) {
                                    M1(A, n, i, c) = v;
                                    if (more && c >= k0n + 1 && c <= kbn + 1)
                                        a.B0[(size_t)(c - k0n - 1) * n + (i - 1)] = v;
                                }
                            }
                        }
                    }
                } else {
                    // top rows 1..k0 of panel columns c0..c0+3 (F:1635-1672)
                    const int tt = task - ntr;
                    const int rt = tt / ((nbp + 3) / 4), cg = tt % ((nbp + 3) / 4);
                    const int i = 1 + rt * 32 + lane;
                    const bool act = i <= k0;
                    const int ii = act ? i : 1;
                    double pre[NBMAX + 1];
#pragma unroll
                    for (int c = 0; c < NBMAX + 1; ++c) pre[c] = (c < nbp) ? a.tsnap[(size_t)c * n + (ii - 1)] : 0.0;
                    double acc[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int cc = cg * 4 + q;  // column k0+1+cc
                        double v = (cc < nbp) ? pre[cc] : 0.0;
#pragma unroll
                        for (int j = 0; j < NBMAX + 1; ++j) {
                            if (cc < nbp && j > cc && j < nbp) {
                                const double vj = M1(A, n, k0 + 1 + j, k0 + cc);
                                if (vj != 0.0) v = dadd(v, dmul(vj, pre[j]));
                            }
                        }
                        acc[q] = v;
                    }
                    // one fma chain per element over j = kb+2..n, in order, in chunks of 32 j: the
                    // chunk's multipliers A[j, k0+c0q+q] come in one coalesced load per column
                    // (lane u holds row j0+u) and reach every lane by shuffle; each lane issues its
                    // row's 32 loads of the chunk together
                    const int c0q = cg * 4;
                    const int nq = min(4, nbp - c0q);
                    for (int j0 = kb + 2; j0 <= n; j0 += 32) {
                        const int jl = j0 + lane;
                        double lq[4];
#pragma unroll
                        for (int q = 0; q < 4; ++q) lq[q] = (q < nq && jl <= n) ? M1(A, n, jl, k0 + c0q + q) : 0.0;
                        const int cnt = min(32, n - j0 + 1);
                        if (cnt == 32) {
                            double av[32];
#pragma unroll
                            for (int u = 0; u < 32; ++u) av[u] = M1(A, n, ii, j0 + u);
#pragma unroll
                            for (int u = 0; u < 32; ++u)
#pragma unroll
                                for (int q = 0; q < 4; ++q)
                                    acc[q] = dfma(av[u], __shfl_sync(0xffffffffu, lq[q], u), acc[q]);
                        } else {
                            for (int u = 0; u < cnt; ++u) {
                                const double aij = M1(A, n, ii, j0 + u);
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    const double l = __shfl_sync(0xffffffffu, lq[q], u);
                                    if (q < nq) acc[q] = dfma(aij, l, acc[q]);
                                }
                            }
                        }
                    }
                    if (act) {
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const int cc = cg * 4 + q;
                            if (cc < nbp) M1(A, n, i, k0 + 1 + cc) = acc[q];
                        }
                    }
                }
            }
            // next panel's B0, rows 1..kb+1 (rows below come from the GEMM writers)
            if (more) {
                const int wn = kbn + 1 - k0n;  // columns k0n+1..kbn+1
                for (size_t e = gt; e < (size_t)(kb + 1) * wn; e += gsz) {
                    const int i = (int)(e % (kb + 1)), c = (int)(e / (kb + 1));
                    a.B0[(size_t)c * n + i] = A[(size_t)(k0n + c) * n + i];
                }
            }
        }
        if (!gb.sync()) return false;
        tmark(a, 4, last);
    }
    return true;
}

// ---------------------------------------------------------------------------------
// The reduction kernel: mode 0 = balance only, 1 = unblocked, 2 = blocked.  Balancing,
// when requested, runs first in the same launch.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(RT, 1) reduce_kernel(RedArgs a, int balance, int mode,
                                                        const __grid_constant__ CUtensorMap tmA,
                                                        const __grid_constant__ CUtensorMap tmP)
{
    __shared__ PanelSh S;
    __shared__ __align__(8) uint64_t bars[T64_SLOTS];
    extern __shared__ __align__(1024) double tiles[];
    if (threadIdx.x == 0) {
        for (int s = 0; s < T64_SLOTS; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    GridBarrier gb{a.bar, a.err, a.limit_ns, 0, a.ptimes ? a.ptimes + 5 : nullptr};
    uint64_t t0 = globaltimer_ns(), last = t0;
    if (balance) {
        if (!balance_phase(a, gb)) return;
    }
    tmark(a, 0, last);
    if (mode == 1) {
        unblocked_phase<double>(a, gb, a.A, a.buf2);
        tmark(a, 1, last);
    } else if (mode == 2) {
        blocked_phase<NBMAX>(a, gb, S, last, &tmA, &tmP, bars, tiles);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && a.ptimes) a.ptimes[7] += globaltimer_ns() - t0;
}

// Ht[j,i] = A[i,j] for i <= j+1, zero elsewhere (F:2005-2061); 32x32 tiles.
__global__ void ht_fill_kernel(int n, const double* __restrict__ A, double* __restrict__ Ht)
{
    __shared__ double tile[32][33];
    const int bi = blockIdx.y * 32, bj = blockIdx.x * 32;  // tile of A rows bi.., cols bj..
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = bi + threadIdx.x, j = bj + r;
        tile[r][threadIdx.x] = (i < n && j < n) ? A[(size_t)j * n + i] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = bi + r, j = bj + threadIdx.x;  // Ht[j, i] = A[i, j]
        if (i < n && j < n) Ht[(size_t)i * n + j] = (i <= j + 1) ? tile[threadIdx.x][r] : 0.0;
    }
}

// perm from ipiv (F:376-384) and its inverse (F:385-387): one CTA, shared memory.
__global__ void perm_kernel(int n, const int64_t* __restrict__ ipiv, int64_t* __restrict__ perm,
                            int64_t* __restrict__ iperm)
{
    extern __shared__ int sp[];
    for (int i = threadIdx.x; i < n; i += blockDim.x) sp[i] = i + 1;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k <= n - 2; ++k) {
            const int p = (int)ipiv[k - 1];
            if (p < k + 1 || p > n) continue;  // never produced by a completed reduction
            const int t = sp[k];
            sp[k] = sp[p - 1];
            sp[p - 1] = t;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        perm[i] = sp[i];
        iperm[sp[i] - 1] = i + 1;
    }
}

// Reset of the per-reduction state: ipiv[k] = k+1 (no interchange) and empty candidates,
// so that a reduction that ends early on a barrier timeout leaves only valid indices.
__global__ void reduce_init_kernel(int n, int64_t* ipiv, double* cand_v, int* cand_i, int ncand)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n - 2; k += gridDim.x * blockDim.x) ipiv[k] = k + 2;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncand; c += gridDim.x * blockDim.x) {
        cand_v[c] = 0.0;
        cand_i[c] = 0;
    }
}

constexpr size_t REDUCE_DSMEM = (size_t)T64_SLOTS * TILE64_BYTES > (size_t)PBOX_SLOTS * PBOX_BYTES
                                    ? (size_t)T64_SLOTS * TILE64_BYTES
                                    : (size_t)PBOX_SLOTS * PBOX_BYTES;

int reduce_grid_size()
{
    static int g_of[MAX_DEVICES] = {};
    int dev = 0;
    if (current_device(&dev) != cudaSuccess) return 0;
    if (g_of[dev] == 0) {
        int sms = 0, per = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaFuncSetAttribute(reduce_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)REDUCE_DSMEM) !=
            cudaSuccess)
            return 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, reduce_kernel, RT, REDUCE_DSMEM);
        g_of[dev] = sms * (per > 0 ? 1 : 0);
    }
    return g_of[dev];
}

// 2-D tensor map of a column-major FP64 array (rows x cols, leading dimension ld) in
// boxes of box_r x box_c, for TMA loads.  TMA needs a 16-byte row pitch (even ld).
bool make_tmap_2d(void* tmap, const double* base, int rows, int cols, int ld, int box_r, int box_c)
{
    if ((ld & 1) || rows < 1 || cols < 1) return false;
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    if (!enc) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
            return false;
        enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    const cuuint64_t dims[2] = {(cuuint64_t)rows, (cuuint64_t)cols};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(double)};
    const cuuint32_t box[2] = {(cuuint32_t)box_r, (cuuint32_t)box_c};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = enc((CUtensorMap*)tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void*)base, dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

cudaError_t launch_reduce(RedArgs a, int balance, int mode, cudaStream_t st)
{
    const int grid = reduce_grid_size();
    if (grid <= 0) return cudaErrorCooperativeLaunchTooLarge;
    reduce_init_kernel<<<64, 256, 0, st>>>(a.n, a.ipiv, a.cand_v, a.cand_i, grid);
    cudaError_t e0 = cudaGetLastError();
    if (e0 != cudaSuccess) return e0;
    int bal = balance;
    CUtensorMap tm, tp;
    memset(&tm, 0, sizeof(tm));
    memset(&tp, 0, sizeof(tp));
    if (a.use_tma) {
        const int P = (a.n + GEMV_GROUP - 1) / GEMV_GROUP;
        const bool ok = a.n >= 64 && a.n <= PMAX * GEMV_GROUP && make_tmap_2d(&tm, a.A, a.n, a.n, a.n, 64, 64) &&
                        make_tmap_2d(&tp, a.part, a.n, P, a.n, RT, PBOX_G);
        if (!ok) a.use_tma = 0;
    }
    void* args[] = {&a, &bal, &mode, &tm, &tp};
    return cudaLaunchCooperativeKernel((void*)reduce_kernel, dim3(grid), dim3(RT), args, REDUCE_DSMEM, st);
}

cudaError_t launch_unblocked_assemble(int n, double* A, const double* B2, const int64_t* ipiv, cudaStream_t st)
{
    if (n <= 0 || n > 512) return cudaErrorInvalidValue;
    unblocked_assemble_kernel<double><<<n, RT, 0, st>>>(n, A, A, B2, ipiv);
    return cudaGetLastError();
}

cudaError_t launch_reduce_f32(RedArgs a, int balance, float* A32, float* B32, cudaStream_t st)
{
    if (a.n < 1 || a.n >= 1024) return cudaErrorInvalidValue;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    // one thread per row in warps of 32 rows; the candidate arrays hold one entry per CTA
    const int rows = (a.n + 31) / 32, grid = rows < sms ? rows : sms;
    reduce_init_kernel<<<64, 256, 0, st>>>(a.n, a.ipiv, a.cand_v, a.cand_i, grid);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    void* args[] = {&a, &balance, &A32, &B32};
    return cudaLaunchCooperativeKernel((void*)reduce_f32_kernel, dim3(grid), dim3(RT), args, 0, st);
}

cudaError_t launch_reduce_f32_blocked(RedArgs a, int balance, float* A32, float* B0, float* w, float* pre,
                                     cudaStream_t st)
{
    if (a.n < 3) return cudaErrorInvalidValue;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const int rows = (a.n + 31) / 32, grid = rows < sms ? rows : sms;
    reduce_init_kernel<<<64, 256, 0, st>>>(a.n, a.ipiv, a.cand_v, a.cand_i, grid);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    void* args[] = {&a, &balance, &A32, &B0, &w, &pre};
    return cudaLaunchCooperativeKernel((void*)reduce_f32_blocked_kernel, dim3(grid), dim3(RT), args, 0, st);
}

cudaError_t launch_unblocked_assemble_f32(int n, double* F, const float* A32, const float* B32, const int64_t* ipiv,
                                          cudaStream_t st)
{
    if (n <= 0 || n >= 1024) return cudaErrorInvalidValue;
    unblocked_assemble_kernel<float><<<n, RT, 0, st>>>(n, F, A32, B32, ipiv);
    return cudaGetLastError();
}

cudaError_t launch_ht_perm(int n, const double* A, double* Ht, const int64_t* ipiv, int64_t* perm, int64_t* iperm,
                           cudaStream_t st)
{
    dim3 grid((n + 31) / 32, (n + 31) / 32);
    ht_fill_kernel<<<grid, dim3(32, 8), 0, st>>>(n, A, Ht);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    perm_kernel<<<1, 256, sizeof(int) * (size_t)n, st>>>(n, ipiv, perm, iperm);
    return cudaGetLastError();
}

cudaError_t launch_ht_fill(int n, const double* A, double* Ht, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    dim3 grid((n + 31) / 32, (n + 31) / 32);
    ht_fill_kernel<<<grid, dim3(32, 8), 0, st>>>(n, A, Ht);
    return cudaGetLastError();
}

cudaError_t launch_perm(int n, const int64_t* ipiv, int64_t* perm, int64_t* iperm, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    perm_kernel<<<1, 256, sizeof(int) * (size_t)n, st>>>(n, ipiv, perm, iperm);
    return cudaGetLastError();
}

size_t stepTabBytes() { return sizeof(StepTab); }

__global__ void fill_ones_kernel(double* a, double* b, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        a[i] = 1.0;
        b[i] = 1.0;
    }
}

cudaError_t launch_fill_ones(double* a, double* b, int n, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    fill_ones_kernel<<<(n + 255) / 256, 256, 0, st>>>(a, b, n);
    return cudaGetLastError();
}

__global__ void set_pair_kernel(double* a, double* b, double va, double vb)
{
    *a = va;
    *b = vb;
}

cudaError_t launch_set_pair(double* a, double* b, double va, double vb, cudaStream_t st)
{
    set_pair_kernel<<<1, 1, 0, st>>>(a, b, va, vb);
    return cudaGetLastError();
}

}  // namespace lhl
