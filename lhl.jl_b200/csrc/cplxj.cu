// cplxj.cu -- LHLWorkspace{ComplexF64}: the reduction of a complex J and the solves on it.
//
//   * balancing (F:299-340) with the complex modulus |z| = hypot(re, im) (cplx.cuh);
//   * below _lhl_block_min = 768 (F:703-705) the unblocked ELMHES reduction (F:466-501) with
//     the generic paired sweep (F:508-538); from 768 the generic blocked form (F:765-850 and
//     its helpers), as the reference chooses (F:398-399);
//   * Ht = H transposed (F:2005-2061) and perm / iperm (F:376-387);
//   * lhl_ldiv! on the complex reduction (F:3111-3121): applyZinv! (gather with the real
//     iscale, the generic L^-1 sweep F:2151-2195), the planar Hessenberg solve (complex.cu),
//     applyZ! (the generic L sweep F:2199-2243, scatter with scale);
//   * the residual of lhl_refine! with a complex J (F:3144-3157).
//
// Layout: J, factors and Ht are n x n interleaved complex (re, im pairs, leading dimension n),
// as a CuArray{ComplexF64}; scale and iscale are real.  The complex shift LU on the complex
// Ht is complex.cu's kernel with a complex Ht.
//
// Either reduction is one cooperative launch, one thread per row (rows by warps, spread over up
// to one CTA per SM).  The unblocked one is double-buffered like the real unblocked kernel
// (reduce.cu): step k reads the matrix of step k-1 with rows and columns k+1 <-> p swapped on
// the fly and writes the other buffer, so a step needs one grid barrier (the pivot search).
// The blocked one works in place (cj_blocked).  Every element sees the reference's complex
// operations in its order.
#include "cplx.cuh"
#include "internal.cuh"

namespace lhl {

constexpr int CJT = 256;
constexpr int CJW = CJT / 32;

__device__ __forceinline__ dc ldc(const double* A, int ld, int i, int j)
{
    const double2 w = reinterpret_cast<const double2*>(A)[(size_t)(j - 1) * ld + (i - 1)];
    return {w.x, w.y};
}
__device__ __forceinline__ void stc(double* A, int ld, int i, int j, dc v)
{
    reinterpret_cast<double2*>(A)[(size_t)(j - 1) * ld + (i - 1)] = make_double2(v.re, v.im);
}

// every CTA reads all CTA candidates and reduces them (first max)
__device__ __forceinline__ void cj_combine(const CjArgs& a, int* s_p, double* s_red, int* s_redi)
{
    const int t = threadIdx.x;
    double v = 0.0;
    int vi = 0;
    for (int c = t; c < (int)gridDim.x; c += CJT) {
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
        for (int w = 0; w < CJW; ++w) argmax_combine(bv, bi, s_red[w], s_redi[w]);
        *s_p = bi;
    }
    __syncthreads();
}

__device__ __forceinline__ void cj_publish(const CjArgs& a, double v, int vi, double* s_red, int* s_redi)
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
        for (int w = 0; w < CJW; ++w) argmax_combine(bv, bi, s_red[w], s_redi[w]);
        a.cand_v[blockIdx.x] = bv;
        a.cand_i[blockIdx.x] = bi;
    }
    __syncthreads();
}

// Balancing (F:299-340), organised as the real kernel's: per sweep (1) every index's
// column and row sums of moduli without the diagonal, each summed in the reference's order
// by one thread; (2) CTA 0 walks i = 1..n in order taking the reference's decision, the
// sums of later indices patched for an index that scales; (3) all CTAs apply the sweep's
// power-of-two factors (exact on both parts).
__device__ bool cj_balance(const CjArgs& a, GridBarrier& gb)
{
    const int n = a.n;
    double* A = a.A;
    const int gt = blockIdx.x * CJT + threadIdx.x;
    const int gsz = gridDim.x * CJT;
    for (int i = gt; i < n; i += gsz) {
        a.scale[i] = 1.0;
        a.iscale[i] = 1.0;
    }
    __shared__ int s_first;
    __shared__ double s_f;
    for (int sweep = 0; sweep < 20; ++sweep) {
        for (int i = 1 + gt; i <= n; i += gsz) {
            double c = 0.0, r = 0.0;
            for (int j = 1; j <= n; ++j) {
                if (j == i) continue;
                c = dadd(c, cabs_h(ldc(A, n, j, i)));
                r = dadd(r, cabs_h(ldc(A, n, i, j)));
            }
            a.bsum[i - 1] = c;
            a.bsum[n + i - 1] = r;
            a.bfac[i - 1] = 1.0;
        }
        if (gt == 0) a.bflag[0] = 0;
        if (!gb.sync()) return false;
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
                    base += CJT;
                    continue;
                }
                if (i == si) {
                    s_f = f;
                    a.bflag[0] = 1;
                }
                __syncthreads();
                const double fs = s_f;
                for (int m = si + 1 + threadIdx.x; m <= n; m += CJT) {
                    const double vr = cabs_h(ldc(A, n, si, m));
                    const double vc = cabs_h(ldc(A, n, m, si));
                    a.bsum[m - 1] = (a.bsum[m - 1] - vr) + vr / fs;
                    a.bsum[n + m - 1] = (a.bsum[n + m - 1] - vc) + vc * fs;
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
        for (size_t e = gt; e < (size_t)n * n; e += gsz) {
            const int i = (int)(e % n), j = (int)(e / n);
            const double fi = a.bfac[i], fj = a.bfac[j];
            if (fi != 1.0 || fj != 1.0) {
                A[2 * e] = (A[2 * e] / fi) * fj;
                A[2 * e + 1] = (A[2 * e + 1] / fi) * fj;
            }
        }
        if (!gb.sync()) return false;
    }
    return true;
}

// Unblocked ELMHES with the generic paired sweep (F:466-538), one thread per row.
__device__ bool cj_unblocked(const CjArgs& a, GridBarrier& gb, dc* s_l)
{
    const int n = a.n;
    double* buf[2] = {a.A, a.B};
    __shared__ double s_red[CJW];
    __shared__ int s_redi[CJW];
    __shared__ int s_p;
    const int gt = blockIdx.x * CJT + threadIdx.x;
    // rows by warps spread over the CTAs (global warp w = local warp * grid + CTA holds rows
    // 32 w + 1 .. 32 w + 32), so that every SM streams a share of the matrix each step
    const int i = 32 * ((threadIdx.x >> 5) * (int)gridDim.x + (int)blockIdx.x) + (threadIdx.x & 31) + 1;
    {
        double v = 0.0;
        int vi = 0;
        if (i >= 2 && i <= n) { v = cabs_h(ldc(a.A, n, i, 1)); vi = i; }
        cj_publish(a, v, vi, s_red, s_redi);
    }
    if (!gb.sync()) return false;
    for (int k = 1; k <= n - 2; ++k) {
        const double* R = buf[(k - 1) & 1];
        double* W = buf[k & 1];
        cj_combine(a, &s_p, s_red, s_redi);
        const int p = (s_p >= k + 1 && s_p <= n) ? s_p : k + 1;
        if (gt == 0) a.ipiv[k - 1] = p;
        auto sw = [&](int r) { return r == k + 1 ? p : (r == p ? k + 1 : r); };
        const dc piv = ldc(R, n, p, k);
        const bool pz = ciszero(piv);
        // multipliers l_j = A'[j,k] / piv (F:489-491), j = k+2..n
        for (int j = k + 2 + threadIdx.x; j <= n; j += CJT) {
            const dc v = ldc(R, n, sw(j), k);
            s_l[j - 1] = pz ? v : cdiv(v, piv);
        }
        __syncthreads();
        double cand = 0.0;
        int candi = 0;
        if (i <= n) {
            const int si = sw(i);
            dc ck = ldc(R, n, si, k);
            if (!pz && i >= k + 2) ck = s_l[i - 1];
            stc(W, n, i, k, ck);
            dc ck1 = ldc(R, n, si, p);
            if (pz) {
                // step skipped (F:488): rows and columns still carry the interchange
                for (int j = k + 2; j <= n; ++j) stc(W, n, i, j, ldc(R, n, si, sw(j)));
                stc(W, n, i, k + 1, ck1);
            } else {
                const dc pk = ldc(R, n, p, p);
                const bool low = i >= k + 2;
                const dc li = low ? s_l[i - 1] : dc{0.0, 0.0};
                if (low && !ciszero(pk)) ck1 = csub(ck1, cmul(li, pk));  // F:492-496
                int j = k + 2;
                // eight column pairs at a time: every load of the block is issued before its
                // stores (a store to W could otherwise hold back the next load from R)
                for (; j + 15 <= n; j += 16) {
                    dc v[16], pr[16];
#pragma unroll
                    for (int u = 0; u < 16; ++u) {
                        const int sj = sw(j + u);
                        v[u] = ldc(R, n, si, sj);
                        pr[u] = low ? ldc(R, n, p, sj) : dc{0.0, 0.0};
                    }
#pragma unroll
                    for (int u = 0; u < 16; u += 2) {
                        dc v0 = v[u], v1 = v[u + 1];
                        if (low) {
                            v0 = csub(v0, cmul(li, pr[u]));
                            v1 = csub(v1, cmul(li, pr[u + 1]));
                        }
                        stc(W, n, i, j + u, v0);
                        stc(W, n, i, j + u + 1, v1);
                        ck1 = cadd(ck1, cadd(cmul(s_l[j + u - 1], v0), cmul(s_l[j + u], v1)));
                    }
                }
                while (j + 1 <= n) {  // column pairs (F:515-528)
                    const int sj = sw(j), sj1 = sw(j + 1);
                    dc v0 = ldc(R, n, si, sj), v1 = ldc(R, n, si, sj1);
                    if (low) {
                        v0 = csub(v0, cmul(li, ldc(R, n, p, sj)));
                        v1 = csub(v1, cmul(li, ldc(R, n, p, sj1)));
                    }
                    stc(W, n, i, j, v0);
                    stc(W, n, i, j + 1, v1);
                    ck1 = cadd(ck1, cadd(cmul(s_l[j - 1], v0), cmul(s_l[j], v1)));
                    j += 2;
                }
                if (j <= n) {  // last single column (F:529-536)
                    const int sj = sw(j);
                    dc v0 = ldc(R, n, si, sj);
                    if (low) v0 = csub(v0, cmul(li, ldc(R, n, p, sj)));
                    stc(W, n, i, j, v0);
                    ck1 = cadd(ck1, cmul(s_l[j - 1], v0));
                }
                stc(W, n, i, k + 1, ck1);
            }
            if (i >= k + 2) { cand = cabs_h(ck1); candi = i; }
        }
        cj_publish(a, cand, candi, s_red, s_redi);
        if (!gb.sync()) return false;
    }
    return true;
}

// ---- the blocked form (n >= 768) ---------------------------------------------------
// The generic delayed-update reduction the reference runs for T = ComplexF64 from
// _lhl_block_min = 768 (F:398-399, F:705), nb = 16 (F:706).  Per panel k0..kb: the pre-panel
// copy B0 of the panel columns; per step the pivot search, the step's interchanges
// (F:857-890, CTA 0 alone: the row exchange over the panel columns, then the column exchange
// within the panel or the pulled column with its missed interchanges and left transforms),
// the multipliers and left transforms of the panel columns, the right transforms inside the
// panel, the GEMV against the pre-panel trailing block (F:1418-1440, groups of four columns),
// its interchanges and corrections, and the add into column k+1 (F:787-850).  Panel end: per
// trailing column the row interchanges (F:1336-1342), the TRSM (F:1917-1927) and the rank-nb
// GEMM with b = -one(T) * B element (F:1676-1689); the rows above the panel take their
// in-panel right updates, then the top GEMM (F:1588-1607).  After the last panel the deferred
// interchanges of the panel columns (F:1383-1393).  Every element sees the reference's complex
// operations in its order.  One thread per row for the per-step work (rows by warps spread
// over the CTAs), one CTA per trailing column for the panel-end update.
constexpr int CJ_NB = 16;          // panel width (F:706)
constexpr int CJ_BLOCK_MIN = 768;  // _lhl_block_min(ComplexF64), F:705

// the rows the step interchanges of w touch and where each one's value comes from:
// w[kk+1] <-> w[q] for kk = k0..k in order (F:826-829)
struct CjPerm {
    int row[2 * CJ_NB + 2];
    int src[2 * CJ_NB + 2];
    int cnt;
};

__device__ __forceinline__ int cj_perm_slot(CjPerm& P, int r)
{
    for (int s = 0; s < P.cnt; ++s)
        if (P.row[s] == r) return s;
    P.row[P.cnt] = r;
    P.src[P.cnt] = r;
    return P.cnt++;
}

__device__ __forceinline__ int cj_perm_src(const CjPerm& P, int r)
{
    for (int s = 0; s < P.cnt; ++s)
        if (P.row[s] == r) return P.src[s];
    return r;
}

// The interchange of step k with pivot row p != k+1 (F:806-808, F:857-890), CTA 0 alone.
__device__ void cj_step_swaps(const CjArgs& a, double* B0, int k0, int kb, int k, int p)
{
    const int n = a.n, t = threadIdx.x;
    double* A = a.A;
    if (t == 0)
        for (int j = k0; j <= kb + 1; ++j) {  // column k first in the reference; distinct elements
            const dc x = ldc(A, n, k + 1, j);
            stc(A, n, k + 1, j, ldc(A, n, p, j));
            stc(A, n, p, j, x);
        }
    __syncthreads();
    if (p <= kb + 1) {
        for (int i = 1 + t; i <= n; i += CJT) {
            const dc x = ldc(A, n, i, k + 1);
            stc(A, n, i, k + 1, ldc(A, n, i, p));
            stc(A, n, i, p, x);
            const dc y = ldc(B0, n, i, k + 1 - k0);
            stc(B0, n, i, k + 1 - k0, ldc(B0, n, i, p - k0));
            stc(B0, n, i, p - k0, y);
        }
        __syncthreads();
        return;
    }
    for (int i = 1 + t; i <= n; i += CJT) {
        const dc x = ldc(A, n, i, p);
        stc(A, n, i, p, ldc(B0, n, i, k + 1 - k0));
        stc(B0, n, i, k + 1 - k0, x);
        stc(A, n, i, k + 1, x);
    }
    __syncthreads();
    if (t == 0)
        for (int kk = k0; kk <= k; ++kk) {
            const int q = (int)a.ipiv[kk - 1];
            if (q != kk + 1) {
                const dc x = ldc(A, n, kk + 1, k + 1);
                stc(A, n, kk + 1, k + 1, ldc(A, n, q, k + 1));
                stc(A, n, q, k + 1, x);
            }
        }
    __syncthreads();
    for (int kk = k0; kk <= k - 1; ++kk) {
        const dc x = ldc(A, n, kk + 1, k + 1);
        if (!ciszero(x))
            for (int i = kk + 2 + t; i <= n; i += CJT) stc(A, n, i, k + 1, csub(ldc(A, n, i, k + 1), cmul(ldc(A, n, i, kk), x)));
        __syncthreads();
    }
}

// w for row r: sum over columns c0..c1 of A[j,k] A[r,j], from zero, four columns per pass
__device__ __forceinline__ dc cj_gemv_row(const double* A, int n, int k, int r, int c0, int c1)
{
    dc acc = {0.0, 0.0};
    int j = c0;
#pragma unroll 2
    for (; j + 3 <= c1; j += 4) {
        const dc l1 = ldc(A, n, j, k), l2 = ldc(A, n, j + 1, k), l3 = ldc(A, n, j + 2, k), l4 = ldc(A, n, j + 3, k);
        const dc a1 = ldc(A, n, r, j), a2 = ldc(A, n, r, j + 1), a3 = ldc(A, n, r, j + 2), a4 = ldc(A, n, r, j + 3);
        acc = cadd(acc, cadd(cadd(cmul(l1, a1), cmul(l2, a2)), cadd(cmul(l3, a3), cmul(l4, a4))));
    }
    for (; j <= c1; ++j) {
        const dc lj = ldc(A, n, j, k);
        if (!ciszero(lj)) acc = cadd(acc, cmul(lj, ldc(A, n, r, j)));
    }
    return acc;
}

__device__ bool cj_blocked(const CjArgs& a, GridBarrier& gb)
{
    const int n = a.n;
    double* A = a.A;
    double* B0 = a.B;                                 // n x (nb + 1) complex
    double* w = a.B + 2 * (size_t)n * (CJ_NB + 1);    // the chain rows' GEMV values (n complex)
    __shared__ double s_red[CJW];
    __shared__ int s_redi[CJW];
    __shared__ int s_p;
    __shared__ CjPerm s_perm;
    __shared__ dc s_w[CJ_NB + 2], s_x[CJ_NB + 1], s_b[CJ_NB + 1];
    const int t = threadIdx.x;
    const int gt = blockIdx.x * CJT + t, gsz = gridDim.x * CJT;
    const int r = 32 * ((t >> 5) * (int)gridDim.x + (int)blockIdx.x) + (t & 31) + 1;  // this thread's row
    const dc minus_one = {-1.0, -0.0}, one = {1.0, 0.0};
    {
        double v = 0.0;
        int vi = 0;
        if (r >= 2 && r <= n) { v = cabs_h(ldc(A, n, r, 1)); vi = r; }
        cj_publish(a, v, vi, s_red, s_redi);
    }
    if (!gb.sync()) return false;
    for (int k0 = 1; k0 <= n - 2; k0 += CJ_NB) {
        const int kb = k0 + CJ_NB - 1 < n - 2 ? k0 + CJ_NB - 1 : n - 2;
        const int np = kb + 1 - k0;  // panel columns k0+1..kb+1
        for (size_t e = gt; e < (size_t)n * np; e += gsz) {
            const int i = (int)(e % n) + 1, jj = (int)(e / n) + 1;
            stc(B0, n, i, jj, ldc(A, n, i, k0 + jj));
        }
        if (!gb.sync()) return false;
        for (int k = k0; k <= kb; ++k) {
            cj_combine(a, &s_p, s_red, s_redi);
            const int p = (s_p >= k + 1 && s_p <= n) ? s_p : k + 1;
            if (gt == 0) a.ipiv[k - 1] = p;
            if (p != k + 1) {
                if (blockIdx.x == 0) {
                    __syncthreads();  // ipiv[k-1] from thread 0
                    cj_step_swaps(a, B0, k0, kb, k, p);
                }
                if (!gb.sync()) return false;
            }
            const dc piv = ldc(A, n, k + 1, k);
            if (!ciszero(piv)) {
                // multipliers and the left transforms of the panel columns (F:813-821)
                if (r >= k + 2 && r <= n) {
                    const dc l = cdiv(ldc(A, n, r, k), piv);
                    stc(A, n, r, k, l);
                    for (int j = k + 1; j <= kb + 1; ++j) {
                        const dc pj = ldc(A, n, k + 1, j);
                        if (!ciszero(pj)) stc(A, n, r, j, csub(ldc(A, n, r, j), cmul(l, pj)));
                    }
                }
                if (t == 0) {  // the step interchanges of w, as a map of the touched rows
                    s_perm.cnt = 0;
                    for (int kk = k0; kk <= k; ++kk) {
                        const int q = kk == k ? p : (int)a.ipiv[kk - 1];  // step k's entry may not be visible yet
                        if (q == kk + 1) continue;
                        const int s1 = cj_perm_slot(s_perm, kk + 1), s2 = cj_perm_slot(s_perm, q);
                        const int x = s_perm.src[s1];
                        s_perm.src[s1] = s_perm.src[s2];
                        s_perm.src[s2] = x;
                    }
                }
                if (!gb.sync()) return false;
                // right transforms inside the panel (F:822-827), then the GEMV of the row whose
                // value the interchanges bring to this row (F:829-833)
                dc acc = {0.0, 0.0}, wv = {0.0, 0.0};
                const bool mine = r >= k0 + 1 && r <= n;
                if (mine) {
                    acc = ldc(A, n, r, k + 1);
                    for (int j = k + 2; j <= kb + 1; ++j) {
                        const dc vj = ldc(A, n, j, k);
                        if (!ciszero(vj)) acc = cadd(acc, cmul(vj, ldc(A, n, r, j)));
                    }
                    wv = cj_gemv_row(A, n, k, cj_perm_src(s_perm, r), kb + 2, n);
                    if (r <= k + 1) stc(w, n, r, 1, wv);
                }
                if (!gb.sync()) return false;
                // the corrections' chain on the rows k0+1..k+1, in every CTA (F:834-839)
                if (t == 0) {
                    for (int i = k0 + 1; i <= k + 1; ++i) s_w[i - k0] = ldc(w, n, i, 1);
                    for (int kk = k0; kk <= k; ++kk) {
                        const dc x = s_w[kk + 1 - k0];
                        s_x[kk - k0] = x;
                        if (ciszero(x)) continue;
                        for (int i = kk + 2; i <= k + 1; ++i) s_w[i - k0] = csub(s_w[i - k0], cmul(ldc(A, n, i, kk), x));
                    }
                }
                __syncthreads();
                if (mine) {
                    if (r <= k + 1) {
                        wv = s_w[r - k0];
                    } else {
                        for (int kk = k0; kk <= k; ++kk) {
                            const dc x = s_x[kk - k0];
                            if (!ciszero(x)) wv = csub(wv, cmul(ldc(A, n, r, kk), x));
                        }
                    }
                    stc(A, n, r, k + 1, cadd(acc, wv));  // F:840-842
                }
            }
            // the next step's pivot candidates: column k+1, rows k+2..n
            double v = 0.0;
            int vi = 0;
            if (r >= k + 2 && r <= n) { v = cabs_h(ldc(A, n, r, k + 1)); vi = r; }
            cj_publish(a, v, vi, s_red, s_redi);
            if (!gb.sync()) return false;
        }
        // panel end, trailing columns: interchanges, TRSM, GEMM (one CTA per column)
        for (int c = kb + 2 + (int)blockIdx.x; c <= n; c += gridDim.x) {
            if (t == 0) {
                for (int k = k0; k <= kb; ++k) {
                    const int q = (int)a.ipiv[k - 1];
                    if (q != k + 1) {
                        const dc x = ldc(A, n, k + 1, c);
                        stc(A, n, k + 1, c, ldc(A, n, q, c));
                        stc(A, n, q, c, x);
                    }
                }
                for (int k = k0; k <= kb; ++k) {
                    const dc x = ldc(A, n, k + 1, c);
                    if (ciszero(x)) continue;
                    for (int i = k + 2; i <= kb + 1; ++i) stc(A, n, i, c, csub(ldc(A, n, i, c), cmul(ldc(A, n, i, k), x)));
                }
                for (int j = k0; j <= kb; ++j) s_b[j - k0] = cmul(minus_one, ldc(A, n, j + 1, c));
            }
            __syncthreads();
            for (int i = kb + 2 + t; i <= n; i += CJT) {
                dc x = ldc(A, n, i, c);
                for (int j = k0; j <= kb; ++j) {
                    const dc b = s_b[j - k0];
                    if (!ciszero(b)) x = cadd(x, cmul(ldc(A, n, i, j), b));
                }
                stc(A, n, i, c, x);
            }
            __syncthreads();
        }
        // rows above the panel: the in-panel right updates (F:1597-1606) ...
        for (int i = 1 + gt; i <= k0; i += gsz)
            for (int k = k0; k <= kb; ++k)
                for (int j = k + 2; j <= kb + 1; ++j) {
                    const dc vj = ldc(A, n, j, k);
                    if (!ciszero(vj)) stc(A, n, i, k + 1, cadd(ldc(A, n, i, k + 1), cmul(vj, ldc(A, n, i, j))));
                }
        if (!gb.sync()) return false;
        // ... then the top GEMM A[1:k0, k0+1:kb+1] += A[1:k0, kb+2:n] * (one * A[kb+2:n, k0:kb])
        for (size_t e = gt; e < (size_t)k0 * np; e += gsz) {
            const int i = (int)(e % k0) + 1, c = k0 + 1 + (int)(e / k0);
            dc x = ldc(A, n, i, c);
            for (int j = kb + 2; j <= n; ++j) {
                const dc b = cmul(one, ldc(A, n, j, c - 1));
                if (!ciszero(b)) x = cadd(x, cmul(ldc(A, n, i, j), b));
            }
            stc(A, n, i, c, x);
        }
        if (!gb.sync()) return false;
    }
    // the interchanges deferred on the multipliers (F:1383-1393)
    for (int c = 1 + gt; c <= n - 2; c += gsz) {
        const int kbc = ((c - 1) / CJ_NB + 1) * CJ_NB < n - 2 ? ((c - 1) / CJ_NB + 1) * CJ_NB : n - 2;
        for (int k = kbc + 1; k <= n - 2; ++k) {
            const int q = (int)a.ipiv[k - 1];
            if (q != k + 1) {
                const dc x = ldc(A, n, k + 1, c);
                stc(A, n, k + 1, c, ldc(A, n, q, c));
                stc(A, n, q, c, x);
            }
        }
    }
    return true;
}

__global__ void __launch_bounds__(CJT, 1) cj_blocked_kernel(CjArgs a, int balance)
{
    GridBarrier gb{a.bar, a.err, a.limit_ns, 0, nullptr};
    if (balance && !cj_balance(a, gb)) return;
    if (a.n >= 3) cj_blocked(a, gb);
}

__global__ void __launch_bounds__(CJT, 1) cj_reduce_kernel(CjArgs a, int balance)
{
    extern __shared__ double2 cj_dyn[];
    GridBarrier gb{a.bar, a.err, a.limit_ns, 0, nullptr};
    if (balance && !cj_balance(a, gb)) return;
    if (a.n >= 3) cj_unblocked(a, gb, reinterpret_cast<dc*>(cj_dyn));
}

__global__ void cj_init_kernel(int n, int64_t* ipiv, double* cand_v, int* cand_i, int ncand)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n - 2; k += gridDim.x * blockDim.x) ipiv[k] = k + 2;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncand; c += gridDim.x * blockDim.x) {
        cand_v[c] = 0.0;
        cand_i[c] = 0;
    }
}

// Final assembly: column j from buffer j&1 (columns n-1, n from the last step's buffer) with
// the interchanges of steps j+1..n-2 applied (F:480-485).  One CTA per column.
__global__ void __launch_bounds__(CJT) cj_assemble_kernel(int n, double* A, const double* B2, const int64_t* ipiv)
{
    extern __shared__ double2 col[];
    const int j = blockIdx.x + 1;
    if (j > n) return;
    const double* src;
    int from;
    if (j <= n - 2) {
        src = (j & 1) ? B2 : A;
        from = j + 1;
    } else {
        const int kl = n - 2;
        src = (kl >= 1 && (kl & 1)) ? B2 : A;
        from = n - 1;
    }
    const double2* s2 = reinterpret_cast<const double2*>(src) + (size_t)(j - 1) * n;
    for (int i = threadIdx.x; i < n; i += CJT) col[i] = s2[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = from; k <= n - 2; ++k) {
            const int p = (int)ipiv[k - 1];
            if (p > k + 1 && p <= n) {
                const double2 t = col[k];
                col[k] = col[p - 1];
                col[p - 1] = t;
            }
        }
    }
    __syncthreads();
    double2* d2 = reinterpret_cast<double2*>(A) + (size_t)(j - 1) * n;
    for (int i = threadIdx.x; i < n; i += CJT) d2[i] = col[i];
}

// Ht[j,i] = A[i,j] for i <= j+1, zero elsewhere (F:2005-2061); 32 x 32 tiles.
__global__ void cj_ht_kernel(int n, const double* __restrict__ A, double* __restrict__ Ht)
{
    __shared__ double2 tile[32][33];
    const double2* A2 = reinterpret_cast<const double2*>(A);
    double2* H2 = reinterpret_cast<double2*>(Ht);
    const int bi = blockIdx.y * 32, bj = blockIdx.x * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = bi + threadIdx.x, j = bj + r;
        tile[r][threadIdx.x] = (i < n && j < n) ? A2[(size_t)j * n + i] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = bi + r, j = bj + threadIdx.x;
        if (i < n && j < n) H2[(size_t)i * n + j] = (i <= j + 1) ? tile[threadIdx.x][r] : make_double2(0.0, 0.0);
    }
}

// one CTA per SM at most, at least one warp of rows per CTA; together they hold >= n rows
int cj_grid_size(int n)
{
    static int sms_of[MAX_DEVICES] = {};
    int dev = 0;
    if (current_device(&dev) != cudaSuccess) dev = 0;
    if (sms_of[dev] == 0) {
        int c = 0;
        sms_of[dev] = (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && c > 0) ? c : 1;
    }
    const int sms = sms_of[dev];
    const int warps = (n + 31) / 32;
    int g = warps < sms ? warps : sms;
    if (g < 1) g = 1;
    while ((long long)g * CJT < n) ++g;  // 8 warps per CTA must cover n rows
    return g;
}

size_t cj_smem(int n) { return (size_t)(n > 0 ? n : 1) * sizeof(double2); }

cudaError_t launch_reduce_cj(CjArgs a, int balance, cudaStream_t st)
{
    const int n = a.n;
    if (n <= 0) return cudaSuccess;
    if (n > CJ_NMAX) return cudaErrorInvalidValue;
    const int grid = cj_grid_size(n);
    const size_t smem = cj_smem(n);
    static size_t attr_r[MAX_DEVICES] = {}, attr_a[MAX_DEVICES] = {};
    cudaError_t e = opt_in_smem((const void*)cj_reduce_kernel, smem, attr_r);
    if (e != cudaSuccess) return e;
    e = opt_in_smem((const void*)cj_assemble_kernel, smem, attr_a);
    if (e != cudaSuccess) return e;
    cj_init_kernel<<<16, 256, 0, st>>>(n, a.ipiv, a.cand_v, a.cand_i, grid);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int bal = balance;
    void* args[] = {&a, &bal};
    const bool blocked = n >= CJ_BLOCK_MIN;  // the reference's choice (F:398-399, F:705)
    e = blocked ? cudaLaunchCooperativeKernel((void*)cj_blocked_kernel, dim3(grid), dim3(CJT), args, 0, st)
                : cudaLaunchCooperativeKernel((void*)cj_reduce_kernel, dim3(grid), dim3(CJT), args, smem, st);
    if (e != cudaSuccess) return e;
    if (n >= 3 && !blocked) {
        cj_assemble_kernel<<<n, CJT, smem, st>>>(n, a.A, a.B, a.ipiv);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    dim3 hg((n + 31) / 32, (n + 31) / 32);
    cj_ht_kernel<<<hg, dim3(32, 8), 0, st>>>(n, a.A, a.Ht);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_perm(n, a.ipiv, a.perm, a.iperm, st);
}

// ---- solves ------------------------------------------------------------------------
// One CTA per complex right-hand side; the vector lives in shared memory.  L[i,k] =
// factors[i,k] (i >= k+2), read as the packed Lp of the reference holds it (F:407-464).

// y <- L^-1 y, the generic sweep F:2151-2195: groups of four steps (a serial head triangle,
// then rows k+5:n take all four columns at once as (L1 x1 + L2 x2) + (L3 x3 + L4 x4)), then
// single steps.
__device__ void cj_fwd(int n, const double* F, dc* y)
{
    const int t = threadIdx.x;
    const int G = (n - 2 > 0 ? n - 2 : 0) >> 2;
    for (int g = 1; g <= G; ++g) {
        const int k = 4 * g - 3;
        if (t == 0) {
            const dc x1 = y[k];
            const dc x2 = csub(y[k + 1], cmul(ldc(F, n, k + 2, k), x1));
            y[k + 1] = x2;
            const dc x3 = csub(y[k + 2], cadd(cmul(ldc(F, n, k + 3, k), x1), cmul(ldc(F, n, k + 3, k + 1), x2)));
            y[k + 2] = x3;
            const dc x4 = csub(y[k + 3], cadd(cadd(cmul(ldc(F, n, k + 4, k), x1), cmul(ldc(F, n, k + 4, k + 1), x2)),
                                              cmul(ldc(F, n, k + 4, k + 2), x3)));
            y[k + 3] = x4;
        }
        __syncthreads();
        const dc x1 = y[k], x2 = y[k + 1], x3 = y[k + 2], x4 = y[k + 3];
        for (int i = k + 5 + t; i <= n; i += CJT) {
            const dc s = cadd(cadd(cmul(ldc(F, n, i, k), x1), cmul(ldc(F, n, i, k + 1), x2)),
                              cadd(cmul(ldc(F, n, i, k + 2), x3), cmul(ldc(F, n, i, k + 3), x4)));
            y[i - 1] = csub(y[i - 1], s);
        }
        __syncthreads();
    }
    for (int k = 4 * G + 1; k <= n - 2; ++k) {
        const dc xk = y[k];
        for (int i = k + 2 + t; i <= n; i += CJT) y[i - 1] = csub(y[i - 1], cmul(ldc(F, n, i, k), xk));
        __syncthreads();
    }
}

// y <- L y, the generic sweep F:2199-2243: single steps in reverse, then groups in reverse;
// a group reads its four values first (step k+c touches rows k+c+2:n only).
__device__ void cj_bwd(int n, const double* F, dc* y)
{
    const int t = threadIdx.x;
    const int G = (n - 2 > 0 ? n - 2 : 0) >> 2;
    for (int k = n - 2; k >= 4 * G + 1; --k) {
        const dc xk = y[k];
        for (int i = k + 2 + t; i <= n; i += CJT) y[i - 1] = cadd(y[i - 1], cmul(ldc(F, n, i, k), xk));
        __syncthreads();
    }
    for (int g = G; g >= 1; --g) {
        const int k = 4 * g - 3;
        const dc x1 = y[k], x2 = y[k + 1], x3 = y[k + 2], x4 = y[k + 3];
        __syncthreads();
        if (t == 0) {
            y[k + 1] = cadd(x2, cmul(ldc(F, n, k + 2, k), x1));
            y[k + 2] = cadd(x3, cadd(cmul(ldc(F, n, k + 3, k), x1), cmul(ldc(F, n, k + 3, k + 1), x2)));
            y[k + 3] = cadd(x4, cadd(cadd(cmul(ldc(F, n, k + 4, k), x1), cmul(ldc(F, n, k + 4, k + 1), x2)),
                                     cmul(ldc(F, n, k + 4, k + 2), x3)));
        }
        for (int i = k + 5 + t; i <= n; i += CJT) {
            const dc s = cadd(cadd(cmul(ldc(F, n, i, k), x1), cmul(ldc(F, n, i, k + 1), x2)),
                              cadd(cmul(ldc(F, n, i, k + 2), x3), cmul(ldc(F, n, i, k + 3), x4)));
            y[i - 1] = cadd(y[i - 1], s);
        }
        __syncthreads();
    }
}

// applyZinv! (F:2104-2112): y = P^-1 D^-1 x (F:2130-2140), y <- L^-1 y.  Column c = col0 +
// blockIdx.x of X (interleaved, ld ldx complex); out to X itself, or (planar != 0) to columns
// 2 b, 2 b + 1 of Y (ld ldy) as two planes for the Hessenberg solve.
__global__ void __launch_bounds__(CJT) cj_zinv_kernel(int n, const double* __restrict__ F,
                                                       const int64_t* __restrict__ perm,
                                                       const double* __restrict__ iscale, double* X, int ldx,
                                                       int col0, double* Y, int ldy, int planar,
                                                       const double* __restrict__ done, double tol)
{
    extern __shared__ double2 yv[];
    dc* y = reinterpret_cast<dc*>(yv);
    const int b = blockIdx.x, c = col0 + b;
    if (done && done[c] <= tol) return;
    double2* x2 = reinterpret_cast<double2*>(X) + (size_t)c * ldx;
    for (int i = threadIdx.x; i < n; i += CJT) {
        const int p = (int)perm[i] - 1;
        const double2 v = x2[p];
        const double s = iscale[p];
        y[i] = {dmul(v.x, s), dmul(v.y, s)};
    }
    __syncthreads();
    cj_fwd(n, F, y);
    __syncthreads();
    if (planar) {
        double* yr = Y + (size_t)(2 * b) * ldy;
        double* yi = yr + ldy;
        for (int i = threadIdx.x; i < n; i += CJT) {
            yr[i] = y[i].re;
            yi[i] = y[i].im;
        }
    } else {
        for (int i = threadIdx.x; i < n; i += CJT) x2[i] = make_double2(y[i].re, y[i].im);
    }
}

// applyZ! (F:2069-2082): y <- L y, x = D P y (x[i] = y[iperm[i]] * scale[i]).  In from X
// itself, or (planar != 0) from the planes in columns 2 b, 2 b + 1 of Y.
__global__ void __launch_bounds__(CJT) cj_z_kernel(int n, const double* __restrict__ F,
                                                    const int64_t* __restrict__ iperm,
                                                    const double* __restrict__ scale, double* X, int ldx, int col0,
                                                    const double* Y, int ldy, int planar,
                                                    const double* __restrict__ done, double tol)
{
    extern __shared__ double2 yv[];
    dc* y = reinterpret_cast<dc*>(yv);
    const int b = blockIdx.x, c = col0 + b;
    if (done && done[c] <= tol) return;
    double2* x2 = reinterpret_cast<double2*>(X) + (size_t)c * ldx;
    if (planar) {
        const double* yr = Y + (size_t)(2 * b) * ldy;
        const double* yi = yr + ldy;
        for (int i = threadIdx.x; i < n; i += CJT) y[i] = {yr[i], yi[i]};
    } else {
        for (int i = threadIdx.x; i < n; i += CJT) y[i] = {x2[i].x, x2[i].y};
    }
    __syncthreads();
    cj_bwd(n, F, y);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += CJT) {
        const dc v = y[(int)iperm[i] - 1];
        const double s = scale[i];
        x2[i] = make_double2(dmul(v.re, s), dmul(v.im, s));
    }
}

cudaError_t launch_ldiv_cj(const LdivArgs& a, int nrhs, cudaStream_t st)
{
    const int n = a.n;
    if (nrhs <= 0 || n <= 0) return cudaSuccess;
    if (n > CJ_NMAX || !a.Y || a.ycap < 2) return cudaErrorInvalidValue;
    const size_t smem = cj_smem(n);
    static size_t attr_zi[MAX_DEVICES] = {}, attr_z[MAX_DEVICES] = {};
    cudaError_t e = opt_in_smem((const void*)cj_zinv_kernel, smem, attr_zi);
    if (e != cudaSuccess) return e;
    e = opt_in_smem((const void*)cj_z_kernel, smem, attr_z);
    if (e != cudaSuccess) return e;
    if (a.mode == 1) {  // applyZinv!
        cj_zinv_kernel<<<nrhs, CJT, smem, st>>>(n, a.F, a.perm, a.iscale, a.X, a.ldx, 0, nullptr, 0, 0, a.done, a.tol);
        return cudaGetLastError();
    }
    if (a.mode == 2) {  // applyZ!
        cj_z_kernel<<<nrhs, CJT, smem, st>>>(n, a.F, a.iperm, a.scale, a.X, a.ldx, 0, nullptr, 0, 0, a.done, a.tol);
        return cudaGetLastError();
    }
    // lhl_ldiv! (F:3111-3121): applyZinv!, planar Hessenberg solve, applyZ!
    const int chunk = a.ycap / 2;
    for (int c0 = 0; c0 < nrhs; c0 += chunk) {
        const int cnt = min(chunk, nrhs - c0);
        cj_zinv_kernel<<<cnt, CJT, smem, st>>>(n, a.F, a.perm, a.iscale, a.X, a.ldx, c0, a.Y, n, 1, a.done, a.tol);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = launch_hess_cplx(n, a.Gt, a.ldg, a.po, a.swp, a.rdiag, a.Y, n, c0, cnt, a.rhs_per_shift, a.done,
                                 a.tol, st);
        if (e == cudaSuccess) {
            cj_z_kernel<<<cnt, CJT, smem, st>>>(n, a.F, a.iperm, a.scale, a.X, a.ldx, c0, a.Y, n, 1, a.done, a.tol);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// ---- residual r = b - (sigma_s x + tau_s J x), J complex; b, x, r interleaved complex ----
// Tiles of 16 rows x 8 complex right-hand sides, k in chunks of 32 through shared memory.
constexpr int RM = 16, RC = 8, RK = 32, RTT = 128;

__global__ void __launch_bounds__(RTT) cj_residual_kernel(int n, const double* __restrict__ J, int ldj,
                                                          const double* __restrict__ B, int ldb,
                                                          const double* __restrict__ X, int ldx,
                                                          double* __restrict__ R, int ldr, int nrhs,
                                                          int rhs_per_shift, const double* __restrict__ sig,
                                                          const double* __restrict__ tau,
                                                          const double* __restrict__ done, double tol)
{
    __shared__ double2 Js[RK][RM + 1];
    __shared__ double2 Xs[RK][RC + 1];
    const int i0 = blockIdx.x * RM, c0 = blockIdx.y * RC;
    if (done) {
        bool all = true;
        for (int c = c0; c < c0 + RC && c < nrhs; ++c) all = all && (done[c] <= tol);
        if (all) return;
    }
    const double2* J2 = reinterpret_cast<const double2*>(J);
    const double2* X2 = reinterpret_cast<const double2*>(X);
    const int t = threadIdx.x;
    const int r = t % RM, cq = t / RM;
    double ar = 0.0, ai = 0.0;
    for (int k0 = 0; k0 < n; k0 += RK) {
        for (int e = t; e < RM * RK; e += RTT) {
            const int ii = e % RM, kk = e / RM;
            const int i = i0 + ii, k = k0 + kk;
            Js[kk][ii] = (i < n && k < n) ? J2[(size_t)k * ldj + i] : make_double2(0.0, 0.0);
        }
        for (int e = t; e < RK * RC; e += RTT) {
            const int kk = e % RK, cc = e / RK;
            const int k = k0 + kk, c = c0 + cc;
            Xs[kk][cc] = (k < n && c < nrhs) ? X2[(size_t)c * ldx + k] : make_double2(0.0, 0.0);
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < RK; ++kk) {
            const double2 jv = Js[kk][r], xv = Xs[kk][cq];
            ar = dfma(jv.x, xv.x, ar);
            ar = dfma(-jv.y, xv.y, ar);
            ai = dfma(jv.x, xv.y, ai);
            ai = dfma(jv.y, xv.x, ai);
        }
        __syncthreads();
    }
    const int i = i0 + r, c = c0 + cq;
    if (i < n && c < nrhs) {
        const int s = c / rhs_per_shift;
        const dc sg = {sig[2 * s], sig[2 * s + 1]}, tu = {tau[2 * s], tau[2 * s + 1]};
        const double2 xw = X2[(size_t)c * ldx + i];
        const dc xv = {xw.x, xw.y};
        dc bv = {0.0, 0.0};  // no B: -W X
        if (B) {
            const double2 bw = reinterpret_cast<const double2*>(B)[(size_t)c * ldb + i];
            bv = {bw.x, bw.y};
        }
        const dc w = cadd(cmul(sg, xv), cmul(tu, dc{ar, ai}));
        reinterpret_cast<double2*>(R)[(size_t)c * ldr + i] = make_double2(bv.re - w.re, bv.im - w.im);
    }
}

cudaError_t launch_residual_cj(int n, const double* J, int ldj, const double* B, int ldb, const double* X, int ldx,
                               double* R, int ldr, int nrhs, int rhs_per_shift, const double* sig, const double* tau,
                               cudaStream_t st, const double* done, double tol)
{
    if (nrhs <= 0 || n <= 0) return cudaSuccess;
    dim3 grid((n + RM - 1) / RM, (nrhs + RC - 1) / RC);
    cj_residual_kernel<<<grid, RTT, 0, st>>>(n, J, ldj, B, ldb, X, ldx, R, ldr, nrhs, rhs_per_shift, sig, tau, done,
                                             tol);
    return cudaGetLastError();
}

}  // namespace lhl
