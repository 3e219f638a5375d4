/*
 * lhl_oracle.c -- CPU restatement of LHLFactorization.jl's hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA library and
 * the timed CPU baseline ("port") of bench.py.  Nothing in the product path links it.
 *
 * Parity status: the reference is Julia and no Julia runtime exists where this build
 * runs, so the oracle cannot be compared with the reference's own outputs.  It is pinned
 * instead by the reference's relation tests (test/core_tests.jl), ported to pytest:
 * reconstruction Z H Z^-1 = J, |l| <= 1, blocked ipiv == unblocked ipiv, solves against a
 * dense LU, the bit-exact shift-LU reference of test/core_tests.jl:119-171, refinement
 * backward errors; and by an exact-rational restatement on small integer matrices.
 *
 * Every function cites the reference lines it restates ("F:" = src/LHLFactorization.jl).
 * Index conventions follow the reference: loops are 1-based, matrices column-major, and
 * ipiv / perm / iperm hold 1-based row indices.  Floating-point operation order follows
 * the path the reference runs for Float64 on x86-64 (vector width W = 4): explicit fused
 * multiply-adds (fma()) exactly where the reference calls llvm.fmuladd, plain IEEE
 * operations everywhere else.  Build with -ffp-contract=off so the compiler adds no
 * contractions of its own.
 *
 * OpenMP is used only over independent rows, columns or shifts, so results do not depend
 * on the thread count (the reference makes the same guarantee, F:708-725).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define M1(A, ld, i, j) ((A)[(size_t)((j) - 1) * (size_t)(ld) + (size_t)((i) - 1)])

static inline void dswap(double* a, double* b) { double t = *a; *a = *b; *b = t; }

/* ------------------------------------------------------------------------------------ */
/* Balancing: Parlett-Reinsch power-of-two scaling, Gauss-Seidel over i, <= 20 sweeps.    */
/* F:299-340.                                                                              */
/* ------------------------------------------------------------------------------------ */
void lhlo_balance(int n, double* A, int ld, double* d, double* isc)
{
    for (int i = 1; i <= n; ++i) { d[i - 1] = 1.0; isc[i - 1] = 1.0; }
    for (int sweep = 0; sweep < 20; ++sweep) {
        int converged = 1;
        for (int i = 1; i <= n; ++i) {
            double c = 0.0, r = 0.0;
            for (int j = 1; j <= n; ++j) {
                if (j == i) continue;
                c += fabs(M1(A, ld, j, i));
                r += fabs(M1(A, ld, i, j));
            }
            if (c == 0.0 || r == 0.0) continue;
            double f = 1.0;
            double s = c + r;
            /* the device's bounds: never reached by finite norms (at most ~2100 steps), they end
             * the loops where the reference's would not (an infinite norm keeps c >= 2r true) */
            int guard = 0;
            while (c < r / 2.0 && guard < 4200) { c *= 2.0; r /= 2.0; f *= 2.0; ++guard; }
            while (c >= 2.0 * r && guard < 8400) { c /= 2.0; r *= 2.0; f /= 2.0; ++guard; }
            if (c + r < 0.95 * s) {
                converged = 0;
                d[i - 1] *= f;
                isc[i - 1] /= f;
                for (int j = 1; j <= n; ++j) {
                    M1(A, ld, i, j) /= f;
                    M1(A, ld, j, i) *= f;
                }
            }
        }
        if (converged) break;
    }
}

/* ------------------------------------------------------------------------------------ */
/* Unblocked ELMHES, F:466-501.  The trailing update is the reference's row-block kernel  */
/* for n >= 8 (F:547-678: per row, left update a = fma(l_i, -p_j, a), accumulator         */
/* s = fma(v_j, a, s) over j = k+2..n in order, then A[i,k+1] += s) and the generic       */
/* paired sweep below that (F:508-538).                                                    */
/* ------------------------------------------------------------------------------------ */
static void trailing_generic(int n, double* A, int ld, int k)
{
    int j = k + 2;
    while (j + 1 <= n) {
        double pj = M1(A, ld, k + 1, j), pj1 = M1(A, ld, k + 1, j + 1);
        for (int i = k + 2; i <= n; ++i) {
            double l = M1(A, ld, i, k);
            M1(A, ld, i, j) -= l * pj;
            M1(A, ld, i, j + 1) -= l * pj1;
        }
        double vj = M1(A, ld, j, k), vj1 = M1(A, ld, j + 1, k);
        for (int i = 1; i <= n; ++i)
            M1(A, ld, i, k + 1) += vj * M1(A, ld, i, j) + vj1 * M1(A, ld, i, j + 1);
        j += 2;
    }
    if (j <= n) {
        double pj = M1(A, ld, k + 1, j);
        for (int i = k + 2; i <= n; ++i) M1(A, ld, i, j) -= M1(A, ld, i, k) * pj;
        double vj = M1(A, ld, j, k);
        for (int i = 1; i <= n; ++i) M1(A, ld, i, k + 1) += vj * M1(A, ld, i, j);
    }
}

static void trailing_rowblock(int n, double* A, int ld, int k)
{
#pragma omp parallel for schedule(static) if (n >= 256)
    for (int i = 1; i <= n; ++i) {
        double s = 0.0;
        if (i >= k + 2) {
            double li = M1(A, ld, i, k);
            for (int j = k + 2; j <= n; ++j) {
                double a = fma(li, -M1(A, ld, k + 1, j), M1(A, ld, i, j));
                M1(A, ld, i, j) = a;
                s = fma(M1(A, ld, j, k), a, s);
            }
        } else {
            for (int j = k + 2; j <= n; ++j) s = fma(M1(A, ld, j, k), M1(A, ld, i, j), s);
        }
        M1(A, ld, i, k + 1) = M1(A, ld, i, k + 1) + s;
    }
}

void lhlo_reduce_unblocked(int n, double* A, int ld, int64_t* ipiv)
{
    for (int k = 1; k <= n - 2; ++k) {
        int p = k + 1;
        double amax = fabs(M1(A, ld, k + 1, k));
        for (int i = k + 2; i <= n; ++i) {
            double a = fabs(M1(A, ld, i, k));
            if (a > amax) { amax = a; p = i; }
        }
        ipiv[k - 1] = p;
        if (p != k + 1) {
            for (int j = 1; j <= n; ++j) dswap(&M1(A, ld, k + 1, j), &M1(A, ld, p, j));
            for (int i = 1; i <= n; ++i) dswap(&M1(A, ld, i, k + 1), &M1(A, ld, i, p));
        }
        double piv = M1(A, ld, k + 1, k);
        if (piv == 0.0) continue;
        for (int i = k + 2; i <= n; ++i) M1(A, ld, i, k) /= piv;
        double pk = M1(A, ld, k + 1, k + 1);
        if (pk != 0.0)
            for (int i = k + 2; i <= n; ++i) M1(A, ld, i, k + 1) -= M1(A, ld, i, k) * pk;
        if (n < 8) trailing_generic(n, A, ld, k);
        else trailing_rowblock(n, A, ld, k);
    }
}

/* ------------------------------------------------------------------------------------ */
/* Blocked (delayed-update) reduction: the reference's generic path.                      */
/* Driver F:765-783; panel steps F:787-850; interchanges F:857-890; row swap sweep        */
/* F:1336-1342; deferred swaps F:1383-1393; GEMV F:1418-1440; top GEMM F:1588-1607;       */
/* GEMM F:1676-1689; TRSM F:1917-1927.                                                     */
/* ------------------------------------------------------------------------------------ */

/* w[r0:r1] = sum_{j=c0}^{c1} A[j,k] * A[r0:r1, j], four columns per pass (F:1418-1440).  */
static void gemv_cols(double* w, const double* A, int ld, int k, int r0, int r1, int c0, int c1)
{
#pragma omp parallel for schedule(static) if (r1 - r0 >= 512)
    for (int i = r0; i <= r1; ++i) {
        double acc = 0.0;
        int j = c0;
        while (j + 3 <= c1) {
            double l1 = M1(A, ld, j, k), l2 = M1(A, ld, j + 1, k), l3 = M1(A, ld, j + 2, k),
                   l4 = M1(A, ld, j + 3, k);
            acc += (l1 * M1(A, ld, i, j) + l2 * M1(A, ld, i, j + 1)) +
                   (l3 * M1(A, ld, i, j + 2) + l4 * M1(A, ld, i, j + 3));
            j += 4;
        }
        while (j <= c1) {
            double lj = M1(A, ld, j, k);
            if (lj != 0.0) acc += lj * M1(A, ld, i, j);
            j += 1;
        }
        w[i - 1] = acc;
    }
}

/* A[i0:i1, c0:c1] += sgn * A[i0:i1, j0:j1] * A[r0:r0+K-1, cB:cB+(c1-c0)]  (F:1676-1689). */
static void gemm_generic(double* A, int ld, int i0, int i1, int j0, int j1, int r0, int cB,
                         int c0, int c1, double sgn)
{
    if (i1 < i0 || j1 < j0 || c1 < c0) return;
#pragma omp parallel for schedule(static) if ((long)(c1 - c0 + 1) * (i1 - i0 + 1) >= 65536)
    for (int c = c0; c <= c1; ++c) {
        for (int j = j0; j <= j1; ++j) {
            int jj = j - j0 + 1;
            double b = sgn * M1(A, ld, r0 + jj - 1, cB + c - c0);
            if (b == 0.0) continue;
            for (int i = i0; i <= i1; ++i) M1(A, ld, i, c) += M1(A, ld, i, j) * b;
        }
    }
}

/* F:857-890 */
static void step_swaps(int n, double* A, int ld, double* B0, int ldb, const int64_t* ipiv,
                       int k0, int kb, int k, int p)
{
    for (int j = k0; j <= kb + 1; ++j) {
        if (j == k) continue;
        dswap(&M1(A, ld, k + 1, j), &M1(A, ld, p, j));
    }
    if (p <= kb + 1) {
        for (int i = 1; i <= n; ++i) {
            dswap(&M1(A, ld, i, k + 1), &M1(A, ld, i, p));
            dswap(&M1(B0, ldb, i, k + 1 - k0), &M1(B0, ldb, i, p - k0));
        }
    } else {
        for (int i = 1; i <= n; ++i) {
            double t = M1(A, ld, i, p);
            M1(A, ld, i, p) = M1(B0, ldb, i, k + 1 - k0);
            M1(B0, ldb, i, k + 1 - k0) = t;
            M1(A, ld, i, k + 1) = t;
        }
        for (int kk = k0; kk <= k; ++kk) {
            int q = (int)ipiv[kk - 1];
            if (q != kk + 1) dswap(&M1(A, ld, kk + 1, k + 1), &M1(A, ld, q, k + 1));
        }
        for (int kk = k0; kk <= k - 1; ++kk) {
            double x = M1(A, ld, kk + 1, k + 1);
            if (x == 0.0) continue;
            for (int i = kk + 2; i <= n; ++i) M1(A, ld, i, k + 1) -= M1(A, ld, i, kk) * x;
        }
    }
}

/* F:787-850 (generic panel steps) */
static void panel_steps(int n, double* A, int ld, int64_t* ipiv, double* B0, int ldb, double* w,
                        int k0, int kb)
{
    for (int j = k0 + 1; j <= kb + 1; ++j)
        for (int i = 1; i <= n; ++i) M1(B0, ldb, i, j - k0) = M1(A, ld, i, j);
    for (int k = k0; k <= kb; ++k) {
        int p = k + 1;
        double amax = fabs(M1(A, ld, k + 1, k));
        for (int i = k + 2; i <= n; ++i) {
            double a = fabs(M1(A, ld, i, k));
            if (a > amax) { amax = a; p = i; }
        }
        ipiv[k - 1] = p;
        if (p != k + 1) {
            dswap(&M1(A, ld, k + 1, k), &M1(A, ld, p, k));
            step_swaps(n, A, ld, B0, ldb, ipiv, k0, kb, k, p);
        }
        double piv = M1(A, ld, k + 1, k);
        if (piv == 0.0) continue;
        for (int i = k + 2; i <= n; ++i) M1(A, ld, i, k) /= piv;
        for (int j = k + 1; j <= kb + 1; ++j) {
            double pj = M1(A, ld, k + 1, j);
            if (pj == 0.0) continue;
            for (int i = k + 2; i <= n; ++i) M1(A, ld, i, j) -= M1(A, ld, i, k) * pj;
        }
        for (int j = k + 2; j <= kb + 1; ++j) {
            double vj = M1(A, ld, j, k);
            if (vj == 0.0) continue;
            for (int i = k0 + 1; i <= n; ++i) M1(A, ld, i, k + 1) += vj * M1(A, ld, i, j);
        }
        if (!(kb + 2 <= n)) continue;
        gemv_cols(w, A, ld, k, k0 + 1, n, kb + 2, n);
        for (int kk = k0; kk <= k; ++kk) {
            int q = (int)ipiv[kk - 1];
            if (q != kk + 1) dswap(&w[kk], &w[q - 1]);
        }
        for (int kk = k0; kk <= k; ++kk) {
            double x = w[kk];
            if (x == 0.0) continue;
            for (int i = kk + 2; i <= n; ++i) w[i - 1] -= M1(A, ld, i, kk) * x;
        }
        for (int i = k0 + 1; i <= n; ++i) M1(A, ld, i, k + 1) += w[i - 1];
    }
}

void lhlo_reduce_blocked(int n, double* A, int ld, int64_t* ipiv, int nb)
{
    if (n < 3) return;
    int ldb = n;
    double* B0 = (double*)malloc(sizeof(double) * (size_t)n * (size_t)(nb + 1));
    double* w = (double*)malloc(sizeof(double) * (size_t)n);
    for (int k0 = 1; k0 <= n - 2; k0 += nb) {
        int kb = k0 + nb - 1 < n - 2 ? k0 + nb - 1 : n - 2;
        panel_steps(n, A, ld, ipiv, B0, ldb, w, k0, kb);
        if (kb + 2 <= n) {
            /* interchange sweep on the trailing block, F:1336-1342 */
#pragma omp parallel for schedule(static) if (n >= 512)
            for (int c = kb + 2; c <= n; ++c)
                for (int k = k0; k <= kb; ++k) {
                    int p = (int)ipiv[k - 1];
                    if (p != k + 1) dswap(&M1(A, ld, k + 1, c), &M1(A, ld, p, c));
                }
            /* small unit-lower TRSM on rows k0+1:kb+1, F:1917-1927 */
#pragma omp parallel for schedule(static) if (n >= 512)
            for (int c = kb + 2; c <= n; ++c)
                for (int k = k0; k <= kb; ++k) {
                    double x = M1(A, ld, k + 1, c);
                    if (x == 0.0) continue;
                    for (int i = k + 2; i <= kb + 1; ++i) M1(A, ld, i, c) -= M1(A, ld, i, k) * x;
                }
            /* rank-nb trailing GEMM, sign -1, F:777 */
            gemm_generic(A, ld, kb + 2, n, k0, kb, k0 + 1, kb + 2, kb + 2, n, -1.0);
        }
        /* deferred right updates of rows 1:k0 of the panel columns, F:1588-1607 */
        for (int k = k0; k <= kb; ++k)
            for (int j = k + 2; j <= kb + 1; ++j) {
                double vj = M1(A, ld, j, k);
                if (vj == 0.0) continue;
                for (int i = 1; i <= k0; ++i) M1(A, ld, i, k + 1) += vj * M1(A, ld, i, j);
            }
        for (int kk = kb + 2; kk <= n; kk += nb) {
            int ke = kk + nb - 1 < n ? kk + nb - 1 : n;
            gemm_generic(A, ld, 1, k0, kk, ke, kk, k0, k0 + 1, kb + 1, 1.0);
        }
    }
    /* interchanges deferred on the multipliers, F:1383-1393 */
    for (int k0 = 1; k0 <= n - 2; k0 += nb) {
        int kb = k0 + nb - 1 < n - 2 ? k0 + nb - 1 : n - 2;
        for (int c = k0; c <= kb; ++c)
            for (int k = kb + 1; k <= n - 2; ++k) {
                int p = (int)ipiv[k - 1];
                if (p != k + 1) dswap(&M1(A, ld, k + 1, c), &M1(A, ld, p, c));
            }
    }
    free(B0);
    free(w);
}

/* ------------------------------------------------------------------------------------ */
/* Blocked reduction, the pointer path the reference runs for Float64 (F:907-1006 and its */
/* helpers), restated per element:                                                        */
/*  - GEMV in 64-column groups (F:1451-1553): per row, the first four-column pass assigns */
/*    (l1 a1 + l2 a2) + (l3 a3 + l4 a4), later passes add it, single tail columns add    */
/*    l a (skipped when l == 0); group sums added in group order (F:1558-1583);           */
/*  - the row kernel F:1166-1296 (interchange, pulled column, panel left / right updates, */
/*    correction by the panel's interchanges and left transforms, pivot search);          */
/*  - the pulled-column tables F:1088-1132;                                                */
/*  - panel end: interchange sweep F:1344-1379, TRSM as an explicit (M^-1 - I) product    */
/*    F:1933-2001, trailing GEMM F:1860-1911 and top GEMM F:1613-1672, where every output */
/*    element is one fused multiply-add chain over K in order (F:1729-1857);              */
/*  - deferred swaps F:1395-1415.                                                           */
/* ------------------------------------------------------------------------------------ */
#define LHL_GEMV_GROUP 64

/* F:1088-1132: the pulled column p's values at rows k0+1..k+1 and at the swap partners of */
/* steps k0..k, after those interchanges and the left transforms k0..k-1 (rows <= k+1).   */
static int pulled_tables(const double* A, int ld, const double* RP, double* OV, int* OR, double* CX,
                         const int64_t* ipiv, int k0, int k, int p)
{
    int m = k - k0 + 1;
    for (int kk = k0; kk <= k; ++kk) {
        OV[kk - k0] = M1(A, ld, kk + 1, p);
        OR[kk - k0] = kk + 1;
    }
    int nov = m;
    for (int kk = k0; kk <= k; ++kk) {
        int q = (int)ipiv[kk - 1];
        if (q == kk + 1) continue;
        int s = -1;
        for (int r = 0; r < nov; ++r)
            if (OR[r] == q) { s = r; break; }
        if (s < 0) {
            s = nov++;
            OV[s] = M1(A, ld, q, p);
            OR[s] = q;
        }
        double a = OV[kk - k0];
        OV[kk - k0] = OV[s];
        OV[s] = a;
    }
    for (int kk = k0; kk <= k - 1; ++kk) {
        double x = OV[kk - k0];
        CX[kk - k0] = x;
        if (x == 0.0) continue;
        for (int i = kk + 2; i <= k + 1; ++i) {
            double aik = (i == k + 1) ? RP[kk - k0] : M1(A, ld, i, kk);
            OV[i - k0 - 1] = OV[i - k0 - 1] - aik * x;
        }
    }
    return nov;
}

/* One 64-column group's partial for rows r0..r1 (F:1496-1553).  The multipliers A[c0:c1,k] */
/* are already divided by the pivot; column psub is read from `sub`.                       */
static void gemv_group(double* out, const double* A, int ld, int k, int r0, int r1, int c0, int c1,
                       int psub, const double* sub)
{
#define COLP(j) ((j) == psub ? sub : A + (size_t)((j) - 1) * ld)
    /* per row: the same operation order as the reference's vector loop; rows run innermost */
    int j = c0;
    if (j + 3 <= c1) {
        const double *p1 = COLP(j), *p2 = COLP(j + 1), *p3 = COLP(j + 2), *p4 = COLP(j + 3);
        double l1 = M1(A, ld, j, k), l2 = M1(A, ld, j + 1, k), l3 = M1(A, ld, j + 2, k), l4 = M1(A, ld, j + 3, k);
        for (int i = r0; i <= r1; ++i)
            out[i - 1] = (l1 * p1[i - 1] + l2 * p2[i - 1]) + (l3 * p3[i - 1] + l4 * p4[i - 1]);
        j += 4;
    } else {
        const double* p1 = COLP(j);
        double lj = M1(A, ld, j, k);
        for (int i = r0; i <= r1; ++i) out[i - 1] = lj * p1[i - 1];
        j += 1;
    }
    while (j + 3 <= c1) {
        const double *p1 = COLP(j), *p2 = COLP(j + 1), *p3 = COLP(j + 2), *p4 = COLP(j + 3);
        double l1 = M1(A, ld, j, k), l2 = M1(A, ld, j + 1, k), l3 = M1(A, ld, j + 2, k), l4 = M1(A, ld, j + 3, k);
        for (int i = r0; i <= r1; ++i)
            out[i - 1] = out[i - 1] + ((l1 * p1[i - 1] + l2 * p2[i - 1]) + (l3 * p3[i - 1] + l4 * p4[i - 1]));
        j += 4;
    }
    while (j <= c1) {
        double lj = M1(A, ld, j, k);
        if (lj != 0.0) {
            const double* p1 = COLP(j);
            for (int i = r0; i <= r1; ++i) out[i - 1] = out[i - 1] + lj * p1[i - 1];
        }
        j += 1;
    }
#undef COLP
}

static void panel_steps_ptr(int n, double* A, int ld, int64_t* ipiv, double* B0, int ldb, double* w,
                            double* part, int k0, int kb, int nb)
{
    double R1[64], RP[64], PJ[64], OV[160], CX[64], LW[64], LQ[64], XS[64];
    int OR[160], LR[64];
    for (int j = k0 + 1; j <= kb + 1; ++j)
        for (int i = 1; i <= n; ++i) M1(B0, ldb, i, j - k0) = M1(A, ld, i, j);
    for (int k = k0; k <= kb; ++k) {
        int p = k + 1;
        double amax = fabs(M1(A, ld, k + 1, k));
        for (int i = k + 2; i <= n; ++i) {
            double a = fabs(M1(A, ld, i, k));
            if (a > amax) { amax = a; p = i; }
        }
        ipiv[k - 1] = p;
        for (int j = k0; j <= kb + 1; ++j) {
            R1[j - k0] = M1(A, ld, k + 1, j);
            RP[j - k0] = M1(A, ld, p, j);
        }
        if (p != k + 1) dswap(&M1(A, ld, k + 1, k), &M1(A, ld, p, k));
        double piv = M1(A, ld, k + 1, k);
        int pulled = p > kb + 1;
        if (piv == 0.0) {
            if (p != k + 1) step_swaps(n, A, ld, B0, ldb, ipiv, k0, kb, k, p);
            continue;
        }
        for (int i = k + 2; i <= kb + 1; ++i) M1(A, ld, i, k) /= piv;
        int nov = pulled ? pulled_tables(A, ld, RP, OV, OR, CX, ipiv, k0, k, p) : 0;
        for (int j = k + 1; j <= kb + 1; ++j) PJ[j - k - 1] = RP[j - k0];
        if (pulled) PJ[0] = OV[k - k0];
        else if (p != k + 1) {
            PJ[0] = RP[p - k0];
            PJ[p - k - 1] = RP[k + 1 - k0];
        }
        int trailing = kb + 2 <= n;
        if (trailing) {
            /* groups: scale their rows of the multiplier column, then their partials */
            int c0 = kb + 2, P = (n - c0 + 1 + LHL_GEMV_GROUP - 1) / LHL_GEMV_GROUP;
            const double* sub = pulled ? B0 + (size_t)(k - k0) * ldb : NULL;
            int psub = pulled ? p : 0;
#pragma omp parallel for schedule(static) if (n - k0 >= 256)
            for (int g = 1; g <= P; ++g) {
                int ga = c0 + (g - 1) * LHL_GEMV_GROUP;
                int gb = ga + LHL_GEMV_GROUP - 1 < n ? ga + LHL_GEMV_GROUP - 1 : n;
                for (int j = ga; j <= gb; ++j) M1(A, ld, j, k) = M1(A, ld, j, k) / piv;
            }
#pragma omp parallel for schedule(static) if (n - k0 >= 256)
            for (int g = 1; g <= P; ++g) {
                int ga = c0 + (g - 1) * LHL_GEMV_GROUP;
                int gb = ga + LHL_GEMV_GROUP - 1 < n ? ga + LHL_GEMV_GROUP - 1 : n;
                gemv_group(part + (size_t)(g - 1) * n, A, ld, k, k0 + 1, n, ga, gb, psub, sub);
            }
#pragma omp parallel for schedule(static) if (n - k0 >= 256)
            for (int i = k0 + 1; i <= n; ++i) {
                double s = part[i - 1];
                for (int g = 2; g <= P; ++g) s += part[(size_t)(g - 1) * n + i - 1];
                w[i - 1] = s;
            }
        }
        /* the row kernel (F:1166-1296) over rows k0+1..n */
        if (p != k + 1) {
            for (int j = k0; j <= kb + 1; ++j) {
                if (j == k) continue;
                M1(A, ld, k + 1, j) = RP[j - k0];
                M1(A, ld, p, j) = R1[j - k0];
            }
            for (int i = 1; i <= n; ++i) { /* column part of the interchange, all rows (F:1135-1161) */
                if (p <= kb + 1) {
                    dswap(&M1(A, ld, i, k + 1), &M1(A, ld, i, p));
                    dswap(&M1(B0, ldb, i, k + 1 - k0), &M1(B0, ldb, i, p - k0));
                } else {
                    double t = M1(A, ld, i, p);
                    M1(A, ld, i, p) = M1(B0, ldb, i, k + 1 - k0);
                    M1(B0, ldb, i, k + 1 - k0) = t;
                    M1(A, ld, i, k + 1) = t;
                }
            }
        }
        if (pulled) {
            for (int r = 0; r < nov; ++r) M1(A, ld, OR[r], k + 1) = OV[r];
            for (int kk = k0; kk <= k - 1; ++kk) {
                double x = CX[kk - k0];
                if (x == 0.0) continue;
                for (int i = k + 2; i <= n; ++i)
                    M1(A, ld, i, k + 1) = M1(A, ld, i, k + 1) - M1(A, ld, i, kk) * x;
            }
        }
        for (int j = k + 1; j <= kb + 1; ++j) {
            double pj = PJ[j - k - 1];
            if (pj == 0.0) continue;
            for (int i = k + 2; i <= n; ++i) M1(A, ld, i, j) = M1(A, ld, i, j) - M1(A, ld, i, k) * pj;
        }
        for (int j = k + 2; j <= kb + 1; ++j) {
            double vj = M1(A, ld, j, k);
            if (vj == 0.0) continue;
            for (int i = k0 + 1; i <= n; ++i) M1(A, ld, i, k + 1) = M1(A, ld, i, k + 1) + vj * M1(A, ld, i, j);
        }
        if (trailing) {
            int m = k - k0 + 1;
            for (int i = k0 + 1; i <= k + 1; ++i) LW[i - k0 - 1] = w[i - 1];
            int nq = 0;
            for (int kk = k0; kk <= k; ++kk) {
                int q = (int)ipiv[kk - 1];
                if (q == kk + 1) continue;
                if (q <= k + 1) {
                    double a = LW[kk - k0];
                    LW[kk - k0] = LW[q - k0 - 1];
                    LW[q - k0 - 1] = a;
                } else {
                    int s = -1;
                    for (int r = 0; r < nq; ++r)
                        if (LR[r] == q) { s = r; break; }
                    if (s < 0) { s = nq++; LQ[s] = w[q - 1]; LR[s] = q; }
                    double a = LW[kk - k0];
                    LW[kk - k0] = LQ[s];
                    LQ[s] = a;
                }
            }
            (void)m;
            for (int kk = k0; kk <= k; ++kk) {
                double x = LW[kk - k0];
                XS[kk - k0] = x;
                if (x == 0.0) continue;
                for (int i = kk + 2; i <= k; ++i) LW[i - k0 - 1] = LW[i - k0 - 1] - M1(A, ld, i, kk) * x;
                if (kk + 2 <= k + 1) LW[k - k0] = LW[k - k0] - RP[kk - k0] * x;
            }
            for (int i = k0 + 1; i <= k + 1; ++i) {
                double v = LW[i - k0 - 1];
                w[i - 1] = v;
                M1(A, ld, i, k + 1) = M1(A, ld, i, k + 1) + v;
            }
            for (int r = 0; r < nq; ++r) w[LR[r] - 1] = LQ[r];
            for (int kk = k0; kk <= k; ++kk) {
                double x = XS[kk - k0];
                if (x == 0.0) continue;
                for (int i = k + 2; i <= n; ++i) w[i - 1] = w[i - 1] - M1(A, ld, i, kk) * x;
            }
            for (int i = k + 2; i <= n; ++i) M1(A, ld, i, k + 1) = M1(A, ld, i, k + 1) + w[i - 1];
        }
    }
    (void)nb;
}

void lhlo_reduce_blocked_ptr(int n, double* A, int ld, int64_t* ipiv, int nb)
{
    if (n < 3) return;
    int ldb = n;
    double* B0 = (double*)malloc(sizeof(double) * (size_t)n * (size_t)(nb + 1));
    double* w = (double*)malloc(sizeof(double) * (size_t)n);
    int Pmax = (n + LHL_GEMV_GROUP - 1) / LHL_GEMV_GROUP;
    double* part = (double*)malloc(sizeof(double) * (size_t)n * (size_t)Pmax);
    double* Pm = (double*)malloc(sizeof(double) * (size_t)nb * (size_t)nb);
    double* Tsnap = (double*)malloc(sizeof(double) * (size_t)n * (size_t)(nb + 1));
    for (int k0 = 1; k0 <= n - 2; k0 += nb) {
        int kb = k0 + nb - 1 < n - 2 ? k0 + nb - 1 : n - 2;
        panel_steps_ptr(n, A, ld, ipiv, B0, ldb, w, part, k0, kb, nb);
        if (kb + 2 <= n) {
            int nbp = kb - k0 + 1;
            /* P = M^-1 - I, M[r,s] = A[k0+r, k0+s-1] for r > s (F:1944-1955) */
            for (int q = 1; q <= nbp; ++q) {
                for (int r = 1; r <= q; ++r) Pm[(r - 1) + (size_t)(q - 1) * nbp] = 0.0;
                for (int r = q + 1; r <= nbp; ++r) {
                    double acc = -M1(A, ld, k0 + r, k0 + q - 1);
                    for (int s = q + 1; s <= r - 1; ++s)
                        acc = acc - M1(A, ld, k0 + r, k0 + s - 1) * Pm[(s - 1) + (size_t)(q - 1) * nbp];
                    Pm[(r - 1) + (size_t)(q - 1) * nbp] = acc;
                }
            }
#pragma omp parallel for schedule(static) if (n >= 512)
            for (int c = kb + 2; c <= n; ++c) {
                double Bs[64];
                for (int k = k0; k <= kb; ++k) {
                    int p = (int)ipiv[k - 1];
                    if (p != k + 1) dswap(&M1(A, ld, k + 1, c), &M1(A, ld, p, c));
                }
                if (nbp >= 2) {
                    for (int s = 1; s <= nbp; ++s) Bs[s - 1] = M1(A, ld, k0 + s, c);
                    for (int r = 1; r <= nbp; ++r) {
                        double v = M1(A, ld, k0 + r, c);
                        for (int s = 1; s <= nbp; ++s) v = fma(Pm[(r - 1) + (size_t)(s - 1) * nbp], Bs[s - 1], v);
                        M1(A, ld, k0 + r, c) = v;
                    }
                }
                for (int i = kb + 2; i <= n; ++i) {
                    double v = M1(A, ld, i, c);
                    for (int kk = 1; kk <= nbp; ++kk)
                        v = fma(-M1(A, ld, i, k0 + kk - 1), M1(A, ld, k0 + kk, c), v);
                    M1(A, ld, i, c) = v;
                }
            }
        }
        /* top rows 1..k0 of the panel columns: panel part (plain), then one fma chain over
         * j = kb+2..n per element (F:1635-1672); rows run innermost, same per-element order */
        {
            int ncp = kb - k0 + 1;
            double* pre = Tsnap; /* k0 x ncp snapshot of the panel columns' top rows */
            for (int c = k0 + 1; c <= kb + 1; ++c)
                for (int i = 1; i <= k0; ++i) pre[(size_t)(c - k0 - 1) * k0 + i - 1] = M1(A, ld, i, c);
#pragma omp parallel for schedule(dynamic, 1) if (k0 >= 128)
            for (int c = k0 + 1; c <= kb + 1; ++c) {
                double* v = A + (size_t)(c - 1) * ld;
                for (int j = c + 1; j <= kb + 1; ++j) {
                    double vj = M1(A, ld, j, c - 1);
                    if (vj == 0.0) continue;
                    const double* pj = pre + (size_t)(j - k0 - 1) * k0;
                    for (int i = 1; i <= k0; ++i) v[i - 1] = v[i - 1] + vj * pj[i - 1];
                }
                for (int j = kb + 2; j <= n; ++j) {
                    double b = M1(A, ld, j, c - 1);
                    const double* aj = A + (size_t)(j - 1) * ld;
                    for (int i = 1; i <= k0; ++i) v[i - 1] = fma(aj[i - 1], b, v[i - 1]);
                }
            }
            (void)ncp;
        }
    }
    for (int k0 = 1; k0 <= n - 2; k0 += nb) {
        int kb = k0 + nb - 1 < n - 2 ? k0 + nb - 1 : n - 2;
        for (int c = k0; c <= kb; ++c)
            for (int k = kb + 1; k <= n - 2; ++k) {
                int p = (int)ipiv[k - 1];
                if (p != k + 1) dswap(&M1(A, ld, k + 1, c), &M1(A, ld, p, c));
            }
    }
    free(B0); free(w); free(part); free(Pm); free(Tsnap);
}

/* ------------------------------------------------------------------------------------ */
/* lhl_reduce! driver, F:355-405 (balance, path choice at n >= 500 for Float64, Ht fill   */
/* F:2024-2039, perm / iperm F:376-387).  path: 0 = the reference's choice, 1 = unblocked,  */
/* 2 = blocked.  F receives the n x n factors (leading dimension ldf), Ht n x n with      */
/* Ht[j,i] = H[i,j] for i <= j+1 and zero elsewhere.                                       */
/* ------------------------------------------------------------------------------------ */
int lhlo_reduce(int n, const double* J, int ldj, int balance, int path, int nb, double* F, int ldf,
                int64_t* ipiv, double* scale, double* iscale, int64_t* perm, int64_t* iperm, double* Ht)
{
    if (n < 0 || ldj < n || ldf < n) return -1;
    for (int j = 1; j <= n; ++j)
        for (int i = 1; i <= n; ++i) M1(F, ldf, i, j) = M1(J, ldj, i, j);
    if (balance) lhlo_balance(n, F, ldf, scale, iscale);
    else for (int i = 0; i < n; ++i) { scale[i] = 1.0; iscale[i] = 1.0; }
    /* path: 0 = the reference's choice (pointer blocked path at n >= 500, F:398-402),
     * 1 = unblocked, 2 = generic blocked, 3 = pointer blocked */
    if (nb <= 0 || nb > 48) nb = 16;
    if (path == 0) path = n >= 500 ? 3 : 1;
    if (path == 3) lhlo_reduce_blocked_ptr(n, F, ldf, ipiv, nb);
    else if (path == 2) lhlo_reduce_blocked(n, F, ldf, ipiv, nb);
    else lhlo_reduce_unblocked(n, F, ldf, ipiv);
    if (Ht) {
        memset(Ht, 0, sizeof(double) * (size_t)n * (size_t)n);
        for (int i = 1; i <= n; ++i)
            for (int j = (i - 1 > 1 ? i - 1 : 1); j <= n; ++j) M1(Ht, n, j, i) = M1(F, ldf, i, j);
    }
    for (int i = 1; i <= n; ++i) perm[i - 1] = i;
    for (int k = 1; k <= n - 2; ++k) {
        int64_t p = ipiv[k - 1];
        int64_t t = perm[k]; perm[k] = perm[p - 1]; perm[p - 1] = t;
    }
    for (int i = 1; i <= n; ++i) iperm[perm[i - 1] - 1] = i;
    return 0;
}

/* ------------------------------------------------------------------------------------ */
/* Shift LU of G = sigma I + tau H (real), F:2529-2594 == test/core_tests.jl:119-171.     */
/* Gt is (ldg x n), column k holds row k of U (Gt[j,k] = U[k,j], j >= k); Gt[k,k+1] holds */
/* the multiplier l_k.  Returns info (first zero pivot, 0 if none).                        */
/* ------------------------------------------------------------------------------------ */
int lhlo_shift(int n, const double* Ht, int ldh, double sigma, double tau, double* Gt, int ldg,
               uint8_t* swp, double* rdiag, double* r /* work, n */)
{
    if (n == 0) return 0;
    for (int j = 1; j <= n; ++j) r[j - 1] = tau * M1(Ht, ldh, j, 1);
    r[0] = r[0] + sigma;
    int info = 0;
    for (int k = 1; k <= n - 1; ++k) {
        double a = r[k - 1];
        double b = tau * M1(Ht, ldh, k, k + 1);
        if (fabs(b) > fabs(a)) {
            swp[k - 1] = 1;
            M1(Gt, ldg, k, k) = b;
            double l = a / b;
            M1(Gt, ldg, k, k + 1) = l;
            for (int j = k + 1; j <= n; ++j) {
                double g = tau * M1(Ht, ldh, j, k + 1);
                M1(Gt, ldg, j, k) = g;
                r[j - 1] = r[j - 1] - l * g;
            }
            M1(Gt, ldg, k + 1, k) = M1(Gt, ldg, k + 1, k) + sigma;
            r[k] = r[k] - l * sigma;
        } else {
            swp[k - 1] = 0;
            M1(Gt, ldg, k, k) = a;
            double l;
            if (a == 0.0) { if (info == 0) info = k; l = 0.0; }
            else l = b / a;
            M1(Gt, ldg, k, k + 1) = l;
            for (int j = k + 1; j <= n; ++j) {
                double rj = r[j - 1];
                M1(Gt, ldg, j, k) = rj;
                r[j - 1] = tau * M1(Ht, ldh, j, k + 1) - l * rj;
            }
            r[k] = r[k] + sigma;
        }
    }
    double rn = r[n - 1];
    M1(Gt, ldg, n, n) = rn;
    swp[n - 1] = 0;
    if (rn == 0.0 && info == 0) info = n;
    for (int j = 1; j <= n; ++j) rdiag[j - 1] = 1.0 / M1(Gt, ldg, j, j);
    return info;
}

/* ------------------------------------------------------------------------------------ */
/* lhl_reduce! for LHLWorkspace{Float32} below _lhl_block_min(Float32) = 1024 (F:703-705): */
/* balancing (F:299-340 with Tr = Float32: sums, halvings and Tr(0.95) in float, scale in  */
/* float) and the unblocked ELMHES (F:466-501) with the Float32 trailing update: the row-  */
/* block kernel for n >= max(W, 8) = 8 (F:547-552, W = 32 / 4 = 8 on x86-64, F:1713), whose */
/* per-row order does not depend on W (each lane is one row), and the paired sweep below.  */
/* J is rounded to float first (copyto! into the Float32 fstore).  The outputs are float   */
/* values in double storage.  From n = 1024 the blocked Float32 form (lhlo_reduce_blocked_  */
/* ptr_f32, below).                                                                        */
/* ------------------------------------------------------------------------------------ */
#define M1F(A, ld, i, j) ((A)[(size_t)((j) - 1) * (size_t)(ld) + (size_t)((i) - 1)])

static void balance_f32(int n, float* A, int ld, float* d, float* isc)
{
    for (int i = 1; i <= n; ++i) { d[i - 1] = 1.0f; isc[i - 1] = 1.0f; }
    for (int sweep = 0; sweep < 20; ++sweep) {
        int converged = 1;
        for (int i = 1; i <= n; ++i) {
            float c = 0.0f, r = 0.0f;
            for (int j = 1; j <= n; ++j) {
                if (j == i) continue;
                c += fabsf(M1F(A, ld, j, i));
                r += fabsf(M1F(A, ld, i, j));
            }
            if (c == 0.0f || r == 0.0f) continue;
            float f = 1.0f;
            float s = c + r;
            int guard = 0;  /* the device's bounds, as in lhlo_balance */
            while (c < r / 2.0f && guard < 4200) { c *= 2.0f; r /= 2.0f; f *= 2.0f; ++guard; }
            while (c >= 2.0f * r && guard < 8400) { c /= 2.0f; r *= 2.0f; f /= 2.0f; ++guard; }
            if (c + r < 0.95f * s) {
                converged = 0;
                d[i - 1] *= f;
                isc[i - 1] /= f;
                for (int j = 1; j <= n; ++j) {
                    M1F(A, ld, i, j) /= f;
                    M1F(A, ld, j, i) *= f;
                }
            }
        }
        if (converged) break;
    }
}

static void reduce_unblocked_f32(int n, float* A, int ld, int64_t* ipiv)
{
    for (int k = 1; k <= n - 2; ++k) {
        int p = k + 1;
        float amax = fabsf(M1F(A, ld, k + 1, k));
        for (int i = k + 2; i <= n; ++i) {
            float a = fabsf(M1F(A, ld, i, k));
            if (a > amax) { amax = a; p = i; }
        }
        ipiv[k - 1] = p;
        if (p != k + 1) {
            for (int j = 1; j <= n; ++j) {
                float t = M1F(A, ld, k + 1, j); M1F(A, ld, k + 1, j) = M1F(A, ld, p, j); M1F(A, ld, p, j) = t;
            }
            for (int i = 1; i <= n; ++i) {
                float t = M1F(A, ld, i, k + 1); M1F(A, ld, i, k + 1) = M1F(A, ld, i, p); M1F(A, ld, i, p) = t;
            }
        }
        float piv = M1F(A, ld, k + 1, k);
        if (piv == 0.0f) continue;
        for (int i = k + 2; i <= n; ++i) M1F(A, ld, i, k) /= piv;
        float pk = M1F(A, ld, k + 1, k + 1);
        if (pk != 0.0f)
            for (int i = k + 2; i <= n; ++i) M1F(A, ld, i, k + 1) -= M1F(A, ld, i, k) * pk;
        if (n < 8) {  /* F:508-538 */
            int j = k + 2;
            while (j + 1 <= n) {
                float pj = M1F(A, ld, k + 1, j), pj1 = M1F(A, ld, k + 1, j + 1);
                for (int i = k + 2; i <= n; ++i) {
                    float l = M1F(A, ld, i, k);
                    M1F(A, ld, i, j) -= l * pj;
                    M1F(A, ld, i, j + 1) -= l * pj1;
                }
                float vj = M1F(A, ld, j, k), vj1 = M1F(A, ld, j + 1, k);
                for (int i = 1; i <= n; ++i)
                    M1F(A, ld, i, k + 1) += vj * M1F(A, ld, i, j) + vj1 * M1F(A, ld, i, j + 1);
                j += 2;
            }
            if (j <= n) {
                float pj = M1F(A, ld, k + 1, j);
                for (int i = k + 2; i <= n; ++i) M1F(A, ld, i, j) -= M1F(A, ld, i, k) * pj;
                float vj = M1F(A, ld, j, k);
                for (int i = 1; i <= n; ++i) M1F(A, ld, i, k + 1) += vj * M1F(A, ld, i, j);
            }
        } else {  /* F:547-678, per row */
#pragma omp parallel for schedule(static) if (n >= 256)
            for (int i = 1; i <= n; ++i) {
                float s = 0.0f;
                if (i >= k + 2) {
                    float li = M1F(A, ld, i, k);
                    for (int j = k + 2; j <= n; ++j) {
                        float a = fmaf(li, -M1F(A, ld, k + 1, j), M1F(A, ld, i, j));
                        M1F(A, ld, i, j) = a;
                        s = fmaf(M1F(A, ld, j, k), a, s);
                    }
                } else {
                    for (int j = k + 2; j <= n; ++j) s = fmaf(M1F(A, ld, j, k), M1F(A, ld, i, j), s);
                }
                M1F(A, ld, i, k + 1) = M1F(A, ld, i, k + 1) + s;
            }
        }
    }
}

/* The reference's blocked Float32 form (n >= _lhl_block_min(Float32) = 1024): the pointer
 * path of F:765-1006 and its helpers with T = Float32.  Its vector width W = 8 only spreads
 * rows over lanes; every element sees the Float64 path's operations in the same order (the
 * GEMV's 64-column groups and four-column passes, the group sums in order, the fused
 * multiply-add chains of the TRSM, the trailing GEMM and the top GEMM), so this is
 * lhlo_reduce_blocked_ptr above with float arithmetic (fmaf where that one calls fma). */
static inline void fswap(float* a, float* b) { float t = *a; *a = *b; *b = t; }

static void step_swaps_f32(int n, float* A, int ld, float* B0, int ldb, const int64_t* ipiv,
                       int k0, int kb, int k, int p)
{
    for (int j = k0; j <= kb + 1; ++j) {
        if (j == k) continue;
        fswap(&M1(A, ld, k + 1, j), &M1(A, ld, p, j));
    }
    if (p <= kb + 1) {
        for (int i = 1; i <= n; ++i) {
            fswap(&M1(A, ld, i, k + 1), &M1(A, ld, i, p));
            fswap(&M1(B0, ldb, i, k + 1 - k0), &M1(B0, ldb, i, p - k0));
        }
    } else {
        for (int i = 1; i <= n; ++i) {
            float t = M1(A, ld, i, p);
            M1(A, ld, i, p) = M1(B0, ldb, i, k + 1 - k0);
            M1(B0, ldb, i, k + 1 - k0) = t;
            M1(A, ld, i, k + 1) = t;
        }
        for (int kk = k0; kk <= k; ++kk) {
            int q = (int)ipiv[kk - 1];
            if (q != kk + 1) fswap(&M1(A, ld, kk + 1, k + 1), &M1(A, ld, q, k + 1));
        }
        for (int kk = k0; kk <= k - 1; ++kk) {
            float x = M1(A, ld, kk + 1, k + 1);
            if (x == 0.0f) continue;
            for (int i = kk + 2; i <= n; ++i) M1(A, ld, i, k + 1) -= M1(A, ld, i, kk) * x;
        }
    }
}

/* F:1088-1132: the pulled column p's values at rows k0+1..k+1 and at the swap partners of */
/* steps k0..k, after those interchanges and the left transforms k0..k-1 (rows <= k+1).   */
static int pulled_tables_f32(const float* A, int ld, const float* RP, float* OV, int* OR, float* CX,
                         const int64_t* ipiv, int k0, int k, int p)
{
    int m = k - k0 + 1;
    for (int kk = k0; kk <= k; ++kk) {
        OV[kk - k0] = M1(A, ld, kk + 1, p);
        OR[kk - k0] = kk + 1;
    }
    int nov = m;
    for (int kk = k0; kk <= k; ++kk) {
        int q = (int)ipiv[kk - 1];
        if (q == kk + 1) continue;
        int s = -1;
        for (int r = 0; r < nov; ++r)
            if (OR[r] == q) { s = r; break; }
        if (s < 0) {
            s = nov++;
            OV[s] = M1(A, ld, q, p);
            OR[s] = q;
        }
        float a = OV[kk - k0];
        OV[kk - k0] = OV[s];
        OV[s] = a;
    }
    for (int kk = k0; kk <= k - 1; ++kk) {
        float x = OV[kk - k0];
        CX[kk - k0] = x;
        if (x == 0.0f) continue;
        for (int i = kk + 2; i <= k + 1; ++i) {
            float aik = (i == k + 1) ? RP[kk - k0] : M1(A, ld, i, kk);
            OV[i - k0 - 1] = OV[i - k0 - 1] - aik * x;
        }
    }
    return nov;
}

/* One 64-column group's partial for rows r0..r1 (F:1496-1553).  The multipliers A[c0:c1,k] */
/* are already divided by the pivot; column psub is read from `sub`.                       */
static void gemv_group_f32(float* out, const float* A, int ld, int k, int r0, int r1, int c0, int c1,
                       int psub, const float* sub)
{
#define COLP(j) ((j) == psub ? sub : A + (size_t)((j) - 1) * ld)
    /* per row: the same operation order as the reference's vector loop; rows run innermost */
    int j = c0;
    if (j + 3 <= c1) {
        const float *p1 = COLP(j), *p2 = COLP(j + 1), *p3 = COLP(j + 2), *p4 = COLP(j + 3);
        float l1 = M1(A, ld, j, k), l2 = M1(A, ld, j + 1, k), l3 = M1(A, ld, j + 2, k), l4 = M1(A, ld, j + 3, k);
        for (int i = r0; i <= r1; ++i)
            out[i - 1] = (l1 * p1[i - 1] + l2 * p2[i - 1]) + (l3 * p3[i - 1] + l4 * p4[i - 1]);
        j += 4;
    } else {
        const float* p1 = COLP(j);
        float lj = M1(A, ld, j, k);
        for (int i = r0; i <= r1; ++i) out[i - 1] = lj * p1[i - 1];
        j += 1;
    }
    while (j + 3 <= c1) {
        const float *p1 = COLP(j), *p2 = COLP(j + 1), *p3 = COLP(j + 2), *p4 = COLP(j + 3);
        float l1 = M1(A, ld, j, k), l2 = M1(A, ld, j + 1, k), l3 = M1(A, ld, j + 2, k), l4 = M1(A, ld, j + 3, k);
        for (int i = r0; i <= r1; ++i)
            out[i - 1] = out[i - 1] + ((l1 * p1[i - 1] + l2 * p2[i - 1]) + (l3 * p3[i - 1] + l4 * p4[i - 1]));
        j += 4;
    }
    while (j <= c1) {
        float lj = M1(A, ld, j, k);
        if (lj != 0.0f) {
            const float* p1 = COLP(j);
            for (int i = r0; i <= r1; ++i) out[i - 1] = out[i - 1] + lj * p1[i - 1];
        }
        j += 1;
    }
#undef COLP
}

static void panel_steps_ptr_f32(int n, float* A, int ld, int64_t* ipiv, float* B0, int ldb, float* w,
                            float* part, int k0, int kb, int nb)
{
    float R1[64], RP[64], PJ[64], OV[160], CX[64], LW[64], LQ[64], XS[64];
    int OR[160], LR[64];
    for (int j = k0 + 1; j <= kb + 1; ++j)
        for (int i = 1; i <= n; ++i) M1(B0, ldb, i, j - k0) = M1(A, ld, i, j);
    for (int k = k0; k <= kb; ++k) {
        int p = k + 1;
        float amax = fabsf(M1(A, ld, k + 1, k));
        for (int i = k + 2; i <= n; ++i) {
            float a = fabsf(M1(A, ld, i, k));
            if (a > amax) { amax = a; p = i; }
        }
        ipiv[k - 1] = p;
        for (int j = k0; j <= kb + 1; ++j) {
            R1[j - k0] = M1(A, ld, k + 1, j);
            RP[j - k0] = M1(A, ld, p, j);
        }
        if (p != k + 1) fswap(&M1(A, ld, k + 1, k), &M1(A, ld, p, k));
        float piv = M1(A, ld, k + 1, k);
        int pulled = p > kb + 1;
        if (piv == 0.0f) {
            if (p != k + 1) step_swaps_f32(n, A, ld, B0, ldb, ipiv, k0, kb, k, p);
            continue;
        }
        for (int i = k + 2; i <= kb + 1; ++i) M1(A, ld, i, k) /= piv;
        int nov = pulled ? pulled_tables_f32(A, ld, RP, OV, OR, CX, ipiv, k0, k, p) : 0;
        for (int j = k + 1; j <= kb + 1; ++j) PJ[j - k - 1] = RP[j - k0];
        if (pulled) PJ[0] = OV[k - k0];
        else if (p != k + 1) {
            PJ[0] = RP[p - k0];
            PJ[p - k - 1] = RP[k + 1 - k0];
        }
        int trailing = kb + 2 <= n;
        if (trailing) {
            /* groups: scale their rows of the multiplier column, then their partials */
            int c0 = kb + 2, P = (n - c0 + 1 + LHL_GEMV_GROUP - 1) / LHL_GEMV_GROUP;
            const float* sub = pulled ? B0 + (size_t)(k - k0) * ldb : NULL;
            int psub = pulled ? p : 0;
#pragma omp parallel for schedule(static) if (n - k0 >= 256)
            for (int g = 1; g <= P; ++g) {
                int ga = c0 + (g - 1) * LHL_GEMV_GROUP;
                int gb = ga + LHL_GEMV_GROUP - 1 < n ? ga + LHL_GEMV_GROUP - 1 : n;
                for (int j = ga; j <= gb; ++j) M1(A, ld, j, k) = M1(A, ld, j, k) / piv;
            }
#pragma omp parallel for schedule(static) if (n - k0 >= 256)
            for (int g = 1; g <= P; ++g) {
                int ga = c0 + (g - 1) * LHL_GEMV_GROUP;
                int gb = ga + LHL_GEMV_GROUP - 1 < n ? ga + LHL_GEMV_GROUP - 1 : n;
                gemv_group_f32(part + (size_t)(g - 1) * n, A, ld, k, k0 + 1, n, ga, gb, psub, sub);
            }
#pragma omp parallel for schedule(static) if (n - k0 >= 256)
            for (int i = k0 + 1; i <= n; ++i) {
                float s = part[i - 1];
                for (int g = 2; g <= P; ++g) s += part[(size_t)(g - 1) * n + i - 1];
                w[i - 1] = s;
            }
        }
        /* the row kernel (F:1166-1296) over rows k0+1..n */
        if (p != k + 1) {
            for (int j = k0; j <= kb + 1; ++j) {
                if (j == k) continue;
                M1(A, ld, k + 1, j) = RP[j - k0];
                M1(A, ld, p, j) = R1[j - k0];
            }
            for (int i = 1; i <= n; ++i) { /* column part of the interchange, all rows (F:1135-1161) */
                if (p <= kb + 1) {
                    fswap(&M1(A, ld, i, k + 1), &M1(A, ld, i, p));
                    fswap(&M1(B0, ldb, i, k + 1 - k0), &M1(B0, ldb, i, p - k0));
                } else {
                    float t = M1(A, ld, i, p);
                    M1(A, ld, i, p) = M1(B0, ldb, i, k + 1 - k0);
                    M1(B0, ldb, i, k + 1 - k0) = t;
                    M1(A, ld, i, k + 1) = t;
                }
            }
        }
        if (pulled) {
            for (int r = 0; r < nov; ++r) M1(A, ld, OR[r], k + 1) = OV[r];
            for (int kk = k0; kk <= k - 1; ++kk) {
                float x = CX[kk - k0];
                if (x == 0.0f) continue;
                for (int i = k + 2; i <= n; ++i)
                    M1(A, ld, i, k + 1) = M1(A, ld, i, k + 1) - M1(A, ld, i, kk) * x;
            }
        }
        for (int j = k + 1; j <= kb + 1; ++j) {
            float pj = PJ[j - k - 1];
            if (pj == 0.0f) continue;
            for (int i = k + 2; i <= n; ++i) M1(A, ld, i, j) = M1(A, ld, i, j) - M1(A, ld, i, k) * pj;
        }
        for (int j = k + 2; j <= kb + 1; ++j) {
            float vj = M1(A, ld, j, k);
            if (vj == 0.0f) continue;
            for (int i = k0 + 1; i <= n; ++i) M1(A, ld, i, k + 1) = M1(A, ld, i, k + 1) + vj * M1(A, ld, i, j);
        }
        if (trailing) {
            int m = k - k0 + 1;
            for (int i = k0 + 1; i <= k + 1; ++i) LW[i - k0 - 1] = w[i - 1];
            int nq = 0;
            for (int kk = k0; kk <= k; ++kk) {
                int q = (int)ipiv[kk - 1];
                if (q == kk + 1) continue;
                if (q <= k + 1) {
                    float a = LW[kk - k0];
                    LW[kk - k0] = LW[q - k0 - 1];
                    LW[q - k0 - 1] = a;
                } else {
                    int s = -1;
                    for (int r = 0; r < nq; ++r)
                        if (LR[r] == q) { s = r; break; }
                    if (s < 0) { s = nq++; LQ[s] = w[q - 1]; LR[s] = q; }
                    float a = LW[kk - k0];
                    LW[kk - k0] = LQ[s];
                    LQ[s] = a;
                }
            }
            (void)m;
            for (int kk = k0; kk <= k; ++kk) {
                float x = LW[kk - k0];
                XS[kk - k0] = x;
                if (x == 0.0f) continue;
                for (int i = kk + 2; i <= k; ++i) LW[i - k0 - 1] = LW[i - k0 - 1] - M1(A, ld, i, kk) * x;
                if (kk + 2 <= k + 1) LW[k - k0] = LW[k - k0] - RP[kk - k0] * x;
            }
            for (int i = k0 + 1; i <= k + 1; ++i) {
                float v = LW[i - k0 - 1];
                w[i - 1] = v;
                M1(A, ld, i, k + 1) = M1(A, ld, i, k + 1) + v;
            }
            for (int r = 0; r < nq; ++r) w[LR[r] - 1] = LQ[r];
            for (int kk = k0; kk <= k; ++kk) {
                float x = XS[kk - k0];
                if (x == 0.0f) continue;
                for (int i = k + 2; i <= n; ++i) w[i - 1] = w[i - 1] - M1(A, ld, i, kk) * x;
            }
            for (int i = k + 2; i <= n; ++i) M1(A, ld, i, k + 1) = M1(A, ld, i, k + 1) + w[i - 1];
        }
    }
    (void)nb;
}

void lhlo_reduce_blocked_ptr_f32(int n, float* A, int ld, int64_t* ipiv, int nb)
{
    if (n < 3) return;
    int ldb = n;
    float* B0 = (float*)malloc(sizeof(float) * (size_t)n * (size_t)(nb + 1));
    float* w = (float*)malloc(sizeof(float) * (size_t)n);
    int Pmax = (n + LHL_GEMV_GROUP - 1) / LHL_GEMV_GROUP;
    float* part = (float*)malloc(sizeof(float) * (size_t)n * (size_t)Pmax);
    float* Pm = (float*)malloc(sizeof(float) * (size_t)nb * (size_t)nb);
    float* Tsnap = (float*)malloc(sizeof(float) * (size_t)n * (size_t)(nb + 1));
    for (int k0 = 1; k0 <= n - 2; k0 += nb) {
        int kb = k0 + nb - 1 < n - 2 ? k0 + nb - 1 : n - 2;
        panel_steps_ptr_f32(n, A, ld, ipiv, B0, ldb, w, part, k0, kb, nb);
        if (kb + 2 <= n) {
            int nbp = kb - k0 + 1;
            /* P = M^-1 - I, M[r,s] = A[k0+r, k0+s-1] for r > s (F:1944-1955) */
            for (int q = 1; q <= nbp; ++q) {
                for (int r = 1; r <= q; ++r) Pm[(r - 1) + (size_t)(q - 1) * nbp] = 0.0f;
                for (int r = q + 1; r <= nbp; ++r) {
                    float acc = -M1(A, ld, k0 + r, k0 + q - 1);
                    for (int s = q + 1; s <= r - 1; ++s)
                        acc = acc - M1(A, ld, k0 + r, k0 + s - 1) * Pm[(s - 1) + (size_t)(q - 1) * nbp];
                    Pm[(r - 1) + (size_t)(q - 1) * nbp] = acc;
                }
            }
#pragma omp parallel for schedule(static) if (n >= 512)
            for (int c = kb + 2; c <= n; ++c) {
                float Bs[64];
                for (int k = k0; k <= kb; ++k) {
                    int p = (int)ipiv[k - 1];
                    if (p != k + 1) fswap(&M1(A, ld, k + 1, c), &M1(A, ld, p, c));
                }
                if (nbp >= 2) {
                    for (int s = 1; s <= nbp; ++s) Bs[s - 1] = M1(A, ld, k0 + s, c);
                    for (int r = 1; r <= nbp; ++r) {
                        float v = M1(A, ld, k0 + r, c);
                        for (int s = 1; s <= nbp; ++s) v = fmaf(Pm[(r - 1) + (size_t)(s - 1) * nbp], Bs[s - 1], v);
                        M1(A, ld, k0 + r, c) = v;
                    }
                }
                for (int i = kb + 2; i <= n; ++i) {
                    float v = M1(A, ld, i, c);
                    for (int kk = 1; kk <= nbp; ++kk)
                        v = fmaf(-M1(A, ld, i, k0 + kk - 1), M1(A, ld, k0 + kk, c), v);
                    M1(A, ld, i, c) = v;
                }
            }
        }
        /* top rows 1..k0 of the panel columns: panel part (plain), then one fma chain over
         * j = kb+2..n per element (F:1635-1672); rows run innermost, same per-element order */
        {
            int ncp = kb - k0 + 1;
            float* pre = Tsnap; /* k0 x ncp snapshot of the panel columns' top rows */
            for (int c = k0 + 1; c <= kb + 1; ++c)
                for (int i = 1; i <= k0; ++i) pre[(size_t)(c - k0 - 1) * k0 + i - 1] = M1(A, ld, i, c);
#pragma omp parallel for schedule(dynamic, 1) if (k0 >= 128)
            for (int c = k0 + 1; c <= kb + 1; ++c) {
                float* v = A + (size_t)(c - 1) * ld;
                for (int j = c + 1; j <= kb + 1; ++j) {
                    float vj = M1(A, ld, j, c - 1);
                    if (vj == 0.0f) continue;
                    const float* pj = pre + (size_t)(j - k0 - 1) * k0;
                    for (int i = 1; i <= k0; ++i) v[i - 1] = v[i - 1] + vj * pj[i - 1];
                }
                for (int j = kb + 2; j <= n; ++j) {
                    float b = M1(A, ld, j, c - 1);
                    const float* aj = A + (size_t)(j - 1) * ld;
                    for (int i = 1; i <= k0; ++i) v[i - 1] = fmaf(aj[i - 1], b, v[i - 1]);
                }
            }
            (void)ncp;
        }
    }
    for (int k0 = 1; k0 <= n - 2; k0 += nb) {
        int kb = k0 + nb - 1 < n - 2 ? k0 + nb - 1 : n - 2;
        for (int c = k0; c <= kb; ++c)
            for (int k = kb + 1; k <= n - 2; ++k) {
                int p = (int)ipiv[k - 1];
                if (p != k + 1) fswap(&M1(A, ld, k + 1, c), &M1(A, ld, p, c));
            }
    }
    free(B0); free(w); free(part); free(Pm); free(Tsnap);
}


/* The blocked Float32 form on its own (no balancing), at any n: A (float values in double
 * storage) is reduced in place; for the relation tests of test/threading.jl:58-79. */
int lhlo_reduce_blocked_ptr_f32_raw(int n, double* A, int ld, int64_t* ipiv)
{
    if (n < 0 || ld < n) return -1;
    float* Af = (float*)malloc(sizeof(float) * ((size_t)n * (size_t)n + 1));
    if (!Af) return -3;
    for (int j = 1; j <= n; ++j)
        for (int i = 1; i <= n; ++i) M1F(Af, n, i, j) = (float)M1(A, ld, i, j);
    lhlo_reduce_blocked_ptr_f32(n, Af, n, ipiv, 16);
    for (int j = 1; j <= n; ++j)
        for (int i = 1; i <= n; ++i) M1(A, ld, i, j) = M1F(Af, n, i, j);
    free(Af);
    return 0;
}

int lhlo_reduce_f32(int n, const double* J, int ldj, int balance, double* F, int ldf, int64_t* ipiv, double* scale,
                    double* iscale, int64_t* perm, int64_t* iperm, double* Ht)
{
    if (n < 0 || ldj < n || ldf < n) return -1;
    float* A = (float*)malloc(sizeof(float) * ((size_t)n * (size_t)n + 2 * (size_t)n + 1));
    if (!A) return -3;
    float* d = A + (size_t)n * (size_t)n;
    float* isc = d + n;
    for (int j = 1; j <= n; ++j)
        for (int i = 1; i <= n; ++i) M1F(A, n, i, j) = (float)M1(J, ldj, i, j);
    if (balance) balance_f32(n, A, n, d, isc);
    else for (int i = 0; i < n; ++i) { d[i] = 1.0f; isc[i] = 1.0f; }
    if (n >= 1024) lhlo_reduce_blocked_ptr_f32(n, A, n, ipiv, 16);
    else reduce_unblocked_f32(n, A, n, ipiv);
    for (int j = 1; j <= n; ++j)
        for (int i = 1; i <= n; ++i) M1(F, ldf, i, j) = M1F(A, n, i, j);
    for (int i = 0; i < n; ++i) { scale[i] = d[i]; iscale[i] = isc[i]; }
    free(A);
    if (Ht) {
        memset(Ht, 0, sizeof(double) * (size_t)n * (size_t)n);
        for (int i = 1; i <= n; ++i)
            for (int j = (i - 1 > 1 ? i - 1 : 1); j <= n; ++j) M1(Ht, n, j, i) = M1(F, ldf, i, j);
    }
    for (int i = 1; i <= n; ++i) perm[i - 1] = i;
    for (int k = 1; k <= n - 2; ++k) {
        int64_t p = ipiv[k - 1];
        int64_t t = perm[k]; perm[k] = perm[p - 1]; perm[p - 1] = t;
    }
    for (int i = 1; i <= n; ++i) iperm[perm[i - 1] - 1] = i;
    return 0;
}

/* lhl_shift! for LHLWorkspace{Float32} (F:2529-2594 with T = Float32): the same steps in
 * float arithmetic, sigma and tau rounded to float first (T(sigma), T(tau)).  Ht holds float
 * values in double storage; Gt and rdiag receive float values in double storage. */
int lhlo_shift_f32(int n, const double* Ht, int ldh, double sigma_d, double tau_d, double* Gt, int ldg,
                   uint8_t* swp, double* rdiag, double* rw /* work, n */)
{
    if (n == 0) return 0;
    const float sigma = (float)sigma_d, tau = (float)tau_d;
    float* r = (float*)rw;
    for (int j = 1; j <= n; ++j) r[j - 1] = tau * (float)M1(Ht, ldh, j, 1);
    r[0] = r[0] + sigma;
    int info = 0;
    for (int k = 1; k <= n - 1; ++k) {
        float a = r[k - 1];
        float b = tau * (float)M1(Ht, ldh, k, k + 1);
        if (fabsf(b) > fabsf(a)) {
            swp[k - 1] = 1;
            M1(Gt, ldg, k, k) = b;
            float l = a / b;
            M1(Gt, ldg, k, k + 1) = l;
            for (int j = k + 1; j <= n; ++j) {
                float g = tau * (float)M1(Ht, ldh, j, k + 1);
                M1(Gt, ldg, j, k) = g;
                r[j - 1] = r[j - 1] - l * g;
            }
            M1(Gt, ldg, k + 1, k) = (float)M1(Gt, ldg, k + 1, k) + sigma;
            r[k] = r[k] - l * sigma;
        } else {
            swp[k - 1] = 0;
            M1(Gt, ldg, k, k) = a;
            float l;
            if (a == 0.0f) { if (info == 0) info = k; l = 0.0f; }
            else l = b / a;
            M1(Gt, ldg, k, k + 1) = l;
            for (int j = k + 1; j <= n; ++j) {
                float rj = r[j - 1];
                M1(Gt, ldg, j, k) = rj;
                r[j - 1] = tau * (float)M1(Ht, ldh, j, k + 1) - l * rj;
            }
            r[k] = r[k] + sigma;
        }
    }
    float rn = r[n - 1];
    M1(Gt, ldg, n, n) = rn;
    swp[n - 1] = 0;
    if (rn == 0.0f && info == 0) info = n;
    for (int j = 1; j <= n; ++j) rdiag[j - 1] = 1.0f / (float)M1(Gt, ldg, j, j);
    return info;
}

/* ------------------------------------------------------------------------------------ */
/* Solves.  L (the multipliers) is read from the factors F: L[i,k] = F[i,k], i >= k+2.    */
/* Sweeps follow the Float64 padded-buffer kernels (F:2265-2434: fused multiply-adds in a */
/* group of four steps, head triangle first); the Hessenberg solve follows F:2967-3039.  */
/* ------------------------------------------------------------------------------------ */
static void zinvsweep(int n, const double* F, int ldf, double* y)
{
    int G = (n - 2 > 0 ? n - 2 : 0) >> 2;
    for (int g = 1; g <= G; ++g) {
        int k = 4 * g - 3;
        double x1 = y[k];
        double x2 = fma(-M1(F, ldf, k + 2, k), x1, y[k + 1]);
        y[k + 1] = x2;
        double x3 = fma(-M1(F, ldf, k + 3, k + 1), x2, fma(-M1(F, ldf, k + 3, k), x1, y[k + 2]));
        y[k + 2] = x3;
        double x4 = fma(-M1(F, ldf, k + 4, k + 2), x3,
                        fma(-M1(F, ldf, k + 4, k + 1), x2, fma(-M1(F, ldf, k + 4, k), x1, y[k + 3])));
        y[k + 3] = x4;
        for (int i = k + 5; i <= n; ++i) {
            double v = y[i - 1];
            v = fma(M1(F, ldf, i, k), -x1, v);
            v = fma(M1(F, ldf, i, k + 1), -x2, v);
            v = fma(M1(F, ldf, i, k + 2), -x3, v);
            v = fma(M1(F, ldf, i, k + 3), -x4, v);
            y[i - 1] = v;
        }
    }
    for (int k = 4 * G + 1; k <= n - 2; ++k) {
        double b = -y[k];
        for (int i = k + 2; i <= n; ++i) y[i - 1] = fma(M1(F, ldf, i, k), b, y[i - 1]);
    }
}

static void zsweep(int n, const double* F, int ldf, double* y)
{
    int G = (n - 2 > 0 ? n - 2 : 0) >> 2;
    for (int k = n - 2; k >= 4 * G + 1; --k) {
        double b = y[k];
        for (int i = k + 2; i <= n; ++i) y[i - 1] = fma(M1(F, ldf, i, k), b, y[i - 1]);
    }
    for (int g = G; g >= 1; --g) {
        int k = 4 * g - 3;
        double x1 = y[k], x2 = y[k + 1], x3 = y[k + 2], x4 = y[k + 3];
        y[k + 1] = fma(M1(F, ldf, k + 2, k), x1, x2);
        y[k + 2] = fma(M1(F, ldf, k + 3, k + 1), x2, fma(M1(F, ldf, k + 3, k), x1, x3));
        y[k + 3] = fma(M1(F, ldf, k + 4, k + 2), x3,
                       fma(M1(F, ldf, k + 4, k + 1), x2, fma(M1(F, ldf, k + 4, k), x1, x4)));
        for (int i = k + 5; i <= n; ++i) {
            double v = y[i - 1];
            v = fma(M1(F, ldf, i, k), x1, v);
            v = fma(M1(F, ldf, i, k + 1), x2, v);
            v = fma(M1(F, ldf, i, k + 2), x3, v);
            v = fma(M1(F, ldf, i, k + 3), x4, v);
            y[i - 1] = v;
        }
    }
}

/* Forward 2x2 select-swap steps F:2806-2816, then the four-row pipelined back substitution
 * F:2967-3039 with four-lane vector accumulators (lane = (i - j - 1) mod 4) summed in
 * lane order. */
static void hess_solve(int n, const double* Gt, int ldg, const uint8_t* swp, const double* rd, double* y)
{
    for (int k = 1; k <= n - 1; ++k) {
        int s = swp[k - 1];
        double a = y[k - 1], b = y[k];
        double xk = s ? b : a;
        y[k - 1] = xk;
        y[k] = (s ? a : b) - M1(Gt, ldg, k, k + 1) * xk;
    }
#define G1(i, j) M1(Gt, ldg, i, j)
    int j = n;
    double s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
    while (j - 3 >= 1) {
        double xj = (y[j - 1] - s1) * rd[j - 1];
        y[j - 1] = xj;
        s2 = fma(G1(j, j - 1), xj, s2);
        s3 = fma(G1(j, j - 2), xj, s3);
        s4 = fma(G1(j, j - 3), xj, s4);
        double xj1 = (y[j - 2] - s2) * rd[j - 2];
        y[j - 2] = xj1;
        s3 = fma(G1(j - 1, j - 2), xj1, s3);
        s4 = fma(G1(j - 1, j - 3), xj1, s4);
        double xj2 = (y[j - 3] - s3) * rd[j - 3];
        y[j - 3] = xj2;
        s4 = fma(G1(j - 2, j - 3), xj2, s4);
        double xj3 = (y[j - 4] - s4) * rd[j - 4];
        y[j - 4] = xj3;
        int jn = j - 4;
        if (jn - 3 >= 1) {
            double a[4][4] = {{0}};
            for (int i = j + 1; i <= n; ++i) {
                int lane = (i - j - 1) & 3;
                double v = y[i - 1];
                a[0][lane] = fma(G1(i, jn), v, a[0][lane]);
                a[1][lane] = fma(G1(i, jn - 1), v, a[1][lane]);
                a[2][lane] = fma(G1(i, jn - 2), v, a[2][lane]);
                a[3][lane] = fma(G1(i, jn - 3), v, a[3][lane]);
            }
            double t[4];
            for (int c = 0; c < 4; ++c) t[c] = ((a[c][0] + a[c][1]) + a[c][2]) + a[c][3];
            s1 = t[0] + ((G1(j, jn) * xj + G1(j - 1, jn) * xj1) + (G1(j - 2, jn) * xj2 + G1(j - 3, jn) * xj3));
            s2 = t[1] + ((G1(j, jn - 1) * xj + G1(j - 1, jn - 1) * xj1) +
                         (G1(j - 2, jn - 1) * xj2 + G1(j - 3, jn - 1) * xj3));
            s3 = t[2] + ((G1(j, jn - 2) * xj + G1(j - 1, jn - 2) * xj1) +
                         (G1(j - 2, jn - 2) * xj2 + G1(j - 3, jn - 2) * xj3));
            s4 = t[3] + ((G1(j, jn - 3) * xj + G1(j - 1, jn - 3) * xj1) +
                         (G1(j - 2, jn - 3) * xj2 + G1(j - 3, jn - 3) * xj3));
        }
        j = jn;
    }
    while (j >= 1) {
        double s = 0.0;
        for (int i = j + 1; i <= n; ++i) s += G1(i, j) * y[i - 1];
        y[j - 1] = (y[j - 1] - s) * rd[j - 1];
        j -= 1;
    }
#undef G1
}

/* lhl_ldiv! for a real shift, F:3052-3068: gather, L^-1 sweep, Hessenberg solve, L sweep,
 * scatter.  y is a work vector of length n. */
void lhlo_ldiv(int n, const double* F, int ldf, const int64_t* perm, const int64_t* iperm,
               const double* scale, const double* iscale, const double* Gt, int ldg,
               const uint8_t* swp, const double* rdiag, double* x, double* y)
{
    for (int i = 1; i <= n; ++i) {
        int64_t p = perm[i - 1];
        y[i - 1] = x[p - 1] * iscale[p - 1];
    }
    zinvsweep(n, F, ldf, y);
    hess_solve(n, Gt, ldg, swp, rdiag, y);
    zsweep(n, F, ldf, y);
    for (int i = 1; i <= n; ++i) x[i - 1] = y[iperm[i - 1] - 1] * scale[i - 1];
}

/* x <- Z x and x <- Z^-1 x (F:2069-2126), real vectors. */
void lhlo_applyZ(int n, const double* F, int ldf, const int64_t* iperm, const double* scale,
                 double* x, double* y)
{
    for (int i = 0; i < n; ++i) y[i] = x[i];
    zsweep(n, F, ldf, y);
    for (int i = 1; i <= n; ++i) x[i - 1] = y[iperm[i - 1] - 1] * scale[i - 1];
}

void lhlo_applyZinv(int n, const double* F, int ldf, const int64_t* perm, const double* iscale,
                    double* x, double* y)
{
    for (int i = 1; i <= n; ++i) {
        int64_t p = perm[i - 1];
        y[i - 1] = x[p - 1] * iscale[p - 1];
    }
    zinvsweep(n, F, ldf, y);
    for (int i = 0; i < n; ++i) x[i] = y[i];
}

/* lhl_refine!, F:3144-3157, with A = sigma I + tau J applied as r = sigma x + tau (J x):
 * r = b - A x; ldiv(r); x += r; `steps` times. */
void lhlo_refine(int n, const double* J, int ldj, double sigma, double tau, const double* b,
                 const double* F, int ldf, const int64_t* perm, const int64_t* iperm,
                 const double* scale, const double* iscale, const double* Gt, int ldg,
                 const uint8_t* swp, const double* rdiag, double* x, int steps, double* r, double* y)
{
    for (int s = 0; s < steps; ++s) {
        for (int i = 0; i < n; ++i) r[i] = 0.0;
        for (int j = 1; j <= n; ++j) {
            double xj = x[j - 1];
            for (int i = 1; i <= n; ++i) r[i - 1] += M1(J, ldj, i, j) * xj;
        }
        for (int i = 0; i < n; ++i) r[i] = b[i] - (sigma * x[i] + tau * r[i]);
        lhlo_ldiv(n, F, ldf, perm, iperm, scale, iscale, Gt, ldg, swp, rdiag, r, y);
        for (int i = 0; i < n; ++i) x[i] += r[i];
    }
}

/* ------------------------------------------------------------------------------------ */
/* Batched driver used as the timed CPU baseline: S shifts, one RHS each, shift LU +      */
/* ldiv + `steps` refinement steps per shift; shifts run in parallel (independent).       */
/* ------------------------------------------------------------------------------------ */
int lhlo_shift_solve_batch(int n, const double* J, int ldj, const double* Ht, const double* F, int ldf,
                           const int64_t* perm, const int64_t* iperm, const double* scale,
                           const double* iscale, int S, const double* sigma, const double* tau,
                           const double* B, double* X, int steps, int* info_out)
{
    int ldg = n + 4;
    int bad = 0;
#pragma omp parallel reduction(| : bad)
    {
        double* Gt = (double*)calloc((size_t)ldg * (size_t)n, sizeof(double));
        double* rd = (double*)malloc(sizeof(double) * (size_t)n);
        uint8_t* sw = (uint8_t*)malloc((size_t)n);
        double* w = (double*)malloc(sizeof(double) * (size_t)n * 3);
        if (!Gt || !rd || !sw || !w) bad = 1;
        else {
#pragma omp for schedule(dynamic, 1)
            for (int s = 0; s < S; ++s) {
                int info = lhlo_shift(n, Ht, n, sigma[s], tau[s], Gt, ldg, sw, rd, w);
                info_out[s] = info;
                double* x = X + (size_t)s * n;
                for (int i = 0; i < n; ++i) x[i] = B[(size_t)s * n + i];
                lhlo_ldiv(n, F, ldf, perm, iperm, scale, iscale, Gt, ldg, sw, rd, x, w);
                if (steps > 0)
                    lhlo_refine(n, J, ldj, sigma[s], tau[s], B + (size_t)s * n, F, ldf, perm, iperm, scale,
                                iscale, Gt, ldg, sw, rd, x, steps, w + n, w + 2 * (size_t)n);
            }
        }
        free(Gt); free(rd); free(sw); free(w);
    }
    return bad ? -1 : 0;
}

int lhlo_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------------------ */
/* Complex shifts on a real reduction (LHLShift{ComplexF64} on LHLWorkspace{Float64}).    */
/* Shift LU: F:2529-2594 with TG = ComplexF64 (every complex product written out as        */
/* Julia's Complex arithmetic: (ac - bd, ad + bc); complex x real scales both parts; the    */
/* pivot magnitude is |re| + |im|, F:2519-2520).  Gt is planar: real parts in rows          */
/* 1..n, imaginary parts in rows po+1..po+n of each column (F:117-129).  Division is the    */
/* robust complex division of Baudin & Smith (2012), which Julia's Base uses for            */
/* ComplexF64 (the reference calls `/` and `inv`, F:2548, F:2555, F:2590); rdiag =         */
/* 1 / U[j,j] by the same division.  The planar solve is F:2146-2156 (gather into planes),  */
/* the real L sweeps on each plane, F:2823-2910 (planar Hessenberg solve, here without the  */
/* 4-row pipelining of its back substitution: the same sums in plain order), scatter.      */
/* ------------------------------------------------------------------------------------ */
typedef struct { double re, im; } cplx;

static cplx c_mul(cplx a, cplx b) { cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static cplx c_sub(cplx a, cplx b) { cplx r = {a.re - b.re, a.im - b.im}; return r; }
static cplx c_add(cplx a, cplx b) { cplx r = {a.re + b.re, a.im + b.im}; return r; }
static cplx c_scale(cplx a, double s) { cplx r = {a.re * s, a.im * s}; return r; }
static double c_mag(cplx a) { return fabs(a.re) + fabs(a.im); }

/* Baudin & Smith, "A robust complex division in Scilab" (2012), without its rescaling of  */
/* operands near overflow/underflow (not reached by the tested inputs).                     */
static double cdiv2(double a, double b, double c, double d, double r, double t)
{
    if (r != 0.0) {
        double br = b * r;
        return br != 0.0 ? (a + br) * t : a * t + (b * t) * r;
    }
    return (a + d * (b / c)) * t;
}
static cplx c_div(cplx x, cplx y)
{
    double a = x.re, b = x.im, c = y.re, d = y.im;
    cplx q;
    if (fabs(d) <= fabs(c)) {
        double r = d / c, t = 1.0 / (c + d * r);
        q.re = cdiv2(a, b, c, d, r, t);
        q.im = cdiv2(b, -a, c, d, r, t);
    } else {
        double r = c / d, t = 1.0 / (d + c * r);
        q.re = cdiv2(b, a, d, c, r, t);
        q.im = -cdiv2(a, -b, d, c, r, t);
    }
    return q;
}

#define CG(G, ldg, po, i, c) ((cplx){M1(G, ldg, i, c), M1(G, ldg, (po) + (i), c)})
#define CSET(G, ldg, po, i, c, v) do { cplx v_ = (v); M1(G, ldg, i, c) = v_.re; M1(G, ldg, (po) + (i), c) = v_.im; } while (0)

int lhlo_shift_complex(int n, const double* Ht, int ldh, double sr, double si, double tr, double ti, double* Gt,
                       int ldg, int po, uint8_t* swp, double* rdiag /* 2n interleaved */, double* rw /* 2n */)
{
    if (n == 0) return 0;
    cplx sigma = {sr, si}, tau = {tr, ti};
    cplx* r = (cplx*)rw;
    for (int j = 1; j <= n; ++j) r[j - 1] = c_scale(tau, M1(Ht, ldh, j, 1));
    r[0] = c_add(r[0], sigma);
    int info = 0;
    for (int k = 1; k <= n - 1; ++k) {
        cplx a = r[k - 1];
        cplx b = c_scale(tau, M1(Ht, ldh, k, k + 1));
        if (c_mag(b) > c_mag(a)) {
            swp[k - 1] = 1;
            CSET(Gt, ldg, po, k, k, b);
            cplx l = c_div(a, b);
            CSET(Gt, ldg, po, k, k + 1, l);
            for (int j = k + 1; j <= n; ++j) {
                cplx g = c_scale(tau, M1(Ht, ldh, j, k + 1));
                CSET(Gt, ldg, po, j, k, g);
                r[j - 1] = c_sub(r[j - 1], c_mul(l, g));
            }
            CSET(Gt, ldg, po, k + 1, k, c_add(CG(Gt, ldg, po, k + 1, k), sigma));
            r[k] = c_sub(r[k], c_mul(l, sigma));
        } else {
            swp[k - 1] = 0;
            CSET(Gt, ldg, po, k, k, a);
            cplx l;
            if (a.re == 0.0 && a.im == 0.0) { if (info == 0) info = k; l.re = 0.0; l.im = 0.0; }
            else l = c_div(b, a);
            CSET(Gt, ldg, po, k, k + 1, l);
            for (int j = k + 1; j <= n; ++j) {
                cplx rj = r[j - 1];
                CSET(Gt, ldg, po, j, k, rj);
                r[j - 1] = c_sub(c_scale(tau, M1(Ht, ldh, j, k + 1)), c_mul(l, rj));
            }
            r[k] = c_add(r[k], sigma);
        }
    }
    cplx rn = r[n - 1];
    CSET(Gt, ldg, po, n, n, rn);
    swp[n - 1] = 0;
    if (rn.re == 0.0 && rn.im == 0.0 && info == 0) info = n;
    cplx one = {1.0, 0.0};
    for (int j = 1; j <= n; ++j) {
        cplx q = c_div(one, CG(Gt, ldg, po, j, j));
        rdiag[2 * (j - 1)] = q.re;
        rdiag[2 * (j - 1) + 1] = q.im;
    }
    return info;
}

/* planar Hessenberg solve, F:2823-2910 (y: re plane y[0..n-1], im plane y[po..po+n-1]) */
static void hess_solve_planar(int n, const double* Gt, int ldg, int po, const uint8_t* swp, const double* rd,
                              double* y)
{
    for (int k = 1; k <= n - 1; ++k) {
        int s = swp[k - 1];
        cplx a = {y[k - 1], y[po + k - 1]}, b = {y[k], y[po + k]};
        cplx xk = s ? b : a;
        y[k - 1] = xk.re;
        y[po + k - 1] = xk.im;
        cplx v = c_sub(s ? a : b, c_mul(CG(Gt, ldg, po, k, k + 1), xk));
        y[k] = v.re;
        y[po + k] = v.im;
    }
    for (int j = n; j >= 1; --j) {
        double sr = 0.0, si = 0.0;
        for (int i = j + 1; i <= n; ++i) {
            double xr = y[i - 1], xi = y[po + i - 1];
            double gr = M1(Gt, ldg, i, j), gi = M1(Gt, ldg, po + i, j);
            sr += gr * xr - gi * xi;
            si += gr * xi + gi * xr;
        }
        cplx rj = {rd[2 * (j - 1)], rd[2 * (j - 1) + 1]};
        cplx xj = c_mul(c_sub((cplx){y[j - 1], y[po + j - 1]}, (cplx){sr, si}), rj);
        y[j - 1] = xj.re;
        y[po + j - 1] = xj.im;
    }
}

/* lhl_ldiv!(x, sh::LHLShift{ComplexF64}, ws::LHLWorkspace{Float64}), F:3080-3110.          */
/* x: n complex (interleaved); y: 2 po doubles of scratch.                                  */
void lhlo_ldiv_complex(int n, const double* F, int ldf, const int64_t* perm, const int64_t* iperm,
                       const double* scale, const double* iscale, const double* Gt, int ldg, int po,
                       const uint8_t* swp, const double* rdiag, double* x, double* y)
{
    for (int i = 1; i <= n; ++i) {
        int64_t p = perm[i - 1];
        y[i - 1] = x[2 * (p - 1)] * iscale[p - 1];
        y[po + i - 1] = x[2 * (p - 1) + 1] * iscale[p - 1];
    }
    zinvsweep(n, F, ldf, y);
    zinvsweep(n, F, ldf, y + po);
    hess_solve_planar(n, Gt, ldg, po, swp, rdiag, y);
    zsweep(n, F, ldf, y);
    zsweep(n, F, ldf, y + po);
    for (int i = 1; i <= n; ++i) {
        int64_t p = iperm[i - 1];
        x[2 * (i - 1)] = y[p - 1] * scale[i - 1];
        x[2 * (i - 1) + 1] = y[po + p - 1] * scale[i - 1];
    }
}

/* ------------------------------------------------------------------------------------ */
/* A complex J (LHLWorkspace{ComplexF64}).  J, F and Ht are interleaved complex (re, im    */
/* pairs), column-major.  The reference runs the generic Julia code with T = ComplexF64:    */
/* balancing F:299-340 and the pivot search F:470-477 on abs(z) = hypot(re, im); the        */
/* unblocked ELMHES F:466-501 with the generic paired sweep F:508-538 (the SIMD variants are */
/* Float32/Float64 only, F:547); below _lhl_block_min(ComplexF64) = 768 (F:703-705) that is  */
/* the reference's own path, at and above it the reference's blocked form has the same       */
/* pivots and factors equal to rounding (test/threading.jl:58-79).  Solves: applyZinv!      */
/* (gather, generic L^-1 sweep F:2151-2195), planar Hessenberg solve (F:2823-2910), applyZ! */
/* (generic L sweep F:2199-2243, scatter), as lhl_ldiv! does for a complex workspace         */
/* (F:3111-3121).                                                                            */
/* ------------------------------------------------------------------------------------ */
#define CM1(A, ld, i, j) (((cplx*)(A))[(size_t)((j) - 1) * (size_t)(ld) + (size_t)((i) - 1)])

/* |z| = hypot(re, im).  Borges, "An improved algorithm for hypot(a, b)" (arXiv:1904.09481,  */
/* 2019): sqrt of a fused x^2 + y^2 and one fused correction step, operands first scaled by  */
/* a power of two when very large or very small.  The device library computes the same      */
/* steps (IEEE sqrt and division, exact fma), so the two agree bit for bit.                  */
static double c_abs(cplx z)
{
    double ax = fabs(z.re), ay = fabs(z.im);
    if (isinf(ax) || isinf(ay)) return INFINITY;
    if (isnan(ax) || isnan(ay)) return ax + ay;
    double x = fmax(ax, ay), y = fmin(ax, ay);
    if (y == 0.0) return x;
    double s = 1.0;
    if (x > 0x1p+500) { x *= 0x1p-600; y *= 0x1p-600; s = 0x1p+600; }
    else if (x < 0x1p-500) { x *= 0x1p+600; y *= 0x1p+600; s = 0x1p-600; }
    double h = sqrt(fma(x, x, y * y));
    double h2 = h * h, x2 = x * x;
    double c = (fma(-y, y, h2 - x2) + fma(h, h, -h2)) - fma(x, x, -x2);
    h = h - c / (2.0 * h);
    return h * s;
}

double lhlo_cabs(double re, double im) { cplx z = {re, im}; return c_abs(z); }

static int c_iszero(cplx a) { return a.re == 0.0 && a.im == 0.0; }
static void cswap(cplx* a, cplx* b) { cplx t = *a; *a = *b; *b = t; }

/* F:299-340 with T = ComplexF64: the norms sum abs(z), the factors are real powers of two. */
static void cbalance(int n, double* A, int ld, double* d, double* isc)
{
    for (int i = 1; i <= n; ++i) { d[i - 1] = 1.0; isc[i - 1] = 1.0; }
    for (int sweep = 0; sweep < 20; ++sweep) {
        int converged = 1;
        for (int i = 1; i <= n; ++i) {
            double c = 0.0, r = 0.0;
            for (int j = 1; j <= n; ++j) {
                if (j == i) continue;
                c += c_abs(CM1(A, ld, j, i));
                r += c_abs(CM1(A, ld, i, j));
            }
            if (c == 0.0 || r == 0.0) continue;
            double f = 1.0;
            double s = c + r;
            int guard = 0;  /* the device's bounds (see lhlo_balance) */
            while (c < r / 2.0 && guard < 4200) { c *= 2.0; r /= 2.0; f *= 2.0; ++guard; }
            while (c >= 2.0 * r && guard < 8400) { c /= 2.0; r *= 2.0; f /= 2.0; ++guard; }
            if (c + r < 0.95 * s) {
                converged = 0;
                d[i - 1] *= f;
                isc[i - 1] /= f;
                for (int j = 1; j <= n; ++j) {
                    CM1(A, ld, i, j).re /= f;
                    CM1(A, ld, i, j).im /= f;
                    CM1(A, ld, j, i).re *= f;
                    CM1(A, ld, j, i).im *= f;
                }
            }
        }
        if (converged) break;
    }
}

/* F:466-501 and the generic paired sweep F:508-538, T = ComplexF64. */
static void creduce_unblocked(int n, double* A, int ld, int64_t* ipiv)
{
    for (int k = 1; k <= n - 2; ++k) {
        int p = k + 1;
        double amax = c_abs(CM1(A, ld, k + 1, k));
        for (int i = k + 2; i <= n; ++i) {
            double a = c_abs(CM1(A, ld, i, k));
            if (a > amax) { amax = a; p = i; }
        }
        ipiv[k - 1] = p;
        if (p != k + 1) {
            for (int j = 1; j <= n; ++j) cswap(&CM1(A, ld, k + 1, j), &CM1(A, ld, p, j));
            for (int i = 1; i <= n; ++i) cswap(&CM1(A, ld, i, k + 1), &CM1(A, ld, i, p));
        }
        cplx piv = CM1(A, ld, k + 1, k);
        if (c_iszero(piv)) continue;
        for (int i = k + 2; i <= n; ++i) CM1(A, ld, i, k) = c_div(CM1(A, ld, i, k), piv);
        cplx pk = CM1(A, ld, k + 1, k + 1);
        if (!c_iszero(pk))
            for (int i = k + 2; i <= n; ++i) CM1(A, ld, i, k + 1) = c_sub(CM1(A, ld, i, k + 1), c_mul(CM1(A, ld, i, k), pk));
        int j = k + 2;
        while (j + 1 <= n) {
            cplx pj = CM1(A, ld, k + 1, j), pj1 = CM1(A, ld, k + 1, j + 1);
            for (int i = k + 2; i <= n; ++i) {
                cplx l = CM1(A, ld, i, k);
                CM1(A, ld, i, j) = c_sub(CM1(A, ld, i, j), c_mul(l, pj));
                CM1(A, ld, i, j + 1) = c_sub(CM1(A, ld, i, j + 1), c_mul(l, pj1));
            }
            cplx vj = CM1(A, ld, j, k), vj1 = CM1(A, ld, j + 1, k);
            for (int i = 1; i <= n; ++i)
                CM1(A, ld, i, k + 1) = c_add(CM1(A, ld, i, k + 1),
                                             c_add(c_mul(vj, CM1(A, ld, i, j)), c_mul(vj1, CM1(A, ld, i, j + 1))));
            j += 2;
        }
        if (j <= n) {
            cplx pj = CM1(A, ld, k + 1, j);
            for (int i = k + 2; i <= n; ++i) CM1(A, ld, i, j) = c_sub(CM1(A, ld, i, j), c_mul(CM1(A, ld, i, k), pj));
            cplx vj = CM1(A, ld, j, k);
            for (int i = 1; i <= n; ++i) CM1(A, ld, i, k + 1) = c_add(CM1(A, ld, i, k + 1), c_mul(vj, CM1(A, ld, i, j)));
        }
    }
}

/* ------------------------------------------------------------------------------------ */
/* Blocked reduction for a complex J: the generic path the reference takes for ComplexF64  */
/* at n >= 768 (F:398-399, F:705), restated with Julia's Complex arithmetic (products      */
/* (ac - bd, ad + bc), no fused operations, robust division, pivot on the modulus):        */
/* driver F:765-783; panel steps F:787-850; interchanges F:857-890; row swap sweep        */
/* F:1336-1342; GEMV F:1418-1440; TRSM F:1917-1927; GEMM F:1676-1689 (b = sgn * B          */
/* element, sgn = -one(T) = (-1, -0) or one(T) = (1, 0)); top GEMM F:1588-1607 with its    */
/* fix-up F:1598-1606; deferred swaps F:1383-1393.                                         */
/* ------------------------------------------------------------------------------------ */

/* w[r0:r1] = sum_{j=c0}^{c1} A[j,k] * A[r0:r1, j] from w = 0, four columns per pass.      */
static void cgemv_cols(cplx* w, const double* A, int ld, int k, int r0, int r1, int c0, int c1)
{
#pragma omp parallel for schedule(static) if (r1 - r0 >= 512)
    for (int i = r0; i <= r1; ++i) {
        cplx acc = {0.0, 0.0};
        int j = c0;
        while (j + 3 <= c1) {
            cplx l1 = CM1(A, ld, j, k), l2 = CM1(A, ld, j + 1, k), l3 = CM1(A, ld, j + 2, k),
                 l4 = CM1(A, ld, j + 3, k);
            acc = c_add(acc, c_add(c_add(c_mul(l1, CM1(A, ld, i, j)), c_mul(l2, CM1(A, ld, i, j + 1))),
                                   c_add(c_mul(l3, CM1(A, ld, i, j + 2)), c_mul(l4, CM1(A, ld, i, j + 3)))));
            j += 4;
        }
        while (j <= c1) {
            cplx lj = CM1(A, ld, j, k);
            if (!c_iszero(lj)) acc = c_add(acc, c_mul(lj, CM1(A, ld, i, j)));
            j += 1;
        }
        w[i - 1] = acc;
    }
}

/* A[i0:i1, c0:c1] += A[i0:i1, j0:j1] * (sgn * A[r0:r0+K-1, cB:cB+(c1-c0)]). */
static void cgemm_generic(double* A, int ld, int i0, int i1, int j0, int j1, int r0, int cB, int c0, int c1,
                          cplx sgn)
{
    if (i1 < i0 || j1 < j0 || c1 < c0) return;
#pragma omp parallel for schedule(static) if ((long)(c1 - c0 + 1) * (i1 - i0 + 1) >= 65536)
    for (int c = c0; c <= c1; ++c) {
        for (int j = j0; j <= j1; ++j) {
            int jj = j - j0 + 1;
            cplx b = c_mul(sgn, CM1(A, ld, r0 + jj - 1, cB + c - c0));
            if (c_iszero(b)) continue;
            for (int i = i0; i <= i1; ++i) CM1(A, ld, i, c) = c_add(CM1(A, ld, i, c), c_mul(CM1(A, ld, i, j), b));
        }
    }
}

static void cstep_swaps(int n, double* A, int ld, double* B0, int ldb, const int64_t* ipiv, int k0, int kb, int k,
                        int p)
{
    for (int j = k0; j <= kb + 1; ++j) {
        if (j == k) continue;
        cswap(&CM1(A, ld, k + 1, j), &CM1(A, ld, p, j));
    }
    if (p <= kb + 1) {
        for (int i = 1; i <= n; ++i) {
            cswap(&CM1(A, ld, i, k + 1), &CM1(A, ld, i, p));
            cswap(&CM1(B0, ldb, i, k + 1 - k0), &CM1(B0, ldb, i, p - k0));
        }
    } else {
        for (int i = 1; i <= n; ++i) {
            cplx t = CM1(A, ld, i, p);
            CM1(A, ld, i, p) = CM1(B0, ldb, i, k + 1 - k0);
            CM1(B0, ldb, i, k + 1 - k0) = t;
            CM1(A, ld, i, k + 1) = t;
        }
        for (int kk = k0; kk <= k; ++kk) {
            int q = (int)ipiv[kk - 1];
            if (q != kk + 1) cswap(&CM1(A, ld, kk + 1, k + 1), &CM1(A, ld, q, k + 1));
        }
        for (int kk = k0; kk <= k - 1; ++kk) {
            cplx x = CM1(A, ld, kk + 1, k + 1);
            if (c_iszero(x)) continue;
            for (int i = kk + 2; i <= n; ++i)
                CM1(A, ld, i, k + 1) = c_sub(CM1(A, ld, i, k + 1), c_mul(CM1(A, ld, i, kk), x));
        }
    }
}

static void cpanel_steps(int n, double* A, int ld, int64_t* ipiv, double* B0, int ldb, cplx* w, int k0, int kb)
{
    for (int j = k0 + 1; j <= kb + 1; ++j)
        for (int i = 1; i <= n; ++i) CM1(B0, ldb, i, j - k0) = CM1(A, ld, i, j);
    for (int k = k0; k <= kb; ++k) {
        int p = k + 1;
        double amax = c_abs(CM1(A, ld, k + 1, k));
        for (int i = k + 2; i <= n; ++i) {
            double a = c_abs(CM1(A, ld, i, k));
            if (a > amax) { amax = a; p = i; }
        }
        ipiv[k - 1] = p;
        if (p != k + 1) {
            cswap(&CM1(A, ld, k + 1, k), &CM1(A, ld, p, k));
            cstep_swaps(n, A, ld, B0, ldb, ipiv, k0, kb, k, p);
        }
        cplx piv = CM1(A, ld, k + 1, k);
        if (c_iszero(piv)) continue;
        for (int i = k + 2; i <= n; ++i) CM1(A, ld, i, k) = c_div(CM1(A, ld, i, k), piv);
        for (int j = k + 1; j <= kb + 1; ++j) {
            cplx pj = CM1(A, ld, k + 1, j);
            if (c_iszero(pj)) continue;
            for (int i = k + 2; i <= n; ++i) CM1(A, ld, i, j) = c_sub(CM1(A, ld, i, j), c_mul(CM1(A, ld, i, k), pj));
        }
        for (int j = k + 2; j <= kb + 1; ++j) {
            cplx vj = CM1(A, ld, j, k);
            if (c_iszero(vj)) continue;
            for (int i = k0 + 1; i <= n; ++i)
                CM1(A, ld, i, k + 1) = c_add(CM1(A, ld, i, k + 1), c_mul(vj, CM1(A, ld, i, j)));
        }
        if (!(kb + 2 <= n)) continue;
        cgemv_cols(w, A, ld, k, k0 + 1, n, kb + 2, n);
        for (int kk = k0; kk <= k; ++kk) {
            int q = (int)ipiv[kk - 1];
            if (q != kk + 1) cswap(&w[kk], &w[q - 1]);
        }
        for (int kk = k0; kk <= k; ++kk) {
            cplx x = w[kk];
            if (c_iszero(x)) continue;
            for (int i = kk + 2; i <= n; ++i) w[i - 1] = c_sub(w[i - 1], c_mul(CM1(A, ld, i, kk), x));
        }
        for (int i = k0 + 1; i <= n; ++i) CM1(A, ld, i, k + 1) = c_add(CM1(A, ld, i, k + 1), w[i - 1]);
    }
}

static void creduce_blocked(int n, double* A, int ld, int64_t* ipiv, int nb)
{
    if (n < 3) return;
    const cplx minus_one = {-1.0, -0.0}, one = {1.0, 0.0};
    int ldb = n;
    double* B0 = (double*)malloc(sizeof(cplx) * (size_t)n * (size_t)(nb + 1));
    cplx* w = (cplx*)malloc(sizeof(cplx) * (size_t)n);
    for (int k0 = 1; k0 <= n - 2; k0 += nb) {
        int kb = k0 + nb - 1 < n - 2 ? k0 + nb - 1 : n - 2;
        cpanel_steps(n, A, ld, ipiv, B0, ldb, w, k0, kb);
        if (kb + 2 <= n) {
#pragma omp parallel for schedule(static) if (n >= 512)
            for (int c = kb + 2; c <= n; ++c)
                for (int k = k0; k <= kb; ++k) {
                    int p = (int)ipiv[k - 1];
                    if (p != k + 1) cswap(&CM1(A, ld, k + 1, c), &CM1(A, ld, p, c));
                }
#pragma omp parallel for schedule(static) if (n >= 512)
            for (int c = kb + 2; c <= n; ++c)
                for (int k = k0; k <= kb; ++k) {
                    cplx x = CM1(A, ld, k + 1, c);
                    if (c_iszero(x)) continue;
                    for (int i = k + 2; i <= kb + 1; ++i)
                        CM1(A, ld, i, c) = c_sub(CM1(A, ld, i, c), c_mul(CM1(A, ld, i, k), x));
                }
            cgemm_generic(A, ld, kb + 2, n, k0, kb, k0 + 1, kb + 2, kb + 2, n, minus_one);
        }
        for (int k = k0; k <= kb; ++k)
            for (int j = k + 2; j <= kb + 1; ++j) {
                cplx vj = CM1(A, ld, j, k);
                if (c_iszero(vj)) continue;
                for (int i = 1; i <= k0; ++i)
                    CM1(A, ld, i, k + 1) = c_add(CM1(A, ld, i, k + 1), c_mul(vj, CM1(A, ld, i, j)));
            }
        for (int kk = kb + 2; kk <= n; kk += nb) {
            int ke = kk + nb - 1 < n ? kk + nb - 1 : n;
            cgemm_generic(A, ld, 1, k0, kk, ke, kk, k0, k0 + 1, kb + 1, one);
        }
    }
    for (int k0 = 1; k0 <= n - 2; k0 += nb) {
        int kb = k0 + nb - 1 < n - 2 ? k0 + nb - 1 : n - 2;
        for (int c = k0; c <= kb; ++c)
            for (int k = kb + 1; k <= n - 2; ++k) {
                int p = (int)ipiv[k - 1];
                if (p != k + 1) cswap(&CM1(A, ld, k + 1, c), &CM1(A, ld, p, c));
            }
    }
    free(B0);
    free(w);
}

/* lhl_reduce! for a complex J (F:355-405): copy, balance, reduction, Ht fill               */
/* (Ht[j,i] = H[i,j] for i <= j+1, zero elsewhere), perm / iperm.                            */
/* path 0: the unblocked order at every n (the device's); 1: the generic blocked order     */
/* (panels of nb); 2: the reference's choice, blocked with nb = 16 iff n >= 768 (F:398).    */
int lhlo_reduce_c128_path(int n, const double* J, int ldj, int balance, double* F, int ldf, int64_t* ipiv,
                          double* scale, double* iscale, int64_t* perm, int64_t* iperm, double* Ht, int path, int nb)
{
    if (n < 0 || ldj < n || ldf < n || path < 0 || path > 2 || nb < 1) return -1;
    for (int j = 1; j <= n; ++j)
        for (int i = 1; i <= n; ++i) CM1(F, ldf, i, j) = CM1(J, ldj, i, j);
    if (balance) cbalance(n, F, ldf, scale, iscale);
    else for (int i = 0; i < n; ++i) { scale[i] = 1.0; iscale[i] = 1.0; }
    if (path == 2) { path = n >= 768 ? 1 : 0; nb = 16; }
    if (path == 1) creduce_blocked(n, F, ldf, ipiv, nb);
    else creduce_unblocked(n, F, ldf, ipiv);
    if (Ht) {
        memset(Ht, 0, sizeof(double) * 2 * (size_t)n * (size_t)n);
        for (int i = 1; i <= n; ++i)
            for (int j = (i - 1 > 1 ? i - 1 : 1); j <= n; ++j) CM1(Ht, n, j, i) = CM1(F, ldf, i, j);
    }
    for (int i = 1; i <= n; ++i) perm[i - 1] = i;
    for (int k = 1; k <= n - 2; ++k) {
        int64_t p = ipiv[k - 1];
        int64_t t = perm[k]; perm[k] = perm[p - 1]; perm[p - 1] = t;
    }
    for (int i = 1; i <= n; ++i) iperm[perm[i - 1] - 1] = i;
    return 0;
}

int lhlo_reduce_c128(int n, const double* J, int ldj, int balance, double* F, int ldf, int64_t* ipiv, double* scale,
                     double* iscale, int64_t* perm, int64_t* iperm, double* Ht)
{
    return lhlo_reduce_c128_path(n, J, ldj, balance, F, ldf, ipiv, scale, iscale, perm, iperm, Ht, 0, 16);
}

/* The shift LU of lhlo_shift_complex with tau * Ht[j,k] a complex product (Ht complex). */
int lhlo_shift_c128(int n, const double* Ht, int ldh, double sr, double si, double tr, double ti, double* Gt, int ldg,
                    int po, uint8_t* swp, double* rdiag /* 2n interleaved */, double* rw /* 2n */)
{
    if (n == 0) return 0;
    cplx sigma = {sr, si}, tau = {tr, ti};
    cplx* r = (cplx*)rw;
    for (int j = 1; j <= n; ++j) r[j - 1] = c_mul(tau, CM1(Ht, ldh, j, 1));
    r[0] = c_add(r[0], sigma);
    int info = 0;
    for (int k = 1; k <= n - 1; ++k) {
        cplx a = r[k - 1];
        cplx b = c_mul(tau, CM1(Ht, ldh, k, k + 1));
        if (c_mag(b) > c_mag(a)) {
            swp[k - 1] = 1;
            CSET(Gt, ldg, po, k, k, b);
            cplx l = c_div(a, b);
            CSET(Gt, ldg, po, k, k + 1, l);
            for (int j = k + 1; j <= n; ++j) {
                cplx g = c_mul(tau, CM1(Ht, ldh, j, k + 1));
                CSET(Gt, ldg, po, j, k, g);
                r[j - 1] = c_sub(r[j - 1], c_mul(l, g));
            }
            CSET(Gt, ldg, po, k + 1, k, c_add(CG(Gt, ldg, po, k + 1, k), sigma));
            r[k] = c_sub(r[k], c_mul(l, sigma));
        } else {
            swp[k - 1] = 0;
            CSET(Gt, ldg, po, k, k, a);
            cplx l;
            if (c_iszero(a)) { if (info == 0) info = k; l.re = 0.0; l.im = 0.0; }
            else l = c_div(b, a);
            CSET(Gt, ldg, po, k, k + 1, l);
            for (int j = k + 1; j <= n; ++j) {
                cplx rj = r[j - 1];
                CSET(Gt, ldg, po, j, k, rj);
                r[j - 1] = c_sub(c_mul(tau, CM1(Ht, ldh, j, k + 1)), c_mul(l, rj));
            }
            r[k] = c_add(r[k], sigma);
        }
    }
    cplx rn = r[n - 1];
    CSET(Gt, ldg, po, n, n, rn);
    swp[n - 1] = 0;
    if (c_iszero(rn) && info == 0) info = n;
    cplx one = {1.0, 0.0};
    for (int j = 1; j <= n; ++j) {
        cplx q = c_div(one, CG(Gt, ldg, po, j, j));
        rdiag[2 * (j - 1)] = q.re;
        rdiag[2 * (j - 1) + 1] = q.im;
    }
    return info;
}

/* x <- L^-1 x, the generic sweep F:2151-2195 (L[i,k] = F[i,k], i >= k+2): groups of four
 * steps with a serial head triangle, rows k+5:n as (L1 x1 + L2 x2) + (L3 x3 + L4 x4). */
static void czinvsweep(int n, const double* F, int ldf, cplx* x)
{
    int G = (n - 2 > 0 ? n - 2 : 0) >> 2;
    for (int g = 1; g <= G; ++g) {
        int k = 4 * g - 3;
        cplx x1 = x[k];
        cplx x2 = c_sub(x[k + 1], c_mul(CM1(F, ldf, k + 2, k), x1));
        x[k + 1] = x2;
        cplx x3 = c_sub(x[k + 2], c_add(c_mul(CM1(F, ldf, k + 3, k), x1), c_mul(CM1(F, ldf, k + 3, k + 1), x2)));
        x[k + 2] = x3;
        cplx x4 = c_sub(x[k + 3], c_add(c_add(c_mul(CM1(F, ldf, k + 4, k), x1), c_mul(CM1(F, ldf, k + 4, k + 1), x2)),
                                        c_mul(CM1(F, ldf, k + 4, k + 2), x3)));
        x[k + 3] = x4;
        for (int i = k + 5; i <= n; ++i) {
            cplx s = c_add(c_add(c_mul(CM1(F, ldf, i, k), x1), c_mul(CM1(F, ldf, i, k + 1), x2)),
                           c_add(c_mul(CM1(F, ldf, i, k + 2), x3), c_mul(CM1(F, ldf, i, k + 3), x4)));
            x[i - 1] = c_sub(x[i - 1], s);
        }
    }
    for (int k = 4 * G + 1; k <= n - 2; ++k) {
        cplx xk = x[k];
        for (int i = k + 2; i <= n; ++i) x[i - 1] = c_sub(x[i - 1], c_mul(CM1(F, ldf, i, k), xk));
    }
}

/* x <- L x, the generic sweep F:2199-2243: single steps in reverse, then groups in reverse,
 * each reading its four values first. */
static void czsweep(int n, const double* F, int ldf, cplx* x)
{
    int G = (n - 2 > 0 ? n - 2 : 0) >> 2;
    for (int k = n - 2; k >= 4 * G + 1; --k) {
        cplx xk = x[k];
        for (int i = k + 2; i <= n; ++i) x[i - 1] = c_add(x[i - 1], c_mul(CM1(F, ldf, i, k), xk));
    }
    for (int g = G; g >= 1; --g) {
        int k = 4 * g - 3;
        cplx x1 = x[k], x2 = x[k + 1], x3 = x[k + 2], x4 = x[k + 3];
        x[k + 1] = c_add(x2, c_mul(CM1(F, ldf, k + 2, k), x1));
        x[k + 2] = c_add(x3, c_add(c_mul(CM1(F, ldf, k + 3, k), x1), c_mul(CM1(F, ldf, k + 3, k + 1), x2)));
        x[k + 3] = c_add(x4, c_add(c_add(c_mul(CM1(F, ldf, k + 4, k), x1), c_mul(CM1(F, ldf, k + 4, k + 1), x2)),
                                   c_mul(CM1(F, ldf, k + 4, k + 2), x3)));
        for (int i = k + 5; i <= n; ++i) {
            cplx s = c_add(c_add(c_mul(CM1(F, ldf, i, k), x1), c_mul(CM1(F, ldf, i, k + 1), x2)),
                           c_add(c_mul(CM1(F, ldf, i, k + 2), x3), c_mul(CM1(F, ldf, i, k + 3), x4)));
            x[i - 1] = c_add(x[i - 1], s);
        }
    }
}

/* applyZinv! (F:2104-2112) and applyZ! (F:2069-2082) for a complex reduction; x n complex. */
void lhlo_applyZinv_c128(int n, const double* F, int ldf, const int64_t* perm, const double* iscale, double* x)
{
    cplx* xv = (cplx*)x;
    cplx* w = (cplx*)malloc(sizeof(cplx) * (size_t)(n > 0 ? n : 1));
    for (int i = 1; i <= n; ++i) {
        int64_t p = perm[i - 1];
        w[i - 1] = c_scale(xv[p - 1], iscale[p - 1]);
    }
    czinvsweep(n, F, ldf, w);
    for (int i = 0; i < n; ++i) xv[i] = w[i];
    free(w);
}

void lhlo_applyZ_c128(int n, const double* F, int ldf, const int64_t* iperm, const double* scale, double* x)
{
    cplx* xv = (cplx*)x;
    cplx* w = (cplx*)malloc(sizeof(cplx) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) w[i] = xv[i];
    czsweep(n, F, ldf, w);
    for (int i = 1; i <= n; ++i) xv[i - 1] = c_scale(w[iperm[i - 1] - 1], scale[i - 1]);
    free(w);
}

/* lhl_ldiv!(x, sh, ws) on a complex reduction (F:3111-3121): applyZinv!, the planar        */
/* Hessenberg solve, applyZ!.  y: 2 po doubles of scratch.                                   */
void lhlo_ldiv_c128(int n, const double* F, int ldf, const int64_t* perm, const int64_t* iperm, const double* scale,
                    const double* iscale, const double* Gt, int ldg, int po, const uint8_t* swp, const double* rdiag,
                    double* x, double* y)
{
    cplx* xv = (cplx*)x;
    lhlo_applyZinv_c128(n, F, ldf, perm, iscale, x);
    for (int i = 0; i < n; ++i) { y[i] = xv[i].re; y[po + i] = xv[i].im; }
    for (int i = n; i < po; ++i) { y[i] = 0.0; y[po + i] = 0.0; }
    hess_solve_planar(n, Gt, ldg, po, swp, rdiag, y);
    for (int i = 0; i < n; ++i) { xv[i].re = y[i]; xv[i].im = y[po + i]; }
    lhlo_applyZ_c128(n, F, ldf, iperm, scale, x);
}
