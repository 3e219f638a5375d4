// batch.cu -- lhl_reduce! of many independent matrices of uneven order in one launch
// (config 4's "4096 Jacobians, n in [16, 256]"): one CTA per matrix, in place in global memory
// (the matrix stays in L2 while its CTA works on it).  Orders n <= 512 take the reference's
// unblocked path (F:398-402 chooses it below 500), with the same operations in the same order
// as the single-matrix kernels, so every matrix is bit-identical to the oracle:
//   balancing (F:299-340): per sweep every index's column and row 1-norm summed sequentially
//     by one thread, then the ordered decision walk over the indices, 256 at a time, patching
//     the sums of later indices after an in-sweep scaling (as reduce.cu's balance_phase);
//   for k = 1..n-2 (F:466-501): pivot = first maximum of |A[k+1:n, k]|, row and column
//     interchanges, multipliers, the pk left update, then the trailing update with the
//     row-block kernel's per-row fma order (F:547-678) for n >= 8 and the paired sweep
//     (F:508-538) below; one thread per row;
//   Ht = H transposed (F:2005-2061), perm and iperm from ipiv (F:376-387).
#include "internal.cuh"

namespace lhl {

constexpr int BT = 256;  // threads per matrix

__device__ __forceinline__ bool bal_decide(double c, double r, double& f)
{
    if (c == 0.0 || r == 0.0) return false;
    f = 1.0;
    const double s = c + r;
    int guard = 0;
    while (c < r / 2.0 && guard < 4200) { c *= 2.0; r /= 2.0; f *= 2.0; ++guard; }
    while (c >= 2.0 * r && guard < 8400) { c /= 2.0; r *= 2.0; f /= 2.0; ++guard; }
    return c + r < 0.95 * s;
}

__global__ void __launch_bounds__(BT) reduce_batch_kernel(BatchDesc d, const double* __restrict__ J, int balance)
{
    const int m = blockIdx.x;
    const int n = d.n[m];
    if (n <= 0) return;
    double* A = d.F + d.off2[m];
    double* Ht = d.Ht + d.off2[m];
    const double* Jm = J + d.off2[m];
    int64_t* ipiv = d.ipiv + d.off1[m];
    int64_t* perm = d.perm + d.off1[m];
    int64_t* iperm = d.iperm + d.off1[m];
    double* sc = d.scale + d.off1[m];
    double* isc = d.iscale + d.off1[m];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    __shared__ double bsum[2 * 512], bfac[512];
    __shared__ double s_rv[BT / 32];
    __shared__ int s_ri[BT / 32];
    __shared__ int s_first, s_scaled, s_p;
    __shared__ double s_f;
    __shared__ int sp[512];

    for (size_t e = t; e < (size_t)n * n; e += BT) A[e] = Jm[e];
    for (int i = t; i < n; i += BT) {
        sc[i] = 1.0;
        isc[i] = 1.0;
        if (i < n - 2) ipiv[i] = i + 2;  // "no interchange" until step i+1 runs
    }
    __syncthreads();

    // ---- balancing ----
    for (int sweep = 0; balance && sweep < 20; ++sweep) {
        for (int i = 1 + t; i <= n; i += BT) {
            double c = 0.0, r = 0.0;
            for (int j = 1; j <= n; ++j) {
                if (j == i) continue;
                c += fabs(M1(A, n, j, i));
                r += fabs(M1(A, n, i, j));
            }
            bsum[i - 1] = c;
            bsum[n + i - 1] = r;
            bfac[i - 1] = 1.0;
        }
        if (t == 0) s_scaled = 0;
        __syncthreads();
        int base = 1;
        while (base <= n) {
            if (t == 0) s_first = 0x7fffffff;
            __syncthreads();
            const int i = base + t;
            double f = 1.0;
            if (i <= n && bal_decide(bsum[i - 1], bsum[n + i - 1], f)) atomicMin(&s_first, i);
            __syncthreads();
            const int si = s_first;
            if (si == 0x7fffffff) {
                base += BT;
                continue;
            }
            if (i == si) {
                s_f = f;
                s_scaled = 1;
            }
            __syncthreads();
            const double fs = s_f;
            for (int mm = si + 1 + t; mm <= n; mm += BT) {
                const double vr = fabs(M1(A, n, si, mm));
                const double vc = fabs(M1(A, n, mm, si));
                bsum[mm - 1] = (bsum[mm - 1] - vr) + vr / fs;
                bsum[n + mm - 1] = (bsum[n + mm - 1] - vc) + vc * fs;
            }
            if (t == 0) {
                bfac[si - 1] = fs;
                sc[si - 1] *= fs;
                isc[si - 1] /= fs;
            }
            __syncthreads();
            base = si + 1;
        }
        if (!s_scaled) break;
        for (size_t e = t; e < (size_t)n * n; e += BT) {
            const int i = (int)(e % n), j = (int)(e / n);
            const double fi = bfac[i], fj = bfac[j];
            if (fi != 1.0 || fj != 1.0) A[e] = (A[e] / fi) * fj;
        }
        __syncthreads();
    }

    // ---- elimination ----
    const bool generic = n < 8;
    for (int k = 1; k <= n - 2; ++k) {
        double bv = 0.0;
        int bi = 0;
        for (int i = k + 1 + t; i <= n; i += BT) argmax_combine(bv, bi, fabs(M1(A, n, i, k)), i);
        warp_argmax(bv, bi);
        if (lane == 0) {
            s_rv[warp] = bv;
            s_ri[warp] = bi;
        }
        __syncthreads();
        if (t == 0) {
            double v = 0.0;
            int vi = 0;
            for (int w = 0; w < BT / 32; ++w) argmax_combine(v, vi, s_rv[w], s_ri[w]);
            s_p = (vi >= k + 1 && vi <= n) ? vi : k + 1;
            ipiv[k - 1] = s_p;
        }
        __syncthreads();
        const int p = s_p;
        if (p != k + 1) {
            for (int j = 1 + t; j <= n; j += BT) {
                const double u = M1(A, n, k + 1, j);
                M1(A, n, k + 1, j) = M1(A, n, p, j);
                M1(A, n, p, j) = u;
            }
            __syncthreads();
            for (int i = 1 + t; i <= n; i += BT) {
                const double u = M1(A, n, i, k + 1);
                M1(A, n, i, k + 1) = M1(A, n, i, p);
                M1(A, n, i, p) = u;
            }
            __syncthreads();
        }
        const double piv = M1(A, n, k + 1, k);
        if (piv == 0.0) continue;  // F:488
        for (int i = k + 2 + t; i <= n; i += BT) M1(A, n, i, k) = M1(A, n, i, k) / piv;
        __syncthreads();
        const double pk = M1(A, n, k + 1, k + 1);
        if (pk != 0.0)
            for (int i = k + 2 + t; i <= n; i += BT) M1(A, n, i, k + 1) = dsub(M1(A, n, i, k + 1), dmul(M1(A, n, i, k), pk));
        __syncthreads();
        for (int i = 1 + t; i <= n; i += BT) {
            const double li = (i >= k + 2) ? M1(A, n, i, k) : 0.0;
            double ck1 = M1(A, n, i, k + 1);
            if (!generic) {
                double s = 0.0;
                const bool low = i >= k + 2;
                int j = k + 2;
                // eight columns at a time: the block's loads (this row, the pivot row, column k;
                // none of them is stored this step) are issued before its stores
                for (; j + 7 <= n; j += 8) {
                    double v[8], pr[8], lk[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        v[u] = M1(A, n, i, j + u);
                        pr[u] = low ? M1(A, n, k + 1, j + u) : 0.0;
                        lk[u] = M1(A, n, j + u, k);
                    }
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        double x = v[u];
                        if (low) {
                            x = dfma(li, -pr[u], x);
                            M1(A, n, i, j + u) = x;
                        }
                        s = dfma(lk[u], x, s);
                    }
                }
                for (; j <= n; ++j) {
                    double v = M1(A, n, i, j);
                    if (low) {
                        v = dfma(li, -M1(A, n, k + 1, j), v);
                        M1(A, n, i, j) = v;
                    }
                    s = dfma(M1(A, n, j, k), v, s);
                }
                ck1 = dadd(ck1, s);
            } else {
                int j = k + 2;
                while (j + 1 <= n) {
                    double v0 = M1(A, n, i, j), v1 = M1(A, n, i, j + 1);
                    if (i >= k + 2) {
                        v0 = dsub(v0, dmul(li, M1(A, n, k + 1, j)));
                        v1 = dsub(v1, dmul(li, M1(A, n, k + 1, j + 1)));
                        M1(A, n, i, j) = v0;
                        M1(A, n, i, j + 1) = v1;
                    }
                    ck1 = dadd(ck1, dadd(dmul(M1(A, n, j, k), v0), dmul(M1(A, n, j + 1, k), v1)));
                    j += 2;
                }
                if (j <= n) {
                    double v0 = M1(A, n, i, j);
                    if (i >= k + 2) {
                        v0 = dsub(v0, dmul(li, M1(A, n, k + 1, j)));
                        M1(A, n, i, j) = v0;
                    }
                    ck1 = dadd(ck1, dmul(M1(A, n, j, k), v0));
                }
            }
            M1(A, n, i, k + 1) = ck1;
        }
        __syncthreads();
    }

    // ---- Ht and the permutations ----
    for (size_t e = t; e < (size_t)n * n; e += BT) {
        const int j = (int)(e % n), i = (int)(e / n);  // Ht[j, i] = A[i, j] for i <= j + 1
        Ht[e] = (i <= j + 1) ? A[(size_t)j * n + i] : 0.0;
    }
    for (int i = t; i < n; i += BT) sp[i] = i + 1;
    __syncthreads();
    if (t == 0)
        for (int k = 1; k <= n - 2; ++k) {
            const int p = (int)ipiv[k - 1];
            const int u = sp[k];
            sp[k] = sp[p - 1];
            sp[p - 1] = u;
        }
    __syncthreads();
    for (int i = t; i < n; i += BT) {
        perm[i] = sp[i];
        iperm[sp[i] - 1] = i + 1;
    }
}

cudaError_t launch_reduce_batch(const BatchDesc& d, const double* J, int balance, cudaStream_t st)
{
    if (d.count <= 0) return cudaSuccess;
    reduce_batch_kernel<<<d.count, BT, 0, st>>>(d, J, balance);
    return cudaGetLastError();
}

}  // namespace lhl
