// solve.cu -- lhl_ldiv! (F:3052-3068), applyZ! / applyZinv! (F:2069-2126) and the residual
// of lhl_refine! (F:3144-3157) on sm_100a.
//
// x <- W^-1 x with W = Z (sigma I + tau H) Z^-1, Z = D P L:
//   gather y = P^-1 D^-1 x  ->  y <- L^-1 y  ->  Hessenberg solve with the shift's LU
//   ->  y <- L y  ->  scatter x = D P y.
// One CTA per right-hand side; the vector lives in shared memory for the whole chain.
// The triangular solves are blocked by 32: a warp solves the 32x32 diagonal triangle with
// shuffles, then the whole CTA applies the block to the remaining rows, so a solve costs
// 2n/32 CTA barriers instead of n.  The L product needs no recurrence (y <- L y reads the
// original y only) and runs as one row-parallel triangular matvec.  The Hessenberg
// forward pass (n-1 select-swap steps, F:2806-2816) is one scalar recurrence on
// shared-memory operands.  Summation order differs from the reference's (results agree to
// rounding; the solve's contract is its residual, not its bits).
#include "internal.cuh"

namespace lhl {

constexpr int SOLVE_T = 512;
constexpr int BS = 32;


// y <- L^-1 y, L[i,c] = F[i,c-1] for i >= c+1, c = 2..n-1 (unit lower; column 1 is e1).
__device__ void lsolve_fwd(const LdivArgs& a, double* y)
{
    const int n = a.n;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int c0 = 2; c0 <= n - 1; c0 += BS) {
        const int cb = min(c0 + BS - 1, n - 1);
        if (warp == 0) {
            // diagonal triangle: rows c0..cb+1? no -- rows within the block c0..cb
            const int i = c0 + lane;
            double yi = (i <= cb) ? y[i - 1] : 0.0;
            for (int c = c0; c < cb; ++c) {
                const double xc = __shfl_sync(0xffffffffu, yi, c - c0);
                if (i > c && i <= cb) yi = dfma(-M1(a.F, a.ldf, i, c - 1), xc, yi);
            }
            if (i <= cb) y[i - 1] = yi;
        }
        __syncthreads();
        // rows below the block: y[i] -= sum_{c=c0..cb} L[i,c] y[c]
        for (int i = cb + 1 + t; i <= n; i += SOLVE_T) {
            double v = y[i - 1];
            for (int c = c0; c <= cb; ++c) v = dfma(-M1(a.F, a.ldf, i, c - 1), y[c - 1], v);
            y[i - 1] = v;
        }
        __syncthreads();
    }
}

// y <- L y (original y on the right): (Ly)[i] = y[i] + sum_{c=2}^{i-1} L[i,c] y[c].
__device__ void lmul(const LdivArgs& a, double* y, double* y2)
{
    const int n = a.n;
    const int t = threadIdx.x;
    for (int i = 1 + t; i <= n; i += SOLVE_T) {
        double v = y[i - 1];
        for (int c = 2; c <= i - 1; ++c) v = dfma(M1(a.F, a.ldf, i, c - 1), y[c - 1], v);
        y2[i - 1] = v;
    }
    __syncthreads();
    for (int i = 1 + t; i <= n; i += SOLVE_T) y[i - 1] = y2[i - 1];
    __syncthreads();
}

// Hessenberg solve with the shift's LU (F:2746-2816): forward select-swap steps, then
// U x = y with U[k,j] = Gt[j,k] (j >= k) and rdiag = 1 / U[k,k].
__device__ void hess_solve(const LdivArgs& a, const double* Gt, const uint8_t* swp, const double* rd, double* y,
                           double* sm, uint8_t* ssw)
{
    const int n = a.n;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int k = 1 + t; k <= n - 1; k += SOLVE_T) {
        sm[k - 1] = M1(Gt, a.ldg, k, k + 1);
        ssw[k - 1] = swp[k - 1];
    }
    __syncthreads();
    if (t == 0 && n >= 2) {
        double c = y[0];
        for (int k = 1; k <= n - 1; ++k) {
            const double b = y[k];
            const bool s = ssw[k - 1] != 0;
            const double xk = s ? b : c;
            y[k - 1] = xk;
            c = (s ? c : b) - sm[k - 1] * xk;
        }
        y[n - 1] = c;
    }
    __syncthreads();
    // back substitution in blocks of 32 rows from the bottom, left-looking: the block's
    // sums over the rows already solved are dot products with columns of Gt (column j of Gt
    // is row j of U, contiguous), one warp per column, coalesced.  The same warp stages the
    // block's part of that column (U[j, r0..r1]) in shared memory, and warp 0 then solves
    // the 32 x 32 triangle from there.
    __shared__ double tri[BS][BS + 1];
    double* sj = sm;  // block partial sums (the multiplier copy in sm is no longer needed)
    const int nwarps = SOLVE_T / 32;
    for (int r1 = n; r1 >= 1; r1 -= BS) {
        const int r0 = max(r1 - BS + 1, 1);
        const int bs = r1 - r0 + 1;
        for (int jj = warp; jj < bs; jj += nwarps) {
            const int j = r0 + jj;
            const double* g = Gt + (size_t)(j - 1) * a.ldg;  // Gt column j = row j of U
            if (r0 + lane <= r1) tri[jj][lane] = g[r0 + lane - 1];  // U[j, r0 + lane]
            double acc = 0.0;
            for (int i = r1 + 1 + lane; i <= n; i += 32) acc = dfma(g[i - 1], y[i - 1], acc);
            acc = warp_sum(acc);
            if (lane == 0) sj[jj] = acc;
        }
        __syncthreads();
        if (warp == 0) {
            const int i = r0 + lane;
            double yi = (i <= r1) ? y[i - 1] - sj[lane] : 0.0;
            for (int j = r1; j >= r0; --j) {
                double xj = 0.0;
                if (i == j) {
                    yi = yi * rd[j - 1];
                    xj = yi;
                }
                xj = __shfl_sync(0xffffffffu, xj, j - r0);
                if (i < j && i >= r0) yi = dfma(-tri[lane][j - r0], xj, yi);  // U[i, j]
            }
            if (i <= r1) y[i - 1] = yi;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(SOLVE_T) ldiv_kernel(LdivArgs a)
{
    extern __shared__ double smem[];
    const int n = a.n;
    double* y = smem;
    double* y2 = smem + n;
    uint8_t* ssw = (uint8_t*)(smem + 2 * n);
    const int col = blockIdx.x;
    if (a.done && a.done[col] <= a.tol) return;  // converged column (refinement to a tolerance)
    double* x = a.X + (size_t)col * a.ldx;
    const int t = threadIdx.x;

    if (a.mode != 2) {  // gather y = P^-1 D^-1 x (F:2130-2140)
        for (int i = 1 + t; i <= n; i += SOLVE_T) {
            const int64_t p = a.perm[i - 1];
            y[i - 1] = x[p - 1] * a.iscale[p - 1];
        }
    } else {
        for (int i = 1 + t; i <= n; i += SOLVE_T) y[i - 1] = x[i - 1];
    }
    __syncthreads();
    if (a.mode != 2) lsolve_fwd(a, y);
    if (a.mode == 0) {
        const int s = col / a.rhs_per_shift;
        const double* Gt = a.Gt + (size_t)s * a.ldg * n;
        hess_solve(a, Gt, a.swp + (size_t)s * n, a.rdiag + (size_t)s * n, y, y2, ssw);
    }
    if (a.mode != 1) {
        lmul(a, y, y2);
        for (int i = 1 + t; i <= n; i += SOLVE_T) x[i - 1] = y[a.iperm[i - 1] - 1] * a.scale[i - 1];
    } else {
        for (int i = 1 + t; i <= n; i += SOLVE_T) x[i - 1] = y[i - 1];
    }
}

cudaError_t launch_ldiv(const LdivArgs& a, int nrhs, cudaStream_t st)
{
    if (nrhs <= 0 || a.n <= 0) return cudaSuccess;
    const size_t smem = (size_t)a.n * 2 * sizeof(double) + (size_t)a.n + 16;
    // dynamic + static shared memory must stay within the 227 KB a CTA may use
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static size_t attr = 0;
    if (smem > 32 * 1024 && smem > attr) {  // the kernel's static shared arrays add about 8.5 KB
        cudaError_t e = cudaFuncSetAttribute(ldiv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr = smem;
    }
    ldiv_kernel<<<nrhs, SOLVE_T, smem, st>>>(a);
    return cudaGetLastError();
}

// ---- residual r = b - (sigma_s I + tau_s J) x, one tile of 64 rows x 8 columns per CTA ----
constexpr int RT_M = 64, RT_N = 8, RT_K = 32;

__global__ void __launch_bounds__(256) residual_kernel(int n, const double* __restrict__ J, int ldj,
                                                       const double* __restrict__ B, int ldb,
                                                       const double* __restrict__ X, int ldx, double* __restrict__ R,
                                                       int ldr, int nrhs, int rhs_per_shift,
                                                       const double* __restrict__ sig, const double* __restrict__ tau)
{
    __shared__ double sJ[RT_K][RT_M + 1];
    __shared__ double sX[RT_N][RT_K + 1];
    const int i0 = blockIdx.x * RT_M, c0 = blockIdx.y * RT_N;
    const int t = threadIdx.x;
    const int ti = t & 63, tc = t >> 6;  // 64 rows x 4 column pairs
    double acc0 = 0.0, acc1 = 0.0;
    for (int k0 = 0; k0 < n; k0 += RT_K) {
        for (int e = t; e < RT_K * RT_M; e += 256) {
            const int ii = e % RT_M, kk = e / RT_M;
            const int i = i0 + ii, k = k0 + kk;
            sJ[kk][ii] = (i < n && k < n) ? J[(size_t)k * ldj + i] : 0.0;
        }
        for (int e = t; e < RT_K * RT_N; e += 256) {
            const int kk = e % RT_K, cc = e / RT_K;
            const int k = k0 + kk, c = c0 + cc;
            sX[cc][kk] = (k < n && c < nrhs) ? X[(size_t)c * ldx + k] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < RT_K; ++kk) {
            const double jv = sJ[kk][ti];
            acc0 = dfma(jv, sX[2 * tc][kk], acc0);
            acc1 = dfma(jv, sX[2 * tc + 1][kk], acc1);
        }
        __syncthreads();
    }
    const int i = i0 + ti;
    if (i < n) {
        for (int q = 0; q < 2; ++q) {
            const int c = c0 + 2 * tc + q;
            if (c < nrhs) {
                const int s = c / rhs_per_shift;
                const double xv = X[(size_t)c * ldx + i];
                const double jx = q == 0 ? acc0 : acc1;
                R[(size_t)c * ldr + i] = B[(size_t)c * ldb + i] - (sig[s] * xv + tau[s] * jx);
            }
        }
    }
}

cudaError_t launch_residual(int n, const double* J, int ldj, const double* B, int ldb, const double* X, int ldx,
                            double* R, int ldr, int nrhs, int rhs_per_shift, const double* sig, const double* tau,
                            cudaStream_t st)
{
    if (nrhs <= 0 || n <= 0) return cudaSuccess;
    dim3 grid((n + RT_M - 1) / RT_M, (nrhs + RT_N - 1) / RT_N);
    residual_kernel<<<grid, 256, 0, st>>>(n, J, ldj, B, ldb, X, ldx, R, ldr, nrhs, rhs_per_shift, sig, tau);
    return cudaGetLastError();
}

__global__ void axpy_cols_kernel(int n, double* __restrict__ X, int ldx, const double* __restrict__ R, int ldr,
                                 const double* __restrict__ done, double tol)
{
    const int c = blockIdx.y;
    if (done && done[c] <= tol) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        X[(size_t)c * ldx + i] += R[(size_t)c * ldr + i];
}

cudaError_t launch_axpy_cols(int n, double* X, int ldx, const double* R, int ldr, int nrhs, cudaStream_t st,
                             const double* done, double tol)
{
    if (nrhs <= 0 || n <= 0) return cudaSuccess;
    dim3 grid((n + 255) / 256 < 64 ? (n + 255) / 256 : 64, nrhs);
    axpy_cols_kernel<<<grid, 256, 0, st>>>(n, X, ldx, R, ldr, done, tol);
    return cudaGetLastError();
}

// ||R[:,c]||_2 / ||B[:,c]||_2 per column
__global__ void __launch_bounds__(256) relres_kernel(int n, const double* __restrict__ R, int ldr,
                                                     const double* __restrict__ B, int ldb, double* __restrict__ out)
{
    __shared__ double s_r[8], s_b[8];
    const int c = blockIdx.x;
    double r2 = 0.0, b2 = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) {
        const double rv = R[(size_t)c * ldr + i], bv = B[(size_t)c * ldb + i];
        r2 = dfma(rv, rv, r2);
        b2 = dfma(bv, bv, b2);
    }
    r2 = warp_sum(r2);
    b2 = warp_sum(b2);
    if ((threadIdx.x & 31) == 0) {
        s_r[threadIdx.x >> 5] = r2;
        s_b[threadIdx.x >> 5] = b2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < 8; ++w) { a += s_r[w]; b += s_b[w]; }
        out[c] = b > 0.0 ? sqrt(a) / sqrt(b) : sqrt(a);
    }
}

cudaError_t launch_relres(int n, const double* R, int ldr, const double* B, int ldb, double* out, int nrhs,
                          cudaStream_t st)
{
    if (nrhs <= 0 || n <= 0) return cudaSuccess;
    relres_kernel<<<nrhs, 256, 0, st>>>(n, R, ldr, B, ldb, out);
    return cudaGetLastError();
}

}  // namespace lhl
