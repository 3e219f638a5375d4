// solve.cu -- lhl_ldiv! (F:3052-3068), applyZ! / applyZinv! (F:2069-2126) and the residual
// of lhl_refine! (F:3144-3157) on sm_100a.
//
// x <- W^-1 x with W = Z (sigma I + tau H) Z^-1, Z = D P L:
//   gather y = P^-1 D^-1 x  ->  y <- L^-1 y  ->  Hessenberg solve with the shift's LU
//   ->  y <- L y  ->  scatter x = D P y.
// Three launches, so that L (shared by every shift) is read once per tile of right-hand
// sides and not once per right-hand side:
//   zinv_kernel  -- gather and y <- L^-1 y for RT right-hand sides per CTA, the vectors in
//                   shared memory.  Column blocks of 32: the block's 32 x 32 triangle is staged
//                   in shared memory and solved by one warp per right-hand side (shuffles),
//                   then every thread applies the block to its rows with 32 independent loads
//                   of L in flight.
//   hess_kernel  -- the Hessenberg solve with each right-hand side's shift LU, one CTA per
//                   right-hand side (the forward select-swap recurrence, F:2806-2816, then a
//                   left-looking back substitution over Gt's contiguous columns).
//   zmul_kernel  -- y <- L y (no recurrence: original y on the right), rows split over CTAs,
//                   and the scatter x[perm[i]] = (L y)[i] * scale[perm[i]].
// Summation order differs from the reference's (results agree to rounding; the solve's
// contract is its residual, not its bits).
#include "internal.cuh"

namespace lhl {

constexpr int SOLVE_T = 512;
constexpr int BS = 32;


constexpr int ZT = 512;

// L[i, c] (1-based) = F[i, c-1] for 2 <= c <= n-1, i >= c+1 (unit lower; column 1 is e1).
__device__ __forceinline__ const double* lcol(const ZArgs& z, int c) { return z.F + (size_t)(c - 2) * z.ldf; }

// y <- L^-1 P^-1 D^-1 x (gather = 1) or y <- L^-1 x, for RT right-hand sides per CTA.
template <int RT>
__global__ void __launch_bounds__(ZT) zinv_kernel(ZArgs z)
{
    extern __shared__ double ys[];  // RT x n, right-hand side j at ys + j n
    __shared__ double tri[BS][BS + 1];
    const int n = z.n;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int c0 = blockIdx.x * RT;
    for (int j = 0; j < RT; ++j) {
        const double* x = z.src + (size_t)(c0 + j) * z.lds;
        for (int i = t; i < n; i += ZT) {
            double v = 0.0;
            if (c0 + j < z.m) {
                if (z.gather) {
                    const int64_t p = z.perm[i];
                    v = x[p - 1] * z.iscale[p - 1];
                } else {
                    v = x[i];
                }
            }
            ys[j * n + i] = v;
        }
    }
    __syncthreads();
    for (int cb0 = 2; cb0 <= n - 1; cb0 += BS) {
        const int cb1 = min(cb0 + BS - 1, n - 1);
        const int bw = cb1 - cb0 + 1;
        for (int e = t; e < BS * BS; e += ZT) {
            const int r = e & (BS - 1), q = e >> 5;
            if (q < bw && r < bw && r > q) tri[r][q] = lcol(z, cb0 + q)[cb0 + r - 1];
        }
        __syncthreads();
        if (warp < RT) {
            double* y = ys + warp * n;
            double yi = lane < bw ? y[cb0 + lane - 1] : 0.0;
            for (int q = 0; q < bw - 1; ++q) {
                const double xq = __shfl_sync(0xffffffffu, yi, q);
                if (lane > q && lane < bw) yi = dfma(-tri[lane][q], xq, yi);
            }
            if (lane < bw) y[cb0 + lane - 1] = yi;
        }
        __syncthreads();
        for (int i = cb1 + 1 + t; i <= n; i += ZT) {
            double l[BS];
#pragma unroll
            for (int q = 0; q < BS; ++q) l[q] = q < bw ? lcol(z, cb0 + q)[i - 1] : 0.0;
#pragma unroll
            for (int j = 0; j < RT; ++j) {
                const double* y = ys + j * n;
                double v = y[i - 1];
#pragma unroll
                for (int q = 0; q < BS; ++q)
                    if (q < bw) v = dfma(-l[q], y[cb0 + q - 1], v);
                ys[j * n + i - 1] = v;
            }
        }
        __syncthreads();
    }
    for (int j = 0; j < RT; ++j) {
        if (c0 + j >= z.m) break;
        double* d = z.dst + (size_t)(c0 + j) * z.ldd;
        for (int i = t; i < n; i += ZT) d[i] = ys[j * n + i];
    }
}

// x <- D P L y for RT right-hand sides per CTA; blockIdx.y splits the rows (row i costs i).
template <int RT>
__global__ void __launch_bounds__(ZT) zmul_kernel(ZArgs z)
{
    extern __shared__ double ys[];  // RT x n
    const int n = z.n;
    const int t = threadIdx.x;
    const int c0 = blockIdx.x * RT;
    for (int j = 0; j < RT; ++j) {
        const double* y = z.src + (size_t)(c0 + j) * z.lds;
        for (int i = t; i < n; i += ZT) ys[j * n + i] = (c0 + j < z.m) ? y[i] : 0.0;
    }
    __syncthreads();
    // rows [i0, i1) of this CTA: equal shares of the n^2/2 work
    const int S = gridDim.y, s = blockIdx.y;
    const int i0 = (int)((double)n * sqrt((double)s / S)), i1 = s + 1 == S ? n : (int)((double)n * sqrt((double)(s + 1) / S));
    for (int i = i0 + 1 + t; i <= i1; i += ZT) {
        double acc[RT];
#pragma unroll
        for (int j = 0; j < RT; ++j) acc[j] = ys[j * n + i - 1];
        for (int cb0 = 2; cb0 <= i - 1; cb0 += BS) {
            const int bw = min(BS, i - cb0);
            double l[BS];
#pragma unroll
            for (int q = 0; q < BS; ++q) l[q] = q < bw ? lcol(z, cb0 + q)[i - 1] : 0.0;
#pragma unroll
            for (int j = 0; j < RT; ++j) {
                const double* y = ys + j * n;
#pragma unroll
                for (int q = 0; q < BS; ++q)
                    if (q < bw) acc[j] = dfma(l[q], y[cb0 + q - 1], acc[j]);
            }
        }
        const int64_t p = z.perm[i - 1];
#pragma unroll
        for (int j = 0; j < RT; ++j)
            if (c0 + j < z.m) z.dst[(size_t)(c0 + j) * z.ldd + (p - 1)] = acc[j] * z.scale[p - 1];
    }
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
            double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
            int i = r1 + 1 + lane;
            for (; i + 96 <= n; i += 128) {
                acc0 = dfma(g[i - 1], y[i - 1], acc0);
                acc1 = dfma(g[i + 31], y[i + 31], acc1);
                acc2 = dfma(g[i + 63], y[i + 63], acc2);
                acc3 = dfma(g[i + 95], y[i + 95], acc3);
            }
            for (; i <= n; i += 32) acc0 = dfma(g[i - 1], y[i - 1], acc0);
            double acc = warp_sum((acc0 + acc1) + (acc2 + acc3));
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

// The Hessenberg solve of one right-hand side of Y (column blockIdx.x) with its shift's LU.
__global__ void __launch_bounds__(SOLVE_T) hess_kernel(LdivArgs a, double* Y, int ldy, int col0)
{
    extern __shared__ double smem[];
    const int n = a.n;
    double* y = smem;
    double* y2 = smem + n;
    uint8_t* ssw = (uint8_t*)(smem + 2 * n);
    const int col = col0 + blockIdx.x;
    if (a.done && a.done[col] <= a.tol) return;  // converged column (refinement to a tolerance)
    double* yg = Y + (size_t)blockIdx.x * ldy;
    const int t = threadIdx.x;
    for (int i = t; i < n; i += SOLVE_T) y[i] = yg[i];
    __syncthreads();
    const int s = col / a.rhs_per_shift;
    const double* Gt = a.Gt + (size_t)s * a.ldg * n;
    hess_solve(a, Gt, a.swp + (size_t)s * n, a.rdiag + (size_t)s * n, y, y2, ssw);
    for (int i = t; i < n; i += SOLVE_T) yg[i] = y[i];
}

template <int RT>
static cudaError_t launch_z(bool inv, const ZArgs& z, int zsplit, cudaStream_t st)
{
    const size_t smem = (size_t)RT * z.n * sizeof(double);
    static size_t attr[2] = {0, 0};
    const void* fn = inv ? (const void*)zinv_kernel<RT> : (const void*)zmul_kernel<RT>;
    if (smem > 32 * 1024 && smem > attr[inv]) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr[inv] = smem;
    }
    const dim3 grid((z.m + RT - 1) / RT, inv ? 1 : zsplit);
    if (inv) zinv_kernel<RT><<<grid, ZT, smem, st>>>(z);
    else zmul_kernel<RT><<<grid, ZT, smem, st>>>(z);
    return cudaGetLastError();
}

static cudaError_t run_z(bool inv, const ZArgs& z, cudaStream_t st)
{
    // right-hand sides per CTA: as many as fit in shared memory, at most 4
    const size_t per = (size_t)z.n * sizeof(double);
    const int tiles4 = (z.m + 3) / 4;
    const int zsplit = inv ? 1 : (tiles4 >= 64 ? 2 : (tiles4 >= 16 ? 8 : 16));
    if (4 * per <= 190 * 1024) return launch_z<4>(inv, z, zsplit, st);
    if (2 * per <= 190 * 1024) return launch_z<2>(inv, z, zsplit * 2, st);
    return launch_z<1>(inv, z, zsplit * 4, st);
}

cudaError_t launch_ldiv(const LdivArgs& a, int nrhs, cudaStream_t st)
{
    if (nrhs <= 0 || a.n <= 0) return cudaSuccess;
    ZArgs z;
    memset(&z, 0, sizeof(z));
    z.n = a.n;
    z.F = a.F;
    z.ldf = a.ldf;
    z.perm = a.perm;
    z.scale = a.scale;
    z.iscale = a.iscale;
    if (a.mode == 1) {  // applyZinv: x <- L^-1 P^-1 D^-1 x (in place)
        z.src = a.X; z.lds = a.ldx; z.dst = a.X; z.ldd = a.ldx; z.m = nrhs; z.gather = 1;
        return run_z(true, z, st);
    }
    if (!a.Y || a.ycap <= 0) return cudaErrorInvalidValue;
    if (a.mode == 2) {  // applyZ: x <- D P L x, through the scratch (CTAs split the rows)
        for (int c0 = 0; c0 < nrhs; c0 += a.ycap) {
            const int cnt = min(a.ycap, nrhs - c0);
            cudaError_t e = cudaMemcpy2DAsync(a.Y, (size_t)a.n * sizeof(double), a.X + (size_t)c0 * a.ldx,
                                              (size_t)a.ldx * sizeof(double), (size_t)a.n * sizeof(double), cnt,
                                              cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return e;
            z.src = a.Y; z.lds = a.n; z.dst = a.X + (size_t)c0 * a.ldx; z.ldd = a.ldx; z.m = cnt; z.gather = 0;
            e = run_z(false, z, st);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    const size_t hsm = (size_t)a.n * 2 * sizeof(double) + (size_t)a.n + 16;
    // dynamic + static shared memory must stay within the 227 KB a CTA may use
    if (hsm > 200 * 1024) return cudaErrorInvalidValue;
    static size_t attr = 0;
    if (hsm > 32 * 1024 && hsm > attr) {  // the kernel's static shared arrays add about 8.5 KB
        cudaError_t e = cudaFuncSetAttribute(hess_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsm);
        if (e != cudaSuccess) return e;
        attr = hsm;
    }
    for (int c0 = 0; c0 < nrhs; c0 += a.ycap) {
        const int cnt = min(a.ycap, nrhs - c0);
        z.src = a.X + (size_t)c0 * a.ldx; z.lds = a.ldx; z.dst = a.Y; z.ldd = a.n; z.m = cnt; z.gather = 1;
        cudaError_t e = run_z(true, z, st);
        if (e != cudaSuccess) return e;
        hess_kernel<<<cnt, SOLVE_T, hsm, st>>>(a, a.Y, a.n, c0);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        z.src = a.Y; z.lds = a.n; z.dst = a.X + (size_t)c0 * a.ldx; z.ldd = a.ldx; z.gather = 0;
        e = run_z(false, z, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
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
