// solve.cu -- lhl_ldiv! (F:3052-3068), applyZ! / applyZinv! (F:2069-2126) and the residual
// of lhl_refine! (F:3144-3157) on sm_100a.
//
// x <- W^-1 x with W = Z (sigma I + tau H) Z^-1, Z = D P L:
//   gather y = P^-1 D^-1 x  ->  y <- L^-1 y  ->  Hessenberg solve with the shift's LU
//   ->  y <- L y  ->  scatter x = D P y.
// Three launches, so that L (shared by every shift) is read once per tile of right-hand
// sides and not once per right-hand side:
//   zl_kernel<false> -- gather and y <- L^-1 y: a blocked forward substitution over a
//                   cooperative grid, tasks (64-row block, 4 right-hand sides) with ready flags.
//   hess_kernel  -- the Hessenberg solve with each right-hand side's shift LU, one CTA per
//                   right-hand side (the forward select-swap recurrence, F:2806-2816, then a
//                   left-looking back substitution over Gt's contiguous columns).
//   zl_kernel<true>  -- y <- L y (no recurrence: original y on the right), the same tasks
//                   without flags, and the scatter x[perm[i]] = (L y)[i] * scale[perm[i]].
// Summation order differs from the reference's (results agree to rounding; the solve's
// contract is its residual, not its bits).
#include "internal.cuh"

namespace lhl {

constexpr int SOLVE_T = 512;
constexpr int BS = 32;


constexpr int ZT = 512;

// true when every column c0..c0+cnt-1 (< m) is marked converged; with cs = 1 the columns
// are the two parts of complex right-hand sides and done[] is indexed by c >> 1
__device__ __forceinline__ bool tile_done(const double* done, double tol, int c0, int cnt, int m, int cs = 0)
{
    if (!done) return false;
    for (int c = c0; c < c0 + cnt && c < m; ++c)
        if (!(done[c >> cs] <= tol)) return false;
    return true;
}

// L[i, c] (1-based) = F[i, c-1] for 2 <= c <= n-1, i >= c+1 (unit lower; column 1 is e1).
__device__ __forceinline__ const double* lcol(const ZArgs& z, int c) { return z.F + (size_t)(c - 2) * z.ldf; }

// MUL = false: y <- L^-1 P^-1 D^-1 x (gather = 1) or y <- L^-1 x, a blocked forward
// substitution spread over a cooperative grid.  MUL = true: x <- D P L y with the same tiles
// and no dependencies between tasks.  Task (i, c) owns rows 64i..64i+63 of right-hand sides 4c..4c+3;
// tasks are numbered block-major and handed out in order, so every task it waits for runs
// earlier (on a co-resident CTA).  A task folds in L_ij y_j for each earlier block j as soon
// as that block's ready flag is set (the L tile is loaded before the wait), then solves its
// unit lower 64 x 64 diagonal block (one warp per right-hand side, shuffles), stores y_i and
// sets its own flag with release semantics.  Every wait is bounded in wall time.
constexpr int ZR = 64;   // rows per block
constexpr int ZC = 4;    // right-hand sides per task
constexpr int ZIT = 256;

template <bool MUL>
__global__ void __launch_bounds__(ZIT, 2) zl_kernel(ZArgs z)
{
    __shared__ double Lt[ZR][ZR + 1];
    __shared__ double Ys[ZR][ZC];
    __shared__ int s_ok;
    const int n = z.n, m = z.m;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nblk = (n + ZR - 1) / ZR, ntile = (m + ZC - 1) / ZC;
    const int r = t & (ZR - 1), jr = t >> 6;  // this thread's row in the block and right-hand side
    for (int task = blockIdx.x; task < nblk * ntile; task += gridDim.x) {
        const int ib = task / ntile, c = task - ib * ntile;
        const int i = MUL ? nblk - 1 - ib : ib;  // L y: the longest rows first
        if (tile_done(z.done, z.tol, c * ZC, ZC, m, z.cplx)) continue;  // all of its tasks skip alike
        const int row = i * ZR + r, col = c * ZC + jr;
        const bool live = row < n && col < m;
        double acc = 0.0;
        if (live) {
            if (!MUL && z.gather && z.cplx) {  // part col & 1 of interleaved complex column col >> 1
                const int64_t p = z.perm[row];
                acc = z.src[2 * ((size_t)(col >> 1) * z.lds + (p - 1)) + (col & 1)] * z.iscale[p - 1];
            } else if (!MUL && z.gather) {
                const int64_t p = z.perm[row];
                acc = z.src[(size_t)col * z.lds + (p - 1)] * z.iscale[p - 1];
            } else {
                acc = z.src[(size_t)col * z.lds + row];
            }
        }
        // L tiles are software-pipelined: tile j+1 is in registers while tile j is used
        constexpr int PER = ZR * ZR / ZIT;  // 16 entries per thread
        double lreg[PER];
        const bool dinv = !MUL && z.linv != nullptr;  // mixed form: diagonal blocks by their inverses
        auto load_tile = [&](int j) {
#pragma unroll
            for (int u = 0; u < PER; ++u) {
                const int e = t + u * ZIT;
                const int rr = e & (ZR - 1), qq = e >> 6;
                const int gr = i * ZR + rr, q = j * ZR + qq;
                if (dinv && j == i) {
                    lreg[u] = z.linv[((size_t)i * ZR + rr) * ZR + qq];  // (L_ii)^-1, row-major
                } else {
                    // L[row][q] = F[(q-1) ldf + row] for 1 <= q <= n-2 and row >= q+1, else 0
                    lreg[u] = (gr < n && q >= 1 && q <= n - 2 && gr >= q + 1) ? z.F[(size_t)(q - 1) * z.ldf + gr] : 0.0;
                }
            }
        };
        load_tile(0);
        for (int j = 0; j <= i; ++j) {
#pragma unroll
            for (int u = 0; u < PER; ++u) {
                const int e = t + u * ZIT;
                Lt[e & (ZR - 1)][e >> 6] = lreg[u];
            }
            if (j < i) load_tile(j + 1);
            if (MUL || j < i) {
                if (!MUL) {
                    if (t == 0) {
                        int ok = 1;
                        const int* f = z.flags + (size_t)j * ntile + c;
                        const uint64_t t0 = globaltimer_ns();
                        unsigned spins = 0;
                        while (ld_acquire_i32(f) != 1) {
                            if ((++spins & 63u) == 0) {
                                if (ld_acquire_i32(z.err) != 0) { ok = 0; break; }
                                if (globaltimer_ns() - t0 > z.limit_ns) {
                                    atomicCAS(z.err, 0, (int)LHL_ERR_TIMEOUT);
                                    ok = 0;
                                    break;
                                }
                            }
                        }
                        s_ok = ok;
                    }
                    __syncthreads();
                    if (!s_ok) return;
                }
                {
                    const int qq = t & (ZR - 1), cc = t >> 6;
                    const int q = j * ZR + qq;
                    const double* yb = MUL ? z.src : z.dst;  // L y reads the input; L^-1 y the solved blocks
                    const int ldy = MUL ? z.lds : z.ldd;
                    Ys[qq][cc] = (q < n && c * ZC + cc < m) ? __ldcg(&yb[(size_t)(c * ZC + cc) * ldy + q]) : 0.0;
                }
                __syncthreads();
                double s0 = 0.0, s1 = 0.0;
#pragma unroll 8
                for (int qq = 0; qq < ZR; qq += 2) {
                    s0 = dfma(Lt[r][qq], Ys[qq][jr], s0);
                    s1 = dfma(Lt[r][qq + 1], Ys[qq + 1][jr], s1);
                }
                if (MUL) acc += s0 + s1;
                else acc -= s0 + s1;
                __syncthreads();
            } else if (dinv) {
                // diagonal block: y_i = (L_ii)^-1 acc, a 64 x 64 product
                Ys[r][jr] = acc;
                __syncthreads();
                double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll 4
                for (int qq = 0; qq < ZR; qq += 4) {
                    s0 = dfma(Lt[r][qq], Ys[qq][jr], s0);
                    s1 = dfma(Lt[r][qq + 1], Ys[qq + 1][jr], s1);
                    s2 = dfma(Lt[r][qq + 2], Ys[qq + 2][jr], s2);
                    s3 = dfma(Lt[r][qq + 3], Ys[qq + 3][jr], s3);
                }
                if (live) z.dst[(size_t)col * z.ldd + row] = (s0 + s1) + (s2 + s3);
                __syncthreads();
                if (t == 0) {
                    __threadfence();
                    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(z.flags + (size_t)i * ntile + c), "r"(1)
                                 : "memory");
                }
            } else {
                // diagonal block: unit lower solve, one warp per right-hand side
                Ys[r][jr] = acc;
                __syncthreads();
                if (warp < ZC && c * ZC + warp < m) {
                    double y0 = Ys[lane][warp], y1 = Ys[lane + 32][warp];
                    for (int q = 0; q < ZR - 1; ++q) {
                        const double xq = __shfl_sync(0xffffffffu, q < 32 ? y0 : y1, q & 31);
                        if (lane > q) y0 = dfma(-Lt[lane][q], xq, y0);
                        if (lane + 32 > q) y1 = dfma(-Lt[lane + 32][q], xq, y1);
                    }
                    double* d = z.dst + (size_t)(c * ZC + warp) * z.ldd;
                    if (i * ZR + lane < n) d[i * ZR + lane] = y0;
                    if (i * ZR + lane + 32 < n) d[i * ZR + lane + 32] = y1;
                }
                __syncthreads();
                if (t == 0) {
                    __threadfence();
                    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(z.flags + (size_t)i * ntile + c), "r"(1)
                                 : "memory");
                }
            }
        }
        if (MUL && live) {  // x[perm[row]] = (L y)[row] * scale[perm[row]]
            const int64_t p = z.perm[row];
            if (z.cplx) z.dst[2 * ((size_t)(col >> 1) * z.ldd + (p - 1)) + (col & 1)] = acc * z.scale[p - 1];
            else z.dst[(size_t)col * z.ldd + (p - 1)] = acc * z.scale[p - 1];
        }
    }
}

// Hessenberg solve with the shift's LU (F:2746-2816): forward select-swap steps, then
// U x = y with U[k,j] = Gt[j,k] (j >= k) and rdiag = 1 / U[k,k].
template <int NT = SOLVE_T>
__device__ void hess_solve(const LdivArgs& a, const double* Gt, const uint8_t* swp, const double* rd, double* y,
                           double* sm, uint8_t* ssw)
{
    const int n = a.n;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int k = 1 + t; k <= n - 1; k += NT) {
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
    const int nwarps = NT / 32;
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

// Mixed form: inverses of the unit lower 64 x 64 diagonal blocks of L (shift-independent,
// formed once per reduction), so that the forward substitution's diagonal step is a
// product.  One CTA of 64 threads per block; thread c forms column c by substitution on e_c.
// Stored row-major: linv[(i * 64 + r) * 64 + c].
__global__ void __launch_bounds__(ZR) linv_kernel(int n, const double* __restrict__ F, int ldf,
                                                  double* __restrict__ linv)
{
    extern __shared__ double lsm[];
    double(*T)[ZR + 1] = reinterpret_cast<double(*)[ZR + 1]>(lsm);
    double(*X)[ZR + 1] = reinterpret_cast<double(*)[ZR + 1]>(lsm + ZR * (ZR + 1));
    const int i = blockIdx.x, c = threadIdx.x;
    for (int rr = 0; rr < ZR; ++rr) {  // T[rr][q] = L[row][col] strictly below the diagonal
        const int gr = i * ZR + rr, q = i * ZR + c;
        T[rr][c] = (gr < n && q >= 1 && q <= n - 2 && gr >= q + 1) ? F[(size_t)(q - 1) * ldf + gr] : 0.0;
    }
    __syncthreads();
    for (int rr = 0; rr < ZR; ++rr) {
        double acc = 0.0;
        if (rr == c) acc = 1.0;
        else if (rr > c)
            for (int q = c; q < rr; ++q) acc = dfma(-T[rr][q], X[q][c], acc);
        X[rr][c] = acc;
    }
    __syncthreads();
    for (int rr = 0; rr < ZR; ++rr) linv[((size_t)i * ZR + rr) * ZR + c] = X[rr][c];
}

cudaError_t launch_linv(int n, const double* F, int ldf, double* linv, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    const size_t smem = 2 * (size_t)ZR * (ZR + 1) * sizeof(double);
    static size_t attr[MAX_DEVICES] = {};
    cudaError_t e = opt_in_smem((const void*)linv_kernel, smem, attr);
    if (e != cudaSuccess) return e;
    linv_kernel<<<(n + ZR - 1) / ZR, ZR, smem, st>>>(n, F, ldf, linv);
    return cudaGetLastError();
}

// Mixed form: inverses of the 32 x 32 diagonal blocks of each shift's U (the blocks of the
// back substitution below: rows r0..r1, r1 = n - 32 b), so that the back substitution's
// triangle step is a matrix-vector product instead of a 32-step recurrence.  One warp per
// (shift, block); lane c forms column c of the inverse by substitution on e_c.  Stored
// column by column: element (i, c) at uinv[((s * nblocks + b) * 32 + c) * 32 + i].  Not used by the plain form, whose
// solves keep the backward-stable substitution.
constexpr int UW = 2;  // warps (blocks) per CTA

__global__ void __launch_bounds__(UW * 32) uinv_kernel(int n, const double* __restrict__ Gt_all, int ldg,
                                                      const double* __restrict__ rd_all, int s0,
                                                      double* __restrict__ uinv_all)
{
    __shared__ double T[UW][BS][BS + 1];
    __shared__ double X[UW][BS][BS + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nblocks = (n + BS - 1) / BS;
    const int b = blockIdx.x * UW + warp;
    if (b >= nblocks) return;
    const int s = s0 + blockIdx.y;
    const double* Gt = Gt_all + (size_t)s * ldg * n;
    const double* rd = rd_all + (size_t)s * n;
    const int r1 = n - BS * b, r0 = max(r1 - (BS - 1), 1), bw = r1 - r0 + 1;
    for (int i = 0; i < BS; ++i)  // T[i][j] = U[r0 + i, r0 + j] = Gt[r0 + j, r0 + i]
        T[warp][i][lane] = (i < bw && lane < bw && lane >= i) ? M1(Gt, ldg, r0 + lane, r0 + i) : 0.0;
    __syncwarp();
    for (int i = BS - 1; i >= 0; --i) {
        if (lane < bw && i <= lane) {
            double acc = (i == lane) ? 1.0 : 0.0;
            for (int j = i + 1; j <= lane; ++j) acc = dfma(-T[warp][i][j], X[warp][j][lane], acc);
            X[warp][i][lane] = acc * rd[r0 + i - 1];
        } else {
            X[warp][i][lane] = 0.0;
        }
        __syncwarp();
    }
    double* out = uinv_all + ((size_t)blockIdx.y * nblocks + b) * BS * BS;  // column c at out + 32 c
    for (int c = 0; c < BS; ++c) out[c * BS + lane] = X[warp][lane][c];
}

cudaError_t launch_uinv(int n, const double* Gt, int ldg, const double* rd, int s0, int count, double* uinv,
                        cudaStream_t st)
{
    if (n <= 0 || count <= 0) return cudaSuccess;
    const int nblocks = (n + BS - 1) / BS;
    uinv_kernel<<<dim3((nblocks + UW - 1) / UW, count), UW * 32, 0, st>>>(n, Gt, ldg, rd, s0,
                                                                       uinv + (size_t)s0 * nblocks * BS * BS);
    return cudaGetLastError();
}

// The same Hessenberg solve with Gt streamed by TMA (even n): the back substitution's 32-row
// blocks read their 32 columns of Gt (rows r0..n) as 128 x 32 boxes through a ring of `ns`
// shared-memory slots.  Warp 16 is the producer: it requests boxes in consumption order as
// slots free up (per-slot "full" and "empty" mbarriers), starting before the forward
// recurrence runs.  Warps 0-15 consume, two Gt columns each, and synchronise among
// themselves (named barrier 1) only at block boundaries.  Every wait is bounded in time.
constexpr int HB_ROWS = 128, HB_COLS = 32, HB_MAXSLOTS = 8;
constexpr uint32_t HB_BYTES = HB_ROWS * HB_COLS * sizeof(double);
constexpr int HCONS = 16;                 // consumer warps
constexpr int HT = (HCONS + 1) * 32;      // + one producer warp

__device__ __forceinline__ void cons_sync() { asm volatile("bar.sync 1, %0;" ::"r"(HCONS * 32) : "memory"); }

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Forward select-swap recurrence of the Hessenberg solve (F:2806-2816) as a parallel scan.
// Step k (1..n-1) maps c -> alpha_k c + beta_k: with an interchange x_k = y_k and
// c <- c - l_k y_k (alpha = 1, beta = -l_k y_k); without, x_k = c and c <- y_k - l_k c
// (alpha = -l_k, beta = y_k).  |l_k| <= 1 (the LU's pivoting), so composing the maps is
// stable.  Each of the NT threads composes one contiguous chunk of steps, the chunk maps are
// scanned across the threads (shuffles, then warp totals), and every thread replays its
// chunk from the prefix value.  In place on y (x_k -> y[k-1], the last c -> y[n-1]).
// Called by all NT threads (warps 0..NT/32-1); `sync` synchronises exactly those threads.
template <int NT, class Sync>
__device__ __forceinline__ void forward_scan(int n, double* y, const double* sm, const uint8_t* ssw, double* wA,
                                             double* wB, Sync sync)
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    constexpr int NW = NT / 32;
    const int C = (n - 1 + NT - 1) / NT;
    const int k0 = 1 + t * C, k1 = min(k0 + C, n);  // steps [k0, k1)
    double A = 1.0, B = 0.0;                          // chunk map: c_out = A c_in + B
    for (int k = k0; k < k1; ++k) {
        const double l = sm[k - 1], b = y[k];
        if (ssw[k - 1]) {
            B = B - l * b;
        } else {
            A = -l * A;
            B = b - l * B;
        }
    }
    const double blast = k0 < k1 ? y[k1 - 1] : 0.0;  // the next thread overwrites y[k1-1] below
    // inclusive scan of the maps in thread order: earlier (pA, pB) then own (A, B)
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double pA = __shfl_up_sync(0xffffffffu, A, o), pB = __shfl_up_sync(0xffffffffu, B, o);
        if (lane >= o) {
            B = A * pB + B;
            A = A * pA;
        }
    }
    if (lane == 31) {
        wA[warp] = A;
        wB[warp] = B;
    }
    sync();
    if (warp == 0) {
        double a = lane < NW ? wA[lane] : 1.0, bb = lane < NW ? wB[lane] : 0.0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double pA = __shfl_up_sync(0xffffffffu, a, o), pB = __shfl_up_sync(0xffffffffu, bb, o);
            if (lane >= o) {
                bb = a * pB + bb;
                a = a * pA;
            }
        }
        if (lane < NW) {
            wA[lane] = a;
            wB[lane] = bb;
        }
    }
    sync();
    double eA = __shfl_up_sync(0xffffffffu, A, 1), eB = __shfl_up_sync(0xffffffffu, B, 1);
    if (lane == 0) {
        eA = 1.0;
        eB = 0.0;
    }
    const double pA = warp > 0 ? wA[warp - 1] : 1.0, pB = warp > 0 ? wB[warp - 1] : 0.0;
    double c = eA * (pA * y[0] + pB) + eB;  // c before step k0
    sync();                                 // y[0] and every chunk's last input read
    for (int k = k0; k < k1; ++k) {
        const double l = sm[k - 1], b = k == k1 - 1 ? blast : y[k];
        double x;
        if (ssw[k - 1]) {
            x = b;
            c = c - l * b;
        } else {
            x = c;
            c = b - l * c;
        }
        y[k - 1] = x;
    }
    if (k1 == n && k0 < k1) y[n - 1] = c;
    sync();
}

__global__ void __launch_bounds__(HT) hess_tma_kernel(LdivArgs a, double* Y, int ldy, int col0, int ns,
                                                      const __grid_constant__ CUtensorMap tmG)
{
    extern __shared__ __align__(1024) double hsm[];
    __shared__ __align__(8) uint64_t full[HB_MAXSLOTS], empty[HB_MAXSLOTS];
    __shared__ __align__(16) double Xs[BS * BS];  // mixed form: the current block's inverse
    __shared__ double tri[BS][BS + 1];
    __shared__ double sj[BS];
    __shared__ int s_bad;
    const int n = a.n;
    double* box = hsm;  // ns boxes, column jj of a box at box + jj * HB_ROWS
    double* y = hsm + (size_t)ns * HB_ROWS * HB_COLS;
    double* sm = y + n;
    uint8_t* ssw = (uint8_t*)(sm + n);
    const int col = col0 + blockIdx.x;
    if (a.done && a.done[col] <= a.tol) return;  // converged column: nothing requested yet
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int s = col / a.rhs_per_shift;
    const uint8_t* swp = a.swp + (size_t)s * n;
    const double* rd = a.rdiag + (size_t)s * n;
    const double* Gt = a.Gt + (size_t)s * a.ldg * n;
    // blocks b = 0.. from the bottom: r1 = n - 32 b, r0 = max(r1 - 31, 1) (odd for even n);
    // block b needs ceil((n - r0 + 1) / 128) boxes
    const int nblocks = (n + BS - 1) / BS;
    if (t == 0) {
        for (int u = 0; u < ns; ++u) {
            mbar_init(&full[u], 1);
            mbar_init(&empty[u], HCONS);
        }
        mbar_fence_init();
        s_bad = 0;
    }
    __syncthreads();
    if (warp == HCONS) {
        // ---- producer ----
        if (lane == 0) {
            int u = 0;
            for (int b = 0; b < nblocks && !s_bad; ++b) {
                const int r1 = n - BS * b, r0 = max(r1 - (BS - 1), 1);
                const int nk = (n - r0 + HB_ROWS) / HB_ROWS;
                for (int k = 0; k < nk; ++k, ++u) {
                    const int slot = u % ns;
                    if (u >= ns && !mbar_wait_ns(&empty[slot], (uint32_t)((u / ns - 1) & 1), a.limit_ns)) {
                        atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
                        s_bad = 1;
                        break;
                    }
                    mbar_expect_tx(&full[slot], HB_BYTES);
                    tma_load_2d(box + (size_t)slot * HB_ROWS * HB_COLS, &tmG, r0 - 1 + HB_ROWS * k, s * n + r0 - 1,
                                &full[slot]);
                }
            }
            // drain: wait (bounded) for the last copies of every slot, so that none lands after
            // the block exits (on the normal path they completed long ago)
            for (int v = max(u - ns, 0); v < u; ++v) mbar_wait_ns(&full[v % ns], (uint32_t)((v / ns) & 1), a.limit_ns);
        }
        return;
    }
    // ---- consumers (warps 0-15) ----
    for (int i = t; i < n; i += HCONS * 32) y[i] = Y[(size_t)blockIdx.x * ldy + i];
    for (int k = 1 + t; k <= n - 1; k += HCONS * 32) {
        sm[k - 1] = M1(Gt, a.ldg, k, k + 1);
        ssw[k - 1] = swp[k - 1];
    }
    cons_sync();
    if (n >= 2) forward_scan<HCONS * 32>(n, y, sm, ssw, sj, sj + 16, []() { cons_sync(); });
    cons_sync();
    int u = 0;
    bool bad = false;
    for (int b = 0; b < nblocks; ++b) {
        const int r1 = n - BS * b, r0 = max(r1 - (BS - 1), 1);
        const int bw = r1 - r0 + 1;
        const int nk = (n - r0 + HB_ROWS) / HB_ROWS;
        double acc0 = 0.0, acc1 = 0.0;  // columns jj = warp and warp + 16
        if (a.uinv && warp == 0) {  // mixed form: the block's inverse into shared memory, async
            const char* X = reinterpret_cast<const char*>(a.uinv + ((size_t)s * nblocks + b) * BS * BS);
#pragma unroll
            for (int q = 0; q < BS * BS * 8 / 16 / 32; ++q) {
                const int off = (q * 32 + lane) * 16;
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(reinterpret_cast<char*>(Xs) + off)),
                             "l"(X + off)
                             : "memory");
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
        }
        for (int k = 0; k < nk; ++k, ++u) {
            const int slot = u % ns;
            if (!bad && !mbar_wait_ns(&full[slot], (uint32_t)((u / ns) & 1), a.limit_ns)) {
                atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
                bad = true;
            }
            const double* bx = box + (size_t)slot * HB_ROWS * HB_COLS;
            const int rb = r0 + HB_ROWS * k;  // 1-based row of box row 0
            if (k == 0)
                for (int e = t; e < BS * BS; e += HCONS * 32) {
                    const int jj = e >> 5, rr = e & 31;
                    tri[jj][rr] = bx[jj * HB_ROWS + rr];  // Gt[r0 + rr, r0 + jj] = U[r0 + jj, r0 + rr]
                }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int jj = warp + HCONS * h;
                if (jj < bw) {
                    double p = 0.0;
#pragma unroll
                    for (int rr = lane; rr < HB_ROWS; rr += 32) {
                        const int i = rb + rr;
                        if (i > r1 && i <= n) p = dfma(bx[jj * HB_ROWS + rr], y[i - 1], p);
                    }
                    if (h == 0) acc0 += p;
                    else acc1 += p;
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[slot]);  // this warp is done with the slot
        }
        acc0 = warp_sum(acc0);
        acc1 = warp_sum(acc1);
        if (lane == 0) {
            if (warp < bw) sj[warp] = acc0;
            if (warp + HCONS < bw) sj[warp + HCONS] = acc1;
        }
        cons_sync();
        if (warp == 0 && a.uinv) {
            // x_block = Ub^-1 (y_block - sums): a 32 x 32 matrix-vector product
            const int i = r0 + lane;
            const double rhs = (i <= r1) ? y[i - 1] - sj[lane] : 0.0;
            asm volatile("cp.async.wait_all;" ::: "memory");
            __syncwarp();
            double p0 = 0.0, p1 = 0.0, p2 = 0.0, p3 = 0.0;
#pragma unroll
            for (int c = 0; c < BS; c += 4) {
                p0 = dfma(Xs[c * BS + lane], __shfl_sync(0xffffffffu, rhs, c), p0);
                p1 = dfma(Xs[(c + 1) * BS + lane], __shfl_sync(0xffffffffu, rhs, c + 1), p1);
                p2 = dfma(Xs[(c + 2) * BS + lane], __shfl_sync(0xffffffffu, rhs, c + 2), p2);
                p3 = dfma(Xs[(c + 3) * BS + lane], __shfl_sync(0xffffffffu, rhs, c + 3), p3);
            }
            __syncwarp();  // Xs is refilled at the next block's start
            if (i <= r1) y[i - 1] = (p0 + p1) + (p2 + p3);
        } else if (warp == 0) {
            const int i = r0 + lane;
            double yi = (i <= r1) ? y[i - 1] - sj[lane] : 0.0;
            const double rdi = (i <= r1) ? rd[i - 1] : 0.0;
#pragma unroll
            for (int jj = BS - 1; jj >= 0; --jj) {
                if (jj < bw) {
                    double xj = 0.0;
                    if (lane == jj) {
                        yi = yi * rdi;
                        xj = yi;
                    }
                    xj = __shfl_sync(0xffffffffu, xj, jj);
                    if (lane < jj) yi = dfma(-tri[lane][jj], xj, yi);  // U[r0 + lane, r0 + jj]
                }
            }
            if (i <= r1) y[i - 1] = yi;
        }
        cons_sync();
    }
    if (bad) return;
    for (int i = t; i < n; i += HCONS * 32) Y[(size_t)blockIdx.x * ldy + i] = y[i];
}

// ---- batches of small independent matrices: one CTA per (matrix, shift, right-hand side),
// the solve and its refinement entirely on chip (lhl_solve_batched) ----
// y <- L^-1 y, blocked by 32: the block's triangle staged in shared memory and solved by one
// warp with shuffles, then every thread applies the block to its rows.
template <int NT>
__device__ void small_lsolve(int n, const double* __restrict__ F, double* y)
{
    __shared__ double tri[BS][BS + 1];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int c0 = 2; c0 <= n - 1; c0 += BS) {
        const int cb = min(c0 + BS - 1, n - 1), bw = cb - c0 + 1;
        for (int e = t; e < BS * BS; e += NT) {
            const int r = e & 31, q = e >> 5;  // L[c0 + r, c0 + q] = F[c0 + r, c0 + q - 1]
            if (q < bw && r < bw && r > q) tri[r][q] = M1(F, n, c0 + r, c0 + q - 1);
        }
        __syncthreads();
        if (warp == 0) {
            double yr = lane < bw ? y[c0 + lane - 1] : 0.0;
            for (int q = 0; q < bw - 1; ++q) {
                const double xq = __shfl_sync(0xffffffffu, yr, q);
                if (lane > q && lane < bw) yr = dfma(-tri[lane][q], xq, yr);
            }
            if (lane < bw) y[c0 + lane - 1] = yr;
        }
        __syncthreads();
        for (int i = cb + 1 + t; i <= n; i += NT) {
            double v = y[i - 1];
            for (int q = 0; q < bw; ++q) v = dfma(-M1(F, n, i, c0 + q - 1), y[c0 + q - 1], v);
            y[i - 1] = v;
        }
        __syncthreads();
    }
}

// y <- L y (original y on the right): (L y)[i] = y[i] + sum_{c=2}^{i-1} L[i,c] y[c]
template <int NT>
__device__ void small_lmul(int n, const double* __restrict__ F, double* y, double* y2)
{
    const int t = threadIdx.x;
    for (int i = 1 + t; i <= n; i += NT) {
        double v = y[i - 1];
        for (int c = 2; c <= i - 1; ++c) v = dfma(M1(F, n, i, c - 1), y[c - 1], v);
        y2[i - 1] = v;
    }
    __syncthreads();
    for (int i = t; i < n; i += NT) y[i] = y2[i];
    __syncthreads();
}

template <int NT>
__device__ double block_sum(double v, double* red)
{
    const int t = threadIdx.x;
    v = warp_sum(v);
    __syncthreads();
    if ((t & 31) == 0) red[t >> 5] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < NT / 32; ++w) s += red[w];
    return s;
}

// threads per CTA of the batched solve: one per row of a matrix of order <= 256 (most of config
// 4), four CTAs per SM within the 64-register cap
constexpr int SB_T = 256;

__global__ void __launch_bounds__(SB_T, 4) solve_batch_kernel(BatchDesc d, const double* __restrict__ J,
                                                              const double* __restrict__ B, double* __restrict__ X,
                                                              int R, const double* __restrict__ sig,
                                                              const double* __restrict__ tau, double tol,
                                                              int max_steps, double* __restrict__ res)
{
    const int SR = d.S * R;
    const int m = blockIdx.x / SR, q = blockIdx.x - m * SR, s = q / R;
    const int n = d.n[m];
    if (n <= 0) return;
    __shared__ double xs[512], rs[512], ys[512], ys2[512];
    __shared__ uint8_t ssw[512];
    __shared__ double red[SB_T / 32];
    const int t = threadIdx.x;
    const double* Jm = J + d.off2[m];
    const double* F = d.F + d.off2[m];
    const int64_t* perm = d.perm + d.off1[m];
    const int64_t* iperm = d.iperm + d.off1[m];
    const double* sc = d.scale + d.off1[m];
    const double* isc = d.iscale + d.off1[m];
    const int ldg = n + 4;
    const double* Gt = d.Gt + d.offg[m] + (size_t)s * ldg * n;
    const uint8_t* swp = d.swap + (size_t)d.S * d.off1[m] + (size_t)s * n;
    const double* rd = d.rdiag + (size_t)d.S * d.off1[m] + (size_t)s * n;
    const double sigma = sig[(size_t)m * d.S + s], tauv = tau[(size_t)m * d.S + s];
    const double* b = B + (size_t)SR * d.off1[m] + (size_t)q * n;
    double* x = X + (size_t)SR * d.off1[m] + (size_t)q * n;
    LdivArgs la;
    la.n = n;
    la.ldg = ldg;
    // v <- W^-1 v in place (F:3052-3068)
    auto solve = [&](double* v) {
        for (int i = t; i < n; i += SB_T) {
            const int64_t p = perm[i];
            ys[i] = v[p - 1] * isc[p - 1];
        }
        __syncthreads();
        small_lsolve<SB_T>(n, F, ys);
        hess_solve<SB_T>(la, Gt, swp, rd, ys, ys2, ssw);
        small_lmul<SB_T>(n, F, ys, ys2);
        for (int i = t; i < n; i += SB_T) v[i] = ys[iperm[i] - 1] * sc[i];
        __syncthreads();
    };
    double bb = 0.0;
    for (int i = t; i < n; i += SB_T) {
        const double v = b[i];
        xs[i] = v;
        bb = dfma(v, v, bb);
    }
    const double bnorm = sqrt(block_sum<SB_T>(bb, red));
    __syncthreads();
    solve(xs);  // x = W^-1 b
    double rel = 0.0;
    for (int it = 0; it <= max_steps; ++it) {
        // r = b - (sigma x + tau J x), FP64 with the caller's J
        double rr = 0.0;
        for (int i = t; i < n; i += SB_T) {
            double acc = 0.0;
            for (int j = 0; j < n; ++j) acc = dfma(Jm[(size_t)j * n + i], xs[j], acc);
            const double r = b[i] - (sigma * xs[i] + tauv * acc);
            rs[i] = r;
            rr = dfma(r, r, rr);
        }
        const double rn = sqrt(block_sum<SB_T>(rr, red));
        rel = bnorm > 0.0 ? rn / bnorm : rn;
        if (rel <= tol || it == max_steps) break;
        __syncthreads();
        solve(rs);
        for (int i = t; i < n; i += SB_T) xs[i] += rs[i];
        __syncthreads();
    }
    for (int i = t; i < n; i += SB_T) x[i] = xs[i];
    if (t == 0 && res) res[blockIdx.x] = rel;
}

cudaError_t launch_solve_batch(const BatchDesc& d, const double* J, const double* B, double* X, int R,
                               const double* sig, const double* tau, double tol, int max_steps, double* res,
                               cudaStream_t st)
{
    if (d.count <= 0 || d.S <= 0 || R <= 0) return cudaSuccess;
    solve_batch_kernel<<<d.count * d.S * R, SB_T, 0, st>>>(d, J, B, X, R, sig, tau, tol, max_steps, res);
    return cudaGetLastError();
}

// Columns from which the 64-wide tensor-pipe sweeps (zlw_kernel) replace zl_kernel's 4-wide tasks.
constexpr int ZW_MIN_COLUMNS = 1024;
static cudaError_t run_zinv_wide(ZArgs z, cudaStream_t st);

static cudaError_t run_zinv(ZArgs z, cudaStream_t st)
{
    if (z.m >= ZW_MIN_COLUMNS) return run_zinv_wide(z, st);
    const int nblk = (z.n + ZR - 1) / ZR, ntile = (z.m + ZC - 1) / ZC;
    if ((size_t)nblk * ntile > (size_t)z.nflags) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(z.flags, 0, (size_t)nblk * ntile * sizeof(int), st);
    if (e != cudaSuccess) return e;
    static int maxgrid_of[MAX_DEVICES] = {};
    int dev = 0;
    e = current_device(&dev);
    if (e != cudaSuccess) return e;
    if (maxgrid_of[dev] == 0) {
        int sms = 0, per = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, zl_kernel<false>, ZIT, 0);
        maxgrid_of[dev] = sms * (per > 0 ? per : 1);
    }
    const int grid = min(nblk * ntile, maxgrid_of[dev]);
    void* args[] = {&z};
    return cudaLaunchCooperativeKernel((void*)zl_kernel<false>, dim3(grid), dim3(ZIT), args, 0, st);
}

// x <- D P L y: independent tasks (row block, 4 right-hand sides), no flags; the blocks of
// the last rows (the most work) are handed out first.
// ---- the same sweeps for many right-hand sides: tiles of 64 rows x 64 columns on the FP64
// tensor pipe ----
// zl_kernel re-reads each 64 x 64 tile of L once per four right-hand sides; with thousands of
// them (config 5's 4096 complex vectors are 8192 real columns) that is hundreds of GB of L2
// traffic per sweep.  Here a task owns 64 rows x 64 columns, so a tile of L serves 64
// columns, and the products L_ij y_j run as mma.sync m8n8k4 FP64 (eight warps, each 32 rows x
// 16 columns: 4 x 2 tiles of 8 x 8), with the L and y tiles staged by cp.async in K chunks of 32 (double buffered,
// padded so that fragment loads hit 16 distinct 8-byte banks per half-warp).  The structure is
// zl_kernel's: MUL = false is the blocked forward substitution over a cooperative grid with
// ready flags per (row block, column tile), tasks block-major; the unit lower diagonal block is
// then solved one column per lane group (plain form: substitution with shuffles) or multiplied
// by its precomputed inverse (mixed form); MUL = true has no dependencies.
constexpr int ZWR = 64;          // rows per block (the L blocks of zl_kernel)
constexpr int ZWC = 64;          // columns per task
constexpr int ZWK = 32;          // K chunk
constexpr int ZWT = 256;
constexpr int ZWAP = ZWR + 4, ZWBP = ZWC + 4;
struct ZwSmem {
    double A[2][ZWK][ZWAP];  // L tile [q][row]
    double B[2][ZWK][ZWBP];  // y tile [q][column]
    double D[ZWR][ZWC + 1];  // diagonal block: the block's values [row][column]
    int ok;
};

template <bool MUL>
__global__ void __launch_bounds__(ZWT, 2) zlw_kernel(ZArgs z)
{
    extern __shared__ __align__(16) unsigned char zw_raw[];
    ZwSmem& sm = *reinterpret_cast<ZwSmem*>(zw_raw);
    const int n = z.n, m = z.m;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wm = warp & 1, wn = warp >> 1;  // warp tile: rows 32 wm .., columns 16 wn ..
    const int g = lane >> 2, t4 = lane & 3;
    const int nblk = (n + ZWR - 1) / ZWR, ntile = (m + ZWC - 1) / ZWC;
    const bool dinv = !MUL && z.linv != nullptr;
    for (int task = blockIdx.x; task < nblk * ntile; task += gridDim.x) {
        const int ib = task / ntile, c = task - ib * ntile;
        const int i = MUL ? nblk - 1 - ib : ib;
        if (tile_done(z.done, z.tol, c * ZWC, ZWC, m, z.cplx)) continue;
        double acc[4][2][2];
        // initial values: the gathered x (L^-1 sweep) or y itself (L sweep), at this thread's
        // fragment positions (row 32 wm + 8 a + g, column 16 wn + 8 b + 2 t4 + e)
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int row = i * ZWR + 32 * wm + 8 * a + g;
                    const int col = c * ZWC + 16 * wn + 8 * b + 2 * t4 + e;
                    double v = 0.0;
                    if (row < n && col < m) {
                        if (!MUL && z.gather && z.cplx) {
                            const int64_t p = z.perm[row];
                            v = z.src[2 * ((size_t)(col >> 1) * z.lds + (p - 1)) + (col & 1)] * z.iscale[p - 1];
                        } else if (!MUL && z.gather) {
                            const int64_t p = z.perm[row];
                            v = z.src[(size_t)col * z.lds + (p - 1)] * z.iscale[p - 1];
                        } else {
                            v = z.src[(size_t)col * z.lds + row];
                        }
                    }
                    acc[a][b][e] = v;
                }
        const double sgn = MUL ? 1.0 : -1.0;
        const double* yb = MUL ? z.src : z.dst;  // L y reads the input; L^-1 y the solved blocks
        const int ldy = MUL ? z.lds : z.ldd;
        // products with the blocks j < i (L^-1 sweep) or j <= i (L sweep; L's diagonal is
        // stored as zero and the unit part is the initial value above)
        const int jend = MUL ? i : i - 1;
        // block j's readiness (its flag, set when that block of this column tile is solved); the
        // wait is bounded and ends the kernel with LHL_ERR_TIMEOUT
        auto ready = [&](int j) -> bool {
            if (MUL) return true;
            if (t == 0) {
                int ok = 1;
                const int* f = z.flags + (size_t)j * ntile + c;
                const uint64_t t0 = globaltimer_ns();
                unsigned spins = 0;
                while (ld_acquire_i32(f) != 1) {
                    if ((++spins & 63u) == 0) {
                        if (ld_acquire_i32(z.err) != 0) { ok = 0; break; }
                        if (globaltimer_ns() - t0 > z.limit_ns) {
                            atomicCAS(z.err, 0, (int)LHL_ERR_TIMEOUT);
                            ok = 0;
                            break;
                        }
                    }
                }
                sm.ok = ok;
            }
            __syncthreads();
            return sm.ok != 0;
        };
        auto stage = [&](int q, int st) {  // K chunk q: half q & 1 (columns 32 (q & 1) ..) of block q >> 1
            const int j = q >> 1, h = q & 1;
            for (int e = t; e < ZWK * ZWR; e += ZWT) {
                const int rr = e % ZWR, qq = e / ZWR;
                const int gr = i * ZWR + rr, k = j * ZWR + h * ZWK + qq;
                // L[gr][k] = F[(k-1) ldf + gr] for 1 <= k <= n-2 and gr >= k+1, else 0
                const bool ok = gr < n && k >= 1 && k <= n - 2 && gr >= k + 1;
                cp_async8(&sm.A[st][qq][rr], ok ? &z.F[(size_t)(k - 1) * z.ldf + gr] : z.F, ok, z.F);
            }
            for (int e = t; e < ZWK * ZWC; e += ZWT) {
                const int qq = e % ZWK, cc = e / ZWK;
                const int k = j * ZWR + h * ZWK + qq, col = c * ZWC + cc;
                const bool ok = k < n && col < m;
                cp_async8(&sm.B[st][qq][cc], ok ? &yb[(size_t)col * ldy + k] : z.F, ok, z.F);
            }
            cp_async_commit();
        };
        // products with the blocks j < i (L^-1 sweep) or j <= i (L sweep; L's diagonal is
        // stored as zero and the unit part is the initial value above), as one stream of K
        // chunks over the two stages: chunk q + 1 (the next block's first half included) is in
        // flight while chunk q is multiplied
        const int nq = 2 * (jend + 1);
        if (nq > 0) {
            if (!ready(0)) return;
            stage(0, 0);
        }
        for (int q = 0; q < nq; ++q) {
            const int st = q & 1;
            if (q + 1 < nq) {
                if (((q + 1) & 1) == 0 && !ready((q + 1) >> 1)) {
                    cp_async_wait<0>();  // nothing of this CTA's stays in flight into shared memory
                    return;
                }
                stage(q + 1, st ^ 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < ZWK; kk += 4) {
                double fa[4], fb[2];
#pragma unroll
                for (int a = 0; a < 4; ++a) fa[a] = sgn * sm.A[st][kk + t4][32 * wm + 8 * a + g];
#pragma unroll
                for (int b = 0; b < 2; ++b) fb[b] = sm.B[st][kk + t4][16 * wn + 8 * b + g];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 2; ++b) dmma_8x8x4(acc[a][b], fa[a], fb[b]);
            }
            __syncthreads();  // stage st is refilled by the next iteration's copy
        }
        if constexpr (MUL) {  // x[perm[row]] = (L y)[row] * scale[perm[row]]
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int row = i * ZWR + 32 * wm + 8 * a + g;
                        const int col = c * ZWC + 16 * wn + 8 * b + 2 * t4 + e;
                        if (row < n && col < m) {
                            const int64_t p = z.perm[row];
                            if (z.cplx)
                                z.dst[2 * ((size_t)(col >> 1) * z.ldd + (p - 1)) + (col & 1)] = acc[a][b][e] * z.scale[p - 1];
                            else
                                z.dst[(size_t)col * z.ldd + (p - 1)] = acc[a][b][e] * z.scale[p - 1];
                        }
                    }
        } else {
        // ---- the diagonal block: unit lower L_ii, values of this block in sm.D ----
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int e = 0; e < 2; ++e) sm.D[32 * wm + 8 * a + g][16 * wn + 8 * b + 2 * t4 + e] = acc[a][b][e];
        // L_ii (strictly lower part, or its inverse) into sm.A as [row][q] pairs of halves
        double* Lii = &sm.A[0][0][0];  // 64 x 65 doubles, row-major, fits in the two A stages
        for (int e = t; e < ZWR * ZWR; e += ZWT) {
            const int rr = e % ZWR, qq = e / ZWR;
            const int gr = i * ZWR + rr, q = i * ZWR + qq;
            double v;
            if (dinv) v = z.linv[((size_t)i * ZWR + rr) * ZWR + qq];  // (L_ii)^-1, row-major
            else v = (gr < n && q >= 1 && q <= n - 2 && gr >= q + 1) ? z.F[(size_t)(q - 1) * z.ldf + gr] : 0.0;
            Lii[rr * (ZWR + 1) + qq] = v;
        }
        __syncthreads();
        if (dinv) {
            // y_i = (L_ii)^-1 D: one column per thread quarter, 64-term dot products
            for (int e = t; e < ZWR * ZWC; e += ZWT) {
                const int rr = e % ZWR, cc = e / ZWR;
                double s0 = 0.0, s1 = 0.0;
#pragma unroll 8
                for (int q = 0; q < ZWR; q += 2) {
                    s0 = dfma(Lii[rr * (ZWR + 1) + q], sm.D[q][cc], s0);
                    s1 = dfma(Lii[rr * (ZWR + 1) + q + 1], sm.D[q + 1][cc], s1);
                }
                const int row = i * ZWR + rr, col = c * ZWC + cc;
                if (row < n && col < m) z.dst[(size_t)col * z.ldd + row] = s0 + s1;
            }
        } else {
            // forward substitution: warp w solves columns 8w .. 8w+7; lane holds rows lane, lane+32
            double y0[8], y1[8];
#pragma unroll
            for (int v = 0; v < 8; ++v) {
                y0[v] = sm.D[lane][8 * warp + v];
                y1[v] = sm.D[lane + 32][8 * warp + v];
            }
            for (int q = 0; q < ZWR - 1; ++q) {
                const double l0 = Lii[lane * (ZWR + 1) + q], l1 = Lii[(lane + 32) * (ZWR + 1) + q];
#pragma unroll
                for (int v = 0; v < 8; ++v) {
                    const double xq = __shfl_sync(0xffffffffu, q < 32 ? y0[v] : y1[v], q & 31);
                    if (lane > q) y0[v] = dfma(-l0, xq, y0[v]);
                    if (lane + 32 > q) y1[v] = dfma(-l1, xq, y1[v]);
                }
            }
#pragma unroll
            for (int v = 0; v < 8; ++v) {
                const int col = c * ZWC + 8 * warp + v;
                if (col < m) {
                    double* d = z.dst + (size_t)col * z.ldd;
                    if (i * ZWR + lane < n) d[i * ZWR + lane] = y0[v];
                    if (i * ZWR + lane + 32 < n) d[i * ZWR + lane + 32] = y1[v];
                }
            }
        }
        __syncthreads();
        if (t == 0) {
            __threadfence();
            asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(z.flags + (size_t)i * ntile + c), "r"(1)
                         : "memory");
        }
        }
    }
}

static cudaError_t run_zinv_wide(ZArgs z, cudaStream_t st)
{
    const int nblk = (z.n + ZWR - 1) / ZWR, ntile = (z.m + ZWC - 1) / ZWC;
    if ((size_t)nblk * ntile > (size_t)z.nflags) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(z.flags, 0, (size_t)nblk * ntile * sizeof(int), st);
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(ZwSmem);
    static int maxgrid_of[MAX_DEVICES] = {};
    int dev = 0;
    e = current_device(&dev);
    if (e != cudaSuccess) return e;
    if (maxgrid_of[dev] == 0) {
        e = cudaFuncSetAttribute(zlw_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int sms = 0, per = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, zlw_kernel<false>, ZWT, smem);
        maxgrid_of[dev] = sms * (per > 0 ? per : 1);
    }
    const int grid = min(nblk * ntile, maxgrid_of[dev]);
    void* args[] = {&z};
    return cudaLaunchCooperativeKernel((void*)zlw_kernel<false>, dim3(grid), dim3(ZWT), args, smem, st);
}

static cudaError_t run_zmul(const ZArgs& z, cudaStream_t st)
{
    if (z.m >= ZW_MIN_COLUMNS) {
        const size_t smem = sizeof(ZwSmem);
        static size_t attr[MAX_DEVICES] = {};
        cudaError_t e = opt_in_smem((const void*)zlw_kernel<true>, smem, attr);
        if (e != cudaSuccess) return e;
        const int nblk = (z.n + ZWR - 1) / ZWR, ntile = (z.m + ZWC - 1) / ZWC;
        zlw_kernel<true><<<nblk * ntile, ZWT, smem, st>>>(z);
        return cudaGetLastError();
    }
    const int nblk = (z.n + ZR - 1) / ZR, ntile = (z.m + ZC - 1) / ZC;
    zl_kernel<true><<<nblk * ntile, ZIT, 0, st>>>(z);
    return cudaGetLastError();
}

cudaError_t launch_ldiv(const LdivArgs& a, int nrhs, cudaStream_t st)
{
    if (nrhs <= 0 || a.n <= 0) return cudaSuccess;
    if (a.cj) return launch_ldiv_cj(a, nrhs, st);  // complex reduction: complex L (cplxj.cu)
    ZArgs z;
    memset(&z, 0, sizeof(z));
    z.n = a.n;
    z.F = a.F;
    z.ldf = a.ldf;
    z.perm = a.perm;
    z.scale = a.scale;
    z.iscale = a.iscale;
    z.flags = a.zflags;
    z.nflags = a.nzflags;
    z.err = a.err;
    z.limit_ns = a.limit_ns;
    z.tol = a.tol;
    z.linv = a.linv;
    if (!a.Y || a.ycap <= 0 || !a.zflags || !a.err) return cudaErrorInvalidValue;
    if (a.mode == 0 && a.cplx) {
        // complex shift on a real reduction: each complex right-hand side is two real columns
        // of Y (its planes) for the L sweeps (F:3092-3104)
        const int chunk = a.ycap / 2;
        for (int c0 = 0; c0 < nrhs; c0 += chunk) {
            const int cnt = min(chunk, nrhs - c0);
            z.cplx = 1;
            z.src = a.X + 2 * (size_t)c0 * a.ldx; z.lds = a.ldx; z.dst = a.Y; z.ldd = a.n; z.m = 2 * cnt;
            z.gather = 1;
            z.done = a.done ? a.done + c0 : nullptr;
            cudaError_t e = run_zinv(z, st);
            // several right-hand sides per shift: one CTA per group of them streams the shift's
            // Gt once for the group; otherwise one CTA per right-hand side
            if (e == cudaSuccess && a.rhs_per_shift >= 4)
                e = launch_hess_cplx_mrhs(a.n, a.Gt, a.ldg, a.po, a.swp, a.rdiag, a.Y, a.n, c0, cnt,
                                          a.rhs_per_shift, a.done, a.tol, st, a.tail, a.err, a.limit_ns);
            else if (e == cudaSuccess)
                e = launch_hess_cplx(a.n, a.Gt, a.ldg, a.po, a.swp, a.rdiag, a.Y, a.n, c0, cnt, a.rhs_per_shift,
                                     a.done, a.tol, st);
            if (e != cudaSuccess) return e;
            z.src = a.Y; z.lds = a.n; z.dst = a.X + 2 * (size_t)c0 * a.ldx; z.ldd = a.ldx; z.gather = 0;
            e = run_zmul(z, st);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    if (a.mode == 1) {  // applyZinv: x <- L^-1 P^-1 D^-1 x, through the scratch
        for (int c0 = 0; c0 < nrhs; c0 += a.ycap) {
            const int cnt = min(a.ycap, nrhs - c0);
            z.src = a.X + (size_t)c0 * a.ldx; z.lds = a.ldx; z.dst = a.Y; z.ldd = a.n; z.m = cnt; z.gather = 1;
            cudaError_t e = run_zinv(z, st);
            if (e == cudaSuccess)
                e = cudaMemcpy2DAsync(a.X + (size_t)c0 * a.ldx, (size_t)a.ldx * sizeof(double), a.Y,
                                      (size_t)a.n * sizeof(double), (size_t)a.n * sizeof(double), cnt,
                                      cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    if (a.mode == 2) {  // applyZ: x <- D P L x, through the scratch (CTAs split the rows)
        for (int c0 = 0; c0 < nrhs; c0 += a.ycap) {
            const int cnt = min(a.ycap, nrhs - c0);
            cudaError_t e = cudaMemcpy2DAsync(a.Y, (size_t)a.n * sizeof(double), a.X + (size_t)c0 * a.ldx,
                                              (size_t)a.ldx * sizeof(double), (size_t)a.n * sizeof(double), cnt,
                                              cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return e;
            z.src = a.Y; z.lds = a.n; z.dst = a.X + (size_t)c0 * a.ldx; z.ldd = a.ldx; z.m = cnt; z.gather = 0;
            e = run_zmul(z, st);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    const size_t hsm = (size_t)a.n * 2 * sizeof(double) + (size_t)a.n + 16;
    // dynamic + static shared memory must stay within the 227 KB a CTA may use
    if (hsm > 200 * 1024) return cudaErrorInvalidValue;
    static size_t attr[MAX_DEVICES] = {};
    if (hsm > 32 * 1024) {  // the kernel's static shared arrays add about 8.5 KB
        cudaError_t e = opt_in_smem((const void*)hess_kernel, hsm, attr);
        if (e != cudaSuccess) return e;
    }
    // Gt through TMA: even n (16-byte row pitch and box origins) and room for >= 2 slots
    const size_t vec = (size_t)a.n * 2 * sizeof(double) + (size_t)a.n + 16;
    const int ns = (int)min((size_t)HB_MAXSLOTS, vec < 210 * 1024 ? (210 * 1024 - vec) / HB_BYTES : (size_t)0);
    const size_t tsm = (size_t)ns * HB_BYTES + vec;
    CUtensorMap tmG;
    bool use_tma = (a.n % 2 == 0) && a.n >= 2 && ns >= 2 && a.nshifts > 0 &&
                   make_tmap_2d(&tmG, a.Gt, a.ldg, a.nshifts * a.n, a.ldg, HB_ROWS, HB_COLS);
    if (use_tma) {
        static size_t tattr[MAX_DEVICES] = {};
        if (opt_in_smem((const void*)hess_tma_kernel, tsm, tattr) != cudaSuccess) use_tma = false;
    }
    for (int c0 = 0; c0 < nrhs; c0 += a.ycap) {
        const int cnt = min(a.ycap, nrhs - c0);
        z.src = a.X + (size_t)c0 * a.ldx; z.lds = a.ldx; z.dst = a.Y; z.ldd = a.n; z.m = cnt; z.gather = 1;
        z.done = a.done ? a.done + c0 : nullptr;
        cudaError_t e = run_zinv(z, st);
        if (e != cudaSuccess) return e;
        if (use_tma) hess_tma_kernel<<<cnt, HT, tsm, st>>>(a, a.Y, a.n, c0, ns, tmG);
        else hess_kernel<<<cnt, SOLVE_T, hsm, st>>>(a, a.Y, a.n, c0);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        z.src = a.Y; z.lds = a.n; z.dst = a.X + (size_t)c0 * a.ldx; z.ldd = a.ldx; z.gather = 0;
        e = run_zmul(z, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// ---- residual r = b - (sigma_s I + tau_s J) x: tiles of 16 rows x 64 right-hand sides ----
// 256 threads, thread (row r = t % 16, columns 4 (t / 16) .. +3); k in chunks of 64 through
// shared memory, the next chunk prefetched into registers while the current one is used.
constexpr int RM = 16, RK = 64, RTT = 256;

template <int CPT>  // columns per thread: tiles of 16 CPT right-hand sides
__global__ void __launch_bounds__(RTT) residual_kernel(int n, const double* __restrict__ J, int ldj,
                                                       const double* __restrict__ B, int ldb,
                                                       const double* __restrict__ X, int ldx, double* __restrict__ R,
                                                       int ldr, int nrhs, int rhs_per_shift,
                                                       const double* __restrict__ sig, const double* __restrict__ tau,
                                                       const double* __restrict__ done, double tol)
{
    constexpr int RN = 16 * CPT;
    __shared__ double Js[RK][RM + 1];
    __shared__ double Xs[RK][RN + 1];
    const int i0 = blockIdx.x * RM, c0 = blockIdx.y * RN;
    if (tile_done(done, tol, c0, RN, nrhs)) return;  // converged columns keep their residual
    const int t = threadIdx.x;
    const int r = t % RM, cg = t / RM;  // cg in 0..15, columns cg*CPT ..
    constexpr int JPER = RM * RK / RTT, XPER = RK * RN / RTT;  // 4 and 16
    double jr[JPER], xr[XPER];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int u = 0; u < JPER; ++u) {
            const int e = t + u * RTT;
            const int ii = e % RM, kk = e / RM;  // J rows contiguous
            const int i = i0 + ii, k = k0 + kk;
            jr[u] = (i < n && k < n) ? J[(size_t)k * ldj + i] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < XPER; ++u) {
            const int e = t + u * RTT;
            const int kk = e % RK, cc = e / RK;  // X columns contiguous
            const int k = k0 + kk, c = c0 + cc;
            xr[u] = (k < n && c < nrhs) ? X[(size_t)c * ldx + k] : 0.0;
        }
    };
    double acc[CPT];
#pragma unroll
    for (int q = 0; q < CPT; ++q) acc[q] = 0.0;
    fetch(0);
    for (int k0 = 0; k0 < n; k0 += RK) {
#pragma unroll
        for (int u = 0; u < JPER; ++u) {
            const int e = t + u * RTT;
            Js[e / RM][e % RM] = jr[u];
        }
#pragma unroll
        for (int u = 0; u < XPER; ++u) {
            const int e = t + u * RTT;
            Xs[e % RK][e / RK] = xr[u];
        }
        __syncthreads();
        if (k0 + RK < n) fetch(k0 + RK);
#pragma unroll 16
        for (int kk = 0; kk < RK; ++kk) {
            const double jv = Js[kk][r];
#pragma unroll
            for (int q = 0; q < CPT; ++q) acc[q] = dfma(jv, Xs[kk][cg * CPT + q], acc[q]);
        }
        __syncthreads();
    }
    const int i = i0 + r;
    if (i < n) {
#pragma unroll
        for (int q = 0; q < CPT; ++q) {
            const int c = c0 + cg * CPT + q;
            if (c < nrhs) {
                const int s = c / rhs_per_shift;
                const double xv = X[(size_t)c * ldx + i];
                const double bv = B ? B[(size_t)c * ldb + i] : 0.0;  // no B: R = -W X
                R[(size_t)c * ldr + i] = bv - (sig[s] * xv + tau[s] * acc[q]);
            }
        }
    }
}

cudaError_t launch_residual(int n, const double* J, int ldj, const double* B, int ldb, const double* X, int ldx,
                            double* R, int ldr, int nrhs, int rhs_per_shift, const double* sig, const double* tau,
                            cudaStream_t st, const double* done, double tol)
{
    if (nrhs <= 0 || n <= 0) return cudaSuccess;
    if (done) {  // refinement steps: narrow tiles, so that converged columns cost nothing
        dim3 grid((n + RM - 1) / RM, (nrhs + 15) / 16);
        residual_kernel<1><<<grid, RTT, 0, st>>>(n, J, ldj, B, ldb, X, ldx, R, ldr, nrhs, rhs_per_shift, sig, tau, done,
                                                 tol);
    } else {
        dim3 grid((n + RM - 1) / RM, (nrhs + 63) / 64);
        residual_kernel<4><<<grid, RTT, 0, st>>>(n, J, ldj, B, ldb, X, ldx, R, ldr, nrhs, rhs_per_shift, sig, tau, done,
                                                 tol);
    }
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
