// complex.cu -- complex shifts on a real reduction (LHLShift{ComplexF64} on
// LHLWorkspace{Float64}): the shift LU of G = sigma I + tau H with complex sigma, tau
// (F:2529-2594 with TG = ComplexF64), its planar Hessenberg solve (F:2823-2910) and the
// complex residual of lhl_refine! (F:3144-3157).  The L sweeps of the solve are the real
// ones (solve.cu), applied to the two planes as two real right-hand sides.
//
// Layout: Gt is planar, (2 po) x n per shift: real parts in rows 1..n, imaginary parts in
// rows po+1..po+n of each column (po = n + 4 rounded up to even).  rdiag, sigma, tau and
// every complex vector of the C ABI are interleaved (re, im) pairs, as CuArray{ComplexF64}.
//
// Arithmetic is Julia's Complex arithmetic written out on the parts, every operation
// rounded separately (no fused multiply-adds): (a+bi)(c+di) = (ac - bd) + (ad + bc)i,
// complex x real scales both parts, the pivot magnitude is |re| + |im| (F:2519-2520).
// Division is Baudin & Smith's robust complex division (the one Julia's Base uses for
// ComplexF64, without its rescaling near overflow and underflow); rdiag = 1 / U[j,j] by the
// same division.  The CPU oracle uses the same operations in the same order, so the device
// shift LU is bit-identical to it.
#include "cplx.cuh"
#include "internal.cuh"

namespace lhl {

// ---- shift LU, one CTA per shift (the real kernel's structure, shift.cu) ----
// HV = double: complex shifts on a real Ht; HV = dc: a complex reduction's Ht (interleaved).
__device__ __forceinline__ void ht_load(const double* Ht, int ldh, int j, int k, double& v) { v = M1(Ht, ldh, j, k); }
__device__ __forceinline__ void ht_load(const double* Ht, int ldh, int j, int k, dc& v)
{
    const double2 w = reinterpret_cast<const double2*>(Ht)[(size_t)(k - 1) * ldh + (j - 1)];
    v = {w.x, w.y};
}
template <class HV> __device__ __forceinline__ HV hzero();
template <> __device__ __forceinline__ double hzero<double>() { return 0.0; }
template <> __device__ __forceinline__ dc hzero<dc>() { return {0.0, 0.0}; }

template <int T, int E, class HV>
__global__ void __launch_bounds__(T, 1) shift_lu_cplx_kernel(int n, const double* __restrict__ Ht, int ldh,
                                                          const double* __restrict__ sig, const double* __restrict__ tau_,
                                                          int s0, double* __restrict__ Gt_all, int ldg, int po,
                                                          uint8_t* __restrict__ swap_all, double* __restrict__ rdiag_all,
                                                          int32_t* __restrict__ info_all)
{
    const int s = s0 + blockIdx.x;
    const dc sigma = {sig[2 * blockIdx.x], sig[2 * blockIdx.x + 1]};
    const dc tau = {tau_[2 * blockIdx.x], tau_[2 * blockIdx.x + 1]};
    double* Gt = Gt_all + (size_t)s * ldg * n;
    uint8_t* swp = swap_all + (size_t)s * n;
    double* rdiag = rdiag_all + (size_t)s * 2 * n;
    const int t = threadIdx.x;
    __shared__ dc s_next[2];
    __shared__ dc s_l[2], s_a[2], s_b[2];
    __shared__ int s_sw[2];
    __shared__ int s_info;

    dc r[E];
    HV h[E];  // Ht[j, k+1] for the current step, reloaded in place for the next one
    // Ht[j, j+1] for the one element j whose pivot decision this thread takes next (step j,
    // taken during step j - 1): loaded a step ahead by the owner of element k + 2
    HV hs = hzero<HV>();
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int j = 1 + t + e * T;
        HV h1 = hzero<HV>();
        if (j <= n) ht_load(Ht, ldh, j, 1, h1);
        r[e] = (j <= n) ? tmul(tau, h1) : dc{0.0, 0.0};
        if (j == 1) r[e] = cadd(r[e], sigma);
        h[e] = hzero<HV>();
        if (j <= n && n >= 2) ht_load(Ht, ldh, j, 2, h[e]);
        if (j == 2 && j + 1 <= n) ht_load(Ht, ldh, j, j + 1, hs);  // decides step 2, during step 1
    }
    auto decide = [&](int k, dc a, HV hs) {
        const dc b = tmul(tau, hs);
        const bool sw = cmag(b) > cmag(a);
        dc l;
        if (sw) l = cdiv(a, b);
        else if (a.re == 0.0 && a.im == 0.0) l = {0.0, 0.0};
        else l = cdiv(b, a);
        s_l[k & 1] = l;
        s_a[k & 1] = a;
        s_b[k & 1] = b;
        s_sw[k & 1] = sw ? 1 : 0;
    };
    if (t == 0) {
        s_next[1] = r[0];
        s_info = 0;
        if (n >= 2) {
            HV h12 = hzero<HV>();
            ht_load(Ht, ldh, 1, 2, h12);
            decide(1, r[0], h12);
        }
    }
    __syncthreads();
    for (int k = 1; k <= n - 1; ++k) {
        const dc l = s_l[k & 1];
        const bool sw = s_sw[k & 1] != 0;
        if (t == 0) {
            const dc a = s_a[k & 1], b = s_b[k & 1];
            const dc d = sw ? b : a;
            swp[k - 1] = sw ? 1 : 0;
            M1(Gt, ldg, k, k) = d.re;
            M1(Gt, ldg, po + k, k) = d.im;
            M1(Gt, ldg, k, k + 1) = l.re;
            M1(Gt, ldg, po + k, k + 1) = l.im;
            if (!sw && a.re == 0.0 && a.im == 0.0 && s_info == 0) s_info = k;
        }
        // the subdiagonal entry of the decision this thread takes next step (element k + 2)
        HV hs_next = hs;
        if (k + 3 <= n && (k + 1) % T == t) ht_load(Ht, ldh, k + 2, k + 3, hs_next);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int j = 1 + t + e * T;
            if (j >= k + 1 && j <= n) {
                dc gk;
                if (sw) {
                    const dc g = tmul(tau, h[e]);
                    gk = g;
                    dc rj = csub(r[e], cmul(l, g));
                    if (j == k + 1) {
                        gk = cadd(g, sigma);              // Gt[k+1,k] += sigma
                        rj = csub(rj, cmul(l, sigma));    // r[k+1] -= l*sigma
                    }
                    r[e] = rj;
                } else {
                    const dc rj = r[e];
                    gk = rj;
                    dc rn = csub(tmul(tau, h[e]), cmul(l, rj));
                    if (j == k + 1) rn = cadd(rn, sigma); // r[k+1] += sigma
                    r[e] = rn;
                }
                M1(Gt, ldg, j, k) = gk.re;
                M1(Gt, ldg, po + j, k) = gk.im;
                if (j == k + 1) {  // owner of element k+1: publish it and decide step k+1
                    s_next[(k + 1) & 1] = r[e];
                    if (k + 1 <= n - 1) decide(k + 1, r[e], hs);
                }
            }
            // Ht[j, k+2] for the next step, into the same register
            if (j >= k + 1 && j <= n && k + 2 <= n) ht_load(Ht, ldh, j, k + 2, h[e]);
        }
        hs = hs_next;
        __syncthreads();
    }
    if (t == 0) {  // finish (F:2579-2594)
        const dc rn = s_next[n & 1];
        M1(Gt, ldg, n, n) = rn.re;
        M1(Gt, ldg, po + n, n) = rn.im;
        swp[n - 1] = 0;
        int info = s_info;
        if (rn.re == 0.0 && rn.im == 0.0 && info == 0) info = n;
        info_all[s] = info;
    }
    __syncthreads();
    for (int j = 1 + t; j <= n; j += T) {
        const dc q = cdiv(dc{1.0, 0.0}, dc{M1(Gt, ldg, j, j), M1(Gt, ldg, po + j, j)});
        rdiag[2 * (j - 1)] = q.re;
        rdiag[2 * (j - 1) + 1] = q.im;
    }
}

// Launch shapes of the complex shift LU (threads T, elements per thread E), selectable per
// workspace like the real ones (same bits for every shape); shape v serves n <= T E.
static const int kCShiftShapes[][2] = {{256, 1}, {512, 2}, {512, 4}, {512, 8}, {1024, 8}, {1024, 2}, {1024, 4}, {256, 4},
                                        {512, 16}, {256, 32}};
constexpr int kNumCShiftShapes = sizeof(kCShiftShapes) / sizeof(kCShiftShapes[0]);

int shift_shape_cplx(int variant, int* T, int* E)
{
    if (variant < 1 || variant > kNumCShiftShapes) return 0;
    *T = kCShiftShapes[variant - 1][0];
    *E = kCShiftShapes[variant - 1][1];
    return 1;
}

cudaError_t launch_shift_lu_cplx(int n, const double* Ht, int ldh, const double* sig, const double* tau, int s0,
                                 int count, double* Gt, int ldg, int po, uint8_t* swp, double* rd, int32_t* info,
                                 cudaStream_t st, int ht_complex, int variant)
{
    if (count <= 0 || n <= 0) return cudaSuccess;
#define L_(T, E)                                                                                                  \
    do {                                                                                                          \
        if (ht_complex)                                                                                           \
            shift_lu_cplx_kernel<T, E, dc><<<count, T, 0, st>>>(n, Ht, ldh, sig, tau, s0, Gt, ldg, po, swp, rd, info); \
        else                                                                                                      \
            shift_lu_cplx_kernel<T, E, double><<<count, T, 0, st>>>(n, Ht, ldh, sig, tau, s0, Gt, ldg, po, swp, rd,  \
                                                                    info);                                        \
    } while (0)
    if (variant > 0) {
        int T, E;
        if (!shift_shape_cplx(variant, &T, &E) || T * E < n) return cudaErrorInvalidValue;
        switch (variant) {
            case 1: L_(256, 1); break;
            case 2: L_(512, 2); break;
            case 3: L_(512, 4); break;
            case 4: L_(512, 8); break;
            case 5: L_(1024, 8); break;
            case 6: L_(1024, 2); break;
            case 7: L_(1024, 4); break;
            case 8: L_(256, 4); break;
            case 9: L_(512, 16); break;
            case 10: L_(256, 32); break;
            default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
    if (n <= 256) L_(256, 1);
    else if (n <= 1024) L_(512, 2);
    else if (n <= 2048) L_(512, 4);
    else if (n <= 4096) L_(512, 8);
    else if (n <= 8192) L_(512, 16);
    else return cudaErrorInvalidValue;
#undef L_
    return cudaGetLastError();
}

// ---- planar Hessenberg solve, one CTA per complex right-hand side ----
// Y holds each complex right-hand side as two real columns (real parts in column 2c,
// imaginary parts in column 2c + 1, leading dimension ldy), as the L sweeps left them.
constexpr int CT = 512;
constexpr int CB = 32;

__global__ void __launch_bounds__(CT) hess_cplx_kernel(int n, const double* __restrict__ Gt_all, int ldg, int po,
                                                       const uint8_t* __restrict__ swap_all,
                                                       const double* __restrict__ rdiag_all, double* Y, int ldy,
                                                       int col0, int rhs_per_shift, const double* __restrict__ done,
                                                       double tol)
{
    extern __shared__ double csm[];
    const int cc = col0 + blockIdx.x;  // complex right-hand side
    if (done && done[cc] <= tol) return;
    const int n_ = n;
    double* yr = csm;
    double* yi = csm + n_;
    __shared__ double tr_[CB][CB + 1], ti_[CB][CB + 1];
    __shared__ double sjr[CB], sji[CB];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int s = cc / rhs_per_shift;
    const double* Gt = Gt_all + (size_t)s * ldg * n_;
    const uint8_t* swp = swap_all + (size_t)s * n_;
    const double* rd = rdiag_all + (size_t)s * 2 * n_;
    double* Yr = Y + (size_t)(2 * blockIdx.x) * ldy;
    double* Yi = Y + (size_t)(2 * blockIdx.x + 1) * ldy;
    for (int i = t; i < n_; i += CT) {
        yr[i] = Yr[i];
        yi[i] = Yi[i];
    }
    __syncthreads();
    if (t == 0 && n_ >= 2) {  // forward select-swap recurrence (F:2827-2838), complex multipliers
        dc c = {yr[0], yi[0]};
        for (int k = 1; k <= n_ - 1; ++k) {
            const dc b = {yr[k], yi[k]};
            const bool sw = swp[k - 1] != 0;
            const dc xk = sw ? b : c;
            yr[k - 1] = xk.re;
            yi[k - 1] = xk.im;
            const dc lk = {M1(Gt, ldg, k, k + 1), M1(Gt, ldg, po + k, k + 1)};
            c = csub(sw ? c : b, cmul(lk, xk));
        }
        yr[n_ - 1] = c.re;
        yi[n_ - 1] = c.im;
    }
    __syncthreads();
    // back substitution in blocks of 32 rows from the bottom, left-looking: complex dot
    // products with the contiguous columns of both planes of Gt, then a warp solves the block
    const int nwarps = CT / 32;
    for (int r1 = n_; r1 >= 1; r1 -= CB) {
        const int r0 = max(r1 - CB + 1, 1);
        const int bs = r1 - r0 + 1;
        for (int jj = warp; jj < bs; jj += nwarps) {
            const int j = r0 + jj;
            const double* gr = Gt + (size_t)(j - 1) * ldg;  // real plane of column j = row j of U
            const double* gi = gr + po;
            if (r0 + lane <= r1) {
                tr_[jj][lane] = gr[r0 + lane - 1];
                ti_[jj][lane] = gi[r0 + lane - 1];
            }
            double ar = 0.0, ai = 0.0;
            for (int i = r1 + 1 + lane; i <= n_; i += 32) {
                const double xr = yr[i - 1], xi = yi[i - 1], g_r = gr[i - 1], g_i = gi[i - 1];
                ar += g_r * xr - g_i * xi;
                ai += g_r * xi + g_i * xr;
            }
            ar = warp_sum(ar);
            ai = warp_sum(ai);
            if (lane == 0) {
                sjr[jj] = ar;
                sji[jj] = ai;
            }
        }
        __syncthreads();
        if (warp == 0) {
            const int i = r0 + lane;
            dc yv = (i <= r1) ? csub(dc{yr[i - 1], yi[i - 1]}, dc{sjr[lane], sji[lane]}) : dc{0.0, 0.0};
            const dc rdi = (i <= r1) ? dc{rd[2 * (i - 1)], rd[2 * (i - 1) + 1]} : dc{0.0, 0.0};
            for (int j = r1; j >= r0; --j) {
                dc xj = {0.0, 0.0};
                if (i == j) {
                    yv = cmul(yv, rdi);
                    xj = yv;
                }
                xj.re = __shfl_sync(0xffffffffu, xj.re, j - r0);
                xj.im = __shfl_sync(0xffffffffu, xj.im, j - r0);
                if (i < j && i >= r0) {  // U[i, j] = Gt[j, i] (staged as tr_[i - r0][j - r0])
                    const dc u = {tr_[lane][j - r0], ti_[lane][j - r0]};
                    yv = csub(yv, cmul(u, xj));
                }
            }
            if (i <= r1) {
                yr[i - 1] = yv.re;
                yi[i - 1] = yv.im;
            }
        }
        __syncthreads();
    }
    for (int i = t; i < n_; i += CT) {
        Yr[i] = yr[i];
        Yi[i] = yi[i];
    }
}

cudaError_t launch_hess_cplx(int n, const double* Gt, int ldg, int po, const uint8_t* swp, const double* rd,
                             double* Y, int ldy, int col0, int count, int rhs_per_shift, const double* done,
                             double tol, cudaStream_t st)
{
    if (count <= 0 || n <= 0) return cudaSuccess;
    const size_t smem = (size_t)2 * n * sizeof(double);
    if (smem > 150 * 1024) return cudaErrorInvalidValue;
    static size_t attr[MAX_DEVICES] = {};  // opt in for any size: the static tiles (17 KB) come on top of it
    cudaError_t e = opt_in_smem((const void*)hess_cplx_kernel, smem, attr);
    if (e != cudaSuccess) return e;
    hess_cplx_kernel<<<count, CT, smem, st>>>(n, Gt, ldg, po, swp, rd, Y, ldy, col0, rhs_per_shift, done, tol);
    return cudaGetLastError();
}

// ---- planar Hessenberg solve of several right-hand sides of one shift per CTA ----
// The same solve as hess_cplx_kernel (F:2823-2884) for a group of up to MG complex
// right-hand sides that share a shift, so that the shift's Gt (0.5 GB per plane pair at
// n = 8192) is streamed once per group instead of once per right-hand side.  The vectors stay
// in the scratch Y (global memory, L2-resident); the CTA works on them in place:
//   1. the forward select-swap recurrence (F:2827-2838), one thread per right-hand side, on
//      chunks of 32 steps staged in shared memory by the whole CTA;
//   2. the back substitution in blocks of 32 rows from the bottom, left-looking: for block b
//      the products U[b, j] x[j] over the solved rows j below it form a real GEMM
//          [Re S  Im S] (32 x 2 MG) = [Re U  Im U] (32 x 2K) [[Re X, Im X]; [-Im X, Re X]]
//      run as mma.sync m8n8k4 FP64 tiles: K in chunks of 64 staged by cp.async (double
//      buffered, pitches chosen so that fragment loads hit 16 distinct 8-byte banks per
//      half-warp), each warp a share of the chunk's k-steps over the whole 32 x 16 output,
//      the eight warps' sums added in a fixed order; then one warp per right-hand side solves
//      the 32 x 32 triangle with rdiag (shuffles, as the one-vector kernel does).
// Results agree with the one-vector kernel to rounding (the summation order differs).
constexpr int MG = 8;        // complex right-hand sides per CTA
constexpr int MT = 256;      // threads
constexpr int MRB = 32;      // rows per back-substitution block
constexpr int MKC = 64;      // K chunk
constexpr int MUP = MKC + 4; // row pitch of the staged U tile (= 4 mod 16 doubles)
constexpr int MXP = MKC + 4; // pitch of the staged x tile (= 4 mod 16 doubles)
constexpr int MFC = 32;      // forward-recurrence chunk (steps)
constexpr int MW8 = MT / 32; // warps
struct MrhsSmem {
    union {  // used in turn: the K chunks, then the warps' sums, then the diagonal block
        double U[2][2][MRB][MUP];          // [stage][plane][row][k]
        double red[MW8][MRB][2 * MG + 1];  // the warps' block sums [warp][row][part * MG + rhs]
        double T[2][MRB][MRB + 1];         // diagonal block U_bb: [plane][row][col]
    };
    double X[2][2][MG][MXP];     // [stage][part][rhs][k]
    double D[2][MRB][MG + 1];    // block sums: [part][row][rhs]
    double F[2][MFC + 1][MG];    // forward recurrence: y chunk [part][step][rhs]
    double FL[2][MFC];           // forward recurrence: multipliers l_k [part][step]
    unsigned char FS[MFC];       // forward recurrence: swaps
};

// the few-groups path of the solve (hess_cplx_tail_kernel, below)
constexpr int HT_MAX = 16;  // active groups the grid takes on, each on its own share of the CTAs
constexpr int HT_T = 256;   // threads per CTA
constexpr int HT_BAR = 32;  // the plan's words for the groups' barrier counters (HT_MAX of them)
constexpr int HT_WORDS = 64;

// The forward select-swap recurrence (F:2827-2838) of ng <= MG complex right-hand sides of one
// shift, in place in their scratch columns (part p of right-hand side v: Yg + (2 v + p) ldy):
// chunks of MFC steps staged in shared memory by the CTA's NT threads, then one thread per
// right-hand side through the chunk.  Every thread of the CTA calls it.
template <int NT>
__device__ __forceinline__ void hess_cplx_forward(int n, const double* __restrict__ Gt, int ldg, int po,
                                                  const uint8_t* __restrict__ swp, double* Yg, int ldy, int ng,
                                                  double (&F)[2][MFC + 1][MG], double (&FL)[2][MFC],
                                                  unsigned char (&FS)[MFC])
{
    const int t = threadIdx.x;
    auto col = [&](int v, int p) { return Yg + (size_t)(2 * v + p) * ldy; };
    if (n >= 2) {
        dc c = {0.0, 0.0};
        if (t < ng) c = {col(t, 0)[0], col(t, 1)[0]};
        for (int k0 = 1; k0 <= n - 1; k0 += MFC) {
            const int cnt = min(MFC, n - k0);  // steps k0 .. k0 + cnt - 1
            // stage y[k] (0-based index k, k = k0 .. k0+cnt-1), l_k and swap_k
            for (int e = t; e < 2 * MG * MFC; e += NT) {
                const int i = e % MFC, v = (e / MFC) % MG, p = e / (MFC * MG);
                F[p][i][v] = (i < cnt && v < ng) ? col(v, p)[k0 + i] : 0.0;
            }
            if (t < 2 * MFC) {
                const int i = t % MFC, p = t / MFC;
                const int k = k0 + i;
                FL[p][i] = i < cnt ? M1(Gt, ldg, p * po + k, k + 1) : 0.0;
            }
            if (t < MFC) FS[t] = t < cnt ? swp[k0 + t - 1] : 0;
            __syncthreads();
            if (t < ng) {
                for (int i = 0; i < cnt; ++i) {
                    const dc b = {F[0][i][t], F[1][i][t]};
                    const bool sw = FS[i] != 0;
                    const dc xk = sw ? b : c;
                    F[0][i][t] = xk.re;  // becomes y[k - 1]
                    F[1][i][t] = xk.im;
                    const dc lk = {FL[0][i], FL[1][i]};
                    c = csub(sw ? c : b, cmul(lk, xk));
                }
            }
            __syncthreads();
            for (int e = t; e < 2 * MG * MFC; e += NT) {  // y[k-1] for k = k0 .. k0+cnt-1
                const int i = e % MFC, v = (e / MFC) % MG, p = e / (MFC * MG);
                if (i < cnt && v < ng) col(v, p)[k0 + i - 1] = F[p][i][v];
            }
            __syncthreads();
        }
        if (t < ng) {
            col(t, 0)[n - 1] = c.re;
            col(t, 1)[n - 1] = c.im;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(MT, 2) hess_cplx_mrhs_kernel(int n, const double* __restrict__ Gt_all, int ldg,
                                                               int po, const uint8_t* __restrict__ swap_all,
                                                               const double* __restrict__ rdiag_all, double* Y,
                                                               int ldy, int col0, int count, int rhs_per_shift,
                                                               int s_first, int groups_per_shift,
                                                               const double* __restrict__ done, double tol,
                                                               const int* __restrict__ plan)
{
    if (plan && plan[0] <= HT_MAX) return;  // hess_cplx_tail_kernel has the work (or none is left)
    extern __shared__ __align__(16) unsigned char mrhs_raw[];
    MrhsSmem& sm = *reinterpret_cast<MrhsSmem*>(mrhs_raw);
    const int s = s_first + blockIdx.x / groups_per_shift;
    const int g = blockIdx.x % groups_per_shift;
    // this CTA's complex right-hand sides: [c_lo, c_hi) of the chunk (global indices)
    const int c_lo = max(col0, s * rhs_per_shift + g * MG);
    const int c_hi = min(min(col0 + count, (s + 1) * rhs_per_shift), s * rhs_per_shift + g * MG + MG);
    if (c_lo >= c_hi) return;
    const int ng = c_hi - c_lo;
    if (done) {
        bool all = true;
        for (int c = c_lo; c < c_hi; ++c) all = all && (done[c] <= tol);
        if (all) return;
    }
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const double* Gt = Gt_all + (size_t)s * ldg * n;
    const uint8_t* swp = swap_all + (size_t)s * n;
    const double* rd = rdiag_all + (size_t)s * 2 * n;
    // part p of right-hand side v (0 <= v < ng): column 2 (c_lo - col0 + v) + p of Y
    auto ycol = [&](int v, int p) -> double* { return Y + (size_t)(2 * (c_lo - col0 + v) + p) * ldy; };

    // ---- 1. forward recurrence, chunks of MFC steps: element k (1-based) of the chunk at row k0 + i
    hess_cplx_forward<MT>(n, Gt, ldg, po, swp, ycol(0, 0), ldy, ng, sm.F, sm.FL, sm.FS);

    // ---- 2. back substitution
    const int g8 = lane >> 2, t4 = lane & 3;  // mma fragment coordinates
    const bool vec16 = (n % 2) == 0 && ((ldg | po | ldy) % 2) == 0 &&
                       (reinterpret_cast<uintptr_t>(Gt_all) % 16) == 0 && (reinterpret_cast<uintptr_t>(Y) % 16) == 0;
    for (int r1 = n; r1 >= 1; r1 -= MRB) {
        const int r0 = max(r1 - MRB + 1, 1);
        const int bs = r1 - r0 + 1;
        // acc[a][b]: rows 8 a + g8 of the block; b = 0: real parts, b = 1: imaginary parts of
        // right-hand sides 2 t4, 2 t4 + 1
        double acc[4][2][2];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
        const int K = n - r1;  // solved rows r1+1 .. n
        const int nch = (K + MKC - 1) / MKC;
        // even n: every row of a chunk starts on an odd index (1-based), so the pairs (j, j+1)
        // are 16-byte aligned in Gt (ldg and po even) and in Y (ldy = n): 16-byte copies
        auto stage = [&](int ch, int st) {
            const int j0 = r1 + 1 + ch * MKC;  // first row (1-based) of the chunk
            if (vec16) {
                for (int e = t; e < MRB * MKC; e += MT) {  // 2 planes x 32 rows x 32 pairs
                    const int kk = 2 * (e % (MKC / 2)), a = (e / (MKC / 2)) % MRB, p = e / (MKC / 2 * MRB);
                    const int j = j0 + kk;
                    const int bytes = (a < bs && j <= n) ? (j + 1 <= n ? 16 : 8) : 0;
                    cp_async16(&sm.U[st][p][a][kk], bytes ? &M1(Gt, ldg, p * po + j, r0 + a) : Gt, bytes, Gt);
                }
                for (int e = t; e < MKC * MG; e += MT) {  // 2 parts x 8 vectors x 32 pairs
                    const int kk = 2 * (e % (MKC / 2)), v = (e / (MKC / 2)) % MG, p = e / (MKC / 2 * MG);
                    const int j = j0 + kk;
                    const int bytes = (v < ng && j <= n) ? (j + 1 <= n ? 16 : 8) : 0;
                    cp_async16(&sm.X[st][p][v][kk], bytes ? &ycol(v, p)[j - 1] : Gt, bytes, Gt);
                }
            } else {
                for (int e = t; e < 2 * MRB * MKC; e += MT) {
                    const int kk = e % MKC, a = (e / MKC) % MRB, p = e / (MKC * MRB);
                    const int j = j0 + kk;
                    const bool ok = a < bs && j <= n;
                    cp_async8(&sm.U[st][p][a][kk], ok ? &M1(Gt, ldg, p * po + j, r0 + a) : Gt, ok, Gt);
                }
                for (int e = t; e < 2 * MKC * MG; e += MT) {
                    const int kk = e % MKC, v = (e / MKC) % MG, p = e / (MKC * MG);
                    const int j = j0 + kk;
                    const bool ok = v < ng && j <= n;
                    cp_async8(&sm.X[st][p][v][kk], ok ? &ycol(v, p)[j - 1] : Gt, ok, Gt);
                }
            }
            cp_async_commit();
        };
        if (nch > 0) stage(0, 0);
        for (int ch = 0; ch < nch; ++ch) {
            const int st = ch & 1;
            if (ch + 1 < nch) {
                stage(ch + 1, st ^ 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            // this warp's k-steps of the chunk: kk = 4 (warp + 8 u), u = 0, 1, in both planes
#pragma unroll
            for (int u = 0; u < MKC / (4 * MW8); ++u) {
                const int kk = 4 * (warp + MW8 * u) + t4;
                const double xr = sm.X[st][0][g8][kk], xi = sm.X[st][1][g8][kk];
                double far[4], fai[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    far[a] = sm.U[st][0][8 * a + g8][kk];
                    fai[a] = sm.U[st][1][8 * a + g8][kk];
                }
                // two passes over the eight accumulators, so that the two products into one
                // accumulator are eight instructions apart (each waits for the previous result)
                const double nxi = -xi;
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    dmma_8x8x4(acc[a][0], far[a], xr);   // Re U Re x
                    dmma_8x8x4(acc[a][1], far[a], xi);   // Re U Im x
                }
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    dmma_8x8x4(acc[a][0], fai[a], nxi);  // - Im U Im x
                    dmma_8x8x4(acc[a][1], fai[a], xr);   // Im U Re x
                }
            }
            __syncthreads();  // the stage this chunk used is refilled two chunks on
        }
        // the eight warps' sums, added in a fixed order (the U stages are free now)
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int e = 0; e < 2; ++e) sm.red[warp][8 * a + g8][b * MG + 2 * t4 + e] = acc[a][b][e];
        __syncthreads();
        for (int e = t; e < MRB * 2 * MG; e += MT) {
            const int row = e % MRB, col = e / MRB;  // col = part * MG + rhs
            double sum = 0.0;
#pragma unroll
            for (int w = 0; w < MW8; ++w) sum += sm.red[w][row][col];
            sm.D[col / MG][row][col % MG] = sum;
        }
        __syncthreads();
        // diagonal block U[r0 + a, r0 + b] = Gt[r0 + b, r0 + a] (b >= a), both planes
        for (int e = t; e < 2 * MRB * MRB; e += MT) {
            const int bb = e % MRB, a = (e / MRB) % MRB, p = e / (MRB * MRB);
            sm.T[p][a][bb] = (a < bs && bb < bs && bb >= a) ? M1(Gt, ldg, p * po + r0 + bb, r0 + a) : 0.0;
        }
        __syncthreads();
        // triangle: warp v solves right-hand side v
        if (warp < ng) {
            const int v = warp;
            const int i = r0 + lane;  // this lane's row
            dc yv = {0.0, 0.0}, rdi = {0.0, 0.0};
            if (i <= r1) {
                yv = csub(dc{ycol(v, 0)[i - 1], ycol(v, 1)[i - 1]}, dc{sm.D[0][lane][v], sm.D[1][lane][v]});
                rdi = dc{rd[2 * (i - 1)], rd[2 * (i - 1) + 1]};
            }
            for (int j = r1; j >= r0; --j) {
                dc xj = {0.0, 0.0};
                if (i == j) {
                    yv = cmul(yv, rdi);
                    xj = yv;
                }
                xj.re = __shfl_sync(0xffffffffu, xj.re, j - r0);
                xj.im = __shfl_sync(0xffffffffu, xj.im, j - r0);
                if (i < j) yv = csub(yv, cmul(dc{sm.T[0][lane][j - r0], sm.T[1][lane][j - r0]}, xj));
            }
            if (i <= r1) {
                ycol(v, 0)[i - 1] = yv.re;
                ycol(v, 1)[i - 1] = yv.im;
            }
        }
        __syncthreads();  // x of this block is in Y before the next block's K chunks read it
    }
}

// ---- the planar Hessenberg solve when only a few groups of right-hand sides still refine ----
// After the first refinement steps only the right-hand sides of shifts near the spectrum stay
// above the tolerance, and one CTA per group (hess_cplx_mrhs_kernel) streams its shift's whole
// planar Gt at one SM's rate: about 21 ms at n = 8192 however few vectors are left.  With at
// most HT_MAX groups active, a cooperative grid of one CTA per SM takes them all at once, the
// CTAs dealt out to the groups (CTA c to group c mod A, at least 9 CTAs per group), each group
// with its own bounded barrier:
//   * the forward recurrence of the group (its CTA 0, hess_cplx_forward), then a barrier;
//   * the back substitution right-looking, in blocks of 32 rows from the bottom, block q owned
//     by the group's CTA q mod G: the owner solves the block's triangle (rdiag, shuffles, as the
//     multi-vector kernel does) and a barrier makes x_q visible; then every CTA of the group
//     subtracts U[i, block q] x_q from the rows i of the blocks it owns above q (a row of U is a
//     contiguous column of Gt: each lane streams its own row, both planes).  The owner of block
//     q+1 has that block's rows complete after its own update and solves it: one barrier per
//     block.
// hess_tail_plan_kernel counts the active groups first; the multi-vector kernel returns at once
// when this kernel takes the work, and this one when it does not.  Results agree with the
// multi-vector kernel's to rounding (the sums run in another order).

__global__ void hess_tail_plan_kernel(int col0, int count, int rhs_per_shift, int s_first, int gps, int ngroups,
                                      const double* __restrict__ done, double tol, int* __restrict__ plan)
{
    __shared__ int s_cnt;
    __shared__ int s_ids[HT_MAX];
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    for (int gid = threadIdx.x; gid < ngroups; gid += blockDim.x) {
        const int s = s_first + gid / gps, g = gid % gps;
        const int c_lo = max(col0, s * rhs_per_shift + g * MG);
        const int c_hi = min(min(col0 + count, (s + 1) * rhs_per_shift), s * rhs_per_shift + g * MG + MG);
        bool act = false;  // the multi-vector kernel's test: some column not at the tolerance
        for (int c = c_lo; c < c_hi; ++c) act = act || !(done[c] <= tol);
        if (act) {
            const int slot = atomicAdd(&s_cnt, 1);
            if (slot < HT_MAX) s_ids[slot] = gid;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int m = min(s_cnt, HT_MAX);
        for (int i = 1; i < m; ++i)  // ascending, so the groups are taken in a fixed order
            for (int j = i; j > 0 && s_ids[j - 1] > s_ids[j]; --j) {
                const int x = s_ids[j];
                s_ids[j] = s_ids[j - 1];
                s_ids[j - 1] = x;
            }
        plan[0] = s_cnt;
        for (int i = 0; i < HT_MAX; ++i) plan[1 + i] = i < m ? s_ids[i] : -1;
        for (int i = 0; i < HT_MAX; ++i) plan[HT_BAR + i] = 0;
    }
}

struct TailSmem {
    double F[2][MFC + 1][MG];   // forward recurrence (CTA 0)
    double FL[2][MFC];
    unsigned char FS[MFC];
    double X[2][MRB][MG];       // x of the block just solved: [part][row][rhs]
    double T[2][MRB][MRB + 1];  // the diagonal block being solved: [plane][row][col]
};

__global__ void __launch_bounds__(HT_T, 1) hess_cplx_tail_kernel(int n, const double* __restrict__ Gt_all, int ldg,
                                                                 int po, const uint8_t* __restrict__ swap_all,
                                                                 const double* __restrict__ rdiag_all, double* Y,
                                                                 int ldy, int col0, int count, int rhs_per_shift,
                                                                 int s_first, int gps, int* plan, int* err,
                                                                 unsigned long long limit_ns)
{
    __shared__ TailSmem sm;
    __shared__ int s_ok;
    const int A = plan[0];
    if (A <= 0 || A > HT_MAX || (int)gridDim.x < A) return;  // the multi-vector kernel has the work
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    // CTA blockIdx.x takes group a = blockIdx.x mod A, as CTA b of that group's G CTAs
    const int a = blockIdx.x % A, b = blockIdx.x / A, G = ((int)gridDim.x - a + A - 1) / A;
    unsigned int* counter = reinterpret_cast<unsigned int*>(plan + HT_BAR + a);
    unsigned int seq = 0;
    // barrier of the group's G CTAs, bounded in wall time like GridBarrier
    auto group_sync = [&]() -> bool {
        ++seq;
        __syncthreads();
        if (t == 0) {
            int ok = 1;
            __threadfence();
            atomicAdd(counter, 1u);
            const unsigned int target = seq * (unsigned)G;
            const uint64_t t0 = globaltimer_ns();
            unsigned int spins = 0;
            while (ld_acquire_u32(counter) < target) {
                if (ld_acquire_i32(err) != 0) { ok = 0; break; }
                if ((++spins & 63u) == 0 && globaltimer_ns() - t0 > limit_ns) {
                    atomicCAS(err, 0, (int)LHL_ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
            if (ok && ld_acquire_i32(err) != 0) ok = 0;
            __threadfence();
            s_ok = ok;
        }
        __syncthreads();
        return s_ok != 0;
    };
    const int nq = (n + MRB - 1) / MRB;
    {
        const int gid = plan[1 + a];
        const int s = s_first + gid / gps, g = gid % gps;
        const int c_lo = max(col0, s * rhs_per_shift + g * MG);
        const int c_hi = min(min(col0 + count, (s + 1) * rhs_per_shift), s * rhs_per_shift + g * MG + MG);
        const int ng = c_hi - c_lo;
        const double* Gt = Gt_all + (size_t)s * ldg * n;
        const uint8_t* swp = swap_all + (size_t)s * n;
        const double* rd = rdiag_all + (size_t)s * 2 * n;
        double* Yg = Y + (size_t)2 * (c_lo - col0) * ldy;
        auto col = [&](int v, int p) { return Yg + (size_t)(2 * v + p) * ldy; };

        if (b == 0) hess_cplx_forward<HT_T>(n, Gt, ldg, po, swp, Yg, ldy, ng, sm.F, sm.FL, sm.FS);
        if (!group_sync()) return;

        // the triangle of block q (rows r0 .. r1, 1-based), by its owner: every thread calls it
        auto solve_block = [&](int q) {
            const int r1 = n - MRB * q, r0 = max(r1 - MRB + 1, 1), bs = r1 - r0 + 1;
            for (int e = t; e < 2 * MRB * MRB; e += HT_T) {
                const int bb = e % MRB, aa = (e / MRB) % MRB, p = e / (MRB * MRB);
                sm.T[p][aa][bb] = (aa < bs && bb < bs && bb >= aa) ? M1(Gt, ldg, p * po + r0 + bb, r0 + aa) : 0.0;
            }
            __syncthreads();
            if (warp < ng) {  // warp v solves right-hand side v
                const int v = warp;
                const int i = r0 + lane;
                dc yv = {0.0, 0.0}, rdi = {0.0, 0.0};
                if (i <= r1) {
                    yv = {col(v, 0)[i - 1], col(v, 1)[i - 1]};
                    rdi = {rd[2 * (i - 1)], rd[2 * (i - 1) + 1]};
                }
                for (int j = r1; j >= r0; --j) {
                    dc xj = {0.0, 0.0};
                    if (i == j) {
                        yv = cmul(yv, rdi);
                        xj = yv;
                    }
                    xj.re = __shfl_sync(0xffffffffu, xj.re, j - r0);
                    xj.im = __shfl_sync(0xffffffffu, xj.im, j - r0);
                    if (i < j) yv = csub(yv, cmul(dc{sm.T[0][lane][j - r0], sm.T[1][lane][j - r0]}, xj));
                }
                if (i <= r1) {
                    col(v, 0)[i - 1] = yv.re;
                    col(v, 1)[i - 1] = yv.im;
                }
            }
            __syncthreads();
        };
        if (b == 0) solve_block(0);  // the bottom block has nothing below it
        if (!group_sync()) return;
        for (int q = 0; q + 1 < nq; ++q) {
            const int r1 = n - MRB * q, r0 = max(r1 - MRB + 1, 1), bs = r1 - r0 + 1;
            for (int e = t; e < 2 * MRB * MG; e += HT_T) {  // x_q, solved by another CTA
                const int jj = e % MRB, v = (e / MRB) % MG, p = e / (MRB * MG);
                sm.X[p][jj][v] = (jj < bs && v < ng) ? __ldcg(&col(v, p)[r0 + jj - 1]) : 0.0;
            }
            __syncthreads();
            // this CTA's blocks above q (q' > q, q' = b mod G): warp w takes every (HT_T/32)-th
            const int first = q + 1 + ((b - (q + 1)) % G + G) % G;
            for (int qq = first + warp * G; qq < nq; qq += (HT_T / 32) * G) {
                const int s1 = n - MRB * qq, s0 = max(s1 - MRB + 1, 1);
                const int i = s0 + lane;  // this lane's row
                if (i <= s1) {
                    dc acc[MG];
#pragma unroll
                    for (int v = 0; v < MG; ++v) acc[v] = {0.0, 0.0};
                    const double* ur = &M1(Gt, ldg, r0, i);       // U[i, r0 ..] = Gt[r0 .., i], real plane
                    const double* ui = &M1(Gt, ldg, po + r0, i);  // and imaginary plane
                    for (int jj = 0; jj < bs; ++jj) {
                        const dc u = {ur[jj], ui[jj]};
#pragma unroll
                        for (int v = 0; v < MG; ++v) acc[v] = cadd(acc[v], cmul(u, dc{sm.X[0][jj][v], sm.X[1][jj][v]}));
                    }
#pragma unroll
                    for (int v = 0; v < MG; ++v)
                        if (v < ng) {
                            col(v, 0)[i - 1] -= acc[v].re;
                            col(v, 1)[i - 1] -= acc[v].im;
                        }
                }
            }
            __syncthreads();
            if (b == (q + 1) % G) solve_block(q + 1);
            if (!group_sync()) return;
        }
    }
}

cudaError_t launch_hess_cplx_mrhs(int n, const double* Gt, int ldg, int po, const uint8_t* swp, const double* rd,
                                  double* Y, int ldy, int col0, int count, int rhs_per_shift, const double* done,
                                  double tol, cudaStream_t st, int* tail, int* err, unsigned long long limit_ns)
{
    if (count <= 0 || n <= 0) return cudaSuccess;
    const int s_first = col0 / rhs_per_shift, s_last = (col0 + count - 1) / rhs_per_shift;
    const int gps = (rhs_per_shift + MG - 1) / MG;
    const long long grid = (long long)(s_last - s_first + 1) * gps;
    if (grid > 0x7fffffffll) return cudaErrorInvalidValue;
    const size_t smem = sizeof(MrhsSmem);
    static size_t attr[MAX_DEVICES] = {};
    {
        cudaError_t e = opt_in_smem((const void*)hess_cplx_mrhs_kernel, smem, attr);
        if (e != cudaSuccess) return e;
    }
    // refinement steps (done given): the few-groups path takes over when at most HT_MAX groups
    // are left; its plan is counted on the device, so neither launch waits for the host
    const bool tail_path = done && tail && err;
    if (tail_path) {
        hess_tail_plan_kernel<<<1, 256, 0, st>>>(col0, count, rhs_per_shift, s_first, gps, (int)grid, done, tol, tail);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    hess_cplx_mrhs_kernel<<<(unsigned)grid, MT, smem, st>>>(n, Gt, ldg, po, swp, rd, Y, ldy, col0, count,
                                                             rhs_per_shift, s_first, gps, done, tol,
                                                             tail_path ? tail : nullptr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !tail_path) return e;
    static int sms_of[MAX_DEVICES] = {};
    int dev = 0;
    e = current_device(&dev);
    if (e != cudaSuccess) return e;
    if (!sms_of[dev]) {
        e = cudaDeviceGetAttribute(&sms_of[dev], cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
    }
    const int sms = sms_of[dev];
    int sf = s_first, gp = gps;
    void* args[] = {&n, &Gt, &ldg, &po, &swp, &rd, &Y, &ldy, &col0, &count, &rhs_per_shift, &sf, &gp,
                    &tail, &err, &limit_ns};
    return cudaLaunchCooperativeKernel((const void*)hess_cplx_tail_kernel, dim3(sms), dim3(HT_T), args, 0, st);
}

// ---- complex residual r = b - (sigma_s x + tau_s J x), J real; b, x, r interleaved complex ----
// Tiles of 16 rows x 8 complex right-hand sides (16 real columns), one complex column pair
// per thread; k in chunks of 64 through shared memory.
constexpr int QM = 16, QC = 8, QK = 64, QT = 128;

__global__ void __launch_bounds__(QT) residual_cplx_kernel(int n, const double* __restrict__ J, int ldj,
                                                            const double* __restrict__ B, int ldb,
                                                            const double* __restrict__ X, int ldx,
                                                            double* __restrict__ R, int ldr, int nrhs,
                                                            int rhs_per_shift, const double* __restrict__ sig,
                                                            const double* __restrict__ tau,
                                                            const double* __restrict__ done, double tol)
{
    __shared__ double Js[QK][QM + 1];
    __shared__ double Xs[QK][2 * QC + 1];
    const int i0 = blockIdx.x * QM, c0 = blockIdx.y * QC;
    if (done) {
        bool all = true;
        for (int c = c0; c < c0 + QC && c < nrhs; ++c) all = all && (done[c] <= tol);
        if (all) return;
    }
    const int t = threadIdx.x;
    const int r = t % QM, cq = t / QM;  // cq in 0..7: complex column c0 + cq
    double ar = 0.0, ai = 0.0;
    for (int k0 = 0; k0 < n; k0 += QK) {
        for (int e = t; e < QM * QK; e += QT) {
            const int ii = e % QM, kk = e / QM;
            const int i = i0 + ii, k = k0 + kk;
            Js[kk][ii] = (i < n && k < n) ? J[(size_t)k * ldj + i] : 0.0;
        }
        for (int e = t; e < QK * 2 * QC; e += QT) {
            const int kk = e % QK, cp = e / QK;  // cp = 2 (column) + part
            const int k = k0 + kk, c = c0 + (cp >> 1);
            Xs[kk][cp] = (k < n && c < nrhs) ? X[2 * ((size_t)c * ldx + k) + (cp & 1)] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < QK; ++kk) {
            const double jv = Js[kk][r];
            ar = dfma(jv, Xs[kk][2 * cq], ar);
            ai = dfma(jv, Xs[kk][2 * cq + 1], ai);
        }
        __syncthreads();
    }
    const int i = i0 + r, c = c0 + cq;
    if (i < n && c < nrhs) {
        const int s = c / rhs_per_shift;
        const dc sg = {sig[2 * s], sig[2 * s + 1]}, tu = {tau[2 * s], tau[2 * s + 1]};
        const dc xv = {X[2 * ((size_t)c * ldx + i)], X[2 * ((size_t)c * ldx + i) + 1]};
        const dc bv = B ? dc{B[2 * ((size_t)c * ldb + i)], B[2 * ((size_t)c * ldb + i) + 1]} : dc{0.0, 0.0};  // no B: -W X
        const dc w = cadd(cmul(sg, xv), cmul(tu, dc{ar, ai}));
        R[2 * ((size_t)c * ldr + i)] = bv.re - w.re;
        R[2 * ((size_t)c * ldr + i) + 1] = bv.im - w.im;
    }
}

// ---- the same residual for many right-hand sides: J X on the FP64 tensor pipe ----
// J X is an n x n by n x 2m real product (the two planes of m complex vectors), so it runs as
// a tiled GEMM with mma.sync m8n8k4 FP64 (D = A B + C, FP64 products and sums): a CTA owns 128
// rows of J x 32 complex right-hand sides (64 real columns), eight warps of 32 x 32; K in chunks
// of 32 staged by cp.async (double buffered) into padded tiles [k][row] and [k][column] whose
// fragment loads hit 16 distinct 8-byte banks per half-warp.  The epilogue forms
// r = b - (sigma_s x + tau_s (J x)) as the one-tile kernel above does.
constexpr int RM = 128, RC = 32, RN = 2 * RC, RK = 32, RTT = 256;
constexpr int RAP = RM + 4, RBP = RN + 4;
struct ResSmem {
    double A[2][RK][RAP];  // J tile [k][row]
    double B[2][RK][RBP];  // X tile [k][2 c + part]
};

__global__ void __launch_bounds__(RTT, 2) residual_cplx_mma_kernel(int n, const double* __restrict__ J, int ldj,
                                                                   const double* __restrict__ B, int ldb,
                                                                   const double* __restrict__ X, int ldx,
                                                                   double* __restrict__ R, int ldr, int nrhs,
                                                                   int rhs_per_shift, const double* __restrict__ sig,
                                                                   const double* __restrict__ tau,
                                                                   const double* __restrict__ done, double tol)
{
    extern __shared__ __align__(16) unsigned char rsm_raw[];
    ResSmem& sm = *reinterpret_cast<ResSmem*>(rsm_raw);
    const int i0 = blockIdx.x * RM, c0 = blockIdx.y * RC;
    if (done) {
        bool all = true;
        for (int c = c0; c < c0 + RC && c < nrhs; ++c) all = all && (done[c] <= tol);
        if (all) return;
    }
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wm = warp & 3, wn = warp >> 2;  // warp tile: rows 32 wm .., real columns 32 wn ..
    const int g = lane >> 2, t4 = lane & 3;
    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    const int nch = (n + RK - 1) / RK;
    auto stage = [&](int kc, int st) {
        const int k0 = kc * RK;
        for (int e = t; e < RK * RM; e += RTT) {
            const int m = e % RM, kk = e / RM;
            const int i = i0 + m, k = k0 + kk;
            const bool ok = i < n && k < n;
            cp_async8(&sm.A[st][kk][m], ok ? &J[(size_t)k * ldj + i] : J, ok, J);
        }
        for (int e = t; e < RK * RC; e += RTT) {
            const int kk = e % RK, cc = e / RK;
            const int k = k0 + kk, c = c0 + cc;
            const bool ok = k < n && c < nrhs;
            const double* src = ok ? &X[2 * ((size_t)c * ldx + k)] : X;
            cp_async8(&sm.B[st][kk][2 * cc], src, ok, X);
            cp_async8(&sm.B[st][kk][2 * cc + 1], ok ? src + 1 : X, ok, X);
        }
        cp_async_commit();
    };
    stage(0, 0);
    for (int kc = 0; kc < nch; ++kc) {
        const int st = kc & 1;
        if (kc + 1 < nch) {
            stage(kc + 1, st ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < RK; kk += 4) {
            double fa[4], fb[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) fa[a] = sm.A[st][kk + t4][32 * wm + 8 * a + g];
#pragma unroll
            for (int b = 0; b < 4; ++b) fb[b] = sm.B[st][kk + t4][32 * wn + 8 * b + g];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) dmma_8x8x4(acc[a][b], fa[a], fb[b]);
        }
        __syncthreads();
    }
    // epilogue: thread holds (J x) at row 32 wm + 8 a + g, complex column (32 wn + 8 b) / 2 + t4
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int i = i0 + 32 * wm + 8 * a + g;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int c = c0 + (32 * wn + 8 * b) / 2 + t4;
            if (i < n && c < nrhs) {
                const int s = c / rhs_per_shift;
                const dc sg = {sig[2 * s], sig[2 * s + 1]}, tu = {tau[2 * s], tau[2 * s + 1]};
                const dc xv = {X[2 * ((size_t)c * ldx + i)], X[2 * ((size_t)c * ldx + i) + 1]};
                const dc bv = B ? dc{B[2 * ((size_t)c * ldb + i)], B[2 * ((size_t)c * ldb + i) + 1]} : dc{0.0, 0.0};
                const dc w = cadd(cmul(sg, xv), cmul(tu, dc{acc[a][b][0], acc[a][b][1]}));
                R[2 * ((size_t)c * ldr + i)] = bv.re - w.re;
                R[2 * ((size_t)c * ldr + i) + 1] = bv.im - w.im;
            }
        }
    }
}

cudaError_t launch_residual_cplx(int n, const double* J, int ldj, const double* B, int ldb, const double* X, int ldx,
                                 double* R, int ldr, int nrhs, int rhs_per_shift, const double* sig, const double* tau,
                                 cudaStream_t st, const double* done, double tol)
{
    if (nrhs <= 0 || n <= 0) return cudaSuccess;
    if (nrhs >= 16 && (nrhs + RC - 1) / RC <= 65535) {  // many right-hand sides: the tensor-pipe GEMM
        const size_t smem = sizeof(ResSmem);
        static size_t attr[MAX_DEVICES] = {};
        cudaError_t e = opt_in_smem((const void*)residual_cplx_mma_kernel, smem, attr);
        if (e != cudaSuccess) return e;
        dim3 grid((n + RM - 1) / RM, (nrhs + RC - 1) / RC);
        residual_cplx_mma_kernel<<<grid, RTT, smem, st>>>(n, J, ldj, B, ldb, X, ldx, R, ldr, nrhs, rhs_per_shift, sig,
                                                           tau, done, tol);
        return cudaGetLastError();
    }
    dim3 grid((n + QM - 1) / QM, (nrhs + QC - 1) / QC);
    residual_cplx_kernel<<<grid, QT, 0, st>>>(n, J, ldj, B, ldb, X, ldx, R, ldr, nrhs, rhs_per_shift, sig, tau, done,
                                              tol);
    return cudaGetLastError();
}

__global__ void real_to_cplx_kernel(const double* __restrict__ re, double* __restrict__ out, int count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        out[2 * i] = re[i];
        out[2 * i + 1] = 0.0;
    }
}

cudaError_t launch_real_to_cplx(const double* re, double* out, int count, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    real_to_cplx_kernel<<<(count + 255) / 256, 256, 0, st>>>(re, out, count);
    return cudaGetLastError();
}

}  // namespace lhl
