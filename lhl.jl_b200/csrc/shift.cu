// shift.cu -- lhl_shift!: LU with partial pivoting of G = sigma I + tau H, H upper
// Hessenberg, stored transposed (Gt[j,k] = U[k,j]) -- src/LHLFactorization.jl F:2529-2594,
// identical to the bit-exact reference of test/core_tests.jl:119-171.
//
// One CTA per shift.  Element j of the pending row r (the not-yet-chosen candidate row,
// F:2522-2527) lives in a register of thread (j-1) mod T for the whole elimination, so a
// step costs one CTA barrier: the owner of element k+1 updates it first, takes the pivot
// decision of step k+1 (the compare and the one division) and publishes it in shared
// memory; every other thread only reads the decision.  Rows of H (Ht[j, k+1]) are requested D
// steps before they are used (D = 4 up to n = 2048), into a register ring indexed at
// compile time, so that a step does not wait for its loads.  Every operation is the reference's, in its order, with no fused
// multiply-add, so Gt, swap, rdiag and info are bit-identical to the reference.
#include "internal.cuh"

namespace lhl {

// Rounded operations of the elimination's arithmetic type V: double (LHLWorkspace{Float64}) or
// float (LHLWorkspace{Float32}: Ht, sigma and tau hold float values, every operation rounds to
// float, and Gt / rdiag receive float values in double storage).  No fused multiply-add.
__device__ __forceinline__ double vmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double vadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double vsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float vmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float vadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float vsub(float a, float b) { return __fsub_rn(a, b); }

// The elimination of one shift; every thread of the CTA calls it (T threads).
template <int T, int E, int D, class V = double>
__device__ __forceinline__ void shift_lu_body(int n, const double* __restrict__ Ht, int ldh, double sigma_in,
                                              double tau_in, double* __restrict__ Gt, int ldg,
                                              uint8_t* __restrict__ swp, double* __restrict__ rdiag,
                                              int32_t* __restrict__ info_out)
{
    const int t = threadIdx.x;
    const V sigma = (V)sigma_in, tau = (V)tau_in;

    __shared__ V s_next[2];  // r[k+1] after step k, double-buffered by step parity
    __shared__ V s_l[2], s_a[2], s_b[2];  // the decision of step k (by parity)
    __shared__ int s_sw[2];
    __shared__ int s_info;

    // D rows of H in flight: the row for step k is requested at step k - D
    V r[E];
    V hq[D][E];           // hq[d]: H row k+1 (Ht[j, k+1]) for the step k = d + 1 (mod D)
    V hsub[E];            // Ht[j, j+1] = H[j+1, j]: the subdiagonal entry of the step this
                          // thread decides (the owner of element j decides step j)
    // row 1 of G: r[j] = tau * Ht[j, 1], r[1] += sigma (F:2536-2539)
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int j = 1 + t + e * T;
        r[e] = (j <= n) ? vmul(tau, (V)M1(Ht, ldh, j, 1)) : (V)0;
        if (j == 1) r[e] = vadd(r[e], sigma);
        hsub[e] = (j + 1 <= n) ? (V)M1(Ht, ldh, j, j + 1) : (V)0;
    }
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const int k = d + 1;  // step
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int j = 1 + t + e * T;
            hq[d][e] = (j <= n && k + 1 <= n) ? (V)M1(Ht, ldh, j, k + 1) : (V)0;
        }
    }
    // the pivot decision of step k (F:2541-2556): |b| > |a| swaps; l = a/b, b/a, or 0
    auto decide = [&](int k, V a, V hs) {
        const V b = vmul(tau, hs);
        const bool sw = fabs(b) > fabs(a);
        V l;
        if (sw) {
            l = a / b;
        } else if (a == (V)0) {
            l = (V)0;
        } else {
            l = b / a;
        }
        s_l[k & 1] = l;
        s_a[k & 1] = a;
        s_b[k & 1] = b;
        s_sw[k & 1] = sw ? 1 : 0;
    };
    if (t == 0) {
        s_next[1] = r[0];
        s_info = 0;
        if (n >= 2) decide(1, r[0], hsub[0]);
    }
    __syncthreads();

    // running column pointers, so that a step computes no 64-bit addresses: this thread's
    // element e of Gt column k is gcol[e * T], of Ht column k + D + 1 (the prefetch) hcol[e * T]
    double* gcol = Gt + t;
    const double* hcol = Ht + (size_t)(D + 1) * ldh + t;
    for (int k0 = 1; k0 <= n - 1; k0 += D) {
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const int k = k0 + d;
            if (k > n - 1) break;
            const V l = s_l[k & 1];
            const bool sw = s_sw[k & 1] != 0;
            if (t == 0) {
                const V a = s_a[k & 1], b = s_b[k & 1];
                swp[k - 1] = sw ? 1 : 0;
                M1(Gt, ldg, k, k) = sw ? b : a;
                M1(Gt, ldg, k, k + 1) = l;
                if (!sw && a == (V)0 && s_info == 0) s_info = k;
            }
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int j = 1 + t + e * T;
                if (j >= k + 1 && j <= n) {
                    if (sw) {
                        const V g = vmul(tau, hq[d][e]);
                        V gk = g;
                        V rj = vsub(r[e], vmul(l, g));
                        if (j == k + 1) {
                            gk = vadd(g, sigma);              // Gt[k+1,k] += sigma
                            rj = vsub(rj, vmul(l, sigma));    // r[k+1] -= l*sigma
                        }
                        gcol[e * T] = gk;
                        r[e] = rj;
                    } else {
                        const V rj = r[e];
                        gcol[e * T] = rj;
                        V rn = vsub(vmul(tau, hq[d][e]), vmul(l, rj));
                        if (j == k + 1) rn = vadd(rn, sigma); // r[k+1] += sigma
                        r[e] = rn;
                    }
                    if (j == k + 1) {  // owner of element k+1: publish it and decide step k+1
                        s_next[(k + 1) & 1] = r[e];
                        if (k + 1 <= n - 1) decide(k + 1, r[e], hsub[e]);
                    }
                }
            }
            // request the row for step k + D into the slot just used
            const int kf = k + D;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int j = 1 + t + e * T;
                hq[d][e] = (j >= kf && j <= n && kf + 1 <= n) ? (V)hcol[e * T] : (V)0;
            }
            gcol += ldg;
            hcol += ldh;
            __syncthreads();
        }
    }
    // finish (F:2579-2594)
    if (t == 0) {
        const V rn = s_next[n & 1];
        M1(Gt, ldg, n, n) = rn;
        swp[n - 1] = 0;
        int info = s_info;
        if (rn == (V)0 && info == 0) info = n;
        *info_out = info;
    }
    __syncthreads();
    for (int j = 1 + t; j <= n; j += T) rdiag[j - 1] = (V)1 / (V)M1(Gt, ldg, j, j);
}

template <int T, int E, int D, class V = double>
__global__ void __launch_bounds__(T) shift_lu_kernel(int n, const double* __restrict__ Ht, int ldh,
                                                     const double* __restrict__ sig, const double* __restrict__ tau_,
                                                     int s0, double* __restrict__ Gt_all, int ldg,
                                                     uint8_t* __restrict__ swap_all, double* __restrict__ rdiag_all,
                                                     int32_t* __restrict__ info_all)
{
    const int s = s0 + blockIdx.x;
    shift_lu_body<T, E, D, V>(n, Ht, ldh, sig[blockIdx.x], tau_[blockIdx.x], Gt_all + (size_t)s * ldg * n, ldg,
                           swap_all + (size_t)s * n, rdiag_all + (size_t)s * n, info_all + s);
}

// Many independent matrices (lhl_shift_batched_all): CTA b takes shift b % S of matrix b / S;
// the matrix's order and offsets come from the batch descriptor.
__global__ void __launch_bounds__(256) shift_lu_batch_kernel(BatchDesc d, const double* __restrict__ sig,
                                                             const double* __restrict__ tau)
{
    const int m = blockIdx.x / d.S, s = blockIdx.x - m * d.S;
    const int n = d.n[m];
    if (n <= 0) return;
    const size_t ms = (size_t)m * d.S + s;
    shift_lu_body<256, 2, 2>(n, d.Ht + d.off2[m], n, sig[ms], tau[ms], d.Gt + d.offg[m] + (size_t)s * (n + 4) * n,
                             n + 4, d.swap + d.S * d.off1[m] + (size_t)s * n, d.rdiag + d.S * d.off1[m] + (size_t)s * n,
                             d.info + ms);
}

cudaError_t launch_shift_lu_batch(const BatchDesc& d, const double* sig, const double* tau, cudaStream_t st)
{
    if (d.count <= 0 || d.S <= 0) return cudaSuccess;
    shift_lu_batch_kernel<<<d.count * d.S, 256, 0, st>>>(d, sig, tau);
    return cudaGetLastError();
}

template <int T, int E, int D>
static cudaError_t launch_shift_T(int n, const double* Ht, int ldh, const double* sig, const double* tau, int s0,
                                  int count, double* Gt, int ldg, uint8_t* swp, double* rd, int32_t* info,
                                  cudaStream_t st, int f32)
{
    if (f32) shift_lu_kernel<T, E, D, float><<<count, T, 0, st>>>(n, Ht, ldh, sig, tau, s0, Gt, ldg, swp, rd, info);
    else shift_lu_kernel<T, E, D, double><<<count, T, 0, st>>>(n, Ht, ldh, sig, tau, s0, Gt, ldg, swp, rd, info);
    return cudaGetLastError();
}

// Launch shapes of the real shift LU (threads T, elements per thread E, rows of H in flight D),
// selectable per workspace (lhl_ws_set_shift_variant) so that a tuner can time them; every shape
// runs the same operations in the same order, so all give the same bits.  Shape v serves orders
// n <= T E.  Variant 0 is the rule by order below.
static const int kShiftShapes[][3] = {{256, 1, 4}, {512, 2, 4}, {512, 4, 4}, {512, 8, 2}, {1024, 8, 1},
                                      {1024, 16, 1}, {1024, 2, 4}, {1024, 4, 2}, {256, 4, 4}, {256, 8, 2}};
constexpr int kNumShiftShapes = sizeof(kShiftShapes) / sizeof(kShiftShapes[0]);

int shift_shape(int variant, int* T, int* E, int* D)
{
    if (variant < 1 || variant > kNumShiftShapes) return 0;
    *T = kShiftShapes[variant - 1][0];
    *E = kShiftShapes[variant - 1][1];
    *D = kShiftShapes[variant - 1][2];
    return 1;
}

cudaError_t launch_shift_lu(int n, const double* Ht, int ldh, const double* sig, const double* tau, int s0, int count,
                            double* Gt, int ldg, uint8_t* swp, double* rd, int32_t* info, cudaStream_t st, int f32,
                            int variant)
{
    if (count <= 0 || n <= 0) return cudaSuccess;
    if (variant > 0) {
        int T, E, D;
        if (!shift_shape(variant, &T, &E, &D) || T * E < n) return cudaErrorInvalidValue;
#define V_(k, T_, E_, D_) \
    case k: return launch_shift_T<T_, E_, D_>(n, Ht, ldh, sig, tau, s0, count, Gt, ldg, swp, rd, info, st, f32);
        switch (variant) {
            V_(1, 256, 1, 4) V_(2, 512, 2, 4) V_(3, 512, 4, 4) V_(4, 512, 8, 2) V_(5, 1024, 8, 1)
            V_(6, 1024, 16, 1) V_(7, 1024, 2, 4) V_(8, 1024, 4, 2) V_(9, 256, 4, 4) V_(10, 256, 8, 2)
            default: return cudaErrorInvalidValue;
        }
#undef V_
    }
    if (n <= 256) return launch_shift_T<256, 1, 4>(n, Ht, ldh, sig, tau, s0, count, Gt, ldg, swp, rd, info, st, f32);
    if (n <= 1024) return launch_shift_T<512, 2, 4>(n, Ht, ldh, sig, tau, s0, count, Gt, ldg, swp, rd, info, st, f32);
    if (n <= 2048) return launch_shift_T<512, 4, 4>(n, Ht, ldh, sig, tau, s0, count, Gt, ldg, swp, rd, info, st, f32);
    if (n <= 4096) return launch_shift_T<512, 8, 2>(n, Ht, ldh, sig, tau, s0, count, Gt, ldg, swp, rd, info, st, f32);
    if (n <= 8192) return launch_shift_T<1024, 8, 1>(n, Ht, ldh, sig, tau, s0, count, Gt, ldg, swp, rd, info, st, f32);
    if (n <= 16384) return launch_shift_T<1024, 16, 1>(n, Ht, ldh, sig, tau, s0, count, Gt, ldg, swp, rd, info, st, f32);
    return cudaErrorInvalidValue;
}

}  // namespace lhl
