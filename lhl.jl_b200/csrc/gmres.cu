// gmres.cu -- refinement by GMRES-IR (lhl_refine_gmres): restarted GMRES on the correction
// equation W d = r, left-preconditioned by the shift's factorisation, in place of the
// reference's fixed-point refinement (lhl_refine!, F:3144-3157) where that converges slowly
// (the mixed form near a shift where sigma I + tau J is close to singular).
//
// Per cycle, for every column whose relative residual is still above tol:
//   r = b - W x                    (residual kernel, FP64)
//   the columns that take the cycle: above tol, and not stagnated (gm_mark_kernel)
//   z = W~^-1 r                    (lhl_ldiv's kernels)
//   v0 = z / beta, g = beta e1     (gm_begin_kernel)
//   for j = 0 .. m-1, while the column is active:
//       w = W~^-1 (0 - W v_j)      (residual kernel with b = 0, then lhl_ldiv's kernels;
//                                   the sign is folded in below)
//       CGS2 of -w against v_0..v_j, h_{j+1,j} = ||w||, v_{j+1} = w / h_{j+1,j}; the earlier
//       Givens rotations applied to the new column of H and a new one computed, so that
//       |g_{j+1}| is the preconditioned residual of the least-squares solution
//       (gm_arnoldi_kernel); the column leaves the cycle once |g_{j+1}| / beta <= eta, with
//       eta = min(0.5, 0.1 tol / (relative residual at the cycle's start))
//   x += V y with R y = g           (gm_update_kernel)
// Every kernel takes the per-column activity flags, so finished columns cost nothing and the
// whole cycle is launched without a host round trip.
//
// Per-column state (GS(m) doubles): beta, eta, j done, spare; g[0..m]; cs[0..m-1];
// sn[0..m-1]; the rotated H's upper triangle, column-major m x m.
// Krylov basis: V + c (m+1) n, vector i at + i n.
#include "internal.cuh"

namespace lhl {

constexpr int GT = 256;
constexpr int GW = GT / 32;

__host__ __device__ constexpr int gm_state_size(int m) { return 4 + (m + 1) + 2 * m + m * m; }

__device__ __forceinline__ double block_sum_gm(double v, double* red)
{
    v = warp_sum(v);
    __syncthreads();  // red may still be read from an earlier call
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < GW; ++w) s += red[w];
    return s;
}

// Which columns take the next cycle: those above tol (not NaN) whose relative residual at
// least halved over the last cycle.  One that did not is at its attainable accuracy (its FP64
// floor for this shift, or the limit of the preconditioner): it is marked (prev < 0) and sits
// out every later cycle, keeping its last iterate.
__global__ void gm_mark_kernel(const double* __restrict__ res, double* __restrict__ prev, double* __restrict__ act,
                               double tol, int first, int nrhs)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nrhs) return;
    const double rc = res[c];
    bool go = rc > tol;
    if (first) {
        prev[c] = rc;
    } else if (prev[c] < 0.0) {
        go = false;
    } else if (go && !(rc <= 0.5 * prev[c])) {
        prev[c] = -1.0;
        go = false;
    } else {
        prev[c] = rc;
    }
    act[c] = go ? 1.0 : 0.0;
}

// Starts a cycle for the columns gm_mark_kernel chose.  z = W~^-1 r is in R's column c.
__global__ void __launch_bounds__(GT) gm_begin_kernel(int n, int m, const double* __restrict__ R, int ldr,
                                                      double* __restrict__ V, double* __restrict__ S,
                                                      double* __restrict__ act, const double* __restrict__ res,
                                                      double tol)
{
    __shared__ double red[GW];
    const int c = blockIdx.x;
    double* st = S + (size_t)c * gm_state_size(m);
    const double rc = res[c];
    if (!(act[c] > 0.5)) {
        if (threadIdx.x == 0) st[2] = 0.0;
        return;
    }
    const double* z = R + (size_t)c * ldr;
    double p = 0.0;
    for (int i = threadIdx.x; i < n; i += GT) p = dfma(z[i], z[i], p);
    const double beta = sqrt(block_sum_gm(p, red));
    const bool ok = beta > 0.0 && isfinite(beta);
    double* v0 = V + (size_t)c * (m + 1) * n;
    const double ib = ok ? 1.0 / beta : 0.0;
    for (int i = threadIdx.x; i < n; i += GT) v0[i] = z[i] * ib;
    if (threadIdx.x == 0) {
        st[0] = beta;
        st[1] = fmin(0.5, 0.1 * tol / rc);
        st[2] = 0.0;
        for (int q = 0; q <= m; ++q) st[4 + q] = 0.0;
        st[4] = beta;
        act[c] = ok ? 1.0 : 0.0;
    }
}

// One Arnoldi step j for every active column: R's column c holds -(W~^-1 W v_j).
__global__ void __launch_bounds__(GT) gm_arnoldi_kernel(int n, int m, int j, double* __restrict__ R, int ldr,
                                                        double* __restrict__ V, double* __restrict__ S,
                                                        double* __restrict__ act)
{
    __shared__ double h1[33], h2[33];
    __shared__ double red[GW];
    const int c = blockIdx.x;
    if (!(act[c] > 0.5)) return;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    double* w = R + (size_t)c * ldr;
    const double* Vc = V + (size_t)c * (m + 1) * n;
    // pass 1: h1_i = v_i . (-R), one warp per basis vector
    for (int i = warp; i <= j; i += GW) {
        const double* vi = Vc + (size_t)i * n;
        double p = 0.0;
        for (int e = lane; e < n; e += 32) p = dfma(vi[e], -w[e], p);
        p = warp_sum(p);
        if (lane == 0) h1[i] = p;
    }
    __syncthreads();
    // pass 2: w' = -R - V h1, stored in R
    for (int e = t; e < n; e += GT) {
        double x = -w[e];
        for (int i = 0; i <= j; ++i) x = dfma(-h1[i], Vc[(size_t)i * n + e], x);
        w[e] = x;
    }
    __syncthreads();
    // pass 3: h2_i = v_i . w' (the second Gram-Schmidt sweep)
    for (int i = warp; i <= j; i += GW) {
        const double* vi = Vc + (size_t)i * n;
        double p = 0.0;
        for (int e = lane; e < n; e += 32) p = dfma(vi[e], w[e], p);
        p = warp_sum(p);
        if (lane == 0) h2[i] = p;
    }
    __syncthreads();
    // pass 4: w'' = w' - V h2 and its norm
    double p = 0.0;
    for (int e = t; e < n; e += GT) {
        double x = w[e];
        for (int i = 0; i <= j; ++i) x = dfma(-h2[i], Vc[(size_t)i * n + e], x);
        w[e] = x;
        p = dfma(x, x, p);
    }
    const double hn = sqrt(block_sum_gm(p, red));
    // pass 5: v_{j+1}
    double* vn = V + ((size_t)c * (m + 1) + j + 1) * n;
    const double ih = (hn > 0.0 && isfinite(hn)) ? 1.0 / hn : 0.0;
    for (int e = t; e < n; e += GT) vn[e] = w[e] * ih;
    if (t == 0) {
        double* st = S + (size_t)c * gm_state_size(m);
        double* g = st + 4;
        double* cs = g + (m + 1);
        double* sn = cs + m;
        double* Hr = sn + m;  // column-major m x m
        double hc[33];
        for (int i = 0; i <= j; ++i) hc[i] = h1[i] + h2[i];
        hc[j + 1] = hn;
        for (int i = 0; i < j; ++i) {
            const double a = hc[i], b = hc[i + 1];
            hc[i] = cs[i] * a + sn[i] * b;
            hc[i + 1] = -sn[i] * a + cs[i] * b;
        }
        const double a = hc[j], b = hc[j + 1];
        const double r = hypot(a, b);
        const double cj = r > 0.0 ? a / r : 1.0, sj = r > 0.0 ? b / r : 0.0;
        cs[j] = cj;
        sn[j] = sj;
        for (int i = 0; i < j; ++i) Hr[i + (size_t)m * j] = hc[i];
        Hr[j + (size_t)m * j] = r;
        const double gj = g[j];
        g[j] = cj * gj;
        g[j + 1] = -sj * gj;
        st[2] = (double)(j + 1);
        const double est = fabs(g[j + 1]) / st[0];
        if (!(est > st[1]) || j + 1 >= m || !(hn > 0.0) || !isfinite(est)) act[c] = 0.0;
    }
}

// x += V y, R y = g over the column's j done steps.
__global__ void __launch_bounds__(GT) gm_update_kernel(int n, int m, double* __restrict__ X, int ldx,
                                                       const double* __restrict__ V, const double* __restrict__ S)
{
    __shared__ double y[32];
    const int c = blockIdx.x;
    const double* st = S + (size_t)c * gm_state_size(m);
    const int jd = (int)st[2];
    if (jd <= 0) return;
    if (threadIdx.x == 0) {
        const double* g = st + 4;
        const double* Hr = g + (m + 1) + 2 * m;
        for (int i = jd - 1; i >= 0; --i) {
            double v = g[i];
            for (int k = i + 1; k < jd; ++k) v = dfma(-Hr[i + (size_t)m * k], y[k], v);
            const double d = Hr[i + (size_t)m * i];
            y[i] = d != 0.0 ? v / d : 0.0;
        }
    }
    __syncthreads();
    const double* Vc = V + (size_t)c * (m + 1) * n;
    double* x = X + (size_t)c * ldx;
    for (int e = threadIdx.x; e < n; e += GT) {
        double v = x[e];
        for (int i = 0; i < jd; ++i) v = dfma(y[i], Vc[(size_t)i * n + e], v);
        x[e] = v;
    }
}

size_t gm_state_doubles(int m) { return (size_t)gm_state_size(m); }

cudaError_t launch_gm_mark(const double* res, double* prev, double* act, double tol, int first, int nrhs,
                           cudaStream_t st)
{
    if (nrhs <= 0) return cudaSuccess;
    gm_mark_kernel<<<(nrhs + 127) / 128, 128, 0, st>>>(res, prev, act, tol, first, nrhs);
    return cudaGetLastError();
}

cudaError_t launch_gm_begin(int n, int m, const double* R, int ldr, double* V, double* S, double* act,
                            const double* res, double tol, int nrhs, cudaStream_t st)
{
    if (nrhs <= 0 || n <= 0) return cudaSuccess;
    gm_begin_kernel<<<nrhs, GT, 0, st>>>(n, m, R, ldr, V, S, act, res, tol);
    return cudaGetLastError();
}

cudaError_t launch_gm_arnoldi(int n, int m, int j, double* R, int ldr, double* V, double* S, double* act, int nrhs,
                              cudaStream_t st)
{
    if (nrhs <= 0 || n <= 0) return cudaSuccess;
    gm_arnoldi_kernel<<<nrhs, GT, 0, st>>>(n, m, j, R, ldr, V, S, act);
    return cudaGetLastError();
}

cudaError_t launch_gm_update(int n, int m, double* X, int ldx, const double* V, const double* S, int nrhs,
                             cudaStream_t st)
{
    if (nrhs <= 0 || n <= 0) return cudaSuccess;
    gm_update_kernel<<<nrhs, GT, 0, st>>>(n, m, X, ldx, V, S);
    return cudaGetLastError();
}

}  // namespace lhl
