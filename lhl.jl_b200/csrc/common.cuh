// common.cuh -- shared device helpers for the LHL sm_100a kernels.
//
// Conventions (mirroring src/LHLFactorization.jl): matrices are column-major FP64,
// indices in the algorithm text are 1-based, pivot / permutation vectors hold 1-based
// int64 row indices.  Device code indexes with the 1-based macro M1 below so the
// kernels read like the reference they restate.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/lhl_gpu.h"

#define M1(A, ld, i, j) ((A)[(size_t)((j) - 1) * (size_t)(ld) + (size_t)((i) - 1)])

namespace lhl {

// IEEE operations that the compiler must not fuse: the plain FP64 form reproduces the
// reference's operation order exactly (fused multiply-adds only where it calls fmuladd).
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dfma(double a, double b, double c) { return __fma_rn(a, b, c); }
// the same four in single precision (the Float32 workspace's reduction)
__device__ __forceinline__ float dmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float dadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float dsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float dfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_acquire_i32(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// 8-byte asynchronous copy global -> shared (cp.async); a masked copy reads nothing (source
// size 0, the destination is zero-filled) and is given `base`, a valid address, as its source
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid, const double* base)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const int sz = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(valid ? src : base), "r"(sz)
                 : "memory");
}
// 16-byte asynchronous copy global -> shared, L2 only (.cg): both addresses 16-byte aligned;
// `bytes` (0, 8 or 16) are read and the rest of the 16 zero-filled; a copy reading nothing is
// given `base`, a valid address, as its source
__device__ __forceinline__ void cp_async16(double* dst, const double* src, int bytes, const double* base)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(bytes > 0 ? src : base), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// D = A B + D on the FP64 tensor pipe, one 8 x 8 x 4 tile per warp (mma.sync m8n8k4 .f64):
// lane (g = lane / 4, t = lane % 4) holds A[g][t], B[t][g] and D[g][2t], D[g][2t+1]
__device__ __forceinline__ void dmma_8x8x4(double (&c)[2], double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// Grid-wide barrier for a cooperative (co-resident) grid.  `counter` only grows: the
// b-th barrier of a launch waits until it reaches b * gridDim.x.  The wait is bounded
// by `limit_ns` of wall time; on expiry the CTA records LHL_ERR_TIMEOUT in *err and
// returns false, and every CTA that sees *err set also returns false, so a lost CTA
// ends the kernel with an error status instead of a hang.
struct GridBarrier {
    unsigned int* counter;
    int* err;
    unsigned long long limit_ns;
    unsigned int seq;
    unsigned long long* wait_ns;  // optional: CTA 0 accumulates its wait (arrival -> release)

    __device__ __forceinline__ bool sync()
    {
        __shared__ int s_ok;
        ++seq;
        __syncthreads();
        if (threadIdx.x == 0) {
            int ok = 1;
            __threadfence();
            atomicAdd(counter, 1u);
            const unsigned int target = seq * gridDim.x;
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
            if (wait_ns && blockIdx.x == 0) *wait_ns += globaltimer_ns() - t0;
            s_ok = ok;
        }
        __syncthreads();
        return s_ok != 0;
    }
};

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// First-maximum combine: larger |value| wins, ties go to the lower row (the reference's
// strict `>` scan in increasing row order, F:799-806).  Row 0 means "no candidate".
__device__ __forceinline__ void argmax_combine(double& a, int& ia, double b, int ib)
{
    if (ib == 0) return;
    if (ia == 0 || b > a || (b == a && ib < ia)) { a = b; ia = ib; }
}

__device__ __forceinline__ void warp_argmax(double& a, int& ia)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double b = __shfl_xor_sync(0xffffffffu, a, o);
        int ib = __shfl_xor_sync(0xffffffffu, ia, o);
        argmax_combine(a, ia, b, ib);
    }
}

// Balancing decision for one index (F:313-327): the power-of-two factor f that brings the
// column and row norms c, r within a factor 2, and whether it reduces c + r below 0.95 of
// its value.  The loops are bounded by the exponent range.
__device__ __forceinline__ bool balance_decide(double c, double r, double& f)
{
    if (c == 0.0 || r == 0.0) return false;
    f = 1.0;
    const double s = c + r;
    int guard = 0;
    while (c < r / 2.0 && guard < 4200) { c *= 2.0; r /= 2.0; f *= 2.0; ++guard; }
    while (c >= 2.0 * r && guard < 8400) { c /= 2.0; r *= 2.0; f /= 2.0; ++guard; }
    return c + r < 0.95 * s;
}

}  // namespace lhl

// ---- TMA (cp.async.bulk.tensor) and mbarrier helpers -------------------------------------
namespace lhl {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait on an mbarrier phase; returns false if it did not complete in `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit)
{
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Bounded wait on an mbarrier phase by wall time; returns false after limit_ns.
__device__ __forceinline__ bool mbar_wait_ns(uint64_t* bar, uint32_t parity, unsigned long long limit_ns)
{
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 0;; ++it) {
        if (mbar_wait(bar, parity, 64)) return true;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
}

// Order this thread's view of global memory (generic proxy) before its later TMA reads.
__device__ __forceinline__ void fence_proxy_async_global()
{
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 2-D tiled TMA load of box (x, y) of `tmap` into shared memory, completing on `bar`.
// x (the contiguous coordinate) must be a multiple of 2 for FP64 (16-byte rule).
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int x, int y, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(tmap), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace lhl
