// mixed_common.cuh -- the exchange between CTAs of the mixed-precision reductions
// (reduce_mixed.cu, reduce_lazy.cu): tagged 64-bit words, relaxed polling loads, the pivot
// choice among candidates.
#pragma once
#include "internal.cuh"

namespace lhl {

constexpr int MT = 512;
constexpr int MW = MT / 32;
constexpr int MIX_FLUSH = 16;  // float4 iterations per lane before the FP32 partials go to FP64
constexpr int MIX_RPC_MAX = 64;
constexpr unsigned MIX_POLL_GAP_NS = 300;  // offset of the second header-poll stream

// Polling load: relaxed, so that a lane's loads of several headers are in flight together.
// No acquire is needed: every word read after the poll carries its own step tag.
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Exchange words carry their step: value bits << 32 | (step & 0xffff) << 16.  A reader that
// has seen a CTA's header for step k may still see older words of that CTA (the stores are
// not ordered), so it re-reads a word until its tag is k, bounded in wall time.
__device__ __forceinline__ unsigned long long mix_tag(unsigned step, float v)
{
    return ((unsigned long long)__float_as_uint(v) << 32) | ((unsigned long long)(step & 0xffffu) << 16);
}

__device__ __forceinline__ float ld_tagged(const unsigned long long* p, unsigned step, unsigned long long limit_ns,
                                           bool& ok)
{
    unsigned long long v = ld_relaxed_u64(p);
    if (((unsigned)(v >> 16) & 0xffffu) != (step & 0xffffu)) {
        const uint64_t t0 = globaltimer_ns();
        do {
            v = ld_relaxed_u64(p);
            if (globaltimer_ns() - t0 > limit_ns) {
                ok = false;
                break;
            }
        } while (((unsigned)(v >> 16) & 0xffffu) != (step & 0xffffu));
    }
    return __uint_as_float((unsigned)(v >> 32));
}

// header word: value bits << 32 | (step & 0xffff) << 16 | logical row (0 = none)
__device__ __forceinline__ unsigned long long mix_pack(unsigned int step, int idx, float val)
{
    return ((unsigned long long)__float_as_uint(val) << 32) | ((unsigned long long)(step & 0xffffu) << 16) |
           (unsigned long long)(idx & 0xffff);
}

// Better candidate: larger |v|; ties go to the lower logical row; row 0 = none.
__device__ __forceinline__ bool mix_better(float v, int i, float bv, int bi)
{
    if (i == 0) return false;
    if (bi == 0) return true;
    const float a = fabsf(v), b = fabsf(bv);
    return a > b || (a == b && i < bi);
}

__device__ __forceinline__ void warp_best(float& bv, int& bi, int& bl)
{
    // the same order as mix_better as a key: |v| (its bits order like unsigned integers), plus one
    // so that a zero candidate beats "none" (key 0); then the lowest row among the largest keys
    const unsigned key = bi == 0 ? 0u : __float_as_uint(fabsf(bv)) + 1u;
    const unsigned m = __reduce_max_sync(0xffffffffu, key);
    const unsigned lo = __reduce_min_sync(0xffffffffu, key == m ? (unsigned)bi : 0xffffffffu);
    const unsigned who = __ballot_sync(0xffffffffu, key == m && (unsigned)bi == lo);
    const int src = __ffs(who) - 1;
    bv = __shfl_sync(0xffffffffu, bv, src);
    bi = __shfl_sync(0xffffffffu, bi, src);
    bl = __shfl_sync(0xffffffffu, bl, src);
}


}  // namespace lhl
