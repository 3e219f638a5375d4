// reduce_lazy.cu -- the mixed-precision reduction (LHL_PREC_MIXED) for orders whose FP32 rows
// do not fit in shared memory: ELMHES (F:466-501) with the row updates of each panel of LZ_NB
// steps delayed and applied at the panel's end as one rank-LZ_NB update -- the delayed panel
// updates of the reference's blocked reduction (F:765-783, F:1676-1705), restated for rows that
// stay with the CTA that owns them.
//
// Layout and exchange are reduce_mixed.cu's: one CTA per SM owns `rpc` physical rows of the
// balanced matrix, FP32, here in global memory; rows never move (row interchanges swap logical
// labels); each step one exchange between CTAs (headers, column values, candidate rows: tagged
// words, relaxed stores, polls bounded in wall time) and no grid barrier.
//
// What is delayed.  At step k the eager kernel subtracts l_i R from every own row below the
// pivot (a read and a write of the whole trailing block per step).  Here the stored rows keep
// their values from the start of the panel; row i's true entries are
//     A[i, c] = S[i, c] - sum_{s in panel, s < k} l_i^(s) U_s[c]
// for every column c not yet complete, where U_s is step s's pivot row and l_i^(s) row i's
// multiplier at step s (zero unless the row was below that pivot).  Step k then needs:
//   * the column update A[:, k+1] += A[:, k+2:n] l (the GEMV): with the stored rows,
//         A[i, :] . l = S[i, :] . l - sum_s l_i^(s) (U_s . l),
//     so every CTA also takes the panel's U_s rows against l (at most LZ_NB dot products);
//   * the new column k+1 of row i, written into the stored row (the column is complete):
//         c'_i = S[i, k+1] + S[i, :] . l - sum_{s <= k} l_i^(s) Gamma_s,
//         Gamma_s = U_s[k+1] + U_s . l   (U_k = R, the pivot row, l_i^(k) = l_i);
//   * the candidate row for step k+1 in its true form, computed from its stored values and the
//     U_s when it is published (the winner's published row is U_{k+1}).
// The candidate rows live in a ring of LZ_NS slots, so every CTA can read the panel's U_s from
// the winners' slots until the panel ends.  Column interchanges are not applied to the stored
// rows during a panel (that would put them out of step with the published U_s): logical column
// L sits at physical position L - 1 except for the few positions the panel's interchanges
// touched, kept in a small table; at the panel's end each CTA applies the rank-LZ_NB update
//     S[i, c] -= sum_s l_i^(s) U_s[c]   for every column c after the panel,
// then moves the touched positions to their logical places, so that each panel starts in
// logical column order.  The dot products start at the panel's first column.
//
// Arithmetic: FP32 storage; dot products of FP32 products with FP64 accumulation; the new
// column value and the Gamma corrections in FP64, rounded once to FP32 when stored; the
// rank-LZ_NB update in FP32 fused multiply-adds.  The pivot search is the eager kernel's (the
// reference's first maximum on the FP32 column values).  At the end every CTA writes its rows
// in FP64 to their logical positions of `factors`, and CTA 0 writes perm / iperm: the same
// outputs, in the same layout, as the eager kernel.
#include "mixed_common.cuh"

namespace lhl {

constexpr int LZ_NB = 16;               // steps per panel
constexpr int LZ_NS = MIX_LAZY_RING;    // slots of the candidate-row ring
static_assert(LZ_NS >= LZ_NB + 2, "the ring holds a panel's pivot rows and the next step's candidates");
constexpr int LZ_TMAX = 2 * LZ_NB + 2;  // column positions a panel's interchanges can touch
constexpr int LZ_CH = 256;              // columns per staged chunk of the panel update

struct LazyShared {
    int tP[LZ_TMAX];      // touched physical positions (0-based) ...
    int tL[LZ_TMAX];      // ... and the logical column (1-based) each now holds
    float tdl[LZ_TMAX];   // per step: l_{tL} - lv[tP] (the dot-product fix at touched positions)
    int ntouch;
    int win[LZ_NB];       // winning CTA of each panel step
    float ucol[LZ_NB];    // U_s[k+1] at the step's new column
    double gam[LZ_NB];    // U_s . l
    int K0;               // the panel's first step
    int pk, pk1;          // physical positions of logical columns k and k+1
};

// the physical position (0-based) of logical column L (1-based), through the panel's table of
// touched positions
__device__ __forceinline__ int lz_cph(const LazyShared& z, int L)
{
    for (int q = 0; q < z.ntouch; ++q)
        if (z.tL[q] == L) return z.tP[q];
    return L - 1;
}

// barrier of the `count` threads of warps 1-15 (id 1; warp 0 is polling meanwhile)
__device__ __forceinline__ void named_bar_sync(int id, int count)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// U_s[P] from the ring: winner w's row of step s, tagged with the step
__device__ __forceinline__ const unsigned long long* lz_urow(const MixArgs& a, int s, int w, int G)
{
    return a.crow + ((size_t)(s % LZ_NS) * G + w) * a.ldr;
}

__global__ void __launch_bounds__(MT, 1) reduce_mixed_lazy_kernel(MixArgs a)
{
    extern __shared__ __align__(16) float slz[];
    __shared__ double s_part[(MIX_RPC_MAX + 4) * 4];
    __shared__ float s_li[MIX_RPC_MAX];
    __shared__ float s_lm[MIX_RPC_MAX][LZ_NB];
    __shared__ LazyShared z;
    __shared__ int s_win, s_p, s_ok, s_cand;
    __shared__ float s_piv;

    const int n = a.n, rpc = a.rpc, ldr = a.ldr, G = gridDim.x, b = blockIdx.x;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int r0 = b * rpc;
    const int nr = min(rpc, n - r0);
    float* R = slz;              // pivot row, physical column order; pads zero
    float* lv = R + ldr;         // multipliers by logical row (slot L-1)
    int* lg = (int*)(lv + ldr);  // physical row -> logical (1-based)
    int* ph = lg + ldr;          // logical (1-based) -> physical row, ph[0] unused
    float* Us = (float*)(ph + ldr + 4);  // panel update: the panel's U_s at LZ_CH columns (ph[n] may be ph[ldr])
    unsigned* tbits = (unsigned*)(Us + LZ_NB * LZ_CH);  // bit P: position P is in the touched table
    float* rows = a.grows + (size_t)r0 * ldr;  // nr x ldr, FP32, global
    unsigned long long* hdr = a.hdr;

    // ---- load own rows (FP64 -> FP32, zero pads), labels ----
    for (int e = t; e < nr * ldr; e += MT) {
        const int c = e % ldr, i = e / ldr;  // along the row: coalesced stores, strided reads of A
        rows[(size_t)i * ldr + c] = c < n ? (float)a.A[(size_t)c * n + r0 + i] : 0.f;
    }
    for (int q = t; q < ldr; q += MT) {
        R[q] = 0.f;
        lv[q] = 0.f;
        if (q < n) {
            lg[q] = q + 1;
            ph[q + 1] = q;
        }
    }
    for (int e = t; e < MIX_RPC_MAX * LZ_NB; e += MT) s_lm[e / LZ_NB][e % LZ_NB] = 0.f;
    for (int q = t; q < (ldr + 31) / 32; q += MT) tbits[q] = 0u;
    if (t == 0) {
        z.ntouch = 0;
        z.K0 = 1;
    }
    __syncthreads();

    auto prefetch_cval = [&](int st) {  // warps 1-15: column values of step st by logical row
        constexpr int PF = 8;
        const unsigned long long* cv = a.cval + (size_t)(st & 1) * n;
        const unsigned want = (unsigned)st & 0xffffu;
        bool ok = true;
        for (int base = t - 32; base < n; base += PF * (MT - 32)) {
            unsigned long long w[PF];
#pragma unroll
            for (int u = 0; u < PF; ++u) {
                const int q = base + u * (MT - 32);
                w[u] = q < n ? ld_relaxed_u64(&cv[q]) : 0ull;
            }
#pragma unroll
            for (int u = 0; u < PF; ++u) {
                const int q = base + u * (MT - 32);
                if (q < n) {
                    float v = __uint_as_float((unsigned)(w[u] >> 32));
                    if (((unsigned)(w[u] >> 16) & 0xffffu) != want) v = ok ? ld_tagged(&cv[q], (unsigned)st, a.limit_ns, ok) : 0.f;
                    lv[lg[q] - 1] = v;
                }
            }
        }
        if (!ok) atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
    };

    // ---- publish step 1: column 1 values, candidate among logical rows >= 2 (its row as stored:
    // nothing is delayed yet), into ring slot 1 ----
    if (warp != 0) prefetch_cval(1);
    if (warp == 0) {
        float bv = 0.f;
        int bi = 0, bl = -1;
        for (int i = lane; i < nr; i += 32) {
            const int L = r0 + i + 1;
            const float v = rows[(size_t)i * ldr];
            __stcg(&a.cval[(1 & 1) * n + r0 + i], mix_tag(1u, v));
            if (L >= 2 && mix_better(v, L, bv, bi)) { bv = v; bi = L; bl = i; }
        }
        warp_best(bv, bi, bl);
        if (bl >= 0) {
            const float* src = rows + (size_t)bl * ldr;
            unsigned long long* dst = a.crow + ((size_t)(1 % LZ_NS) * G + b) * ldr;
            for (int c = lane; c < ldr; c += 32) __stcg(&dst[c], mix_tag(1u, src[c]));
        }
        __syncwarp();
        if (lane == 0) st_relaxed_u64(&hdr[(1 & 1) * G + b], mix_pack(1u, bi, bv));
    }

    const uint64_t t_start = globaltimer_ns();
    for (int k = 1; k <= n - 2; ++k) {
        const int par = k & 1;
        // ---- wait for step k from every CTA; pick the pivot (the eager kernel's poll) ----
        if (warp == 0) {
            const unsigned long long* H = hdr + par * G;
            const unsigned want = (unsigned)k & 0xffffu;
            unsigned long long hv[5];  // G <= 160
            unsigned pending = 0;
            {
                int q = 0;
                for (int s = lane; s < G; s += 32, ++q) pending |= 1u << q;
            }
            const uint64_t t0 = globaltimer_ns();
            unsigned spins = 0;
            int ok = 1;
            unsigned long long wa[5] = {0, 0, 0, 0, 0}, wc[5] = {0, 0, 0, 0, 0};
            auto issue = [&](unsigned long long (&w)[5]) {
#pragma unroll
                for (int qq = 0; qq < 5; ++qq) {
                    const int s = lane + 32 * qq;
                    if (s < G && ((pending >> qq) & 1u)) w[qq] = ld_relaxed_u64(&H[s]);
                }
            };
            auto absorb = [&](const unsigned long long (&w)[5]) {
#pragma unroll
                for (int qq = 0; qq < 5; ++qq)
                    if (((pending >> qq) & 1u) && ((unsigned)(w[qq] >> 16) & 0xffffu) == want) {
                        hv[qq] = w[qq];
                        pending &= ~(1u << qq);
                    }
            };
            issue(wa);
            __nanosleep(MIX_POLL_GAP_NS);
            issue(wc);
            for (;;) {
                absorb(wa);
                if (__all_sync(0xffffffffu, pending == 0)) break;
                issue(wa);
                absorb(wc);
                if (__all_sync(0xffffffffu, pending == 0)) break;
                issue(wc);
                if (((spins += 2) & 15u) == 0) {
                    int bad = 0;
                    if (lane == 0) {
                        if (ld_acquire_i32(a.err) != 0) bad = 1;
                        else if (globaltimer_ns() - t0 > a.limit_ns) {
                            atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
                            bad = 1;
                        }
                    }
                    if (__shfl_sync(0xffffffffu, bad, 0)) { ok = 0; break; }
                }
            }
            float bv = 0.f;
            int bi = 0, bs = -1;
            if (ok) {
#pragma unroll
                for (int qq = 0; qq < 5; ++qq) {
                    const int s = lane + 32 * qq;
                    if (s < G) {
                        const int i = (int)(hv[qq] & 0xffffu);
                        const float v = __uint_as_float((unsigned)(hv[qq] >> 32));
                        if (mix_better(v, i, bv, bi)) { bv = v; bi = i; bs = s; }
                    }
                }
                warp_best(bv, bi, bs);
            }
            if (lane == 0) {
                s_ok = ok;
                const int p = (ok && bs >= 0 && bi >= k + 1 && bi <= n) ? bi : k + 1;
                s_p = p;
                s_win = (ok && bs >= 0 && bi >= k + 1 && bi <= n) ? bs : -1;
                s_piv = s_win >= 0 ? bv : 0.f;
                if (ok && b == 0) a.ipiv[k - 1] = p;
            }
        }
        __syncthreads();
        if (!s_ok) return;
        const int p = s_p;
        const int win = s_win;
        const float piv = s_piv;
        const int K0 = z.K0;
        const int js = k - K0;  // this step's index in the panel
        const bool last = (js == LZ_NB - 1) || (k == n - 2);  // the panel ends with this step
        // ---- interchange k+1 <-> p: row labels, and the column table (no data moves) ----
        if (t == 0) {
            if (p != k + 1) {
                const int x = ph[k + 1], w = ph[p];
                ph[k + 1] = w;
                ph[p] = x;
                lg[w] = k + 1;
                lg[x] = p;
                const int Pa = lz_cph(z, k + 1), Pb = lz_cph(z, p);
                int qa = -1, qb = -1;
                for (int q = 0; q < z.ntouch; ++q) {
                    if (z.tP[q] == Pa) qa = q;
                    if (z.tP[q] == Pb) qb = q;
                }
                if (qa < 0) { qa = z.ntouch++; z.tP[qa] = Pa; tbits[Pa >> 5] |= 1u << (Pa & 31); }
                if (qb < 0) { qb = z.ntouch++; z.tP[qb] = Pb; tbits[Pb >> 5] |= 1u << (Pb & 31); }
                z.tL[qa] = p;      // Pa held logical k+1, now p
                z.tL[qb] = k + 1;  // Pb held logical p, now k+1
            }
            z.win[js] = win;
            z.pk = lz_cph(z, k);
            z.pk1 = lz_cph(z, k + 1);
        }
        __syncthreads();
        const int pk1 = z.pk1;
        // ---- pivot row (physical order, from the winner's ring slot), multipliers by logical row
        // (from the prefetched column values, slots by the labels before the interchange) ----
        {
            const unsigned long long* src = win >= 0 ? lz_urow(a, k, win, G) : nullptr;
            const unsigned want = (unsigned)k & 0xffffu;
            bool ok = true;
            const int P0 = K0;  // the panel's first column (0-based position of logical K0 + 1)
            for (int base = P0; base < ldr; base += 4 * MT) {
                unsigned long long rv[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int P = base + t + u * MT;
                    rv[u] = (src && P < n) ? ld_relaxed_u64(&src[P]) : mix_tag((unsigned)k, 0.f);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int P = base + t + u * MT;
                    float r = __uint_as_float((unsigned)(rv[u] >> 32));
                    if (src && P < n && ((unsigned)(rv[u] >> 16) & 0xffffu) != want) r = ld_tagged(&src[P], k, a.limit_ns, ok);
                    if (P < ldr) R[P] = P < n ? r : 0.f;
                }
            }
            if (!ok) atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
            for (int jj = k + 1 + t; jj < n; jj += MT) {  // slot of logical row jj + 1 >= k + 2
                const float cq = lv[jj == p - 1 ? k : jj];
                lv[jj] = piv != 0.f ? cq / piv : 0.f;
            }
        }
        __syncthreads();
        // slots of logical rows K0+1 .. k+1 are no multipliers (zero for the dot products, which
        // start at the panel's first column); U_s[k+1] of the panel's earlier steps
        for (int jj = K0 + t; jj <= k; jj += MT) lv[jj] = 0.f;
        if (t < js) {
            bool ok = true;
            const unsigned long long* u = lz_urow(a, K0 + t, z.win[t], G);
            z.ucol[t] = z.win[t] >= 0 ? ld_tagged(&u[pk1], K0 + t, a.limit_ns, ok) : 0.f;
            if (!ok) atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
        }
        __syncthreads();
        // the dot-product fix at touched positions: l_{logical(P)} - lv[P]
        if (t < z.ntouch) {
            const int P = z.tP[t], L = z.tL[t];
            z.tdl[t] = (L >= k + 2 ? lv[L - 1] : 0.f) - lv[P];
        }
        __syncthreads();

        // ---- dot products (FP64 accumulation of FP32 products) from the panel's first column:
        // own stored rows and R as in the eager kernel's items (4 rows x one of 4 column parts per
        // warp, the touched-position fix in part 0), then the panel's U_s rows, one warp each ----
        const int ntouch = z.ntouch;
        {
            const int nv = nr + 1;  // own rows, then R
            const int c0 = K0, c4 = (c0 + 3) & ~3;
            const int g0 = c4 >> 2, g1 = ldr >> 2;
            const int per = (g1 - g0 + 3) >> 2;
            const float4* l4 = reinterpret_cast<const float4*>(lv);
            const int nitems = ((nv + 3) >> 2) * 4;
            for (int item = warp; item < nitems + js; item += MW) {
                if (item >= nitems) {  // U_s . l for the panel's step s = K0 + (item - nitems)
                    const int si = item - nitems;
                    double acc = 0.0;
                    const int w = z.win[si];
                    if (w >= 0) {
                        const unsigned long long* u = lz_urow(a, K0 + si, w, G);
                        bool ok = true;
                        for (int P = c0 + lane; P < n; P += 32) {
                            const unsigned long long v = ld_relaxed_u64(&u[P]);
                            float x = __uint_as_float((unsigned)(v >> 32));
                            if (((unsigned)(v >> 16) & 0xffffu) != ((unsigned)(K0 + si) & 0xffffu))
                                x = ld_tagged(&u[P], K0 + si, a.limit_ns, ok);
                            acc += (double)(x * lv[P]);
                        }
                        for (int q = lane; q < ntouch; q += 32) {
                            const float x = ld_tagged(&u[z.tP[q]], K0 + si, a.limit_ns, ok);
                            acc += (double)(x * z.tdl[q]);
                        }
                        if (!ok) atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
                    }
                    acc = warp_sum(acc);
                    if (lane == 0) z.gam[si] = acc;
                    continue;
                }
                const int rg = item >> 2, cp = item & 3;
                const float* xq[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int v = min(rg * 4 + q, nr);
                    xq[q] = v < nr ? rows + (size_t)v * ldr : R;
                }
                double acc[4] = {0.0, 0.0, 0.0, 0.0};
                if (cp == 0) {
                    if (c0 + lane < c4 && c0 + lane < ldr) {  // the unaligned head
#pragma unroll
                        for (int q = 0; q < 4; ++q) acc[q] = (double)(xq[q][c0 + lane] * lv[c0 + lane]);
                    }
                    for (int q2 = lane; q2 < ntouch; q2 += 32) {  // touched positions
                        const int P = z.tP[q2];
                        const float d = z.tdl[q2];
#pragma unroll
                        for (int q = 0; q < 4; ++q) acc[q] += (double)(xq[q][P] * d);
                    }
                }
                float pp[4][4];
#pragma unroll
                for (int q = 0; q < 4; ++q) pp[q][0] = pp[q][1] = pp[q][2] = pp[q][3] = 0.f;
                int it = 0;
                const int ga = g0 + cp * per, gb = min(ga + per, g1);
                for (int g = ga + lane; g < gb; g += 32) {
                    const float4 l = l4[g];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float4 x = reinterpret_cast<const float4*>(xq[q])[g];
                        pp[q][0] = fmaf(x.x, l.x, pp[q][0]);
                        pp[q][1] = fmaf(x.y, l.y, pp[q][1]);
                        pp[q][2] = fmaf(x.z, l.z, pp[q][2]);
                        pp[q][3] = fmaf(x.w, l.w, pp[q][3]);
                    }
                    if (++it == MIX_FLUSH) {
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            acc[q] += ((double)pp[q][0] + (double)pp[q][1]) + ((double)pp[q][2] + (double)pp[q][3]);
                            pp[q][0] = pp[q][1] = pp[q][2] = pp[q][3] = 0.f;
                        }
                        it = 0;
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    acc[q] += ((double)pp[q][0] + (double)pp[q][1]) + ((double)pp[q][2] + (double)pp[q][3]);
                const bool h16 = lane & 16, h8 = lane & 8;
                const double e0 = __shfl_xor_sync(0xffffffffu, h16 ? acc[0] : acc[2], 16);
                const double e1 = __shfl_xor_sync(0xffffffffu, h16 ? acc[1] : acc[3], 16);
                const double k0 = (h16 ? acc[2] : acc[0]) + e0, k1 = (h16 ? acc[3] : acc[1]) + e1;
                double sum = (h8 ? k1 : k0) + __shfl_xor_sync(0xffffffffu, h8 ? k0 : k1, 8);
                sum += __shfl_xor_sync(0xffffffffu, sum, 4);
                sum += __shfl_xor_sync(0xffffffffu, sum, 2);
                sum += __shfl_xor_sync(0xffffffffu, sum, 1);
                const int q = lane >> 3;
                if ((lane & 7) == 0 && rg * 4 + q < nv) s_part[(rg * 4 + q) * 4 + cp] = sum;
            }
        }
        __syncthreads();
        // ---- warp 0: new column k+1 of own rows (completed in the stored rows), multipliers into
        // column k, the next candidate and its header ----
        if (warp == 0) {
            float bv = 0.f;
            int bi = 0, bl = -1;
            const int np = (k + 1) & 1;
            auto dot = [&](int v) {
                return (s_part[4 * v] + s_part[4 * v + 1]) + (s_part[4 * v + 2] + s_part[4 * v + 3]);
            };
            const double gk = (double)R[pk1] + dot(nr);  // Gamma_k
            const int pk = z.pk;
            for (int i = lane; i < nr; i += 32) {
                float* ri = rows + (size_t)i * ldr;
                const int L = lg[r0 + i];
                const float li = L >= k + 2 ? lv[L - 1] : 0.f;
                double cn = (double)ri[pk1] + dot(i);
                for (int s = 0; s < js; ++s) {
                    const float lm = s_lm[i][s];
                    if (lm != 0.f) cn -= (double)lm * ((double)z.ucol[s] + z.gam[s]);
                }
                cn -= (double)li * gk;
                const float c32 = (float)cn;
                ri[pk1] = c32;
                if (L >= k + 2) ri[pk] = li;
                s_li[i] = li;
                s_lm[i][js] = li;
                if (k + 1 <= n - 2) __stcg(&a.cval[(size_t)np * n + r0 + i], mix_tag((unsigned)(k + 1), c32));
                if (L >= k + 2 && mix_better(c32, L, bv, bi)) { bv = c32; bi = L; bl = i; }
            }
            warp_best(bv, bi, bl);
            if (lane == 0) {
                s_cand = bl;
                if (k + 1 <= n - 2) st_relaxed_u64(&hdr[np * G + b], mix_pack((unsigned)(k + 1), bi, bv));
            }
        }
        __syncthreads();
        const int cl = s_cand;
        if (warp != 0) {
            const int tw = t - 32, TW = MT - 32;  // warps 1-15
            // ---- publish step k+1's candidate row in its true form:
            //   S[cl, P] - sum_{s <= k} l_cl^(s) U_s[P] at columns not yet complete (logical >= k+2),
            // the stored value elsewhere; in the next panel's column order if this step ends the panel
            if (k + 1 <= n - 2 && cl >= 0) {
                const float* rc = rows + (size_t)cl * ldr;
                unsigned long long* dst = a.crow + ((size_t)((k + 1) % LZ_NS) * G + b) * ldr;
                const unsigned st = (unsigned)(k + 1);
                const int nsd = js + 1;  // steps of the panel so far, this one included
                bool ok = true;
                // every word of the row is stored once (a reader may take any stored word whose tag
                // is the step's): the touched positions only by the second loop below
                for (int P = K0 + tw; P < ldr; P += TW) {
                    if ((tbits[P >> 5] >> (P & 31)) & 1u) continue;
                    float x = rc[P];
                    // identity positions: complete iff P + 1 <= k + 1
                    if (P >= k + 1 && P < n) {
                        for (int s = 0; s < nsd; ++s) {
                            const float lm = s_lm[cl][s];
                            if (lm == 0.f) continue;
                            const float u = s == js ? R[P] : ld_tagged(&lz_urow(a, K0 + s, z.win[s], G)[P], K0 + s,
                                                                       a.limit_ns, ok);
                            x = fmaf(-lm, u, x);
                        }
                    }
                    __stcg(&dst[P], mix_tag(st, x));
                }
                if (!ok) atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
                named_bar_sync(1, TW);
                // touched positions: their own completeness; and the move to logical order at a panel end
                for (int q = tw; q < ntouch; q += TW) {
                    const int P = z.tP[q], L = z.tL[q];
                    float x = rc[P];
                    if (L >= k + 2) {
                        for (int s = 0; s < nsd; ++s) {
                            const float lm = s_lm[cl][s];
                            if (lm == 0.f) continue;
                            const float u = s == js ? R[P] : ld_tagged(&lz_urow(a, K0 + s, z.win[s], G)[P], K0 + s,
                                                                       a.limit_ns, ok);
                            x = fmaf(-lm, u, x);
                        }
                    }
                    z.tdl[q] = x;  // the value at P (tdl is free until the next step)
                }
                named_bar_sync(1, TW);
                for (int q = tw; q < ntouch; q += TW) {
                    const int P = z.tP[q], L = z.tL[q];
                    __stcg(&dst[last ? L - 1 : P], mix_tag(st, z.tdl[q]));
                }
                if (!ok) atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
            }
            if (last) {
                // ---- panel end: S[i, P] -= sum_s l_i^(s) U_s[P] at the columns after the panel
                // (logical >= k + 2), chunks of LZ_CH columns staged in lv, then the touched
                // positions moved to their logical places ----
                named_bar_sync(1, TW);
                const int nsd = js + 1;
                for (int i = tw; i < nr; i += TW) {  // rows with a delayed update
                    int any = 0;
                    for (int s = 0; s < nsd; ++s) any |= s_lm[i][s] != 0.f;
                    s_li[i] = any ? 1.f : 0.f;
                }
                bool ok = true;
                for (int c0 = K0; c0 < n; c0 += LZ_CH) {
                    for (int e = tw; e < nsd * LZ_CH; e += TW) {
                        const int s = e / LZ_CH, P = c0 + e % LZ_CH;
                        float u = 0.f;
                        if (P < n && (s == js || z.win[s] >= 0)) {
                            int L = P + 1;
                            for (int q = 0; q < ntouch; ++q)
                                if (z.tP[q] == P) L = z.tL[q];
                            if (L >= k + 2)
                                u = s == js ? R[P] : ld_tagged(&lz_urow(a, K0 + s, z.win[s], G)[P], K0 + s, a.limit_ns, ok);
                        }
                        Us[e] = u;
                    }
                    named_bar_sync(1, TW);
                    for (int e = tw; e < nr * LZ_CH; e += TW) {
                        const int i = e / LZ_CH, cc = e % LZ_CH, P = c0 + cc;
                        if (P >= n || s_li[i] == 0.f) continue;
                        float* ri = rows + (size_t)i * ldr;
                        float x = ri[P];
                        for (int s = 0; s < nsd; ++s) {
                            const float lm = s_lm[i][s];
                            if (lm != 0.f) x = fmaf(-lm, Us[s * LZ_CH + cc], x);
                        }
                        ri[P] = x;
                    }
                    named_bar_sync(1, TW);
                }
                if (!ok) atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
                // move the touched positions: row i's value at P goes to L - 1 (at most 2 LZ_NB + 2
                // of them: two per lane)
                for (int i = warp - 1; i < nr; i += MW - 1) {
                    float* ri = rows + (size_t)i * ldr;
                    float v0 = 0.f, v1 = 0.f;
                    if (lane < ntouch) v0 = ri[z.tP[lane]];
                    if (lane + 32 < ntouch) v1 = ri[z.tP[lane + 32]];
                    __syncwarp();
                    if (lane < ntouch) ri[z.tL[lane] - 1] = v0;
                    if (lane + 32 < ntouch) ri[z.tL[lane + 32] - 1] = v1;
                }
                named_bar_sync(1, TW);
                // the next panel starts in logical column order with no delayed rows
                for (int e = tw; e < MIX_RPC_MAX * LZ_NB; e += TW) s_lm[e / LZ_NB][e % LZ_NB] = 0.f;
                if (tw == 0) {
                    for (int q = 0; q < ntouch; ++q) tbits[z.tP[q] >> 5] &= ~(1u << (z.tP[q] & 31));
                    z.ntouch = 0;
                    z.K0 = k + 1;
                }
            }
            if (k + 1 <= n - 2) prefetch_cval(k + 1);
        }
    }
    __syncthreads();
    if (b == 0 && t == 0 && a.ptimes) a.ptimes[6] += globaltimer_ns() - t_start;

    // ---- write own rows to their logical positions (FP64) ----
    for (int e = t; e < nr * n; e += MT) {
        const int i = e % nr, c = e / nr;
        a.A[(size_t)c * n + (lg[r0 + i] - 1)] = (double)rows[(size_t)i * ldr + c];
    }
    if (b == 0)
        for (int q = t; q < n; q += MT) {
            a.perm[q] = ph[q + 1] + 1;
            a.iperm[q] = lg[q];
        }
}

size_t lazy_smem_bytes(int ldr)
{
    return (size_t)ldr * 4 * sizeof(float) + 4 * sizeof(int) + (size_t)LZ_NB * LZ_CH * sizeof(float) +
           (size_t)((ldr + 31) / 32) * sizeof(unsigned);
}

cudaError_t launch_reduce_mixed_lazy(MixArgs a, const MixPlan& pl, cudaStream_t st)
{
    if (!pl.ok) return cudaErrorInvalidValue;
    a.rpc = pl.rpc;
    a.ldr = pl.ldr;
    const size_t smem = lazy_smem_bytes(pl.ldr);
    if (smem > MIX_SMEM_MAX) return cudaErrorInvalidValue;
    static size_t attr = 0;
    if (smem > attr) {
        cudaError_t e = cudaFuncSetAttribute(reduce_mixed_lazy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        attr = smem;
    }
    void* args[] = {&a};
    return cudaLaunchCooperativeKernel((const void*)reduce_mixed_lazy_kernel, dim3(pl.grid), dim3(MT), args, smem,
                                       st);
}

}  // namespace lhl
