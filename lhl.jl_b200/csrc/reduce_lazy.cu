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
// What is delayed.  The eager kernel subtracts l_i R from every own row below the pivot at
// every step (a read and a write of the trailing block per step).  Here the stored rows S keep
// their values from the start of the panel.  With U_s the true pivot row of panel step s and
// l_i^(s) row i's multiplier at that step (zero unless the row was below that pivot), row i's
// true entries in every column not yet complete are
//     A[i, c] = S[i, c] - sum_{s < k} l_i^(s) U_s[c].
// The winner of a step publishes its STORED row and its multipliers of the panel so far; the
// true pivot rows then follow from the stored ones, V_s, through a unit lower triangular
// transform: U_s = V_s - sum_{t < s} T[s][t] U_t with T[s][t] = l_{w_s}^(t), the multipliers of
// step s's winning row (the form of a blocked Householder product, here for Gauss transforms).
// Step k needs (l = the step's multipliers, P the physical column order):
//   * g_s = V_s . l and V_s[k+1] for the panel's steps s <= k: each V_s is still one of its
//     owner's rows, so its owner has both (its own dot product and stored value) and publishes
//     them, with the row T[k] of this step's winner; nobody else reads the pivot rows during
//     the panel.  Then by the transform
//         gamma_s = g_s - sum_{t < s} T[s][t] gamma_t,   u_s = V_s[k+1] - sum_{t < s} T[s][t] u_t;
//   * the new column k+1 of own row i (the column update A[:, k+1] += A[:, k+2:n] l after the
//     row update), written into the stored row -- the column is complete from then on:
//         c'_i = S[i, k+1] + S[i, :] . l - sum_{s <= k} l_i^(s) (u_s + gamma_s);
//   * at the panel's end, S[i, c] -= sum_s l_i^(s) U_s[c] = sum_s w_i^(s) V_s[c] for every
//     column c after the panel, with (I + T)^T w_i = l_i (a back substitution of 16 terms),
//     then the candidate row of the next step is published in its updated form.
// The published rows live in a ring of LZ_NS slots, so every CTA reads the panel's V_s from the
// winners' slots until the panel ends.  Column interchanges are not applied to the stored rows
// during a panel (the published V_s would go out of step): logical column L sits at physical
// position L - 1 except at the few positions the panel's interchanges touched, kept in a small
// table; at the panel's end each CTA moves those positions to their logical places, so each
// panel starts in logical column order.  The dot products start at the panel's first column.
// Every exchange word is stored once per step: a reader takes any word whose tag is the step's.
//
// Arithmetic: FP32 storage; dot products of FP32 products with FP64 accumulation; the
// transform and the new column value in FP64, rounded once when stored; the rank-LZ_NB update
// in FP32 fused multiply-adds.  The pivot search is the eager kernel's (the reference's first
// maximum on the FP32 column values).  At the end every CTA writes its rows in FP64 to their
// logical positions of `factors`, and CTA 0 writes perm / iperm: the eager kernel's outputs.
#include "mixed_common.cuh"

namespace lhl {

constexpr int LZ_NB = MIX_LAZY_LM;      // steps per panel
constexpr int LZ_NS = MIX_LAZY_RING;    // slots of the ring of published rows
static_assert(LZ_NS >= LZ_NB + 2, "the ring holds a panel's pivot rows and the next step's candidates");
constexpr int LZ_TMAX = 2 * LZ_NB + 2;  // column positions a panel's interchanges can touch
constexpr int LZ_XW = 4 * LZ_NB;        // words per step parity of the pivot rows' exchange
constexpr int LZ_RING_MAX = 24;         // rows in flight per thread in the panel update (cp.async ring)

struct LazyShared {
    int tP[LZ_TMAX];          // touched physical positions (0-based) ...
    int tL[LZ_TMAX];          // ... and the logical column (1-based) each now holds
    float tdl[LZ_TMAX];       // per step: l_{tL} - lv[tP] (the dot-product fix at touched positions)
    int ntouch;
    int win[LZ_NB];           // winning CTA of each panel step
    float T[LZ_NB][LZ_NB];    // T[s][t] = l_{w_s}^(t), t < s
    float vcol[LZ_NB];        // V_s[pk1] of the panel's pivot rows s <= js (from their owners)
    double gsum[LZ_NB];       // V_s . l of the panel's pivot rows s <= js (from their owners)
    double Gam[LZ_NB + 1];    // u_s + gamma_s for s < k, [js]: this step's pivot row's
    int K0;                   // the panel's first step
    int pk, pk1;              // physical positions of logical columns k and k+1
};


// 8-byte asynchronous copy of 2 floats global -> shared (cp.async); both addresses 8-byte
// aligned
__device__ __forceinline__ void lz_cp8(float* dst, const float* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}

// barrier of the `count` threads of warps 1-15 (id 1; warp 0 is polling meanwhile)
__device__ __forceinline__ void named_bar_sync(int id, int count)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// winner w's published row of step s (ldr words, then LZ_NB multipliers), tagged with the step
__device__ __forceinline__ const unsigned long long* lz_urow(const MixArgs& a, int s, int w, int G)
{
    return a.crow + ((size_t)(s % LZ_NS) * G + w) * (size_t)(a.ldr + LZ_NB);
}

// The panel end's rank-LZ_NB update S[i, P] -= sum_s w_i^(s) V_s[P] for the rows in `ul`
// (nu rows with a delayed update), every column P from the panel's first one whose logical
// column is >= k + 2.  Thread tw of the TW threads of warps 1-15 takes pairs of columns: it
// holds the 2 columns of every V_s in registers (from the winners' ring slots, every one of
// them published before this step ended) and streams the rows
// through a ring of D 8-byte slots of its own, filled by cp.async D rows ahead, so that D rows
// of its columns are in flight at once.  A slot is refilled only after its value has been used
// (the refill follows the store that depends on it).  Columns that take no update keep their
// values (V is zero there) and their exchange words are not read.
template <int D>
__device__ __forceinline__ void lz_panel_update(const MixArgs& a, float* rows, int ldr, int n, int k, int K0,
                                                int js, int G, const LazyShared& z,
                                                const float (*w)[LZ_NB], const int* ul, int nu, float2* ring,
                                                int tw, int TW, bool& ok)
{
    float2* mine = ring + (size_t)tw * D;
    const int g0 = K0 >> 1, g1 = ldr >> 1;
    const int ntouch = z.ntouch;
    for (int g = g0 + tw; g < g1; g += TW) {
        const int P0 = 2 * g;
        // logical columns >= k + 2 take the update: positions >= k + 1 unless touched, and the
        // touched positions by their table entry
        bool m0 = P0 >= k + 1 && P0 < n, m1 = P0 + 1 >= k + 1 && P0 + 1 < n;
        for (int q = 0; q < ntouch; ++q) {
            const int P = z.tP[q];
            if (P == P0) m0 = z.tL[q] >= k + 2;
            if (P == P0 + 1) m1 = z.tL[q] >= k + 2;
        }
        if (!m0 && !m1) continue;
        float v[LZ_NB][2];
#pragma unroll
        for (int s = 0; s < LZ_NB; ++s) {
            v[s][0] = v[s][1] = 0.f;
            if (s <= js && z.win[s] >= 0) {
                const unsigned long long* u = lz_urow(a, K0 + s, z.win[s], G) + P0;
                const ulonglong2 p = __ldcg(reinterpret_cast<const ulonglong2*>(u));
                const unsigned want = (unsigned)(K0 + s) & 0xffffu;
                float x0 = __uint_as_float((unsigned)(p.x >> 32)), x1 = __uint_as_float((unsigned)(p.y >> 32));
                if (m0 && ((unsigned)(p.x >> 16) & 0xffffu) != want) x0 = ld_tagged(u, K0 + s, a.limit_ns, ok);
                if (m1 && ((unsigned)(p.y >> 16) & 0xffffu) != want) x1 = ld_tagged(u + 1, K0 + s, a.limit_ns, ok);
                v[s][0] = m0 ? x0 : 0.f;
                v[s][1] = m1 ? x1 : 0.f;
            }
        }
#pragma unroll
        for (int q = 0; q < D; ++q) {
            if (q < nu) lz_cp8(reinterpret_cast<float*>(&mine[q]), rows + (size_t)ul[q] * ldr + P0);
            cp_async_commit();
        }
        for (int q = 0; q < nu; ++q) {
            cp_async_wait<D - 1>();
            float2 x = mine[q % D];
            const float* wi = w[ul[q]];
#pragma unroll
            for (int s = 0; s < LZ_NB; ++s) {
                const float ws = wi[s];
                x.x = fmaf(-ws, v[s][0], x.x);
                x.y = fmaf(-ws, v[s][1], x.y);
            }
            *reinterpret_cast<float2*>(rows + (size_t)ul[q] * ldr + P0) = x;
            if (q + D < nu) lz_cp8(reinterpret_cast<float*>(&mine[q % D]), rows + (size_t)ul[q + D] * ldr + P0);
            cp_async_commit();
        }
        cp_async_wait<0>();
    }
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
    __shared__ int s_ul[MIX_RPC_MAX];  // panel end: own rows with a delayed update
    __shared__ int s_nu;
    __shared__ int s_act[MIX_RPC_MAX];  // own rows below the panel's first step (logical label > K0)
    __shared__ int s_nact;
    __shared__ int s_pos[MIX_RPC_MAX];  // own row -> its place in s_act (-1: above the panel)

    const int n = a.n, rpc = a.rpc, ldr = a.ldr, G = gridDim.x, b = blockIdx.x;
    const int ldrr = ldr + LZ_NB;  // words per CTA in a ring slot
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int r0 = b * rpc;
    const int nr = min(rpc, n - r0);
    float* lv = slz;             // multipliers by logical row (slot L-1)
    int* lg = (int*)(lv + ldr);  // physical row -> logical (1-based)
    int* ph = lg + ldr;          // logical (1-based) -> physical row, ph[0] unused
    float2* ring = (float2*)(ph + ldr + 4);  // panel update: 8-byte slots (a.ring per thread of warps 1-15)
    float* rows = a.grows + (size_t)r0 * ldr;  // nr x ldr, FP32, global
    unsigned long long* hdr = a.hdr;

    // ---- load own rows (FP64 -> FP32, zero pads), labels ----
    for (int e = t; e < nr * ldr; e += MT) {
        const int c = e % ldr, i = e / ldr;
        rows[(size_t)i * ldr + c] = c < n ? (float)a.A[(size_t)c * n + r0 + i] : 0.f;
    }
    for (int q = t; q < ldr; q += MT) {
        lv[q] = 0.f;
        if (q < n) {
            lg[q] = q + 1;
            ph[q + 1] = q;
        }
    }
    for (int e = t; e < MIX_RPC_MAX * LZ_NB; e += MT) s_lm[e / LZ_NB][e % LZ_NB] = 0.f;
    if (t == 0) {
        z.ntouch = 0;
        z.K0 = 1;
        int c = 0;
        for (int i = 0; i < nr; ++i) {
            s_pos[i] = -1;
            if (r0 + i + 1 > 1) {
                s_pos[i] = c;
                s_act[c++] = i;
            }
        }
        s_nact = c;
    }
    __syncthreads();

    // warps 1-15: column values of step st by logical row, of the rows with labels > kmin (the
    // rows above the panel publish none)
    auto prefetch_cval = [&](int st, int kmin) {
        constexpr int PF = 8;
        const unsigned long long* cv = a.cval + (size_t)(st & 1) * n;
        const unsigned want = (unsigned)st & 0xffffu;
        bool ok = true;
        for (int base = t - 32; base < n; base += PF * (MT - 32)) {
            unsigned long long w[PF];
#pragma unroll
            for (int u = 0; u < PF; ++u) {
                const int q = base + u * (MT - 32);
                w[u] = (q < n && lg[q] > kmin) ? ld_relaxed_u64(&cv[q]) : 0ull;
            }
#pragma unroll
            for (int u = 0; u < PF; ++u) {
                const int q = base + u * (MT - 32);
                if (q < n && lg[q] > kmin) {
                    float v = __uint_as_float((unsigned)(w[u] >> 32));
                    if (((unsigned)(w[u] >> 16) & 0xffffu) != want) v = ok ? ld_tagged(&cv[q], (unsigned)st, a.limit_ns, ok) : 0.f;
                    lv[lg[q] - 1] = v;
                }
            }
        }
        if (!ok) atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
    };
    // the candidate row of step st (own row cl) as stored, from position p0, and its multipliers
    // lm (null: zeros), into ring slot st; every word stored once (warps 1-15)
    auto publish = [&](int st, int cl, int p0, const float* lm) {
        const int tw = t - 32, TW = MT - 32;
        const float* rc = rows + (size_t)cl * ldr;
        unsigned long long* dst = a.crow + ((size_t)(st % LZ_NS) * G + b) * (size_t)ldrr;
        for (int P = p0 + tw; P < ldr; P += TW) __stcg(&dst[P], mix_tag((unsigned)st, rc[P]));
        if (tw < LZ_NB) __stcg(&dst[ldr + tw], mix_tag((unsigned)st, lm ? lm[tw] : 0.f));
    };

    // ---- publish step 1: column 1 values, candidate among logical rows >= 2 ----
    if (warp != 0) prefetch_cval(1, 1);
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
        if (lane == 0) s_cand = bl;
        __syncwarp();
        if (lane == 0) st_relaxed_u64(&hdr[(1 & 1) * G + b], mix_pack(1u, bi, bv));
    }
    __syncthreads();
    if (warp != 0 && s_cand >= 0) publish(1, s_cand, 0, nullptr);

    const uint64_t t_start = globaltimer_ns();
    // CTA 0's time per phase, summed over steps (lhl_ws_set_probes).  Thread 0: slot 0 the wait
    // for step k (warp 0's poll, and warps 1-15's work of the step before), 1 interchange and
    // pivot row, 2 dot products, 3 transform, 4 new column; slot 5 the poll alone.  Thread 32
    // (warps 1-15): slot 8 publishing a candidate row, 9 the panel end, 10 the column-value
    // prefetch.
    unsigned long long* probe = (b == 0 && (t == 0 || t == 32) && a.ptimes) ? a.ptimes + 8 : nullptr;
    uint64_t tp = t_start;
    auto mark = [&](int slot) {
        if (probe) {
            const uint64_t now = globaltimer_ns();
            probe[slot] += now - tp;
            tp = now;
        }
    };
    for (int k = 1; k <= n - 2; ++k) {
        const int par = k & 1;
        if (t == 0) tp = globaltimer_ns();
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
            if (probe && t == 0) probe[5] += globaltimer_ns() - tp;
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
        if (t == 0) mark(0);
        if (!s_ok) return;
        const int p = s_p;
        const int win = s_win;
        const float piv = s_piv;
        const int K0 = z.K0;
        const int nact = s_nact;  // own rows below K0 (the rows above wait for the deferred product)
        const int js = k - K0;  // this step's index in the panel
        const bool last = (js == LZ_NB - 1) || (k == n - 2);  // the panel ends with this step
        // ---- interchange k+1 <-> p: row labels, and the column table (no data moves) ----
        // (warp 0: the table's at most 2 LZ_NB + 2 entries two per lane, looked up by ballots)
        if (warp == 0) {
            const int nt = z.ntouch;
            const int P0v = lane < nt ? z.tP[lane] : -1, L0v = lane < nt ? z.tL[lane] : -1;
            const int P1v = lane + 32 < nt ? z.tP[lane + 32] : -1, L1v = lane + 32 < nt ? z.tL[lane + 32] : -1;
            auto cph = [&](int L) {  // physical position (0-based) of logical column L (1-based)
                const unsigned m0 = __ballot_sync(0xffffffffu, L0v == L), m1 = __ballot_sync(0xffffffffu, L1v == L);
                if (m0) return __shfl_sync(0xffffffffu, P0v, __ffs(m0) - 1);
                if (m1) return __shfl_sync(0xffffffffu, P1v, __ffs(m1) - 1);
                return L - 1;
            };
            auto entry = [&](int P) {  // the table entry of position P, or -1
                const unsigned m0 = __ballot_sync(0xffffffffu, P0v == P), m1 = __ballot_sync(0xffffffffu, P1v == P);
                return m0 ? __ffs(m0) - 1 : (m1 ? 32 + __ffs(m1) - 1 : -1);
            };
            const int pkv = cph(k);  // logical k is not part of this step's interchange
            int pk1v;
            if (p != k + 1) {
                const int Pa = cph(k + 1), Pb = cph(p);
                int qa = entry(Pa), qb = entry(Pb);
                if (lane == 0) {
                    const int x = ph[k + 1], w = ph[p];
                    ph[k + 1] = w;
                    ph[p] = x;
                    lg[w] = k + 1;
                    lg[x] = p;
                    int nt2 = nt;
                    if (qa < 0) { qa = nt2++; z.tP[qa] = Pa; }
                    if (qb < 0) { qb = nt2++; z.tP[qb] = Pb; }
                    z.tL[qa] = p;      // Pa held logical k+1, now p
                    z.tL[qb] = k + 1;  // Pb held logical p, now k+1
                    z.ntouch = nt2;
                }
                pk1v = Pb;
            } else {
                pk1v = cph(k + 1);
            }
            if (lane == 0) {
                z.win[js] = win;
                z.pk = pkv;
                z.pk1 = pk1v;
            }
        }
        __syncthreads();
        const int pk1 = z.pk1;
        // ---- multipliers by logical row from the prefetched column values (slots by the labels
        // before the interchange).  The pivot row itself is not loaded: what the step needs of it
        // (its product with l, its value at the new column, its panel multipliers) comes from its
        // owner after the dot products ----
        {
            const float rp = piv != 0.f ? 1.f / piv : 0.f;  // FP32 form: one division per step
            for (int jj = k + 1 + t; jj < n; jj += MT) {  // slot of logical row jj + 1 >= k + 2
                const float cq = lv[jj == p - 1 ? k : jj];
                lv[jj] = cq * rp;
            }
        }
        __syncthreads();
        // slots of logical rows K0+1 .. k+1 are no multipliers (zero for the dot products, which
        // start at the panel's first column)
        for (int jj = K0 + t; jj <= k; jj += MT) lv[jj] = 0.f;
        __syncthreads();
        if (t < z.ntouch) {  // the dot-product fix at touched positions: l_{logical(P)} - lv[P]
            const int P = z.tP[t], L = z.tL[t];
            z.tdl[t] = (L >= k + 2 ? lv[L - 1] : 0.f) - lv[P];
        }
        __syncthreads();
        if (t == 0) mark(1);

        // ---- dot products (FP64 accumulation of FP32 products) from the panel's first column:
        // own stored rows in the eager kernel's items (4 rows x one of 4 column parts per warp,
        // the touched-position fix in part 0) ----
        const int ntouch = z.ntouch;
        const int c0 = K0;
        {
            const int nv = nact;  // own rows below the panel's first step
            const int c4 = (c0 + 3) & ~3;
            const int g0 = c4 >> 2, g1 = ldr >> 2;
            const int per = (g1 - g0 + 3) >> 2;
            const float4* l4 = reinterpret_cast<const float4*>(lv);
            const int nitems = ((nv + 3) >> 2) * 4;
            for (int item = warp; item < nitems; item += MW) {
                const int rg = item >> 2, cp = item & 3;
                const float* xq[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int v = min(rg * 4 + q, nact);
                    xq[q] = v < nact ? rows + (size_t)s_act[v] * ldr : rows;  // rows: a pad, never stored
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
                int g = ga + lane;
                // two iterations' loads (8 float4 per lane) issued before their multiply-adds
                for (; g + 32 < gb; g += 64) {
                    float4 x0[4], x1[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        x0[q] = reinterpret_cast<const float4*>(xq[q])[g];
                        x1[q] = reinterpret_cast<const float4*>(xq[q])[g + 32];
                    }
                    const float4 la = l4[g], lb = l4[g + 32];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        pp[q][0] = fmaf(x0[q].x, la.x, pp[q][0]);
                        pp[q][1] = fmaf(x0[q].y, la.y, pp[q][1]);
                        pp[q][2] = fmaf(x0[q].z, la.z, pp[q][2]);
                        pp[q][3] = fmaf(x0[q].w, la.w, pp[q][3]);
                        pp[q][0] = fmaf(x1[q].x, lb.x, pp[q][0]);
                        pp[q][1] = fmaf(x1[q].y, lb.y, pp[q][1]);
                        pp[q][2] = fmaf(x1[q].z, lb.z, pp[q][2]);
                        pp[q][3] = fmaf(x1[q].w, lb.w, pp[q][3]);
                    }
                    if ((it += 2) == MIX_FLUSH) {
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            acc[q] += ((double)pp[q][0] + (double)pp[q][1]) + ((double)pp[q][2] + (double)pp[q][3]);
                            pp[q][0] = pp[q][1] = pp[q][2] = pp[q][3] = 0.f;
                        }
                        it = 0;
                    }
                }
                for (; g < gb; g += 32) {
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
        auto dot = [&](int v) {
            return (s_part[4 * v] + s_part[4 * v + 1]) + (s_part[4 * v + 2] + s_part[4 * v + 3]);
        };
        // ---- the panel's pivot rows V_s, s = 0 .. js (js: this step's): each is still one of its
        // owner's rows below K0, and in every column where l is not zero its stored values are
        // the ones it published, so the owner's dot product above is V_s . l, and its stored value
        // at the new column is V_s[pk1].  Owners publish both (the FP64 product as two tagged
        // 32-bit halves), and this step's winner its panel multipliers, the row T[js]; the others
        // read them.  Words by step parity: [3 s, 3 s + 1] V_s . l, [3 s + 2] V_s[pk1], then
        // [3 LZ_NB + t] T[js][t] ----
        {
            unsigned long long* gx = a.cval + 2 * (size_t)n + (size_t)(k & 1) * LZ_XW;
            const unsigned long long tag = (unsigned long long)((unsigned)k & 0xffffu) << 16;
            if (t <= js) {
                const int w = z.win[t];
                double g = 0.0;
                float u = 0.f;
                if (w == b) {
                    const int i = ph[K0 + t + 1] - r0;  // the pivot row of panel step t
                    g = dot(s_pos[i]);
                    u = rows[(size_t)i * ldr + pk1];
                    const unsigned long long bits = (unsigned long long)__double_as_longlong(g);
                    __stcg(&gx[3 * t], ((bits >> 32) << 32) | tag);
                    __stcg(&gx[3 * t + 1], ((bits & 0xffffffffull) << 32) | tag);
                    __stcg(&gx[3 * t + 2], mix_tag((unsigned)k, u));
                } else if (w >= 0) {
                    bool ok = true;
                    const unsigned hi = __float_as_uint(ld_tagged(&gx[3 * t], (unsigned)k, a.limit_ns, ok));
                    const unsigned lo = __float_as_uint(ld_tagged(&gx[3 * t + 1], (unsigned)k, a.limit_ns, ok));
                    u = ld_tagged(&gx[3 * t + 2], (unsigned)k, a.limit_ns, ok);
                    if (!ok) atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
                    g = __longlong_as_double((long long)(((unsigned long long)hi << 32) | lo));
                }
                z.gsum[t] = g;
                z.vcol[t] = u;
            }
            if (t < js) {  // T[js][t]: this step's pivot row's multiplier of panel step t
                float x = 0.f;
                if (win == b) {
                    x = s_lm[ph[k + 1] - r0][t];  // s_lm is by own row, s_part by place in s_act
                    __stcg(&gx[3 * LZ_NB + t], mix_tag((unsigned)k, x));
                } else if (win >= 0) {
                    bool ok = true;
                    x = ld_tagged(&gx[3 * LZ_NB + t], (unsigned)k, a.limit_ns, ok);
                    if (!ok) atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
                }
                z.T[js][t] = x;
            }
        }
        __syncthreads();
        if (t == 0) mark(2);
        // ---- the transform: true gamma_s and u_s of the panel's pivot rows, in step order, then
        // Gamma = u + gamma.  Warp 0, lane s for step s: V_s . l and V_s[pk1] from the exchange, then a forward substitution by columns: once lane s is final
        // it is broadcast and every later lane subtracts T[r][s] times it (the same terms in the
        // same order as a row-by-row substitution) ----
        if (warp == 0) {
            double g = 0.0, u = 0.0;
            if (lane <= js) {
                g = z.gsum[lane];
                u = (double)z.vcol[lane];
            }
            for (int s2 = 0; s2 < js; ++s2) {
                const double gs = __shfl_sync(0xffffffffu, g, s2), us = __shfl_sync(0xffffffffu, u, s2);
                if (lane > s2 && lane <= js) {
                    const double tr = (double)z.T[lane][s2];
                    g -= tr * gs;
                    u -= tr * us;
                }
            }
            if (lane <= js) z.Gam[lane] = g + u;
        }
        __syncthreads();
        if (t == 0) mark(3);
        // ---- warp 0: new column k+1 of own rows (completed in the stored rows), multipliers into
        // column k, the next candidate and its header ----
        if (warp == 0) {
            float bv = 0.f;
            int bi = 0, bl = -1;
            const int np = (k + 1) & 1;
            const int pk = z.pk;
            for (int q = lane; q < nact; q += 32) {  // rows above the panel take no step
                const int i = s_act[q];
                float* ri = rows + (size_t)i * ldr;
                const int L = lg[r0 + i];
                const float li = L >= k + 2 ? lv[L - 1] : 0.f;
                double cn = (double)ri[pk1] + dot(q);
                for (int s = 0; s < js; ++s) {
                    const float lm = s_lm[i][s];
                    if (lm != 0.f) cn -= (double)lm * z.Gam[s];
                }
                cn -= (double)li * z.Gam[js];
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
        if (t == 0) mark(4);
        const int cl = s_cand;
        if (warp != 0) {
            const int tw = t - 32, TW = MT - 32;  // warps 1-15
            if (t == 32) tp = globaltimer_ns();
            if (!last) {
                // ---- publish step k+1's candidate: its stored row and its multipliers so far ----
                if (k + 1 <= n - 2 && cl >= 0) publish(k + 1, cl, K0, s_lm[cl]);
                if (t == 32) mark(8);
            } else {
                // ---- panel end: S[i, P] -= sum_s w_i^(s) V_s[P] at the columns after the panel
                // (logical >= k + 2), (I + T)^T w_i = l_i (lz_panel_update); then the touched
                // positions moved to their logical places ----
                const int nsd = js + 1;
                for (int i = tw; i < nr; i += TW) {  // w_i over l_i, in place; rows with a delayed update
                    int any = 0;
                    for (int s = nsd - 1; s >= 0; --s) {
                        float x = s_lm[i][s];
                        for (int s2 = s + 1; s2 < nsd; ++s2) x = fmaf(-z.T[s2][s], s_lm[i][s2], x);
                        s_lm[i][s] = x;
                        any |= x != 0.f;
                    }
                    s_li[i] = any ? 1.f : 0.f;
                }
                named_bar_sync(1, TW);
                if (warp == 1) {  // the list of rows with a delayed update, in row order
                    int cnt = 0;
                    for (int i0 = 0; i0 < nr; i0 += 32) {
                        const int i = i0 + lane;
                        const bool has = i < nr && s_li[i] != 0.f;
                        const unsigned bal = __ballot_sync(0xffffffffu, has);
                        if (has) s_ul[cnt + __popc(bal & ((1u << lane) - 1u))] = i;
                        cnt += __popc(bal);
                    }
                    if (lane == 0) s_nu = cnt;
                    // the rows below the next panel's first step k + 1 (labels are final for step k)
                    cnt = 0;
                    for (int i0 = 0; i0 < nr; i0 += 32) {
                        const int i = i0 + lane;
                        const bool has = i < nr && lg[r0 + i] > k + 1;
                        const unsigned bal = __ballot_sync(0xffffffffu, has);
                        if (has) s_act[cnt + __popc(bal & ((1u << lane) - 1u))] = i;
                        cnt += __popc(bal);
                    }
                    if (lane == 0) s_nact = cnt;
                    __syncwarp();
                    for (int i = lane; i < nr; i += 32) s_pos[i] = -1;
                    __syncwarp();
                    for (int q = lane; q < cnt; q += 32) s_pos[s_act[q]] = q;
                }
                named_bar_sync(1, TW);
                bool ok = true;
                if (a.ring >= 24)
                    lz_panel_update<24>(a, rows, ldr, n, k, K0, js, G, z, s_lm, s_ul, s_nu, ring, tw, TW, ok);
                else if (a.ring >= 16)
                    lz_panel_update<16>(a, rows, ldr, n, k, K0, js, G, z, s_lm, s_ul, s_nu, ring, tw, TW, ok);
                else if (a.ring >= 8)
                    lz_panel_update<8>(a, rows, ldr, n, k, K0, js, G, z, s_lm, s_ul, s_nu, ring, tw, TW, ok);
                else
                    lz_panel_update<4>(a, rows, ldr, n, k, K0, js, G, z, s_lm, s_ul, s_nu, ring, tw, TW, ok);
                named_bar_sync(1, TW);
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
                // the candidate of step k+1 opens the next panel: its row is now complete and in
                // logical order, with no delayed multipliers
                if (k + 1 <= n - 2 && cl >= 0) publish(k + 1, cl, k + 1, nullptr);
                for (int e = tw; e < MIX_RPC_MAX * LZ_NB; e += TW) s_lm[e / LZ_NB][e % LZ_NB] = 0.f;
                if (tw == 0) {
                    z.ntouch = 0;
                    z.K0 = k + 1;
                }
                if (t == 32) mark(9);
            }
            if (k + 1 <= n - 2) prefetch_cval(k + 1, last ? k + 1 : K0);
            if (t == 32) mark(10);
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

// dynamic shared memory with a panel-update ring of `ring` slots per thread of warps 1-15
size_t lazy_smem_bytes(int ldr, int ring)
{
    return (size_t)ldr * 3 * sizeof(float) + 4 * sizeof(int) + (size_t)(MT - 32) * ring * sizeof(float2);
}

// the deepest ring (24, 16, 8 or 4 slots) whose shared memory fits beside the kernel's static arrays
static int lazy_ring(int ldr)
{
    cudaFuncAttributes fa;
    size_t stat = 16 * 1024;
    if (cudaFuncGetAttributes(&fa, reduce_mixed_lazy_kernel) == cudaSuccess) stat = fa.sharedSizeBytes;
    for (int r : {LZ_RING_MAX, 16, 8, 4})
        if (lazy_smem_bytes(ldr, r) + stat <= MIX_SMEM_TOTAL) return r;
    return 0;
}

bool lazy_fits(int ldr) { return lazy_ring(ldr) > 0; }

cudaError_t launch_reduce_mixed_lazy(MixArgs a, const MixPlan& pl, cudaStream_t st)
{
    if (!pl.ok) return cudaErrorInvalidValue;
    a.rpc = pl.rpc;
    a.ldr = pl.ldr;
    a.ring = lazy_ring(pl.ldr);
    if (a.ring == 0) return cudaErrorInvalidValue;
    const size_t smem = lazy_smem_bytes(pl.ldr, a.ring);
    static size_t attr[MAX_DEVICES] = {};
    cudaError_t e = opt_in_smem((const void*)reduce_mixed_lazy_kernel, smem, attr);
    if (e != cudaSuccess) return e;
    void* args[] = {&a};
    return cudaLaunchCooperativeKernel((const void*)reduce_mixed_lazy_kernel, dim3(pl.grid), dim3(MT), args, smem,
                                       st);
}

}  // namespace lhl

namespace lhl {

// ---- the deferred right updates of the rows above each panel ----------------------------
// The panel-delayed kernel leaves out of every step the rows whose logical label is at most the
// panel's first step K0 (the reference's rows 1:k0, whose right updates F:1588-1672 delays to the
// panel end as its top GEMM).  Nothing in the elimination reads those rows' later columns: after
// a row rises above a panel only the right updates A[:, c] += A[:, c+1:n] l_(c-1) still change
// it, one column per step, from its stored values.  So the kernel writes them unchanged, and
// row r (0-based) receives, for every column q >= qmin(r) = 1 + 16 ceil(r / 16),
//     H[r, q] = F[r, q] + sum_{p > q} F[r, p] F[p, q - 1]
// with F the written factors: the stored values in the upper part and the multipliers of
// column q - 1 below its subdiagonal (final row order on both sides, as the similarity keeps).
// One product of the upper part with the unit lower factor, here on the FP64 tensor pipe
// (mma.sync m8n8k4: FP64 products and sums), added into Ht at the transposed positions; then
// the same entries are copied back into the factors' upper part.
constexpr int TPM = 64, TPN = 64, TPK = 32, TPT = 128;
struct TopSmem {
    double A[2][TPK][TPM + 4];  // F[r, p]: [k][row]
    double B[2][TPK][TPN + 4];  // F[p, q - 1], zero unless p > q: [k][column]
};

__device__ __forceinline__ int top_qmin(int r) { return 1 + LZ_NB * ((r + LZ_NB - 1) / LZ_NB); }

__global__ void __launch_bounds__(TPT) lz_top_kernel(int n, const double* __restrict__ F, double* __restrict__ Ht)
{
    extern __shared__ __align__(16) unsigned char top_raw[];
    TopSmem& sm = *reinterpret_cast<TopSmem*>(top_raw);
    const int r0 = blockIdx.y * TPM, q0 = blockIdx.x * TPN;
    if (r0 >= n || q0 >= n || q0 + TPN - 1 < top_qmin(r0)) return;  // nothing deferred in this tile
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wm = warp & 1, wn = warp >> 1;  // warp tile: rows 32 wm .., columns 32 wn ..
    const int g = lane >> 2, t4 = lane & 3;
    double acc[4][4][2];
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y][0] = acc[x][y][1] = 0.0;
    const int pbeg = q0 + 1;  // the smallest p any column of the tile takes
    const int nch = (n - pbeg + TPK - 1) / TPK;
    auto stage = [&](int kc, int st) {
        const int pk = pbeg + kc * TPK;
        for (int e = t; e < TPK * TPM; e += TPT) {
            const int m = e % TPM, kk = e / TPM;
            const int r = r0 + m, p = pk + kk;
            const bool ok = r < n && p < n;
            cp_async8(&sm.A[st][kk][m], ok ? &F[(size_t)p * n + r] : F, ok, F);
        }
        for (int e = t; e < TPK * TPN; e += TPT) {
            const int kk = e % TPK, j = e / TPK;
            const int p = pk + kk, q = q0 + j;
            const bool ok = p < n && q < n && q >= 1 && p > q;  // the multipliers of column q - 1 below row q
            cp_async8(&sm.B[st][kk][j], ok ? &F[(size_t)(q - 1) * n + p] : F, ok, F);
        }
        cp_async_commit();
    };
    if (nch > 0) stage(0, 0);
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
        for (int kk = 0; kk < TPK; kk += 4) {
            double fa[4], fb[4];
#pragma unroll
            for (int x = 0; x < 4; ++x) fa[x] = sm.A[st][kk + t4][32 * wm + 8 * x + g];
#pragma unroll
            for (int y = 0; y < 4; ++y) fb[y] = sm.B[st][kk + t4][32 * wn + 8 * y + g];
#pragma unroll
            for (int x = 0; x < 4; ++x)
#pragma unroll
                for (int y = 0; y < 4; ++y) dmma_8x8x4(acc[x][y], fa[x], fb[y]);
        }
        __syncthreads();
    }
    // thread holds D at row 32 wm + 8 x + g, columns 32 wn + 8 y + 2 t4 + {0, 1}
#pragma unroll
    for (int x = 0; x < 4; ++x) {
        const int r = r0 + 32 * wm + 8 * x + g;
        if (r >= n) continue;
        const int qm = top_qmin(r);
#pragma unroll
        for (int y = 0; y < 4; ++y)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int q = q0 + 32 * wn + 8 * y + 2 * t4 + h;
                if (q < n && q >= qm) Ht[(size_t)r * n + q] += acc[x][y][h];
            }
    }
}

// F[r, q] = Ht[q, r] at the deferred positions (q >= qmin(r)), 32 x 32 tiles through shared memory
__global__ void lz_top_copy_kernel(int n, const double* __restrict__ Ht, double* __restrict__ F)
{
    __shared__ double tile[32][33];
    const int rb = blockIdx.y * 32, qb = blockIdx.x * 32;
    if (qb + 31 < top_qmin(rb)) return;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {  // Ht column r = rb + y, rows q = qb + x
        const int r = rb + y, q = qb + threadIdx.x;
        tile[y][threadIdx.x] = (r < n && q < n) ? Ht[(size_t)r * n + q] : 0.0;
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {  // F column q = qb + y, rows r = rb + x
        const int q = qb + y, r = rb + threadIdx.x;
        if (r < n && q < n && q >= top_qmin(r)) F[(size_t)q * n + r] = tile[threadIdx.x][y];
    }
}

// After the panel-delayed kernel: Ht from the factors, the deferred updates added into Ht, and
// copied back into the factors' upper part.
cudaError_t launch_lazy_finish(int n, double* F, double* Ht, cudaStream_t st)
{
    cudaError_t e = launch_ht_fill(n, F, Ht, st);
    if (e != cudaSuccess || n < 3) return e;
    static size_t attr[MAX_DEVICES] = {};
    e = opt_in_smem((const void*)lz_top_kernel, sizeof(TopSmem), attr);
    if (e != cudaSuccess) return e;
    dim3 grid((n + TPN - 1) / TPN, (n + TPM - 1) / TPM);
    lz_top_kernel<<<grid, TPT, sizeof(TopSmem), st>>>(n, F, Ht);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dim3 g2((n + 31) / 32, (n + 31) / 32);
    lz_top_copy_kernel<<<g2, dim3(32, 8), 0, st>>>(n, Ht, F);
    return cudaGetLastError();
}

}  // namespace lhl
