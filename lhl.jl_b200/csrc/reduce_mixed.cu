// reduce_mixed.cu -- the mixed-precision reduction (LHL_PREC_MIXED): ELMHES (F:466-501,
// the unblocked algorithm) with the matrix held in FP32 and every column-update dot product
// accumulated in FP64, for use as the preconditioner of FP64 refinement (lhl_refine!,
// F:3144-3157).  Balancing (F:299-340) runs before it in FP64, in the plain reduction
// kernel's balance-only mode.
//
// Layout: one CTA per SM, each owning a contiguous block of `rpc` physical rows of the
// (balanced) matrix, FP32, in shared memory (rows in global memory when they do not fit).
// Rows never move: a row interchange only swaps logical labels (ph: logical -> physical,
// lg: physical -> logical), which every CTA tracks identically.  Column interchanges are
// applied in place by each owner.
//
// Step k (1-based, k = 1..n-2), per CTA:
//   wait   -- warp 0 polls until every CTA has published step k: a 64-bit header per CTA
//             (step number, best candidate's logical row and signed column value), stored
//             after the CTA's rows' column-k values (cval) and before the candidate's row
//             (crow), which is written while the header travels.
//             Every exchange word carries its step number, so no store waits for an earlier
//             one to be acknowledged (no release fences): a reader re-reads a word whose tag
//             is not yet the step's.  Polls and re-reads are bounded in wall time.
//             Warp 0 then picks the pivot p (largest |value|, ties to the lowest logical row:
//             the reference's first maximum, F:799-806) and swaps labels k+1 <-> p.
//   load   -- swap columns k+1 <-> p in own rows; load the pivot row R from the winner's crow
//             (one L2 round trip) and form every multiplier l_j = c_j / piv from the column
//             values, which warps 1-15 prefetched from cval while warp 0 polled.
//   update -- new column k+1 of own row i (the column update A[:,k+1] += A[:,k+2:n] l after
//             the row update A[i,:] -= l_i R):
//                 c'_i = (A[i,k+1] - l_i R[k+1]) + A[i,k+2:n].l - l_i (R[k+2:n].l)
//             with both dot products in FP64 (FP32 partial sums of at most 16 terms, added in
//             FP64).  Warp 0 publishes the next step's header and returns to polling, while
//             warps 1-15 update the candidate row and publish it in the same pass, then apply
//             the rank-1 row update to the other own rows.
// At the end every CTA writes its rows, in FP64, to their logical positions of `factors`:
// the same layout as the plain form (H in the upper Hessenberg part, multipliers below); CTA 0
// also writes perm and iperm, read off its final labels.
#include "mixed_common.cuh"

namespace lhl {

// r[c] -= li * R[c] for c in [c0, ldr) (0-based), warp-collective; pads stay zero.
__device__ __forceinline__ void mix_axpy(float* __restrict__ r, const float* __restrict__ R, float li, int c0, int ldr,
                                         int lane)
{
    const int c4 = (c0 + 3) & ~3;
    if (c0 + lane < c4 && c0 + lane < ldr) r[c0 + lane] = fmaf(-li, R[c0 + lane], r[c0 + lane]);
    float4* r4 = reinterpret_cast<float4*>(r);
    const float4* R4 = reinterpret_cast<const float4*>(R);
    for (int g = (c4 >> 2) + lane; g < (ldr >> 2); g += 32) {
        float4 a = r4[g];
        const float4 b = R4[g];
        a.x = fmaf(-li, b.x, a.x);
        a.y = fmaf(-li, b.y, a.y);
        a.z = fmaf(-li, b.z, a.z);
        a.w = fmaf(-li, b.w, a.w);
        r4[g] = a;
    }
}

template <bool SROWS>
__global__ void __launch_bounds__(MT, 1) reduce_mixed_kernel(MixArgs a)
{
    extern __shared__ __align__(16) float smx[];
    __shared__ double s_part[(MIX_RPC_MAX + 4) * 4];  // dot products by (row, column part)
    __shared__ float s_li[MIX_RPC_MAX];
    __shared__ int s_win, s_p, s_ok, s_cand;
    __shared__ float s_piv;

    const int n = a.n, rpc = a.rpc, ldr = a.ldr, G = gridDim.x, b = blockIdx.x;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int r0 = b * rpc;
    const int nr = min(rpc, n - r0);
    float* R = smx;                      // pivot row, logical column c at R[c-1]; pads zero
    float* lv = R + ldr;                 // multipliers by logical row; pads zero
    int* lg = (int*)(lv + ldr);          // physical -> logical (1-based)
    int* ph = lg + ldr;                  // logical (1-based) -> physical, ph[0] unused
    float* rows = SROWS ? (float*)(ph + ldr + 4) : a.grows + (size_t)r0 * ldr;  // nr x ldr
    unsigned long long* hdr = a.hdr;

    // ---- load own rows (FP64 -> FP32, zero pads), labels ----
    for (int e = t; e < nr * ldr; e += MT) {
        const int i = e % nr, c = e / nr;
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
    for (int i = t; i < nr; i += MT) s_li[i] = 0.f;
    __syncthreads();

    // Warps 1-15: the column values of step st into lv, by the labels before step st's
    // interchange (the multipliers are formed from them once the pivot is known).  All of a
    // thread's loads are in flight together; a stale word is re-read, bounded in wall time.
    auto prefetch_cval = [&](int st) {
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

    // ---- publish step 1: column 1 values, candidate among logical rows >= 2 ----
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
            const float2* src = reinterpret_cast<const float2*>(rows + (size_t)bl * ldr);
            ulonglong2* dst = reinterpret_cast<ulonglong2*>(a.crow + ((size_t)(1 & 1) * G + b) * ldr);
            for (int g = lane; g < (ldr >> 1); g += 32) {
                const float2 x = src[g];
                __stcg(&dst[g], make_ulonglong2(mix_tag(1u, x.x), mix_tag(1u, x.y)));
            }
        }
        __syncwarp();
        if (lane == 0) st_relaxed_u64(&hdr[(1 & 1) * G + b], mix_pack(1u, bi, bv));
    }

    const uint64_t t_start = globaltimer_ns();
    // CTA 0's time per sub-phase on warp 0, summed over steps (probe slots 0-2: wait and pivot
    // choice, interchange and loads, dot products and new column; slot 4: from there to the next
    // wait; slots 5 and 6 split slots 0 and 2: the poll alone, the dot products alone.  Slot 3
    // is unused: warps 1-15 publish the candidate row)
    unsigned long long* probe = (b == 0 && t == 0 && a.ptimes) ? a.ptimes + 8 : nullptr;
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
        mark(4);
        // ---- wait for step k from every CTA; pick the pivot; relabel ----
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
            // two streams of header loads, the second started about half an L2 round trip after
            // the first, each re-issued as soon as its data is in: a header is seen about half
            // a round trip sooner than by one stream of samples
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
            if (probe) {  // the poll alone (slot 5)
                const uint64_t now = globaltimer_ns();
                probe[5] += now - tp;
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
        mark(0);
        const int p = s_p;
        const int win = s_win;
        const float piv = s_piv;
        // relabel k+1 <-> p only now: until the barrier above, warps 1-15 were prefetching
        // this step's column values by the old labels (nothing below reads the labels before
        // the next barrier)
        if (t == 0 && p != k + 1) {
            const int x = ph[k + 1], w = ph[p];
            ph[k + 1] = w;
            ph[p] = x;
            lg[w] = k + 1;
            lg[x] = p;
        }

        // ---- interchange own columns; pivot row and multipliers (one L2 round trip) ----
        if (p != k + 1)
            for (int i = t; i < nr; i += MT) {
                float* ri = rows + (size_t)i * ldr;
                const float u = ri[k];
                ri[k] = ri[p - 1];
                ri[p - 1] = u;
            }
        {
            // the pivot row from the winner; the multipliers from the prefetched column values,
            // whose slots are by the labels before this interchange: the row now labelled p was
            // labelled k+1 (its value is at lv[k]); every other label in k+2..n is unchanged
            const unsigned long long* src = win >= 0 ? a.crow + ((size_t)par * G + win) * ldr : nullptr;
            const unsigned want = (unsigned)k & 0xffffu;
            bool ok = true;
            for (int base = 0; base < n; base += 4 * MT) {
                unsigned long long rv[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int c = k + 1 + base + t + u * MT;  // logical column of R (1-based)
                    const int sc = c == k + 1 ? p : (c == p ? k + 1 : c);
                    rv[u] = (src && c <= n) ? ld_relaxed_u64(&src[sc - 1]) : mix_tag((unsigned)k, 0.f);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int jj = k + 1 + base + t + u * MT;  // 0-based slot of logical row jj + 1 >= k + 2
                    if (jj < n) {
                        const float cq = lv[jj == p - 1 ? k : jj];
                        lv[jj] = piv != 0.f ? cq / piv : 0.f;
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int c = k + 1 + base + t + u * MT;
                    const int sc = c == k + 1 ? p : (c == p ? k + 1 : c);
                    float r = __uint_as_float((unsigned)(rv[u] >> 32));
                    if (((unsigned)(rv[u] >> 16) & 0xffffu) != want) r = ld_tagged(&src[sc - 1], k, a.limit_ns, ok);
                    if (c <= n) R[c - 1] = r;
                }
            }
            if (!ok) atomicCAS(a.err, 0, (int)LHL_ERR_TIMEOUT);
        }
        __syncthreads();
        mark(1);

        // ---- dot products: own rows and the pivot row against l (FP64 accumulation of FP32
        // partials).  A warp item is 4 rows x one of 4 column parts, so that l is read from
        // shared memory once per 4 rows; the parts are added in a fixed order below ----
        {
            const int nv = nr + 1;  // own rows, then R
            const int c0 = k + 1, c4 = (c0 + 3) & ~3;
            const int g0 = c4 >> 2, g1 = ldr >> 2;
            const int per = (g1 - g0 + 3) >> 2;
            const float4* l4 = reinterpret_cast<const float4*>(lv);
            for (int item = warp; item < ((nv + 3) >> 2) * 4; item += MW) {
                const int rg = item >> 2, cp = item & 3;
                const float* xq[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int v = min(rg * 4 + q, nr);
                    xq[q] = v < nr ? rows + (size_t)v * ldr : R;
                }
                double acc[4] = {0.0, 0.0, 0.0, 0.0};
                if (cp == 0 && c0 + lane < c4 && c0 + lane < ldr) {  // the unaligned head
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc[q] = (double)(xq[q][c0 + lane] * lv[c0 + lane]);
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
                // the four sums over the warp in six shuffles: halves of the lanes keep two of the
                // values, quarters one; lanes 8q .. 8q+7 end with row q's sum
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
        if (probe) {  // the dot products alone (slot 6)
            const uint64_t now = globaltimer_ns();
            probe[6] += now - tp;
        }
        // warp 0: new column k+1 of own rows, multipliers into column k, the next candidate
        if (warp == 0) {
            float bv = 0.f;
            int bi = 0, bl = -1;
            const int np = (k + 1) & 1;
            auto dot = [&](int v) {
                return (s_part[4 * v] + s_part[4 * v + 1]) + (s_part[4 * v + 2] + s_part[4 * v + 3]);
            };
            const double dR = dot(nr);
            for (int i = lane; i < nr; i += 32) {
                float* ri = rows + (size_t)i * ldr;
                const int L = lg[r0 + i];
                double cn;
                float li = 0.f;
                if (L >= k + 2) {
                    li = lv[L - 1];
                    const float a1 = fmaf(-li, R[k], ri[k]);
                    cn = ((double)a1 + dot(i)) - (double)li * dR;
                    ri[k - 1] = li;
                } else {
                    cn = (double)ri[k] + dot(i);
                }
                const float c32 = (float)cn;
                ri[k] = c32;
                s_li[i] = li;
                if (k + 1 <= n - 2) __stcg(&a.cval[(size_t)np * n + r0 + i], mix_tag((unsigned)(k + 1), c32));
                if (L >= k + 2 && mix_better(c32, L, bv, bi)) { bv = c32; bi = L; bl = i; }
            }
            warp_best(bv, bi, bl);
            if (lane == 0) {
                s_cand = bl;
                s_piv = bv;
                s_p = bi;
                // publish step k+1's header now: the candidate row follows below, and a reader
                // re-reads any row word whose tag is not yet k+1
                if (k + 1 <= n - 2) st_relaxed_u64(&hdr[np * G + b], mix_pack((unsigned)(k + 1), bi, bv));
            }
        }
        __syncthreads();
        mark(2);
        const int cl = s_cand;
        if (warp != 0) {
            // ---- publish step k+1: the candidate row after this step's row update, written to
            // the exchange and back into its own row in one pass, by warps 1-15 (warp 0 is
            // already polling for step k+1) ----
            const int np = (k + 1) & 1;
            const bool pub = k + 1 <= n - 2;
            if (cl >= 0) {
                float* rc = rows + (size_t)cl * ldr;
                const float li = s_li[cl];
                ulonglong2* dst = reinterpret_cast<ulonglong2*>(a.crow + ((size_t)np * G + b) * ldr);
                const unsigned st = (unsigned)(k + 1);
                for (int g = ((k + 1) >> 1) + (t - 32); g < (ldr >> 1); g += MT - 32) {
                    const int c = 2 * g;  // 0-based columns c, c+1; only c >= k+1 change
                    float x0 = rc[c], x1 = rc[c + 1];
                    if (c >= k + 1) x0 = fmaf(-li, R[c], x0);
                    x1 = fmaf(-li, R[c + 1], x1);  // c + 1 >= k + 1 always
                    if (pub) __stcg(&dst[g], make_ulonglong2(mix_tag(st, x0), mix_tag(st, x1)));
                    rc[c] = x0;
                    rc[c + 1] = x1;
                }
            }
            // ---- rank-1 row update of the other own active rows ----
            for (int v = warp - 1; v < nr; v += MW - 1) {
                const float li = s_li[v];
                if (v == cl || li == 0.f) continue;
                mix_axpy(rows + (size_t)v * ldr, R, li, k + 1, ldr, lane);
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
    // ---- perm / iperm (F:376-387) from the final labels: the labels went through the same
    // interchanges k+1 <-> p, so logical position L holds original row ph[L] + 1 ----
    if (b == 0)
        for (int q = t; q < n; q += MT) {
            a.perm[q] = ph[q + 1] + 1;
            a.iperm[q] = lg[q];
        }
}

static size_t mixed_fixed_smem(int ldr) { return (size_t)ldr * 4 * sizeof(float) + 16 * sizeof(float); }

void mixed_plan(int n, int sms, MixPlan* pl)
{
    memset(pl, 0, sizeof(*pl));
    if (n < 3 || sms <= 0) return;
    if (sms > 160) sms = 160;
    const int rpc = (n + sms - 1) / sms;
    pl->rpc = rpc;
    pl->grid = (n + rpc - 1) / rpc;
    pl->ldr = (n + 3) & ~3;
    const size_t fixed = mixed_fixed_smem(pl->ldr);
    const size_t srows = (size_t)rpc * pl->ldr * sizeof(float);
    pl->smem_rows = fixed + srows <= MIX_SMEM_MAX;
    pl->smem = pl->smem_rows ? fixed + srows : fixed;
    pl->ok = rpc <= MIX_RPC_MAX && fixed <= MIX_SMEM_MAX && n <= 16384;
}

cudaError_t launch_reduce_mixed(MixArgs a, const MixPlan& pl, cudaStream_t st)
{
    if (!pl.ok) return cudaErrorInvalidValue;
    a.rpc = pl.rpc;
    a.ldr = pl.ldr;
    static size_t attr[2][MAX_DEVICES] = {};
    const void* fn = pl.smem_rows ? (const void*)reduce_mixed_kernel<true> : (const void*)reduce_mixed_kernel<false>;
    cudaError_t e = opt_in_smem(fn, pl.smem, attr[pl.smem_rows ? 1 : 0]);
    if (e != cudaSuccess) return e;
    void* args[] = {&a};
    return cudaLaunchCooperativeKernel(fn, dim3(pl.grid), dim3(MT), args, pl.smem, st);
}

}  // namespace lhl
