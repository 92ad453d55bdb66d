// Search kind of the masked SpGEMM engine (included by spgemm.cu): sorted-list
// intersection of the mask row with the B rows by binary search, one warp per
// row.
//
// The streaming kinds read every element of every B row B_k of a row's A
// entries and test it against the mask row; when the mask row is short and the
// B rows are long almost all of those elements miss (triangle counting on a
// power-law graph: rows with 4 mask entries stream B rows of ~2,000).  Here a
// warp instead takes, for each A entry k, only the mask columns that fall
// inside B_k's column range [B_k first, B_k last] (two loads per k, then a
// search in the mask chunk held in shared memory) and looks each of them up
// in B_k by binary search: the cost per (k, mask column) pair is log2 nnz(B_k)
// dependent loads instead of nnz(B_k) streamed elements.  The reference's
// mask-compressed accumulator walks B_k against M_i (matrix_la.h:505-526); this
// is the same intersection driven from the mask side.
//
//  * The (A entry, mask column) pairs of 32 A entries are packed onto the
//    lanes: each lane computes its entry's pair count, a warp scan gives the
//    offsets, and every lane takes pairs lane, lane+32, ... locating the pair's
//    A entry by a five-step search over the scan held in the lanes' registers
//    (shuffles).  No lane idles on an A entry with few pairs.  A lane runs
//    several pairs' binary searches interleaved (three dependent-load chains
//    in flight for a warp per row, two for the smaller groups: the kernel is
//    bound by the latency of those loads).
//  * Mask rows longer than CAP are taken in chunks of CAP columns; a pair is
//    seen in exactly one chunk, so chunking adds no lookups.
//  * Integer terms are summed exactly as in the other kinds (32-bit wrapping
//    per lane, 64-bit row totals).
//  * G lanes per row: a warp (variant 17), or half- and quarter-warps that
//    take two and four short rows at a time (variants 22 and 23, the small
//    rows of a many-graph batch), every collective confined to the group.
#pragma once

// Pairs whose binary searches a lane runs interleaved, and the resident
// 256-thread CTAs per SM its register cap aims at: a warp per row (variant 17)
// runs three chains at five CTAs (RMAT-24: 54.4 -> 52.5 ms against two at six,
// four at four 55.3 ms); half- and quarter-warp groups keep two chains and get
// four CTAs, whose 64 registers hold their per-group state without spills
// (4,096-graph batch, variant 23: 46.5 -> 42.4 ms against five CTAs).  With
// values written (k-truss support) the warp shape keeps two chains at six
// CTAs: its accumulator updates need the registers (three chains at five CTAs
// spilled and took variant 17's k-truss passes from 6.9 to 8.2 ms).
#ifndef GK_SEARCH_PAIRS
#define GK_SEARCH_PAIRS 3
#endif
#ifndef GK_SEARCH_PAIRS_SUB
#define GK_SEARCH_PAIRS_SUB 2
#endif
#ifndef GK_SEARCH_MINB
#define GK_SEARCH_MINB 5
#endif
#ifndef GK_SEARCH_MINB_SUB
#define GK_SEARCH_MINB_SUB 4
#endif
#ifndef GK_SEARCH_MINB_WRITE
#define GK_SEARCH_MINB_WRITE 6
#endif

// First index q in [0, n) of the sorted shared-memory array k with k[q] >= x
// (strict = false) or k[q] > x (strict = true); n when there is none.
template <bool STRICT>
__device__ __forceinline__ int smem_bound(const int *k, int n, int x) {
    int lo = 0;
    while (n > 0) {
        const int half = n >> 1;
        const int v = k[lo + half];
        if (STRICT ? (v <= x) : (v < x)) {
            lo += half + 1;
            n -= half + 1;
        } else {
            n = half;
        }
    }
    return lo;
}

template <int G>
__device__ __forceinline__ int64_t shfl64(int64_t v, int src, unsigned gmask) {
    const int lo = __shfl_sync(gmask, static_cast<int>(v & 0xFFFFFFFF), src, G);
    const int hi = __shfl_sync(gmask, static_cast<int>(v >> 32), src, G);
    return (static_cast<int64_t>(hi) << 32) | static_cast<uint32_t>(lo);
}

// One (A entry, mask column) lookup of the search kernel: a 32-bit search
// range inside one B row (B rows hold fewer than 2^31 entries).
struct Pair {
    const int32_t *row;  // B.col + b0 of the pair's B row
    int lo, len;         // remaining search range, relative to row
    int c, q;            // the mask column and its position in the chunk
    uint32_t av;         // the A entry's value (1 for patterns)
    bool live;
};

// G lanes per row (G = 32: a warp; 16 and 8: two and four short rows per
// warp), CAP mask columns per chunk in shared memory.  Sub-warp groups hold
// more per-lane state (group masks, shuffle widths).
template <int NT, int G, int CAP, int EPI, bool VAL>
__global__ void __launch_bounds__(NT, G < 32 ? GK_SEARCH_MINB_SUB
                                             : (EPI == EPI_WRITE ? GK_SEARCH_MINB_WRITE : GK_SEARCH_MINB))
    k_search(KArgs p) {
    static_assert(NT == 256, "the register caps assume 256-thread CTAs");
    constexpr bool ACC = (EPI == EPI_WRITE);
    constexpr int NP = (G < 32 || ACC) ? GK_SEARCH_PAIRS_SUB : GK_SEARCH_PAIRS;
    constexpr int NG = NT / G;
    const unsigned gmask = group_mask<G>();
    extern __shared__ int smem[];
    const int grp = threadIdx.x / G, lane = threadIdx.x % G;
    int *mk = smem + grp * CAP;
    int *acc = smem + NG * CAP + grp * CAP;  // EPI_WRITE only
    const int begin = p.voff[p.v], end = p.voff[p.v + 1];
    unsigned long long local = 0;
    int cur_key = -1;
    unsigned long long cur_sum = 0;
    constexpr int FB = 2;  // rows per fetch
    int got = 0, left = 0;

    while (true) {
        if (left == 0) {
            if (lane == 0) got = static_cast<int>(atomicAdd(p.fetch + p.v, static_cast<unsigned>(FB)));
            got = __shfl_sync(gmask, got, 0, G);
            left = FB;
        }
        const int idx = begin + got + (FB - left);
        --left;
        if (idx >= end) break;
        const int row = p.rowlist[idx];
        const int64_t m0 = p.M.rp[row];
        const int mlen = static_cast<int>(p.M.rp[row + 1] - m0);
        const int64_t a0 = p.A.rp[row], a1 = p.A.rp[row + 1];
        unsigned long long rowsum = 0;
        for (int c0 = 0; c0 < mlen; c0 += CAP) {
            const int clen = min(CAP, mlen - c0);
            for (int q = lane; q < clen; q += G) {
                mk[q] = __ldg(p.M.col + m0 + c0 + q);
                if (ACC) acc[q] = 0;
            }
            __syncwarp(gmask);
            const int lo_col = mk[0], hi_col = mk[clen - 1];
            unsigned cnt = 0;
            for (int64_t tb = a0; tb < a1; tb += G) {
                const int64_t t = tb + lane;
                int64_t b0 = 0;
                int blen = 0, qlo = 0, n = 0;
                uint32_t av = 1u;
                if (t < a1) {
                    const int k = __ldg(p.A.col + t);
                    b0 = __ldg(p.B.rp + k);
                    blen = static_cast<int>(__ldg(p.B.rp + k + 1) - b0);
                    if (blen > 0) {
                        const int first = __ldg(p.B.col + b0), last = __ldg(p.B.col + b0 + blen - 1);
                        if (last >= lo_col && first <= hi_col) {
                            qlo = smem_bound<false>(mk, clen, first);
                            n = smem_bound<true>(mk, clen, last) - qlo;
                        }
                    }
                    if (VAL && p.A.val) av = static_cast<uint32_t>(__ldg(p.A.val + t));
                }
                int incl = n;
#pragma unroll
                for (int o = 1; o < G; o <<= 1) {
                    const int y = __shfl_up_sync(gmask, incl, o, G);
                    if (lane >= o) incl += y;
                }
                const int total = __shfl_sync(gmask, incl, G - 1, G);
                const int excl = incl - n;
                // NP pairs per lane per round (pairs pb + lane, pb + G +
                // lane, ...), their binary searches interleaved so that NP
                // dependent-load chains are in flight per lane
                for (int pb = 0; pb < total; pb += NP * G) {
                    Pair P[NP];
#pragma unroll
                    for (int h = 0; h < NP; ++h) {
                        const int pp = pb + G * h + lane;
                        // the pair's A entry: the first lane j whose inclusive
                        // count exceeds pp (binary lifting over the lanes)
                        int j = 0;
#pragma unroll
                        for (int s = G / 2; s > 0; s >>= 1) {
                            const int v = __shfl_sync(gmask, incl, j + s - 1, G);
                            if (v <= pp) j += s;
                        }
                        const int ex_j = __shfl_sync(gmask, excl, j, G);
                        const int qlo_j = __shfl_sync(gmask, qlo, j, G);
                        const int blen_j = __shfl_sync(gmask, blen, j, G);
                        const int64_t b0_j = shfl64<G>(b0, j, gmask);
                        P[h].av = VAL ? static_cast<uint32_t>(__shfl_sync(gmask, static_cast<int>(av), j, G)) : 1u;
                        P[h].live = pp < total;
                        P[h].q = P[h].live ? qlo_j + (pp - ex_j) : 0;
                        P[h].c = P[h].live ? mk[P[h].q] : 0;
                        P[h].row = p.B.col + b0_j;
                        P[h].lo = 0;
                        P[h].len = P[h].live ? blen_j : 1;
                    }
                    // last position with B.col <= c in each pair's B row
                    // (row[0] <= c holds: c lies inside the row's range)
                    while (true) {
                        bool more = false;
#pragma unroll
                        for (int h = 0; h < NP; ++h) more |= P[h].len > 1;
                        if (!more) break;
                        int x[NP];
#pragma unroll
                        for (int h = 0; h < NP; ++h)
                            if (P[h].len > 1) x[h] = __ldg(P[h].row + P[h].lo + (P[h].len >> 1));
#pragma unroll
                        for (int h = 0; h < NP; ++h)
                            if (P[h].len > 1) {
                                const int half = P[h].len >> 1;
                                if (x[h] <= P[h].c) P[h].lo += half;
                                P[h].len -= half;
                            }
                    }
#pragma unroll
                    for (int h = 0; h < NP; ++h) {
                        if (P[h].live && __ldg(P[h].row + P[h].lo) == P[h].c) {
                            const uint32_t w =
                                (VAL && p.B.val)
                                    ? P[h].av * static_cast<uint32_t>(__ldg(p.B.val + (P[h].row - p.B.col) + P[h].lo))
                                    : P[h].av;
                            if (ACC) atomicAdd(reinterpret_cast<unsigned *>(acc + P[h].q), w);
                            else cnt += w;
                        }
                    }
                }
            }
            __syncwarp(gmask);
            if (ACC) {
                for (int q = lane; q < clen; q += G) p.c_val[m0 + c0 + q] = acc[q];
            } else {
                rowsum += cnt;
            }
            __syncwarp(gmask);
        }
        if (EPI == EPI_SUM) local += rowsum;
        if (EPI == EPI_KEYED) {
            const int key = p.row_key ? p.row_key[row] : row;
            if (key != cur_key) {
                const unsigned long long tot = group_sum<G>(cur_sum, gmask);
                if (lane == 0 && tot) atomicAdd(p.sums + cur_key, tot);
                cur_key = key;
                cur_sum = 0;
            }
            cur_sum += rowsum;
        }
    }
    if (EPI == EPI_KEYED && cur_key >= 0) {
        const unsigned long long tot = group_sum<G>(cur_sum, gmask);
        if (lane == 0 && tot) atomicAdd(p.sums + cur_key, tot);
    }
    if (EPI == EPI_SUM) {
        const unsigned long long tot = group_sum<G>(local, gmask);
        if (lane == 0 && tot) atomicAdd(p.sums, tot);
    }
}
