// Masked SpGEMM engine C<M> = A·B on sm_100a.
//
// Reference: mxmm_msa (include/matrix_la.h:562-635) and mxmm_mca (:478-528)
// — a row-wise Gustavson product that, for every row i, streams the rows B_k
// of the entries k of A_i and accumulates a·b at the columns that the mask
// row M_i allows; C has exactly M's pattern.  The reference runs one row per
// OpenMP thread with a dense accumulator of B.n entries per thread.
//
// B200 design (all device-side, no host synchronisation, graph-capturable):
//  1. k_row_stats   eight lanes per row (a warp for long rows): work_i = sum over
//                   k in A_i of nnz(B_k), and the largest nnz(B_k), from B's row
//                   lengths as 32-bit words (k_row_lengths)
//  2. k_bin_rows    bin each row by (log2 nnz(M_i), log2 mean nnz(B_k)); per-bin stats
//  3. sched_choose  one variant per bin (plain heuristic or learned MLP)
//  4. k_count/k_scatter  counting sort of the rows by variant; block kinds also
//                   get their item count (mask chunks x A-entry splits)
//  5. one persistent kernel per variant over its rows / items (the catalogue
//     of 24 variants is the table in gk_sched.cuh):
//       HASH_GROUP  4, 8 or 32 threads per row, the mask row's columns in a
//                   shared-memory bucketed hash set (slot = accumulator)
//       MCA_GROUP   32 threads per row, mask row sorted in shared memory,
//                   binary search (mask-compressed accumulator, matrix_la.h:437-461)
//       HASH_BLOCK  one CTA per item (row x mask chunk x A-entry split), a
//                   512- to 16K-slot table, warps take A entries dynamically;
//                   a bitmap filter in front of the table, or none (every
//                   element looked up), or an exact map of the low columns
//       MCA_BLOCK   one CTA per item, up to 16K sorted mask columns
//       MSA_BLOCK   one CTA per item, dense column-window accumulator
//                   (the reference's MSA, matrix_la.h:611-631) or bitmap
//       SEARCH      a warp (or half-/quarter-warp) per row, each mask column
//                   inside B_k's column range looked up in B_k by binary
//                   search (gk_ksearch.cuh)
// B rows are streamed with 16-byte vector loads; mask chunks that do not cover
// a whole mask row only stream the part of B_k inside the chunk's column range
// (group-cooperative search).  Integer terms are summed in 32-bit wrapping
// arithmetic, so any assignment of rows to variants gives identical values.
#include <cub/cub.cuh>

#include "gk_common.cuh"
#include "gk_device.cuh"
#include "gk_sched.cuh"
#include "gk_spgemm.cuh"

namespace gk {

// ---------------------------------------------------------------------------
// kernel arguments
// ---------------------------------------------------------------------------
struct KArgs {
    DevCsr A, B, M;
    const int32_t *rowlist;  // rows sorted by variant
    const int *voff;         // [NV+1] offsets into rowlist
    const int *vsimple;      // [NV] rows of each variant that are a single item (listed first)
    const int64_t *item_ex;  // exclusive prefix of items per rowlist entry (block kinds)
    const int64_t *work;     // per-row work
    unsigned int *fetch;     // [NV] dynamic item counters (block kinds)
    int32_t *c_val;
    unsigned long long *sums;
    const int32_t *row_key;
    int v;    // variant id
    int vec;  // B.col is 16-byte aligned: vector loads allowed
};

// ---------------------------------------------------------------------------
// plan kernels
// ---------------------------------------------------------------------------
// Per row r of A: work[r] = sum of the B-row lengths of its entries, maxb[r] =
// the longest of them.  Eight lanes per row, four rows per warp step (most rows
// have a few dozen entries, so a warp per row left most lanes idle through its
// dependent loads); a row of up to 32 entries is one dependent load chain of
// its eight lanes.  Rows longer than ROW_STATS_LONG entries are taken by the
// whole warp afterwards, eight independent load pairs in flight per lane, so
// that a hub row (10^5 entries) is one warp's loop.
constexpr int ROW_STATS_LONG = 256;

// B's row lengths as 32-bit words: the row statistics gather one per A entry
// at random, and 4 bytes a row stay in L2 where B's 8-byte row pointers (two
// per lookup, 134 MB at 2^24 rows) do not.
__global__ void k_row_lengths(DevCsr B, int32_t *blen) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < B.m; k += stride)
        blen[k] = static_cast<int32_t>(B.rp[k + 1] - B.rp[k]);
}

// Entries t, t + step, ... < a1 of a row, U of them per lane in flight at a
// time: the U column loads, then the U row lengths they name, so that a row of
// at most step * U entries costs one dependent load chain.
template <int U>
__device__ __forceinline__ void row_stats_entries(const DevCsr &A, const int32_t *__restrict__ blen, int64_t t,
                                                  int64_t a1, int step, long long &w, int &mb) {
    for (; t < a1; t += static_cast<int64_t>(step) * U) {
        int k[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t q = t + static_cast<int64_t>(step) * u;
            k[u] = q < a1 ? __ldg(A.col + q) : -1;
        }
        int len[U];
#pragma unroll
        for (int u = 0; u < U; ++u) len[u] = k[u] >= 0 ? __ldg(blen + k[u]) : 0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            w += len[u];
            mb = max(mb, len[u]);
        }
    }
}

__global__ void k_row_stats(DevCsr A, const int32_t *__restrict__ blen, int64_t *work, int32_t *maxb) {
    constexpr unsigned FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31, sl = lane & 7;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t base = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 4; base < A.m; base += warps * 4) {
        const int64_t r = base + (lane >> 3);
        int64_t a0 = 0, a1 = 0;
        if (r < A.m) {
            a0 = A.rp[r];
            a1 = A.rp[r + 1];
        }
        const bool lng = a1 - a0 > ROW_STATS_LONG;
        long long w = 0;
        int mb = 0;
        if (!lng) row_stats_entries<4>(A, blen, a0 + sl, a1, 8, w, mb);
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
            w += __shfl_xor_sync(FULL, w, o);
            mb = max(mb, __shfl_xor_sync(FULL, mb, o));
        }
        if (sl == 0 && r < A.m && !lng) {
            work[r] = w;
            maxb[r] = mb;
        }
        // the step's long rows, one at a time with all 32 lanes
        for (unsigned lm = __ballot_sync(FULL, lng && sl == 0); lm; lm &= lm - 1) {
            const int g = (__ffs(lm) - 1) >> 3;
            const int64_t rr = base + g;
            const int64_t b0 = __shfl_sync(FULL, a0, 8 * g), b1 = __shfl_sync(FULL, a1, 8 * g);
            long long lw = 0;
            int lmb = 0;
            row_stats_entries<8>(A, blen, b0 + lane, b1, 32, lw, lmb);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                lw += __shfl_xor_sync(FULL, lw, o);
                lmb = max(lmb, __shfl_xor_sync(FULL, lmb, o));
            }
            if (lane == 0) {
                work[rr] = lw;
                maxb[rr] = lmb;
            }
        }
    }
}

__global__ void k_bin_rows(DevCsr A, DevCsr M, const int64_t *work, const int32_t *maxb, uint16_t *bin,
                           BinStats *bins) {
    __shared__ unsigned long long s_rows[NBINS], s_m[NBINS], s_a[NBINS], s_w[NBINS];
    __shared__ unsigned int s_b[NBINS];
    for (int b = threadIdx.x; b < NBINS; b += blockDim.x) {
        s_rows[b] = s_m[b] = s_a[b] = s_w[b] = 0;
        s_b[b] = 0;
    }
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < A.m; r += stride) {
        const int64_t mlen = M.rp[r + 1] - M.rp[r];
        const int64_t alen = A.rp[r + 1] - A.rp[r];
        const int64_t w = work[r];
        if (mlen == 0 || w == 0) {
            bin[r] = BIN_SKIP;
            continue;
        }
        const int qm = min(NB_M - 1, ilog2_u64(static_cast<unsigned long long>(mlen)));
        const int qb = min(NB_B - 1, ilog2_u64(static_cast<unsigned long long>(w / alen)));
        const int b = qm * NB_B + qb;
        bin[r] = static_cast<uint16_t>(b);
        atomicAdd(&s_rows[b], 1ull);
        atomicAdd(&s_m[b], static_cast<unsigned long long>(mlen));
        atomicAdd(&s_a[b], static_cast<unsigned long long>(alen));
        atomicAdd(&s_w[b], static_cast<unsigned long long>(w));
        atomicMax(&s_b[b], static_cast<unsigned int>(maxb[r]));
    }
    __syncthreads();
    for (int b = threadIdx.x; b < NBINS; b += blockDim.x) {
        if (s_rows[b] == 0) continue;
        atomicAdd(&bins[b].rows, s_rows[b]);
        atomicAdd(&bins[b].sum_m, s_m[b]);
        atomicAdd(&bins[b].sum_a, s_a[b]);
        atomicAdd(&bins[b].sum_work, s_w[b]);
        atomicMax(&bins[b].max_b, s_b[b]);
    }
}

__device__ __forceinline__ int64_t items_of_row(int v, bool write, int64_t mlen, int64_t alen, int64_t w,
                                                const int32_t *mcol_row) {
    const Variant V = c_variants[v];
    if (V.kind == K_HASH_GROUP || V.kind == K_MCA_GROUP || V.kind == K_SEARCH) return 1;
    int64_t nch;
    if (V.kind == K_MSA_BLOCK) {
        const int lw = write ? V.cap_write : V.cap;
        nch = (int64_t)(mcol_row[mlen - 1] >> lw) - (int64_t)(mcol_row[0] >> lw) + 1;
    } else {
        const int ch = write ? V.chunk_write : V.chunk;
        nch = (mlen + ch - 1) / ch;
    }
    return nch * num_splits(w, alen, V.split_log2);
}

// Variant and item count of row r (-1 when the row has no work).
__device__ __forceinline__ int row_variant(int64_t r, const uint16_t *bin, const int *var_of_bin, int force_variant) {
    const uint16_t b = bin[r];
    if (b == BIN_SKIP) return -1;
    return force_variant >= 0 ? force_variant : var_of_bin[b];
}

__device__ __forceinline__ int64_t row_items(const DevCsr &A, const DevCsr &M, const int64_t *work, int64_t r, int v,
                                             bool write) {
    const int64_t m0 = M.rp[r], mlen = M.rp[r + 1] - m0;
    return items_of_row(v, write, mlen, A.rp[r + 1] - A.rp[r], work[r], M.col + m0);
}

// Counting sort of the rows by variant.  Within a variant's segment the rows
// that are a single item come first, so the kernels map those items to rows
// without a search; rows split into several items follow.
__global__ void k_count_rows(DevCsr A, DevCsr M, const int64_t *work, const uint16_t *bin, const int *var_of_bin,
                             int force_variant, bool write, int *vcount, int *vsimple) {
    __shared__ int s_cnt[NV], s_simple[NV];
    if (threadIdx.x < NV) s_cnt[threadIdx.x] = s_simple[threadIdx.x] = 0;
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < A.m; r += stride) {
        const int v = row_variant(r, bin, var_of_bin, force_variant);
        if (v < 0) continue;
        atomicAdd(&s_cnt[v], 1);
        if (row_items(A, M, work, r, v, write) == 1) atomicAdd(&s_simple[v], 1);
    }
    __syncthreads();
    if (threadIdx.x < NV && s_cnt[threadIdx.x]) {
        atomicAdd(&vcount[threadIdx.x], s_cnt[threadIdx.x]);
        atomicAdd(&vsimple[threadIdx.x], s_simple[threadIdx.x]);
    }
}

// vcursor[2v]: next single-item slot of variant v, vcursor[2v+1]: next multi-item slot.
__global__ void k_offsets(const int *vcount, const int *vsimple, int *voff, int *vcursor, unsigned int *fetch) {
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int v = 0; v < NV; ++v) {
            voff[v] = acc;
            vcursor[2 * v] = acc;
            vcursor[2 * v + 1] = acc + vsimple[v];
            fetch[v] = 0;
            acc += vcount[v];
        }
        voff[NV] = acc;
    }
}

__global__ void k_scatter_rows(DevCsr A, DevCsr M, const int64_t *work, const uint16_t *bin,
                               const int *var_of_bin, int force_variant, bool write, int *vcursor,
                               int32_t *rowlist, int64_t *item_n) {
    __shared__ int s_cnt[2 * NV], s_base[2 * NV];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < A.m; base += stride) {
        if (threadIdx.x < 2 * NV) s_cnt[threadIdx.x] = 0;
        __syncthreads();
        const int64_t r = base + threadIdx.x;
        int slot = -1, local = 0;
        int64_t items = 0;
        if (r < A.m) {
            const int v = row_variant(r, bin, var_of_bin, force_variant);
            if (v >= 0) {
                items = row_items(A, M, work, r, v, write);
                slot = 2 * v + (items == 1 ? 0 : 1);
                local = atomicAdd(&s_cnt[slot], 1);
            }
        }
        __syncthreads();
        if (threadIdx.x < 2 * NV && s_cnt[threadIdx.x])
            s_base[threadIdx.x] = atomicAdd(&vcursor[threadIdx.x], s_cnt[threadIdx.x]);
        __syncthreads();
        if (slot >= 0) {
            const int pos = s_base[slot] + local;
            rowlist[pos] = static_cast<int32_t>(r);
            item_n[pos] = items;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// group kinds: one row per group of G threads
// ---------------------------------------------------------------------------
// Probe kinds: the mask structure a B-row element is looked up in.
enum : int { PK_HASH = 0, PK_MCA = 1, PK_MSA = 2 };

// One B-row element against the mask structure of the current row/chunk:
// HASH  slot of x in a CAP-slot hash set;  MCA  position of x in the sorted
// chunk keys[0, clen);  MSA  x - base if its bit is set in a 2^CAP-column
// window bitmap (keys reinterpreted as words).
template <int CAP, int PK, bool ACC, int FLOG = 0, int LOWB = 0>
__device__ __forceinline__ void probe_elem(int x, uint32_t w, const int *keys, int *acc, int clen, unsigned &cnt,
                                           const unsigned *filt = nullptr) {
    int s;
    if constexpr (PK == PK_HASH && FLOG > 0) {
        // bitmap filter first: most B elements are not mask columns
        const uint32_t h = filter_pos<FLOG, LOWB>(x);
        if (!((filt[h >> 5] >> (h & 31)) & 1u)) return;
        if constexpr (!ACC && LOWB > 0) {
            if (static_cast<uint32_t>(x) < (1u << LOWB)) {  // exact part of the filter: a hit
                cnt += w;
                return;
            }
        }
    }
    if constexpr (PK == PK_MSA) {
        const int y = x - clen;  // clen carries the window base for MSA
        s = (y >= 0 && y < (1 << CAP) && ((reinterpret_cast<const unsigned *>(keys)[y >> 5] >> (y & 31)) & 1u)) ? y : -1;
    } else if constexpr (PK == PK_MCA) {
        s = sorted_find(keys, clen, x);
    } else if constexpr (ACC) {
        s = hash_find<CAP>(keys, x);
    } else {
        s = hash_has<CAP>(keys, x) ? 0 : -1;  // no slot needed without accumulators
    }
    if (s >= 0) {
        if (ACC) atomicAdd(reinterpret_cast<unsigned *>(acc + s), w);
        else cnt += w;
    }
}

// Filter bit of x placed at bit E of the result (0 elsewhere): the word's
// bit h moves to position E by one rotate (funnel shift, amount taken mod 32),
// and the caller's OR with the other elements' bits folds into the AND.
template <int FLOG, int LOWB, int E>
__device__ __forceinline__ uint32_t cand_at(int x, const unsigned *filt) {
    const uint32_t h = filter_pos<FLOG, LOWB>(x);
    const uint32_t w = filt[h >> 5];
    return __funnelshift_r(w, w, h - E) & (1u << E);
}

template <int CAP, bool ACC>
__device__ __forceinline__ void exact_hash(int x, uint32_t w, const int *keys, int *acc, unsigned &cnt) {
    if constexpr (ACC) {
        const int s = hash_find<CAP>(keys, x);
        if (s >= 0) atomicAdd(reinterpret_cast<unsigned *>(acc + s), w);
    } else {
        if (hash_has<CAP>(keys, x)) cnt += w;
    }
}

// Element e (0..7) of the eight held in x (0..3) and y (4..7).
__device__ __forceinline__ int elem8(const int4 &x, const int4 &y, int e) {
    const int lo = (e & 1) ? ((e & 4) ? y.y : x.y) : ((e & 4) ? y.x : x.x);
    const int hi = (e & 1) ? ((e & 4) ? y.w : x.w) : ((e & 4) ? y.z : x.z);
    return (e & 2) ? hi : lo;
}

// Exact lookups of the filter candidates among the eight elements of x, y
// (bit e of m set = element e passed the filter).  Each lane walks only its
// own set bits, so a warp iterates as often as its busiest lane has
// candidates instead of once per element position with a lane or two active.
template <int CAP, bool ACC, int LOWB = 0>
__device__ __forceinline__ void exact_cands(uint32_t m, const int4 &x, const int4 &y, uint32_t av,
                                            const int *keys, int *acc, unsigned &cnt) {
    if constexpr (!ACC && LOWB > 0) {
        // candidates below 2^LOWB passed an exact bit: counted at once,
        // without a trip through the per-candidate loop
        constexpr uint32_t L = 1u << LOWB;
        const uint32_t low = uint32_t(uint32_t(x.x) < L) | (uint32_t(uint32_t(x.y) < L) << 1) |
                             (uint32_t(uint32_t(x.z) < L) << 2) | (uint32_t(uint32_t(x.w) < L) << 3) |
                             (uint32_t(uint32_t(y.x) < L) << 4) | (uint32_t(uint32_t(y.y) < L) << 5) |
                             (uint32_t(uint32_t(y.z) < L) << 6) | (uint32_t(uint32_t(y.w) < L) << 7);
        cnt += av * static_cast<uint32_t>(__popc(m & low));
        m &= ~low;
    }
    while (m) {
        const int e = __ffs(m) - 1;
        m &= m - 1;
        exact_hash<CAP, ACC>(elem8(x, y, e), av, keys, acc, cnt);
    }
}

// Vector part of a B row for the high-hit-rate kinds (hub rows, whose mask
// covers a large share of the B rows they stream): instead of every lane
// walking its own filter candidates through the table (a loop as long as the
// busiest lane's candidates), the candidates of the whole sub-group are
// packed into a shared-memory queue (a scan of the per-lane counts) and
// checked one per lane.  The loop runs a uniform number of rounds over the
// row's 16-byte vectors so that the sub-group's collectives stay converged;
// lanes past the item's last mask column contribute nothing.
template <int SUB, int CAP, bool ACC, int FLOG, int LOWB>
__device__ __forceinline__ void stream_vectors_compact(const int4 *__restrict__ base, int n4, int sl, unsigned smask,
                                                       uint32_t av, const int *keys, int *acc, unsigned &cnt,
                                                       const unsigned *filt, int hi_col, int *queue) {
    const int rounds = (n4 + 2 * SUB - 1) / (2 * SUB);
    bool past = false;
    for (int it = 0; it < rounds; ++it) {
        const int q = it * 2 * SUB + sl;
        int4 x = make_int4(0, 0, 0, 0), y = make_int4(0, 0, 0, 0);
        uint32_t m = 0;
        if (!past && q < n4) {
            x = __ldg(base + q);
            m = cand_at<FLOG, LOWB, 0>(x.x, filt) | cand_at<FLOG, LOWB, 1>(x.y, filt) |
                cand_at<FLOG, LOWB, 2>(x.z, filt) | cand_at<FLOG, LOWB, 3>(x.w, filt);
            if (q + SUB < n4) {
                y = __ldg(base + q + SUB);
                m |= cand_at<FLOG, LOWB, 4>(y.x, filt) | cand_at<FLOG, LOWB, 5>(y.y, filt) |
                     cand_at<FLOG, LOWB, 6>(y.z, filt) | cand_at<FLOG, LOWB, 7>(y.w, filt);
                past = y.w > hi_col;
            } else {
                past = x.w > hi_col;
            }
        }
        if constexpr (!ACC && LOWB > 0) {  // exact part of the filter: hits counted at once
            constexpr uint32_t L = 1u << LOWB;
            const uint32_t low = uint32_t(uint32_t(x.x) < L) | (uint32_t(uint32_t(x.y) < L) << 1) |
                                 (uint32_t(uint32_t(x.z) < L) << 2) | (uint32_t(uint32_t(x.w) < L) << 3) |
                                 (uint32_t(uint32_t(y.x) < L) << 4) | (uint32_t(uint32_t(y.y) < L) << 5) |
                                 (uint32_t(uint32_t(y.z) < L) << 6) | (uint32_t(uint32_t(y.w) < L) << 7);
            cnt += av * static_cast<uint32_t>(__popc(m & low));
            m &= ~low;
        }
        const int nc = __popc(m);
        int incl = nc;
#pragma unroll
        for (int o = 1; o < SUB; o <<= 1) {
            const int t = __shfl_up_sync(smask, incl, o, SUB);
            if (sl >= o) incl += t;
        }
        const int total = __shfl_sync(smask, incl, SUB - 1, SUB);
        int w = incl - nc;
        while (m) {
            const int e = __ffs(m) - 1;
            m &= m - 1;
            queue[w++] = elem8(x, y, e);
        }
        __syncwarp(smask);
        for (int c = sl; c < total; c += SUB) exact_hash<CAP, ACC>(queue[c], av, keys, acc, cnt);
        __syncwarp(smask);
        if (__all_sync(smask, past || q >= n4)) break;
    }
}

// The SUB lanes of a sub-group stream B[b0, b1): 16-byte vector loads, two in
// flight per lane, scalar head/tail; with values, scalar loads of col and val.
// With a filter, the eight elements of two vectors are tested against the
// filter without branches and only the candidates take the exact lookup.  A
// lane stops once its elements pass hi_col, the last mask column of the
// item (B rows are sorted); elements beyond it could never match.
template <int SUB, int CAP, int PK, bool ACC, bool VAL, int FLOG = 0, int LOWB = 0, int COMP = 0>
__device__ __forceinline__ void stream_row(const KArgs &p, int64_t b0, int64_t b1, int sl, uint32_t av,
                                           const int *keys, int *acc, int clen, unsigned &cnt,
                                           const unsigned *filt, int hi_col, int *queue = nullptr) {
    const int32_t *__restrict__ bc = p.B.col;
    if constexpr (PK == PK_HASH && FLOG > 0 && !VAL) {
        if (p.vec) {
            int64_t h1 = (b0 + 3) & ~int64_t(3);
            if (h1 > b1) h1 = b1;
            if (b0 + sl < h1) probe_elem<CAP, PK, ACC, FLOG, LOWB>(__ldg(bc + b0 + sl), av, keys, acc, clen, cnt, filt);
            const int4 *__restrict__ base = reinterpret_cast<const int4 *>(bc) + (h1 >> 2);
            const int n4 = static_cast<int>((b1 >> 2) - (h1 >> 2));
            if constexpr (COMP) {
                stream_vectors_compact<SUB, CAP, ACC, FLOG, LOWB>(base, n4, sl, group_mask<SUB>(), av, keys, acc,
                                                                   cnt, filt, hi_col, queue);
                int64_t tl = (b1 >> 2) << 2;
                if (tl < h1) tl = h1;
                if (tl + sl < b1)
                    probe_elem<CAP, PK, ACC, FLOG, LOWB>(__ldg(bc + tl + sl), av, keys, acc, clen, cnt, filt);
                return;
            }
            int q = sl;
            bool past = false;  // this lane's elements went beyond the mask's last column
            for (; q + SUB < n4; q += 2 * SUB) {
                const int4 x = __ldg(base + q);
                const int4 y = __ldg(base + q + SUB);
                const uint32_t m = cand_at<FLOG, LOWB, 0>(x.x, filt) | cand_at<FLOG, LOWB, 1>(x.y, filt) |
                                   cand_at<FLOG, LOWB, 2>(x.z, filt) | cand_at<FLOG, LOWB, 3>(x.w, filt) |
                                   cand_at<FLOG, LOWB, 4>(y.x, filt) | cand_at<FLOG, LOWB, 5>(y.y, filt) |
                                   cand_at<FLOG, LOWB, 6>(y.z, filt) | cand_at<FLOG, LOWB, 7>(y.w, filt);
                exact_cands<CAP, ACC, LOWB>(m, x, y, av, keys, acc, cnt);
                if (y.w > hi_col) {  // B rows are sorted: the rest cannot be mask columns
                    past = true;
                    break;
                }
            }
            if (!past && q < n4) {
                const int4 x = __ldg(base + q);
                const uint32_t m = cand_at<FLOG, LOWB, 0>(x.x, filt) | cand_at<FLOG, LOWB, 1>(x.y, filt) |
                                   cand_at<FLOG, LOWB, 2>(x.z, filt) | cand_at<FLOG, LOWB, 3>(x.w, filt);
                exact_cands<CAP, ACC, LOWB>(m, x, x, av, keys, acc, cnt);
            }
            int64_t tl = (b1 >> 2) << 2;
            if (tl < h1) tl = h1;
            if (tl + sl < b1) probe_elem<CAP, PK, ACC, FLOG, LOWB>(__ldg(bc + tl + sl), av, keys, acc, clen, cnt, filt);
            return;
        }
    }
    if (!VAL && p.vec) {
        int64_t h1 = (b0 + 3) & ~int64_t(3);
        if (h1 > b1) h1 = b1;
        if (b0 + sl < h1) probe_elem<CAP, PK, ACC, FLOG, LOWB>(__ldg(bc + b0 + sl), av, keys, acc, clen, cnt, filt);
        const int64_t v1 = b1 >> 2;
        const int4 *__restrict__ bv = reinterpret_cast<const int4 *>(bc);
        int64_t q = (h1 >> 2) + sl;
        bool past = false;
        for (; q + SUB < v1; q += 2 * SUB) {
            const int4 x = __ldg(bv + q);
            const int4 y = __ldg(bv + q + SUB);
            probe_elem<CAP, PK, ACC, FLOG, LOWB>(x.x, av, keys, acc, clen, cnt, filt);
            probe_elem<CAP, PK, ACC, FLOG, LOWB>(x.y, av, keys, acc, clen, cnt, filt);
            probe_elem<CAP, PK, ACC, FLOG, LOWB>(x.z, av, keys, acc, clen, cnt, filt);
            probe_elem<CAP, PK, ACC, FLOG, LOWB>(x.w, av, keys, acc, clen, cnt, filt);
            probe_elem<CAP, PK, ACC, FLOG, LOWB>(y.x, av, keys, acc, clen, cnt, filt);
            probe_elem<CAP, PK, ACC, FLOG, LOWB>(y.y, av, keys, acc, clen, cnt, filt);
            probe_elem<CAP, PK, ACC, FLOG, LOWB>(y.z, av, keys, acc, clen, cnt, filt);
            probe_elem<CAP, PK, ACC, FLOG, LOWB>(y.w, av, keys, acc, clen, cnt, filt);
            if (y.w > hi_col) {
                past = true;
                break;
            }
        }
        if (!past && q < v1) {
            const int4 x = __ldg(bv + q);
            probe_elem<CAP, PK, ACC, FLOG, LOWB>(x.x, av, keys, acc, clen, cnt, filt);
            probe_elem<CAP, PK, ACC, FLOG, LOWB>(x.y, av, keys, acc, clen, cnt, filt);
            probe_elem<CAP, PK, ACC, FLOG, LOWB>(x.z, av, keys, acc, clen, cnt, filt);
            probe_elem<CAP, PK, ACC, FLOG, LOWB>(x.w, av, keys, acc, clen, cnt, filt);
        }
        int64_t tl = v1 << 2;
        if (tl < h1) tl = h1;
        if (tl + sl < b1) probe_elem<CAP, PK, ACC, FLOG, LOWB>(__ldg(bc + tl + sl), av, keys, acc, clen, cnt, filt);
    } else {
        const int32_t *__restrict__ bvals = VAL ? p.B.val : nullptr;
        for (int64_t j = b0 + sl; j < b1; j += SUB) {
            const int x = __ldg(bc + j);
            if (x > hi_col) break;
            const uint32_t w = (VAL && bvals) ? av * static_cast<uint32_t>(__ldg(bvals + j)) : av;
            probe_elem<CAP, PK, ACC, FLOG, LOWB>(x, w, keys, acc, clen, cnt, filt);
        }
    }
}

// Row bounds of B_k for A entry t (b0 == b1 when outside [lo_col, hi_col]).
struct BRow {
    int64_t b0, b1;
    uint32_t av;
};

template <bool VAL>
__device__ __forceinline__ BRow brow_of(const KArgs &p, int k, int64_t t) {
    BRow r;
    r.b0 = __ldg(p.B.rp + k);
    r.b1 = __ldg(p.B.rp + k + 1);
    r.av = (VAL && p.A.val) ? static_cast<uint32_t>(__ldg(p.A.val + t)) : 1u;
    return r;
}

// Streams the B rows of A entries t = first, first+step, ... < a1 with one
// sub-group of SUB lanes: the next entry's row bounds and the entry after
// that's column are loaded while the current row streams.
template <int SUB, int CAP, int PK, bool ACC, bool VAL, int FLOG>
__device__ __forceinline__ void stream_entries(const KArgs &p, int64_t first, int64_t a1, int step, int sl,
                                               bool chunked, int lo_col, int hi_col, const int *keys, int *acc,
                                               int clen, unsigned &cnt, const unsigned *filt) {
    const unsigned smask = group_mask<SUB>();
    int64_t t = first;
    if (t >= a1) return;
    BRow nxt = brow_of<VAL>(p, __ldg(p.A.col + t), t);
    int k2 = (t + step < a1) ? __ldg(p.A.col + t + step) : 0;
    while (t < a1) {
        BRow cur = nxt;
        const int64_t tn = t + step;
        if (tn < a1) nxt = brow_of<VAL>(p, k2, tn);
        if (tn + step < a1) k2 = __ldg(p.A.col + tn + step);
        if (cur.b0 < cur.b1) {
            bool skip = false;
            if (chunked && cur.b1 - cur.b0 > CUT_MIN) {
                skip = __ldg(p.B.col + cur.b1 - 1) < lo_col || __ldg(p.B.col + cur.b0) > hi_col;
                if (!skip) {
                    const int64_t lo = group_lower_bound<SUB>(p.B.col, cur.b0, cur.b1, lo_col, sl, smask);
                    cur.b1 = group_lower_bound<SUB>(p.B.col, lo, cur.b1, hi_col + 1, sl, smask);
                    cur.b0 = lo;
                }
            }
            if (!skip)
                stream_row<SUB, CAP, PK, ACC, VAL, FLOG>(p, cur.b0, cur.b1, sl, cur.av, keys, acc, clen, cnt, filt,
                                                         hi_col);
        }
        t = tn;
    }
}

// Rows a group takes per fetch: four for the narrow groups, whose rows are
// short, so that the shared counter is not hit once per row.
template <int G>
__host__ __device__ constexpr int c_group_fetch() { return G >= 32 ? 2 : 4; }

// G threads per row; the row's A entries are dealt round-robin to G/SUB
// sub-groups of SUB lanes that stream their B rows concurrently.  Each group
// takes its next row from a global counter, so groups never wait on each
// other for work.
template <int G, int SUB, int NT, int CAP, int CHUNK, bool MCA, int FLOG, int EPI, bool VAL>
__global__ void __launch_bounds__(NT, GK_LB_THREADS / NT) k_group(KArgs p) {
    constexpr int NG = NT / G;
    constexpr int S = G / SUB;
    constexpr bool ACC = (EPI == EPI_WRITE);
    constexpr int FW = (!MCA && FLOG > 0) ? (1 << FLOG) / 32 : 0;  // filter words per group
    extern __shared__ int smem[];
    const int g = threadIdx.x / G;
    const int lane = threadIdx.x % G;
    const int sg = lane / SUB, sl = lane % SUB;
    // MCA: each group's sorted keys get 4 spare slots (cp.async staging puts
    // them at an offset of 0..3 elements, congruent to the source mod 16 bytes)
    constexpr int KST = MCA ? CAP + 4 : CAP;
    int *const keys0 = smem + g * KST;
    int *keys = keys0;
    int *acc = smem + NG * KST + g * CAP;
    unsigned *filt = reinterpret_cast<unsigned *>(smem + NG * KST + NG * CAP * (ACC ? 1 : 0)) + g * FW;
    const unsigned gmask = group_mask<G>();
    const int begin = p.voff[p.v], end = p.voff[p.v + 1];
    unsigned long long local = 0;
    // keyed sums: consecutive rows of a group mostly share a key (rows of one
    // graph of a batch), so a group adds up per key and flushes on change
    int cur_key = -1;
    unsigned long long cur_sum = 0;
    // the table and filter start empty; every row clears what it set
    if constexpr (!MCA) {
        for (int s = lane; s < CAP; s += G) {
            keys[s] = EMPTY_KEY;
            if (ACC) acc[s] = 0;
        }
        for (int wd = lane; wd < FW; wd += G) filt[wd] = 0u;
    }
    __syncwarp(gmask);
    constexpr int FB = c_group_fetch<G>();
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
        const int32_t *__restrict__ mc = p.M.col + m0;
        const bool chunked = mlen > CHUNK;
        unsigned long long rowsum = 0;
        for (int c0 = 0; c0 < mlen; c0 += CHUNK) {
            const int c1 = min(mlen, c0 + CHUNK);
            const int clen = c1 - c0;
            if (MCA) {
                keys = keys0 + stage_phase(mc + c0);
                stage_ints_async(keys, mc + c0, clen, lane, G);
                if (ACC)
                    for (int q = lane; q < clen; q += G) acc[q] = 0;
                cp_async_wait_all();
            } else {
                for (int q = c0 + lane; q < c1; q += G) {
                    const int x = mc[q];
                    hash_insert<CAP>(keys, x);
                    if constexpr (FW > 0) {
                        const uint32_t h = filter_bit<FLOG>(x);
                        atomicOr(filt + (h >> 5), 1u << (h & 31));
                    }
                }
            }
            __syncwarp(gmask);
            const int lo_col = mc[c0], hi_col = mc[c1 - 1];
            unsigned cnt = 0;
            stream_entries<SUB, CAP, MCA ? PK_MCA : PK_HASH, ACC, VAL, (FW > 0 ? FLOG : 0)>(
                p, a0 + sg, a1, S, sl, chunked, lo_col, hi_col, keys, acc, clen, cnt, filt);
            __syncwarp(gmask);
            if constexpr (MCA) {
                if (ACC)
                    for (int q = c0 + lane; q < c1; q += G) p.c_val[m0 + q] = acc[q - c0];
            } else {
                // find this chunk's slots (writing the values out), then clear
                // them and the filter words only after every lane has found
                // its keys, so that no probe meets a half-cleared bucket
                constexpr int PER = (CHUNK + G - 1) / G;
                int slot[PER];
#pragma unroll
                for (int k = 0; k < PER; ++k) {
                    const int q = c0 + lane + k * G;
                    slot[k] = q < c1 ? hash_find<CAP>(keys, mc[q]) : -1;
                    if (ACC && slot[k] >= 0) p.c_val[m0 + q] = acc[slot[k]];
                }
                __syncwarp(gmask);
#pragma unroll
                for (int k = 0; k < PER; ++k) {
                    const int q = c0 + lane + k * G;
                    if (slot[k] >= 0) {
                        keys[slot[k]] = EMPTY_KEY;
                        if (ACC) acc[slot[k]] = 0;
                    }
                    if constexpr (FW > 0) {
                        if (q < c1) filt[filter_bit<FLOG>(mc[q]) >> 5] = 0u;
                    }
                }
            }
            if (!ACC) rowsum += cnt;
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
        // groups leave at different times: reduce per group, no CTA barrier
        const unsigned long long tot = group_sum<G>(local, gmask);
        if (lane == 0 && tot) atomicAdd(p.sums, tot);
    }
}

#include "gk_kblock.cuh"
#include "gk_ksearch.cuh"

// ---------------------------------------------------------------------------
// host side: launching one variant
// ---------------------------------------------------------------------------
template <int V>
constexpr size_t smem_bytes(bool write) {
    constexpr Variant X = VARIANTS[V];
    if constexpr (X.kind == K_HASH_GROUP || X.kind == K_MCA_GROUP) {
        const int nt = group_cta_threads(V);
        const int ng = nt / X.G;
        const int cap = (X.kind == K_MCA_GROUP) ? X.chunk : X.cap;
        const size_t filter = (X.kind == K_HASH_GROUP && X.flog > 0) ? (size_t(1) << X.flog) / 8 : 0;
        const size_t stage_pad = (X.kind == K_MCA_GROUP) ? 16 : 0;  // cp.async alignment slots
        return size_t(ng) * (size_t(cap) * 4 * (write ? 2 : 1) + filter + stage_pad);
    } else if constexpr (X.kind == K_SEARCH) {
        return size_t(NT_GROUP / X.G) * size_t(write ? X.cap_write : X.cap) * 4 * (write ? 2 : 1);
    } else if constexpr (X.kind == K_MSA_BLOCK) {
        if (write) return (size_t(1) << X.cap_write) / 8 + (size_t(1) << X.cap_write) * 4;
        return (size_t(1) << X.cap) / 8;
    } else {
        const int cap = write ? X.cap_write : X.cap;
        const size_t filter =
            (X.kind == K_HASH_BLOCK && X.flog > 0) ? ((size_t(1) << X.lowb) + (size_t(1) << X.flog)) / 8 : 0;
        const size_t stage_pad = (X.kind == K_MCA_BLOCK) ? 16 : 0;  // cp.async alignment slots
        const size_t queue = (X.kind == K_HASH_BLOCK && X.comp) ? size_t(X.G) * 8 * 4 : 0;  // candidate queues
        return size_t(cap) * 4 * (write ? 2 : 1) + filter + stage_pad + queue;
    }
}

// launch == false: only size the grid (attributes and occupancy), so that a
// later launch inside a stream capture makes no configuration calls.
template <int V, int EPI, bool VAL>
static cudaError_t launch_variant_t(const KArgs &args, int num_sms, cudaStream_t s, bool launch = true) {
    constexpr Variant X = VARIANTS[V];
    constexpr bool W = (EPI == EPI_WRITE);
    constexpr size_t SMEM = smem_bytes<V>(W);
    void (*fn)(KArgs);
    int nt;
    if constexpr (X.kind == K_HASH_GROUP || X.kind == K_MCA_GROUP) {
        constexpr int NTV = group_cta_threads(V);
        constexpr bool MCA = X.kind == K_MCA_GROUP;
        constexpr int CAPV = MCA ? X.chunk : X.cap;
        fn = k_group<X.G, X.sub, NTV, CAPV, X.chunk, MCA, (MCA ? 0 : X.flog), EPI, VAL>;
        nt = NTV;
    } else if constexpr (X.kind == K_SEARCH) {
        fn = k_search<NT_GROUP, X.G, (W ? X.cap_write : X.cap), EPI, VAL>;
        nt = NT_GROUP;
    } else {
        constexpr int CAPV = W ? X.cap_write : X.cap;
        constexpr int CHV = W ? X.chunk_write : X.chunk;
        constexpr int FLOGV = (X.kind == K_HASH_BLOCK) ? X.flog : 0;
        fn = k_block<X.G, X.kind, X.sub, CAPV, CHV, X.split_log2, FLOGV, X.batch, EPI, VAL, (FLOGV > 0 ? X.lowb : 0),
                     (FLOGV > 0 ? X.comp : 0)>;
        nt = X.G;
    }
    // resident CTAs per SM, computed once per kernel instance (and device)
    static int per_sm_cache[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    int &per_sm = per_sm_cache[dev & 63];
    if (per_sm == 0) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(SMEM));
        if (e != cudaSuccess) return e;
        int n = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, nt, SMEM);
        if (e != cudaSuccess) return e;
        per_sm = n < 1 ? 1 : n;
    }
    if (!launch) return cudaSuccess;
    fn<<<num_sms * per_sm, nt, SMEM, s>>>(args);
    return cudaGetLastError();
}

template <int V>
static cudaError_t launch_variant_v(const KArgs &a, int epi, bool val, int sms, cudaStream_t s, bool launch) {
    if (epi == EPI_WRITE) return val ? launch_variant_t<V, EPI_WRITE, true>(a, sms, s, launch)
                                     : launch_variant_t<V, EPI_WRITE, false>(a, sms, s, launch);
    if (epi == EPI_SUM) return launch_variant_t<V, EPI_SUM, false>(a, sms, s, launch);
    return launch_variant_t<V, EPI_KEYED, false>(a, sms, s, launch);
}

static cudaError_t launch_variant(int v, const KArgs &a, int epi, bool val, int sms, cudaStream_t s,
                                  bool launch = true) {
    switch (v) {
        case 0: return launch_variant_v<0>(a, epi, val, sms, s, launch);
        case 1: return launch_variant_v<1>(a, epi, val, sms, s, launch);
        case 2: return launch_variant_v<2>(a, epi, val, sms, s, launch);
        case 3: return launch_variant_v<3>(a, epi, val, sms, s, launch);
        case 4: return launch_variant_v<4>(a, epi, val, sms, s, launch);
        case 5: return launch_variant_v<5>(a, epi, val, sms, s, launch);
        case 6: return launch_variant_v<6>(a, epi, val, sms, s, launch);
        case 7: return launch_variant_v<7>(a, epi, val, sms, s, launch);
        case 8: return launch_variant_v<8>(a, epi, val, sms, s, launch);
        case 9: return launch_variant_v<9>(a, epi, val, sms, s, launch);
        case 10: return launch_variant_v<10>(a, epi, val, sms, s, launch);
        case 11: return launch_variant_v<11>(a, epi, val, sms, s, launch);
        case 12: return launch_variant_v<12>(a, epi, val, sms, s, launch);
        case 13: return launch_variant_v<13>(a, epi, val, sms, s, launch);
        case 14: return launch_variant_v<14>(a, epi, val, sms, s, launch);
        case 15: return launch_variant_v<15>(a, epi, val, sms, s, launch);
        case 16: return launch_variant_v<16>(a, epi, val, sms, s, launch);
        case 17: return launch_variant_v<17>(a, epi, val, sms, s, launch);
        case 18: return launch_variant_v<18>(a, epi, val, sms, s, launch);
        case 19: return launch_variant_v<19>(a, epi, val, sms, s, launch);
        case 20: return launch_variant_v<20>(a, epi, val, sms, s, launch);
        case 21: return launch_variant_v<21>(a, epi, val, sms, s, launch);
        case 22: return launch_variant_v<22>(a, epi, val, sms, s, launch);
        case 23: return launch_variant_v<23>(a, epi, val, sms, s, launch);
        default: return cudaErrorInvalidValue;
    }
}

int spgemm_prepare(int epi, bool values, int sched, int force_accum) {
    KArgs none{};
    for (int v = 0; v < NV; ++v) {
        cudaError_t e = launch_variant(v, none, epi, values, ctx().num_sms, nullptr, false);
        if (e != cudaSuccess) return cuda_fail(e, "masked SpGEMM variant setup");
    }
    return sched_prepare(sched, force_accum);
}

size_t spgemm_scratch_bytes(int64_t m) {
    auto r = [](size_t b) { return (b + 255) & ~size_t(255); };
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, static_cast<int64_t *>(nullptr),
                                  static_cast<int64_t *>(nullptr), m + 1);
    return r(8 * m) + r(4 * m) + r(2 * m) + r(4 * m) + 2 * r(8 * (m + 1)) + r(sizeof(BinStats) * NBINS) +
           r(4 * NBINS) + r(4 * (6 * NV + 4)) + r(4 * NV) + r(tmp_bytes);
}

// NVTX range names of the variant launches
static const char *const kVariantRange[NV] = {
    "gk:variant 0",  "gk:variant 1",  "gk:variant 2",  "gk:variant 3",  "gk:variant 4",  "gk:variant 5",
    "gk:variant 6",  "gk:variant 7",  "gk:variant 8",  "gk:variant 9",  "gk:variant 10", "gk:variant 11",
    "gk:variant 12", "gk:variant 13", "gk:variant 14", "gk:variant 15", "gk:variant 16", "gk:variant 17",
    "gk:variant 18", "gk:variant 19", "gk:variant 20", "gk:variant 21", "gk:variant 22", "gk:variant 23"};

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------
int run_spgemm(const SpgemmRequest &rq, Scratch &scr) {
    NvtxRange range("gk:masked_spgemm");
    const DevCsr &A = rq.A, &B = rq.B, &M = rq.M;
    if (A.m != M.m || A.n != B.m || B.n != M.n)
        return fail(GK_ERR_ARG, "shape mismatch: need A.m == M.m, A.n == B.m, B.n == M.n");
    cudaStream_t s = rq.stream;
    Context &c = ctx();
    const bool write = rq.epi == EPI_WRITE;
    if (write && M.nnz > 0 && rq.zero_output) GK_CUDA(cudaMemsetAsync(rq.c_val, 0, sizeof(int32_t) * M.nnz, s));
    if (A.m == 0 || M.nnz == 0 || A.nnz == 0 || B.nnz == 0) return GK_OK;

    const int64_t m = A.m;
    int64_t *work, *item_n, *item_ex;
    int32_t *maxb, *rowlist;
    uint16_t *bin;
    BinStats *bins;
    int *var_of_bin, *vcount, *voff, *vcursor;
    unsigned int *fetch;
    GK_CHECK(scr.alloc(&work, m));
    GK_CHECK(scr.alloc(&maxb, m));
    GK_CHECK(scr.alloc(&bin, m));
    GK_CHECK(scr.alloc(&rowlist, m));
    GK_CHECK(scr.alloc(&item_n, m + 1));
    GK_CHECK(scr.alloc(&item_ex, m + 1));
    GK_CHECK(scr.alloc(&bins, NBINS));
    GK_CHECK(scr.alloc(&var_of_bin, NBINS));
    GK_CHECK(scr.alloc(&vcount, 6 * NV + 4));
    voff = vcount + NV;
    vcursor = voff + NV + 1;          // 2 * NV
    int *vsimple = vcursor + 2 * NV;  // NV
    GK_CHECK(scr.alloc(&fetch, NV));
    GK_CUDA(cudaMemsetAsync(bins, 0, sizeof(BinStats) * NBINS, s));
    GK_CUDA(cudaMemsetAsync(vcount, 0, sizeof(int) * (6 * NV + 4), s));
    GK_CUDA(cudaMemsetAsync(item_n, 0, sizeof(int64_t) * (m + 1), s));

    const int sms = c.num_sms;
    // B's row lengths live in item_ex until the item scan overwrites it (after
    // the row statistics, in stream order); a B with more rows than that holds
    // gets its own buffer (fixed-scratch callers are square and never do)
    int32_t *blen = reinterpret_cast<int32_t *>(item_ex);
    if (B.m > 2 * (m + 1)) GK_CHECK(scr.alloc(&blen, B.m));
    k_row_lengths<<<sms * 8, 256, 0, s>>>(B, blen);
    k_row_stats<<<sms * 8, 256, 0, s>>>(A, blen, work, maxb);
    GK_CUDA(cudaGetLastError());
    k_bin_rows<<<sms * 2, 256, 0, s>>>(A, M, work, maxb, bin, bins);
    GK_CUDA(cudaGetLastError());
    if (rq.bin_variant) {
        GK_CUDA(cudaMemcpyAsync(var_of_bin, rq.bin_variant, sizeof(int) * NBINS, cudaMemcpyHostToDevice, s));
    } else if (rq.force_variant < 0) {
        GK_CHECK(sched_choose(bins, var_of_bin, rq.sched, rq.force_accum, rq.epi, rq.use_values, s));
    }
    if (rq.bin_stats_out)
        GK_CUDA(cudaMemcpyAsync(rq.bin_stats_out, bins, sizeof(BinStats) * NBINS, cudaMemcpyDeviceToDevice, s));
    if (rq.variant_of_bin_out && rq.force_variant < 0)
        GK_CUDA(cudaMemcpyAsync(rq.variant_of_bin_out, var_of_bin, sizeof(int) * NBINS, cudaMemcpyDeviceToDevice, s));
    if (rq.stats_only) {
        note_launches(3);
        return GK_OK;
    }
    k_count_rows<<<sms * 2, 256, 0, s>>>(A, M, work, bin, var_of_bin, rq.force_variant, write, vcount, vsimple);
    GK_CUDA(cudaGetLastError());
    k_offsets<<<1, 32, 0, s>>>(vcount, vsimple, voff, vcursor, fetch);
    GK_CUDA(cudaGetLastError());
    k_scatter_rows<<<sms * 2, 256, 0, s>>>(A, M, work, bin, var_of_bin, rq.force_variant, write, vcursor,
                                           rowlist, item_n);
    GK_CUDA(cudaGetLastError());
    size_t tmp_bytes = 0;
    GK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, item_n, item_ex, m + 1, s));
    void *tmp;
    GK_CHECK(scr.alloc(reinterpret_cast<char **>(&tmp), tmp_bytes));
    GK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, item_n, item_ex, m + 1, s));

    note_launches(6);

    KArgs args;
    args.A = A;
    args.B = B;
    args.M = M;
    args.rowlist = rowlist;
    args.voff = voff;
    args.vsimple = vsimple;
    args.item_ex = item_ex;
    args.work = work;
    args.fetch = fetch;
    args.c_val = rq.c_val;
    args.sums = rq.sums;
    args.row_key = rq.row_key;
    args.vec = (reinterpret_cast<uintptr_t>(B.col) % 16) == 0;
    const bool val = rq.use_values && (A.val || B.val);
    // the variant kernels are independent: with GK_CONCURRENT_VARIANTS=1 they
    // are forked onto side streams and joined (capturable).  Off by default:
    // each variant is a persistent grid that fills the GPU by itself.
    static const bool concurrent = [] {
        const char *e = getenv("GK_CONCURRENT_VARIANTS");
        return e && e[0] == '1';
    }();
    static_assert(NV <= kSideStreams, "one side stream per variant");
    SideStreams &side = side_streams();
    const bool fork = concurrent && rq.force_variant < 0;
    if (fork) GK_CUDA(cudaEventRecord(side.fork, s));
    ProfWindow prof(s, NV);
    cudaEvent_t tev[NV + 1];
    const bool timed = rq.variant_ms_out != nullptr;
    if (timed) {
        for (int v = 0; v <= NV; ++v) GK_CUDA(cudaEventCreate(&tev[v]));
        GK_CUDA(cudaEventRecord(tev[0], s));
    }
    for (int v = 0; v < NV; ++v) {
        if (rq.force_variant >= 0 && v != rq.force_variant) {
            if (timed) GK_CUDA(cudaEventRecord(tev[v + 1], s));
            continue;
        }
        args.v = v;
        cudaStream_t vs = s;
        if (fork) {
            vs = side.s[v];
            GK_CUDA(cudaStreamWaitEvent(vs, side.fork, 0));
        }
        NvtxRange vrange(kVariantRange[v]);
        prof.begin(v, vs);
        cudaError_t e = launch_variant(v, args, rq.epi, val, sms, vs);
        if (e != cudaSuccess) return cuda_fail(e, "masked SpGEMM variant launch");
        prof.end(v, vs);
        note_launches(1);
        if (fork) {
            GK_CUDA(cudaEventRecord(side.join[v], vs));
            GK_CUDA(cudaStreamWaitEvent(s, side.join[v], 0));
        }
        if (timed) GK_CUDA(cudaEventRecord(tev[v + 1], s));
    }
    if (timed) {
        GK_CUDA(cudaEventSynchronize(tev[NV]));
        for (int v = 0; v < NV; ++v) {
            float ms = 0.f;
            GK_CUDA(cudaEventElapsedTime(&ms, tev[v], tev[v + 1]));
            rq.variant_ms_out[v] = ms;
        }
        for (int v = 0; v <= NV; ++v) cudaEventDestroy(tev[v]);
    }
    if (prof.active()) {
        // attribute the bins' work to the variants that ran them
        BinStats hb[NBINS];
        int hv[NBINS];
        GK_CUDA(cudaMemcpyAsync(hb, bins, sizeof(hb), cudaMemcpyDeviceToHost, s));
        GK_CUDA(cudaMemcpyAsync(hv, var_of_bin, sizeof(hv), cudaMemcpyDeviceToHost, s));
        GK_CUDA(cudaStreamSynchronize(s));
        ProfTotals tot[NV] = {};
        for (int b = 0; b < NBINS; ++b) {
            if (!hb[b].rows) continue;
            const int v = rq.force_variant >= 0 ? rq.force_variant : (rq.bin_variant ? rq.bin_variant[b] : hv[b]);
            if (v < 0 || v >= NV) continue;
            tot[v].rows += hb[b].rows;
            tot[v].sum_a += hb[b].sum_a;
            tot[v].sum_m += hb[b].sum_m;
            tot[v].sum_work += hb[b].sum_work;
        }
        GK_CHECK(prof.finish(tot));
    }
    return GK_OK;
}

}  // namespace gk
