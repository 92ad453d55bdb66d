// Block kinds of the masked SpGEMM engine (included by spgemm.cu): one CTA
// per item, an item being (row, mask chunk or column window, A-entry split).
//
//  * Items are taken from a per-variant counter NB at a time.  Rows that are
//    a single item sit first in the variant's row list, so their items map
//    to rows directly; only split rows need a binary search over the prefix
//    of item counts.
//  * The mask chunk is built into shared memory: a hash set (load factor
//    <= 1/4) behind a bitmap filter of 2^FLOG bits (one load rejects most
//    misses without entering the probe loop), a sorted list (MCA), or a dense
//    column-window bitmap + accumulator (MSA).
//  * Sub-groups of SUB lanes take the item's A entries dynamically; the next
//    entry's B-row bounds are loaded while the current B row streams.
#pragma once

// Resident CTAs a block kind is register-capped for: GK_LB_THREADS / NT, or
// fewer when its shared memory (table, accumulators, filter) admits fewer per
// SM anyway, so that the large-table kinds get the registers of the residency
// they can actually reach.
__host__ __device__ constexpr int block_min_ctas(int nt, int kind, int cap, int flog, int lowb, bool acc,
                                                 int comp = 0) {
    const int by_threads = GK_LB_THREADS / nt < 1 ? 1 : GK_LB_THREADS / nt;
    if (kind != K_HASH_BLOCK) return by_threads;
    const long smem = long(cap) * 4 * (acc ? 2 : 1) + (flog > 0 ? ((1l << lowb) + (1l << flog)) / 8 : 0) +
                      (comp ? long(nt) * 8 * 4 : 0);
    const int by_smem = int((228l * 1024) / (smem + 1024));
    return by_smem < 1 ? 1 : (by_smem < by_threads ? by_smem : by_threads);
}

template <int NT, int KIND, int SUB, int CAP, int CHUNK, int SPLIT, int FLOG, int NB, int EPI, bool VAL, int LOWB = 0,
          int COMP = 0>
__global__ void __launch_bounds__(NT, block_min_ctas(NT, KIND, CAP, FLOG, LOWB, EPI == EPI_WRITE, COMP))
    k_block(KArgs p) {
    constexpr bool ACC = (EPI == EPI_WRITE);
    constexpr int NW = NT / 32;
    constexpr int WIN = (KIND == K_MSA_BLOCK) ? (1 << CAP) : 0;  // MSA: CAP = log2 window width
    // filter words: 2^LOWB exact bits for the low columns, then 2^FLOG hashed bits
    constexpr int FWORDS = (KIND == K_HASH_BLOCK && FLOG > 0) ? ((1 << LOWB) + (1 << FLOG)) / 32 : 0;
    constexpr int PKV = (KIND == K_MSA_BLOCK) ? PK_MSA : ((KIND == K_MCA_BLOCK) ? PK_MCA : PK_HASH);
    extern __shared__ int smem[];
    __shared__ unsigned long long s_red[NW];
    __shared__ int64_t s_item, s_base;
    __shared__ int s_pos, s_left, s_next;
    const int sl = threadIdx.x % SUB;
    const unsigned smask = group_mask<SUB>();
    const int begin = p.voff[p.v], end = p.voff[p.v + 1];
    if (begin == end) return;
    const int nsimple = p.vsimple[p.v];
    const int64_t ibeg = p.item_ex[begin], iend = p.item_ex[end];
    if (threadIdx.x == 0) s_left = 0;
    unsigned long long local = 0;

    while (true) {
        if (threadIdx.x == 0) {
            if (s_left == 0) {
                s_base = static_cast<int64_t>(atomicAdd(p.fetch + p.v, static_cast<unsigned>(NB)));
                s_left = NB;
            }
            const int64_t rel = s_base + (NB - s_left);
            --s_left;
            const int64_t I = ibeg + rel;
            s_item = I;
            if (I < iend) {
                if (rel < nsimple) {
                    s_pos = begin + static_cast<int>(rel);
                } else {  // last position in the split-row part whose prefix <= I
                    int lo = begin + nsimple, hi = end;
                    while (hi - lo > 1) {
                        const int mid = (lo + hi) >> 1;
                        if (p.item_ex[mid] <= I) lo = mid;
                        else hi = mid;
                    }
                    s_pos = lo;
                }
            }
        }
        __syncthreads();
        const int64_t I = s_item;
        if (I >= iend) break;
        const int pos = s_pos;
        const int row = p.rowlist[pos];
        const int64_t l = I - p.item_ex[pos];
        const int64_t m0 = p.M.rp[row];
        const int mlen = static_cast<int>(p.M.rp[row + 1] - m0);
        const int64_t a0 = p.A.rp[row], alen = p.A.rp[row + 1] - a0;
        const int64_t nsp = num_splits(p.work[row], alen, SPLIT);
        const int64_t ch = l / nsp, sp = l % nsp;
        const int64_t t0 = a0 + alen * sp / nsp, t1 = a0 + alen * (sp + 1) / nsp;
        const int32_t *__restrict__ mc = p.M.col + m0;

        // ---- build the mask structure of this item ----
        int c0, c1;  // mask positions covered
        int lo_col, hi_col;
        int *keys = smem;
        // MCA: the sorted keys sit at an offset of 0..3 elements (cp.async
        // staging keeps them congruent to the source modulo 16 bytes)
        int *acc = smem + ((KIND == K_MSA_BLOCK) ? (ACC ? WIN / 32 : 0) : (KIND == K_MCA_BLOCK ? CAP + 4 : CAP));
        unsigned *bits = reinterpret_cast<unsigned *>(smem);
        unsigned *filt = reinterpret_cast<unsigned *>(smem + CAP * (ACC ? 2 : 1));
        bool cut;
        if constexpr (KIND == K_MSA_BLOCK) {
            const int64_t wbase = ((int64_t)(mc[0] >> CAP) + ch) << CAP;
            lo_col = static_cast<int>(wbase);
            {
                const int64_t hc = wbase + WIN - 1;
                hi_col = static_cast<int>(hc < 0x7FFFFFFF ? hc : 0x7FFFFFFF);
            }
            int lo = 0, hi = mlen;  // mask positions inside the window
            while (lo < hi) {
                const int md = (lo + hi) >> 1;
                if (mc[md] < lo_col) lo = md + 1;
                else hi = md;
            }
            c0 = lo;
            hi = mlen;
            while (lo < hi) {
                const int md = (lo + hi) >> 1;
                if (mc[md] <= hi_col) lo = md + 1;
                else hi = md;
            }
            c1 = lo;
            for (int wd = threadIdx.x; wd < WIN / 32; wd += NT) bits[wd] = 0u;
            __syncthreads();
            for (int q = c0 + threadIdx.x; q < c1; q += NT) {
                const int x = mc[q] - lo_col;
                atomicOr(bits + (x >> 5), 1u << (x & 31));
                if (ACC) acc[x] = 0;
            }
            cut = (mc[0] >> CAP) != (mc[mlen - 1] >> CAP);
        } else {
            c0 = static_cast<int>(ch) * CHUNK;
            c1 = min(mlen, c0 + CHUNK);
            if constexpr (KIND == K_MCA_BLOCK) {
                // the sorted chunk is copied verbatim: cp.async staging
                keys = smem + stage_phase(mc + c0);
                stage_ints_async(keys, mc + c0, c1 - c0, threadIdx.x, NT);
                if (ACC)
                    for (int q = threadIdx.x; q < c1 - c0; q += NT) acc[q] = 0;
                cp_async_wait_all();
            } else {
                for (int s = threadIdx.x; s < CAP; s += NT) {
                    keys[s] = EMPTY_KEY;
                    if (ACC) acc[s] = 0;
                }
                for (int wd = threadIdx.x; wd < FWORDS; wd += NT) filt[wd] = 0u;
                __syncthreads();
                for (int q = c0 + threadIdx.x; q < c1; q += NT) {
                    const int x = mc[q];
                    // without accumulators a low column needs no slot: its
                    // filter bit is exact
                    if (ACC || LOWB == 0 || static_cast<uint32_t>(x) >= (1u << LOWB)) hash_insert<CAP>(keys, x);
                    if constexpr (FWORDS > 0) {
                        const uint32_t h = filter_pos<FLOG, LOWB>(x);
                        atomicOr(filt + (h >> 5), 1u << (h & 31));
                    }
                }
            }
            lo_col = mc[c0];
            hi_col = mc[c1 - 1];
            cut = mlen > CHUNK;
        }
        if (threadIdx.x == 0) s_next = 0;
        __syncthreads();

        // ---- stream the B rows of A entries [t0, t1): sub-groups fetch entries
        //      dynamically; the next entry's bounds load during the current row ----
        unsigned cnt = 0;
        const int clen = c1 - c0;
        if (c1 > c0) {
            const int probe_arg = (KIND == K_MSA_BLOCK) ? lo_col : clen;
            const int *pkeys = (KIND == K_MSA_BLOCK) ? reinterpret_cast<const int *>(bits) : keys;
            const unsigned *pfilt = FWORDS > 0 ? filt : nullptr;
            // candidate queue of this sub-group (COMP kinds): 8 elements per lane
            int *queue = COMP ? reinterpret_cast<int *>(filt + FWORDS) + (threadIdx.x / SUB) * 8 * SUB : nullptr;
            auto fetch = [&]() -> int64_t {
                int tt = 0;
                if (sl == 0) tt = atomicAdd(&s_next, 1);
                return t0 + __shfl_sync(smask, tt, 0, SUB);
            };
            int64_t tc = fetch();
            if (tc < t1) {
                BRow nxt = brow_of<VAL>(p, __ldg(p.A.col + tc), tc);
                int64_t tn = fetch();
                int k2 = tn < t1 ? __ldg(p.A.col + tn) : 0;
                while (tc < t1) {
                    BRow cur = nxt;
                    if (tn < t1) nxt = brow_of<VAL>(p, k2, tn);
                    const int64_t tnn = (tn < t1) ? fetch() : t1;
                    if (tnn < t1) k2 = __ldg(p.A.col + tnn);
                    if (cur.b0 < cur.b1) {
                        bool skip = false;
                        if (cut && cur.b1 - cur.b0 > CUT_MIN) {
                            skip = __ldg(p.B.col + cur.b1 - 1) < lo_col || __ldg(p.B.col + cur.b0) > hi_col;
                            if (!skip) {
                                const int64_t lo = group_lower_bound<SUB>(p.B.col, cur.b0, cur.b1, lo_col, sl, smask);
                                cur.b1 = group_lower_bound<SUB>(p.B.col, lo, cur.b1, hi_col + 1, sl, smask);
                                cur.b0 = lo;
                            }
                        }
                        if (!skip)
                            stream_row<SUB, CAP, PKV, ACC, VAL, (FWORDS > 0 ? FLOG : 0), (FWORDS > 0 ? LOWB : 0),
                                       (FWORDS > 0 ? COMP : 0)>(p, cur.b0, cur.b1, sl, cur.av, pkeys, acc, probe_arg,
                                                                 cnt, pfilt, hi_col, queue);
                    }
                    tc = tn;
                    tn = tnn;
                }
            }
        }
        __syncthreads();

        // ---- epilogue ----
        if (ACC) {
            for (int q = c0 + threadIdx.x; q < c1; q += NT) {
                int s;
                if constexpr (KIND == K_MSA_BLOCK) s = mc[q] - lo_col;
                else if constexpr (KIND == K_MCA_BLOCK) s = q - c0;
                else s = hash_find<CAP>(keys, mc[q]);
                const int val = acc[s];
                if (nsp == 1) p.c_val[m0 + q] = val;
                else if (val) atomicAdd(p.c_val + m0 + q, val);
            }
        } else if (EPI == EPI_KEYED) {
            const unsigned long long tot = block_sum(static_cast<unsigned long long>(cnt), s_red);
            if (threadIdx.x == 0 && tot) atomicAdd(p.sums + (p.row_key ? p.row_key[row] : row), tot);
        } else {
            local += cnt;
        }
        __syncthreads();
    }
    if (EPI == EPI_SUM) {
        const unsigned long long tot = block_sum(local, s_red);
        if (threadIdx.x == 0 && tot) atomicAdd(p.sums, tot);
    }
}
