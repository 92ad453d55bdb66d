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
//    (shuffles).  No lane idles on an A entry with few pairs.
//  * Mask rows longer than CAP are taken in chunks of CAP columns; a pair is
//    seen in exactly one chunk, so chunking adds no lookups.
//  * Integer terms are summed exactly as in the other kinds (32-bit wrapping
//    per lane, 64-bit row totals).
#pragma once

// Last position in [lo, lo + len) whose value is <= x, for sorted a with
// a[lo] <= x (len >= 1): ceil(log2 len) dependent loads.
__device__ __forceinline__ int64_t last_le(const int32_t *__restrict__ a, int64_t lo, int64_t len, int x) {
    while (len > 1) {
        const int64_t half = len >> 1;
        lo = (__ldg(a + lo + half) <= x) ? lo + half : lo;
        len -= half;
    }
    return lo;
}

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

__device__ __forceinline__ int64_t shfl64(int64_t v, int src) {
    const int lo = __shfl_sync(0xFFFFFFFFu, static_cast<int>(v & 0xFFFFFFFF), src);
    const int hi = __shfl_sync(0xFFFFFFFFu, static_cast<int>(v >> 32), src);
    return (static_cast<int64_t>(hi) << 32) | static_cast<uint32_t>(lo);
}

template <int NT, int CAP, int EPI, bool VAL>
__global__ void __launch_bounds__(NT, GK_LB_THREADS / NT) k_search(KArgs p) {
    constexpr bool ACC = (EPI == EPI_WRITE);
    constexpr int NWARP = NT / 32;
    constexpr unsigned FULL = 0xFFFFFFFFu;
    extern __shared__ int smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int *mk = smem + warp * CAP;
    int *acc = smem + NWARP * CAP + warp * CAP;  // EPI_WRITE only
    const int begin = p.voff[p.v], end = p.voff[p.v + 1];
    unsigned long long local = 0;
    int cur_key = -1;
    unsigned long long cur_sum = 0;
    constexpr int FB = 2;  // rows per fetch
    int got = 0, left = 0;

    while (true) {
        if (left == 0) {
            if (lane == 0) got = static_cast<int>(atomicAdd(p.fetch + p.v, static_cast<unsigned>(FB)));
            got = __shfl_sync(FULL, got, 0);
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
            for (int q = lane; q < clen; q += 32) {
                mk[q] = __ldg(p.M.col + m0 + c0 + q);
                if (ACC) acc[q] = 0;
            }
            __syncwarp();
            const int lo_col = mk[0], hi_col = mk[clen - 1];
            unsigned cnt = 0;
            for (int64_t tb = a0; tb < a1; tb += 32) {
                const int64_t t = tb + lane;
                int64_t b0 = 0, b1 = 0;
                int qlo = 0, n = 0;
                uint32_t av = 1u;
                if (t < a1) {
                    const int k = __ldg(p.A.col + t);
                    b0 = __ldg(p.B.rp + k);
                    b1 = __ldg(p.B.rp + k + 1);
                    if (b1 > b0) {
                        const int first = __ldg(p.B.col + b0), last = __ldg(p.B.col + b1 - 1);
                        if (last >= lo_col && first <= hi_col) {
                            qlo = smem_bound<false>(mk, clen, first);
                            n = smem_bound<true>(mk, clen, last) - qlo;
                        }
                    }
                    if (VAL && p.A.val) av = static_cast<uint32_t>(__ldg(p.A.val + t));
                }
                int incl = n;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += y;
                }
                const int total = __shfl_sync(FULL, incl, 31);
                const int excl = incl - n;
                for (int pb = 0; pb < total; pb += 32) {
                    const int pp = pb + lane;
                    // the pair's A entry: the first lane j whose inclusive
                    // count exceeds pp (binary lifting over the lanes)
                    int j = 0;
#pragma unroll
                    for (int s = 16; s > 0; s >>= 1) {
                        const int v = __shfl_sync(FULL, incl, j + s - 1);
                        if (v <= pp) j += s;
                    }
                    const int ex_j = __shfl_sync(FULL, excl, j);
                    const int qlo_j = __shfl_sync(FULL, qlo, j);
                    const int64_t b0_j = shfl64(b0, j), b1_j = shfl64(b1, j);
                    const uint32_t av_j = VAL ? static_cast<uint32_t>(__shfl_sync(FULL, static_cast<int>(av), j)) : 1u;
                    if (pp < total) {
                        const int q = qlo_j + (pp - ex_j);
                        const int c = mk[q];
                        const int64_t pos = last_le(p.B.col, b0_j, b1_j - b0_j, c);
                        if (__ldg(p.B.col + pos) == c) {
                            const uint32_t w =
                                (VAL && p.B.val) ? av_j * static_cast<uint32_t>(__ldg(p.B.val + pos)) : av_j;
                            if (ACC) atomicAdd(reinterpret_cast<unsigned *>(acc + q), w);
                            else cnt += w;
                        }
                    }
                }
            }
            __syncwarp();
            if (ACC) {
                for (int q = lane; q < clen; q += 32) p.c_val[m0 + c0 + q] = acc[q];
            } else {
                rowsum += cnt;
            }
            __syncwarp();
        }
        if (EPI == EPI_SUM) local += rowsum;
        if (EPI == EPI_KEYED) {
            const int key = p.row_key ? p.row_key[row] : row;
            if (key != cur_key) {
                const unsigned long long tot = group_sum<32>(cur_sum, FULL);
                if (lane == 0 && tot) atomicAdd(p.sums + cur_key, tot);
                cur_key = key;
                cur_sum = 0;
            }
            cur_sum += rowsum;
        }
    }
    if (EPI == EPI_KEYED && cur_key >= 0) {
        const unsigned long long tot = group_sum<32>(cur_sum, FULL);
        if (lane == 0 && tot) atomicAdd(p.sums + cur_key, tot);
    }
    if (EPI == EPI_SUM) {
        const unsigned long long tot = group_sum<32>(local, FULL);
        if (lane == 0 && tot) atomicAdd(p.sums, tot);
    }
}
