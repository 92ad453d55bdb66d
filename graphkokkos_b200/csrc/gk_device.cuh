// Device-side building blocks of the masked SpGEMM kernels: thread-group
// masks, shared-memory hash sets of mask columns, group-cooperative search in
// sorted CSR rows, and reductions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// Resident threads per SM the engine kernels are register-capped for
// (launch bounds NT, GK_LB_THREADS / NT).
#ifndef GK_LB_THREADS
#define GK_LB_THREADS 1536
#endif

namespace gk {

constexpr int EMPTY_KEY = -1;

// When a row's mask is processed in chunks (column ranges), a B row longer
// than this is cut to the chunk's column range by two group searches; a
// shorter one is streamed whole, since its columns outside the range are not
// in the chunk's structure and cost less to test than the searches' round
// trips to memory.
constexpr int64_t CUT_MIN = 256;

// Lanes of the calling thread's aligned group of G threads inside its warp.
template <int G>
__device__ __forceinline__ unsigned group_mask() {
    if constexpr (G >= 32) {
        return 0xFFFFFFFFu;
    } else {
        const unsigned base = (threadIdx.x & 31) / G * G;
        return ((1u << G) - 1u) << base;
    }
}

template <int G>
__device__ __forceinline__ unsigned low_bits() {
    if constexpr (G >= 32) return 0xFFFFFFFFu;
    else return (1u << G) - 1u;
}

// Bit of x in a 2^FLOG-bit filter (a second multiplicative hash, independent
// of the table's bucket hash).
template <int FLOG>
__device__ __forceinline__ uint32_t filter_bit(int x) {
    return (static_cast<uint32_t>(x) * 0x85EBCA77u) >> (32 - FLOG);
}

// Position of x in a filter whose first 2^LOWB bits map columns below 2^LOWB
// one to one (an exact bitmap of the low columns, where power-law graphs
// without relabelling keep their hubs) followed by the 2^FLOG hashed bits.
template <int FLOG, int LOWB>
__device__ __forceinline__ uint32_t filter_pos(int x) {
    if constexpr (LOWB > 0) {
        const uint32_t ux = static_cast<uint32_t>(x);
        return ux < (1u << LOWB) ? ux : (1u << LOWB) + filter_bit<FLOG>(x);
    } else {
        return filter_bit<FLOG>(x);
    }
}

// The mask tables are bucketed open addressing: CAP slots as CAP/4 buckets
// of four adjacent slots, read with one 16-byte shared-memory load.  A key
// lives in its home bucket or, when that bucket is full, in the following
// ones (linear probing over buckets).  The slots of a bucket fill in order,
// so a bucket with an empty last slot ends every probe sequence.
template <int CAP>
__device__ __forceinline__ int home_bucket(int x) {
    constexpr int LOG2 = __builtin_ctz(CAP / 4);
    static_assert(CAP >= 8 && (CAP & (CAP - 1)) == 0, "table size must be a power of two >= 8");
    return static_cast<int>((static_cast<uint32_t>(x) * 0x9E3779B1u) >> (32 - LOG2));
}

// Inserts x; concurrent inserts of distinct keys are safe (a slot is claimed
// by compare-and-swap only after the slots before it were seen taken).  The
// caller guarantees fewer than CAP keys; the probe count is bounded anyway.
template <int CAP>
__device__ __forceinline__ void hash_insert(int *keys, int x) {
    int b = home_bucket<CAP>(x);
#pragma unroll 1
    for (int probe = 0; probe < CAP / 4; ++probe) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int prev = atomicCAS(keys + 4 * b + i, EMPTY_KEY, x);
            if (prev == EMPTY_KEY || prev == x) return;
        }
        b = (b + 1) & (CAP / 4 - 1);
    }
}

// Slot of x, or -1 when x is not a key.
template <int CAP>
__device__ __forceinline__ int hash_find(const int *keys, int x) {
    int b = home_bucket<CAP>(x);
#pragma unroll 1
    for (int probe = 0; probe < CAP / 4; ++probe) {
        const int4 k = *reinterpret_cast<const int4 *>(keys + 4 * b);
        if (k.x == x) return 4 * b;
        if (k.y == x) return 4 * b + 1;
        if (k.z == x) return 4 * b + 2;
        if (k.w == x) return 4 * b + 3;
        if (k.w == EMPTY_KEY) return -1;
        b = (b + 1) & (CAP / 4 - 1);
    }
    return -1;
}

// Whether x is a key (no slot needed: the sum epilogues).
template <int CAP>
__device__ __forceinline__ bool hash_has(const int *keys, int x) {
    int b = home_bucket<CAP>(x);
#pragma unroll 1
    for (int probe = 0; probe < CAP / 4; ++probe) {
        const int4 k = *reinterpret_cast<const int4 *>(keys + 4 * b);
        if ((k.x == x) | (k.y == x) | (k.z == x) | (k.w == x)) return true;
        if (k.w == EMPTY_KEY) return false;
        b = (b + 1) & (CAP / 4 - 1);
    }
    return false;
}

// Index of x in sorted keys[0, n), or -1.
__device__ __forceinline__ int sorted_find(const int *keys, int n, int x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (keys[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return (lo < n && keys[lo] == x) ? lo : -1;
}

// First index in [lo, hi) with a[idx] >= x, for a sorted ascending; computed
// cooperatively by the G lanes of a group (a G-ary search: every round each
// lane probes one pivot, a ballot counts the pivots below x).  All lanes of
// the group must call it with the same arguments; all get the result.
template <int G>
__device__ __forceinline__ int64_t group_lower_bound(const int32_t *__restrict__ a, int64_t lo, int64_t hi,
                                                     int x, int lane, unsigned gmask) {
    const unsigned shift = (G >= 32) ? 0u : ((threadIdx.x & 31) / G * G);
#pragma unroll 1
    while (hi - lo > G) {
        const int64_t len = hi - lo;
        const int64_t piv = lo + (len * (lane + 1)) / (G + 1);
        const bool below = a[piv] < x;
        const unsigned bal = (__ballot_sync(gmask, below) >> shift) & low_bits<G>();
        const int c = __popc(bal);
        const int64_t new_lo = (c == 0) ? lo : lo + (len * c) / (G + 1) + 1;
        const int64_t new_hi = (c == G) ? hi : lo + (len * (c + 1)) / (G + 1);
        lo = new_lo;
        hi = new_hi;
    }
    const bool below = (lo + lane < hi) && a[lo + lane] < x;
    const unsigned bal = (__ballot_sync(gmask, below) >> shift) & low_bits<G>();
    return lo + __popc(bal);
}

// Sum over the G lanes of a group (all lanes get the total).
template <int G, class T>
__device__ __forceinline__ T group_sum(T v, unsigned gmask) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gmask, v, o, G);
    return v;
}

// Block-wide sum; every thread of the block must call it.  Result valid in
// thread 0.  `red` is shared scratch of at least blockDim.x/32 entries.
template <class T>
__device__ __forceinline__ T block_sum(T v, T *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    T t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += red[w];
    return t;
}

__device__ __forceinline__ int ilog2_u64(unsigned long long x) { return x ? 63 - __clzll(x) : 0; }

// ----- asynchronous staging of a sorted mask chunk into shared memory ---------
// cp.async copies global memory to shared memory without passing through
// registers; the copies of a chunk are issued by all of the group's lanes and
// complete at cp_async_wait_all() (a hardware wait, no polling loop).
__device__ __forceinline__ void cp_async_4(void *dst, const void *src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_16(void *dst, const void *src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Element offset (0..3) that puts a shared-memory copy of src on the same
// position modulo 16 bytes as src, so that its interior can move in 16-byte
// copies.  The shared buffer must hold n + 3 elements.
__device__ __forceinline__ int stage_phase(const int32_t *src) {
    return static_cast<int>((reinterpret_cast<uintptr_t>(src) >> 2) & 3);
}

// dst[0, n) = src[0, n) by cp.async, issued by `lane` of `lanes` threads; dst
// is congruent to src modulo 16 bytes (stage_phase).  The 16-byte-aligned
// interior moves in 16-byte copies, the ragged ends (at most 3 elements each)
// in 4-byte copies, so no copy reads outside src[0, n).
__device__ __forceinline__ void stage_ints_async(int *dst, const int32_t *src, int n, int lane, int lanes) {
    int head = (4 - stage_phase(src)) & 3;
    if (head > n) head = n;
    const int body = (n - head) & ~3;
    for (int q = lane; q < head; q += lanes) cp_async_4(dst + q, src + q);
    for (int q = head + 4 * lane; q < head + body; q += 4 * lanes) cp_async_16(dst + q, src + q);
    for (int q = head + body + lane; q < n; q += lanes) cp_async_4(dst + q, src + q);
}

// Number of A-entry splits of a row in the block kinds.
__host__ __device__ __forceinline__ int64_t num_splits(int64_t work, int64_t a_len, int split_log2) {
    if (split_log2 <= 0 || a_len <= 1) return 1;
    int64_t s = (work + (int64_t(1) << split_log2) - 1) >> split_log2;
    if (s < 1) s = 1;
    if (s > a_len) s = a_len;
    if (s > 4096) s = 4096;
    return s;
}

}  // namespace gk
