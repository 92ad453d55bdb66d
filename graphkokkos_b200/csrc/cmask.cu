// Complement-masked product C<!M> = A·B: gk_mxmm_cmask.
//
// Reference: mxmm_msa_cmask (include/matrix_la.h:733-934).  Row i of C holds
// every column j reached by some product A(i,k)·B(k,j) — structurally, kept
// even where the sum is zero — that is not a column of M's row i, in
// ascending order, with the sum of the products.  The reference sizes C with
// a symbolic pass over a dense per-thread state array and then scans all B.n
// columns for every row to emit them in order (:834-843).
//
// Here: expand, sort, compress, over batches of rows whose products fit a
// fixed budget.
//   1. work per row (sum of nnz(B_k) over the row's A entries), on the host
//      once to cut the batches;
//   2. per batch, the products' offsets (a scan over the batch's A entries)
//      and one warp per row writing a 64-bit key (row << 32 | column) and the
//      product for every B element, the key of a column of M's row (binary
//      search in the sorted mask row) replaced by a sentinel that sorts last;
//   3. one radix sort of (key, product) and one reduce-by-key: the runs are
//      C's entries in CSR order, so the batch's run j is entry rp[r0] + j.
// Two calls, as the reference's symbolic and numeric passes: without C_col the
// row pointers are computed; with them (and C_rowptr from the first call) the
// columns and values are written.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "gk_common.cuh"

namespace gk {

constexpr int64_t CMASK_BUDGET = int64_t(1) << 26;  // products per batch
constexpr unsigned long long CMASK_SENTINEL = ~0ull;

__global__ void k_cmask_row_work(DevCsr A, DevCsr B, int64_t *work) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < A.m; i += warps) {
        int64_t w = 0;
        for (int64_t t = A.rp[i] + lane; t < A.rp[i + 1]; t += 32) {
            const int k = A.col[t];
            w += B.rp[k + 1] - B.rp[k];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xFFFFFFFFu, w, o);
        if (lane == 0) work[i] = w;
    }
}

__global__ void k_cmask_entry_len(DevCsr A, DevCsr B, int64_t t0, int64_t t1, int64_t *len) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = t0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < t1; t += stride) {
        const int k = A.col[t];
        len[t - t0] = B.rp[k + 1] - B.rp[k];
    }
}

// One warp per row of [r0, r1): every product of the row at off[t - t0] + q.
__global__ void k_cmask_expand(DevCsr A, DevCsr B, DevCsr M, int64_t r0, int64_t r1, int64_t t0, const int64_t *off,
                               bool values, unsigned long long *keys, int32_t *prods) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = r0 + (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < r1; i += warps) {
        const int64_t m0 = M.rp[i], m1 = M.rp[i + 1];
        for (int64_t t = A.rp[i]; t < A.rp[i + 1]; ++t) {
            const int k = A.col[t];
            const uint32_t a = (values && A.val) ? static_cast<uint32_t>(A.val[t]) : 1u;
            const int64_t b0 = B.rp[k], b1 = B.rp[k + 1], o = off[t - t0] - b0;
            for (int64_t j = b0 + lane; j < b1; j += 32) {
                const int c = B.col[j];
                int64_t lo = m0, hi = m1;  // is c a column of M's row i?
                while (lo < hi) {
                    const int64_t md = (lo + hi) >> 1;
                    if (M.col[md] < c) lo = md + 1;
                    else hi = md;
                }
                const bool masked = lo < m1 && M.col[lo] == c;
                const uint32_t b = (values && B.val) ? static_cast<uint32_t>(B.val[j]) : 1u;
                keys[o + j] = masked ? CMASK_SENTINEL
                                     : ((static_cast<unsigned long long>(i) << 32) | static_cast<uint32_t>(c));
                prods[o + j] = static_cast<int32_t>(a * b);
            }
        }
    }
}

// Entries per row from the sorted unique keys (the sentinel run excluded).
__global__ void k_cmask_row_counts(const unsigned long long *uniq, const int64_t *nruns, int64_t *cnt) {
    const int64_t n = *nruns;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        const unsigned long long k = uniq[r];
        if (k != CMASK_SENTINEL) atomicAdd(reinterpret_cast<unsigned long long *>(cnt + (k >> 32)), 1ull);
    }
}

__global__ void k_cmask_write(const unsigned long long *uniq, const int32_t *sums, const int64_t *nruns, int64_t base,
                              int32_t *c_col, int32_t *c_val) {
    const int64_t n = *nruns;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        const unsigned long long k = uniq[r];
        if (k == CMASK_SENTINEL) continue;
        c_col[base + r] = static_cast<int32_t>(k & 0xFFFFFFFFull);
        if (c_val) c_val[base + r] = sums[r];
    }
}

// wrapping int32 sum, as the reference accumulates int values
struct WrapSum {
    __device__ __forceinline__ int32_t operator()(int32_t a, int32_t b) const {
        return static_cast<int32_t>(static_cast<uint32_t>(a) + static_cast<uint32_t>(b));
    }
};

}  // namespace gk

using namespace gk;

extern "C" int gk_mxmm_cmask(const gk_csr *A, const gk_csr *B, const gk_csr *M, int semiring, int64_t *C_rowptr,
                             int32_t *C_col, int32_t *C_val, void *stream) {
    NvtxRange range("gk:mxmm_cmask");
    GK_CHECK(validate_csr_shape(A, "A"));
    GK_CHECK(validate_csr_shape(B, "B"));
    GK_CHECK(validate_csr_shape(M, "M"));
    if (A->m != M->m || A->n != B->m || B->n != M->n)
        return fail(GK_ERR_ARG, "shape mismatch: need A.m == M.m, A.n == B.m, B.n == M.n");
    if (semiring != GK_PLUS_TIMES && semiring != GK_PLUS_PAIR) return fail(GK_ERR_ARG, "unknown semiring");
    if (!C_rowptr) return fail(GK_ERR_ARG, "C_rowptr is null");
    if (A->m >= (int64_t(1) << 31) || B->n >= (int64_t(1) << 31))
        return fail(GK_ERR_UNSUPPORTED, "complement-masked product: dimensions must be < 2^31");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    DevCsr a, b, mk;
    GK_CHECK(stage_csr(A, &a, scr, s, nullptr, CSR_STRUCTURE, "A"));
    GK_CHECK(stage_csr(B, &b, scr, s, nullptr, CSR_STRUCTURE, "B"));
    GK_CHECK(stage_csr(M, &mk, scr, s, nullptr, CSR_SORTED, "M"));
    const bool values = semiring == GK_PLUS_TIMES;
    const int64_t m = A->m;
    const bool fill = C_col != nullptr;
    const int sms = ctx().num_sms;

    // work per row on the host, to cut the batches
    int64_t *work;
    GK_CHECK(scr.alloc(&work, m > 0 ? m : 1));
    if (m > 0) {
        k_cmask_row_work<<<sms * 8, 256, 0, s>>>(a, b, work);
        note_launches(1);
    }
    std::vector<int64_t> hwork(m), arp(m + 1), crp(m + 1, 0);
    if (m > 0) GK_CUDA(cudaMemcpyAsync(hwork.data(), work, sizeof(int64_t) * m, cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaMemcpyAsync(arp.data(), a.rp, sizeof(int64_t) * (m + 1), cudaMemcpyDeviceToHost, s));
    if (fill) GK_CUDA(cudaMemcpyAsync(crp.data(), C_rowptr, sizeof(int64_t) * (m + 1), cudaMemcpyDefault, s));
    GK_CUDA(cudaStreamSynchronize(s));
    int64_t maxb = 0;  // largest batch (a row above the budget is a batch of its own)
    for (int64_t i = 0, acc = 0; i < m; ++i) {
        if (acc > 0 && acc + hwork[i] > CMASK_BUDGET) acc = 0;
        acc += hwork[i];
        if (acc > maxb) maxb = acc;
    }
    int64_t *cnt = nullptr;
    int32_t *dcol = C_col, *dval = C_val;
    const int64_t cnnz = fill ? crp[m] : 0;
    if (fill && crp[0] != 0) return fail(GK_ERR_ARG, "C_rowptr[0] must be 0 (pass the first call's row pointers)");
    if (!fill) {
        GK_CHECK(scr.alloc(&cnt, m + 1));
        GK_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int64_t) * (m + 1), s));
    } else {
        if (cnnz > 0 && !is_device_pointer(C_col)) GK_CHECK(scr.alloc(&dcol, cnnz));
        if (cnnz > 0 && C_val && !is_device_pointer(C_val)) GK_CHECK(scr.alloc(&dval, cnnz));
    }
    unsigned long long *keys = nullptr, *keys2 = nullptr, *uniq = nullptr;
    int32_t *prods = nullptr, *prods2 = nullptr, *sums = nullptr;
    int64_t *off = nullptr, *nruns = nullptr;
    int64_t max_entries = 0;
    for (int64_t i = 0; i < m; ++i) max_entries = std::max(max_entries, arp[i + 1] - arp[i]);
    size_t sort_bytes = 0, red_bytes = 0, scan_bytes = 0;
    void *tmp = nullptr;
    if (maxb > 0) {
        GK_CHECK(scr.alloc(&keys, maxb));
        GK_CHECK(scr.alloc(&keys2, maxb));
        GK_CHECK(scr.alloc(&uniq, maxb));
        GK_CHECK(scr.alloc(&prods, maxb));
        GK_CHECK(scr.alloc(&prods2, maxb));
        GK_CHECK(scr.alloc(&sums, maxb));
        GK_CHECK(scr.alloc(&nruns, 1));
        const int nmax = static_cast<int>(std::min<int64_t>(maxb, (int64_t(1) << 31) - 1));
        GK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, keys, keys2, prods, prods2, nmax, 0, 64, s));
        GK_CUDA(cub::DeviceReduce::ReduceByKey(nullptr, red_bytes, keys2, uniq, prods2, sums, nruns, WrapSum(), nmax,
                                               s));
    }
    // entry offsets: the largest batch's A entries
    int64_t max_batch_entries = 1;
    {
        int64_t r0 = 0;
        while (r0 < m) {
            int64_t r1 = r0, acc = 0;
            while (r1 < m && (r1 == r0 || acc + hwork[r1] <= CMASK_BUDGET)) acc += hwork[r1++];
            max_batch_entries = std::max(max_batch_entries, arp[r1] - arp[r0] + 1);
            r0 = r1;
        }
    }
    if (maxb >= (int64_t(1) << 31)) return fail(GK_ERR_UNSUPPORTED, "complement-masked product: a row has >= 2^31 products");
    int64_t *len;
    GK_CHECK(scr.alloc(&len, max_batch_entries));
    GK_CHECK(scr.alloc(&off, max_batch_entries));
    GK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, len, off, max_batch_entries, s));
    GK_CHECK(scr.alloc(reinterpret_cast<char **>(&tmp), std::max(std::max(sort_bytes, red_bytes), scan_bytes)));
    const size_t tmp_bytes = std::max(std::max(sort_bytes, red_bytes), scan_bytes);

    for (int64_t r0 = 0; r0 < m;) {
        int64_t r1 = r0, acc = 0;
        while (r1 < m && (r1 == r0 || acc + hwork[r1] <= CMASK_BUDGET)) acc += hwork[r1++];
        const int64_t n = acc;
        const int64_t t0 = arp[r0], t1 = arp[r1];
        if (n > 0) {
            k_cmask_entry_len<<<sms * 4, 256, 0, s>>>(a, b, t0, t1, len);
            GK_CUDA(cudaMemsetAsync(len + (t1 - t0), 0, sizeof(int64_t), s));
            size_t tb = tmp_bytes;
            GK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, len, off, t1 - t0 + 1, s));
            k_cmask_expand<<<sms * 8, 256, 0, s>>>(a, b, mk, r0, r1, t0, off, values, keys, prods);
            tb = tmp_bytes;
            GK_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys2, prods, prods2, static_cast<int>(n), 0, 64, s));
            tb = tmp_bytes;
            GK_CUDA(cub::DeviceReduce::ReduceByKey(tmp, tb, keys2, uniq, prods2, sums, nruns, WrapSum(),
                                                   static_cast<int>(n), s));
            if (!fill)
                k_cmask_row_counts<<<sms * 4, 256, 0, s>>>(uniq, nruns, cnt);
            else
                k_cmask_write<<<sms * 4, 256, 0, s>>>(uniq, sums, nruns, crp[r0], dcol, dval);
            note_launches(4);
            GK_CUDA(cudaGetLastError());
            if (fill) {  // the batch must produce exactly the entries the row pointers give it
                int64_t runs = 0;
                unsigned long long last = 0;
                GK_CUDA(cudaMemcpyAsync(&runs, nruns, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
                GK_CUDA(cudaStreamSynchronize(s));
                if (runs > 0)
                    GK_CUDA(cudaMemcpyAsync(&last, uniq + runs - 1, sizeof(last), cudaMemcpyDeviceToHost, s));
                GK_CUDA(cudaStreamSynchronize(s));
                const int64_t got = runs - (runs > 0 && last == CMASK_SENTINEL ? 1 : 0);
                if (got != crp[r1] - crp[r0])
                    return fail(GK_ERR_ARG, "C_rowptr does not match this product (pass the first call's row pointers)");
            }
        }
        r0 = r1;
    }
    if (!fill) {
        int64_t *rp_dev;
        GK_CHECK(scr.alloc(&rp_dev, m + 1));
        size_t tb = tmp_bytes;
        GK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, rp_dev, m + 1, s));
        void *t2;
        GK_CHECK(scr.alloc(reinterpret_cast<char **>(&t2), tb));
        GK_CUDA(cub::DeviceScan::ExclusiveSum(t2, tb, cnt, rp_dev, m + 1, s));
        GK_CUDA(cudaMemcpyAsync(C_rowptr, rp_dev, sizeof(int64_t) * (m + 1), cudaMemcpyDefault, s));
    } else {
        if (cnnz > 0 && dcol != C_col)
            GK_CUDA(cudaMemcpyAsync(C_col, dcol, sizeof(int32_t) * cnnz, cudaMemcpyDeviceToHost, s));
        if (cnnz > 0 && C_val && dval != C_val)
            GK_CUDA(cudaMemcpyAsync(C_val, dval, sizeof(int32_t) * cnnz, cudaMemcpyDeviceToHost, s));
    }
    GK_CUDA(cudaStreamSynchronize(s));
    return GK_OK;
}
