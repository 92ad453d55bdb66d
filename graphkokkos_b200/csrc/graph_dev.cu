// Device graph ingest: seeded RMAT / Erdos-Renyi generation and CSR
// construction on the GPU — symmetrise, drop self-loops, deduplicate and sort
// rows — producing exactly the CSR of the host builder (graph_host.cpp).
//
// Reference counterparts: the .rmat edge-list reader (include/matrix.h:488-533)
// plus build_symm_from_lower / extract_lower_triangle (include/matrix.h:662-726)
// which the reference runs serially before its algorithms (src/main.cpp:215).
//
// Pipeline: every edge (u,v) becomes the two keys u<<b|v and v<<b|u
// (b = bits per vertex id; self-loops become the all-ones sentinel), one
// radix sort orders them row-major, a flag/scan pass drops duplicates and
// sentinels, and row pointers are found by binary search in the unique keys.
#include <cub/cub.cuh>

#include "gk_common.cuh"
#include "gk_gen.h"

namespace gk {

struct GenParams {
    int kind;  // 0 RMAT, 1 ER
    int scale;
    uint32_t ta, tab, tabc;
    uint64_t key;
    uint64_t n;  // vertices
    uint64_t nedges;
    int bits;    // bits per vertex id
};

__global__ void k_gen_keys(GenParams g, uint64_t *keys) {
    const uint64_t sentinel = (g.bits * 2 >= 64) ? ~0ull : ((1ull << (2 * g.bits)) - 1);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < g.nedges; e += stride) {
        uint32_t u, v;
        if (g.kind == 0) gk_rmat_edge(g.key, e, g.scale, g.ta, g.tab, g.tabc, &u, &v);
        else gk_er_edge(g.key, e, g.n, &u, &v);
        if (u == v) {
            keys[2 * e] = sentinel;
            keys[2 * e + 1] = sentinel;
        } else {
            keys[2 * e] = (static_cast<uint64_t>(u) << g.bits) | v;
            keys[2 * e + 1] = (static_cast<uint64_t>(v) << g.bits) | u;
        }
    }
}

__global__ void k_flag_unique(const uint64_t *k, int64_t n, uint64_t sentinel, int32_t *flag) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        flag[i] = (k[i] != sentinel) && (i == 0 || k[i] != k[i - 1]);
}

__global__ void k_compact_keys(const uint64_t *k, int64_t n, const int32_t *flag, const int64_t *pos,
                               uint64_t *ukeys) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        if (flag[i]) ukeys[pos[i]] = k[i];
}

__global__ void k_keys_to_csr(const uint64_t *ukeys, int64_t nnz, int64_t m, int bits, int64_t *rp, int32_t *col) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const uint64_t mask = (1ull << bits) - 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += stride)
        col[i] = static_cast<int32_t>(ukeys[i] & mask);
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= m; r += stride) {
        const uint64_t target = static_cast<uint64_t>(r) << bits;
        int64_t lo = 0, hi = nnz;
        while (lo < hi) {
            const int64_t md = (lo + hi) >> 1;
            if (ukeys[md] < target) lo = md + 1;
            else hi = md;
        }
        rp[r] = lo;
    }
}

// Builds the graph; if rowptr is null only *nnz is produced.
static int build_graph(const GenParams &gp, int64_t *nnz_out, int64_t *rowptr, int32_t *col, cudaStream_t s) {
    Scratch scr(s);
    const int64_t nk = static_cast<int64_t>(gp.nedges) * 2;
    const int64_t m = static_cast<int64_t>(gp.n);
    const int sms = ctx().num_sms;
    uint64_t *k0, *k1;
    GK_CHECK(scr.alloc(&k0, nk > 0 ? nk : 1));
    GK_CHECK(scr.alloc(&k1, nk > 0 ? nk : 1));
    if (nk > 0) {
        k_gen_keys<<<sms * 16, 256, 0, s>>>(gp, k0);
        note_launches(1);
        GK_CUDA(cudaGetLastError());
    }
    cub::DoubleBuffer<uint64_t> db(k0, k1);
    const int end_bit = 2 * gp.bits;
    if (nk > 0) {
        size_t tb = 0;
        GK_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, db, nk, 0, end_bit, s));
        void *tmp;
        GK_CHECK(scr.alloc(reinterpret_cast<char **>(&tmp), tb));
        GK_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tb, db, nk, 0, end_bit, s));
    }
    const uint64_t *sorted = db.Current();
    uint64_t *ukeys = db.Alternate();
    int32_t *flag;
    int64_t *pos;
    GK_CHECK(scr.alloc(&flag, nk + 1));
    GK_CHECK(scr.alloc(&pos, nk + 1));
    GK_CUDA(cudaMemsetAsync(flag + nk, 0, sizeof(int32_t), s));
    const uint64_t sentinel = (end_bit >= 64) ? ~0ull : ((1ull << end_bit) - 1);
    if (nk > 0) {
        k_flag_unique<<<sms * 8, 256, 0, s>>>(sorted, nk, sentinel, flag);
        note_launches(1);
        GK_CUDA(cudaGetLastError());
    }
    size_t tb2 = 0;
    GK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb2, flag, pos, nk + 1, s));
    void *tmp2;
    GK_CHECK(scr.alloc(reinterpret_cast<char **>(&tmp2), tb2));
    GK_CUDA(cub::DeviceScan::ExclusiveSum(tmp2, tb2, flag, pos, nk + 1, s));
    int64_t nnz = 0;
    GK_CUDA(cudaMemcpyAsync(&nnz, pos + nk, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaStreamSynchronize(s));
    *nnz_out = nnz;
    if (!rowptr) return GK_OK;
    if (nk > 0) {
        k_compact_keys<<<sms * 8, 256, 0, s>>>(sorted, nk, flag, pos, ukeys);
        note_launches(1);
        GK_CUDA(cudaGetLastError());
    }
    const bool host_out = !is_device_pointer(rowptr);
    int64_t *drp = rowptr;
    int32_t *dcol = col;
    if (host_out) {
        GK_CHECK(scr.alloc(&drp, m + 1));
        GK_CHECK(scr.alloc(&dcol, nnz > 0 ? nnz : 1));
    }
    k_keys_to_csr<<<sms * 8, 256, 0, s>>>(ukeys, nnz, m, gp.bits, drp, dcol);
    note_launches(1);
    GK_CUDA(cudaGetLastError());
    if (host_out) {
        GK_CUDA(cudaMemcpyAsync(rowptr, drp, sizeof(int64_t) * (m + 1), cudaMemcpyDeviceToHost, s));
        if (nnz) GK_CUDA(cudaMemcpyAsync(col, dcol, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, s));
    }
    GK_CUDA(cudaStreamSynchronize(s));
    return GK_OK;
}

}  // namespace gk

extern "C" {

int gk_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int64_t *nnz,
                int64_t *rowptr, int32_t *col, void *stream) {
    if (scale < 1 || scale > 30 || edge_factor < 1 || !nnz) return gk::fail(GK_ERR_ARG, "gk_gen_rmat: bad arguments");
    if (rowptr && !col) return gk::fail(GK_ERR_ARG, "gk_gen_rmat: col is null");
    gk::GenParams gp{};
    gp.kind = 0;
    gp.scale = scale;
    gk_rmat_thresholds(a, b, c, &gp.ta, &gp.tab, &gp.tabc);
    gp.key = gk_seed_key(seed);
    gp.n = uint64_t(1) << scale;
    gp.nedges = static_cast<uint64_t>(edge_factor) << scale;
    gp.bits = scale;
    return gk::build_graph(gp, nnz, rowptr, col, static_cast<cudaStream_t>(stream));
}

int gk_gen_er(int64_t n, int64_t nedges, uint64_t seed, int64_t *nnz, int64_t *rowptr, int32_t *col, void *stream) {
    if (n < 1 || n >= (int64_t(1) << 31) || nedges < 0 || !nnz) return gk::fail(GK_ERR_ARG, "gk_gen_er: bad arguments");
    if (rowptr && !col) return gk::fail(GK_ERR_ARG, "gk_gen_er: col is null");
    gk::GenParams gp{};
    gp.kind = 1;
    gp.key = gk_seed_key(seed);
    gp.n = static_cast<uint64_t>(n);
    gp.nedges = static_cast<uint64_t>(nedges);
    int bits = 1;
    while ((int64_t(1) << bits) < n) ++bits;
    gp.bits = bits;
    return gk::build_graph(gp, nnz, rowptr, col, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
