// C-ABI entry points of the masked SpGEMM family: gk_mxmm_masked,
// gk_tc_count, gk_tc_row_sums, gk_tc_count_batched, gk_extract_lower,
// gk_transpose.  Each stages host inputs to HBM, runs the device pipeline on
// the caller's stream and returns outputs to host or device memory.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "gk_common.cuh"
#include "gk_spgemm.cuh"

namespace gk {

// Copies `bytes` from device `src` to `dst` (host or device) on the stream;
// synchronises when dst is host memory.
static int deliver(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return GK_OK;
    if (is_device_pointer(dst)) {
        GK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
    } else {
        GK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        GK_CUDA(cudaStreamSynchronize(s));
    }
    return GK_OK;
}

// (sum >> 1) as the reference's int per vertex (src/main.cpp:27-31)
__global__ void k_half_int(int64_t m, const unsigned long long *sums, int32_t *out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] = static_cast<int32_t>(static_cast<int64_t>(sums[i]) >> 1);
}

__global__ void k_half_u64(const unsigned long long *sum, unsigned long long *half) { *half = *sum >> 1; }

static int check_square_pattern(const gk_csr *L, const char *name) {
    GK_CHECK(validate_csr_shape(L, name));
    if (L->m != L->n) return fail(GK_ERR_ARG, std::string(name) + ": matrix must be square");
    return GK_OK;
}

// A side stream for host-to-device copies that run ahead of the caller's
// stream, with one event per stage.  Released on every return path; the
// caller's stream first waits for the side stream, so that scratch freed in
// order on the caller's stream outlives every copy into it.
struct CopyPipe {
    cudaStream_t s, cs = nullptr;
    std::vector<cudaEvent_t> ev;
    explicit CopyPipe(cudaStream_t s_) : s(s_) {}
    CopyPipe(const CopyPipe &) = delete;
    CopyPipe &operator=(const CopyPipe &) = delete;
    // creates the side stream and `stages` + 1 events; the last one orders the
    // side stream after the work already queued on the caller's stream
    int open(int stages) {
        GK_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        ev.resize(static_cast<size_t>(stages) + 1, nullptr);
        for (auto &e : ev) GK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        GK_CUDA(cudaEventRecord(ev[stages], s));
        GK_CUDA(cudaStreamWaitEvent(cs, ev[stages], 0));
        return GK_OK;
    }
    // the caller's stream waits for the copies queued so far as stage q
    int stage_done(int q) {
        GK_CUDA(cudaEventRecord(ev[q], cs));
        GK_CUDA(cudaStreamWaitEvent(s, ev[q], 0));
        return GK_OK;
    }
    ~CopyPipe() {
        if (cs) {
            cudaEvent_t done;
            if (cudaEventCreateWithFlags(&done, cudaEventDisableTiming) == cudaSuccess) {
                cudaEventRecord(done, cs);
                cudaStreamWaitEvent(s, done, 0);
                cudaEventDestroy(done);
            } else {
                cudaStreamSynchronize(cs);
            }
        }
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        if (cs) cudaStreamDestroy(cs);
    }
};

static int tc_common(const gk_csr *L, int epi, unsigned long long *dev_sums, int sched, cudaStream_t s,
                     Scratch &scr, int force_variant = -1) {
    DevCsr d;
    GK_CHECK(stage_csr(L, &d, scr, s, nullptr, CSR_SORTED, "L"));
    d.val = nullptr;  // plus-pair: an adjacency pattern
    SpgemmRequest rq;
    rq.A = rq.B = rq.M = d;
    rq.epi = epi;
    rq.use_values = false;
    rq.sched = sched;
    rq.sums = dev_sums;
    rq.stream = s;
    rq.force_variant = force_variant;
    return run_spgemm(rq, scr);
}

// ---- batched graphs: block-diagonal concatenation -------------------------------
struct GraphSlot {
    const int64_t *rp;
    const int32_t *col;
    int64_t m, nnz, vbase, ebase;
};

// Graph key_base + blockIdx.x of the batch into the combined matrix (slots
// points at that graph's slot for blockIdx.x == 0).  Row pointers must run
// from 0 to nnz (spMtx's invariant, matrix.h:33-43); a pointer outside [0, nnz]
// is clamped into the graph's own entry range, so the combined matrix never
// points outside its buffers; a column outside [0, m) is replaced by 0 (the
// graph's first vertex).  Each defect is flagged in *bad for the check that
// follows.
__global__ void k_concat_graphs(const GraphSlot *slots, int key_base, int64_t *rp_out, int32_t *col_out,
                                int32_t *key_out, unsigned int *bad) {
    const GraphSlot g = slots[blockIdx.x];
    const int64_t stride = (int64_t)gridDim.y * blockDim.x;
    const int64_t start = (int64_t)blockIdx.y * blockDim.x + threadIdx.x;
    if (start == 0 && (g.rp[0] != 0 || g.rp[g.m] != g.nnz)) atomicOr(bad, CSR_BAD_ENDS);
    for (int64_t i = start; i < g.m; i += stride) {
        int64_t p = g.rp[i];
        if (p < 0 || p > g.nnz) {
            atomicOr(bad, CSR_BAD_ROWPTR);
            p = p < 0 ? 0 : g.nnz;
        }
        rp_out[g.vbase + i] = p + g.ebase;
        key_out[g.vbase + i] = key_base + static_cast<int32_t>(blockIdx.x);
    }
    for (int64_t j = start; j < g.nnz; j += stride) {
        int32_t x = g.col[j];
        if (x < 0 || x >= g.m) {  // outside the graph's own vertices
            atomicOr(bad, CSR_BAD_COL);
            x = 0;
        }
        col_out[g.ebase + j] = x + static_cast<int32_t>(g.vbase);
    }
}

__global__ void k_set_last(int64_t *rp, int64_t idx, int64_t value) { rp[idx] = value; }

// ---- CSR transforms ---------------------------------------------------------------
__global__ void k_lower_counts(DevCsr A, int64_t *cnt) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < A.m; r += warps) {
        const int64_t a0 = A.rp[r], a1 = A.rp[r + 1];
        // rows are sorted: count entries with col < r
        int64_t c = 0;
        for (int64_t t = a0 + lane; t < a1; t += 32) c += (A.col[t] < r);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
        if (lane == 0) cnt[r] = c;
    }
}

__global__ void k_lower_copy(DevCsr A, const int64_t *orp, int32_t *ocol) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < A.m; r += warps) {
        const int64_t a0 = A.rp[r], n = orp[r + 1] - orp[r], o0 = orp[r];
        for (int64_t t = lane; t < n; t += 32) ocol[o0 + t] = A.col[a0 + t];
    }
}

__global__ void k_row_ids(DevCsr A, int32_t *rows, int32_t *idx) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < A.m; r += warps)
        for (int64_t t = A.rp[r] + lane; t < A.rp[r + 1]; t += 32) {
            rows[t] = static_cast<int32_t>(r);
            idx[t] = static_cast<int32_t>(t);
        }
}

__global__ void k_col_hist(const int32_t *col, int64_t nnz, unsigned long long *cnt) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += stride)
        atomicAdd(cnt + col[j], 1ull);
}

__global__ void k_transpose_fill(int64_t nnz, const int32_t *sorted_idx, const int32_t *rows, const int32_t *val,
                                 int32_t *ocol, int32_t *oval) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += stride) {
        const int32_t src = sorted_idx[j];
        ocol[j] = rows[src];
        if (oval) oval[j] = val ? val[src] : 1;
    }
}

int transpose_device(const DevCsr &A, int64_t *orp, int32_t *ocol, int32_t *oval, cudaStream_t s, Scratch &scr) {
    const int64_t nnz = A.nnz;
    if (A.nnz >= (int64_t(1) << 31)) return fail(GK_ERR_UNSUPPORTED, "transpose: nnz must be < 2^31");
    unsigned long long *cnt;
    GK_CHECK(scr.alloc(&cnt, A.n + 1));
    GK_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * (A.n + 1), s));
    const int sms = ctx().num_sms;
    if (nnz > 0) {
        k_col_hist<<<sms * 4, 256, 0, s>>>(A.col, nnz, cnt);
        note_launches(1);
        GK_CUDA(cudaGetLastError());
    }
    size_t tb = 0;
    GK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, reinterpret_cast<int64_t *>(cnt), orp, A.n + 1, s));
    void *tmp;
    GK_CHECK(scr.alloc(reinterpret_cast<char **>(&tmp), tb));
    GK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, reinterpret_cast<int64_t *>(cnt), orp, A.n + 1, s));
    if (nnz == 0) return GK_OK;
    int32_t *rows, *idx, *keys_out, *idx_out;
    GK_CHECK(scr.alloc(&rows, nnz));
    GK_CHECK(scr.alloc(&idx, nnz));
    GK_CHECK(scr.alloc(&keys_out, nnz));
    GK_CHECK(scr.alloc(&idx_out, nnz));
    k_row_ids<<<sms * 8, 256, 0, s>>>(A, rows, idx);
    note_launches(1);
    GK_CUDA(cudaGetLastError());
    int bits = 1;
    while ((int64_t(1) << bits) < A.n) ++bits;
    size_t sb = 0;
    GK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sb, A.col, keys_out, idx, idx_out, static_cast<int>(nnz), 0,
                                            bits, s));
    void *stmp;
    GK_CHECK(scr.alloc(reinterpret_cast<char **>(&stmp), sb));
    GK_CUDA(cub::DeviceRadixSort::SortPairs(stmp, sb, A.col, keys_out, idx, idx_out, static_cast<int>(nnz), 0,
                                            bits, s));
    k_transpose_fill<<<sms * 4, 256, 0, s>>>(nnz, idx_out, rows, A.val, ocol, oval);
    note_launches(1);
    GK_CUDA(cudaGetLastError());
    return GK_OK;
}

int extract_lower_device(const DevCsr &A, int64_t *orp, int32_t *ocol, cudaStream_t s, Scratch &scr) {
    int64_t *cnt;
    GK_CHECK(scr.alloc(&cnt, A.m + 1));
    GK_CUDA(cudaMemsetAsync(cnt + A.m, 0, sizeof(int64_t), s));
    const int sms = ctx().num_sms;
    if (A.m > 0) {
        k_lower_counts<<<sms * 8, 256, 0, s>>>(A, cnt);
        note_launches(1);
        GK_CUDA(cudaGetLastError());
    }
    size_t tb = 0;
    GK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, orp, A.m + 1, s));
    void *tmp;
    GK_CHECK(scr.alloc(reinterpret_cast<char **>(&tmp), tb));
    GK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, orp, A.m + 1, s));
    if (A.m > 0) {
        k_lower_copy<<<sms * 8, 256, 0, s>>>(A, orp, ocol);
        note_launches(1);
        GK_CUDA(cudaGetLastError());
    }
    return GK_OK;
}

}  // namespace gk

using namespace gk;

extern "C" {

int gk_mxmm_masked(const gk_csr *A, const gk_csr *B, const gk_csr *M, int32_t *C_val, int semiring, int sched,
                   int accum, void *stream) {
    GK_CHECK(validate_csr_shape(A, "A"));
    GK_CHECK(validate_csr_shape(B, "B"));
    GK_CHECK(validate_csr_shape(M, "M"));
    if (semiring != GK_PLUS_TIMES && semiring != GK_PLUS_PAIR) return fail(GK_ERR_ARG, "unknown semiring");
    if (M->nnz > 0 && !C_val) return fail(GK_ERR_ARG, "C_val is null");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    SpgemmRequest rq;
    GK_CHECK(stage_csr(A, &rq.A, scr, s, nullptr, CSR_STRUCTURE, "A"));
    GK_CHECK(stage_csr(B, &rq.B, scr, s, nullptr, CSR_SORTED, "B"));
    GK_CHECK(stage_csr(M, &rq.M, scr, s, nullptr, CSR_SORTED, "M"));
    rq.M.val = nullptr;
    rq.epi = EPI_WRITE;
    rq.use_values = semiring == GK_PLUS_TIMES;
    if (!rq.use_values) rq.A.val = rq.B.val = nullptr;
    rq.sched = sched;
    rq.force_accum = accum;
    rq.stream = s;
    const bool host_out = M->nnz > 0 && !is_device_pointer(C_val);
    int32_t *dc = C_val;
    if (host_out) GK_CHECK(scr.alloc(&dc, M->nnz));
    rq.c_val = dc;
    GK_CHECK(run_spgemm(rq, scr));
    if (host_out) GK_CHECK(deliver(C_val, dc, sizeof(int32_t) * M->nnz, s));
    return GK_OK;
}

int gk_tc_count(const gk_csr *L, uint64_t *count, int sched, void *stream) {
    GK_CHECK(check_square_pattern(L, "L"));
    if (!count) return fail(GK_ERR_ARG, "count is null");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    unsigned long long *d;
    GK_CHECK(scr.alloc(&d, 1));
    GK_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), s));
    GK_CHECK(tc_common(L, EPI_SUM, d, sched, s, scr));
    return deliver(count, d, sizeof(uint64_t), s);
}

int gk_tc_count_variant(const gk_csr *L, int variant, uint64_t *count, void *stream) {
    GK_CHECK(check_square_pattern(L, "L"));
    if (!count) return fail(GK_ERR_ARG, "count is null");
    if (variant < 0 || variant >= NV) return fail(GK_ERR_ARG, "variant out of range");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    unsigned long long *d;
    GK_CHECK(scr.alloc(&d, 1));
    GK_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), s));
    GK_CHECK(tc_common(L, EPI_SUM, d, GK_SCHED_PLAIN, s, scr, variant));
    return deliver(count, d, sizeof(uint64_t), s);
}

int gk_mxmm_masked_variant(const gk_csr *A, const gk_csr *B, const gk_csr *M, int32_t *C_val, int semiring,
                           int variant, void *stream) {
    GK_CHECK(validate_csr_shape(A, "A"));
    GK_CHECK(validate_csr_shape(B, "B"));
    GK_CHECK(validate_csr_shape(M, "M"));
    if (semiring != GK_PLUS_TIMES && semiring != GK_PLUS_PAIR) return fail(GK_ERR_ARG, "unknown semiring");
    if (variant < 0 || variant >= NV) return fail(GK_ERR_ARG, "variant out of range");
    if (M->nnz > 0 && !C_val) return fail(GK_ERR_ARG, "C_val is null");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    SpgemmRequest rq;
    GK_CHECK(stage_csr(A, &rq.A, scr, s, nullptr, CSR_STRUCTURE, "A"));
    GK_CHECK(stage_csr(B, &rq.B, scr, s, nullptr, CSR_SORTED, "B"));
    GK_CHECK(stage_csr(M, &rq.M, scr, s, nullptr, CSR_SORTED, "M"));
    rq.M.val = nullptr;
    rq.epi = EPI_WRITE;
    rq.use_values = semiring == GK_PLUS_TIMES;
    if (!rq.use_values) rq.A.val = rq.B.val = nullptr;
    rq.force_variant = variant;
    rq.stream = s;
    const bool host_out = M->nnz > 0 && !is_device_pointer(C_val);
    int32_t *dc = C_val;
    if (host_out) GK_CHECK(scr.alloc(&dc, M->nnz));
    rq.c_val = dc;
    GK_CHECK(run_spgemm(rq, scr));
    if (host_out) GK_CHECK(deliver(C_val, dc, sizeof(int32_t) * M->nnz, s));
    return GK_OK;
}

int gk_tc_row_sums(const gk_csr *L, uint64_t *row_sums, int sched, void *stream) {
    GK_CHECK(check_square_pattern(L, "L"));
    if (!row_sums && L->m > 0) return fail(GK_ERR_ARG, "row_sums is null");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    unsigned long long *d;
    GK_CHECK(scr.alloc(&d, L->m + 1));
    GK_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long) * (L->m + 1), s));
    GK_CHECK(tc_common(L, EPI_KEYED, d, sched, s, scr));
    return deliver(row_sums, d, sizeof(uint64_t) * L->m, s);
}

int gk_tc_vertex(const gk_csr *A, int32_t *counts, int sched, void *stream) {
    GK_CHECK(check_square_pattern(A, "A"));
    if (!counts && A->m > 0) return fail(GK_ERR_ARG, "counts is null");
    if (A->m == 0) return GK_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    DevCsr d;
    GK_CHECK(stage_csr(A, &d, scr, s, nullptr, CSR_SORTED, "A"));
    d.val = nullptr;
    unsigned long long *sums;
    int32_t *out;
    GK_CHECK(scr.alloc(&sums, A->m + 1));
    GK_CHECK(scr.alloc(&out, A->m));
    GK_CUDA(cudaMemsetAsync(sums, 0, sizeof(unsigned long long) * (A->m + 1), s));
    SpgemmRequest rq;
    rq.A = rq.B = rq.M = d;
    rq.epi = EPI_KEYED;  // row sums of C<A> = A·A
    rq.sched = sched;
    rq.sums = sums;
    rq.stream = s;
    GK_CHECK(run_spgemm(rq, scr));
    k_half_int<<<ceil_div(A->m, 256), 256, 0, s>>>(A->m, sums, out);
    note_launches(1);
    GK_CUDA(cudaGetLastError());
    return deliver(counts, out, sizeof(int32_t) * A->m, s);
}

int gk_tc_count_lu(const gk_csr *A, uint64_t *count, int sched, void *stream) {
    GK_CHECK(check_square_pattern(A, "A"));
    if (!count) return fail(GK_ERR_ARG, "count is null");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    DevCsr d;
    GK_CHECK(stage_csr(A, &d, scr, s, nullptr, CSR_SORTED, "A"));
    d.val = nullptr;
    const int64_t m = A->m;
    int64_t *lrp, *urp;
    int32_t *lcol, *ucol;
    GK_CHECK(scr.alloc(&lrp, m + 1));
    GK_CHECK(scr.alloc(&lcol, d.nnz > 0 ? d.nnz : 1));
    GK_CHECK(extract_lower_device(d, lrp, lcol, s, scr));
    int64_t lnnz = 0;
    GK_CUDA(cudaMemcpyAsync(&lnnz, lrp + m, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaStreamSynchronize(s));
    DevCsr L{m, m, lnnz, lrp, lcol, nullptr};
    GK_CHECK(scr.alloc(&urp, m + 1));
    GK_CHECK(scr.alloc(&ucol, lnnz > 0 ? lnnz : 1));
    GK_CHECK(transpose_device(L, urp, ucol, nullptr, s, scr));
    unsigned long long *sum, *half;
    GK_CHECK(scr.alloc(&sum, 2));
    half = sum + 1;
    GK_CUDA(cudaMemsetAsync(sum, 0, 2 * sizeof(unsigned long long), s));
    SpgemmRequest rq;
    rq.A = L;
    rq.B = DevCsr{m, m, lnnz, urp, ucol, nullptr};
    rq.M = d;
    rq.epi = EPI_SUM;
    rq.sched = sched;
    rq.sums = sum;
    rq.stream = s;
    GK_CHECK(run_spgemm(rq, scr));
    k_half_u64<<<1, 1, 0, s>>>(sum, half);
    note_launches(1);
    GK_CUDA(cudaGetLastError());
    return deliver(count, half, sizeof(uint64_t), s);
}

int gk_tc_count_batched(const gk_csr *graphs, int ngraphs, uint64_t *counts, int sched, void *stream) {
    NvtxRange range("gk:tc_count_batched");
    if (ngraphs < 0 || (ngraphs > 0 && (!graphs || !counts))) return fail(GK_ERR_ARG, "bad batch arguments");
    if (ngraphs == 0) return GK_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    std::vector<GraphSlot> slots(ngraphs);
    int64_t vtot = 0, etot = 0;
    bool any_host = false;
    for (int g = 0; g < ngraphs; ++g) {
        GK_CHECK(check_square_pattern(&graphs[g], "graphs[g]"));
        slots[g].m = graphs[g].m;
        slots[g].nnz = graphs[g].nnz;
        slots[g].vbase = vtot;
        slots[g].ebase = etot;
        vtot += graphs[g].m;
        etot += graphs[g].nnz;
        if (graphs[g].m > 0 && !is_device_pointer(graphs[g].rowptr)) any_host = true;
    }
    if (vtot >= (int64_t(1) << 31)) return fail(GK_ERR_UNSUPPORTED, "batched graphs exceed 2^31 vertices in total");
    int64_t *rp;
    int32_t *col, *key;
    GK_CHECK(scr.alloc(&rp, vtot + 1));
    GK_CHECK(scr.alloc(&col, etot > 0 ? etot : 1));
    GK_CHECK(scr.alloc(&key, vtot > 0 ? vtot : 1));
    unsigned long long *d;
    GK_CHECK(scr.alloc(&d, ngraphs));
    GK_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long) * ngraphs, s));
    int64_t *rp_raw = nullptr;
    if (any_host) {
        // host graphs are staged raw into the combined buffers (columns at their
        // final positions, offset in place by k_concat_graphs)
        GK_CHECK(scr.alloc(&rp_raw, vtot + ngraphs));
        int64_t roff = 0;
        for (int g = 0; g < ngraphs; ++g) {
            slots[g].rp = rp_raw + roff;
            slots[g].col = col + slots[g].ebase;
            roff += graphs[g].m + 1;
        }
    } else {
        for (int g = 0; g < ngraphs; ++g) {
            slots[g].rp = graphs[g].rowptr;
            slots[g].col = graphs[g].col;
        }
    }
    GraphSlot *dslots;
    GK_CHECK(scr.alloc(&dslots, ngraphs));
    GK_CUDA(cudaMemcpyAsync(dslots, slots.data(), sizeof(GraphSlot) * ngraphs, cudaMemcpyHostToDevice, s));
    // per-graph entry ranges for the content check, and its flags
    std::vector<int64_t> ranges(static_cast<size_t>(ngraphs) + 1);
    for (int g = 0; g < ngraphs; ++g) ranges[g] = slots[g].ebase;
    ranges[ngraphs] = etot;
    int64_t *dranges;
    unsigned int *bad;
    GK_CHECK(scr.alloc(&dranges, ranges.size()));
    GK_CHECK(scr.alloc(&bad, 1));
    GK_CUDA(cudaMemcpyAsync(dranges, ranges.data(), sizeof(int64_t) * ranges.size(), cudaMemcpyHostToDevice, s));
    GK_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned int), s));

    // Groups of consecutive graphs.  With host inputs the copies of group q+1
    // run on a side stream while group q is counted (the graphs are
    // independent, so a group needs only its own rows); device inputs form one
    // group.  A group holds about etot/8 entries, at least GK_BATCH_STAGE_MIN
    // (default 2^24, whose copy takes ~1 ms).  All copies are queued at once,
    // so they run back to back while the counts follow them group by group.
    // (Groups that double in size, which expose only a small first copy, were
    // slower on the uneven 4,096-graph batch: its compute-light Erdos-Renyi
    // half comes first and cannot hide the copies of the large groups.)
    std::vector<int> gstart{0};
    if (any_host) {
        int64_t min_entries = int64_t(1) << 24;
        if (const char *e = getenv("GK_BATCH_STAGE_MIN")) min_entries = std::max<int64_t>(1, atoll(e));
        const int64_t target = std::max<int64_t>(etot / 8, min_entries);
        int64_t acc = 0;
        for (int g = 0; g + 1 < ngraphs; ++g) {
            acc += graphs[g].nnz;
            if (acc >= target) {
                gstart.push_back(g + 1);
                acc = 0;
            }
        }
    }
    gstart.push_back(ngraphs);
    const int ngroups = static_cast<int>(gstart.size()) - 1;

    CopyPipe pipe(s);
    cudaStream_t cs = s;
    if (any_host && ngroups > 1) {
        GK_CHECK(pipe.open(ngroups));  // after the buffers' allocation and the sums' zeroing
        cs = pipe.cs;
    }
    for (int q = 0; q < ngroups; ++q) {
        const int g0 = gstart[q], g1 = gstart[q + 1];
        if (any_host) {
            for (int g = g0; g < g1; ++g) {
                GK_CUDA(cudaMemcpyAsync(const_cast<int64_t *>(slots[g].rp), graphs[g].rowptr,
                                        sizeof(int64_t) * (graphs[g].m + 1), cudaMemcpyDefault, cs));
                if (graphs[g].nnz)
                    GK_CUDA(cudaMemcpyAsync(col + slots[g].ebase, graphs[g].col, sizeof(int32_t) * graphs[g].nnz,
                                            cudaMemcpyDefault, cs));
            }
            if (cs != s) GK_CHECK(pipe.stage_done(q));
        }
        const int64_t v0 = slots[g0].vbase, e0 = slots[g0].ebase;
        const int64_t v1 = g1 < ngraphs ? slots[g1].vbase : vtot, e1 = g1 < ngraphs ? slots[g1].ebase : etot;
        dim3 grid(g1 - g0, 8);
        k_concat_graphs<<<grid, 256, 0, s>>>(dslots + g0, g0, rp, col, key, bad);
        k_set_last<<<1, 1, 0, s>>>(rp, v1, e1);  // the group's end (the next group writes the same value)
        note_launches(2);
        GK_CUDA(cudaGetLastError());
        // rows [v0, v1) against the whole combined matrix: their columns lie in
        // [v0, v1), so only this group's B rows are read
        DevCsr rows{v1 - v0, vtot, e1 - e0, rp + v0, col, nullptr};
        DevCsr all{vtot, vtot, etot, rp, col, nullptr};
        SpgemmRequest rq;
        rq.A = rq.M = rows;
        rq.B = all;
        rq.epi = EPI_KEYED;
        rq.row_key = key + v0;
        rq.sums = d;
        rq.sched = sched;
        rq.stream = s;
        Scratch gs(s);  // the group's plan, freed in stream order before the next group's
        GK_CHECK(check_csr_batch(rows, e0, v0, key, dranges, bad, CSR_SORTED, "graphs", s, gs));
        GK_CHECK(run_spgemm(rq, gs));
    }
    return deliver(counts, d, sizeof(uint64_t) * ngraphs, s);
}

int gk_extract_lower(const gk_csr *A, int64_t *out_rowptr, int32_t *out_col, int64_t *out_nnz, void *stream) {
    GK_CHECK(check_square_pattern(A, "A"));
    if (!out_rowptr || !out_nnz || (A->nnz > 0 && !out_col)) return fail(GK_ERR_ARG, "null output");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    DevCsr d;
    GK_CHECK(stage_csr(A, &d, scr, s, nullptr, CSR_SORTED, "A"));
    const bool host_out = !is_device_pointer(out_rowptr);
    int64_t *orp = out_rowptr;
    int32_t *ocol = out_col;
    if (host_out) {
        GK_CHECK(scr.alloc(&orp, A->m + 1));
        GK_CHECK(scr.alloc(&ocol, A->nnz > 0 ? A->nnz : 1));
    }
    GK_CHECK(extract_lower_device(d, orp, ocol, s, scr));
    int64_t nnz = 0;
    GK_CUDA(cudaMemcpyAsync(&nnz, orp + A->m, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaStreamSynchronize(s));
    *out_nnz = nnz;
    if (host_out) {
        GK_CHECK(deliver(out_rowptr, orp, sizeof(int64_t) * (A->m + 1), s));
        GK_CHECK(deliver(out_col, ocol, sizeof(int32_t) * nnz, s));
    }
    return GK_OK;
}

int gk_transpose(const gk_csr *A, int64_t *out_rowptr, int32_t *out_col, int32_t *out_val, void *stream) {
    GK_CHECK(validate_csr_shape(A, "A"));
    if (!out_rowptr || (A->nnz > 0 && !out_col)) return fail(GK_ERR_ARG, "null output");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    DevCsr d;
    GK_CHECK(stage_csr(A, &d, scr, s, nullptr, CSR_STRUCTURE, "A"));
    const bool host_out = !is_device_pointer(out_rowptr);
    int64_t *orp = out_rowptr;
    int32_t *ocol = out_col, *oval = out_val;
    if (host_out) {
        GK_CHECK(scr.alloc(&orp, A->n + 1));
        GK_CHECK(scr.alloc(&ocol, A->nnz > 0 ? A->nnz : 1));
        if (out_val) GK_CHECK(scr.alloc(&oval, A->nnz > 0 ? A->nnz : 1));
    }
    GK_CHECK(transpose_device(d, orp, ocol, oval, s, scr));
    if (host_out) {
        GK_CHECK(deliver(out_rowptr, orp, sizeof(int64_t) * (A->n + 1), s));
        GK_CHECK(deliver(out_col, ocol, sizeof(int32_t) * A->nnz, s));
        if (out_val) GK_CHECK(deliver(out_val, oval, sizeof(int32_t) * A->nnz, s));
    }
    GK_CUDA(cudaStreamSynchronize(s));
    return GK_OK;
}

}  // extern "C"
