// k-truss on the GPU: gk_ktruss.
//
// Reference: k_truss (src/main.cpp:94-141): repeat Tmp<C> = C·C, drop the
// entries with support < k-2 (keeping the others with value 1), until nnz
// stops changing, at most n passes.  The reference compacts serially on the
// host (:110-119); here one pass is
//   1. support  S<C> = C·C (plus-pair) with the masked SpGEMM engine (EPI_WRITE);
//               for a symmetric C only its lower triangle is computed (below)
//   2. flag     keep[j] = S[j] >= k-2
//   3. scan     exclusive prefix of keep over all entries (one device scan)
//   4. compact  new_rp[i] = pos[rp[i]], new_col[pos[j]] = col[j] for kept j
//   5. copy the pruned matrix back over the current one
// and the loop stops when the kept count equals nnz.  Compaction preserves the
// order within rows, so rows stay sorted and the edge set is bit-exact with the
// reference (whose View-size defect at :99/:118 is not reproduced).
// Every pass reads its sizes on the device, so the loop is one CUDA graph: a
// conditional while node around one captured pass, the condition set by the
// pass's last kernel; the host waits once, at the end.  With profiling on
// (its events cannot be captured) the host runs the passes itself.
#include <cub/cub.cuh>

#include "gk_common.cuh"
#include "gk_spgemm.cuh"

namespace gk {

// Loop state in device memory, so that a pass needs no host value.
struct KtState {
    long long iters;   // passes run
    long long kept;    // nnz after the last pass
};

// keep[j] = S[j] >= k-2 for j < nnz (nnz = rp[m]); 0 up to the capacity, so
// that a scan over capacity+1 entries yields the kept count at pos[cap].
__global__ void k_keep_flags(const int32_t *sup, const int64_t *rp, int64_t m, int64_t cap, int thresh,
                             int32_t *keep) {
    const int64_t nnz = rp[m];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j <= cap; j += stride)
        keep[j] = j < nnz ? (sup[j] >= thresh) : 0;
}

__global__ void k_compact(int64_t m, const int64_t *rp, const int32_t *col, const int32_t *keep, const int64_t *pos,
                          int64_t *nrp, int32_t *ncol) {
    const int64_t nnz = rp[m];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += stride)
        if (keep[j]) ncol[pos[j]] = col[j];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= m; i += stride) nrp[i] = pos[rp[i]];
}

// End of a pass: count it and decide whether another pass follows (the edge
// count changed and fewer than max_iters passes ran).  Inside the graph the
// decision drives the conditional while node.
__global__ void k_pass_end(const int64_t *rp, const int64_t *nrp, int64_t m, long long max_iters, KtState *st,
                           cudaGraphConditionalHandle h, int in_graph) {
    const long long old = rp[m], kept = nrp[m];
    const long long it = st->iters + 1;
    st->iters = it;
    st->kept = kept;
    if (in_graph) cudaGraphSetConditional(h, (kept != old && it < max_iters) ? 1u : 0u);
}

// The pruned matrix becomes the current one.
__global__ void k_copy_back(int64_t m, const int64_t *nrp, const int32_t *ncol, int64_t *rp, int32_t *col) {
    const int64_t nnz = nrp[m];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= m; i += stride) rp[i] = nrp[i];
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += stride) col[j] = ncol[j];
}

// ---- symmetric input: support on the lower triangle only -------------------
// For a symmetric C, S = C·C is symmetric (S_ij = |N(i) ∩ N(j)| = S_ji), so the
// pass computes S<L> = C·C with L the strict lower triangle of C and reads the
// support of an upper entry (i, j > i) at its mirror (j, i) in L.  The B rows
// streamed for row i then stop at row i's largest lower column (the engine
// ends a B row past the mask's last column), which roughly halves the streamed
// entries.  The values are the same integers, so the truss is unchanged.

// Row index of every entry (warp per row, coalesced stores).  The per-entry
// kernels below then spread their work over entries, not rows: with a warp per
// row, a hub row of 10^5 entries is one warp's serial loop of binary searches
// and sets the kernel's duration.
__global__ void k_row_of(int64_t m, const int64_t *rp, int32_t *row) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < m; i += warps)
        for (int64_t p = rp[i] + lane; p < rp[i + 1]; p += 32) row[p] = static_cast<int32_t>(i);
}

// Whether every entry (i, j) has its mirror (j, i): a thread per entry, a
// binary search in row j.
__global__ void k_sym_check(int64_t m, const int64_t *rp, const int32_t *col, const int32_t *row, int *asym) {
    const int64_t nnz = rp[m];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += stride) {
        const int i = row[p], j = col[p];
        int64_t lo = rp[j], hi = rp[j + 1];
        const int64_t end = hi;
        while (lo < hi) {
            const int64_t md = (lo + hi) >> 1;
            if (col[md] < i) lo = md + 1;
            else hi = md;
        }
        if (lo == end || col[lo] != i) atomicExch(asym, 1);
    }
}

// Entries of row i below the diagonal (a prefix of the sorted row).
__global__ void k_lower_len(int64_t m, const int64_t *rp, const int32_t *col, int64_t *len) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        int64_t lo = rp[i], hi = rp[i + 1];
        while (lo < hi) {
            const int64_t md = (lo + hi) >> 1;
            if (col[md] < i) lo = md + 1;
            else hi = md;
        }
        len[i] = lo - rp[i];
    }
}

// Lower-triangle columns, a thread per entry of C (balanced over entries).
__global__ void k_lower_fill(int64_t m, const int64_t *rp, const int32_t *col, const int32_t *row,
                             const int64_t *lrp, int32_t *lcol) {
    const int64_t nnz = rp[m];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += stride) {
        const int i = row[p], j = col[p];
        const int64_t off = p - rp[i];  // below llen[i] for every j < i of a sorted row
        if (j < i && off < lrp[i + 1] - lrp[i]) lcol[lrp[i] + off] = j;
    }
}

// keep[p] for every entry of C from the lower supports, a thread per entry: a
// lower entry reads its own position in L, an upper entry (i, j) the position
// of i in L's row j (binary search).
__global__ void k_keep_sym(int64_t m, int64_t cap, const int64_t *rp, const int32_t *col, const int32_t *row,
                           const int64_t *lrp, const int32_t *lcol, const int32_t *sup, int thresh, int32_t *keep) {
    const int64_t nnz = rp[m];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += stride) {
        const int i = row[p], j = col[p];
        int64_t q;
        if (j < i) {
            q = lrp[i] + (p - rp[i]);
        } else {
            int64_t lo = lrp[j], hi = lrp[j + 1];
            const int64_t end = hi;
            while (lo < hi) {
                const int64_t md = (lo + hi) >> 1;
                if (lcol[md] < i) lo = md + 1;
                else hi = md;
            }
            q = (lo < end && lcol[lo] == i) ? lo : -1;
        }
        keep[p] = (q >= 0 && sup[q] >= thresh) ? 1 : 0;
    }
    for (int64_t p = nnz + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p <= cap; p += stride) keep[p] = 0;
}

struct KtBuffers {
    int64_t m, cap;            // rows, nnz of the input (capacity of every edge array)
    int64_t *rp, *nrp;         // current / pruned row pointers
    int32_t *col, *ncol;       // current / pruned columns
    int32_t *sup, *keep;       // support per entry, keep flags (cap + 1)
    int64_t *pos;              // exclusive scan of keep (cap + 1)
    void *scan_tmp;
    size_t scan_bytes;
    void *arena;               // scratch of the support SpGEMM
    size_t arena_bytes;
    KtState *st;
    int k, sched;
    bool sym;                  // symmetric input: support on the lower triangle
    int64_t *llen, *lrp;       // lower-triangle lengths (m + 1) and row pointers (m + 1)
    int32_t *lcol;             // lower-triangle columns
    int32_t *row;              // row index of every entry of the current matrix
};

// One pass: support S<C> = C·C, flags, scan, compaction, pass end, copy back.
// Every size is read on the device, so the same launches serve every pass.
static int ktruss_pass(const KtBuffers &b, cudaStream_t s, cudaGraphConditionalHandle h, bool in_graph) {
    const int sms = ctx().num_sms;
    Scratch pass(s, b.arena, b.arena_bytes);
    SpgemmRequest rq;
    DevCsr c{b.m, b.m, b.cap, b.rp, b.col, nullptr};
    rq.A = rq.B = rq.M = c;
    rq.epi = EPI_WRITE;
    rq.sched = b.sched;
    rq.c_val = b.sup;
    rq.stream = s;
    size_t scan_bytes = b.scan_bytes;
    if (b.sym) {
        k_row_of<<<sms * 8, 256, 0, s>>>(b.m, b.rp, b.row);
        k_lower_len<<<sms * 4, 256, 0, s>>>(b.m, b.rp, b.col, b.llen);
        GK_CUDA(cub::DeviceScan::ExclusiveSum(b.scan_tmp, scan_bytes, b.llen, b.lrp, b.m + 1, s));
        k_lower_fill<<<sms * 8, 256, 0, s>>>(b.m, b.rp, b.col, b.row, b.lrp, b.lcol);
        rq.M = DevCsr{b.m, b.m, b.cap, b.lrp, b.lcol, nullptr};
        GK_CHECK(run_spgemm(rq, pass));
        k_keep_sym<<<sms * 8, 256, 0, s>>>(b.m, b.cap, b.rp, b.col, b.row, b.lrp, b.lcol, b.sup, b.k - 2, b.keep);
        note_launches(4);
    } else {
        GK_CHECK(run_spgemm(rq, pass));
        k_keep_flags<<<sms * 8, 256, 0, s>>>(b.sup, b.rp, b.m, b.cap, b.k - 2, b.keep);
        note_launches(1);
    }
    scan_bytes = b.scan_bytes;
    GK_CUDA(cub::DeviceScan::ExclusiveSum(b.scan_tmp, scan_bytes, b.keep, b.pos, b.cap + 1, s));
    k_compact<<<sms * 8, 256, 0, s>>>(b.m, b.rp, b.col, b.keep, b.pos, b.nrp, b.ncol);
    k_pass_end<<<1, 1, 0, s>>>(b.rp, b.nrp, b.m, static_cast<long long>(b.m), b.st, h, in_graph ? 1 : 0);
    k_copy_back<<<sms * 8, 256, 0, s>>>(b.m, b.nrp, b.ncol, b.rp, b.col);
    note_launches(5);
    GK_CUDA(cudaGetLastError());
    return GK_OK;
}

// The whole loop as one CUDA graph: a conditional while node whose body is
// one pass, captured once.  Returns GK_ERR_UNSUPPORTED where the graph cannot
// be built (the caller then runs the passes from the host).
static int ktruss_graph(const KtBuffers &b, cudaStream_t s, int *passes_per_launch) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cs = nullptr;
    int status = GK_OK;
    do {
        if (cudaGraphCreate(&g, 0) != cudaSuccess) { status = GK_ERR_UNSUPPORTED; break; }
        cudaGraphConditionalHandle h;
        if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
            status = GK_ERR_UNSUPPORTED;
            break;
        }
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        if (cudaGraphAddNode(&node, g, nullptr, 0, &np) != cudaSuccess) { status = GK_ERR_UNSUPPORTED; break; }
        cudaGraph_t body = np.conditional.phGraph_out[0];
        if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) { status = GK_ERR_UNSUPPORTED; break; }
        if (cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
            cudaSuccess) {
            status = GK_ERR_UNSUPPORTED;
            break;
        }
        const int64_t before = launches_noted();
        const int ps = ktruss_pass(b, cs, h, true);
        *passes_per_launch = static_cast<int>(launches_noted() - before);
        cudaGraph_t captured = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(cs, &captured);
        if (ps != GK_OK) { status = ps; break; }
        if (ce != cudaSuccess) { status = cuda_fail(ce, "k-truss pass capture"); break; }
        if (cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) {
            cudaGetLastError();
            status = GK_ERR_UNSUPPORTED;
            break;
        }
        const cudaError_t le = cudaGraphLaunch(exec, s);
        if (le != cudaSuccess) status = cuda_fail(le, "k-truss graph launch");
    } while (false);
    if (exec) cudaGraphExecDestroy(exec);
    if (g) cudaGraphDestroy(g);
    if (cs) cudaStreamDestroy(cs);
    return status;
}

int ktruss_device(int64_t m, int64_t nnz0, int64_t *rp_a, int32_t *col_a, int k, int sched, int *iters_out,
                  int64_t *nnz_out, int64_t **rp_res, int32_t **col_res, cudaStream_t s, Scratch &scr) {
    NvtxRange range("gk:ktruss");
    *rp_res = rp_a;
    *col_res = col_a;
    if (nnz0 == 0 || m == 0) {  // the reference counts one pass over the empty matrix
        *iters_out = m > 0 ? 1 : 0;
        *nnz_out = 0;
        return GK_OK;
    }
    KtBuffers b;
    b.m = m;
    b.cap = nnz0;
    b.rp = rp_a;
    b.col = col_a;
    b.k = k;
    b.sched = sched;
    GK_CHECK(scr.alloc(&b.nrp, m + 1));
    GK_CHECK(scr.alloc(&b.ncol, nnz0));
    GK_CHECK(scr.alloc(&b.sup, nnz0));
    GK_CHECK(scr.alloc(&b.keep, nnz0 + 1));
    GK_CHECK(scr.alloc(&b.pos, nnz0 + 1));
    GK_CHECK(scr.alloc(&b.st, 1));
    GK_CHECK(scr.alloc(&b.llen, m + 1));
    GK_CHECK(scr.alloc(&b.lrp, m + 1));
    GK_CHECK(scr.alloc(&b.lcol, nnz0));
    GK_CHECK(scr.alloc(&b.row, nnz0));
    GK_CUDA(cudaMemsetAsync(b.llen + m, 0, sizeof(int64_t), s));
    {
        int *asym;
        GK_CHECK(scr.alloc(&asym, 1));
        GK_CUDA(cudaMemsetAsync(asym, 0, sizeof(int), s));
        k_row_of<<<ctx().num_sms * 8, 256, 0, s>>>(m, rp_a, b.row);
        k_sym_check<<<ctx().num_sms * 8, 256, 0, s>>>(m, rp_a, col_a, b.row, asym);
        note_launches(2);
        int h = 1;
        GK_CUDA(cudaMemcpyAsync(&h, asym, sizeof(int), cudaMemcpyDeviceToHost, s));
        GK_CUDA(cudaStreamSynchronize(s));
        b.sym = h == 0;
    }
    b.scan_bytes = 0;
    GK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b.scan_bytes, b.keep, b.pos, nnz0 + 1, s));
    {
        size_t lb = 0;
        GK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, lb, b.llen, b.lrp, m + 1, s));
        if (lb > b.scan_bytes) b.scan_bytes = lb;
    }
    GK_CHECK(scr.alloc(reinterpret_cast<char **>(&b.scan_tmp), b.scan_bytes));
    b.arena_bytes = spgemm_scratch_bytes(m);
    GK_CHECK(scr.alloc(reinterpret_cast<char **>(&b.arena), b.arena_bytes));
    GK_CUDA(cudaMemsetAsync(b.st, 0, sizeof(KtState), s));
    GK_CHECK(spgemm_prepare(EPI_WRITE, false, sched, GK_ACCUM_AUTO));

    int status = GK_ERR_UNSUPPORTED;
    int per_pass = 0;
    if (!prof_any()) status = ktruss_graph(b, s, &per_pass);
    KtState h{};
    if (status == GK_OK) {
        GK_CUDA(cudaMemcpyAsync(&h, b.st, sizeof(KtState), cudaMemcpyDeviceToHost, s));
        GK_CUDA(cudaStreamSynchronize(s));
        note_launches(static_cast<int>(per_pass * (h.iters - 1)));  // replays beyond the captured pass
    } else if (status == GK_ERR_UNSUPPORTED) {
        // passes driven from the host (profiling on, or no conditional graphs)
        long long prev = nnz0;
        for (int64_t t = 0; t < m; ++t) {
            GK_CHECK(ktruss_pass(b, s, cudaGraphConditionalHandle{}, false));
            GK_CUDA(cudaMemcpyAsync(&h, b.st, sizeof(KtState), cudaMemcpyDeviceToHost, s));
            GK_CUDA(cudaStreamSynchronize(s));
            if (h.kept == prev) break;
            prev = h.kept;
        }
    } else {
        return status;
    }
    *iters_out = static_cast<int>(h.iters);
    *nnz_out = h.kept;
    return GK_OK;
}

}  // namespace gk

using namespace gk;

extern "C" int gk_ktruss(gk_csr_mut *inout, int k, int *iters, int sched, void *stream) {
    if (!inout || !iters) return fail(GK_ERR_ARG, "gk_ktruss: null argument");
    if (k < 3) return fail(GK_ERR_ARG, "gk_ktruss: k must be >= 3");
    if (inout->m != inout->n) return fail(GK_ERR_ARG, "gk_ktruss: matrix must be square");
    if (inout->m < 0 || inout->nnz < 0 || !inout->rowptr || (inout->nnz > 0 && !inout->col))
        return fail(GK_ERR_ARG, "gk_ktruss: bad matrix");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    const int64_t m = inout->m, nnz0 = inout->nnz;
    const bool dev = is_device_pointer(inout->rowptr);
    int64_t *rp;
    int32_t *col;
    GK_CHECK(scr.alloc(&rp, m + 1));
    GK_CHECK(scr.alloc(&col, nnz0 > 0 ? nnz0 : 1));
    GK_CUDA(cudaMemcpyAsync(rp, inout->rowptr, sizeof(int64_t) * (m + 1), cudaMemcpyDefault, s));
    if (nnz0) GK_CUDA(cudaMemcpyAsync(col, inout->col, sizeof(int32_t) * nnz0, cudaMemcpyDefault, s));
    GK_CHECK(check_csr(DevCsr{m, m, nnz0, rp, col, nullptr}, CSR_SORTED, "graph", s, scr));
    int64_t nnz = 0;
    int64_t *rp_res;
    int32_t *col_res;
    GK_CHECK(ktruss_device(m, nnz0, rp, col, k, sched, iters, &nnz, &rp_res, &col_res, s, scr));
    GK_CUDA(cudaMemcpyAsync(inout->rowptr, rp_res, sizeof(int64_t) * (m + 1),
                            dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    if (nnz) GK_CUDA(cudaMemcpyAsync(inout->col, col_res, sizeof(int32_t) * nnz,
                                     dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaStreamSynchronize(s));
    inout->nnz = nnz;
    return GK_OK;
}
