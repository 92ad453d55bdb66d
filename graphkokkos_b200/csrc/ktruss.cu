// k-truss on the GPU: gk_ktruss.
//
// Reference: k_truss (src/main.cpp:94-141): repeat Tmp<C> = C·C, drop the
// entries with support < k-2 (keeping the others with value 1), until nnz
// stops changing, at most n passes.  The reference compacts serially on the
// host (:110-119); here one pass is
//   1. support  S<C> = C·C (plus-pair) with the masked SpGEMM engine (EPI_WRITE)
//   2. flag     keep[j] = S[j] >= k-2
//   3. scan     exclusive prefix of keep over all entries (one device scan)
//   4. compact  new_rp[i] = pos[rp[i]], new_col[pos[j]] = col[j] for kept j
// and the loop stops when the kept count equals nnz.  Compaction preserves the
// order within rows, so rows stay sorted and the edge set is bit-exact with the
// reference (whose View-size defect at :99/:118 is not reproduced).
// The host reads the kept count once per pass to decide whether to stop.
#include <cub/cub.cuh>

#include "gk_common.cuh"
#include "gk_spgemm.cuh"

namespace gk {

__global__ void k_keep_flags(const int32_t *sup, int64_t nnz, int thresh, int32_t *keep) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += stride)
        keep[j] = sup[j] >= thresh;
}

__global__ void k_compact(int64_t m, int64_t nnz, const int64_t *rp, const int32_t *col, const int32_t *keep,
                          const int64_t *pos, int64_t *nrp, int32_t *ncol) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += stride)
        if (keep[j]) ncol[pos[j]] = col[j];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= m; i += stride) nrp[i] = pos[rp[i]];
}

int ktruss_device(int64_t m, int64_t nnz0, int64_t *rp_a, int32_t *col_a, int k, int sched, int *iters_out,
                  int64_t *nnz_out, int64_t **rp_res, int32_t **col_res, cudaStream_t s, Scratch &scr) {
    int64_t *rp_b;
    int32_t *col_b, *sup, *keep;
    int64_t *pos;
    GK_CHECK(scr.alloc(&rp_b, m + 1));
    GK_CHECK(scr.alloc(&col_b, nnz0 > 0 ? nnz0 : 1));
    GK_CHECK(scr.alloc(&sup, nnz0 > 0 ? nnz0 : 1));
    GK_CHECK(scr.alloc(&keep, nnz0 + 1));
    GK_CHECK(scr.alloc(&pos, nnz0 + 1));
    size_t tb = 0;
    GK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, keep, pos, nnz0 + 1, s));
    void *tmp;
    GK_CHECK(scr.alloc(reinterpret_cast<char **>(&tmp), tb));
    const int sms = ctx().num_sms;
    int64_t *rp_cur = rp_a, *rp_nxt = rp_b;
    int32_t *col_cur = col_a, *col_nxt = col_b;
    int64_t nnz = nnz0;
    int iters = 0;
    int64_t *h_nnz;
    GK_CUDA(cudaMallocHost(&h_nnz, sizeof(int64_t)));
    int status = GK_OK;
    for (int64_t t = 0; t < m; ++t) {
        if (nnz == 0) {
            ++iters;
            break;
        }
        // the scheduler's plan arrays live for one pass only
        Scratch pass(s);
        SpgemmRequest rq;
        DevCsr c{m, m, nnz, rp_cur, col_cur, nullptr};
        rq.A = rq.B = rq.M = c;
        rq.epi = EPI_WRITE;
        rq.sched = sched;
        rq.c_val = sup;
        rq.stream = s;
        status = run_spgemm(rq, pass);
        if (status != GK_OK) break;
        k_keep_flags<<<sms * 8, 256, 0, s>>>(sup, nnz, k - 2, keep);
        note_launches(1);
        if (cudaMemsetAsync(keep + nnz, 0, sizeof(int32_t), s) != cudaSuccess) {
            status = cuda_fail(cudaGetLastError(), "memset");
            break;
        }
        cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, tb, keep, pos, nnz + 1, s);
        if (e != cudaSuccess) {
            status = cuda_fail(e, "ktruss scan");
            break;
        }
        k_compact<<<sms * 8, 256, 0, s>>>(m, nnz, rp_cur, col_cur, keep, pos, rp_nxt, col_nxt);
        note_launches(1);
        e = cudaMemcpyAsync(h_nnz, pos + nnz, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            status = cuda_fail(e, "ktruss pass");
            break;
        }
        ++iters;
        const int64_t kept = *h_nnz;
        std::swap(rp_cur, rp_nxt);
        std::swap(col_cur, col_nxt);
        const bool same = kept == nnz;
        nnz = kept;
        if (same) break;
    }
    cudaFreeHost(h_nnz);
    if (status != GK_OK) return status;
    *iters_out = iters;
    *nnz_out = nnz;
    *rp_res = rp_cur;
    *col_res = col_cur;
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
