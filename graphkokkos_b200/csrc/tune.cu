// Autotuning entry points of the row-bin scheduler: per-bin statistics and
// features of a product, the plain / learned choices, and timed runs of a
// chosen subset of bins on chosen variants.  No reference counterpart (the
// reference's scheduling is the CLI's accumulator choice, src/main.cpp:194-212).
#include <vector>

#include "gk_common.cuh"
#include "gk_sched.cuh"
#include "gk_spgemm.cuh"

namespace gk {

void bin_features_host(const BinStats &b, int epi, bool values, float *f);
int plain_variant_host(int bin, const BinStats &b);


// mode 0: triangle counting on L (A = B = M = L, sum of C);
// mode 1: k-truss support on a symmetric A as gk_ktruss computes it
//         (A = B = the symmetric matrix, M = its strict lower triangle, values written).
static int tune_request(const gk_csr *G, int mode, SpgemmRequest &rq, Scratch &scr, cudaStream_t s,
                        unsigned long long **sums, int32_t **cval) {
    if (mode != 0 && mode != 1) return fail(GK_ERR_ARG, "tune: mode must be 0 (triangle count) or 1 (k-truss support)");
    GK_CHECK(validate_csr_shape(G, "G"));
    if (G->m != G->n) return fail(GK_ERR_ARG, "tune: matrix must be square");
    DevCsr d;
    GK_CHECK(stage_csr(G, &d, scr, s, nullptr, CSR_SORTED, "graph"));
    d.val = nullptr;
    rq.A = rq.B = rq.M = d;
    rq.stream = s;
    if (mode == 0) {
        GK_CHECK(scr.alloc(sums, 1));
        GK_CUDA(cudaMemsetAsync(*sums, 0, sizeof(unsigned long long), s));
        rq.epi = EPI_SUM;
        rq.sums = *sums;
    } else {
        GK_CHECK(scr.alloc(cval, d.nnz > 0 ? d.nnz : 1));
        rq.epi = EPI_WRITE;
        rq.c_val = *cval;
        int64_t *lrp;
        int32_t *lcol;
        GK_CHECK(scr.alloc(&lrp, d.m + 1));
        GK_CHECK(scr.alloc(&lcol, d.nnz > 0 ? d.nnz : 1));
        GK_CHECK(extract_lower_device(d, lrp, lcol, s, scr));
        rq.M = DevCsr{d.m, d.n, d.nnz, lrp, lcol, nullptr};
    }
    return GK_OK;
}

}  // namespace gk

using namespace gk;

extern "C" {

int gk_sched_num_bins(void) { return NBINS; }

int gk_sched_bins(const gk_csr *G, int mode, gk_bin_stat *stats, int32_t *plain_variant, int32_t *learned_variant,
                  float *features, void *stream) {
    if (!stats) return fail(GK_ERR_ARG, "gk_sched_bins: stats is null");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    SpgemmRequest rq;
    unsigned long long *sums = nullptr;
    int32_t *cval = nullptr;
    GK_CHECK(tune_request(G, mode, rq, scr, s, &sums, &cval));
    BinStats *dbins;
    GK_CHECK(scr.alloc(&dbins, NBINS));
    GK_CUDA(cudaMemsetAsync(dbins, 0, sizeof(BinStats) * NBINS, s));
    rq.bin_stats_out = dbins;
    rq.stats_only = true;
    rq.zero_output = false;
    int *dvar = nullptr;
    if (learned_variant) {
        GK_CHECK(scr.alloc(&dvar, NBINS));
        rq.sched = GK_SCHED_LEARNED;
        rq.variant_of_bin_out = dvar;
    }
    GK_CHECK(run_spgemm(rq, scr));
    std::vector<BinStats> hb(NBINS);
    GK_CUDA(cudaMemcpyAsync(hb.data(), dbins, sizeof(BinStats) * NBINS, cudaMemcpyDeviceToHost, s));
    std::vector<int> hv(NBINS, 0);
    if (dvar) GK_CUDA(cudaMemcpyAsync(hv.data(), dvar, sizeof(int) * NBINS, cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaStreamSynchronize(s));
    for (int b = 0; b < NBINS; ++b) {
        stats[b].rows = static_cast<int64_t>(hb[b].rows);
        stats[b].sum_m = static_cast<int64_t>(hb[b].sum_m);
        stats[b].sum_a = static_cast<int64_t>(hb[b].sum_a);
        stats[b].sum_work = static_cast<int64_t>(hb[b].sum_work);
        stats[b].max_b = static_cast<int64_t>(hb[b].max_b);
        if (plain_variant) plain_variant[b] = hb[b].rows ? plain_variant_host(b, hb[b]) : -1;
        if (learned_variant) learned_variant[b] = hb[b].rows ? hv[b] : -1;
        if (features) {
            if (hb[b].rows) bin_features_host(hb[b], rq.epi, false, features + b * NFEAT);
            else
                for (int f = 0; f < NFEAT; ++f) features[b * NFEAT + f] = 0.f;
        }
    }
    return GK_OK;
}

int gk_tune_run(const gk_csr *G, int mode, const int32_t *bin_variant, float *variant_ms, uint64_t *sum,
                void *stream) {
    if (!bin_variant || !variant_ms) return fail(GK_ERR_ARG, "gk_tune_run: null argument");
    for (int b = 0; b < NBINS; ++b)
        if (bin_variant[b] < -1 || bin_variant[b] >= NV) return fail(GK_ERR_ARG, "gk_tune_run: variant out of range");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    SpgemmRequest rq;
    unsigned long long *sums = nullptr;
    int32_t *cval = nullptr;
    GK_CHECK(tune_request(G, mode, rq, scr, s, &sums, &cval));
    rq.bin_variant = bin_variant;
    rq.variant_ms_out = variant_ms;
    GK_CHECK(run_spgemm(rq, scr));
    if (sum) {
        unsigned long long h = 0;
        if (sums) GK_CUDA(cudaMemcpyAsync(&h, sums, sizeof(h), cudaMemcpyDeviceToHost, s));
        GK_CUDA(cudaStreamSynchronize(s));
        *sum = h;
    }
    return GK_OK;
}

}  // extern "C"
