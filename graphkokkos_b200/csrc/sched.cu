// Row-bin scheduler of the masked SpGEMM engine: the plain binning
// heuristic and the learned MLP (inference on the device), plus the model
// registry behind gk_sched_set_model.
//
// No reference counterpart beyond the CLI's per-call accumulator choice
// (src/main.cpp:194-212).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "gk_common.cuh"
#include "gk_internal_host.h"
#include "gk_sched.cuh"
#include "gk_spgemm.cuh"

namespace gk {

__device__ float d_mlp[MLP_SIZE];

static std::mutex g_model_mutex;
static std::vector<float> g_model;     // host copy
static int g_model_version = 0;
static int g_model_uploaded[64];       // version uploaded per device

__host__ __device__ inline void bin_features(const BinStats &b, int epi, bool values, float *f) {
    const double rows = static_cast<double>(b.rows);
    const double mean_m = b.sum_m / rows;
    const double mean_b = b.sum_a ? static_cast<double>(b.sum_work) / static_cast<double>(b.sum_a) : 0.0;
    const double mean_a = b.sum_a / rows;
    const double mean_w = b.sum_work / rows;
    f[0] = static_cast<float>(log2(1.0 + mean_m));
    f[1] = static_cast<float>(log2(1.0 + mean_b));
    f[2] = static_cast<float>(log2(1.0 + mean_a));
    f[3] = static_cast<float>(log2(1.0 + mean_w));
    f[4] = static_cast<float>(log2(1.0 + static_cast<double>(b.max_b))) - f[1];
    f[5] = static_cast<float>(log2(1.0 + rows));
    f[6] = epi == EPI_WRITE ? 1.0f : 0.0f;
    f[7] = values ? 1.0f : 0.0f;
}

// Plain heuristic: the smallest structure that holds the mask row in one
// chunk, a wider thread group when the streamed B rows are long, and a block
// kind (which splits rows over CTAs) when a row carries a lot of work.
__host__ __device__ inline int plain_variant(int bin, const BinStats &b) {
    const int qm = bin / NB_B, qb = bin % NB_B;  // log2 mask-row length, log2 mean B-row length
    int v;
    if (qm <= 3) v = qb <= 4 ? 0 : 3;       // < 16 mask entries: 4 threads, or a 2-warp CTA for long B rows
    else if (qm == 4) v = qb <= 3 ? 1 : 3;  // < 32
    else if (qm <= 6) v = qb <= 3 ? 2 : 3;  // < 128
    else if (qm == 7) v = qb <= 5 ? 5 : 4;  // < 256: half-warps stream short B rows
    else if (qm <= 9) v = 6;                // < 1024
    else if (qm <= 11) v = 7;               // < 4096
    else v = 8;
    const double mean_w = static_cast<double>(b.sum_work) / static_cast<double>(b.rows ? b.rows : 1);
    if (v <= 2 && mean_w > double(1 << 16)) v = 3;  // heavy rows: CTA kinds split them
    return v;
}

__host__ __device__ inline int forced_variant(int bin, const BinStats &b, int accum) {
    const int qm = bin / NB_B;
    switch (accum) {
        case GK_ACCUM_MSA: return V_MSA_BLOCK;
        case GK_ACCUM_MCA: return qm <= 7 ? V_MCA_GROUP : V_MCA_BLOCK;
        default: return plain_variant(bin, b);
    }
}

// The learned choice replaces the plain one only where the model predicts it
// at least this much faster (log2 of 1.1): small predicted gains are within the
// model's error and are not worth a change of kernel.  GK_LEARNED_MARGIN (a
// log2 ratio) overrides it, for tuning runs.
constexpr float LEARNED_MARGIN = 0.1375f;

static float learned_margin() {
    static const float m = [] {
        const char *e = getenv("GK_LEARNED_MARGIN");
        const float v = e ? static_cast<float>(atof(e)) : LEARNED_MARGIN;
        return std::isfinite(v) && v >= 0.f ? v : LEARNED_MARGIN;
    }();
    return m;
}

__device__ inline int mlp_variant(const float *w, const float *f_raw, int bin, int plain, float margin) {
    const float *W1 = w;
    const float *b1 = W1 + MLP_H * NFEAT;
    const float *W2 = b1 + MLP_H;
    const float *b2 = W2 + MLP_H * MLP_H;
    const float *W3 = b2 + MLP_H;
    const float *b3 = W3 + NV * MLP_H;
    const float *mu = b3 + NV;
    const float *sg = mu + NFEAT;
    float x[NFEAT], h1[MLP_H], h2[MLP_H];
    for (int i = 0; i < NFEAT; ++i) x[i] = (f_raw[i] - mu[i]) / sg[i];
    for (int j = 0; j < MLP_H; ++j) {
        float a = b1[j];
        for (int i = 0; i < NFEAT; ++i) a += W1[j * NFEAT + i] * x[i];
        h1[j] = a > 0.f ? a : 0.f;
    }
    for (int j = 0; j < MLP_H; ++j) {
        float a = b2[j];
        for (int i = 0; i < MLP_H; ++i) a += W2[j * MLP_H + i] * h1[i];
        h2[j] = a > 0.f ? a : 0.f;
    }
    int best = 6;  // allowed for every bin
    float best_s = 3.0e38f, plain_s = 3.0e38f;
    for (int v = 0; v < NV; ++v) {
        if (!variant_allowed(v, bin) && v != plain) continue;
        float a = b3[v];
        for (int i = 0; i < MLP_H; ++i) a += W3[v * MLP_H + i] * h2[i];
        if (v == plain) plain_s = a;
        if (variant_allowed(v, bin) && a < best_s) {
            best_s = a;
            best = v;
        }
    }
    return plain_s - best_s >= margin ? best : plain;
}

__global__ void k_choose(const BinStats *bins, int *var_of_bin, int mode, int accum, int epi, bool values,
                         float margin) {
    // the weights are read by every bin's thread: stage them in shared memory
    // (broadcast reads) instead of chains of dependent global loads
    __shared__ float sw[MLP_SIZE];
    const bool learned = mode == GK_SCHED_LEARNED && accum == GK_ACCUM_AUTO;
    if (learned) {
        for (int i = threadIdx.x; i < MLP_SIZE; i += blockDim.x) sw[i] = d_mlp[i];
        __syncthreads();
    }
    const int b = threadIdx.x + blockIdx.x * blockDim.x;
    if (b >= NBINS) return;
    const BinStats st = bins[b];
    if (st.rows == 0) {
        var_of_bin[b] = 0;
        return;
    }
    int v;
    if (accum != GK_ACCUM_AUTO) v = forced_variant(b, st, accum);
    else if (mode == GK_SCHED_LEARNED) {
        float f[NFEAT];
        bin_features(st, epi, values, f);
        v = mlp_variant(sw, f, b, plain_variant(b, st), margin);
    } else v = plain_variant(b, st);
    var_of_bin[b] = v;
}

void bin_features_host(const BinStats &b, int epi, bool values, float *f) { bin_features(b, epi, values, f); }
int plain_variant_host(int bin, const BinStats &b) { return plain_variant(bin, b); }

static int ensure_model_on_device() {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(g_model_mutex);
    if (g_model.empty()) return fail(GK_ERR_ARG, "learned scheduler requested but no model is loaded (gk_sched_set_model)");
    if (g_model_uploaded[dev & 63] != g_model_version) {
        GK_CUDA(cudaMemcpyToSymbol(d_mlp, g_model.data(), sizeof(float) * MLP_SIZE));
        g_model_uploaded[dev & 63] = g_model_version;
    }
    return GK_OK;
}

int sched_prepare(int sched, int force_accum) {
    if (sched != GK_SCHED_PLAIN && sched != GK_SCHED_LEARNED) return fail(GK_ERR_ARG, "unknown scheduler mode");
    if (force_accum < GK_ACCUM_AUTO || force_accum > GK_ACCUM_HASH) return fail(GK_ERR_ARG, "unknown accumulator");
    if (sched == GK_SCHED_LEARNED && force_accum == GK_ACCUM_AUTO) GK_CHECK(ensure_model_on_device());
    return GK_OK;
}

int sched_choose(const BinStats *bins, int *var_of_bin, int sched, int force_accum, int epi, bool values,
                 cudaStream_t s) {
    GK_CHECK(sched_prepare(sched, force_accum));
    k_choose<<<1, NBINS, 0, s>>>(bins, var_of_bin, sched, force_accum, epi, values, learned_margin());
    GK_CUDA(cudaGetLastError());
    return GK_OK;
}

}  // namespace gk

namespace gk {

std::string read_model_file(const char *path, std::vector<float> &out) {
    if (!path) return "path is null";
    FILE *f = fopen(path, "rb");
    if (!f) return std::string("cannot open ") + path;
    unsigned char head[12];
    std::string err;
    if (fread(head, 1, sizeof(head), f) != sizeof(head) || memcmp(head, "GKMLP001", 8) != 0) {
        err = std::string(path) + " is not a scheduler model file (magic GKMLP001)";
    } else {
        const uint32_t n = uint32_t(head[8]) | (uint32_t(head[9]) << 8) | (uint32_t(head[10]) << 16) |
                           (uint32_t(head[11]) << 24);
        if (n != static_cast<uint32_t>(MLP_SIZE)) {
            err = std::string(path) + " holds " + std::to_string(n) + " weights, the model has " +
                  std::to_string(MLP_SIZE);
        } else {
            std::vector<unsigned char> raw(4 * size_t(n) + 1);
            if (fread(raw.data(), 1, raw.size(), f) != 4 * size_t(n)) {
                err = std::string(path) + ": wrong length (truncated, or bytes after the weights)";
            } else {
                out.resize(n);
                for (uint32_t i = 0; i < n; ++i) {
                    const uint32_t b = uint32_t(raw[4 * i]) | (uint32_t(raw[4 * i + 1]) << 8) |
                                       (uint32_t(raw[4 * i + 2]) << 16) | (uint32_t(raw[4 * i + 3]) << 24);
                    memcpy(&out[i], &b, 4);
                }
            }
        }
    }
    fclose(f);
    return err;
}

}  // namespace gk

extern "C" {

int gk_sched_num_variants(void) { return gk::NV; }
int gk_sched_variant_allowed(int bin, int variant) {
    return (bin >= 0 && bin < gk::NBINS && gk::variant_allowed(variant, bin)) ? 1 : 0;
}
int gk_sched_num_features(void) { return gk::NFEAT; }
size_t gk_sched_model_size(void) { return static_cast<size_t>(gk::MLP_SIZE); }

int gk_sched_set_model(const float *weights, size_t n_floats) {
    if (!weights || n_floats != static_cast<size_t>(gk::MLP_SIZE))
        return gk::fail(GK_ERR_ARG, "gk_sched_set_model: weight count does not match gk_sched_model_size()");
    for (size_t i = 0; i < n_floats; ++i)
        if (!std::isfinite(weights[i])) return gk::fail(GK_ERR_ARG, "gk_sched_set_model: non-finite weight");
    std::lock_guard<std::mutex> lock(gk::g_model_mutex);
    gk::g_model.assign(weights, weights + n_floats);
    ++gk::g_model_version;
    return GK_OK;
}

int gk_sched_has_model(void) {
    std::lock_guard<std::mutex> lock(gk::g_model_mutex);
    return gk::g_model.empty() ? 0 : 1;
}

int gk_sched_load_model_file(const char *path) {
    std::vector<float> w;
    const std::string err = gk::read_model_file(path, w);
    if (!err.empty()) return gk::fail(GK_ERR_ARG, "gk_sched_load_model_file: " + err);
    return gk_sched_set_model(w.data(), w.size());
}

}  // extern "C"
