// Internal interface of the masked SpGEMM engine (spgemm.cu), shared by the
// triangle-counting, k-truss and batched entry points.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "gk_common.cuh"
#include "gk_sched.cuh"

namespace gk {

enum Epi : int {
    EPI_WRITE = 0,  // C_val[p] = sum over k of A(i,k)·B(k, M.col[p])
    EPI_SUM = 1,    // sums[0] += every C value (triangle counting)
    EPI_KEYED = 2   // sums[key(i)] += the C values of row i (key = row_key[i], or i)
};

struct SpgemmRequest {
    DevCsr A, B, M;
    int epi = EPI_WRITE;
    bool use_values = false;  // plus-times with A.val / B.val (missing arrays read as 1)
    int sched = GK_SCHED_PLAIN;
    int force_accum = GK_ACCUM_AUTO;
    int force_variant = -1;    // autotuning: every row goes to this variant
    const int *bin_variant = nullptr;  // autotuning: host table [NBINS] overriding the scheduler
    int32_t *c_val = nullptr;
    unsigned long long *sums = nullptr;
    const int32_t *row_key = nullptr;
    bool zero_output = true;   // memset C_val / sums before accumulating
    cudaStream_t stream = nullptr;
    // optional outputs for the scheduler and the autotuner
    BinStats *bin_stats_out = nullptr;  // device [NBINS]
    int *variant_of_bin_out = nullptr;  // device [NBINS]
    float *variant_ms_out = nullptr;    // host [NV]: CUDA-event time of each variant launch (synchronises)
    bool stats_only = false;            // stop after the bin statistics
};

int run_spgemm(const SpgemmRequest &req, Scratch &scr);

// Scheduler (sched.cu): fills var_of_bin[NBINS] on the device from the bin
// statistics, by the plain heuristic, the learned MLP, or a forced family.
int sched_choose(const BinStats *bins, int *var_of_bin, int sched, int force_accum, int epi, bool values,
                 cudaStream_t s);

}  // namespace gk
