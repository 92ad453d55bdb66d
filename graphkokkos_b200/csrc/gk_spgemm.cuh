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

// Everything run_spgemm configures on its first use (kernel attributes and
// grid sizes of every variant for this epilogue, the learned model's upload),
// done ahead so that later calls can be captured into a CUDA graph.
int spgemm_prepare(int epi, bool values, int sched, int force_accum);
// Device scratch one run_spgemm call on an m-row A takes (arena sizing).
size_t spgemm_scratch_bytes(int64_t m);

// Scheduler (sched.cu): fills var_of_bin[NBINS] on the device from the bin
// statistics, by the plain heuristic, the learned MLP, or a forced family.
int sched_choose(const BinStats *bins, int *var_of_bin, int sched, int force_accum, int epi, bool values,
                 cudaStream_t s);
// Validates the mode and uploads the learned model if it will be used.
int sched_prepare(int sched, int force_accum);

}  // namespace gk
