// Row binning and kernel-variant catalog of the masked SpGEMM engine.
//
// The reference's only scheduling is a choice of accumulator per call
// (src/main.cpp:194-212) and an nnz-balanced split of rows over threads
// (matrix_la.h:590-596).  Here every row of C<M> = A·B is placed in a bin by
// two features — the mask-row length nnz(M_i) and the mean length of the B
// rows it streams, work_i / nnz(A_i) with work_i = sum_{k in A_i} nnz(B_k) —
// and each bin is assigned one kernel variant (accumulator family, threads
// per row, mask-chunk capacity, work per item) by either the plain heuristic
// or the learned MLP.  The variant only decides how a row is computed, never
// what: all variants accumulate the same integer terms.
#pragma once
#include <stdint.h>

namespace gk {

// ---- bins -------------------------------------------------------------------
constexpr int NB_M = 16;  // floor(log2(nnz(M_i))), capped
constexpr int NB_B = 16;  // floor(log2(mean nnz(B_k))), capped
constexpr int NBINS = NB_M * NB_B;
constexpr uint16_t BIN_SKIP = 0xFFFF;  // row with no work or an empty mask row

struct BinStats {
    unsigned long long rows;
    unsigned long long sum_m;     // sum of nnz(M_i)
    unsigned long long sum_a;     // sum of nnz(A_i)
    unsigned long long sum_work;  // sum of work_i
    unsigned int max_b;           // max nnz(B_k) seen by any row of the bin
    unsigned int pad;
};

// ---- variants -----------------------------------------------------------------
enum Kind : int { K_HASH_GROUP = 0, K_HASH_BLOCK = 1, K_MCA_GROUP = 2, K_MCA_BLOCK = 3, K_MSA_BLOCK = 4, K_SEARCH = 5 };

struct Variant {
    int kind;
    int G;          // threads per row (group kinds) or per CTA (block kinds)
    int sub;        // lanes that stream one B row together (G/sub rows of B in flight per row)
    int cap;        // hash slots (HASH), sorted slots (MCA), log2 window columns (MSA)
    int cap_write;  // same when values are written back (WRITE epilogue needs accumulators)
    int chunk;      // mask entries per item (HASH/MCA); unused by MSA
    int chunk_write;
    int split_log2; // block kinds: work per item before a row's A entries are split
    int flog;       // block HASH kinds: log2 bits of the bitmap filter in front of the table
    int batch;      // items a CTA (group kinds: a warp) takes per fetch
    int accum;      // gk_accum family this variant belongs to
    int lowb;       // block HASH kinds: log2 of the low-column range the filter maps exactly (0: none)
    int comp;       // block HASH kinds: filter candidates packed into a per-warp queue and checked one per lane
};

constexpr int NV = 24;
// Shared-memory budget of every variant is below 160 KB; see the kernels.
// Tables are bucketed (four slots per 16-byte load).  The small ones run at
// load factor <= 1/4 (chunk <= cap/4); the large ones of variants 6-8 and
// 12-14 at load <= 1/2.  Variants with a filter (about 64 bits per mask
// entry) send only filter candidates to the table; variants 12-14 have none
// and look every streamed element up in the table directly, which wins on
// rows where a large share of the elements are mask columns.
// Variant 17 (K_SEARCH) does not stream B rows: a warp per row looks each mask
// column inside B_k's column range up in B_k by binary search (mask chunks of
// 256 columns in shared memory), which wins where mask rows are short and B
// rows long.  Variant 18 is variant 5 with quarter-warp (8-lane) sub-groups, for
// B rows shorter than a half-warp's 64-element vector step (small graphs of a
// many-graph batch).  Variant 19 is variant 8 (mask chunks of 8,192 columns
// for hub rows) with variant 15's exact map of the columns below 2^18: a hub
// row's mask and the B rows it streams concentrate on low vertex IDs, where a
// hit then costs one bit test instead of a divergent table lookup.  Variants 20
// and 21 are variants 8 and 15 with the filter candidates of a warp packed into
// a shared-memory queue and checked one per lane (comp = 1), for rows whose
// mask covers a large share of the streamed elements.  Variants 22 and 23 are
// the search kind with half- and quarter-warps per row (two and four short
// rows per warp).
// columns: kind, G, sub, cap, cap (WRITE), chunk, chunk (WRITE), split_log2, filter log2, batch, accum, comp,
// exact low-column bits (variants 15, 16: the filter maps columns below 2^lowb
// one to one, so a hit there needs no table lookup when only sums are kept)
#define GK_VARIANT_TABLE { \
    {K_HASH_GROUP,   4,  4,    64,    64,    16,    16,   0,  0, 1, 3  , 0, 0},   \
    {K_HASH_GROUP,   8,  8,   128,   128,    32,    32,   0,  0, 1, 3  , 0, 0},   \
    {K_HASH_GROUP,  32, 32,   512,   512,   128,   128,   0, 13, 1, 3  , 0, 0},   \
    {K_HASH_BLOCK,  64, 32,   512,   512,   128,   128,  16, 13, 8, 3  , 0, 0},   \
    {K_HASH_BLOCK, 128, 32,  1024,  1024,   256,   256,  17, 14, 4, 3  , 0, 0},   \
    {K_HASH_BLOCK, 128, 16,  1024,  1024,   256,   256,  17, 14, 4, 3  , 0, 0},   \
    {K_HASH_BLOCK, 128, 32,  2048,  2048,  1024,  1024,  18, 16, 2, 3  , 0, 0},   \
    {K_HASH_BLOCK, 256, 32,  8192,  8192,  4096,  4096,  19, 17, 1, 3  , 0, 0},   \
    {K_HASH_BLOCK, 512, 32, 16384, 16384,  8192,  8192,  20, 18, 1, 3  , 0, 0},   \
    {K_MCA_GROUP,   32, 32,   256,   256,   256,   256,   0,  0, 1, 2  , 0, 0},   \
    {K_MCA_BLOCK,  512, 32, 16384, 16384, 16384, 16384,  20,  0, 1, 2  , 0, 0},   \
    {K_MSA_BLOCK,  512, 32,    20,    15,     0,     0,  20,  0, 1, 1  , 0, 0},   \
    {K_HASH_BLOCK, 256, 32,  8192,  8192,  4096,  4096,  19,  0, 1, 3  , 0, 0},   \
    {K_HASH_BLOCK, 128, 32,  2048,  2048,  1024,  1024,  18,  0, 2, 3  , 0, 0},   \
    {K_HASH_BLOCK, 512, 32, 16384, 16384,  8192,  8192,  20,  0, 1, 3  , 0, 0},   \
    {K_HASH_BLOCK, 512, 32,  8192, 16384,  4096,  8192,  20, 16, 1, 3  , 18, 0},  \
    {K_HASH_BLOCK, 128, 32,  2048,  2048,  1024,  1024,  18, 14, 2, 3  , 15, 0},  \
    {K_SEARCH,      32, 32,   256,   256,   256,   256,   0,  0, 2, 0  , 0, 0},   \
    {K_HASH_BLOCK, 128,  8,  1024,  1024,   256,   256,  17, 14, 4, 3  , 0, 0},   \
    {K_HASH_BLOCK, 512, 32, 16384, 16384,  8192,  8192,  20, 16, 1, 3  , 18, 0},  \
    {K_HASH_BLOCK, 512, 32, 16384, 16384,  8192,  8192,  20, 18, 1, 3  , 0, 1},  \
    {K_HASH_BLOCK, 512, 32,  8192, 16384,  4096,  8192,  20, 16, 1, 3  , 18, 1}, \
    {K_SEARCH,      16, 16,    64,    64,    64,    64,   0,  0, 2, 0  , 0, 0},   \
    {K_SEARCH,       8,  8,    32,    32,    32,    32,   0,  0, 2, 0  , 0, 0},   \
}
constexpr Variant VARIANTS[NV] = GK_VARIANT_TABLE;
#ifdef __CUDACC__
__constant__ const Variant c_variants[NV] = GK_VARIANT_TABLE;  // runtime-indexed copy for device code
#endif
constexpr int NT_GROUP = 256;  // CTA size of the group kinds
__host__ __device__ constexpr int group_cta_threads(int) { return NT_GROUP; }
// variant ids the heuristics name
constexpr int V_MCA_GROUP = 9, V_MCA_BLOCK = 10, V_MSA_BLOCK = 11;

// Variants the learned scheduler (and the autotuner) may pick for a bin: a
// variant is excluded where it would split every mask row into many chunks
// (small structures on long mask rows) or rebuild a large structure for every
// short row (large structures on short mask rows).
__host__ __device__ constexpr bool variant_allowed(int v, int bin) {
    const int qm = bin / NB_B;  // floor(log2(nnz(M_i)))
    switch (v) {
        case 0: return qm <= 5;
        case 1: return qm <= 6;
        case 2: return qm <= 8;
        case 3: return qm <= 10;
        case 4:
        case 5: return qm <= 11;
        case 6: return true;
        case 7: return qm >= 5;
        case 8: return qm >= 8;
        case 9: return qm <= 9;
        case 10: return qm >= 7;
        case 11: return qm >= 9;
        case 12: return qm >= 5;
        case 13: return true;
        case 14: return qm >= 8;
        case 15: return qm >= 8;
        case 16: return true;
        case 17: return qm <= 8;  // binary-search lookups: mask rows below 512 columns
        case 18: return qm <= 11;
        case 19: return qm >= 10;
        case 20:
        case 21: return qm >= 8;
        case 22: return qm <= 6;
        case 23: return qm <= 5;
        default: return false;
    }
}

// ---- features of a bin (inputs of the learned scheduler) ---------------------
constexpr int NFEAT = 8;
// f0 log2(1+mean nnz(M_i))   f1 log2(1+mean nnz(B_k))   f2 log2(1+mean nnz(A_i))
// f3 log2(1+mean work_i)     f4 log2(1+max nnz(B_k)) - f1 (degree skew)
// f5 log2(1+rows)            f6 1 if values are written back (WRITE epilogue)
// f7 1 if A or B carries values (plus-times) else 0 (plus-pair)

// ---- MLP of the learned scheduler --------------------------------------------
constexpr int MLP_H = 32;
// layout (float32): W1[MLP_H][NFEAT], b1[MLP_H], W2[MLP_H][MLP_H], b2[MLP_H],
//                   W3[NV][MLP_H], b3[NV], mu[NFEAT], sigma[NFEAT]
constexpr int MLP_SIZE = MLP_H * NFEAT + MLP_H + MLP_H * MLP_H + MLP_H + NV * MLP_H + NV + 2 * NFEAT;

#ifdef __CUDACC__
// Forward pass of the network (mlp.cu): out[NV] from the raw features f;
// x, h1, h2 are caller scratch of NFEAT, MLP_H, MLP_H floats.
__device__ void mlp_forward(const float *w, const float *f, float *x, float *h1, float *h2, float *out);
// outputs 0 and 1 of the same network, computed by one full warp (mlp.cu)
__device__ void mlp_forward_warp2(const float *w, const float *f, float *o0, float *o1);
#endif

}  // namespace gk
