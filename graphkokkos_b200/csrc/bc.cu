// Batched betweenness centrality in FP64: gk_bc_batch.
//
// Reference: betweenness_centrality_batch (include/betweenness_centrality.h:406-506)
// with bc_forward_step (:313-401) and bc_backward_step (:182-242).  Per
// source column s of an m x b batch:
//   forward   Numsp += F_d;  F_{d+1}<!Numsp> = A^T·F_d   (path counts sigma)
//   backward  W = (1/sigma)∘Bcu on level d+1;  Bcu<level d> += (A·W)∘sigma,  Bcu = 1 + delta
//   result    bc[v] = sum_s (Bcu(v,s) - 1)
// The reference keeps int32 sigma / float dependencies and scans all b
// columns of every row per level (:359-363, :391-397).
//
// B200 layout: the batch is processed in chunks of W = 32*T sources (T <= 16).
//   sigma[v*W + s], R[v*W + s]   FP64, row-major: one vertex's chunk is W*8
//                                bytes contiguous (4 KB at W = 512)
//   level bitmaps F_d[v*T + t]   bit l of word t <=> source 32t+l is at depth d
//   visited bitmap V[v*T + t]
// Forward levels run one of two kernel shapes, chosen per level on the device:
//   pull  one warp per vertex with sources still open: its lanes test 32
//         in-neighbours' frontier words at a time, then take the (neighbour,
//         source) hits 32 at a time, one per lane, each adding the neighbour's
//         sigma of its source into the vertex's sum of that source;
//   push  one warp per frontier vertex: its lanes test 32 out-neighbours'
//         visited words at a time, then add sigma into the new vertices with
//         FP64 atomics.  sigma are path counts, integers below 2^53 in FP64, so
//         the order of the additions does not change them.
// The plain rule picks push while the frontier's edges are few against the
// edges still to explore (Beamer's direction-optimising rule); the learned
// rule is an MLP over the level's frontier statistics, trained on measured
// per-level times of both shapes.  Backward levels pull: one warp per vertex
// of level d, lanes testing 32 successors' level-(d+1) words at a time and
// gathering their R words hit by hit in the same way.
// Vertices with more than BC_HEAVY neighbours have their neighbour lists cut
// into items of BC_ITEM_EDGES edges, one CTA each, so that a hub no longer
// holds one CTA for the whole level; the items' partial sums are added per
// vertex in item order.
// R(v,s) = (1+delta)/sigma replaces the reference's Nspinv∘Bcu; delta is summed
// into bc[v] as soon as it is final, in a fixed order (deterministic).
//
// Every kernel reads the level index and the level bitmaps from device state,
// so the level loops are CUDA graphs: a conditional while node around one
// captured level, the condition set by the level's last kernel.  Both forward
// shapes are launched every level and the one not chosen returns at once.
#include <cub/cub.cuh>

#include <cmath>
#include <mutex>
#include <vector>

#include "gk_common.cuh"
#include "gk_internal_host.h"
#include "gk_device.cuh"
#include "gk_sched.cuh"

namespace gk {


// Widest chunk: 32 * GK_BC_TMAX sources (a power of two, at most 16).
#ifndef GK_BC_TMAX
#define GK_BC_TMAX 16
#endif
// Resident CTAs per SM the light level kernels are register-capped for: 4 CTAs
// of 8 warps (32 warps per SM, 64 registers a thread), which their gathers of
// scattered FP64 words need for latency hiding; their accumulators live in
// shared memory (SmemAcc, 32 KB a CTA).
#ifndef GK_BC_MINB
#define GK_BC_MINB 4
#endif
// A gather step whose hits average more than this per hit edge takes its
// edges one at a time (see pull_gather).
#ifndef GK_BC_DENSE_HITS
#define GK_BC_DENSE_HITS 32
#endif
#ifndef GK_BC_HEAVY
#define GK_BC_HEAVY 512
#endif
#ifndef GK_BC_ITEM_EDGES
#define GK_BC_ITEM_EDGES 1024
#endif
constexpr int BC_HEAVY = GK_BC_HEAVY;
constexpr int BC_NW_HEAVY = 8;  // T=16: 8*16*32 doubles = 32 KB of static shared memory
constexpr int BC_PULL = 0, BC_PUSH = 1;
constexpr int BC_LEVEL_BATCH = 16;  // level bitmaps allocated at a time
constexpr int BC_FEAT = NFEAT;
constexpr int BC_ITEM_EDGES = GK_BC_ITEM_EDGES;  // edges of a heavy vertex per CTA work item

// Vertices with more than BC_HEAVY neighbours, their neighbour lists cut
// into items of BC_ITEM_EDGES edges (one CTA each).  Pull-type items write
// per-item partial sums; a warp per heavy vertex adds its items' partials in
// item order (deterministic) and emits.
struct HeavySet {
    const int32_t *list;   // heavy vertices
    const int32_t *first;  // items of list[h]: first[h] .. first[h+1]-1
    const int32_t *item_h; // heavy index of each item
    int n, items;
};

// learned forward-shape model (same network as the row-bin scheduler's;
// outputs 0 and 1 predict log2 microseconds of a pull and a push level)
__device__ float d_mlp_bc[MLP_SIZE];
static std::mutex g_bc_model_mutex;
static std::vector<float> g_bc_model;
static int g_bc_model_version = 0;
static int g_bc_uploaded[64];

struct BcState {
    uint32_t **fptr;               // fptr[d] = F_d (m x T words), d = 1..levels
    int d;                         // forward: deepest level built so far
    int levels;                    // bitmaps allocated
    int bd;                        // backward: level being processed
    int mode;                      // forward shape of the current level
    int done;                      // forward finished (next frontier empty)
    int pad;
    unsigned long long nf, ef, bf;  // F_d: vertices, their out-edges, (vertex, source) pairs
    unsigned long long nn, en, bn;  // F_{d+1} under construction
    unsigned long long visited;     // (vertex, source) pairs reached, sources included
    unsigned long long pushes, pulls;
    unsigned long long cur_pull, cur_push, cur_bwd;  // vertex cursors of the light kernels
    unsigned long long cur_ipull, cur_ipush, cur_ibwd;  // item cursors of the heavy-vertex kernels
};

// Light kernels hand vertices to warps BC_GRAB at a time from a counter, so
// that a warp which met expensive vertices does not hold the level back.
#ifndef GK_BC_GRAB
#define GK_BC_GRAB 2
#endif
constexpr int BC_GRAB = GK_BC_GRAB;
__device__ __forceinline__ int64_t grab_vertices(unsigned long long *cursor, int lane) {
    unsigned long long b = 0;
    if (lane == 0) b = atomicAdd(cursor, static_cast<unsigned long long>(BC_GRAB));
    return static_cast<int64_t>(__shfl_sync(0xFFFFFFFFu, b, 0));
}

// The heavy-vertex item kernels take items one per CTA from a counter too:
// items of one level differ in cost (their hit densities), so a fixed
// round-robin share per CTA left the level waiting on the unluckiest CTA.
// Every thread of the CTA calls it (it contains barriers).
__device__ __forceinline__ int next_item(unsigned long long *cursor) {
    __shared__ int s_item;
    __syncthreads();  // the previous item's index has been read by all
    if (threadIdx.x == 0) s_item = static_cast<int>(atomicAdd(cursor, 1ull));
    __syncthreads();
    return s_item;
}

template <int T>
__device__ __forceinline__ void load_words(const uint32_t *p, uint32_t (&w)[T]) {
    if constexpr (T % 4 == 0) {
#pragma unroll
        for (int q = 0; q < T / 4; ++q) {
            const uint4 x = __ldg(reinterpret_cast<const uint4 *>(p) + q);
            w[4 * q] = x.x;
            w[4 * q + 1] = x.y;
            w[4 * q + 2] = x.z;
            w[4 * q + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int t = 0; t < T; ++t) w[t] = __ldg(p + t);
    }
}

// plain (coherent) loads, for words other CTAs of the same kernel may change
template <int T>
__device__ __forceinline__ void load_words_rw(const uint32_t *p, uint32_t (&w)[T]) {
#pragma unroll
    for (int t = 0; t < T; ++t) w[t] = p[t];
}

// The light level kernels keep each lane's FP64 accumulators of the T source
// words in shared memory (the warp's slice, word t of lane l at 32 t + l:
// conflict-free) instead of 2T registers, which would cap their residency.
struct SmemAcc {
    double *p;
    __device__ __forceinline__ double &operator[](int t) const { return p[32 * t]; }
    // the warp's slice, source s at [s]
    __device__ __forceinline__ double *warp_base(int lane) const { return p - lane; }
};

// One atomic per block and counter.
__device__ __forceinline__ void add_level_stats(unsigned long long n, unsigned long long e, unsigned long long b,
                                                unsigned long long *dst) {
    __shared__ unsigned long long red[32];
    n = block_sum(n, red);
    if (threadIdx.x == 0 && n) atomicAdd(dst, n);
    e = block_sum(e, red);
    if (threadIdx.x == 0 && e) atomicAdd(dst + 1, e);
    b = block_sum(b, red);
    if (threadIdx.x == 0 && b) atomicAdd(dst + 2, b);
}

__global__ void k_bc_seed(DevCsr A, const int32_t *src, int nsrc, int T, int W, uint32_t *F1, uint32_t *V,
                          double *sigma) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < nsrc; j += warps) {
        const int s = src[j];
        const uint32_t bit = 1u << (j & 31);
        const int word = j >> 5;
        for (int64_t e = A.rp[s] + lane; e < A.rp[s + 1]; e += 32) {
            const int v = A.col[e];
            const int a = A.val ? A.val[e] : 1;
            if (v == s || a == 0) continue;
            sigma[(int64_t)v * W + j] = static_cast<double>(a);
            atomicOr(F1 + (int64_t)v * T + word, bit);
            atomicOr(V + (int64_t)v * T + word, bit);
        }
        if (lane == 0) atomicOr(V + (int64_t)s * T + word, bit);
    }
}

// Statistics of F_1 (thread per vertex) into st->nf/ef/bf.
template <int T>
__global__ void k_bc_first_stats(DevCsr A, const uint32_t *F1, BcState *st, int nsrc) {
    unsigned long long n = 0, e = 0, b = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < A.m; v += stride) {
        uint32_t f[T];
        load_words<T>(F1 + v * T, f);
        int c = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) c += __popc(f[t]);
        if (c) {
            ++n;
            e += static_cast<unsigned long long>(A.rp[v + 1] - A.rp[v]);
            b += c;
        }
    }
    add_level_stats(n, e, b, &st->nf);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&st->visited, static_cast<unsigned long long>(nsrc));
}

// Features of the current level (inputs of the learned shape model).
__device__ void bc_features(const BcState *st, int64_t m, int64_t nnz, int W, float *f) {
    const double total = static_cast<double>(m) * W;
    const double unvisited = total > st->visited ? total - static_cast<double>(st->visited) : 0.0;
    const double mu = static_cast<double>(nnz) * unvisited / (total > 0 ? total : 1.0);  // edges left to explore
    f[0] = static_cast<float>(log2(1.0 + st->nf));
    f[1] = static_cast<float>(log2(1.0 + st->ef));
    f[2] = static_cast<float>(log2(1.0 + st->bf));
    f[3] = static_cast<float>(log2(1.0 + mu));
    f[4] = static_cast<float>(log2(1.0 + m));
    f[5] = static_cast<float>(log2(1.0 + nnz));
    f[6] = static_cast<float>(log2(static_cast<double>(W)));
    f[7] = static_cast<float>(st->d);
}

// Plain rule (Beamer's direction-optimising BFS, alpha = 14, beta = 24): push
// while the frontier's out-edges are few against the edges left to explore,
// or while the frontier holds few vertices.
__device__ int bc_plain_shape(const BcState *st, int64_t m, int64_t nnz, int W) {
    const double total = static_cast<double>(m) * W;
    const double unvisited = total > st->visited ? total - static_cast<double>(st->visited) : 0.0;
    const double mu = static_cast<double>(nnz) * unvisited / (total > 0 ? total : 1.0);
    if (static_cast<double>(st->ef) * 14.0 < mu) return BC_PUSH;
    if (static_cast<double>(st->nf) * 24.0 < static_cast<double>(m)) return BC_PUSH;
    return BC_PULL;
}

// Picks the forward shape of level st->d (force >= 0 overrides) and logs the
// level's features when feat_log is given.
// One warp: the lanes stage the model's weights in shared memory, lane 0
// decides.
__global__ void k_bc_choose(BcState *st, int force, int sched, int64_t m, int64_t nnz, int W, float *feat_log,
                            int log_cap) {
    // one warp: the model's hidden units one per lane (mlp_forward_warp2)
    __shared__ float sw[MLP_SIZE];
    const bool learned = force < 0 && sched == GK_SCHED_LEARNED;
    const int lane = threadIdx.x & 31;
    float f[BC_FEAT];
    bc_features(st, m, nnz, W, f);
    int mode;
    if (force >= 0) {
        mode = force;
    } else if (learned) {
        for (int i = lane; i < MLP_SIZE; i += 32) sw[i] = d_mlp_bc[i];
        __syncwarp();
        // the plain rule's shape unless the model predicts the other one at
        // least 10% faster (the row-bin scheduler's margin)
        float o[2];
        mlp_forward_warp2(sw, f, &o[0], &o[1]);
        const int plain = bc_plain_shape(st, m, nnz, W);
        mode = o[plain] - o[1 - plain] >= 0.1375f ? 1 - plain : plain;
    } else {
        mode = bc_plain_shape(st, m, nnz, W);
    }
    __syncwarp();  // every lane has read the state before lane 0 updates it
    if (lane != 0) return;
    st->mode = mode;
    if (mode == BC_PUSH) ++st->pushes;
    else ++st->pulls;
    const int d = st->d;
    if (feat_log && d >= 1 && d <= log_cap)
        for (int i = 0; i < BC_FEAT; ++i) feat_log[(d - 1) * BC_FEAT + i] = f[i];
}

// ---------------------------------------------------------------------------
// forward, pull: in-neighbours (AT) of a vertex with open sources
// ---------------------------------------------------------------------------
// Copies the warp's T selection words (equal in every lane) to its slot in
// shared memory, so that they take no registers through a gather.
template <int T>
__device__ __forceinline__ const uint32_t *stage_sel(uint32_t *slot, const uint32_t (&x)[T], int lane) {
    __syncwarp();
#pragma unroll
    for (int t = 0; t < T; ++t)
        if (lane == t) slot[t] = x[t];
    __syncwarp();
    return slot;
}

// Position of the k-th set bit (from 0) of x, which has more than k set bits.
__device__ __forceinline__ int nth_set_bit(uint32_t x, int k) {
    int p = 0;
    int c = __popc(x & 0xFFFFu);
    if (k >= c) { k -= c; x >>= 16; p += 16; }
    c = __popc(x & 0xFFu);
    if (k >= c) { k -= c; x >>= 8; p += 8; }
    c = __popc(x & 0xFu);
    if (k >= c) { k -= c; x >>= 4; p += 4; }
    c = __popc(x & 0x3u);
    if (k >= c) { k -= c; x >>= 2; p += 2; }
    if (k >= static_cast<int>(x & 1u)) p += 1;
    return p;
}

// Pull gather over the edges [ebeg, e1) of one vertex, 32 edges per warp step
// (estep between a warp's steps).  The edge to neighbour w = G.col[e] carries
// the hits F[w][t] & sel[t] (sel: the warp's T words in shared memory): source
// s = 32 t + l hits when bit l of that word is set, and each hit adds
// a_e * X[w W + s] into the warp's accumulator of source s (acc: the warp's
// T x 32 slice in shared memory, source s at s).  Where a step's hits are
// sparse (at most GK_BC_DENSE_HITS per hit edge on average) they are numbered
// in (edge, word, bit) order and taken 32 at a time, one per lane, so that a
// load instruction carries 32 hits however few sources each (edge, word)
// holds (typically 1.5 to 6 of 32), and the step costs one load latency per
// 32 hits instead of one per hit edge.  Every source's sum is taken in edge
// order: the hits of one source within a batch belong to different edges and
// are applied in lane order.  Returns whether any edge hit (the same in every
// lane).
template <int T>
__device__ __forceinline__ bool pull_gather(const DevCsr &G, int64_t ebeg, int64_t e1, int64_t estep,
                                            const uint32_t *__restrict__ F, const uint32_t *sel,
                                            const double *__restrict__ X, int W, int lane, double *acc) {
    constexpr unsigned FULL = 0xFFFFFFFFu;
    bool any = false;
    for (int64_t base = ebeg; base < e1; base += estep) {
        const int64_t e = base + lane;
        int w = 0;
        uint32_t h[T];
#pragma unroll
        for (int t = 0; t < T; ++t) h[t] = 0u;
        if (e < e1) {
            w = __ldg(G.col + e);
            load_words<T>(F + (int64_t)w * T, h);
#pragma unroll
            for (int t = 0; t < T; ++t) h[t] &= sel[t];
        }
        int c = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) c += __popc(h[t]);
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        const int n = __shfl_sync(FULL, incl, 31);
        if (n) any = true;
        const unsigned edges = __ballot_sync(FULL, c > 0);
        if (n > GK_BC_DENSE_HITS * __popc(edges)) {
            // dense hits (more than GK_BC_DENSE_HITS per hit edge, as at a
            // hub's middle levels): one edge at a time, one load per source
            // word, each carrying many hits, without the per-hit search
            for (unsigned bal = edges; bal; bal &= bal - 1) {
                const int j = __ffs(bal) - 1;
                const int wj = __shfl_sync(FULL, w, j);
                const double a = G.val ? static_cast<double>(__ldg(G.val + base + j)) : 1.0;
                const double *__restrict__ xw = X + (int64_t)wj * W + lane;
#pragma unroll
                for (int t = 0; t < T; ++t) {
                    const uint32_t bits = __shfl_sync(FULL, h[t], j);
                    if ((bits >> lane) & 1u) acc[32 * t + lane] += a * __ldg(xw + 32 * t);
                }
            }
            __syncwarp();
            continue;
        }
        const int excl = incl - c;
        for (int q0 = 0; q0 < n; q0 += 32) {
            const int q = q0 + lane;
            // j = the lane (edge) holding hit q: lanes below j end at or before q
            int j = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1)
                if (__shfl_sync(FULL, incl, j + step - 1) <= q) j += step;
            int r = q - __shfl_sync(FULL, excl, j);
            const int wj = __shfl_sync(FULL, w, j);
            uint32_t word = 0u;
            int tt = 0, rk = 0;
#pragma unroll
            for (int t = 0; t < T; ++t) {
                const uint32_t x = __shfl_sync(FULL, h[t], j);
                const int p = __popc(x);
                if (r >= 0 && r < p) {
                    word = x;
                    tt = t;
                    rk = r;
                }
                r -= p;
            }
            const bool ok = q < n;
            const int s = 32 * tt + nth_set_bit(word, rk);
            double v = 0.0, a = 1.0;
            if (ok) {
                v = __ldg(X + (int64_t)wj * W + s);
                if (G.val) a = static_cast<double>(__ldg(G.val + base + j));
            }
            const int jlast = __shfl_sync(FULL, j, min(n - q0, 32) - 1);
            if (__shfl_sync(FULL, j, 0) == jlast) {
                if (ok) acc[s] += a * v;  // one edge: distinct sources
            } else {
                const unsigned same = __match_any_sync(FULL, ok ? static_cast<unsigned>(s) : W + lane);
                const unsigned rank = __popc(same & ((1u << lane) - 1u));
                const unsigned rounds = __reduce_max_sync(FULL, ok ? rank : 0u);
                for (unsigned k = 0; k <= rounds; ++k) {
                    if (ok && rank == k) acc[s] += a * v;
                    __syncwarp();
                }
            }
            __syncwarp();
        }
    }
    return any;
}

// New level bits, sigma and visited words of vertex i; returns the number of
// new (vertex, source) pairs (valid in every lane).
// V[i] is written only by the warp that emits vertex i, so its visited words
// are re-read here rather than carried in registers through the gather.
template <int T, class AccT>
__device__ __forceinline__ int pull_emit(int64_t i, int W, int lane, const AccT &acc, uint32_t *Fn, uint32_t *V,
                                         double *sigma) {
    int c = 0;
#pragma unroll
    for (int t = 0; t < T; ++t) {
        const double a = acc[t];
        const uint32_t nb = __ballot_sync(0xFFFFFFFFu, a != 0.0);
        c += __popc(nb);
        if ((nb >> lane) & 1u) sigma[i * W + 32 * t + lane] = a;
        if (lane == t) {
            Fn[i * T + t] = nb;
            V[i * T + t] |= nb;
        }
    }
    return c;
}

template <int T>
__global__ void __launch_bounds__(256, GK_BC_MINB) k_bc_pull(DevCsr AT, DevCsr A, BcState *st, uint32_t *V,
                                                             double *sigma, int W, const uint32_t *act) {
    if (st->mode != BC_PULL) return;
    const int d = st->d;
    const uint32_t *__restrict__ Fd = st->fptr[d];
    uint32_t *Fn = st->fptr[d + 1];
    const int lane = threadIdx.x & 31;
    __shared__ double s_acc[8][T][32];
    __shared__ uint32_t s_sel[8][T];
    SmemAcc acc{&s_acc[threadIdx.x >> 5][0][lane]};
    unsigned long long n = 0, e = 0, b = 0;
    for (int64_t base = grab_vertices(&st->cur_pull, lane); base < AT.m; base = grab_vertices(&st->cur_pull, lane))
    for (int64_t i = base, iend = min(base + BC_GRAB, AT.m); i < iend; ++i) {
        const int64_t e0 = AT.rp[i], e1 = AT.rp[i + 1];
        if (e0 == e1 || e1 - e0 > BC_HEAVY) continue;
        uint32_t need[T];
        load_words<T>(V + i * T, need);
        uint32_t open = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) {
            need[t] = ~need[t] & act[t];
            open |= need[t];
        }
        if (!open) continue;
#pragma unroll
        for (int t = 0; t < T; ++t) acc[t] = 0.0;
        const uint32_t *sel = stage_sel<T>(s_sel[threadIdx.x >> 5], need, lane);
        if (!pull_gather<T>(AT, e0, e1, 32, Fd, sel, sigma, W, lane, acc.warp_base(lane))) continue;
        const int c = pull_emit<T>(i, W, lane, acc, Fn, V, sigma);
        if (c && lane == 0) {
            ++n;
            e += static_cast<unsigned long long>(A.rp[i + 1] - A.rp[i]);
            b += c;
        }
    }
    add_level_stats(n, e, b, &st->nn);
}

// Sums the NW warps' T x 32 partial sums of a CTA (each warp accumulated into
// its own slice of part) into dst[32 t + lane], in warp order.
template <int T>
__device__ __forceinline__ void cta_reduce_store(double (*part)[T][32], int warp, int lane, double *dst) {
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int t = 0; t < T; ++t) {
            double sum = 0.0;
            for (int w = 0; w < BC_NW_HEAVY; ++w) sum += part[w][t][lane];
            dst[32 * t + lane] = sum;
        }
    }
}

// Resident CTAs per SM of the heavy-vertex item kernels: their per-lane
// partial sums live in the CTA's reduction buffer (shared memory), not in
// registers, so four 8-warp CTAs fit (64 registers a thread).
constexpr int BC_ITEM_MINB = 4;

template <int T>
__global__ void __launch_bounds__(BC_NW_HEAVY * 32, BC_ITEM_MINB) k_bc_pull_items(DevCsr AT, HeavySet hs, BcState *st,
                                                                    const uint32_t *V, const double *sigma, int W,
                                                                    const uint32_t *act, double *partials) {
    if (st->mode != BC_PULL) return;
    __shared__ double part[BC_NW_HEAVY][T][32];
    __shared__ uint32_t s_sel[BC_NW_HEAVY][T];
    const uint32_t *__restrict__ Fd = st->fptr[st->d];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int it = next_item(&st->cur_ipull); it < hs.items; it = next_item(&st->cur_ipull)) {
        const int h = hs.item_h[it];
        const int64_t i = hs.list[h];
        const int64_t e0 = AT.rp[i] + static_cast<int64_t>(it - hs.first[h]) * BC_ITEM_EDGES;
        const int64_t e1 = min(AT.rp[i + 1], e0 + BC_ITEM_EDGES);
        uint32_t vis[T], need[T];
        load_words<T>(V + i * T, vis);
        uint32_t open = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) {
            need[t] = ~vis[t] & act[t];
            open |= need[t];
        }
        if (!open) continue;  // uniform across the CTA (the emit kernel skips the vertex too)
        SmemAcc acc{&part[warp][0][lane]};
#pragma unroll
        for (int t = 0; t < T; ++t) acc[t] = 0.0;
        const uint32_t *sel = stage_sel<T>(s_sel[warp], need, lane);
        pull_gather<T>(AT, e0 + 32 * warp, e1, 32 * BC_NW_HEAVY, Fd, sel, sigma, W, lane, acc.warp_base(lane));
        cta_reduce_store<T>(part, warp, lane, partials + (int64_t)it * W);
        __syncthreads();
    }
}

template <int T>
__global__ void __launch_bounds__(256) k_bc_pull_heavy_emit(DevCsr A, HeavySet hs, BcState *st, uint32_t *V,
                                                            double *sigma, int W, const uint32_t *act,
                                                            const double *partials) {
    if (st->mode != BC_PULL) return;
    uint32_t *Fn = st->fptr[st->d + 1];
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    unsigned long long n = 0, e = 0, b = 0;
    for (int h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; h < hs.n; h += warps) {
        const int64_t i = hs.list[h];
        uint32_t vis[T];
        load_words<T>(V + i * T, vis);
        uint32_t open = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) open |= ~vis[t] & act[t];
        if (!open) continue;
        double acc[T];
#pragma unroll
        for (int t = 0; t < T; ++t) acc[t] = 0.0;
        for (int it = hs.first[h]; it < hs.first[h + 1]; ++it) {
#pragma unroll
            for (int t = 0; t < T; ++t) acc[t] += partials[(int64_t)it * W + 32 * t + lane];
        }
        const int c = pull_emit<T>(i, W, lane, acc, Fn, V, sigma);
        if (c && lane == 0) {
            ++n;
            e += static_cast<unsigned long long>(A.rp[i + 1] - A.rp[i]);
            b += c;
        }
    }
    add_level_stats(n, e, b, &st->nn);
}

// ---------------------------------------------------------------------------
// forward, push: out-neighbours (A) of frontier vertices
// ---------------------------------------------------------------------------
// V is the visited state before this level (updated by k_bc_push_finish), so
// every depth-d predecessor of a new vertex adds its sigma.
template <int T>
__device__ __forceinline__ void push_sigma(const DevCsr &A, int64_t ebeg, int64_t e1, int64_t estep,
                                           const uint32_t (&fu)[T], const double (&su)[T],
                                           const uint32_t *__restrict__ V, double *sigma, uint32_t *Fn, int W,
                                           int T_, int lane) {
    for (int64_t base = ebeg; base < e1; base += estep) {
        const int64_t e = base + lane;
        int v = 0;
        uint32_t hitw = 0;
        if (e < e1) {
            v = __ldg(A.col + e);
            uint32_t w[T];
            load_words<T>(V + (int64_t)v * T, w);
#pragma unroll
            for (int t = 0; t < T; ++t) hitw |= fu[t] & ~w[t];
        }
        unsigned bal = __ballot_sync(0xFFFFFFFFu, hitw != 0);
        while (bal) {
            const int j = __ffs(bal) - 1;
            bal &= bal - 1;
            const int vv = __shfl_sync(0xFFFFFFFFu, v, j);
            const double a = A.val ? static_cast<double>(__ldg(A.val + base + j)) : 1.0;
            uint32_t w[T];
            load_words<T>(V + (int64_t)vv * T, w);
            double *sv = sigma + (int64_t)vv * W + lane;
            uint32_t mine = 0;
#pragma unroll
            for (int t = 0; t < T; ++t) {
                const uint32_t bits = fu[t] & ~w[t];
                if (bits) {
                    if ((bits >> lane) & 1u) atomicAdd(sv + 32 * t, a * su[t]);
                    if (lane == t) mine = bits;
                }
            }
            if (mine) atomicOr(Fn + (int64_t)vv * T_ + lane, mine);
        }
    }
}

template <int T>
__device__ __forceinline__ bool push_source(int64_t u, const uint32_t *__restrict__ Fd, const double *sigma, int W,
                                            int lane, uint32_t (&fu)[T], double (&su)[T]) {
    load_words<T>(Fd + u * T, fu);
    uint32_t any = 0;
#pragma unroll
    for (int t = 0; t < T; ++t) {
        any |= fu[t];
        su[t] = ((fu[t] >> lane) & 1u) ? sigma[u * W + 32 * t + lane] : 0.0;
    }
    return any != 0;
}

template <int T>
__global__ void __launch_bounds__(256, GK_BC_MINB) k_bc_push(DevCsr A, BcState *st, const uint32_t *V, double *sigma, int W) {
    if (st->mode != BC_PUSH) return;
    const int d = st->d;
    const uint32_t *__restrict__ Fd = st->fptr[d];
    uint32_t *Fn = st->fptr[d + 1];
    const int lane = threadIdx.x & 31;
    for (int64_t base = grab_vertices(&st->cur_push, lane); base < A.m; base = grab_vertices(&st->cur_push, lane))
    for (int64_t u = base, uend = min(base + BC_GRAB, A.m); u < uend; ++u) {
        const int64_t e0 = A.rp[u], e1 = A.rp[u + 1];
        if (e0 == e1 || e1 - e0 > BC_HEAVY) continue;
        uint32_t fu[T];
        double su[T];
        if (!push_source<T>(u, Fd, sigma, W, lane, fu, su)) continue;
        push_sigma<T>(A, e0, e1, 32, fu, su, V, sigma, Fn, W, T, lane);
    }
}

template <int T>
__global__ void __launch_bounds__(BC_NW_HEAVY * 32) k_bc_push_items(DevCsr A, HeavySet hs, BcState *st,
                                                                    const uint32_t *V, double *sigma, int W) {
    if (st->mode != BC_PUSH) return;
    const int d = st->d;
    const uint32_t *__restrict__ Fd = st->fptr[d];
    uint32_t *Fn = st->fptr[d + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int it = next_item(&st->cur_ipush); it < hs.items; it = next_item(&st->cur_ipush)) {
        const int h = hs.item_h[it];
        const int64_t u = hs.list[h];
        const int64_t e0 = A.rp[u] + static_cast<int64_t>(it - hs.first[h]) * BC_ITEM_EDGES;
        const int64_t e1 = min(A.rp[u + 1], e0 + BC_ITEM_EDGES);
        uint32_t fu[T];
        double su[T];
        if (!push_source<T>(u, Fd, sigma, W, lane, fu, su)) continue;
        push_sigma<T>(A, e0 + 32 * warp, e1, 32 * BC_NW_HEAVY, fu, su, V, sigma, Fn, W, T, lane);
    }
}

// After a push level: V |= F_{d+1} and the statistics of F_{d+1}.
template <int T>
__global__ void k_bc_push_finish(DevCsr A, BcState *st, uint32_t *V) {
    if (st->mode != BC_PUSH) return;
    const uint32_t *__restrict__ Fn = st->fptr[st->d + 1];
    unsigned long long n = 0, e = 0, b = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < A.m; v += stride) {
        uint32_t f[T];
        load_words_rw<T>(Fn + v * T, f);
        int c = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) c += __popc(f[t]);
        if (c) {
#pragma unroll
            for (int t = 0; t < T; ++t) V[v * T + t] |= f[t];
            ++n;
            e += static_cast<unsigned long long>(A.rp[v + 1] - A.rp[v]);
            b += c;
        }
    }
    add_level_stats(n, e, b, &st->nn);
}

// End of a forward level: an empty F_{d+1} ends the sweep (F_1..F_d are the
// BFS layers); otherwise F_{d+1} becomes the frontier.  Inside the graph the
// loop continues while a bitmap for the next level is allocated.
__global__ void k_bc_fwd_end(BcState *st, int64_t max_depth, cudaGraphConditionalHandle h, int in_graph) {
    int more = 0;
    if (st->nn == 0) {
        st->done = 1;
    } else {
        st->visited += st->bn;
        st->nf = st->nn;
        st->ef = st->en;
        st->bf = st->bn;
        st->d += 1;
        more = (st->d + 1 <= st->levels && st->d < max_depth) ? 1 : 0;
    }
    st->nn = st->en = st->bn = 0;
    st->cur_pull = st->cur_push = 0;
    st->cur_ipull = st->cur_ipush = 0;
    if (in_graph) cudaGraphSetConditional(h, static_cast<unsigned>(more));
}

// ---------------------------------------------------------------------------
// backward: R = (1 + delta) / sigma from level D up to level 1
// ---------------------------------------------------------------------------
// deepest level: R = 1/sigma (Bcu = 1 there)
template <int T>
__global__ void k_bc_rinit(int64_t m, const BcState *st, const double *sigma, double *R, int W) {
    const uint32_t *__restrict__ Fd = st->fptr[st->d];
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < m; v += warps) {
        uint32_t f[T];
        load_words<T>(Fd + v * T, f);
#pragma unroll
        for (int t = 0; t < T; ++t)
            if ((f[t] >> lane) & 1u) R[v * W + 32 * t + lane] = 1.0 / sigma[v * W + 32 * t + lane];
    }
}

template <int T, class AccT>
__device__ __forceinline__ void bwd_emit(int64_t v, int W, int lane, const uint32_t (&fv)[T], const AccT &sum,
                                         const double *sigma, double *R, double *bc) {
    double tot = 0.0;
#pragma unroll
    for (int t = 0; t < T; ++t) {
        if ((fv[t] >> lane) & 1u) {
            const int64_t o = v * W + 32 * t + lane;
            const double sg = sigma[o];
            const double delta = sg * sum[t];
            R[o] = (1.0 + delta) / sg;
            tot += delta;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xFFFFFFFFu, tot, o);
    if (lane == 0) bc[v] += tot;
}

template <int T>
__global__ void __launch_bounds__(256, GK_BC_MINB) k_bc_backward(DevCsr A, BcState *st, const double *sigma,
                                                                 double *R, int W, double *bc) {
    const int d = st->bd;
    const uint32_t *__restrict__ Fd = st->fptr[d];
    const uint32_t *__restrict__ Fn = st->fptr[d + 1];
    const int lane = threadIdx.x & 31;
    __shared__ double s_sum[8][T][32];
    __shared__ uint32_t s_sel[8][T];
    SmemAcc sum{&s_sum[threadIdx.x >> 5][0][lane]};
    for (int64_t base = grab_vertices(&st->cur_bwd, lane); base < A.m; base = grab_vertices(&st->cur_bwd, lane))
    for (int64_t v = base, vend = min(base + BC_GRAB, A.m); v < vend; ++v) {
        const int64_t e0 = A.rp[v], e1 = A.rp[v + 1];
        if (e1 - e0 > BC_HEAVY) continue;
        uint32_t fv[T];
        load_words<T>(Fd + v * T, fv);
        uint32_t any = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) any |= fv[t];
        if (!any) continue;
#pragma unroll
        for (int t = 0; t < T; ++t) sum[t] = 0.0;
        const uint32_t *sel = stage_sel<T>(s_sel[threadIdx.x >> 5], fv, lane);
        pull_gather<T>(A, e0, e1, 32, Fn, sel, R, W, lane, sum.warp_base(lane));
#pragma unroll
        for (int t = 0; t < T; ++t) fv[t] = sel[t];
        bwd_emit<T>(v, W, lane, fv, sum, sigma, R, bc);
    }
}

template <int T>
__global__ void __launch_bounds__(BC_NW_HEAVY * 32, BC_ITEM_MINB) k_bc_backward_items(DevCsr A, HeavySet hs,
                                                                                     BcState *st,
                                                                        const double *R, int W, double *partials) {
    __shared__ double part[BC_NW_HEAVY][T][32];
    __shared__ uint32_t s_sel[BC_NW_HEAVY][T];
    const int d = st->bd;
    const uint32_t *__restrict__ Fd = st->fptr[d];
    const uint32_t *__restrict__ Fn = st->fptr[d + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int it = next_item(&st->cur_ibwd); it < hs.items; it = next_item(&st->cur_ibwd)) {
        const int h = hs.item_h[it];
        const int64_t v = hs.list[h];
        const int64_t e0 = A.rp[v] + static_cast<int64_t>(it - hs.first[h]) * BC_ITEM_EDGES;
        const int64_t e1 = min(A.rp[v + 1], e0 + BC_ITEM_EDGES);
        uint32_t fv[T];
        load_words<T>(Fd + v * T, fv);
        uint32_t any = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) any |= fv[t];
        if (!any) continue;
        SmemAcc sum{&part[warp][0][lane]};
#pragma unroll
        for (int t = 0; t < T; ++t) sum[t] = 0.0;
        const uint32_t *sel = stage_sel<T>(s_sel[warp], fv, lane);
        pull_gather<T>(A, e0 + 32 * warp, e1, 32 * BC_NW_HEAVY, Fn, sel, R, W, lane, sum.warp_base(lane));
        cta_reduce_store<T>(part, warp, lane, partials + (int64_t)it * W);
        __syncthreads();
    }
}

template <int T>
__global__ void __launch_bounds__(256) k_bc_backward_heavy_emit(HeavySet hs, const BcState *st, const double *sigma,
                                                                double *R, int W, double *bc,
                                                                const double *partials) {
    const uint32_t *__restrict__ Fd = st->fptr[st->bd];
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; h < hs.n; h += warps) {
        const int64_t v = hs.list[h];
        uint32_t fv[T];
        load_words<T>(Fd + v * T, fv);
        uint32_t any = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) any |= fv[t];
        if (!any) continue;
        double sum[T];
#pragma unroll
        for (int t = 0; t < T; ++t) sum[t] = 0.0;
        for (int it = hs.first[h]; it < hs.first[h + 1]; ++it) {
#pragma unroll
            for (int t = 0; t < T; ++t) sum[t] += partials[(int64_t)it * W + 32 * t + lane];
        }
        bwd_emit<T>(v, W, lane, fv, sum, sigma, R, bc);
    }
}

__global__ void k_bc_bwd_end(BcState *st, cudaGraphConditionalHandle h, int in_graph) {
    st->bd -= 1;
    st->cur_bwd = 0;
    st->cur_ibwd = 0;
    if (in_graph) cudaGraphSetConditional(h, st->bd >= 1 ? 1u : 0u);
}

// Row index of every entry (a warp per row), for the per-entry check below.
__global__ void k_bc_entry_rows(DevCsr A, int32_t *row) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < A.m; i += warps)
        for (int64_t p = A.rp[i] + lane; p < A.rp[i + 1]; p += 32) row[p] = static_cast<int32_t>(i);
}

// Symmetry of a pattern with sorted rows.  out[0] = 1 when a row is not
// strictly increasing or an entry (i, j > i) has no mirror (j, i); out[1] and
// out[2] count the entries above and below the diagonal.  Every upper entry
// having its mirror maps the upper entries one to one onto lower ones (no
// duplicates), so equal counts mean that the pattern equals its transpose
// entry for entry; only the upper half is searched.  A thread per entry, one
// binary search of i in row j (a warp per row would serialise on a hub's).
__global__ void k_bc_mirror_check(DevCsr A, const int32_t *row, unsigned long long *out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned up = 0, lo_cnt = 0;
    bool bad = false;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < A.nnz; p += stride) {
        const int i = row[p], j = A.col[p];
        if (p + 1 < A.rp[i + 1] && A.col[p + 1] <= j) bad = true;
        if (j < i) ++lo_cnt;
        if (j <= i) continue;
        ++up;
        int64_t lo = A.rp[j], hi = A.rp[j + 1];
        const int64_t end = hi;
        while (lo < hi) {
            const int64_t md = (lo + hi) >> 1;
            if (A.col[md] < i) lo = md + 1;
            else hi = md;
        }
        if (lo == end || A.col[lo] != i) bad = true;
    }
    if (bad) atomicExch(out, 1ull);
    up = __reduce_add_sync(0xFFFFFFFFu, up);
    lo_cnt = __reduce_add_sync(0xFFFFFFFFu, lo_cnt);
    if ((threadIdx.x & 31) == 0) {
        if (up) atomicAdd(out + 1, static_cast<unsigned long long>(up));
        if (lo_cnt) atomicAdd(out + 2, static_cast<unsigned long long>(lo_cnt));
    }
}

__global__ void k_heavy_list(DevCsr A, int32_t *list, int *count) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < A.m; i += stride)
        if (A.rp[i + 1] - A.rp[i] > BC_HEAVY) list[atomicAdd(count, 1)] = static_cast<int32_t>(i);
}

__global__ void k_heavy_item_counts(DevCsr A, const int32_t *list, int n, int32_t *cnt) {
    for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < n; h += gridDim.x * blockDim.x) {
        const int64_t v = list[h];
        cnt[h] = static_cast<int32_t>((A.rp[v + 1] - A.rp[v] + BC_ITEM_EDGES - 1) / BC_ITEM_EDGES);
    }
}

__global__ void k_heavy_items(const int32_t *first, int n, int32_t *item_h) {
    for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < n; h += gridDim.x * blockDim.x)
        for (int it = first[h]; it < first[h + 1]; ++it) item_h[it] = h;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct BcBuffers {
    DevCsr A, AT;
    HeavySet hA, hAT;  // heavy vertices of A (push, backward) and of AT (pull)
};

// Options of a BC run: scheduler, a forced forward shape (autotuning), and
// per-level logs of the forward levels (host arrays, may be null).
struct BcOptions {
    int sched = GK_SCHED_PLAIN;
    int force = -1;
    bool host_loop = false;  // drive the levels from the host (always with logging)
    float *level_ms = nullptr;
    float *level_feat = nullptr;
    int *level_mode = nullptr;
    int log_cap = 0;
    int *levels_out = nullptr;
};

// A captured level loop: a graph with one conditional while node.
class LevelGraph {
public:
    ~LevelGraph() {
        if (exec_) cudaGraphExecDestroy(exec_);
        if (g_) cudaGraphDestroy(g_);
        if (cs_) cudaStreamDestroy(cs_);
    }
    // Starts capturing the loop body; returns false where conditional graphs
    // are unavailable.
    bool begin(cudaGraphConditionalHandle *h) {
        if (cudaGraphCreate(&g_, 0) != cudaSuccess) return false;
        if (cudaGraphConditionalHandleCreate(h, g_, 1, cudaGraphCondAssignDefault) != cudaSuccess) return false;
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = *h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        if (cudaGraphAddNode(&node, g_, nullptr, 0, &np) != cudaSuccess) return false;
        if (cudaStreamCreateWithFlags(&cs_, cudaStreamNonBlocking) != cudaSuccess) return false;
        if (cudaStreamBeginCaptureToGraph(cs_, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return false;
        capturing_ = true;
        return true;
    }
    cudaStream_t stream() const { return cs_; }
    int end() {
        cudaGraph_t body = nullptr;
        capturing_ = false;
        cudaError_t e = cudaStreamEndCapture(cs_, &body);
        if (e != cudaSuccess) return cuda_fail(e, "BC level capture");
        e = cudaGraphInstantiate(&exec_, g_, 0);
        if (e != cudaSuccess) return cuda_fail(e, "BC level graph instantiate");
        return GK_OK;
    }
    void abort() {
        if (capturing_) {
            cudaGraph_t body = nullptr;
            cudaStreamEndCapture(cs_, &body);
            capturing_ = false;
        }
        cudaGetLastError();
    }
    int launch(cudaStream_t s) {
        cudaError_t e = cudaGraphLaunch(exec_, s);
        return e == cudaSuccess ? GK_OK : cuda_fail(e, "BC level graph launch");
    }

private:
    cudaGraph_t g_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    cudaStream_t cs_ = nullptr;
    bool capturing_ = false;
};

template <int T>
static int bc_chunk(const BcBuffers &g, const int32_t *src, int nsrc, double *bc, const BcOptions &opt,
                    cudaStream_t s) {
    constexpr int W = 32 * T;
    const int64_t m = g.A.m;
    const int64_t nnz = g.A.nnz;
    const int sms = ctx().num_sms;
    double *sigma, *R;
    uint32_t *V, *act;
    BcState *st;
    uint32_t **fptr_dev;
    float *feat_dev = nullptr;
    Scratch local(s);
    GK_CHECK(local.alloc(&sigma, (size_t)m * W));
    GK_CHECK(local.alloc(&R, (size_t)m * W));
    GK_CHECK(local.alloc(&V, (size_t)m * T));
    GK_CHECK(local.alloc(&act, T));
    GK_CHECK(local.alloc(&st, 1));
    if (opt.level_feat && opt.log_cap > 0) GK_CHECK(local.alloc(&feat_dev, (size_t)opt.log_cap * BC_FEAT));
    double *partials;  // per heavy item: W partial sums
    {
        const int items = g.hA.items > g.hAT.items ? g.hA.items : g.hAT.items;
        GK_CHECK(local.alloc(&partials, (size_t)(items > 0 ? items : 1) * W));
    }
    GK_CUDA(cudaMemsetAsync(V, 0, sizeof(uint32_t) * m * T, s));
    GK_CUDA(cudaMemsetAsync(sigma, 0, sizeof(double) * m * W, s));  // push levels add into it
    GK_CUDA(cudaMemsetAsync(st, 0, sizeof(BcState), s));
    uint32_t hact[16];
    for (int t = 0; t < T; ++t) {
        const int lo = 32 * t;
        const int cnt = nsrc - lo <= 0 ? 0 : (nsrc - lo >= 32 ? 32 : nsrc - lo);
        hact[t] = cnt == 32 ? 0xFFFFFFFFu : ((1u << cnt) - 1u);
    }
    GK_CUDA(cudaMemcpyAsync(act, hact, sizeof(uint32_t) * T, cudaMemcpyHostToDevice, s));

    // level bitmaps, allocated BC_LEVEL_BATCH at a time; fptr[0] unused
    std::vector<uint32_t *> levels(1, nullptr);
    size_t fcap = 0;
    fptr_dev = nullptr;
    auto release = [&]() {
        for (size_t i = 1; i < levels.size(); ++i) cudaFreeAsync(levels[i], s);
        if (fptr_dev) cudaFreeAsync(fptr_dev, s);
    };
    auto grow = [&]() -> int {
        const size_t want = levels.size() + BC_LEVEL_BATCH;
        for (int k = 0; k < BC_LEVEL_BATCH; ++k) {
            uint32_t *p = nullptr;
            cudaError_t e = cudaMallocAsync(&p, sizeof(uint32_t) * m * T, s);
            if (e != cudaSuccess) return cuda_fail(e, "BC level bitmap");
            levels.push_back(p);
            e = cudaMemsetAsync(p, 0, sizeof(uint32_t) * m * T, s);
            if (e != cudaSuccess) return cuda_fail(e, "BC level bitmap");
        }
        if (want > fcap) {
            uint32_t **np = nullptr;
            const size_t ncap = want * 2;
            cudaError_t e = cudaMallocAsync(&np, sizeof(uint32_t *) * ncap, s);
            if (e != cudaSuccess) return cuda_fail(e, "BC level table");
            if (fptr_dev) cudaFreeAsync(fptr_dev, s);
            fptr_dev = np;
            fcap = ncap;
        }
        cudaError_t e = cudaMemcpyAsync(fptr_dev, levels.data(), sizeof(uint32_t *) * levels.size(),
                                        cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&st->fptr, &fptr_dev, sizeof(uint32_t **), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_fail(e, "BC level table");
        const int nlev = static_cast<int>(levels.size()) - 1;
        // the host's pointer and level count must stay alive until the copies ran
        e = cudaMemcpyAsync(&st->levels, &nlev, sizeof(int), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(e, "BC level table");
        return GK_OK;
    };
    int status = GK_OK;
    do {
        if ((status = grow()) != GK_OK) break;
        k_bc_seed<<<sms * 4, 256, 0, s>>>(g.A, src, nsrc, T, W, levels[1], V, sigma);
        k_bc_first_stats<T><<<sms * 4, 256, 0, s>>>(g.A, levels[1], st, nsrc);
        {
            const int one = 1;
            GK_CUDA(cudaMemcpyAsync(&st->d, &one, sizeof(int), cudaMemcpyHostToDevice, s));
            GK_CUDA(cudaStreamSynchronize(s));
        }
        note_launches(2);

        // ---- forward levels ----
        auto fwd_level = [&](cudaStream_t ls, cudaGraphConditionalHandle h, bool in_graph) {
            k_bc_choose<<<1, 32, 0, ls>>>(st, opt.force, opt.sched, m, nnz, W, feat_dev, opt.log_cap);
            k_bc_pull<T><<<sms * 8, 256, 0, ls>>>(g.AT, g.A, st, V, sigma, W, act);
            int k = 0;
            if (g.hAT.n) {
                k_bc_pull_items<T><<<sms * BC_ITEM_MINB, BC_NW_HEAVY * 32, 0, ls>>>(g.AT, g.hAT, st, V, sigma, W, act,
                                                                                   partials);
                k_bc_pull_heavy_emit<T><<<sms, 256, 0, ls>>>(g.A, g.hAT, st, V, sigma, W, act, partials);
                k += 2;
            }
            k_bc_push<T><<<sms * 8, 256, 0, ls>>>(g.A, st, V, sigma, W);
            if (g.hA.n) {
                k_bc_push_items<T><<<sms * 2, BC_NW_HEAVY * 32, 0, ls>>>(g.A, g.hA, st, V, sigma, W);
                k += 1;
            }
            k_bc_push_finish<T><<<sms * 4, 256, 0, ls>>>(g.A, st, V);
            k_bc_fwd_end<<<1, 1, 0, ls>>>(st, m, h, in_graph ? 1 : 0);
            return 5 + k;
        };
        BcState hs{};
        bool graph_ok = !opt.host_loop && !prof_any();
        LevelGraph fg;
        cudaGraphConditionalHandle fh{};
        int per_level = 0;
        if (graph_ok) {
            graph_ok = fg.begin(&fh);
            if (graph_ok) {
                per_level = fwd_level(fg.stream(), fh, true);
                if (fg.end() != GK_OK) {
                    fg.abort();
                    graph_ok = false;
                }
            } else {
                fg.abort();
            }
        }
        int lvl_count = 0;
        std::vector<cudaEvent_t> evs;
        while (true) {
            GK_CUDA(cudaMemcpyAsync(&hs, st, sizeof(BcState), cudaMemcpyDeviceToHost, s));
            GK_CUDA(cudaStreamSynchronize(s));
            if (hs.done || hs.d >= m) break;
            if (hs.d + 1 > hs.levels) {
                if ((status = grow()) != GK_OK) break;
                continue;
            }
            if (graph_ok) {
                const int d0 = hs.d;
                if ((status = fg.launch(s)) != GK_OK) break;
                GK_CUDA(cudaMemcpyAsync(&hs, st, sizeof(BcState), cudaMemcpyDeviceToHost, s));
                GK_CUDA(cudaStreamSynchronize(s));
                note_launches(per_level * (hs.d - d0 + (hs.done ? 1 : 0)));
                if (hs.done) break;
                continue;
            }
            // host-driven level (profiling, autotuning, or no conditional graphs)
            cudaEvent_t a = nullptr, b = nullptr;
            if (opt.level_ms) {
                cudaEventCreate(&a);
                cudaEventCreate(&b);
                cudaEventRecord(a, s);
            }
            note_launches(fwd_level(s, cudaGraphConditionalHandle{}, false));
            if (opt.level_ms) {
                cudaEventRecord(b, s);
                evs.push_back(a);
                evs.push_back(b);
            }
            ++lvl_count;
        }
        if (status != GK_OK) break;
        if (opt.level_ms || opt.level_mode) {
            GK_CUDA(cudaStreamSynchronize(s));
            const int n = static_cast<int>(evs.size() / 2);
            for (int i = 0; i < n && i < opt.log_cap; ++i) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, evs[2 * i], evs[2 * i + 1]);
                if (opt.level_ms) opt.level_ms[i] = ms;
            }
            if (opt.levels_out) *opt.levels_out = n;
        }
        for (cudaEvent_t e : evs) cudaEventDestroy(e);
        if (opt.level_feat && feat_dev) {
            const int n = hs.d - 1 + (hs.done ? 1 : 0);
            const int k = n < opt.log_cap ? n : opt.log_cap;
            if (k > 0)
                GK_CUDA(cudaMemcpyAsync(opt.level_feat, feat_dev, sizeof(float) * k * BC_FEAT, cudaMemcpyDeviceToHost,
                                        s));
            GK_CUDA(cudaStreamSynchronize(s));
        }

        // ---- backward levels: D = hs.d ----
        const int D = hs.d;
        k_bc_rinit<T><<<sms * 8, 256, 0, s>>>(m, st, sigma, R, W);
        note_launches(1);
        if (D - 1 < 1) break;
        {
            const int bd = D - 1;
            GK_CUDA(cudaMemcpyAsync(&st->bd, &bd, sizeof(int), cudaMemcpyHostToDevice, s));
            GK_CUDA(cudaStreamSynchronize(s));
        }
        auto bwd_level = [&](cudaStream_t ls, cudaGraphConditionalHandle h, bool in_graph) {
            k_bc_backward<T><<<sms * 8, 256, 0, ls>>>(g.A, st, sigma, R, W, bc);
            int k = 0;
            if (g.hA.n) {
                k_bc_backward_items<T><<<sms * BC_ITEM_MINB, BC_NW_HEAVY * 32, 0, ls>>>(g.A, g.hA, st, R, W, partials);
                k_bc_backward_heavy_emit<T><<<sms, 256, 0, ls>>>(g.hA, st, sigma, R, W, bc, partials);
                k += 2;
            }
            k_bc_bwd_end<<<1, 1, 0, ls>>>(st, h, in_graph ? 1 : 0);
            return 2 + k;
        };
        bool bgraph = !opt.host_loop && !prof_any();
        LevelGraph bg;
        cudaGraphConditionalHandle bh{};
        int per_b = 0;
        if (bgraph) {
            bgraph = bg.begin(&bh);
            if (bgraph) {
                per_b = bwd_level(bg.stream(), bh, true);
                if (bg.end() != GK_OK) {
                    bg.abort();
                    bgraph = false;
                }
            } else {
                bg.abort();
            }
        }
        if (bgraph) {
            if ((status = bg.launch(s)) != GK_OK) break;
            note_launches(per_b * (D - 1));
        } else {
            for (int d = D - 1; d >= 1; --d) note_launches(bwd_level(s, cudaGraphConditionalHandle{}, false));
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) status = cuda_fail(e, "BC backward");
    } while (false);
    cudaError_t e = cudaStreamSynchronize(s);
    release();
    if (status == GK_OK && e != cudaSuccess) status = cuda_fail(e, "BC chunk");
    return status;
}

static int ensure_bc_model(int sched) {
    if (sched != GK_SCHED_LEARNED) return GK_OK;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(g_bc_model_mutex);
    if (g_bc_model.empty())
        return fail(GK_ERR_ARG, "learned BC scheduling requested but no model is loaded (gk_bc_set_model)");
    if (g_bc_uploaded[dev & 63] != g_bc_model_version) {
        GK_CUDA(cudaMemcpyToSymbol(d_mlp_bc, g_bc_model.data(), sizeof(float) * MLP_SIZE));
        g_bc_uploaded[dev & 63] = g_bc_model_version;
    }
    return GK_OK;
}

// Heavy vertices of G and their work items (synchronises once for the counts).
static int heavy_set(const DevCsr &G, HeavySet *hs, cudaStream_t s, Scratch &scr) {
    const int sms = ctx().num_sms;
    int32_t *list, *cnt, *first, *item_h;
    int *n_dev;
    GK_CHECK(scr.alloc(&list, G.m > 0 ? G.m : 1));
    GK_CHECK(scr.alloc(&n_dev, 1));
    GK_CUDA(cudaMemsetAsync(n_dev, 0, sizeof(int), s));
    k_heavy_list<<<sms * 4, 256, 0, s>>>(G, list, n_dev);
    int n = 0;
    GK_CUDA(cudaMemcpyAsync(&n, n_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaStreamSynchronize(s));
    note_launches(1);
    hs->list = list;
    hs->n = n;
    hs->items = 0;
    GK_CHECK(scr.alloc(&cnt, n + 1));
    GK_CHECK(scr.alloc(&first, n + 1));
    GK_CUDA(cudaMemsetAsync(cnt + n, 0, sizeof(int32_t), s));
    if (n > 0) {
        k_heavy_item_counts<<<ceil_div(n, 256), 256, 0, s>>>(G, list, n, cnt);
        note_launches(1);
    }
    size_t tb = 0;
    GK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, first, n + 1, s));
    void *tmp;
    GK_CHECK(scr.alloc(reinterpret_cast<char **>(&tmp), tb));
    GK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, first, n + 1, s));
    int items = 0;
    GK_CUDA(cudaMemcpyAsync(&items, first + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaStreamSynchronize(s));
    GK_CHECK(scr.alloc(&item_h, items > 0 ? items : 1));
    if (n > 0) {
        k_heavy_items<<<ceil_div(n, 256), 256, 0, s>>>(first, n, item_h);
        note_launches(1);
    }
    hs->first = first;
    hs->item_h = item_h;
    hs->items = items;
    return GK_OK;
}

int bc_device(const DevCsr &A, const int32_t *src, int nsrc, double *bc, const BcOptions &opt, cudaStream_t s,
              Scratch &scr) {
    if (opt.sched != GK_SCHED_PLAIN && opt.sched != GK_SCHED_LEARNED) return fail(GK_ERR_ARG, "unknown scheduler mode");
    GK_CHECK(ensure_bc_model(opt.sched));
    const int sms = ctx().num_sms;
    BcBuffers g;
    g.A = A;
    // The pull shapes read A's transpose.  A pattern (no values) with sorted
    // rows that equals its transpose (an undirected graph) is its own: the
    // radix-sort transpose and the second heavy-vertex set are then skipped.
    bool self_transpose = false;
    if (!A.val && A.nnz > 0) {
        Scratch cs(s);
        int32_t *row;
        unsigned long long *chk;
        GK_CHECK(cs.alloc(&row, A.nnz));
        GK_CHECK(cs.alloc(&chk, 3));
        GK_CUDA(cudaMemsetAsync(chk, 0, 3 * sizeof(unsigned long long), s));
        k_bc_entry_rows<<<sms * 8, 256, 0, s>>>(A, row);
        k_bc_mirror_check<<<sms * 8, 256, 0, s>>>(A, row, chk);
        note_launches(2);
        GK_CUDA(cudaGetLastError());
        unsigned long long h[3] = {1, 0, 0};
        GK_CUDA(cudaMemcpyAsync(h, chk, sizeof(h), cudaMemcpyDeviceToHost, s));
        GK_CUDA(cudaStreamSynchronize(s));
        self_transpose = h[0] == 0 && h[1] == h[2];
    }
    if (self_transpose) {
        g.AT = A;
    } else {
        int64_t *trp;
        int32_t *tcol, *tval = nullptr;
        GK_CHECK(scr.alloc(&trp, A.m + 1));
        GK_CHECK(scr.alloc(&tcol, A.nnz > 0 ? A.nnz : 1));
        if (A.val) GK_CHECK(scr.alloc(&tval, A.nnz > 0 ? A.nnz : 1));
        GK_CHECK(transpose_device(A, trp, tcol, tval, s, scr));
        g.AT = DevCsr{A.m, A.m, A.nnz, trp, tcol, tval};
    }
    GK_CHECK(heavy_set(g.A, &g.hA, s, scr));
    if (self_transpose) g.hAT = g.hA;
    else GK_CHECK(heavy_set(g.AT, &g.hAT, s, scr));
    GK_CUDA(cudaMemsetAsync(bc, 0, sizeof(double) * A.m, s));
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    for (int done = 0; done < nsrc;) {
        const int left = nsrc - done;
        int T = GK_BC_TMAX;
        while (T > 1 && 32 * (T / 2) >= left) T /= 2;
        // two FP64 m x W arrays must fit comfortably
        while (T > 1 && (double)A.m * 32 * T * 16 > 0.6 * (double)free_b) T /= 2;
        const int n = left < 32 * T ? left : 32 * T;
        int st;
        switch (T) {
            case 16: st = bc_chunk<16>(g, src + done, n, bc, opt, s); break;
            case 8: st = bc_chunk<8>(g, src + done, n, bc, opt, s); break;
            case 4: st = bc_chunk<4>(g, src + done, n, bc, opt, s); break;
            case 2: st = bc_chunk<2>(g, src + done, n, bc, opt, s); break;
            default: st = bc_chunk<1>(g, src + done, n, bc, opt, s); break;
        }
        GK_CHECK(st);
        done += n;
    }
    return GK_OK;
}

// Validates A and the sources, stages them, runs the batch.
static int bc_entry(const gk_csr *A, const int32_t *sources, int nsources, double *bc, const BcOptions &opt,
                    void *stream) {
    NvtxRange range("gk:bc_batch");
    GK_CHECK(validate_csr_shape(A, "A"));
    if (A->m != A->n) return fail(GK_ERR_ARG, "non-square matrix; BC is only for square matrices");
    if (nsources < 0 || (nsources > 0 && !sources) || (A->m > 0 && !bc)) return fail(GK_ERR_ARG, "bad arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    DevCsr d;
    GK_CHECK(stage_csr(A, &d, scr, s, nullptr, CSR_STRUCTURE, "A"));
    // sources: validate on the host
    std::vector<int32_t> hs(nsources > 0 ? nsources : 1);
    if (nsources > 0) {
        GK_CUDA(cudaMemcpyAsync(hs.data(), sources, sizeof(int32_t) * nsources, cudaMemcpyDefault, s));
        GK_CUDA(cudaStreamSynchronize(s));
    }
    {
        std::vector<char> seen(static_cast<size_t>(A->m), 0);
        for (int j = 0; j < nsources; ++j) {
            if (hs[j] < 0 || hs[j] >= A->m) return fail(GK_ERR_ARG, "source out of range");
            if (seen[hs[j]]) return fail(GK_ERR_ARG, "duplicate source");
            seen[hs[j]] = 1;
        }
    }
    int32_t *dsrc;
    GK_CHECK(scr.alloc(&dsrc, nsources > 0 ? nsources : 1));
    if (nsources > 0) GK_CUDA(cudaMemcpyAsync(dsrc, hs.data(), sizeof(int32_t) * nsources, cudaMemcpyHostToDevice, s));
    const bool host_out = A->m > 0 && !is_device_pointer(bc);
    double *dbc = bc;
    if (host_out) GK_CHECK(scr.alloc(&dbc, A->m));
    if (A->m > 0) GK_CHECK(bc_device(d, dsrc, nsources, dbc, opt, s, scr));
    if (host_out) {
        GK_CUDA(cudaMemcpyAsync(bc, dbc, sizeof(double) * A->m, cudaMemcpyDeviceToHost, s));
    }
    GK_CUDA(cudaStreamSynchronize(s));
    return GK_OK;
}

}  // namespace gk

using namespace gk;

extern "C" int gk_bc_batch(const gk_csr *A, const int32_t *sources, int nsources, double *bc, int sched,
                           void *stream) {
    BcOptions opt;
    opt.sched = sched;
    return bc_entry(A, sources, nsources, bc, opt, stream);
}

extern "C" int gk_bc_tune(const gk_csr *A, const int32_t *sources, int nsources, int shape, double *bc,
                          float *level_ms, float *level_feat, int max_levels, int *nlevels, void *stream) {
    if (shape < -1 || shape > 1) return fail(GK_ERR_ARG, "gk_bc_tune: shape must be -1, 0 (pull) or 1 (push)");
    if (max_levels < 0 || (max_levels > 0 && (!level_ms || !level_feat)) || !nlevels)
        return fail(GK_ERR_ARG, "gk_bc_tune: bad level arrays");
    if (nsources > 512) return fail(GK_ERR_ARG, "gk_bc_tune: at most 512 sources (one chunk)");
    BcOptions opt;
    opt.sched = GK_SCHED_PLAIN;
    opt.force = shape;
    opt.host_loop = true;
    opt.level_ms = level_ms;
    opt.level_feat = level_feat;
    opt.log_cap = max_levels;
    opt.levels_out = nlevels;
    *nlevels = 0;
    return bc_entry(A, sources, nsources, bc, opt, stream);
}

extern "C" int gk_bc_set_model(const float *weights, size_t n_floats) {
    if (!weights || n_floats != static_cast<size_t>(MLP_SIZE))
        return fail(GK_ERR_ARG, "gk_bc_set_model: weight count does not match gk_sched_model_size()");
    for (size_t i = 0; i < n_floats; ++i)
        if (!std::isfinite(weights[i])) return fail(GK_ERR_ARG, "gk_bc_set_model: non-finite weight");
    std::lock_guard<std::mutex> lock(g_bc_model_mutex);
    g_bc_model.assign(weights, weights + n_floats);
    ++g_bc_model_version;
    return GK_OK;
}

extern "C" int gk_bc_load_model_file(const char *path) {
    std::vector<float> w;
    const std::string err = read_model_file(path, w);
    if (!err.empty()) return fail(GK_ERR_ARG, "gk_bc_load_model_file: " + err);
    return gk_bc_set_model(w.data(), w.size());
}

extern "C" int gk_bc_has_model(void) {
    std::lock_guard<std::mutex> lock(g_bc_model_mutex);
    return g_bc_model.empty() ? 0 : 1;
}
