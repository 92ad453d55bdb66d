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
// One warp owns one vertex; lane l owns sources {32t + l}.  A neighbour is
// skipped after one broadcast load of its T bitmap words unless it carries a
// frontier bit this vertex still needs, so sigma/R are only read where the
// algebra has a term.  Vertices with more than HEAVY neighbours are processed
// by a whole CTA (warps split the neighbour list, partial sums reduced in
// shared memory).  R(v,s) = (1+delta)/sigma replaces the reference's
// Nspinv∘Bcu; delta is summed into bc[v] as soon as it is final.
#include <vector>

#include "gk_common.cuh"

namespace gk {

int transpose_device(const DevCsr &A, int64_t *orp, int32_t *ocol, int32_t *oval, cudaStream_t s, Scratch &scr);

constexpr int BC_HEAVY = 512;
constexpr int BC_NW_HEAVY = 8;  // T=16: 8*16*32 doubles = 32 KB of static shared memory

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

// forward pull for one vertex by one warp (or one warp's share of the neighbours)
template <int T>
__device__ __forceinline__ bool fwd_accumulate(const DevCsr &AT, int64_t e0, int64_t e1, int64_t estride,
                                               const uint32_t *__restrict__ Fd, const uint32_t (&need)[T],
                                               const double *__restrict__ sigma, int W, int lane,
                                               double (&acc)[T]) {
    bool any = false;
    for (int64_t e = e0; e < e1; e += estride) {
        const int k = __ldg(AT.col + e);
        uint32_t f[T];
        load_words<T>(Fd + (int64_t)k * T, f);
        uint32_t hit = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) {
            f[t] &= need[t];
            hit |= f[t];
        }
        if (!hit) continue;
        any = true;
        const double a = AT.val ? static_cast<double>(__ldg(AT.val + e)) : 1.0;
        const double *__restrict__ sk = sigma + (int64_t)k * W + lane;
#pragma unroll
        for (int t = 0; t < T; ++t)
            if ((f[t] >> lane) & 1u) acc[t] += a * __ldg(sk + 32 * t);
    }
    return any;
}

template <int T>
__device__ __forceinline__ void fwd_emit(int64_t i, int W, int lane, const uint32_t (&vis)[T], const double (&acc)[T],
                                         uint32_t *Fn, uint32_t *V, double *sigma, unsigned *progress) {
    uint32_t anyb = 0;
#pragma unroll
    for (int t = 0; t < T; ++t) {
        const uint32_t nb = __ballot_sync(0xFFFFFFFFu, acc[t] != 0.0);
        anyb |= nb;
        if ((nb >> lane) & 1u) sigma[i * W + 32 * t + lane] = acc[t];
        if (lane == t) {
            Fn[i * T + t] = nb;
            V[i * T + t] = vis[t] | nb;
        }
    }
    if (lane == 0 && anyb) atomicAdd(progress, 1u);
}

template <int T>
__global__ void __launch_bounds__(256) k_bc_forward(DevCsr AT, const uint32_t *__restrict__ Fd, uint32_t *Fn,
                                                    uint32_t *V, double *sigma, int W, const uint32_t *act,
                                                    unsigned *progress) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < AT.m; i += warps) {
        const int64_t e0 = AT.rp[i], e1 = AT.rp[i + 1];
        if (e0 == e1 || e1 - e0 > BC_HEAVY) continue;
        uint32_t vis[T], need[T];
        load_words<T>(V + i * T, vis);
        uint32_t open = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) {
            need[t] = ~vis[t] & act[t];
            open |= need[t];
        }
        if (!open) continue;
        double acc[T];
#pragma unroll
        for (int t = 0; t < T; ++t) acc[t] = 0.0;
        if (!fwd_accumulate<T>(AT, e0, e1, 1, Fd, need, sigma, W, lane, acc)) continue;
        fwd_emit<T>(i, W, lane, vis, acc, Fn, V, sigma, progress);
    }
}

template <int T>
__global__ void __launch_bounds__(BC_NW_HEAVY * 32) k_bc_forward_heavy(DevCsr AT, const int32_t *heavy, int nheavy,
                                                                      const uint32_t *__restrict__ Fd, uint32_t *Fn,
                                                                      uint32_t *V, double *sigma, int W,
                                                                      const uint32_t *act, unsigned *progress) {
    __shared__ double part[BC_NW_HEAVY][T][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int h = blockIdx.x; h < nheavy; h += gridDim.x) {
        const int64_t i = heavy[h];
        const int64_t e0 = AT.rp[i], e1 = AT.rp[i + 1];
        uint32_t vis[T], need[T];
        load_words<T>(V + i * T, vis);
        uint32_t open = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) {
            need[t] = ~vis[t] & act[t];
            open |= need[t];
        }
        if (!open) continue;  // uniform across the CTA
        double acc[T];
#pragma unroll
        for (int t = 0; t < T; ++t) acc[t] = 0.0;
        fwd_accumulate<T>(AT, e0 + warp, e1, BC_NW_HEAVY, Fd, need, sigma, W, lane, acc);
#pragma unroll
        for (int t = 0; t < T; ++t) part[warp][t][lane] = acc[t];
        __syncthreads();
        if (warp == 0) {
#pragma unroll
            for (int t = 0; t < T; ++t) {
                double sum = 0.0;
                for (int w = 0; w < BC_NW_HEAVY; ++w) sum += part[w][t][lane];
                acc[t] = sum;
            }
            fwd_emit<T>(i, W, lane, vis, acc, Fn, V, sigma, progress);
        }
        __syncthreads();
    }
}

// deepest level: R = 1/sigma (Bcu = 1 there)
template <int T>
__global__ void k_bc_rinit(int64_t m, const uint32_t *__restrict__ Fd, const double *sigma, double *R, int W) {
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

template <int T>
__device__ __forceinline__ void bwd_accumulate(const DevCsr &A, int64_t e0, int64_t e1, int64_t estride,
                                               const uint32_t *__restrict__ Fn, const uint32_t (&fv)[T],
                                               const double *__restrict__ R, int W, int lane, double (&sum)[T]) {
    for (int64_t e = e0; e < e1; e += estride) {
        const int w = __ldg(A.col + e);
        uint32_t f[T];
        load_words<T>(Fn + (int64_t)w * T, f);
        uint32_t hit = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) {
            f[t] &= fv[t];
            hit |= f[t];
        }
        if (!hit) continue;
        const double a = A.val ? static_cast<double>(__ldg(A.val + e)) : 1.0;
        const double *__restrict__ rw = R + (int64_t)w * W + lane;
#pragma unroll
        for (int t = 0; t < T; ++t)
            if ((f[t] >> lane) & 1u) sum[t] += a * __ldg(rw + 32 * t);
    }
}

template <int T>
__device__ __forceinline__ void bwd_emit(int64_t v, int W, int lane, const uint32_t (&fv)[T], const double (&sum)[T],
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
__global__ void __launch_bounds__(256) k_bc_backward(DevCsr A, const uint32_t *__restrict__ Fd,
                                                     const uint32_t *__restrict__ Fn, const double *sigma, double *R,
                                                     int W, double *bc) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < A.m; v += warps) {
        const int64_t e0 = A.rp[v], e1 = A.rp[v + 1];
        if (e1 - e0 > BC_HEAVY) continue;
        uint32_t fv[T];
        load_words<T>(Fd + v * T, fv);
        uint32_t any = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) any |= fv[t];
        if (!any) continue;
        double sum[T];
#pragma unroll
        for (int t = 0; t < T; ++t) sum[t] = 0.0;
        bwd_accumulate<T>(A, e0, e1, 1, Fn, fv, R, W, lane, sum);
        bwd_emit<T>(v, W, lane, fv, sum, sigma, R, bc);
    }
}

template <int T>
__global__ void __launch_bounds__(BC_NW_HEAVY * 32) k_bc_backward_heavy(DevCsr A, const int32_t *heavy, int nheavy,
                                                                       const uint32_t *__restrict__ Fd,
                                                                       const uint32_t *__restrict__ Fn,
                                                                       const double *sigma, double *R, int W,
                                                                       double *bc) {
    __shared__ double part[BC_NW_HEAVY][T][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int h = blockIdx.x; h < nheavy; h += gridDim.x) {
        const int64_t v = heavy[h];
        uint32_t fv[T];
        load_words<T>(Fd + v * T, fv);
        uint32_t any = 0;
#pragma unroll
        for (int t = 0; t < T; ++t) any |= fv[t];
        if (!any) continue;
        double sum[T];
#pragma unroll
        for (int t = 0; t < T; ++t) sum[t] = 0.0;
        bwd_accumulate<T>(A, A.rp[v] + warp, A.rp[v + 1], BC_NW_HEAVY, Fn, fv, R, W, lane, sum);
#pragma unroll
        for (int t = 0; t < T; ++t) part[warp][t][lane] = sum[t];
        __syncthreads();
        if (warp == 0) {
#pragma unroll
            for (int t = 0; t < T; ++t) {
                double x = 0.0;
                for (int w = 0; w < BC_NW_HEAVY; ++w) x += part[w][t][lane];
                sum[t] = x;
            }
            bwd_emit<T>(v, W, lane, fv, sum, sigma, R, bc);
        }
        __syncthreads();
    }
}

__global__ void k_heavy_list(DevCsr A, int32_t *list, int *count) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < A.m; i += stride)
        if (A.rp[i + 1] - A.rp[i] > BC_HEAVY) list[atomicAdd(count, 1)] = static_cast<int32_t>(i);
}

// ---------------------------------------------------------------------------
struct BcBuffers {
    DevCsr A, AT;
    int32_t *heavyA, *heavyAT;
    int nheavyA, nheavyAT;
};

template <int T>
static int bc_chunk(const BcBuffers &g, const int32_t *src, int nsrc, double *bc, cudaStream_t s, Scratch &scr) {
    constexpr int W = 32 * T;
    const int64_t m = g.A.m;
    const int sms = ctx().num_sms;
    double *sigma, *R;
    uint32_t *V, *act;
    unsigned *progress;
    Scratch local(s);
    GK_CHECK(local.alloc(&sigma, (size_t)m * W));
    GK_CHECK(local.alloc(&R, (size_t)m * W));
    GK_CHECK(local.alloc(&V, (size_t)m * T));
    GK_CHECK(local.alloc(&act, T));
    GK_CHECK(local.alloc(&progress, 1));
    GK_CUDA(cudaMemsetAsync(V, 0, sizeof(uint32_t) * m * T, s));
    uint32_t hact[16];
    for (int t = 0; t < T; ++t) {
        const int lo = 32 * t;
        const int cnt = nsrc - lo <= 0 ? 0 : (nsrc - lo >= 32 ? 32 : nsrc - lo);
        hact[t] = cnt == 32 ? 0xFFFFFFFFu : ((1u << cnt) - 1u);
    }
    GK_CUDA(cudaMemcpyAsync(act, hact, sizeof(uint32_t) * T, cudaMemcpyHostToDevice, s));
    std::vector<uint32_t *> levels;
    auto new_level = [&](uint32_t **out) -> int {
        uint32_t *p = nullptr;
        cudaError_t e = cudaMallocAsync(&p, sizeof(uint32_t) * m * T, s);
        if (e != cudaSuccess) return cuda_fail(e, "BC level bitmap");
        levels.push_back(p);
        e = cudaMemsetAsync(p, 0, sizeof(uint32_t) * m * T, s);
        if (e != cudaSuccess) return cuda_fail(e, "BC level bitmap");
        *out = p;
        return GK_OK;
    };
    auto free_levels = [&]() {
        for (uint32_t *p : levels) cudaFreeAsync(p, s);
        levels.clear();
    };
    unsigned *h_prog;
    GK_CUDA(cudaMallocHost(&h_prog, sizeof(unsigned)));
    int status = GK_OK;
    do {
        uint32_t *F1;
        if ((status = new_level(&F1)) != GK_OK) break;
        k_bc_seed<<<sms * 4, 256, 0, s>>>(g.A, src, nsrc, T, W, F1, V, sigma);
        note_launches(1);
        // forward sweep: one level per launch pair, until the frontier is empty
        for (int64_t d = 1; d <= m; ++d) {
            uint32_t *Fn;
            if ((status = new_level(&Fn)) != GK_OK) break;
            cudaMemsetAsync(progress, 0, sizeof(unsigned), s);
            const uint32_t *Fd = levels[levels.size() - 2];
            k_bc_forward<T><<<sms * 8, 256, 0, s>>>(g.AT, Fd, Fn, V, sigma, W, act, progress);
            note_launches(1);
            if (g.nheavyAT)
                k_bc_forward_heavy<T><<<sms * 2, BC_NW_HEAVY * 32, 0, s>>>(g.AT, g.heavyAT, g.nheavyAT, Fd, Fn, V,
                                                                         sigma, W, act, progress);
                note_launches(1);
            cudaMemcpyAsync(h_prog, progress, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
            cudaError_t e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) {
                status = cuda_fail(e, "BC forward level");
                break;
            }
            if (*h_prog == 0) break;  // F_{d+1} empty: levels 1..d are the BFS layers
        }
        if (status != GK_OK) break;
        // levels = [F_1 .. F_D, empty]
        const int D = static_cast<int>(levels.size()) - 1;
        k_bc_rinit<T><<<sms * 8, 256, 0, s>>>(m, levels[D - 1], sigma, R, W);
        note_launches(1);
        for (int d = D - 1; d >= 1; --d) {
            k_bc_backward<T><<<sms * 8, 256, 0, s>>>(g.A, levels[d - 1], levels[d], sigma, R, W, bc);
            note_launches(1);
            if (g.nheavyA)
                k_bc_backward_heavy<T><<<sms * 2, BC_NW_HEAVY * 32, 0, s>>>(g.A, g.heavyA, g.nheavyA, levels[d - 1],
                                                                          levels[d], sigma, R, W, bc);
                note_launches(1);
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) status = cuda_fail(e, "BC backward");
    } while (false);
    free_levels();
    cudaFreeHost(h_prog);
    return status;
}

int bc_device(const DevCsr &A, const int32_t *src, int nsrc, double *bc, cudaStream_t s, Scratch &scr) {
    const int sms = ctx().num_sms;
    BcBuffers g;
    g.A = A;
    int64_t *trp;
    int32_t *tcol, *tval = nullptr;
    GK_CHECK(scr.alloc(&trp, A.m + 1));
    GK_CHECK(scr.alloc(&tcol, A.nnz > 0 ? A.nnz : 1));
    if (A.val) GK_CHECK(scr.alloc(&tval, A.nnz > 0 ? A.nnz : 1));
    GK_CHECK(transpose_device(A, trp, tcol, tval, s, scr));
    g.AT = DevCsr{A.m, A.m, A.nnz, trp, tcol, tval};
    int *cnt;
    GK_CHECK(scr.alloc(&g.heavyA, A.m > 0 ? A.m : 1));
    GK_CHECK(scr.alloc(&g.heavyAT, A.m > 0 ? A.m : 1));
    GK_CHECK(scr.alloc(&cnt, 2));
    GK_CUDA(cudaMemsetAsync(cnt, 0, 2 * sizeof(int), s));
    k_heavy_list<<<sms * 4, 256, 0, s>>>(g.A, g.heavyA, cnt);
    note_launches(1);
    k_heavy_list<<<sms * 4, 256, 0, s>>>(g.AT, g.heavyAT, cnt + 1);
    note_launches(1);
    int hc[2];
    GK_CUDA(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaStreamSynchronize(s));
    g.nheavyA = hc[0];
    g.nheavyAT = hc[1];
    GK_CUDA(cudaMemsetAsync(bc, 0, sizeof(double) * A.m, s));
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    for (int done = 0; done < nsrc;) {
        const int left = nsrc - done;
        int T = 16;
        while (T > 1 && 32 * (T / 2) >= left) T /= 2;
        // two FP64 m x W arrays must fit comfortably
        while (T > 1 && (double)A.m * 32 * T * 16 > 0.6 * (double)free_b) T /= 2;
        const int n = left < 32 * T ? left : 32 * T;
        int st;
        switch (T) {
            case 16: st = bc_chunk<16>(g, src + done, n, bc, s, scr); break;
            case 8: st = bc_chunk<8>(g, src + done, n, bc, s, scr); break;
            case 4: st = bc_chunk<4>(g, src + done, n, bc, s, scr); break;
            case 2: st = bc_chunk<2>(g, src + done, n, bc, s, scr); break;
            default: st = bc_chunk<1>(g, src + done, n, bc, s, scr); break;
        }
        GK_CHECK(st);
        done += n;
    }
    return GK_OK;
}

}  // namespace gk

using namespace gk;

extern "C" int gk_bc_batch(const gk_csr *A, const int32_t *sources, int nsources, double *bc, int sched,
                           void *stream) {
    (void)sched;  // the BC sweep has one kernel shape per level; the scheduler is not consulted
    GK_CHECK(validate_csr_shape(A, "A"));
    if (A->m != A->n) return fail(GK_ERR_ARG, "non-square matrix; BC is only for square matrices");
    if (nsources < 0 || (nsources > 0 && !sources) || (A->m > 0 && !bc)) return fail(GK_ERR_ARG, "bad arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    DevCsr d;
    GK_CHECK(stage_csr(A, &d, scr, s));
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
    if (A->m > 0) GK_CHECK(bc_device(d, dsrc, nsources, dbc, s, scr));
    if (host_out) {
        GK_CUDA(cudaMemcpyAsync(bc, dbc, sizeof(double) * A->m, cudaMemcpyDeviceToHost, s));
        GK_CUDA(cudaStreamSynchronize(s));
    }
    return GK_OK;
}
