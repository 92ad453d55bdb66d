// Runtime plumbing of the library: per-thread last-error string, per-device
// context, stream-ordered scratch memory and host-or-device CSR staging.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "gk_common.cuh"

namespace gk {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s", static_cast<int>(e), cudaGetErrorString(e),
                  what);
    g_last_error = buf;
    if (e == cudaErrorMemoryAllocation) return GK_ERR_OOM;
    return GK_ERR_CUDA;
}

static std::mutex g_ctx_mutex;
static Context g_ctx[64];

Context &ctx() {
    int dev = 0;
    cudaGetDevice(&dev);
    Context &c = g_ctx[dev & 63];
    if (c.device != dev) {
        std::lock_guard<std::mutex> lock(g_ctx_mutex);
        if (c.device != dev) {
            cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, dev);
            cudaDeviceGetAttribute(&c.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
            // keep freed stream-ordered scratch cached in the device's default
            // pool instead of returning it to the driver at every sync
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
                uint64_t threshold = UINT64_MAX;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
                c.pool_ready = true;
            }
            c.device = dev;
        }
    }
    return c;
}

// Allocation-failure injection for testing error paths (gk_inject_alloc_failure):
// the countdown's allocation fails once, -1 is off.
static std::atomic<long long> g_alloc_countdown{-1};

static bool injected_alloc_failure() {
    long long c = g_alloc_countdown.load(std::memory_order_relaxed);
    while (c >= 0) {
        if (g_alloc_countdown.compare_exchange_weak(c, c - 1, std::memory_order_relaxed)) return c == 0;
    }
    return false;
}

int Scratch::raw_alloc(void **p, size_t bytes) {
    if (n_ >= 64) return fail(GK_ERR_OOM, "internal: too many scratch allocations in one call");
    if (injected_alloc_failure()) return fail(GK_ERR_OOM, "injected allocation failure (gk_inject_alloc_failure)");
    bytes = (bytes + 255) & ~size_t(255);
    if (bytes == 0) bytes = 256;
    if (arena_) {
        if (arena_used_ + bytes > arena_bytes_) {
            char buf[160];
            std::snprintf(buf, sizeof(buf), "fixed scratch exhausted: %zu bytes needed, %zu available",
                          arena_used_ + bytes, arena_bytes_);
            return fail(GK_ERR_OOM, buf);
        }
        *p = arena_ + arena_used_;
        arena_used_ += bytes;
        return GK_OK;
    }
    cudaError_t e = cudaMallocAsync(p, bytes, stream_);
    if (e != cudaSuccess) {
        cudaGetLastError();
        char buf[160];
        std::snprintf(buf, sizeof(buf), "device scratch allocation of %zu bytes failed (%s)", bytes,
                      cudaGetErrorString(e));
        return fail(e == cudaErrorMemoryAllocation ? GK_ERR_OOM : GK_ERR_CUDA, buf);
    }
    ptrs_[n_++] = *p;
    return GK_OK;
}

void Scratch::release() {
    for (int i = 0; i < n_; ++i) cudaFreeAsync(ptrs_[i], stream_);
    n_ = 0;
}

bool is_device_pointer(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int validate_csr_shape(const gk_csr *c, const char *name) {
    if (!c) return fail(GK_ERR_ARG, std::string(name) + ": null matrix");
    if (c->m < 0 || c->n < 0 || c->nnz < 0)
        return fail(GK_ERR_ARG, std::string(name) + ": negative dimension");
    if (c->m >= (int64_t(1) << 31) || c->n >= (int64_t(1) << 31))
        return fail(GK_ERR_UNSUPPORTED, std::string(name) + ": dimension exceeds int32 column range");
    if (!c->rowptr) return fail(GK_ERR_ARG, std::string(name) + ": null rowptr");
    if (c->nnz > 0 && !c->col) return fail(GK_ERR_ARG, std::string(name) + ": null col");
    return GK_OK;
}

template <class T>
static int stage_array(const T *src, size_t count, const T **dst, Scratch &scr, cudaStream_t s,
                       int64_t *h2d) {
    if (!src || count == 0) {
        *dst = src;
        return GK_OK;
    }
    if (is_device_pointer(src)) {
        *dst = src;
        return GK_OK;
    }
    T *d = nullptr;
    GK_CHECK(scr.alloc(&d, count));
    GK_CUDA(cudaMemcpyAsync(d, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
    if (h2d) *h2d += static_cast<int64_t>(count * sizeof(T));
    *dst = d;
    return GK_OK;
}

int stage_csr(const gk_csr *in, DevCsr *out, Scratch &scr, cudaStream_t s, int64_t *h2d, int check,
              const char *name) {
    out->m = in->m;
    out->n = in->n;
    out->nnz = in->nnz;
    GK_CHECK(stage_array(in->rowptr, static_cast<size_t>(in->m + 1), &out->rp, scr, s, h2d));
    GK_CHECK(stage_array(in->col, static_cast<size_t>(in->nnz), &out->col, scr, s, h2d));
    GK_CHECK(stage_array(in->val, static_cast<size_t>(in->nnz), &out->val, scr, s, h2d));
    if (check > 0) GK_CHECK(check_csr(*out, check, name, s, scr));
    return GK_OK;
}

// ----- CSR content check -----------------------------------------------------------
struct CsrCheckOut {
    unsigned int flags;
    unsigned int pad;
    unsigned long long first_row;  // smallest bad row (local index)
    unsigned long long descents;   // positions p with col[p+1] <= col[p], over all entries
    unsigned long long boundary;   // the same, counted only where p ends its row
};

// The fast check, balanced over rows and over entries (two kernels, no
// per-row loops): rows are sorted exactly when every descent col[p+1] <=
// col[p] lies on a row boundary, i.e. when the descents counted over all
// entries equal those counted at the row ends.  Only when it finds a defect
// does the window kernel below run, to name the first bad row.
__global__ void __launch_bounds__(256) k_csr_rows(DevCsr c, int64_t ebase, int64_t row_base, const int32_t *key,
                                                  const int64_t *estart, const unsigned int *pre_flags, int sorted,
                                                  CsrCheckOut *out) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (c.rp[0] != ebase || c.rp[c.m] != ebase + c.nnz) atomicOr(&out->flags, CSR_BAD_ENDS);
        if (pre_flags && *pre_flags) atomicOr(&out->flags, *pre_flags);
    }
    const int64_t end = ebase + c.nnz;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned int bad = 0, cnt = 0;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < c.m; r += stride) {
        const int64_t a0 = c.rp[r], a1 = c.rp[r + 1];
        int64_t lo = ebase, hi = end;
        if (key) {
            const int g = key[row_base + r];
            lo = estart[g];
            hi = estart[g + 1];
        }
        if (a0 < lo || a1 < a0 || a1 > hi) {
            bad |= CSR_BAD_ROWPTR;
        } else if (sorted && a1 > a0 && a1 < end) {
            cnt += c.col[a1] <= c.col[a1 - 1];  // the pair across this row's end
        }
    }
    if (bad) atomicOr(&out->flags, bad);
    cnt = __reduce_add_sync(0xFFFFFFFFu, cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&out->boundary, static_cast<unsigned long long>(cnt));
}

__global__ void __launch_bounds__(256) k_csr_entries(DevCsr c, int64_t ebase, int sorted, CsrCheckOut *out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    constexpr int U = 4;  // independent loads in flight per thread
    unsigned int bad = 0, cnt = 0;
    for (int64_t q0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q0 < c.nnz; q0 += U * stride) {
        int32_t x[U], y[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t q = q0 + u * stride;
            x[u] = q < c.nnz ? c.col[ebase + q] : 0;
            y[u] = q + 1 < c.nnz ? c.col[ebase + q + 1] : 0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t q = q0 + u * stride;
            if (q >= c.nnz) continue;
            if (x[u] < 0 || x[u] >= c.n) bad |= CSR_BAD_COL;
            if (sorted && q + 1 < c.nnz) cnt += y[u] <= x[u];
        }
    }
    if (bad) atomicOr(&out->flags, bad);
    cnt = __reduce_add_sync(0xFFFFFFFFu, cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&out->descents, static_cast<unsigned long long>(cnt));
}

// One warp per window of 32 consecutive rows: lane l checks row w*32+l's
// pointers (non-decreasing, inside its entry range), then the warp streams the
// window's entries [rp[first], rp[last+1]) as one flat range in chunks of 256,
// eight loads in flight per lane, so that short rows cost a fraction of a
// load round trip each and a hub row is one warp's stream.  Entry p is
// compared with p+1 unless p ends its row: the rows ending inside the chunk
// mark those entries in a 256-bit shared-memory mask.
constexpr int CSR_CHECK_THREADS = 256;

__global__ void __launch_bounds__(CSR_CHECK_THREADS) k_csr_check(DevCsr c, int64_t ebase, int64_t row_base,
                                                                 const int32_t *key, const int64_t *estart,
                                                                 const unsigned int *pre_flags, int sorted,
                                                                 CsrCheckOut *out) {
    constexpr unsigned FULL = 0xFFFFFFFFu;
    constexpr int U = 8, CHUNK = 32 * U;
    __shared__ unsigned int s_last[CSR_CHECK_THREADS / 32][CHUNK / 32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (c.rp[0] != ebase || c.rp[c.m] != ebase + c.nnz) {
            atomicOr(&out->flags, CSR_BAD_ENDS);
            atomicMin(&out->first_row, c.rp[0] != ebase ? 0ull : static_cast<unsigned long long>(c.m));
        }
        if (pre_flags && *pre_flags) atomicOr(&out->flags, *pre_flags);
    }
    const int64_t nwin = (c.m + 31) / 32;
    for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nwin; w += warps) {
        const int64_t r = w * 32 + lane;
        const bool has = r < c.m;
        int64_t a0 = 0, a1 = 0;
        unsigned int bad = 0;
        if (has) {
            a0 = c.rp[r];
            a1 = c.rp[r + 1];
            int64_t lo = ebase, hi = ebase + c.nnz;
            if (key) {
                const int g = key[row_base + r];
                lo = estart[g];
                hi = estart[g + 1];
            }
            if (a0 < lo || a1 < a0 || a1 > hi) bad = CSR_BAD_ROWPTR;
        }
        if (bad) {
            atomicOr(&out->flags, bad);
            atomicMin(&out->first_row, static_cast<unsigned long long>(r));
        }
        if (__any_sync(FULL, bad)) continue;  // the window's entries are not read
        const int last = static_cast<int>(c.m - 1 - w * 32 < 31 ? c.m - 1 - w * 32 : 31);
        const int64_t w0 = __shfl_sync(FULL, a0, 0), w1 = __shfl_sync(FULL, a1, last);
        for (int64_t c0 = w0; c0 < w1; c0 += CHUNK) {
            __syncwarp();
            if (lane < CHUNK / 32) s_last[wib][lane] = 0u;
            __syncwarp();
            if (has && a1 > a0 && a1 - 1 >= c0 && a1 - 1 < c0 + CHUNK) {
                const int k = static_cast<int>(a1 - 1 - c0);
                atomicOr(&s_last[wib][k >> 5], 1u << (k & 31));
            }
            __syncwarp();
            int32_t x[U], y[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int64_t p = c0 + lane + 32 * u;
                x[u] = p < w1 ? c.col[p] : 0;
                y[u] = p + 1 < w1 ? c.col[p + 1] : 0;
            }
            unsigned int ebad = 0, kbad = FULL;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = lane + 32 * u;
                const int64_t p = c0 + k;
                if (p >= w1) continue;
                unsigned int e = 0;
                if (x[u] < 0 || x[u] >= c.n) e |= CSR_BAD_COL;
                const bool ends_row = (s_last[wib][u] >> lane) & 1u;
                if (sorted && !ends_row && p + 1 < w1 && y[u] <= x[u]) e |= CSR_BAD_ORDER;
                if (e) {
                    ebad |= e;
                    if (static_cast<unsigned int>(k) < kbad) kbad = static_cast<unsigned int>(k);
                }
            }
            ebad = __reduce_or_sync(FULL, ebad);
            if (ebad) {
                // the row holding the first bad entry of the chunk
                const int64_t pbad = c0 + __reduce_min_sync(FULL, kbad);
                const unsigned int owner = __ballot_sync(FULL, has && a0 <= pbad && pbad < a1);
                if (lane == 0) {
                    atomicOr(&out->flags, ebad);
                    atomicMin(&out->first_row, static_cast<unsigned long long>(w * 32 + (owner ? __ffs(owner) - 1 : 0)));
                }
                break;
            }
        }
    }
}

static bool csr_check_enabled() {
    static const bool on = [] {
        const char *e = getenv("GK_CHECK_CSR");
        return !(e && e[0] == '0');
    }();
    return on;
}

int check_csr_batch(const DevCsr &d, int64_t ebase, int64_t row_base, const int32_t *key, const int64_t *estart,
                    const unsigned int *pre_flags, int level, const char *name, cudaStream_t s, Scratch &scr) {
    NvtxRange range("gk:csr_check");
    if (level <= 0 || !csr_check_enabled()) return GK_OK;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
        cudaGetLastError();
        return GK_OK;
    }
    if (cap != cudaStreamCaptureStatusNone) return GK_OK;  // no host read inside a capture
    CsrCheckOut *dout;
    GK_CHECK(scr.alloc(&dout, 1));
    const CsrCheckOut init{0u, 0u, ~0ull, 0ull, 0ull};
    const int sorted = level >= CSR_SORTED ? 1 : 0;
    const int max_blocks = ctx().num_sms * 8;
    GK_CUDA(cudaMemcpyAsync(dout, &init, sizeof(init), cudaMemcpyHostToDevice, s));
    k_csr_rows<<<static_cast<int>(std::min<int64_t>((d.m + 255) / 256 + 1, max_blocks)), 256, 0, s>>>(
        d, ebase, row_base, key, estart, pre_flags, sorted, dout);
    k_csr_entries<<<static_cast<int>(std::min<int64_t>((d.nnz + 255) / 256 + 1, max_blocks)), 256, 0, s>>>(d, ebase, sorted,
                                                                                                    dout);
    note_launches(2);
    GK_CUDA(cudaGetLastError());
    CsrCheckOut h{};
    GK_CUDA(cudaMemcpyAsync(&h, dout, sizeof(h), cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaStreamSynchronize(s));
    if (h.descents != h.boundary) h.flags |= CSR_BAD_ORDER;
    if (!h.flags) return GK_OK;
    // a defect: the window kernel names the first bad row
    GK_CUDA(cudaMemcpyAsync(dout, &init, sizeof(init), cudaMemcpyHostToDevice, s));
    const int64_t windows = (d.m + 31) / 32;
    k_csr_check<<<static_cast<int>(std::min<int64_t>((windows + 7) / 8 + 1, max_blocks)), CSR_CHECK_THREADS, 0, s>>>(
        d, ebase, row_base, key, estart, pre_flags, sorted, dout);
    note_launches(1);
    GK_CUDA(cudaGetLastError());
    CsrCheckOut w{};
    GK_CUDA(cudaMemcpyAsync(&w, dout, sizeof(w), cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaStreamSynchronize(s));
    if (w.flags) h = w;
    if (!h.flags) return GK_OK;
    std::string what;
    if (h.flags & CSR_BAD_ENDS) what = "row pointers must start at 0 and end at nnz";
    else if (h.flags & CSR_BAD_ROWPTR) what = "row pointers decrease or leave [0, nnz]";
    else if (h.flags & CSR_BAD_COL) what = key ? "column index out of range of its graph's vertices" : "column index out of range";
    else what = "columns not strictly increasing within a row (sort the rows, drop duplicates)";
    const std::string where = h.first_row == ~0ull ? std::string()
                                                   : " (first at row " + std::to_string(h.first_row + row_base) + ")";
    return fail(GK_ERR_INVALID_CSR, std::string(name) + ": " + what + where);
}

int check_csr(const DevCsr &d, int level, const char *name, cudaStream_t s, Scratch &scr) {
    return check_csr_batch(d, 0, 0, nullptr, nullptr, nullptr, level, name, s, scr);
}

// ----- launch counter and profiling ---------------------------------------------
static std::atomic<long long> g_launches{0};
static std::atomic<int> g_prof_on{0};
static std::mutex g_prof_mutex;
static std::vector<gk_prof_rec> g_prof;
// events-only mode: launches bracketed without synchronising; resolved by gk_prof_flush
struct Pending {
    int variant;
    cudaEvent_t a, b;
};
static std::vector<Pending> g_pending;

void note_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
bool prof_enabled() { return g_prof_on.load(std::memory_order_relaxed) == 1; }
bool prof_any() { return g_prof_on.load(std::memory_order_relaxed) != 0; }
int64_t launches_noted() { return g_launches.load(std::memory_order_relaxed); }
static bool prof_events_only() { return g_prof_on.load(std::memory_order_relaxed) == 2; }

ProfWindow::ProfWindow(cudaStream_t s, int slots) : s_(s), on_(prof_enabled()), slots_(slots < 64 ? slots : 64) {
    if (prof_events_only()) {
        // bracket each launch with a pair of pooled events, resolved later
        events_only_ = true;
        return;
    }
    for (int i = 0; i < 64; ++i) used_[i] = false;
    if (!on_) return;
    for (int i = 0; i < slots_; ++i) {
        cudaEventCreate(&ev_[i][0]);
        cudaEventCreate(&ev_[i][1]);
    }
}

ProfWindow::~ProfWindow() {
    if (!on_) return;
    for (int i = 0; i < slots_; ++i) {
        cudaEventDestroy(ev_[i][0]);
        cudaEventDestroy(ev_[i][1]);
    }
}

void ProfWindow::begin(int slot, cudaStream_t on) {
    if (events_only_) {
        Pending p{slot, nullptr, nullptr};
        cudaEventCreate(&p.a);
        cudaEventCreate(&p.b);
        cudaEventRecord(p.a, on);
        std::lock_guard<std::mutex> lock(g_prof_mutex);
        g_pending.push_back(p);
        return;
    }
    if (on_ && slot < slots_) cudaEventRecord(ev_[slot][0], on);
}

void ProfWindow::end(int slot, cudaStream_t on) {
    if (events_only_) {
        std::lock_guard<std::mutex> lock(g_prof_mutex);
        for (auto it = g_pending.rbegin(); it != g_pending.rend(); ++it)
            if (it->variant == slot) {
                cudaEventRecord(it->b, on);
                break;
            }
        return;
    }
    if (on_ && slot < slots_) {
        cudaEventRecord(ev_[slot][1], on);
        used_[slot] = true;
    }
}

SideStreams &side_streams() {
    static thread_local SideStreams per_dev[16];
    static thread_local bool ready[16] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    dev &= 15;
    if (!ready[dev]) {
        SideStreams &x = per_dev[dev];
        for (int i = 0; i < kSideStreams; ++i) {
            cudaStreamCreateWithFlags(&x.s[i], cudaStreamNonBlocking);
            cudaEventCreateWithFlags(&x.join[i], cudaEventDisableTiming);
        }
        cudaEventCreateWithFlags(&x.fork, cudaEventDisableTiming);
        ready[dev] = true;
    }
    return per_dev[dev];
}

int ProfWindow::finish(const ProfTotals *totals) {
    if (!on_) return GK_OK;
    GK_CUDA(cudaStreamSynchronize(s_));
    std::lock_guard<std::mutex> lock(g_prof_mutex);
    for (int i = 0; i < slots_; ++i) {
        if (!used_[i]) continue;
        float ms = 0.f;
        GK_CUDA(cudaEventElapsedTime(&ms, ev_[i][0], ev_[i][1]));
        gk_prof_rec r{};
        r.variant = i;
        r.ms = ms;
        if (totals) {
            r.rows = static_cast<int64_t>(totals[i].rows);
            r.sum_a = static_cast<int64_t>(totals[i].sum_a);
            r.sum_m = static_cast<int64_t>(totals[i].sum_m);
            r.sum_work = static_cast<int64_t>(totals[i].sum_work);
        }
        g_prof.push_back(r);
    }
    return GK_OK;
}

}  // namespace gk

extern "C" {

int gk_prof_enable(int on) {
    if (on < 0 || on > 2) return gk::fail(GK_ERR_ARG, "gk_prof_enable: mode must be 0, 1 or 2");
    std::lock_guard<std::mutex> lock(gk::g_prof_mutex);
    gk::g_prof.clear();
    for (auto &p : gk::g_pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    gk::g_pending.clear();
    gk::g_prof_on.store(on);
    return GK_OK;
}

int gk_prof_flush(void) {
    std::lock_guard<std::mutex> lock(gk::g_prof_mutex);
    for (auto &p : gk::g_pending) {
        cudaError_t e = cudaEventSynchronize(p.b);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, p.a, p.b);
        if (e != cudaSuccess) return gk::cuda_fail(e, "gk_prof_flush");
        gk_prof_rec r{};
        r.variant = p.variant;
        r.ms = ms;
        gk::g_prof.push_back(r);
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    gk::g_pending.clear();
    return GK_OK;
}

int gk_prof_count(void) {
    std::lock_guard<std::mutex> lock(gk::g_prof_mutex);
    return static_cast<int>(gk::g_prof.size());
}

int gk_prof_get(int i, gk_prof_rec *out) {
    std::lock_guard<std::mutex> lock(gk::g_prof_mutex);
    if (!out || i < 0 || i >= static_cast<int>(gk::g_prof.size())) return gk::fail(GK_ERR_ARG, "gk_prof_get: index");
    *out = gk::g_prof[i];
    return GK_OK;
}

int64_t gk_launch_count(void) { return gk::g_launches.load(); }

}  // extern "C"

extern "C" const char *gk_last_error_string(void) { return gk::g_last_error.c_str(); }

extern "C" int gk_version(void) { return 100; }

extern "C" int gk_inject_alloc_failure(int64_t after) {
    gk::g_alloc_countdown.store(after < 0 ? -1 : static_cast<long long>(after), std::memory_order_relaxed);
    return GK_OK;
}
