// Runtime plumbing of the library: per-thread last-error string, per-device
// context, stream-ordered scratch memory and host-or-device CSR staging.
#include <cuda_runtime.h>

#include <atomic>
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

int Scratch::raw_alloc(void **p, size_t bytes) {
    if (n_ >= 64) return fail(GK_ERR_OOM, "internal: too many scratch allocations in one call");
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

int stage_csr(const gk_csr *in, DevCsr *out, Scratch &scr, cudaStream_t s, int64_t *h2d) {
    out->m = in->m;
    out->n = in->n;
    out->nnz = in->nnz;
    GK_CHECK(stage_array(in->rowptr, static_cast<size_t>(in->m + 1), &out->rp, scr, s, h2d));
    GK_CHECK(stage_array(in->col, static_cast<size_t>(in->nnz), &out->col, scr, s, h2d));
    GK_CHECK(stage_array(in->val, static_cast<size_t>(in->nnz), &out->val, scr, s, h2d));
    return GK_OK;
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
        for (int i = 0; i < 16; ++i) {
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
