// gk_tc_count_noalloc: triangle counting that allocates no device memory.
//
// Some callers cannot let a library allocate GPU memory while they run: a
// process whose framework's caching allocator has already reserved the device's
// memory (a cudaMalloc from us would fail, or fragment and stall their pool),
// or a host that forbids its plugins from allocating inside its processing loop
// because an allocation can synchronise the device.  For them this entry point
// runs the same masked-SpGEMM triangle count as gk_tc_count, but every scratch
// buffer (the scheduler's per-row plan, the scan's temporary storage and the
// count accumulator) is carved from one fixed array in device memory declared
// below, instead of being allocated per call.
//
//  * The array is a file-scope __device__ variable of GK_NOALLOC_BYTES
//    (36 MiB): every GPU on which this library is loaded holds it until the
//    process exits.  It bounds the graph to GK_NOALLOC_MAX_ROWS rows; larger
//    graphs are rejected with GK_ERR_ARG.
//  * Inputs must already be in device memory (staging host arrays would
//    allocate); the count may be written to host or device memory.
//  * The array's device address is fetched with cudaGetSymbolAddress the first
//    time the entry point is called on a device (with that device current);
//    that first call should therefore come before any stream capture.
//  * L goes through the same content check as every entry point (row
//    pointers, column range, sorted rows), which synchronises the stream once;
//    GK_CHECK_CSR=0 skips it for trusted input.
//  * All calls share the array and it keeps the last call's contents; what
//    must start at zero is cleared by each call.  Calls whose work overlaps on
//    the GPU (other host threads, or other streams without ordering between
//    them) race on the array and give wrong results.
// No counterpart in the reference.
#include <mutex>

#include "gk_common.cuh"
#include "gk_spgemm.cuh"

namespace gk {

constexpr int64_t GK_NOALLOC_MAX_ROWS = int64_t(1) << 20;
constexpr size_t GK_NOALLOC_BYTES = size_t(36) << 20;

// per row: work (8) + maxb (4) + bin (2) + row list (4) + item counts (8) +
// their prefix (8) = 34 bytes -> 34 MiB at the row limit; the rest holds the
// bin table, counters, the scan's temporary storage and the accumulator.
static __device__ __align__(256) unsigned char g_tc_scratch[GK_NOALLOC_BYTES];

constexpr int GK_NOALLOC_MAX_DEVICES = 64;
static std::mutex g_noalloc_mutex;
static void *g_noalloc_ptr[GK_NOALLOC_MAX_DEVICES];

// Device address of g_tc_scratch on the current device (set up once per device).
static int noalloc_arena(void **out) {
    int dev = 0;
    GK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= GK_NOALLOC_MAX_DEVICES)
        return fail(GK_ERR_UNSUPPORTED, "gk_tc_count_noalloc: device ordinals above 63 are not supported");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_tc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_tc_scratch)");
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return GK_OK;
}

}  // namespace gk

using namespace gk;

extern "C" int gk_tc_count_noalloc(const gk_csr *L, uint64_t *count, int sched, void *stream) {
    GK_CHECK(validate_csr_shape(L, "L"));
    if (L->m != L->n) return fail(GK_ERR_ARG, "L: matrix must be square");
    if (!count) return fail(GK_ERR_ARG, "count is null");
    if (L->m > GK_NOALLOC_MAX_ROWS)
        return fail(GK_ERR_ARG, "gk_tc_count_noalloc: L has more than 1048576 rows, the limit of its fixed scratch");
    // the row pointers are read on the device even for an empty graph (rowptr[0], rowptr[m])
    if (!is_device_pointer(L->rowptr) || (L->nnz > 0 && !is_device_pointer(L->col)))
        return fail(GK_ERR_ARG, "gk_tc_count_noalloc: L must be in device memory (staging host arrays would allocate)");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    void *arena = nullptr;
    GK_CHECK(noalloc_arena(&arena));
    Scratch scr(s, arena, GK_NOALLOC_BYTES);
    unsigned long long *d;
    GK_CHECK(scr.alloc(&d, 1));
    GK_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), s));
    DevCsr dl{L->m, L->n, L->nnz, L->rowptr, L->col, nullptr};
    GK_CHECK(check_csr(dl, CSR_SORTED, "L", s, scr));
    SpgemmRequest rq;
    rq.A = rq.B = rq.M = dl;
    rq.epi = EPI_SUM;
    rq.sched = sched;
    rq.sums = d;
    rq.stream = s;
    GK_CHECK(run_spgemm(rq, scr));
    if (is_device_pointer(count)) {
        GK_CUDA(cudaMemcpyAsync(count, d, sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    } else {
        GK_CUDA(cudaMemcpyAsync(count, d, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        GK_CUDA(cudaStreamSynchronize(s));
    }
    return GK_OK;
}
