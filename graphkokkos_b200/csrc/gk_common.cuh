// Common device/host utilities of the B200 library: status handling, the
// device CSR view, stream-ordered scratch allocation and launch sizing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/gk_b200.h"
#include <nvtx3/nvToolsExt.h>  // header-only; ranges are no-ops unless a profiler is attached

namespace gk {

// ----- status / last error ---------------------------------------------------
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

#define GK_CUDA(expr)                                  \
    do {                                               \
        cudaError_t _e = (expr);                       \
        if (_e != cudaSuccess) return gk::cuda_fail(_e, #expr); \
    } while (0)

#define GK_CHECK(expr)                 \
    do {                               \
        int _s = (expr);               \
        if (_s != GK_OK) return _s;    \
    } while (0)

// ----- device CSR view ---------------------------------------------------------
struct DevCsr {
    int64_t m, n, nnz;
    const int64_t *rp;
    const int32_t *col;
    const int32_t *val;  // nullptr: every stored value is 1
};

// ----- per-device context ------------------------------------------------------
struct Context {
    int device = -1;
    int num_sms = 0;
    int max_smem_optin = 0;
    bool pool_ready = false;
};
// Returns the context of the current device (created on first use).
Context &ctx();

// Stream-ordered scratch: a vector of allocations released together, in
// stream order, when the guard goes out of scope.
class Scratch {
public:
    explicit Scratch(cudaStream_t s) : stream_(s) {}
    // Bump allocation inside caller-provided device memory [arena, arena+bytes)
    // instead of cudaMallocAsync; nothing is freed.  Used by the allocation-free
    // entry point (noalloc.cu).
    Scratch(cudaStream_t s, void *arena, size_t bytes)
        : stream_(s), arena_(static_cast<char *>(arena)), arena_bytes_(bytes) {}
    ~Scratch() { release(); }
    Scratch(const Scratch &) = delete;
    Scratch &operator=(const Scratch &) = delete;
    // Allocates `bytes` (rounded up to 256) on the stream; returns GK_OK or an error code.
    template <class T>
    int alloc(T **out, size_t count) {
        void *p = nullptr;
        int s = raw_alloc(&p, count * sizeof(T));
        *out = static_cast<T *>(p);
        return s;
    }
    void release();

private:
    int raw_alloc(void **p, size_t bytes);
    cudaStream_t stream_;
    void *ptrs_[64] = {};
    int n_ = 0;
    char *arena_ = nullptr;
    size_t arena_bytes_ = 0, arena_used_ = 0;
};

// What check_csr verifies beyond the row pointers and the column range.
enum CsrCheck { CSR_STRUCTURE = 1, CSR_SORTED = 2 };

// Content check of a CSR already in device memory, one warp per row: row
// pointers from 0 to nnz and non-decreasing, columns in [0, n), and with
// CSR_SORTED columns strictly increasing within each row (sorted, no
// duplicates).  Returns GK_ERR_INVALID_CSR with the first bad row.  It reads
// the result on the host (one synchronisation); inside a stream capture, or
// with GK_CHECK_CSR=0 in the environment, it is skipped.
int check_csr(const DevCsr &d, int level, const char *name, cudaStream_t s, Scratch &scr);
// The same for rows [row_base, row_base + m) of a block-diagonal batch whose
// row pointers run from ebase to ebase + nnz: row r belongs to graph
// key[row_base + r] (indices into the combined matrix), whose entries must lie
// in [estart[g], estart[g+1]].  pre_flags (device, may be null) holds CsrBad
// flags found while the batch was assembled (a column outside its graph's
// vertex range, a graph's row pointers not from 0 to nnz); they are reported
// like the check's own.
enum CsrBad : unsigned int { CSR_BAD_ENDS = 1, CSR_BAD_ROWPTR = 2, CSR_BAD_COL = 4, CSR_BAD_ORDER = 8 };
int check_csr_batch(const DevCsr &d, int64_t ebase, int64_t row_base, const int32_t *key, const int64_t *estart,
                    const unsigned int *pre_flags, int level, const char *name, cudaStream_t s, Scratch &scr);

// Host-or-device staging of a CSR: if the arrays are host memory they are
// copied to HBM on the stream (into scratch), otherwise used in place.  With
// check > 0 the staged matrix then goes through check_csr at that level.
int stage_csr(const gk_csr *in, DevCsr *out, Scratch &scr, cudaStream_t s, int64_t *h2d_bytes = nullptr,
              int check = CSR_SORTED, const char *name = "matrix");
bool is_device_pointer(const void *p);
int validate_csr_shape(const gk_csr *c, const char *name);

// Device CSR transforms (abi.cu): the transpose (A.n + 1 row pointers out,
// rows sorted; oval may be null) and the strict lower triangle.
int transpose_device(const DevCsr &A, int64_t *orp, int32_t *ocol, int32_t *oval, cudaStream_t s, Scratch &scr);
int extract_lower_device(const DevCsr &A, int64_t *orp, int32_t *ocol, cudaStream_t s, Scratch &scr);

inline int ceil_div(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

// ----- side streams for concurrent kernel variants ----------------------------
// Non-blocking streams and fork/join events, one set per host thread and
// device, so that concurrent callers never share an event.
constexpr int kSideStreams = 32;  // at least the number of kernel variants
struct SideStreams {
    cudaStream_t s[kSideStreams];
    cudaEvent_t fork;
    cudaEvent_t join[kSideStreams];
};
SideStreams &side_streams();

// ----- launch counter and per-variant profiling (gk_launch_count, gk_prof_*) ----
void note_launches(int n);

// An NVTX range around a phase of an operator (nsys timelines, ncu --nvtx
// filters); costs nothing measurable when no tool is attached.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};
bool prof_enabled();
bool prof_any();          // any profiling mode (its events cannot be captured into graphs)
int64_t launches_noted();  // kernel launches counted so far

struct ProfTotals {
    unsigned long long rows, sum_a, sum_m, sum_work;
};

// Brackets kernel launches with CUDA events when profiling is on; finish()
// synchronises the stream and appends one gk_prof_rec per bracketed slot.
class ProfWindow {
public:
    ProfWindow(cudaStream_t s, int slots);
    ~ProfWindow();
    bool active() const { return on_; }
    void begin(int slot, cudaStream_t on);
    void end(int slot, cudaStream_t on);
    int finish(const ProfTotals *totals);

private:
    cudaStream_t s_;
    bool on_;
    bool events_only_ = false;
    int slots_;
    cudaEvent_t ev_[64][2];
    bool used_[64];
};

}  // namespace gk
