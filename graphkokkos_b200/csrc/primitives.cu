// Elementwise and sparse-dense primitives of the reference's alternate BC
// formulation: gk_add_nointersect, gk_dense_ewise_mult_masked,
// gk_dense_fuse_ewise_mult_add, gk_mxmm_spd.
//
// Reference: include/matrix_la.h:182-328 — fuseEWiseMultAdd (:182-187), the
// dense masked eWiseMult (:189-208), mxmm_spd (:230-258) and add_nointersect
// (:287-328), the operators of the commented-out BC in
// include/betweenness_centrality.h:5-123.  FP64 arithmetic keeps the
// reference's order of operations per output value, and its `x += a * b`
// (which the reference's x86-64-v3 build contracts into one fused
// multiply-add) is one fma here, so the results are bit-exact with it.
//
// B200 design: each operator is one or two streaming or gather passes,
// balanced over entries rather than rows (a row index per entry, written once
// with coalesced stores), so a hub row never becomes one warp's serial loop.
//  * add_nointersect: C's row pointers are A's plus B's; an A entry lands at
//    its offset in A's row plus the number of B entries of the row with a
//    column <= its own (B first on equal columns, as the reference's merge),
//    a B entry at its offset plus the A entries with a smaller column — one
//    binary search per entry, no merge loop.
//  * dense masked eWiseMult: C zeroed, then a thread per mask entry.
//  * fuseEWiseMultAdd: one grid-stride fma pass over the m·n values.
//  * mxmm_spd: a thread per mask entry (i, c) sums A(i,j)·B(j,c) over row i
//    of A in order, the reference's order for that output value.
// The reference's defect in add_nointersect (its B-tail copy indexes B with
// A's cursor, matrix_la.h:320-322) is not reproduced: C is the true merge.
#include "gk_common.cuh"

namespace gk {

// Row index of every entry of X (warp per row, coalesced stores).
static __global__ void k_entry_rows(int64_t m, const int64_t *rp, int32_t *row) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < m; i += warps)
        for (int64_t p = rp[i] + lane; p < rp[i + 1]; p += 32) row[p] = static_cast<int32_t>(i);
}

static __global__ void k_add_rowptr(int64_t m, const int64_t *arp, const int64_t *brp, int64_t *crp) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= m; i += stride) crp[i] = arp[i] + brp[i];
}

// Places every entry of X into C: its offset within X's row plus the number of
// Y entries of the row before it (columns < x, or <= x when Y goes first on
// equal columns).
static __global__ void k_add_place(DevCsr X, const int32_t *xrow, DevCsr Y, int y_first_on_tie, const int64_t *crp,
                                   int32_t *ccol, int32_t *cval) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < X.nnz; p += stride) {
        const int i = xrow[p];
        const int32_t x = X.col[p];
        int64_t lo = Y.rp[i], hi = Y.rp[i + 1];
        while (lo < hi) {
            const int64_t md = (lo + hi) >> 1;
            const int32_t y = Y.col[md];
            if (y < x || (y_first_on_tie && y == x)) lo = md + 1;
            else hi = md;
        }
        const int64_t out = crp[i] + (p - X.rp[i]) + (lo - Y.rp[i]);
        ccol[out] = x;
        if (cval) cval[out] = X.val ? X.val[p] : 1;
    }
}

static __global__ void k_ewise_masked(DevCsr M, const int32_t *mrow, int64_t n, const double *A, const double *B,
                                      double *C) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < M.nnz; q += stride) {
        const int64_t idx = (int64_t)mrow[q] * n + M.col[q];
        C[idx] = A[idx] * B[idx];
    }
}

static __global__ void k_fuse_mult_add(int64_t count, const double *A, const double *B, double *C) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        C[i] = fma(A[i], B[i], C[i]);
}

static __global__ void k_spd(DevCsr A, const double *aval, DevCsr M, const int32_t *mrow, int64_t n, const double *B,
                             double *C) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < M.nnz; q += stride) {
        const int64_t i = mrow[q];
        const int32_t c = M.col[q];
        double acc = 0.0;
        for (int64_t t = A.rp[i]; t < A.rp[i + 1]; ++t) {
            const double a = aval ? aval[t] : (A.val ? static_cast<double>(A.val[t]) : 1.0);
            acc = fma(a, B[(int64_t)A.col[t] * n + c], acc);
        }
        C[i * n + c] = acc;
    }
}

// A device copy of `count` values at src (used in place when already there).
template <class T>
static int stage_in(const T *src, size_t count, const T **out, Scratch &scr, cudaStream_t s) {
    if (count == 0 || !src || is_device_pointer(src)) {
        *out = src;
        return GK_OK;
    }
    T *d;
    GK_CHECK(scr.alloc(&d, count));
    GK_CUDA(cudaMemcpyAsync(d, src, sizeof(T) * count, cudaMemcpyHostToDevice, s));
    *out = d;
    return GK_OK;
}

// Device buffer for an output of `count` values: dst itself when it is device
// memory, else scratch that finish_out copies back.
template <class T>
static int out_buffer(T *dst, size_t count, T **out, Scratch &scr) {
    if (count == 0 || !dst || is_device_pointer(dst)) {
        *out = dst;
        return GK_OK;
    }
    return scr.alloc(out, count);
}

template <class T>
static int finish_out(T *dst, const T *dev, size_t count, cudaStream_t s) {
    if (count == 0 || !dst || dst == dev) return GK_OK;
    GK_CUDA(cudaMemcpyAsync(dst, dev, sizeof(T) * count, cudaMemcpyDeviceToHost, s));
    return GK_OK;
}

static int entry_rows(const DevCsr &X, int32_t **row, Scratch &scr, cudaStream_t s) {
    GK_CHECK(scr.alloc(row, X.nnz > 0 ? X.nnz : 1));
    if (X.m > 0 && X.nnz > 0) {
        k_entry_rows<<<ctx().num_sms * 8, 256, 0, s>>>(X.m, X.rp, *row);
        note_launches(1);
        GK_CUDA(cudaGetLastError());
    }
    return GK_OK;
}

static int grid_for(int64_t work) {
    const int64_t blocks = (work + 255) / 256;
    const int64_t cap = int64_t(ctx().num_sms) * 16;
    return static_cast<int>(blocks < 1 ? 1 : (blocks < cap ? blocks : cap));
}

static int check_dense_args(int64_t m, int64_t n, const void *A, const void *B, const void *C) {
    if (m < 0 || n < 0) return fail(GK_ERR_ARG, "negative dense dimension");
    if (m > 0 && n > 0 && (!A || !B || !C)) return fail(GK_ERR_ARG, "null dense operand");
    return GK_OK;
}

}  // namespace gk

using namespace gk;

extern "C" int gk_add_nointersect(const gk_csr *A, const gk_csr *B, int64_t *C_rowptr, int32_t *C_col,
                                  int32_t *C_val, void *stream) {
    GK_CHECK(validate_csr_shape(A, "A"));
    GK_CHECK(validate_csr_shape(B, "B"));
    if (A->m != B->m || A->n != B->n) return fail(GK_ERR_ARG, "add_nointersect: A and B must have the same shape");
    const int64_t m = A->m, nnz = A->nnz + B->nnz;
    if (!C_rowptr || (nnz > 0 && !C_col)) return fail(GK_ERR_ARG, "add_nointersect: null output");
    if (nnz >= (int64_t(1) << 62)) return fail(GK_ERR_UNSUPPORTED, "add_nointersect: too many entries");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    DevCsr a, b;
    GK_CHECK(stage_csr(A, &a, scr, s, nullptr, CSR_SORTED, "A"));
    GK_CHECK(stage_csr(B, &b, scr, s, nullptr, CSR_SORTED, "B"));
    int64_t *crp;
    int32_t *ccol, *cval = nullptr;
    GK_CHECK(out_buffer(C_rowptr, static_cast<size_t>(m + 1), &crp, scr));
    GK_CHECK(out_buffer(C_col, static_cast<size_t>(nnz), &ccol, scr));
    if (C_val) GK_CHECK(out_buffer(C_val, static_cast<size_t>(nnz), &cval, scr));
    k_add_rowptr<<<grid_for(m + 1), 256, 0, s>>>(m, a.rp, b.rp, crp);
    note_launches(1);
    GK_CUDA(cudaGetLastError());
    int32_t *arow, *brow;
    GK_CHECK(entry_rows(a, &arow, scr, s));
    GK_CHECK(entry_rows(b, &brow, scr, s));
    if (a.nnz > 0) {
        k_add_place<<<grid_for(a.nnz), 256, 0, s>>>(a, arow, b, 1, crp, ccol, cval);
        note_launches(1);
    }
    if (b.nnz > 0) {
        k_add_place<<<grid_for(b.nnz), 256, 0, s>>>(b, brow, a, 0, crp, ccol, cval);
        note_launches(1);
    }
    GK_CUDA(cudaGetLastError());
    GK_CHECK(finish_out(C_rowptr, crp, static_cast<size_t>(m + 1), s));
    GK_CHECK(finish_out(C_col, ccol, static_cast<size_t>(nnz), s));
    if (C_val) GK_CHECK(finish_out(C_val, cval, static_cast<size_t>(nnz), s));
    GK_CUDA(cudaStreamSynchronize(s));
    return GK_OK;
}

// build_symm_from_lower (include/matrix.h:662-696): the reference merges row
// i of Low with row i of Upp = transpose(Low), Upp first on equal columns.
// That is add_nointersect(Low, Upp) with the same tie rule, so the device
// path is the transpose (radix sort by column) and the two placement passes.
extern "C" int gk_build_symm_from_lower(const gk_csr *L, int64_t *out_rowptr, int32_t *out_col, int32_t *out_val,
                                        void *stream) {
    GK_CHECK(validate_csr_shape(L, "L"));
    if (L->m != L->n) return fail(GK_ERR_ARG, "build_symm_from_lower: L must be square");
    const int64_t m = L->m, nnz = 2 * L->nnz;
    if (!out_rowptr || (nnz > 0 && !out_col)) return fail(GK_ERR_ARG, "build_symm_from_lower: null output");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    DevCsr low;
    GK_CHECK(stage_csr(L, &low, scr, s, nullptr, CSR_SORTED, "L"));
    DevCsr up{m, m, low.nnz, nullptr, nullptr, nullptr};
    int64_t *urp;
    int32_t *ucol, *uval = nullptr;
    GK_CHECK(scr.alloc(&urp, m + 1));
    GK_CHECK(scr.alloc(&ucol, low.nnz > 0 ? low.nnz : 1));
    if (out_val && low.val) GK_CHECK(scr.alloc(&uval, low.nnz > 0 ? low.nnz : 1));
    GK_CHECK(transpose_device(low, urp, ucol, uval, s, scr));
    up.rp = urp;
    up.col = ucol;
    up.val = uval;
    int64_t *crp;
    int32_t *ccol, *cval = nullptr;
    GK_CHECK(out_buffer(out_rowptr, static_cast<size_t>(m + 1), &crp, scr));
    GK_CHECK(out_buffer(out_col, static_cast<size_t>(nnz), &ccol, scr));
    if (out_val) GK_CHECK(out_buffer(out_val, static_cast<size_t>(nnz), &cval, scr));
    k_add_rowptr<<<grid_for(m + 1), 256, 0, s>>>(m, low.rp, up.rp, crp);
    note_launches(1);
    GK_CUDA(cudaGetLastError());
    int32_t *lrow, *urow;
    GK_CHECK(entry_rows(low, &lrow, scr, s));
    GK_CHECK(entry_rows(up, &urow, scr, s));
    if (low.nnz > 0) {
        k_add_place<<<grid_for(low.nnz), 256, 0, s>>>(low, lrow, up, 1, crp, ccol, cval);
        k_add_place<<<grid_for(up.nnz), 256, 0, s>>>(up, urow, low, 0, crp, ccol, cval);
        note_launches(2);
    }
    GK_CUDA(cudaGetLastError());
    GK_CHECK(finish_out(out_rowptr, crp, static_cast<size_t>(m + 1), s));
    GK_CHECK(finish_out(out_col, ccol, static_cast<size_t>(nnz), s));
    if (out_val) GK_CHECK(finish_out(out_val, cval, static_cast<size_t>(nnz), s));
    GK_CUDA(cudaStreamSynchronize(s));
    return GK_OK;
}

static __global__ void k_fill_ones(int64_t n, int32_t *v) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) v[i] = 1;
}

// build_adjacency_matrix (include/matrix.h:643-660): G's pattern with every
// value 1.
extern "C" int gk_build_adjacency_matrix(const gk_csr *G, int64_t *out_rowptr, int32_t *out_col, int32_t *out_val,
                                         void *stream) {
    GK_CHECK(validate_csr_shape(G, "G"));
    const int64_t m = G->m, nnz = G->nnz;
    if (!out_rowptr || (nnz > 0 && (!out_col || !out_val)))
        return fail(GK_ERR_ARG, "build_adjacency_matrix: null output");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    DevCsr g;
    GK_CHECK(stage_csr(G, &g, scr, s, nullptr, CSR_STRUCTURE, "G"));
    GK_CUDA(cudaMemcpyAsync(out_rowptr, g.rp, sizeof(int64_t) * (m + 1), cudaMemcpyDefault, s));
    if (nnz > 0) {
        GK_CUDA(cudaMemcpyAsync(out_col, g.col, sizeof(int32_t) * nnz, cudaMemcpyDefault, s));
        int32_t *v;
        GK_CHECK(out_buffer(out_val, static_cast<size_t>(nnz), &v, scr));
        k_fill_ones<<<grid_for(nnz), 256, 0, s>>>(nnz, v);
        note_launches(1);
        GK_CUDA(cudaGetLastError());
        GK_CHECK(finish_out(out_val, v, static_cast<size_t>(nnz), s));
    }
    GK_CUDA(cudaStreamSynchronize(s));
    return GK_OK;
}

extern "C" int gk_dense_ewise_mult_masked(int64_t m, int64_t n, const double *A, const double *B, const gk_csr *M,
                                          double *C, void *stream) {
    GK_CHECK(check_dense_args(m, n, A, B, C));
    GK_CHECK(validate_csr_shape(M, "M"));
    if (M->m != m || M->n != n) return fail(GK_ERR_ARG, "dense eWiseMult: M must be m x n");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    const size_t count = static_cast<size_t>(m) * static_cast<size_t>(n);
    DevCsr mk;
    GK_CHECK(stage_csr(M, &mk, scr, s, nullptr, CSR_SORTED, "M"));
    const double *da, *db;
    double *dc;
    GK_CHECK(stage_in(A, count, &da, scr, s));
    GK_CHECK(stage_in(B, count, &db, scr, s));
    GK_CHECK(out_buffer(C, count, &dc, scr));
    if (count > 0) GK_CUDA(cudaMemsetAsync(dc, 0, sizeof(double) * count, s));
    int32_t *mrow;
    GK_CHECK(entry_rows(mk, &mrow, scr, s));
    if (mk.nnz > 0) {
        k_ewise_masked<<<grid_for(mk.nnz), 256, 0, s>>>(mk, mrow, n, da, db, dc);
        note_launches(1);
        GK_CUDA(cudaGetLastError());
    }
    GK_CHECK(finish_out(C, dc, count, s));
    GK_CUDA(cudaStreamSynchronize(s));
    return GK_OK;
}

extern "C" int gk_dense_fuse_ewise_mult_add(int64_t count, const double *A, const double *B, double *C,
                                            void *stream) {
    GK_CHECK(check_dense_args(count, 1, A, B, C));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    const size_t cnt = static_cast<size_t>(count);
    const double *da, *db, *dcin;
    double *dc;
    GK_CHECK(stage_in(A, cnt, &da, scr, s));
    GK_CHECK(stage_in(B, cnt, &db, scr, s));
    GK_CHECK(stage_in(static_cast<const double *>(C), cnt, &dcin, scr, s));  // C is read and written
    dc = const_cast<double *>(dcin);
    if (count > 0) {
        k_fuse_mult_add<<<grid_for(count), 256, 0, s>>>(count, da, db, dc);
        note_launches(1);
        GK_CUDA(cudaGetLastError());
    }
    GK_CHECK(finish_out(C, dc, cnt, s));
    GK_CUDA(cudaStreamSynchronize(s));
    return GK_OK;
}

extern "C" int gk_mxmm_spd(const gk_csr *A, const double *A_val, const double *B, int64_t n, const gk_csr *M,
                           double *C, void *stream) {
    GK_CHECK(validate_csr_shape(A, "A"));
    GK_CHECK(validate_csr_shape(M, "M"));
    if (n < 0) return fail(GK_ERR_ARG, "mxmm_spd: negative n");
    if (M->m != A->m || M->n != n) return fail(GK_ERR_ARG, "mxmm_spd: need M.m == A.m and M.n == n");
    const int64_t m = A->m, k = A->n;
    if ((k > 0 && n > 0 && !B) || (m > 0 && n > 0 && !C)) return fail(GK_ERR_ARG, "mxmm_spd: null dense operand");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    DevCsr a, mk;
    GK_CHECK(stage_csr(A, &a, scr, s, nullptr, CSR_STRUCTURE, "A"));
    GK_CHECK(stage_csr(M, &mk, scr, s, nullptr, CSR_SORTED, "M"));
    const double *dav = nullptr, *db;
    GK_CHECK(stage_in(A_val, static_cast<size_t>(A->nnz), &dav, scr, s));
    const size_t bcount = static_cast<size_t>(k) * static_cast<size_t>(n);
    const size_t ccount = static_cast<size_t>(m) * static_cast<size_t>(n);
    GK_CHECK(stage_in(B, bcount, &db, scr, s));
    // C may be B itself (the reference's mxmm_spd(Af, W, S, W, Wbuf)): then
    // the product goes to scratch first
    double *dc;
    if (ccount > 0 && static_cast<const void *>(C) == static_cast<const void *>(B)) GK_CHECK(scr.alloc(&dc, ccount));
    else GK_CHECK(out_buffer(C, ccount, &dc, scr));
    if (ccount > 0) GK_CUDA(cudaMemsetAsync(dc, 0, sizeof(double) * ccount, s));
    int32_t *mrow;
    GK_CHECK(entry_rows(mk, &mrow, scr, s));
    if (mk.nnz > 0) {
        k_spd<<<grid_for(mk.nnz), 256, 0, s>>>(a, dav, mk, mrow, n, db, dc);
        note_launches(1);
        GK_CUDA(cudaGetLastError());
    }
    if (ccount > 0 && dc != C) {
        GK_CUDA(cudaMemcpyAsync(C, dc, sizeof(double) * ccount, cudaMemcpyDefault, s));
    }
    GK_CUDA(cudaStreamSynchronize(s));
    return GK_OK;
}
