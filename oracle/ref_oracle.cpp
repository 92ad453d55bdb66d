// Reference oracle — TEST INFRASTRUCTURE ONLY.
//
// One translation unit that compiles the reference's own headers
// (GraphKokkos include/matrix.h, include/matrix_la.h,
// include/betweenness_centrality.h — read in place, never copied) against the
// Kokkos-API shim in oracle/kokkos_shim, and exports them through a plain C
// interface so that tests can run the reference algorithms on the same seeded
// inputs as the CUDA path.  The reference functions that live in
// src/main.cpp next to main() are restated here, each with a citation; every
// other call goes into the reference code unmodified.
//
// Built by oracle/Makefile into oracle/_ref/libgk_ref.so.  Only tests/,
// the smoke check and bench.py's CPU-baseline leg may load it.
#include "matrix.h"
#include "matrix_la.h"
#include "betweenness_centrality.h"

#include <cstdint>
#include <cstdio>
#include <sstream>
#include <vector>

template <typename T>
using mxmOp = void (*)(bool, const spMtx<T> &, const spMtx<T> &, const spMtx<T> &, spMtx<T> &);

namespace {

// Builds a reference spMtx<int> from int64 row pointers and int32 columns
// (values default to 1, the adjacency convention of matrix.h:643-660).
spMtx<int> make_mtx(int64_t m, int64_t n, const int64_t *rp, const int32_t *col, const int32_t *val) {
    const int64_t nz = rp[m];
    spMtx<int> A(static_cast<size_t>(m), static_cast<size_t>(n), static_cast<size_t>(nz));
    for (int64_t i = 0; i <= m; ++i) A.Rst(i) = static_cast<int>(rp[i]);
    for (int64_t j = 0; j < nz; ++j) {
        A.Col(j) = col[j];
        A.Val(j) = val ? val[j] : 1;
    }
    std::memcpy(A.matcode, "MCIG", 4);
    return A;
}

// The reference's parallel MSA (matrix_la.h:590-595) splits rows over
// T = Kokkos::num_threads() teams with `if (A.Rst[i] >= A.nz * team_i / T)
// work_distribution(team_i++) = i` over every i <= m.  When A.nz < T the
// threshold A.nz * (T + 1) / T equals A.nz, so each trailing row with
// Rst == nz writes one more entry past the T + 1 the View holds (and with
// A.nz == 0 every row does): a heap overflow.  A.nz >= T keeps every write in
// bounds, so this wrapper runs the reference with min(T, A.nz) threads, and
// for an operand without entries returns what the reference defines without
// calling it: C with M's pattern (matrix_la.h:564-568) and zero values.
struct ThreadCap {
    int saved;
    explicit ThreadCap(int64_t nz) : saved(omp_get_max_threads()) {
        if (nz < saved) omp_set_num_threads(static_cast<int>(nz > 0 ? nz : 1));
    }
    ~ThreadCap() { omp_set_num_threads(saved); }
};

void msa_guarded(bool isParallel, const spMtx<int> &A, const spMtx<int> &B, const spMtx<int> &M, spMtx<int> &C) {
    if (A.nz == 0) {
        C.resizeRows(M.m);
        C.resizeVals(M.nz);
        C.n = M.n;
        Kokkos::deep_copy(C.Col, M.Col);
        Kokkos::deep_copy(C.Rst, M.Rst);
        for (size_t j = 0; j < M.nz; ++j) C.Val(j) = 0;
        return;
    }
    ThreadCap cap(static_cast<int64_t>(A.nz));
    mxmm_msa<int, int>(isParallel, A, B, M, C);
}

mxmOp<int> pick(int accum) {
    switch (accum) {
        case 0: return msa_guarded;
        case 1: return mxmm_mca<int, int>;
        case 2: return mxmm_naive<int>;
        default: return nullptr;
    }
}

// Silences the per-phase timing lines that betweenness_centrality_batch
// prints to std::cerr (betweenness_centrality.h:499-503).
struct MuteCerr {
    std::ostringstream sink;
    std::streambuf *old;
    MuteCerr() : old(std::cerr.rdbuf(sink.rdbuf())) {}
    ~MuteCerr() { std::cerr.rdbuf(old); }
};

// Restatement of triangle_counting_masked_sandia (src/main.cpp:69-90) without
// the stdout lines; L = extract_lower_triangle(A) (matrix.h:698-726) is
// untimed in the reference and computed here the same way.
int64_t tc_sandia(const spMtx<int> &A, mxmOp<int> matrixMult, bool isParallel) {
    int64_t num_of_tr = 0;
    spMtx<int> L = std::move(extract_lower_triangle(A));
    spMtx<int> C;
    matrixMult(isParallel, L, L, L, C);
    Kokkos::parallel_reduce("", C.nz, KOKKOS_LAMBDA(int64_t i, int64_t &sum) { sum += C.Val(i); },
                            Kokkos::Sum<int64_t>(num_of_tr));
    return num_of_tr;
}

// Restatement of triangle_counting_vertex (src/main.cpp:16-39) without the
// timing line: SQ<A> = A·A, nums[i] = (row sum of SQ) >> 1.
void tc_vertex(const spMtx<int> &A, mxmOp<int> matrixMult, bool isParallel, int32_t *nums) {
    spMtx<int> SQ;
    matrixMult(isParallel, A, A, A, SQ);
    for (size_t i = 0; i < A.m; ++i) {
        int num_of_tr = 0;
        for (int j = SQ.Rst(i); j < SQ.Rst(i + 1); ++j) num_of_tr += SQ.Val(j);
        nums[i] = num_of_tr >> 1;
    }
}

// Restatement of triangle_counting_masked_lu (src/main.cpp:42-66) without the
// stdout lines: C<A> = L·U with L = tril(A), U = transpose(L); sum(C) >> 1.
int64_t tc_lu(const spMtx<int> &A, mxmOp<int> matrixMult, bool isParallel) {
    int64_t num_of_tr = 0;
    spMtx<int> L = std::move(extract_lower_triangle(A));
    spMtx<int> U = std::move(transpose(L));
    spMtx<int> C;
    matrixMult(isParallel, L, U, A, C);
    for (int j = 0; j < C.Rst(C.m); ++j) num_of_tr += C.Val(j);
    return num_of_tr >> 1;
}

// Restatement of k_truss (src/main.cpp:94-141) without the stdout lines.
// The one change: tmp_Xdj has n+1 entries (the reference sizes it n at
// main.cpp:99 but writes index n at :118 and deep-copies it into an n+1
// Rst at :120, which leaves Rst(n) stale and stops the loop after one pass).
spMtx<int> k_truss_fixed(const spMtx<int> &A, int k, mxmOp<int> matrixMult, bool isParallel, int *iters) {
    spMtx<int> C = A;
    spMtx<int> Tmp;
    int n = A.m;
    int totalIterationNum = 0;
    Kokkos::View<int *> tmp_Xdj("", n + 1);
    tmp_Xdj(0) = 0;
    for (int t = 0; t < n; ++t) {
        matrixMult(isParallel, C, C, C, Tmp);
        int new_curr_pos = 0;
        for (int i = 0; i < n; ++i) {
            for (int j = Tmp.Rst(i); j < Tmp.Rst(i + 1); ++j) {
                if (Tmp.Val(j) >= k - 2) {
                    Tmp.Col(new_curr_pos) = Tmp.Col[j];
                    Tmp.Val(new_curr_pos++) = 1;
                }
            }
            tmp_Xdj(i + 1) = new_curr_pos;
        }
        Kokkos::deep_copy(Tmp.Rst, tmp_Xdj);
        Tmp.nz = Tmp.Rst(n);
        if (Tmp.nz == C.nz) {
            totalIterationNum = ++t;
            break;
        }
        std::swap(C, Tmp);
    }
    Kokkos::resize(C.Col, C.nz);
    Kokkos::resize(C.Val, C.nz);
    if (iters) *iters = totalIterationNum;
    return C;
}

spMtx<double> make_mtx_d(int64_t m, int64_t n, const int64_t *rp, const int32_t *col, const double *val) {
    const int64_t nz = rp[m];
    spMtx<double> A(static_cast<size_t>(m), static_cast<size_t>(n), static_cast<size_t>(nz));
    for (int64_t i = 0; i <= m; ++i) A.Rst(i) = static_cast<int>(rp[i]);
    for (int64_t j = 0; j < nz; ++j) {
        A.Col(j) = col[j];
        A.Val(j) = val ? val[j] : 1.0;
    }
    return A;
}

denseMtx<double> make_dense(int64_t m, int64_t n, const double *v) {
    denseMtx<double> D(static_cast<size_t>(m), static_cast<size_t>(n));
    for (int64_t i = 0; i < m * n; ++i) D.Val(i) = v[i];
    return D;
}

void export_csr(const spMtx<int> &R, int64_t *rp, int32_t *col, int32_t *val) {
    for (size_t i = 0; i <= R.m; ++i) rp[i] = R.Rst(i);
    for (size_t j = 0; j < R.nz; ++j) {
        if (col) col[j] = R.Col(j);
        if (val) val[j] = R.Val(j);
    }
}

}  // namespace

extern "C" {

int ref_num_threads(void) { return Kokkos::num_threads(); }
int ref_get_threads(void) { return omp_get_max_threads(); }
void ref_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }

// C<M> = A·B through the reference operator selected by `accum`
// (0 mxmm_msa matrix_la.h:562-694, 1 mxmm_mca :478-528, 2 mxmm_naive
// :936-1068).  Writes nnz(M) values in M's pattern order.
int ref_mxmm(int accum, int parallel,
             int64_t am, int64_t an, const int64_t *arp, const int32_t *acol, const int32_t *aval,
             int64_t bm, int64_t bn, const int64_t *brp, const int32_t *bcol, const int32_t *bval,
             int64_t mm, int64_t mn, const int64_t *mrp, const int32_t *mcol,
             int32_t *c_val) {
    try {
        mxmOp<int> op = pick(accum);
        if (!op) return -2;
        spMtx<int> A = make_mtx(am, an, arp, acol, aval);
        spMtx<int> B = make_mtx(bm, bn, brp, bcol, bval);
        spMtx<int> M = make_mtx(mm, mn, mrp, mcol, nullptr);
        spMtx<int> C;
        op(parallel != 0, A, B, M, C);
        if (C.nz != M.nz) return -3;
        for (size_t j = 0; j < C.nz; ++j) c_val[j] = C.Val(j);
        return 0;
    } catch (...) {
        return -1;
    }
}

// The reference's complement-masked product mxmm_msa_cmask (matrix_la.h:733-934).
// Two calls as orc_mxmm_cmask: c_col == nullptr gives c_rp only.
int ref_mxmm_cmask(int parallel,
                   int64_t am, int64_t an, const int64_t *arp, const int32_t *acol, const int32_t *aval,
                   int64_t bm, int64_t bn, const int64_t *brp, const int32_t *bcol, const int32_t *bval,
                   int64_t mm, int64_t mn, const int64_t *mrp, const int32_t *mcol,
                   int64_t *c_rp, int32_t *c_col, int32_t *c_val) {
    try {
        spMtx<int> A = make_mtx(am, an, arp, acol, aval);
        spMtx<int> B = make_mtx(bm, bn, brp, bcol, bval);
        spMtx<int> M = make_mtx(mm, mn, mrp, mcol, nullptr);
        spMtx<int> C;
        mxmm_msa_cmask(parallel != 0, A, B, M, C);
        for (size_t i = 0; i <= C.m; ++i) c_rp[i] = C.Rst(i);
        if (c_col)
            for (size_t j = 0; j < C.nz; ++j) {
                c_col[j] = C.Col(j);
                c_val[j] = C.Val(j);
            }
        return 0;
    } catch (...) {
        return -1;
    }
}

// The reference's add_nointersect (matrix_la.h:287-328).  It sizes its result
// by the output's row count and loops over it (:295-299), so C starts with m
// rows.  Its copy of a row's remaining B entries reads B at A's cursor
// (:320-322): call it only where every row's last entry comes from A.
int ref_add_nointersect(int64_t m, int64_t n, const int64_t *arp, const int32_t *acol, const int32_t *aval,
                        const int64_t *brp, const int32_t *bcol, const int32_t *bval, int64_t *crp, int32_t *ccol,
                        int32_t *cval) {
    try {
        spMtx<int> A = make_mtx(m, n, arp, acol, aval);
        spMtx<int> B = make_mtx(m, n, brp, bcol, bval);
        spMtx<int> C(static_cast<size_t>(m), static_cast<size_t>(n)), Cbuf;
        add_nointersect(A, B, C, Cbuf);
        export_csr(C, crp, ccol, cval);
        return 0;
    } catch (...) {
        return -1;
    }
}

// The reference's dense masked eWiseMult (matrix_la.h:189-208).
int ref_dense_ewise_mult_masked(int64_t m, int64_t n, const double *A, const double *B, const int64_t *mrp,
                                const int32_t *mcol, double *C) {
    denseMtx<double> a = make_dense(m, n, A), b = make_dense(m, n, B), c(static_cast<size_t>(m), static_cast<size_t>(n));
    spMtx<int> M = make_mtx(m, n, mrp, mcol, nullptr);
    eWiseMult(a, b, M, c);
    for (int64_t i = 0; i < m * n; ++i) C[i] = c.Val(i);
    return 0;
}

// The reference's fuseEWiseMultAdd (matrix_la.h:182-187) on a 1 x count matrix.
int ref_fuse_ewise_mult_add(int64_t count, const double *A, const double *B, double *C) {
    denseMtx<double> a = make_dense(1, count, A), b = make_dense(1, count, B), c = make_dense(1, count, C);
    fuseEWiseMultAdd(a, b, c);
    for (int64_t i = 0; i < count; ++i) C[i] = c.Val(i);
    return 0;
}

// The reference's mxmm_spd (matrix_la.h:230-258) with FP64 values.
int ref_mxmm_spd(int64_t m, int64_t k, const int64_t *arp, const int32_t *acol, const double *aval, int64_t n,
                 const double *B, const int64_t *mrp, const int32_t *mcol, double *C) {
    spMtx<double> A = make_mtx_d(m, k, arp, acol, aval);
    denseMtx<double> b = make_dense(k, n, B);
    spMtx<int> M = make_mtx(m, n, mrp, mcol, nullptr);
    denseMtx<double> c(static_cast<size_t>(m), static_cast<size_t>(n)), cbuf(static_cast<size_t>(m), static_cast<size_t>(n));
    mxmm_spd(A, b, M, c, cbuf);
    for (int64_t i = 0; i < m * n; ++i) C[i] = c.Val(i);
    return 0;
}

// Triangle count of a symmetric adjacency matrix (sorted rows, no self-loops).
int ref_tc_sandia(int accum, int parallel, int64_t m, const int64_t *rp, const int32_t *col, int64_t *out) {
    try {
        mxmOp<int> op = pick(accum);
        if (!op) return -2;
        spMtx<int> A = make_mtx(m, m, rp, col, nullptr);
        *out = tc_sandia(A, op, parallel != 0);
        return 0;
    } catch (...) {
        return -1;
    }
}

// The reference's file readers (spMtx(const char *, format), matrix.h:44-60):
// call with null arrays for the sizes, then with arrays of those sizes.
int ref_read_matrix(const char *path, const char *format, int64_t *m, int64_t *n, int64_t *nz, int64_t *rp,
                    int32_t *col, int32_t *val) {
    try {
        spMtx<int> A(path, std::string(format));
        *m = static_cast<int64_t>(A.m);
        *n = static_cast<int64_t>(A.n);
        *nz = static_cast<int64_t>(A.nz);
        if (rp)
            for (size_t i = 0; i <= A.m; ++i) rp[i] = A.Rst(i);
        if (col)
            for (size_t j = 0; j < A.nz; ++j) col[j] = A.Col(j);
        if (val)
            for (size_t j = 0; j < A.nz; ++j) val[j] = A.Val(j);
        return 0;
    } catch (...) {
        return -1;
    }
}

int ref_tc_vertex(int accum, int parallel, int64_t m, const int64_t *rp, const int32_t *col, int32_t *out) {
    try {
        mxmOp<int> op = pick(accum);
        if (!op) return -2;
        spMtx<int> A = make_mtx(m, m, rp, col, nullptr);
        tc_vertex(A, op, parallel != 0, out);
        return 0;
    } catch (...) {
        return -1;
    }
}

int ref_tc_lu(int accum, int parallel, int64_t m, const int64_t *rp, const int32_t *col, int64_t *out) {
    try {
        mxmOp<int> op = pick(accum);
        if (!op) return -2;
        spMtx<int> A = make_mtx(m, m, rp, col, nullptr);
        *out = tc_lu(A, op, parallel != 0);
        return 0;
    } catch (...) {
        return -1;
    }
}

// Same as ref_tc_sandia but starting from the strict lower triangle L, with
// the rows to multiply restricted to [row_begin, row_end): A = M = those rows
// of L, B = all of L.  Used as a bounded CPU sample of a large graph.
int ref_tc_rows(int parallel, int64_t m, const int64_t *rp, const int32_t *col,
                int64_t row_begin, int64_t row_end, int64_t *out) {
    try {
        spMtx<int> L = make_mtx(m, m, rp, col, nullptr);
        spMtx<int> S(static_cast<size_t>(m), static_cast<size_t>(m),
                     static_cast<size_t>(rp[row_end] - rp[row_begin]));
        for (int64_t i = 0; i <= m; ++i) {
            int64_t r = i < row_begin ? row_begin : (i > row_end ? row_end : i);
            S.Rst(i) = static_cast<int>(rp[r] - rp[row_begin]);
        }
        for (int64_t j = rp[row_begin]; j < rp[row_end]; ++j) {
            S.Col(j - rp[row_begin]) = col[j];
            S.Val(j - rp[row_begin]) = 1;
        }
        spMtx<int> C;
        msa_guarded(parallel != 0, S, L, S, C);
        int64_t num_of_tr = 0;
        Kokkos::parallel_reduce("", C.nz, KOKKOS_LAMBDA(int64_t i, int64_t &sum) { sum += C.Val(i); },
                                Kokkos::Sum<int64_t>(num_of_tr));
        *out = num_of_tr;
        return 0;
    } catch (...) {
        return -1;
    }
}

// Bounded sample for CPU timing: C<S> = S·L through the reference mxmm_msa,
// with S = the listed rows of L (a uniform random sample of the rows, sorted),
// compacted to a matrix of those rows only (nrows rows, m columns): the
// reference's per-call costs that scale with the row count (the copy of M's
// pattern into C, matrix_la.h:564-568, and the serial work split, :590-596)
// then follow the sample, not the whole graph, so the measured rate is the
// rate of the reference's row loop.  The shim's per-thread scratch is kept
// between calls and not zero-filled here, as Kokkos' own scratch pool is (the
// MSA clears its accumulator at the mask columns before each row, :614-616).
// Returns the sum of C (the sampled rows' share of the triangle count) and the
// number of sampled L entries; `seconds` receives the time inside mxmm_msa
// plus the sum, the reference's own bracket (src/main.cpp:74-85).
int ref_tc_rows_sample(int64_t m, const int64_t *rp, const int32_t *col, int64_t nrows, const int64_t *rows,
                       int64_t *out, int64_t *sample_nnz, double *seconds) {
    try {
        spMtx<int> L = make_mtx(m, m, rp, col, nullptr);
        int64_t nz = 0;
        for (int64_t r = 0; r < nrows; ++r) nz += rp[rows[r] + 1] - rp[rows[r]];
        if (nz == 0) {  // no entries: the sample's count is 0 (see msa_guarded)
            *out = 0;
            *sample_nnz = 0;
            *seconds = 0.0;
            return 0;
        }
        spMtx<int> S(static_cast<size_t>(nrows), static_cast<size_t>(m), static_cast<size_t>(nz));
        int64_t pos = 0;
        S.Rst(0) = 0;
        for (int64_t r = 0; r < nrows; ++r) {
            const int64_t i = rows[r];
            for (int64_t j = rp[i]; j < rp[i + 1]; ++j) {
                S.Col(pos) = col[j];
                S.Val(pos++) = 1;
            }
            S.Rst(r + 1) = static_cast<int>(pos);
        }
        spMtx<int> C;
        ThreadCap cap(nz);
        kokkos_shim::ScratchZeroFill keep_scratch(false);
        auto t0 = std::chrono::steady_clock::now();
        mxmm_msa(true, S, L, S, C);
        int64_t num_of_tr = 0;
        Kokkos::parallel_reduce("", C.nz, KOKKOS_LAMBDA(int64_t i, int64_t &sum) { sum += C.Val(i); },
                                Kokkos::Sum<int64_t>(num_of_tr));
        auto t1 = std::chrono::steady_clock::now();
        *seconds = std::chrono::duration<double>(t1 - t0).count();
        *out = num_of_tr;
        *sample_nnz = nz;
        return 0;
    } catch (...) {
        return -1;
    }
}

// k-truss (restated loop, see k_truss_fixed).  out_rp has m+1 entries,
// out_col capacity nnz(A).
int ref_ktruss(int accum, int parallel, int64_t m, const int64_t *rp, const int32_t *col, int k,
               int64_t *out_rp, int32_t *out_col, int64_t *out_nnz, int *out_iters) {
    try {
        mxmOp<int> op = pick(accum);
        if (!op) return -2;
        spMtx<int> A = make_mtx(m, m, rp, col, nullptr);
        spMtx<int> R = k_truss_fixed(A, k, op, parallel != 0, out_iters);
        export_csr(R, out_rp, out_col, nullptr);
        *out_nnz = static_cast<int64_t>(R.nz);
        return 0;
    } catch (...) {
        return -1;
    }
}

// Batched BC of the reference (betweenness_centrality.h:406-506) with
// sources 0..b-1, FP32 scores.
int ref_bc_batch(int parallel, int64_t m, const int64_t *rp, const int32_t *col, int64_t b, float *bc_out) {
    try {
        spMtx<int> A = make_mtx(m, m, rp, col, nullptr);
        MuteCerr mute;
        std::vector<float> bc = betweenness_centrality_batch(parallel != 0, A, static_cast<size_t>(b));
        for (int64_t i = 0; i < m; ++i) bc_out[i] = bc[i];
        return 0;
    } catch (...) {
        return -1;
    }
}

// CSR transforms (matrix_la.h:155-179, matrix.h:662-726).
int ref_transpose(int64_t m, int64_t n, const int64_t *rp, const int32_t *col, const int32_t *val,
                  int64_t *out_rp, int32_t *out_col, int32_t *out_val) {
    try {
        spMtx<int> A = make_mtx(m, n, rp, col, val);
        spMtx<int> T = transpose(A);
        export_csr(T, out_rp, out_col, out_val);
        return 0;
    } catch (...) {
        return -1;
    }
}

int ref_extract_lower(int64_t m, const int64_t *rp, const int32_t *col,
                      int64_t *out_rp, int32_t *out_col, int64_t *out_nnz) {
    try {
        spMtx<int> A = make_mtx(m, m, rp, col, nullptr);
        spMtx<int> L = extract_lower_triangle(A);
        export_csr(L, out_rp, out_col, nullptr);
        *out_nnz = static_cast<int64_t>(L.nz);
        return 0;
    } catch (...) {
        return -1;
    }
}

int ref_build_symm_from_lower(int64_t m, const int64_t *rp, const int32_t *col,
                              int64_t *out_rp, int32_t *out_col, int64_t *out_nnz) {
    try {
        spMtx<int> L = make_mtx(m, m, rp, col, nullptr);
        spMtx<int> S = build_symm_from_lower(L);
        export_csr(S, out_rp, out_col, nullptr);
        *out_nnz = static_cast<int64_t>(S.Rst(S.m));
        return 0;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
