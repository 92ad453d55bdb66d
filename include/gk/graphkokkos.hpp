// graphkokkos.hpp — header-only C++ drop-in for GraphKokkos' hot path.
//
// Provides the reference's type and function names with the reference's
// signatures, implemented on top of the C ABI in gk_b200.h (libgk_b200.so):
//
//   spMtx<T>            include/matrix.h:33-175 (m, n, nz, Rst, Col, Val; shallow
//                       reference-counted copies, deep_copy explicit)
//   denseMtx<T>         include/matrix.h:548-630 (row-major Val(i*n+j))
//   mxmOp<T>            src/main.cpp:13-14
//   mxmm_msa / mxmm_mca / mxmm_naive / mxmm_gpu
//                       include/matrix_la.h:478-694, :936-1068 — C<M> = A·B, C
//                       resized to M's pattern with explicit zeros kept (:564-568)
//   mxmm_msa_cmask      include/matrix_la.h:733-934 — C<!M> = A·B
//   add_nointersect / eWiseMult (dense, masked) / fuseEWiseMultAdd / mxmm_spd
//                       include/matrix_la.h:182-328 (FP64 dense operands)
//   triangle_counting_masked_sandia   src/main.cpp:69-90
//   triangle_counting_vertex          src/main.cpp:16-39
//   triangle_counting_masked_lu       src/main.cpp:42-66
//   k_truss                           src/main.cpp:94-141
//   betweenness_centrality_batch      include/betweenness_centrality.h:406-506
//   transpose / extract_lower_triangle / build_symm_from_lower /
//   build_adjacency_matrix            include/matrix_la.h:155-179, include/matrix.h:643-726
//
// Differences from the reference, all deliberate:
//   * storage is host memory owned by std::shared_ptr (no Kokkos); Rst is
//     int64 so graphs beyond 2^31 entries fit;
//   * every operation runs on the GPU through libgk_b200.so; `isParallel` is
//     accepted and ignored;
//   * errors throw std::runtime_error carrying gk_last_error_string() (the
//     reference throws const char* / int);
//   * betweenness_centrality_batch(isParallel, A, b) keeps the reference's
//     float return type and sources 0..b-1 but computes in FP64; the overload
//     taking a source list returns the FP64 scores.
//
// Scheduler.  The reference picks its multiply by name (src/main.cpp:194-212);
// here every call takes the process-wide schedule: the plain row-binning
// heuristic by default, or the learned one after
//   gk::use_learned_scheduler("graphkokkos_b200/sched/model.bin",
//                             "graphkokkos_b200/sched/bc_model.bin");
// or, without code changes, from the environment: GK_SCHED=learned with
// GK_SCHED_MODEL and GK_BC_SCHED_MODEL naming the two model files (a model the
// host already loaded with gk_sched_load_model_file / gk_bc_load_model_file
// is used when the variable is unset).  The schedule changes which kernels
// run, never the results.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../gk_b200.h"

namespace gkb_detail {

inline void check(int status) {
    if (status != GK_OK) throw std::runtime_error(std::string("gk_b200: ") + gk_last_error_string());
}

// Process-wide schedule of the row-bin scheduler and of the BC level shapes.
struct SchedChoice {
    std::atomic<int> rows{GK_SCHED_PLAIN};
    std::atomic<int> bc{GK_SCHED_PLAIN};
    std::once_flag env;
};
inline SchedChoice &sched_choice() {
    static SchedChoice c;
    return c;
}
// GK_SCHED=learned: load the models named by GK_SCHED_MODEL / GK_BC_SCHED_MODEL
// (or keep ones already loaded); a missing model is an error, not a silent
// fallback to the plain schedule.
inline void sched_from_env() {
    std::call_once(sched_choice().env, [] {
        const char *e = std::getenv("GK_SCHED");
        if (!e || std::strcmp(e, "learned") != 0) return;
        const char *rows = std::getenv("GK_SCHED_MODEL");
        const char *bc = std::getenv("GK_BC_SCHED_MODEL");
        if (rows) check(gk_sched_load_model_file(rows));
        else if (!gk_sched_has_model())
            throw std::runtime_error("gk_b200: GK_SCHED=learned needs GK_SCHED_MODEL (path of model.bin)");
        if (bc) check(gk_bc_load_model_file(bc));
        else if (!gk_bc_has_model())
            throw std::runtime_error("gk_b200: GK_SCHED=learned needs GK_BC_SCHED_MODEL (path of bc_model.bin)");
        sched_choice().rows = GK_SCHED_LEARNED;
        sched_choice().bc = GK_SCHED_LEARNED;
    });
}
inline int row_sched() {
    sched_from_env();
    return sched_choice().rows;
}
inline int bc_sched() {
    sched_from_env();
    return sched_choice().bc;
}

// Minimal shared 1-D array with the View call syntax used by the reference
// (operator() and operator[] returning T&, data(), size()).
template <typename T>
class Array {
public:
    Array() = default;
    explicit Array(size_t n) : p_(std::make_shared<std::vector<T>>(n)) {}
    T &operator()(size_t i) const { return (*p_)[i]; }
    T &operator[](size_t i) const { return (*p_)[i]; }
    T *data() const { return p_ ? p_->data() : nullptr; }
    size_t size() const { return p_ ? p_->size() : 0; }
    void resize(size_t n) {
        if (!p_) p_ = std::make_shared<std::vector<T>>(n);
        else if (p_->size() != n) {
            auto q = std::make_shared<std::vector<T>>(n);
            std::copy(p_->begin(), p_->begin() + std::min(n, p_->size()), q->begin());
            p_ = q;
        }
    }
    Array clone() const {
        Array a(size());
        if (size()) std::copy(p_->begin(), p_->end(), a.p_->begin());
        return a;
    }

private:
    std::shared_ptr<std::vector<T>> p_;
};

}  // namespace gkb_detail

namespace gk {
// Loads the learned scheduler's two models from their files and makes every
// following call use them (throws std::runtime_error naming a bad file).
inline void use_learned_scheduler(const char *model_path, const char *bc_model_path) {
    gkb_detail::sched_from_env();
    gkb_detail::check(gk_sched_load_model_file(model_path));
    gkb_detail::check(gk_bc_load_model_file(bc_model_path));
    gkb_detail::sched_choice().rows = GK_SCHED_LEARNED;
    gkb_detail::sched_choice().bc = GK_SCHED_LEARNED;
}
// Back to the plain heuristic for every following call.
inline void use_plain_scheduler() {
    gkb_detail::sched_from_env();
    gkb_detail::sched_choice().rows = GK_SCHED_PLAIN;
    gkb_detail::sched_choice().bc = GK_SCHED_PLAIN;
}
}  // namespace gk

template <typename ValT>
class spMtx {
public:
    size_t m = 0, n = 0, nz = 0;
    gkb_detail::Array<int64_t> Rst;
    gkb_detail::Array<int> Col;
    gkb_detail::Array<ValT> Val;

    spMtx() = default;
    spMtx(size_t m_, size_t n_) : m(m_), n(n_), Rst(m_ + 1) {}
    spMtx(size_t m_, size_t n_, size_t nz_) : m(m_), n(n_), nz(nz_), Rst(m_ + 1), Col(nz_), Val(nz_) {}

    void resizeRows(size_t newM) {
        m = newM;
        Rst.resize(newM + 1);
    }
    void resizeVals(size_t newNz) {
        Col.resize(newNz);
        Val.resize(newNz);
        nz = newNz;
    }
    void deep_copy(const spMtx &src) {
        m = src.m;
        n = src.n;
        nz = src.nz;
        Rst = src.Rst.clone();
        Col = src.Col.clone();
        Val = src.Val.clone();
    }
    spMtx extractRows(size_t begin, size_t end) const {
        spMtx r(end - begin, n, static_cast<size_t>(Rst[end] - Rst[begin]));
        for (size_t i = 0; i <= end - begin; ++i) r.Rst(i) = Rst(i + begin) - Rst(begin);
        for (size_t j = 0; j < r.nz; ++j) {
            r.Col(j) = Col(Rst(begin) + j);
            r.Val(j) = Val(Rst(begin) + j);
        }
        return r;
    }
    bool operator==(const spMtx &o) const {
        if (m != o.m || n != o.n || nz != o.nz) return false;
        for (size_t i = 0; i <= m; ++i)
            if (Rst(i) != o.Rst(i)) return false;
        for (size_t j = 0; j < nz; ++j)
            if (Col(j) != o.Col(j) || Val(j) != o.Val(j)) return false;
        return true;
    }
    // view of this matrix for the C ABI (values as given, or pattern-only)
    gk_csr csr(bool with_values = true) const {
        static_assert(std::is_same<ValT, int>::value, "the GPU operators take int matrices (spMtx<int>)");
        return gk_csr{static_cast<int64_t>(m), static_cast<int64_t>(n), static_cast<int64_t>(nz), Rst.data(),
                      Col.data(), with_values ? Val.data() : nullptr};
    }
};

template <typename ValT>
void deep_copy(spMtx<ValT> &dst, const spMtx<ValT> &src) {
    dst.deep_copy(src);
}

template <typename ValT>
class denseMtx {
public:
    size_t m = 0, n = 0;
    gkb_detail::Array<ValT> Val;
    denseMtx() = default;
    denseMtx(size_t m_, size_t n_) : m(m_), n(n_), Val(m_ * n_) {}
    template <typename V2>
    denseMtx(const spMtx<V2> &s) : m(s.m), n(s.n), Val(s.m * s.n) {
        for (size_t i = 0; i < s.m; ++i)
            for (int64_t k = s.Rst(i); k < s.Rst(i + 1); ++k) Val(i * n + s.Col(k)) = static_cast<ValT>(s.Val(k));
    }
};

template <typename T>
using mxmOp = void (*)(bool, const spMtx<T> &, const spMtx<T> &, const spMtx<T> &, spMtx<T> &);

namespace gkb_detail {
template <typename T, typename U>
void mxmm_with(int accum, const spMtx<T> &A, const spMtx<T> &B, const spMtx<U> &M, spMtx<T> &C) {
    static_assert(std::is_same<T, int>::value, "the GPU operators take int matrices (spMtx<int>)");
    // C takes M's pattern, explicit zeros kept (include/matrix_la.h:564-568)
    spMtx<T> R(M.m, M.n, M.nz);
    std::copy(M.Rst.data(), M.Rst.data() + M.m + 1, R.Rst.data());
    if (M.nz) std::copy(M.Col.data(), M.Col.data() + M.nz, R.Col.data());
    gk_csr a = A.csr(), b = B.csr();
    gk_csr mm{static_cast<int64_t>(M.m), static_cast<int64_t>(M.n), static_cast<int64_t>(M.nz), M.Rst.data(),
              M.Col.data(), nullptr};
    check(gk_mxmm_masked(&a, &b, &mm, R.Val.data(), GK_PLUS_TIMES, row_sched(), accum, nullptr));
    C = R;
}
}  // namespace gkb_detail

// mxmOp family (include/matrix_la.h:87-149).  All run on the GPU; the name
// selects the accumulator family the scheduler is restricted to.
template <typename T, typename U>
void mxmm_msa(bool, const spMtx<T> &A, const spMtx<T> &B, const spMtx<U> &M, spMtx<T> &C) {
    gkb_detail::mxmm_with(GK_ACCUM_MSA, A, B, M, C);
}
template <typename T, typename U>
void mxmm_mca(bool, const spMtx<T> &A, const spMtx<T> &B, const spMtx<U> &M, spMtx<T> &C) {
    gkb_detail::mxmm_with(GK_ACCUM_MCA, A, B, M, C);
}
template <typename T>
void mxmm_naive(bool, const spMtx<T> &A, const spMtx<T> &B, const spMtx<T> &M, spMtx<T> &C) {
    gkb_detail::mxmm_with(GK_ACCUM_HASH, A, B, M, C);
}
// Scheduler's choice per row bin (plain heuristic or learned model, see the top).
template <typename T>
void mxmm_gpu(bool, const spMtx<T> &A, const spMtx<T> &B, const spMtx<T> &M, spMtx<T> &C) {
    gkb_detail::mxmm_with(GK_ACCUM_AUTO, A, B, M, C);
}

// Complement-masked product C<!M> = A·B (include/matrix_la.h:733-934): C is
// resized to the product's pattern minus M's, rows sorted.
template <typename T, typename U>
void mxmm_msa_cmask(bool, const spMtx<T> &A, const spMtx<T> &B, const spMtx<U> &M, spMtx<T> &C) {
    static_assert(std::is_same<T, int>::value, "the GPU operators take int matrices (spMtx<int>)");
    gk_csr a = A.csr(), b = B.csr();
    gk_csr mm{static_cast<int64_t>(M.m), static_cast<int64_t>(M.n), static_cast<int64_t>(M.nz), M.Rst.data(),
              M.Col.data(), nullptr};
    spMtx<T> R(M.m, M.n);
    gkb_detail::check(gk_mxmm_cmask(&a, &b, &mm, GK_PLUS_TIMES, R.Rst.data(), nullptr, nullptr, nullptr));
    R.resizeVals(static_cast<size_t>(R.Rst(M.m)));
    gkb_detail::check(gk_mxmm_cmask(&a, &b, &mm, GK_PLUS_TIMES, R.Rst.data(), R.Col.data(), R.Val.data(), nullptr));
    C = R;
}

// ----- operators of the alternate BC formulation (include/matrix_la.h:182-328) ---
namespace gkb_detail {
template <typename T>
gk_csr pattern_of(const spMtx<T> &X) {
    return gk_csr{static_cast<int64_t>(X.m), static_cast<int64_t>(X.n), static_cast<int64_t>(X.nz), X.Rst.data(),
                  X.Col.data(), nullptr};
}
}  // namespace gkb_detail

// C = A + B for non-intersecting patterns; the result lands in Cbuf and is
// swapped into C, as the reference does (matrix_la.h:287-328).
template <typename T>
void add_nointersect(const spMtx<T> &A, const spMtx<T> &B, spMtx<T> &C, spMtx<T> &Cbuf) {
    static_assert(std::is_same<T, int>::value, "add_nointersect takes int matrices (spMtx<int>)");
    if (A.m != B.m || A.n != B.n) throw std::runtime_error("gk_b200: add_nointersect: shapes differ");
    gk_csr a = A.csr(), b = B.csr();
    spMtx<T> R(A.m, A.n, A.nz + B.nz);
    gkb_detail::check(gk_add_nointersect(&a, &b, R.Rst.data(), R.Col.data(), R.Val.data(), nullptr));
    Cbuf = R;
    std::swap(C, Cbuf);
}

// C<M> = A .* B on dense operands, 0 outside M (matrix_la.h:189-208).
template <typename T, typename U>
void eWiseMult(const denseMtx<T> &A, const denseMtx<T> &B, const spMtx<U> &M, denseMtx<T> &C) {
    static_assert(std::is_same<T, double>::value, "the dense operators take denseMtx<double>");
    gk_csr mm = gkb_detail::pattern_of(M);
    gkb_detail::check(gk_dense_ewise_mult_masked(static_cast<int64_t>(C.m), static_cast<int64_t>(C.n), A.Val.data(),
                                                 B.Val.data(), &mm, C.Val.data(), nullptr));
}

// C += A .* B (matrix_la.h:182-187).
template <typename T>
void fuseEWiseMultAdd(const denseMtx<T> &A, const denseMtx<T> &B, denseMtx<T> &C) {
    static_assert(std::is_same<T, double>::value, "the dense operators take denseMtx<double>");
    gkb_detail::check(gk_dense_fuse_ewise_mult_add(static_cast<int64_t>(A.m * A.n), A.Val.data(), B.Val.data(),
                                                   C.Val.data(), nullptr));
}

// C<M> = A * B with sparse A, dense B and C (0 outside M); the product goes
// through Cbuf and is swapped into C, as the reference does (matrix_la.h:230-258).
template <typename T, typename U>
void mxmm_spd(const spMtx<T> &A, const denseMtx<T> &B, const spMtx<U> &M, denseMtx<T> &C, denseMtx<T> &Cbuf) {
    static_assert(std::is_same<T, double>::value, "mxmm_spd takes FP64 operands (spMtx<double>, denseMtx<double>)");
    gk_csr a = gkb_detail::pattern_of(A), mm = gkb_detail::pattern_of(M);
    if (Cbuf.m != C.m || Cbuf.n != C.n || Cbuf.Val.size() != C.m * C.n) Cbuf = denseMtx<T>(C.m, C.n);
    gkb_detail::check(gk_mxmm_spd(&a, A.Val.data(), B.Val.data(), static_cast<int64_t>(B.n), &mm, Cbuf.Val.data(),
                                  nullptr));
    std::swap(C.Val, Cbuf.Val);
}

// ----- CSR transforms ------------------------------------------------------------
template <typename T>
spMtx<T> transpose(const spMtx<T> &A) {
    spMtx<T> R(A.n, A.m, A.nz);
    gk_csr a = A.csr();
    gkb_detail::check(gk_transpose(&a, R.Rst.data(), R.Col.data(), R.Val.data(), nullptr));
    return R;
}

template <typename T>
spMtx<T> extract_lower_triangle(const spMtx<T> &A) {
    spMtx<T> R(A.m, A.n, A.nz);
    gk_csr a = A.csr(false);
    int64_t nz = 0;
    gkb_detail::check(gk_extract_lower(&a, R.Rst.data(), R.Col.data(), &nz, nullptr));
    // values follow their columns: the lower part of each row is its prefix
    for (size_t i = 0; i < A.m; ++i)
        for (int64_t j = 0; j < R.Rst(i + 1) - R.Rst(i); ++j) R.Val(R.Rst(i) + j) = A.Val(A.Rst(i) + j);
    R.resizeVals(static_cast<size_t>(nz));
    return R;
}

// Both run on the GPU (gk_build_symm_from_lower, gk_build_adjacency_matrix).
template <typename T>
spMtx<T> build_symm_from_lower(const spMtx<T> &Low) {
    static_assert(std::is_same<T, int>::value, "the GPU transforms take int matrices (spMtx<int>)");
    spMtx<T> R(Low.m, Low.n, 2 * Low.nz);
    gk_csr l = Low.csr();
    gkb_detail::check(gk_build_symm_from_lower(&l, R.Rst.data(), R.Col.data(), R.Val.data(), nullptr));
    return R;
}

template <typename T>
spMtx<int> build_adjacency_matrix(const spMtx<T> &G) {
    spMtx<int> R(G.m, G.n, G.nz);
    gk_csr g{static_cast<int64_t>(G.m), static_cast<int64_t>(G.n), static_cast<int64_t>(G.nz), G.Rst.data(),
             G.Col.data(), nullptr};
    gkb_detail::check(gk_build_adjacency_matrix(&g, R.Rst.data(), R.Col.data(), R.Val.data(), nullptr));
    return R;
}

// ----- algorithms --------------------------------------------------------------------
// Triangle count (src/main.cpp:69-90).  With one of this header's operators
// the count runs fused on the GPU (no C materialised); any other mxmOp is
// called as the reference does and C summed on the host.
inline int64_t triangle_counting_masked_sandia(const spMtx<int> &A, mxmOp<int> matrixMult, bool isParallel) {
    spMtx<int> L = extract_lower_triangle(A);
    const bool ours = matrixMult == static_cast<mxmOp<int>>(mxmm_msa<int, int>) ||
                      matrixMult == static_cast<mxmOp<int>>(mxmm_mca<int, int>) ||
                      matrixMult == static_cast<mxmOp<int>>(mxmm_naive<int>) ||
                      matrixMult == static_cast<mxmOp<int>>(mxmm_gpu<int>);
    if (ours) {
        gk_csr l = L.csr(false);
        uint64_t count = 0;
        gkb_detail::check(gk_tc_count(&l, &count, gkb_detail::row_sched(), nullptr));
        return static_cast<int64_t>(count);
    }
    spMtx<int> C;
    matrixMult(isParallel, L, L, L, C);
    int64_t sum = 0;
    for (size_t j = 0; j < C.nz; ++j) sum += C.Val(j);
    return sum;
}

// Triangles through each vertex (src/main.cpp:16-39): a new[]'d array of A.m
// ints the caller deletes, as in the reference.  With one of this header's
// operators the row sums of C<A> = A·A are fused on the GPU.
inline int *triangle_counting_vertex(const spMtx<int> &A, mxmOp<int> matrixMult, bool isParallel) {
    int *nums = new int[A.m];
    const bool ours = matrixMult == static_cast<mxmOp<int>>(mxmm_msa<int, int>) ||
                      matrixMult == static_cast<mxmOp<int>>(mxmm_mca<int, int>) ||
                      matrixMult == static_cast<mxmOp<int>>(mxmm_naive<int>) ||
                      matrixMult == static_cast<mxmOp<int>>(mxmm_gpu<int>);
    if (ours) {
        gk_csr a = A.csr(false);
        try {
            gkb_detail::check(gk_tc_vertex(&a, reinterpret_cast<int32_t *>(nums), gkb_detail::row_sched(), nullptr));
        } catch (...) {
            delete[] nums;
            throw;
        }
        return nums;
    }
    spMtx<int> SQ;
    matrixMult(isParallel, A, A, A, SQ);
    for (size_t i = 0; i < A.m; ++i) {
        int num_of_tr = 0;
        for (int64_t j = SQ.Rst(i); j < SQ.Rst(i + 1); ++j) num_of_tr += SQ.Val(j);
        nums[i] = num_of_tr >> 1;
    }
    return nums;
}

// Triangle count through C<A> = L·U, U = transpose(L) (src/main.cpp:42-66).
inline int64_t triangle_counting_masked_lu(const spMtx<int> &A, mxmOp<int> matrixMult, bool isParallel) {
    const bool ours = matrixMult == static_cast<mxmOp<int>>(mxmm_msa<int, int>) ||
                      matrixMult == static_cast<mxmOp<int>>(mxmm_mca<int, int>) ||
                      matrixMult == static_cast<mxmOp<int>>(mxmm_naive<int>) ||
                      matrixMult == static_cast<mxmOp<int>>(mxmm_gpu<int>);
    if (ours) {
        gk_csr a = A.csr(false);
        uint64_t count = 0;
        gkb_detail::check(gk_tc_count_lu(&a, &count, gkb_detail::row_sched(), nullptr));
        return static_cast<int64_t>(count);
    }
    spMtx<int> L = extract_lower_triangle(A);
    spMtx<int> U = transpose(L);
    spMtx<int> C;
    matrixMult(isParallel, L, U, A, C);
    int64_t sum = 0;
    for (size_t j = 0; j < C.nz; ++j) sum += C.Val(j);
    return sum >> 1;
}

// k-truss (src/main.cpp:94-141).  matrixMult is accepted for signature
// compatibility; the support products run on the GPU engine.
inline spMtx<int> k_truss(const spMtx<int> &A, int k, mxmOp<int>, bool, int *iterations = nullptr) {
    spMtx<int> C(A.m, A.n, A.nz);
    std::copy(A.Rst.data(), A.Rst.data() + A.m + 1, C.Rst.data());
    if (A.nz) std::copy(A.Col.data(), A.Col.data() + A.nz, C.Col.data());
    gk_csr_mut io{static_cast<int64_t>(A.m), static_cast<int64_t>(A.n), static_cast<int64_t>(A.nz), C.Rst.data(),
                  C.Col.data()};
    int iters = 0;
    gkb_detail::check(gk_ktruss(&io, k, &iters, gkb_detail::row_sched(), nullptr));
    C.resizeVals(static_cast<size_t>(io.nnz));
    for (size_t j = 0; j < C.nz; ++j) C.Val(j) = 1;
    if (iterations) *iterations = iters;
    return C;
}

// Batched BC with sources 0..min(n, batchSize)-1, as the reference
// (include/betweenness_centrality.h:406-447); computed in FP64.
inline std::vector<float> betweenness_centrality_batch(bool, const spMtx<int> &A, size_t batchSize) {
    if (A.m != A.n) throw "non-square matrix; BC is only for square matrices";
    const size_t b = std::min(A.n, batchSize);
    std::vector<int32_t> src(b);
    for (size_t j = 0; j < b; ++j) src[j] = static_cast<int32_t>(j);
    std::vector<double> d(A.m);
    gk_csr a = A.csr();
    gkb_detail::check(gk_bc_batch(&a, src.data(), static_cast<int>(b), d.data(), gkb_detail::bc_sched(), nullptr));
    return std::vector<float>(d.begin(), d.end());
}

inline std::vector<double> betweenness_centrality_batch(const spMtx<int> &A, const std::vector<int32_t> &sources) {
    std::vector<double> d(A.m);
    gk_csr a = A.csr();
    gkb_detail::check(gk_bc_batch(&a, sources.data(), static_cast<int>(sources.size()), d.data(),
                                  gkb_detail::bc_sched(), nullptr));
    return d;
}
