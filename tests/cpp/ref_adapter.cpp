// The reference-side adapter of the integration guide, with the plain
// scheduler (which needs no model): an mxmOp-compatible mxmm_b200 over the
// reference's own spMtx (its
// include/matrix.h, compiled here against the Kokkos-API shim of oracle/),
// plus the fused entry points called with spMtx storage.  Compiled and linked
// against libgk_b200.so by tests/test_ref_adapter_cpu.py; run with an
// argument on a GPU host it counts the triangles of K4 both ways.
#include "matrix.h"
#include "gk_b200.h"

#include <cstdio>
#include <numeric>
#include <stdexcept>
#include <vector>

static gk_csr as_gk(const spMtx<int> &X, std::vector<int64_t> &rp, bool values) {
    rp.resize(X.m + 1);
    for (size_t i = 0; i <= X.m; ++i) rp[i] = X.Rst(i);  // int32 -> int64 row pointers
    return gk_csr{(int64_t)X.m, (int64_t)X.n, (int64_t)X.nz, rp.data(), X.Col.data(),
                  values ? X.Val.data() : nullptr};
}

// Drop-in for mxmm_msa / mxmm_mca (matrix_la.h:478-694): C gets M's pattern
// (matrix_la.h:564-568), values computed on the GPU.
template <typename T, typename U>
void mxmm_b200(bool, const spMtx<T> &A, const spMtx<T> &B, const spMtx<U> &M, spMtx<T> &C) {
    C.resizeRows(M.m);
    C.resizeVals(M.nz);
    C.n = M.n;
    Kokkos::deep_copy(C.Col, M.Col);
    Kokkos::deep_copy(C.Rst, M.Rst);
    std::vector<int64_t> ra, rb, rm;
    gk_csr a = as_gk(A, ra, true), b = as_gk(B, rb, true), m = as_gk(M, rm, false);
    if (gk_mxmm_masked(&a, &b, &m, C.Val.data(), GK_PLUS_TIMES, GK_SCHED_PLAIN, GK_ACCUM_AUTO, nullptr))
        throw std::runtime_error(gk_last_error_string());
}

using mxmOpInt = void (*)(bool, const spMtx<int> &, const spMtx<int> &, const spMtx<int> &, spMtx<int> &);

int main(int argc, char **argv) {
    mxmOpInt op = mxmm_b200<int, int>;  // what launch_test would select for "b200"
    if (argc < 2) {
        std::printf("compiled\n");
        return 0;
    }
    // K4: every vertex adjacent to the others
    spMtx<int> A(4, 4, 12);
    int k = 0;
    for (int i = 0; i < 4; ++i) {
        A.Rst(i) = k;
        for (int j = 0; j < 4; ++j)
            if (j != i) {
                A.Col(k) = j;
                A.Val(k++) = 1;
            }
    }
    A.Rst(4) = k;
    spMtx<int> C;
    op(true, A, A, A, C);  // C<A> = A*A: 2 common neighbours per edge
    long long s = 0;
    for (size_t j = 0; j < C.nz; ++j) s += C.Val(j);
    std::vector<int64_t> rl;
    gk_csr l = as_gk(A, rl, false);
    uint64_t sum6 = 0;
    if (gk_tc_count(&l, &sum6, GK_SCHED_PLAIN, nullptr)) throw std::runtime_error(gk_last_error_string());
    std::printf("{\"mxm_sum\": %lld, \"tc_on_A\": %llu}\n", s, (unsigned long long)sum6);
    return (s == 24 && sum6 == 24) ? 0 : 1;
}
