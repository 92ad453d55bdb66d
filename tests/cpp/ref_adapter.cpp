// The reference-side adapter of the integration guide, as written there: an
// mxmOp-compatible mxmm_b200 over the reference's own spMtx (its
// include/matrix.h, compiled against the Kokkos-API shim of oracle/) that
// calls gk_mxmm_masked with the learned scheduler, plus the fused entry
// points called with spMtx storage.  Built against libgk_b200.so by
// __graft_entry__.build() (into oracle/_ref/, since it includes the
// reference's headers) and by tests/test_ref_adapter_cpu.py.
//   ref_adapter                      prints "compiled" (no GPU needed)
//   ref_adapter MODEL.bin BC.bin     loads the learned models from their files
//                                    (gk_sched_load_model_file /
//                                    gk_bc_load_model_file) and checks K4 and
//                                    K64 on the GPU, printing one JSON line
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
    if (gk_mxmm_masked(&a, &b, &m, C.Val.data(), GK_PLUS_TIMES, GK_SCHED_LEARNED, GK_ACCUM_AUTO, nullptr))
        throw std::runtime_error(gk_last_error_string());
}

using mxmOpInt = void (*)(bool, const spMtx<int> &, const spMtx<int> &, const spMtx<int> &, spMtx<int> &);

static spMtx<int> complete_graph(int n) {
    spMtx<int> A(n, n, (size_t)n * (n - 1));
    int k = 0;
    for (int i = 0; i < n; ++i) {
        A.Rst(i) = k;
        for (int j = 0; j < n; ++j)
            if (j != i) {
                A.Col(k) = j;
                A.Val(k++) = 1;
            }
    }
    A.Rst(n) = k;
    return A;
}

int main(int argc, char **argv) {
    mxmOpInt op = mxmm_b200<int, int>;  // what launch_test would select for "b200"
    if (argc < 3) {
        std::printf("compiled\n");
        return 0;
    }
    // the learned scheduler's models, loaded from their files as a C++ host would
    if (gk_sched_load_model_file(argv[1]) || gk_bc_load_model_file(argv[2])) {
        std::printf("{\"error\": \"%s\"}\n", gk_last_error_string());
        return 2;
    }
    bool ok = true;
    std::printf("{");
    for (int n : {4, 64}) {
        spMtx<int> A = complete_graph(n);
        spMtx<int> C;
        op(true, A, A, A, C);  // C<A> = A*A: n-2 common neighbours per edge
        long long s = 0;
        for (size_t j = 0; j < C.nz; ++j) s += C.Val(j);
        // fused count over all of A: every triangle counted 6 times
        std::vector<int64_t> rl;
        gk_csr l = as_gk(A, rl, false);
        uint64_t sum6 = 0;
        if (gk_tc_count(&l, &sum6, GK_SCHED_LEARNED, nullptr)) throw std::runtime_error(gk_last_error_string());
        // BC with the learned level shapes: 0 on a complete graph
        std::vector<int32_t> src(n);
        std::iota(src.begin(), src.end(), 0);
        std::vector<double> bc(n, -1.0);
        gk_csr a = as_gk(A, rl, false);
        if (gk_bc_batch(&a, src.data(), n, bc.data(), GK_SCHED_LEARNED, nullptr))
            throw std::runtime_error(gk_last_error_string());
        double bcs = 0.0;
        for (double x : bc) bcs += x;
        const long long want = (long long)n * (n - 1) * (n - 2);
        ok = ok && s == want && (long long)sum6 == want && bcs == 0.0;
        std::printf("%s\"K%d\": {\"mxm_sum\": %lld, \"tc_on_A\": %llu, \"bc_sum\": %g}", n == 4 ? "" : ", ", n, s,
                    (unsigned long long)sum6, bcs);
    }
    std::printf("}\n");
    return ok ? 0 : 1;
}
