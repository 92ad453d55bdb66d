// Exercises the header-only C++ drop-in (include/gk/graphkokkos.hpp) the way
// the reference's own driver calls its operators (src/main.cpp:69-141,
// :249-251) and prints the results as one JSON line for tests/test_gpu_dropin.py.
#include <cstdio>
#include <cstdlib>
#include <numeric>
#include <vector>

#include "gk/graphkokkos.hpp"

static spMtx<int> rmat(int scale, uint64_t seed) {
    gk_host_graph *g = nullptr;
    gkb_detail::check(gk_gen_rmat_host(scale, 16, 0.57, 0.19, 0.19, seed, &g));
    int64_t m = 0, nnz = 0;
    gk_host_graph_info(g, &m, &nnz);
    spMtx<int> A(static_cast<size_t>(m), static_cast<size_t>(m), static_cast<size_t>(nnz));
    gk_host_graph_copy(g, A.Rst.data(), A.Col.data());
    gk_host_graph_free(g);
    for (size_t j = 0; j < A.nz; ++j) A.Val(j) = 1;
    return A;
}

// A user-supplied operator: triangle_counting_masked_sandia calls it and sums C on the host.
static void user_op(bool p, const spMtx<int> &A, const spMtx<int> &B, const spMtx<int> &M, spMtx<int> &C) {
    mxmm_gpu<int>(p, A, B, M, C);
}

int main(int argc, char **argv) {
    const int scale = argc > 1 ? std::atoi(argv[1]) : 12;
    const uint64_t seed = argc > 2 ? std::strtoull(argv[2], nullptr, 10) : 3;
    spMtx<int> A = rmat(scale, seed);
    const int64_t tc_msa = triangle_counting_masked_sandia(A, mxmm_msa<int, int>, true);
    const int64_t tc_mca = triangle_counting_masked_sandia(A, mxmm_mca<int, int>, true);
    const int64_t tc_user = triangle_counting_masked_sandia(A, user_op, true);
    spMtx<int> C;
    mxmm_msa<int, int>(true, A, A, A, C);
    long long csum = 0;
    for (size_t j = 0; j < C.nz; ++j) csum += C.Val(j);
    int iters = 0;
    spMtx<int> T = k_truss(A, 5, mxmm_msa<int, int>, true, &iters);
    std::vector<float> bcf = betweenness_centrality_batch(true, A, 32);
    double bcsum = 0;
    for (float x : bcf) bcsum += x;
    std::vector<int32_t> src(32);
    std::iota(src.begin(), src.end(), 0);
    std::vector<double> bcd = betweenness_centrality_batch(A, src);
    double bcdsum = 0;
    for (double x : bcd) bcdsum += x;
    spMtx<int> L = extract_lower_triangle(A);
    spMtx<int> S = build_symm_from_lower(L);
    const bool symm_ok = (S == A);
    spMtx<int> AT = transpose(A);
    const bool transpose_ok = (AT.nz == A.nz);
    int *per_vertex = triangle_counting_vertex(A, mxmm_msa<int, int>, true);
    long long vertex_sum = 0;
    for (size_t i = 0; i < A.m; ++i) vertex_sum += per_vertex[i];
    delete[] per_vertex;
    const int64_t tc_lu = triangle_counting_masked_lu(A, mxmm_msa<int, int>, true);
    spMtx<int> NC;  // two-hop pairs that are not edges: C<!A> = A·A
    mxmm_msa_cmask(true, A, A, A, NC);
    long long ncsum = 0;
    for (size_t j = 0; j < NC.nz; ++j) ncsum += NC.Val(j);
    // the alternate-BC operators: L + U merges back into A (disjoint patterns);
    // W = A·1 on A's pattern gives every entry of row i the degree of i
    spMtx<int> U = transpose(L), LU, LUbuf;
    add_nointersect(L, U, LU, LUbuf);
    const bool add_ok = (LU == A);
    spMtx<double> Ad(A.m, A.n, A.nz);
    for (size_t i = 0; i <= A.m; ++i) Ad.Rst(i) = A.Rst(i);
    for (size_t j = 0; j < A.nz; ++j) {
        Ad.Col(j) = A.Col(j);
        Ad.Val(j) = 1.0;
    }
    denseMtx<double> W(A.m, A.m), Wbuf, Sq(A.m, A.m);
    for (size_t i = 0; i < A.m * A.m; ++i) W.Val(i) = 1.0;
    mxmm_spd(Ad, W, A, W, Wbuf);
    bool spd_ok = true;
    for (size_t i = 0; i < A.m && spd_ok; ++i)
        for (int64_t q = A.Rst(i); q < A.Rst(i + 1); ++q)
            if (W.Val(i * A.m + A.Col(q)) != static_cast<double>(A.Rst(i + 1) - A.Rst(i))) spd_ok = false;
    eWiseMult(W, W, A, Sq);   // deg(i)^2 on A's pattern
    fuseEWiseMultAdd(W, W, Sq);  // + deg(i)^2 again
    double sqsum = 0;
    for (size_t i = 0; i < A.m * A.m; ++i) sqsum += Sq.Val(i);
    std::printf("{\"add_nointersect_ok\": %s, \"spd_ok\": %s, \"ewise_sum\": %.17g, ",
                add_ok ? "true" : "false", spd_ok ? "true" : "false", sqsum);
    std::printf("\"scale\": %d, \"seed\": %llu, \"nnz\": %zu, \"tc_msa\": %lld, \"tc_mca\": %lld, \"tc_user\": %lld, "
                "\"mxm_sum\": %lld, \"ktruss_nnz\": %zu, \"ktruss_iters\": %d, \"bc_float_sum\": %.9g, "
                "\"bc_f64_sum\": %.17g, \"symm_roundtrip\": %s, \"transpose_nnz\": %s, \"vertex_sum\": %lld, "
                "\"tc_lu\": %lld, \"cmask_nnz\": %zu, \"cmask_sum\": %lld}\n",
                scale, (unsigned long long)seed, A.nz, (long long)tc_msa, (long long)tc_mca, (long long)tc_user,
                csum, T.nz, iters, bcsum, bcdsum, symm_ok ? "true" : "false", transpose_ok ? "true" : "false",
                vertex_sum, (long long)tc_lu, NC.nz, ncsum);
    return 0;
}
