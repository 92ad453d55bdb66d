// Host code under AddressSanitizer and UndefinedBehaviorSanitizer: the
// library's host graph builder (graph_host.cpp) and matrix-file reader and
// writer (graph_io.cpp), and the CPU restatement of the oracle
// (oracle/gk_oracle.cpp), exercised on seeded graphs.  Built and run by
// tests/test_sanitize_cpu.py; any sanitizer report fails the run.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "gk_b200.h"

namespace gk {
// graph_io.cpp reports errors through the library's error recorder
int fail(int code, const std::string &) { return code; }
}  // namespace gk

extern "C" {
int orc_tc_lower(int64_t m, const int64_t *rp, const int32_t *col, uint64_t *out);
int orc_tc_merge(int64_t m, const int64_t *rp, const int32_t *col, uint64_t *out);
int orc_extract_lower(int64_t m, const int64_t *rp, const int32_t *col, int64_t *orp, int32_t *ocol,
                      int64_t *out_nnz);
int orc_ktruss(int64_t m, const int64_t *rp, const int32_t *col, int k, int64_t *out_rp, int32_t *out_col,
               int64_t *out_nnz, int *out_iters, int64_t *nnz_per_iter, int max_record);
int orc_mxmm_cmask(int64_t am, int64_t an, const int64_t *arp, const int32_t *acol, const int32_t *aval,
                   int64_t bm, int64_t bn, const int64_t *brp, const int32_t *bcol, const int32_t *bval,
                   int64_t mm, int64_t mn, const int64_t *mrp, const int32_t *mcol,
                   int64_t *c_rp, int32_t *c_col, int32_t *c_val);
int orc_bc_f64(int64_t m, const int64_t *rp, const int32_t *col, const int32_t *val, const int32_t *src, int64_t b,
               double *bc_out);
int orc_mxmm_spd(int64_t m, const int64_t *arp, const int32_t *acol, const double *aval, int64_t n,
                 const double *B, const int64_t *mrp, const int32_t *mcol, double *C);
}

static int fails = 0;
#define CHECK(c)                                                     \
    do {                                                             \
        if (!(c)) {                                                  \
            std::fprintf(stderr, "check failed: %s (line %d)\n", #c, __LINE__); \
            ++fails;                                                 \
        }                                                            \
    } while (0)

int main(int argc, char **argv) {
    const std::string dir = argc > 1 ? argv[1] : ".";
    for (int scale = 6; scale <= 10; scale += 2) {
        gk_host_graph *g = nullptr;
        CHECK(gk_gen_rmat_host(scale, 8, 0.57, 0.19, 0.19, 11 + scale, &g) == GK_OK);
        int64_t m = 0, nnz = 0;
        gk_host_graph_info(g, &m, &nnz);
        std::vector<int64_t> rp(m + 1);
        std::vector<int32_t> col(nnz);
        gk_host_graph_copy(g, rp.data(), col.data());
        gk_host_graph_free(g);
        // file round trips (values: none)
        gk_csr A{m, m, nnz, rp.data(), col.data(), nullptr};
        for (const char *ext : {"mtx", "bin"}) {
            const std::string path = dir + "/g" + std::to_string(scale) + "." + ext;
            CHECK(gk_write_matrix(path.c_str(), 0, &A) == GK_OK);
            gk_host_graph *h = nullptr;
            CHECK(gk_read_matrix(path.c_str(), 0, &h) == GK_OK);
            CHECK(gk_host_graph_sort_rows(h) == GK_OK);
            int64_t hm = 0, hn = 0;
            gk_host_graph_info(h, &hm, &hn);
            CHECK(hm == m && hn == nnz);
            gk_host_graph_free(h);
        }
        gk_host_graph *bad = nullptr;
        CHECK(gk_read_matrix((dir + "/missing.mtx").c_str(), 0, &bad) != GK_OK);
        // oracle: two triangle counts, k-truss, the complement-masked product, BC, mxmm_spd
        std::vector<int64_t> lrp(m + 1);
        std::vector<int32_t> lcol(nnz);
        int64_t lnnz = 0;
        orc_extract_lower(m, rp.data(), col.data(), lrp.data(), lcol.data(), &lnnz);
        CHECK(2 * lnnz == nnz);
        uint64_t t1 = 0, t2 = 0;
        orc_tc_lower(m, lrp.data(), lcol.data(), &t1);
        orc_tc_merge(m, lrp.data(), lcol.data(), &t2);
        CHECK(t1 == t2);
        std::vector<int64_t> orp(m + 1), rec(64);
        std::vector<int32_t> ocol(nnz > 0 ? nnz : 1);
        int64_t onnz = 0;
        int iters = 0;
        CHECK(orc_ktruss(m, rp.data(), col.data(), 4, orp.data(), ocol.data(), &onnz, &iters, rec.data(), 64) == 0);
        std::vector<int64_t> crp(m + 1);
        CHECK(orc_mxmm_cmask(m, m, rp.data(), col.data(), nullptr, m, m, rp.data(), col.data(), nullptr, m, m,
                             rp.data(), col.data(), crp.data(), nullptr, nullptr) == 0);
        std::vector<int32_t> ccol(crp[m] > 0 ? crp[m] : 1), cval(ccol.size());
        CHECK(orc_mxmm_cmask(m, m, rp.data(), col.data(), nullptr, m, m, rp.data(), col.data(), nullptr, m, m,
                             rp.data(), col.data(), crp.data(), ccol.data(), cval.data()) == 0);
        std::vector<int32_t> src = {0, 1, 2};
        std::vector<double> bc(m);
        CHECK(orc_bc_f64(m, rp.data(), col.data(), nullptr, src.data(), 3, bc.data()) == 0);
        std::vector<double> B(static_cast<size_t>(m) * 4, 1.0), C(static_cast<size_t>(m) * 4);
        std::vector<int64_t> mrp(m + 1);
        std::vector<int32_t> mcol;
        for (int64_t i = 0; i < m; ++i) {
            mrp[i] = static_cast<int64_t>(mcol.size());
            mcol.push_back(static_cast<int32_t>(i % 4));
        }
        mrp[m] = static_cast<int64_t>(mcol.size());
        CHECK(orc_mxmm_spd(m, rp.data(), col.data(), nullptr, 4, B.data(), mrp.data(), mcol.data(), C.data()) == 0);
        for (int64_t i = 0; i < m; ++i) CHECK(C[i * 4 + i % 4] == static_cast<double>(rp[i + 1] - rp[i]));
    }
    // the text formats, and malformed files that must be refused
    struct TextCase {
        const char *name, *text;
        bool ok;
    };
    const TextCase cases[] = {
        {"a.graph", "4 6\n1 2\n0 3\n0\n1\n", true},
        {"a.rmat", "4 4 3\n0 1\n2 1\n3 0\n", true},
        {"a.crs", "3 3 MCI\n1 2 0\n5 6 7\n0 1 2 3\n", true},
        {"b.mtx", "%%MatrixMarket matrix coordinate integer general\n3 3 2\n1 2 5\n3 1 -4\n", true},
        {"short.mtx", "%%MatrixMarket matrix coordinate pattern general\n3 3 5\n1 2\n", false},
        {"rect.mtx", "%%MatrixMarket matrix coordinate pattern general\n3 4 1\n1 2\n", false},
        {"junk.mtx", "hello\n", false},
        {"range.mtx", "%%MatrixMarket matrix coordinate pattern general\n3 3 1\n1 9\n", false},
    };
    for (const TextCase &c : cases) {
        const std::string path = dir + "/" + c.name;
        FILE *f = std::fopen(path.c_str(), "w");
        std::fputs(c.text, f);
        std::fclose(f);
        gk_host_graph *h = nullptr;
        const int st = gk_read_matrix(path.c_str(), 0, &h);
        CHECK((st == GK_OK) == c.ok);
        if (h) gk_host_graph_free(h);
    }
    std::printf(fails ? "FAILED %d\n" : "OK\n", fails);
    return fails ? 1 : 0;
}
