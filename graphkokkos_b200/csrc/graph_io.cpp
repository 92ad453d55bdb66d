// Sparse-matrix files: gk_read_matrix / gk_write_matrix.
//
// The formats are the reference's (spMtx(const char *filename, format),
// include/matrix.h:44-60, readers :259-533, writers :210-257), re-implemented
// here with their own parser (the NIST mmio library the reference vendors is
// not used).  A read gives the same CSR the reference builds, entry for entry:
//
//   mtx    MatrixMarket coordinate, pattern / integer / real, general or
//          symmetric (matrix.h:259-395).  Square only; diagonal entries are
//          dropped; a symmetric entry (i, j) adds (i, j) then (j, i); rows keep
//          the file's order; pattern values are 1; real values are truncated
//          toward zero (the reference reads them into int).
//   bin    4-byte matrix code, size_t m, n, nz, int32 Rst[m+1], Col[nz],
//          Val[nz] (matrix.h:418-456).  The writer here stores Col and Val;
//          the reference's write_crs_to_bin stores Rst three times (:222-224).
//   crs    text: m nz code, then Col[nz], Val[nz], Rst[m+1] (matrix.h:397-416).
//   graph  text: m nz, then one line of column indices per row (matrix.h:458-486);
//          values 1.  The reference reads the rest of the header line as row 0
//          and shifts every row down by one (:464-475); rows here start on the
//          line after the header.
//   rmat   text: m n nz, then nz pairs x y; each pair adds (x, y) and (y, x),
//          in file order, values 1 (matrix.h:488-533).
//
// Rows are not sorted, as in the reference; gk_host_graph_sort_rows sorts the
// columns of every row (values alongside), which the masked-product kernels
// require.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/gk_b200.h"
#include "gk_internal_host.h"

namespace gk {
int fail(int code, const std::string &msg);  // common.cu: records gk_last_error_string()
}

namespace {

int io_fail(const std::string &msg) { return gk::fail(GK_ERR_ARG, msg); }

// CSR from (row, col, val) triples appended per row in the given order.
void build_in_order(gk_host_graph *g, int64_t m, int64_t n, const std::vector<int64_t> &r,
                    const std::vector<int32_t> &c, const std::vector<int32_t> &v) {
    g->m = m;
    g->n = n;
    g->nnz = static_cast<int64_t>(r.size());
    g->rp.assign(m + 1, 0);
    for (int64_t x : r) ++g->rp[x + 1];
    for (int64_t i = 0; i < m; ++i) g->rp[i + 1] += g->rp[i];
    std::vector<int64_t> next(g->rp.begin(), g->rp.end() - 1);
    g->col.resize(g->nnz);
    g->val.resize(g->nnz);
    for (size_t e = 0; e < r.size(); ++e) {
        const int64_t p = next[r[e]]++;
        g->col[p] = c[e];
        g->val[p] = v[e];
    }
}

std::string lower(std::string s) {
    for (char &ch : s) ch = static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
    return s;
}

int read_mtx(const char *path, gk_host_graph *g) {
    std::ifstream in(path);
    if (!in) return io_fail(std::string("cannot open ") + path);
    std::string line;
    if (!std::getline(in, line)) return io_fail("empty MatrixMarket file");
    std::istringstream banner(line);
    std::string tag, object, layout, field, symmetry;
    banner >> tag >> object >> layout >> field >> symmetry;
    if (tag != "%%MatrixMarket" || lower(object) != "matrix")
        return io_fail("not a MatrixMarket matrix file (first line: " + line + ")");
    layout = lower(layout);
    field = lower(field);
    symmetry = lower(symmetry);
    if (layout != "coordinate") return io_fail("only coordinate MatrixMarket files are supported");
    if (field == "complex") return io_fail("complex MatrixMarket files are not supported");
    const bool pattern = field == "pattern";
    const bool symmetric = symmetry == "symmetric";
    if (symmetry != "general" && !symmetric)
        return io_fail("MatrixMarket symmetry '" + symmetry + "' is not supported");
    while (std::getline(in, line))
        if (!line.empty() && line[0] != '%') break;
    long long m = 0, n = 0, nz = 0;
    if (std::sscanf(line.c_str(), "%lld %lld %lld", &m, &n, &nz) != 3 || m < 0 || n < 0 || nz < 0)
        return io_fail("bad MatrixMarket size line: " + line);
    if (m != n) return io_fail("not a square matrix");
    std::vector<int64_t> r;
    std::vector<int32_t> c, v;
    r.reserve(symmetric ? 2 * nz : nz);
    for (long long e = 0; e < nz; ++e) {
        long long i, j;
        double x = 1.0;
        if (!(in >> i >> j)) return io_fail("MatrixMarket file ends before its " + std::to_string(nz) + " entries");
        if (!pattern && !(in >> x)) return io_fail("MatrixMarket entry without a value");
        if (i < 1 || i > m || j < 1 || j > n) return io_fail("MatrixMarket entry out of range");
        --i;
        --j;
        if (i == j) continue;  // the reference drops loops (matrix.h:323-327)
        const int32_t val = pattern ? 1 : static_cast<int32_t>(std::trunc(x));
        r.push_back(i);
        c.push_back(static_cast<int32_t>(j));
        v.push_back(val);
        if (symmetric) {
            r.push_back(j);
            c.push_back(static_cast<int32_t>(i));
            v.push_back(val);
        }
    }
    build_in_order(g, m, n, r, c, v);
    g->has_val = !pattern;
    return GK_OK;
}

int read_bin(const char *path, gk_host_graph *g) {
    FILE *fp = std::fopen(path, "rb");
    if (!fp) return io_fail(std::string("cannot open ") + path);
    char code[4];
    uint64_t hdr[3];
    int st = GK_OK;
    if (std::fread(code, 1, 4, fp) != 4 || std::fread(hdr, sizeof(uint64_t), 3, fp) != 3) {
        st = io_fail("binary CSR file too short for its header");
    } else {
        const int64_t m = static_cast<int64_t>(hdr[0]), n = static_cast<int64_t>(hdr[1]),
                      nz = static_cast<int64_t>(hdr[2]);
        std::vector<int32_t> rst(m + 1);
        g->m = m;
        g->n = n;
        g->nnz = nz;
        g->col.resize(nz);
        g->val.resize(nz);
        if (std::fread(rst.data(), sizeof(int32_t), m + 1, fp) != static_cast<size_t>(m + 1) ||
            std::fread(g->col.data(), sizeof(int32_t), nz, fp) != static_cast<size_t>(nz) ||
            std::fread(g->val.data(), sizeof(int32_t), nz, fp) != static_cast<size_t>(nz)) {
            st = io_fail("binary CSR file shorter than its header says");
        } else {
            g->rp.assign(rst.begin(), rst.end());
            g->has_val = true;
            if (g->rp[0] != 0 || g->rp[m] != nz) st = io_fail("binary CSR row pointers do not match nz");
        }
    }
    std::fclose(fp);
    return st;
}

int read_crs(const char *path, gk_host_graph *g) {
    std::ifstream in(path);
    if (!in) return io_fail(std::string("cannot open ") + path);
    long long m, nz;
    std::string code;
    if (!(in >> m >> nz >> code) || m < 0 || nz < 0) return io_fail("bad CRS header");
    g->m = g->n = m;
    g->nnz = nz;
    g->col.resize(nz);
    g->val.resize(nz);
    g->rp.resize(m + 1);
    for (long long j = 0; j < nz; ++j)
        if (!(in >> g->col[j])) return io_fail("CRS file ends inside Col");
    for (long long j = 0; j < nz; ++j)
        if (!(in >> g->val[j])) return io_fail("CRS file ends inside Val");
    for (long long i = 0; i <= m; ++i)
        if (!(in >> g->rp[i])) return io_fail("CRS file ends inside Rst");
    g->has_val = true;
    return GK_OK;
}

int read_graph(const char *path, gk_host_graph *g) {
    std::ifstream in(path);
    if (!in) return io_fail(std::string("cannot open ") + path);
    std::string line;
    long long m, nz;
    if (!std::getline(in, line) || std::sscanf(line.c_str(), "%lld %lld", &m, &nz) != 2 || m < 0 || nz < 0)
        return io_fail("bad graph header");
    g->m = g->n = m;
    g->rp.assign(m + 1, 0);
    g->col.clear();
    g->col.reserve(nz);
    for (long long i = 0; i < m; ++i) {
        if (!std::getline(in, line)) line.clear();  // missing trailing rows are empty
        std::istringstream row(line);
        long long c;
        while (row >> c) {
            if (c < 0 || c >= m) return io_fail("graph column out of range");
            g->col.push_back(static_cast<int32_t>(c));
        }
        g->rp[i + 1] = static_cast<int64_t>(g->col.size());
    }
    g->nnz = static_cast<int64_t>(g->col.size());
    g->val.assign(g->nnz, 1);
    g->has_val = false;
    return GK_OK;
}

int read_rmat(const char *path, gk_host_graph *g) {
    std::ifstream in(path);
    if (!in) return io_fail(std::string("cannot open ") + path);
    long long m, n, nz;
    if (!(in >> m >> n >> nz) || m < 0 || nz < 0) return io_fail("bad rmat header");
    std::vector<int64_t> r;
    std::vector<int32_t> c;
    r.reserve(2 * nz);
    c.reserve(2 * nz);
    for (long long e = 0; e < nz; ++e) {
        long long x, y;
        if (!(in >> x >> y)) return io_fail("rmat file ends before its " + std::to_string(nz) + " pairs");
        if (x < 0 || x >= m || y < 0 || y >= m) return io_fail("rmat vertex out of range");
        r.push_back(x);
        c.push_back(static_cast<int32_t>(y));
        r.push_back(y);
        c.push_back(static_cast<int32_t>(x));
    }
    build_in_order(g, m, n, r, c, std::vector<int32_t>(r.size(), 1));
    g->has_val = false;
    return GK_OK;
}

int format_of(const char *path, int format) {
    if (format != GK_FILE_AUTO) return format;
    const char *dot = std::strrchr(path, '.');
    const std::string ext = dot ? lower(dot + 1) : "";
    if (ext == "mtx") return GK_FILE_MTX;
    if (ext == "bin") return GK_FILE_BIN;
    if (ext == "crs") return GK_FILE_CRS;
    if (ext == "graph") return GK_FILE_GRAPH;
    if (ext == "rmat") return GK_FILE_RMAT;
    return -1;
}

}  // namespace

extern "C" {

int gk_read_matrix(const char *path, int format, gk_host_graph **out) {
    if (!path || !out) return io_fail("gk_read_matrix: null argument");
    const int f = format_of(path, format);
    gk_host_graph *g = new (std::nothrow) gk_host_graph();
    if (!g) return io_fail("out of host memory");
    int st;
    switch (f) {
        case GK_FILE_MTX: st = read_mtx(path, g); break;
        case GK_FILE_BIN: st = read_bin(path, g); break;
        case GK_FILE_CRS: st = read_crs(path, g); break;
        case GK_FILE_GRAPH: st = read_graph(path, g); break;
        case GK_FILE_RMAT: st = read_rmat(path, g); break;
        default: st = io_fail(std::string("unknown matrix file format for ") + path);
    }
    if (st != GK_OK) {
        delete g;
        return st;
    }
    *out = g;
    return GK_OK;
}

int gk_write_matrix(const char *path, int format, const gk_csr *A) {
    if (!path || !A || A->m < 0 || A->n < 0 || A->nnz < 0 || !A->rowptr || (A->nnz > 0 && !A->col))
        return io_fail("gk_write_matrix: bad arguments");
    const int f = format_of(path, format);
    const int64_t m = A->m, n = A->n, nz = A->nnz;
    if (f == GK_FILE_BIN) {
        if (nz >= (int64_t(1) << 31)) return io_fail("the binary format stores int32 row pointers: nnz must be < 2^31");
        FILE *fp = std::fopen(path, "wb");
        if (!fp) return io_fail(std::string("cannot create ") + path);
        const char code[4] = {'M', 'C', A->val ? 'I' : 'P', 'G'};  // matrix, coordinate, integer/pattern, general
        const uint64_t hdr[3] = {static_cast<uint64_t>(m), static_cast<uint64_t>(n), static_cast<uint64_t>(nz)};
        std::vector<int32_t> rst(m + 1), val(nz, 1);
        for (int64_t i = 0; i <= m; ++i) rst[i] = static_cast<int32_t>(A->rowptr[i]);
        if (A->val) std::memcpy(val.data(), A->val, sizeof(int32_t) * nz);
        bool ok = std::fwrite(code, 1, 4, fp) == 4 && std::fwrite(hdr, sizeof(uint64_t), 3, fp) == 3 &&
                  std::fwrite(rst.data(), sizeof(int32_t), m + 1, fp) == static_cast<size_t>(m + 1) &&
                  std::fwrite(A->col, sizeof(int32_t), nz, fp) == static_cast<size_t>(nz) &&
                  std::fwrite(val.data(), sizeof(int32_t), nz, fp) == static_cast<size_t>(nz);
        ok = (std::fclose(fp) == 0) && ok;
        return ok ? GK_OK : io_fail(std::string("write failed: ") + path);
    }
    if (f == GK_FILE_MTX) {
        FILE *fp = std::fopen(path, "w");
        if (!fp) return io_fail(std::string("cannot create ") + path);
        std::fprintf(fp, "%%%%MatrixMarket matrix coordinate %s general\n", A->val ? "integer" : "pattern");
        std::fprintf(fp, "%lld %lld %lld\n", static_cast<long long>(m), static_cast<long long>(n),
                     static_cast<long long>(nz));
        for (int64_t i = 0; i < m; ++i)
            for (int64_t p = A->rowptr[i]; p < A->rowptr[i + 1]; ++p) {
                if (A->val)
                    std::fprintf(fp, "%lld %d %d\n", static_cast<long long>(i + 1), A->col[p] + 1, A->val[p]);
                else
                    std::fprintf(fp, "%lld %d\n", static_cast<long long>(i + 1), A->col[p] + 1);
            }
        return std::fclose(fp) == 0 ? GK_OK : io_fail(std::string("write failed: ") + path);
    }
    return io_fail("gk_write_matrix writes the mtx and bin formats");
}

int gk_host_graph_values(const gk_host_graph *g, int32_t *val, int64_t *n) {
    if (!g) return -1;
    if (n) *n = g->n ? g->n : g->m;
    if (!g->has_val) return 0;
    if (val && g->nnz) std::memcpy(val, g->val.data(), sizeof(int32_t) * g->nnz);
    return 1;
}

int gk_host_graph_sort_rows(gk_host_graph *g) {
    if (!g) return GK_ERR_ARG;
    std::vector<int64_t> idx;
    std::vector<int32_t> c, v;
    for (int64_t i = 0; i < g->m; ++i) {
        const int64_t b = g->rp[i], e = g->rp[i + 1];
        if (std::is_sorted(g->col.begin() + b, g->col.begin() + e)) continue;
        idx.resize(e - b);
        std::iota(idx.begin(), idx.end(), b);
        std::stable_sort(idx.begin(), idx.end(), [&](int64_t x, int64_t y) { return g->col[x] < g->col[y]; });
        c.resize(e - b);
        v.resize(e - b);
        for (int64_t k = 0; k < e - b; ++k) {
            c[k] = g->col[idx[k]];
            v[k] = g->val.empty() ? 1 : g->val[idx[k]];
        }
        std::copy(c.begin(), c.end(), g->col.begin() + b);
        if (!g->val.empty()) std::copy(v.begin(), v.end(), g->val.begin() + b);
    }
    return GK_OK;
}


}  // extern "C"
