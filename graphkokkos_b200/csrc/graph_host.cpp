// Host (C++/OpenMP) graph ingest: seeded RMAT / Erdos-Renyi generation and
// CSR construction (symmetrise, drop self-loops, deduplicate, sort rows).
// Produces exactly the CSR that the device builder in graph_dev.cu produces
// (same generator, same canonical form).  Used for CPU-side tests and for the
// reference arm's inputs; the GPU path builds its graphs on the device.
//
// Reference counterparts: the .rmat edge-list reader (matrix.h:488-533) and
// build_symm_from_lower(extract_lower_triangle(.)) (matrix.h:662-726,
// src/main.cpp:215), which together turn an edge list into a sorted
// symmetric CSR; the reference neither sorts nor deduplicates its inputs, so
// the canonical form here is what its algorithms assume (matrix.h:709).
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "gk_gen.h"
#include "gk_internal_host.h"

namespace {

template <class EdgeFn>
void build_symmetric_csr(int64_t m, uint64_t nedges, EdgeFn edge, gk_host_graph *g) {
    std::vector<uint64_t> ed(nedges);
    std::vector<int64_t> deg(m + 1, 0);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < static_cast<int64_t>(nedges); ++e) {
        uint32_t u, v;
        edge(static_cast<uint64_t>(e), &u, &v);
        ed[e] = (static_cast<uint64_t>(u) << 32) | v;
        if (u != v) {
#pragma omp atomic
            ++deg[u];
#pragma omp atomic
            ++deg[v];
        }
    }
    std::vector<int64_t> off(m + 1, 0);
    for (int64_t i = 0; i < m; ++i) off[i + 1] = off[i] + deg[i];
    std::vector<int64_t> cur(off.begin(), off.end() - 1);
    std::vector<int32_t> tmp(static_cast<size_t>(off[m]));
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < static_cast<int64_t>(nedges); ++e) {
        const uint32_t u = static_cast<uint32_t>(ed[e] >> 32), v = static_cast<uint32_t>(ed[e]);
        if (u == v) continue;
        int64_t p, q;
#pragma omp atomic capture
        p = cur[u]++;
#pragma omp atomic capture
        q = cur[v]++;
        tmp[p] = static_cast<int32_t>(v);
        tmp[q] = static_cast<int32_t>(u);
    }
    std::vector<uint64_t>().swap(ed);
    std::vector<int64_t> ucnt(m + 1, 0);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < m; ++i) {
        int32_t *b = tmp.data() + off[i], *e = tmp.data() + off[i + 1];
        std::sort(b, e);
        ucnt[i] = std::unique(b, e) - b;
    }
    g->m = m;
    g->rp.assign(m + 1, 0);
    for (int64_t i = 0; i < m; ++i) g->rp[i + 1] = g->rp[i] + ucnt[i];
    g->nnz = g->rp[m];
    g->col.resize(static_cast<size_t>(g->nnz));
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < m; ++i)
        std::memcpy(g->col.data() + g->rp[i], tmp.data() + off[i], sizeof(int32_t) * ucnt[i]);
}

}  // namespace

extern "C" {

int gk_gen_rmat_host(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                     gk_host_graph **out) {
    if (!out || scale < 1 || scale > 30 || edge_factor < 1) return 1;
    uint32_t ta, tab, tabc;
    gk_rmat_thresholds(a, b, c, &ta, &tab, &tabc);
    const uint64_t key = gk_seed_key(seed);
    const int64_t m = int64_t(1) << scale;
    const uint64_t ne = static_cast<uint64_t>(edge_factor) << scale;
    gk_host_graph *g = new (std::nothrow) gk_host_graph();
    if (!g) return 2;
    build_symmetric_csr(m, ne, [=](uint64_t e, uint32_t *u, uint32_t *v) {
        gk_rmat_edge(key, e, scale, ta, tab, tabc, u, v);
    }, g);
    *out = g;
    return 0;
}

int gk_gen_er_host(int64_t n, int64_t nedges, uint64_t seed, gk_host_graph **out) {
    if (!out || n < 1 || n >= (int64_t(1) << 31) || nedges < 0) return 1;
    const uint64_t key = gk_seed_key(seed);
    gk_host_graph *g = new (std::nothrow) gk_host_graph();
    if (!g) return 2;
    build_symmetric_csr(n, static_cast<uint64_t>(nedges), [=](uint64_t e, uint32_t *u, uint32_t *v) {
        gk_er_edge(key, e, static_cast<uint64_t>(n), u, v);
    }, g);
    *out = g;
    return 0;
}

int gk_host_graph_info(const gk_host_graph *g, int64_t *m, int64_t *nnz) {
    if (!g) return 1;
    if (m) *m = g->m;
    if (nnz) *nnz = g->nnz;
    return 0;
}

int gk_host_graph_copy(const gk_host_graph *g, int64_t *rowptr, int32_t *col) {
    if (!g) return 1;
    if (rowptr) std::memcpy(rowptr, g->rp.data(), sizeof(int64_t) * (g->m + 1));
    if (col && g->nnz) std::memcpy(col, g->col.data(), sizeof(int32_t) * g->nnz);
    return 0;
}

void gk_host_graph_free(gk_host_graph *g) { delete g; }

}  // extern "C"
