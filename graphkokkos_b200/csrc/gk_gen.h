// Deterministic synthetic graph generators shared by the host (C++/OpenMP)
// and device (CUDA) builders, so both produce bit-identical edge lists.
//
// The reference ships no generator: its benchmark graphs were external
// .rmat/.mtx files (matrix.h:488-533) and its test generator is unseeded
// (matrix_utils.h:7-34).  These generators define the synthetic inputs:
//
//  * Counter-based hashing: every random draw is splitmix64's output
//    function (Steele, Lea & Flood, "Fast splittable pseudorandom number
//    generators", OOPSLA 2014) applied to  key ^ counter,  where
//    key = mix(seed) and the counter names the edge and the recursion level.
//    No state is carried between draws, so any edge can be generated by any
//    thread in any order.
//  * RMAT (Chakrabarti, Zhan & Faloutsos, SDM 2004; Graph500 parameters):
//    edge e picks one quadrant per level, most significant bit first, with
//    integer thresholds ta <= tab <= tabc on the high 32 bits of the draw
//    (a: (0,0), b: (0,1), c: (1,0), d: (1,1)).  No noise, no permutation.
//  * Erdos-Renyi G(n, M): edge e is the pair (hi32 * n >> 32, lo32 * n >> 32)
//    of one draw.
// Post-processing (both builders): symmetrise, drop self-loops, remove
// duplicates, sort each row ascending.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define GK_HD __host__ __device__ __forceinline__
#else
#define GK_HD static inline
#endif

GK_HD uint64_t gk_mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

GK_HD uint64_t gk_seed_key(uint64_t seed) { return gk_mix64(seed ^ 0x6A09E667F3BCC909ull); }

// RMAT edge e of a graph with 2^scale vertices.
GK_HD void gk_rmat_edge(uint64_t key, uint64_t e, int scale, uint32_t ta, uint32_t tab, uint32_t tabc,
                        uint32_t *u, uint32_t *v) {
    uint32_t uu = 0, vv = 0;
    for (int l = 0; l < scale; ++l) {
        const uint32_t r = (uint32_t)(gk_mix64(key ^ ((e << 6) | (uint64_t)l)) >> 32);
        const uint32_t bu = r >= tab;                        // quadrants c, d
        const uint32_t bv = (r >= ta && r < tab) | (r >= tabc);  // quadrants b, d
        uu = (uu << 1) | bu;
        vv = (vv << 1) | bv;
    }
    *u = uu;
    *v = vv;
}

// Erdos-Renyi pair e on n vertices (n < 2^32).
GK_HD void gk_er_edge(uint64_t key, uint64_t e, uint64_t n, uint32_t *u, uint32_t *v) {
    const uint64_t h = gk_mix64(key ^ (e << 1));
    *u = (uint32_t)(((h >> 32) * n) >> 32);
    *v = (uint32_t)(((h & 0xFFFFFFFFull) * n) >> 32);
}

// Integer RMAT thresholds from probabilities (computed once on the host).
static inline void gk_rmat_thresholds(double a, double b, double c, uint32_t *ta, uint32_t *tab,
                                      uint32_t *tabc) {
    const double s = 4294967296.0;
    double x = a * s, y = (a + b) * s, z = (a + b + c) * s;
    *ta = x >= s ? 0xFFFFFFFFu : (uint32_t)x;
    *tab = y >= s ? 0xFFFFFFFFu : (uint32_t)y;
    *tabc = z >= s ? 0xFFFFFFFFu : (uint32_t)z;
}
