// Host-side internal types shared by the library's C++ translation units.
#pragma once
#include <cstdint>
#include <vector>

struct gk_host_graph {
    int64_t m = 0;
    int64_t nnz = 0;
    std::vector<int64_t> rp;
    std::vector<int32_t> col;
};
