// Host-side internal types shared by the library's C++ translation units.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

struct gk_host_graph {
    int64_t m = 0;
    int64_t n = 0;  // columns (0: square, n = m)
    int64_t nnz = 0;
    std::vector<int64_t> rp;
    std::vector<int32_t> col;
    std::vector<int32_t> val;  // read from a file that carries values (has_val)
    bool has_val = false;
};

namespace gk {
// Reads a scheduler model file: the 8 bytes "GKMLP001", a little-endian
// uint32 count, then count little-endian float32 weights (written by
// graphkokkos_b200/sched.py).  Returns an empty string on success, else what
// was wrong with the file.
std::string read_model_file(const char *path, std::vector<float> &out);
}  // namespace gk
