// ref_host_shim.cpp -- TEST INFRASTRUCTURE. C entry points over the
// reference's OWN host code (compiled from the reference sources in place by
// oracle/Makefile into oracle/_ref/libref_host.so) so tests can pin the oracle
// and the product against the reference's actual stream generator and loader:
//   generate_init_stream        algorithms/streamgc/src/host/stream_gen.cpp:30-61
//   generate_bench_stream_edges algorithms/streamgc/src/host/stream_gen.cpp:65-177
//   load_graph_csr              algorithms/streamgc/src/host/graph_loader.cpp:29-169
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <utility>
#include <vector>

struct CSRGraph {            // graph_loader.cpp:18-24 (same layout)
    uint32_t  num_vertices;
    uint64_t  num_edges;
    uint32_t* row_ptr;
    uint32_t* col_idx;
    uint32_t* degree;
};
struct StreamConfig {        // stream_gen.cpp:16-20
    uint64_t stream_size;
    uint32_t insert_pct;
    uint64_t random_seed;
};
CSRGraph load_graph_csr(const char* filename);
void free_csr_graph(CSRGraph& graph);
std::vector<std::pair<uint32_t, uint32_t>> generate_init_stream(
    const uint32_t* row_ptr, const uint32_t* col_idx, const uint32_t* degree, uint32_t num_vertices);
std::vector<std::pair<uint32_t, uint32_t>> generate_bench_stream_edges(
    const uint32_t* row_ptr, const uint32_t* col_idx, const uint32_t* degree,
    uint32_t num_vertices, const StreamConfig& config, std::vector<uint8_t>& out_types);

extern "C" {
uint64_t ref_init_stream(uint32_t n, const uint32_t* rp, const uint32_t* col, const uint32_t* deg, uint32_t* out) {
    auto e = generate_init_stream(rp, col, deg, n);
    for (size_t i = 0; i < e.size(); i++) { out[2 * i] = e[i].first; out[2 * i + 1] = e[i].second; }
    return e.size();
}
void ref_bench_stream(uint32_t n, const uint32_t* rp, const uint32_t* col, const uint32_t* deg,
                      uint64_t size, uint32_t pct, uint64_t seed, uint32_t* out, uint8_t* types) {
    StreamConfig c{size, pct, seed};
    std::vector<uint8_t> t;
    auto e = generate_bench_stream_edges(rp, col, deg, n, c, t);
    for (size_t i = 0; i < e.size(); i++) { out[2 * i] = e[i].first; out[2 * i + 1] = e[i].second; types[i] = t[i]; }
}
// Loads an .mtx through the reference loader; returns n and nnz, then copy out.
static CSRGraph g_loaded;
int ref_load_mtx(const char* path, uint32_t* n, uint64_t* nnz) {
    g_loaded = load_graph_csr(path);
    *n = g_loaded.num_vertices;
    *nnz = g_loaded.num_edges;
    return 0;
}
void ref_loaded_copy(uint32_t* rp, uint32_t* col, uint32_t* deg) {
    std::memcpy(rp, g_loaded.row_ptr, (g_loaded.num_vertices + 1ull) * 4);
    std::memcpy(col, g_loaded.col_idx, g_loaded.num_edges * 4);
    std::memcpy(deg, g_loaded.degree, g_loaded.num_vertices * 4ull);
    free_csr_graph(g_loaded);
}
}
