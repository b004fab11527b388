/*
 * sgc_host.h -- host-side helpers of libstreamgc_b200.so (C ABI): graph input,
 * update-stream generation, output files. CSR arrays use 64-bit row offsets.
 */
#ifndef SGC_HOST_H
#define SGC_HOST_H

#include <stdint.h>
#include "../../include/streamgc_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A host CSR owned by the library (free with sgc_csr_free). */
typedef struct sgc_csr {
    uint32_t  n;
    uint64_t  nnz;       /* directed entries = 2 x undirected edges */
    uint64_t* row_ptr;   /* n + 1 */
    uint32_t* col_idx;   /* nnz, each row ascending */
    uint32_t* degree;    /* n */
} sgc_csr;

/* Matrix-Market loader with load_graph_csr semantics
 * (algorithms/streamgc/src/host/graph_loader.cpp:29-169): 1-based ids, self
 * loops dropped, (min,max) normalised, sorted and de-duplicated, symmetric
 * CSR with ascending rows. Returns 0 or a negative code. */
int sgc_load_mtx(const char* path, sgc_csr* out);
/* Same construction from an in-memory 0-based edge list (pairs[2*i], pairs[2*i+1]). */
int sgc_csr_from_edges(uint32_t n, const uint32_t* pairs, uint64_t m, sgc_csr* out);
/* The symmetric closure of rows that may miss mirror entries: an edge is kept
 * when either direction is present (self loops and ids >= n dropped); rows
 * ascending, degrees from the result. */
int sgc_csr_symmetrize(uint32_t n, const uint64_t* row_ptr, const uint32_t* col_idx, sgc_csr* out);
void sgc_csr_free(sgc_csr* g);
/* Writes an undirected .mtx (pattern, one line per edge u > v, 1-based). */
int sgc_write_mtx(const char* path, const sgc_csr* g);

/* Init stream of generate_init_stream (stream_gen.cpp:30-61): every u<v edge,
 * sorted by (min degree desc, max degree desc) with std::sort. out: 2*(nnz/2). */
uint64_t sgc_gen_init_stream(const sgc_csr* g, uint32_t* out_pairs);
/* Churn stream of generate_bench_stream_edges (stream_gen.cpp:65-177): the same
 * std::mt19937_64 / std::uniform_int_distribution draws, so the bytes match the
 * reference built with the same libstdc++. out_pairs: 2*size, out_types: size. */
int sgc_gen_churn_stream(const sgc_csr* g, uint64_t size, uint32_t insert_pct, uint64_t seed,
                         uint32_t* out_pairs, uint8_t* out_types);
/* Dense stream over the k-core at the given core-number percentile: every third
 * event deletes a uniformly chosen live edge inside the core, the other two
 * insert a uniformly chosen non-adjacent pair of core vertices. Writes the core
 * threshold and core size through the out pointers. */
int sgc_gen_kcore_stream(const sgc_csr* g, uint64_t size, double percentile, uint64_t seed,
                         uint32_t* out_pairs, uint8_t* out_types, uint32_t* core_k, uint32_t* core_size);
/* Core numbers (Batagelj-Zaversnik bucket peeling). */
int sgc_core_numbers(const sgc_csr* g, uint32_t* core);

/* Synthetic graphs. R-MAT: 2^scale vertices, edge_factor * 2^scale draws with
 * quadrant probabilities (a, b, c, 1-a-b-c). Chung-Lu: expected degrees from a
 * power law with the given exponent, scaled to avg_degree, capped at max_degree. */
int sgc_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed, sgc_csr* out);
int sgc_gen_chung_lu(uint32_t n, double exponent, double avg_degree, double max_degree, uint64_t seed, sgc_csr* out);

/* static_greedy_coloring (streamgc.cu:559-592): first-fit in id order. */
uint32_t sgc_static_greedy(const sgc_csr* g);

/* write_coloring (streamgc.cu:595-642): raw little-endian uint16 per vertex,
 * plus "<path>.txt" with its 3-line header. */
int sgc_write_coloring(const char* path, const uint16_t* colors, uint32_t n);

#ifdef __cplusplus
}
#endif
#endif
