// stream_gc -- command-line driver with the reference program's flags and
// outputs (algorithms/streamgc/src/streamgc.cu:654-1583), single GPU.
//
//   --graph --stream --insert-pct --seed --num-gpus --hw-tag --output-dir
//   --log-dir --epoch-size --histogram-threshold --validate --profile-hw
//   --init-only                                  (streamgc.cu:670-684)
// plus
//   --mode det|conc        det (default): stream order, reference epochs;
//                          conc: concurrent batches, repaired epochs
//   --stream-kcore <pct>   dense stream over the k-core at that core-number
//                          percentile (2 inserts per delete) instead of churn
//   --slack-pct <p> --max-hist-colors <c>   the reference's compile-time knobs
//   --exact-select         concurrent configuration: exact color selection and
//                          independent-set repair (SGC_OPT_EXACT_SELECT)
//   --graph-publish --sorted-rows            SGC_OPT_GRAPH_PUBLISH, SGC_OPT_SORTED_ROWS
//   --ablation force-bitmap|no-overflow|live-deg   the reference's abl-* builds
//                          (SGC_OPT_ABL_*), with its rules
//
// Output names follow the code (streamgc.cu:1479-1481):
//   <dir>/streamgc_<G>gpu_stream<N>_<pct>pct.coloring (+ .txt, + .meta)
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/streamgc_b200.h"
#include "sgc_host.h"

namespace {

using clk = std::chrono::high_resolution_clock;
double ms_since(clk::time_point t) { return std::chrono::duration<double, std::milli>(clk::now() - t).count(); }

void ensure_dir(const std::string& path) {
    size_t pos = 0;
    while ((pos = path.find('/', pos + 1)) != std::string::npos) mkdir(path.substr(0, pos).c_str(), 0755);
    mkdir(path.c_str(), 0755);
}

#define OK(call)                                                                          \
    do {                                                                                  \
        int r_ = (call);                                                                  \
        if (r_ != 0) {                                                                    \
            fprintf(stderr, "[StreamGC] ERROR %s -> %d: %s\n", #call, r_, sgc_last_error()); \
            return 1;                                                                     \
        }                                                                                 \
    } while (0)

struct Prof {
    double total_ms = 0, local_kernel_ms = 0, epoch_ms = 0, memcpy_ms = 0;
    double query_total_us = 0;
    uint64_t query_count = 0;
};

std::vector<EdgeUpdate> to_updates(const std::vector<uint32_t>& pairs, const std::vector<uint8_t>* types) {
    std::vector<EdgeUpdate> u(pairs.size() / 2);
    for (size_t i = 0; i < u.size(); i++) {
        std::memset(&u[i], 0, sizeof(EdgeUpdate));
        u[i].u = pairs[2 * i];
        u[i].v = pairs[2 * i + 1];
        u[i].type = types ? (*types)[i] : (uint8_t)SGC_UPDATE_ADD;
    }
    return u;
}

}  // namespace

int main(int argc, char** argv) {
    const char* graph_file = nullptr;
    uint64_t stream_size = 1000000;
    uint32_t insert_pct = 50;
    uint64_t seed = 42;
    uint32_t num_gpus = 1;
    const char* hw_tag = nullptr;
    const char* output_dir = nullptr;
    uint32_t epoch_size = SGC_EPOCH_SIZE_DEFAULT;
    uint32_t histogram_threshold = SGC_HISTOGRAM_THRESHOLD_DEFAULT;
    bool validate = false, init_only = false;
    int mode = SGC_MODE_DETERMINISTIC;
    double kcore_pct = -1;
    sgc_options opt;
    sgc_default_options(&opt);
    for (int i = 1; i < argc; i++) {
        auto is = [&](const char* f) { return strcmp(argv[i], f) == 0 && i + 1 < argc; };
        if (is("--graph")) graph_file = argv[++i];
        else if (is("--stream")) stream_size = strtoull(argv[++i], nullptr, 10);
        else if (is("--insert-pct")) insert_pct = (uint32_t)atoi(argv[++i]);
        else if (is("--seed")) seed = strtoull(argv[++i], nullptr, 10);
        else if (is("--num-gpus")) num_gpus = (uint32_t)atoi(argv[++i]);
        else if (is("--hw-tag")) hw_tag = argv[++i];
        else if (is("--output-dir")) output_dir = argv[++i];
        else if (is("--log-dir")) ++i;  // accepted, unused (as in the reference)
        else if (is("--epoch-size")) epoch_size = (uint32_t)atoi(argv[++i]);
        else if (is("--histogram-threshold")) histogram_threshold = (uint32_t)atoi(argv[++i]);
        else if (strcmp(argv[i], "--validate") == 0) validate = true;
        else if (strcmp(argv[i], "--profile-hw") == 0) {}
        else if (strcmp(argv[i], "--init-only") == 0) init_only = true;
        else if (is("--mode")) mode = strcmp(argv[++i], "conc") == 0 ? SGC_MODE_CONCURRENT : SGC_MODE_DETERMINISTIC;
        else if (is("--stream-kcore")) kcore_pct = atof(argv[++i]);
        else if (is("--slack-pct")) opt.slack_pct = (uint32_t)atoi(argv[++i]);
        else if (is("--max-hist-colors")) opt.max_hist_colors = (uint32_t)atoi(argv[++i]);
        else if (strcmp(argv[i], "--exact-select") == 0) opt.flags |= SGC_OPT_EXACT_SELECT;
        else if (strcmp(argv[i], "--graph-publish") == 0) opt.flags |= SGC_OPT_GRAPH_PUBLISH;
        else if (strcmp(argv[i], "--sorted-rows") == 0) opt.flags |= SGC_OPT_SORTED_ROWS;
        else if (is("--ablation")) {  // the reference's abl-* builds (Makefile:55-78)
            const char* a = argv[++i];
            if (!strcmp(a, "force-bitmap")) opt.flags |= SGC_OPT_ABL_FORCE_BITMAP;
            else if (!strcmp(a, "no-overflow")) opt.flags |= SGC_OPT_ABL_NO_OVERFLOW;
            else if (!strcmp(a, "live-deg")) opt.flags |= SGC_OPT_ABL_LIVE_DEG;
            else {
                fprintf(stderr, "[StreamGC] unknown ablation %s (force-bitmap, no-overflow, live-deg)\n", a);
                return 1;
            }
        }
    }
    if (!graph_file) {
        fprintf(stderr, "Usage: %s --graph <path.mtx> [options]\n", argv[0]);
        return 1;
    }
    if (num_gpus != 1) {
        fprintf(stderr, "[StreamGC] --num-gpus %u: this program runs the single-GPU path only\n", num_gpus);
        return 1;
    }
    std::string hw;
    if (hw_tag) {
        hw = hw_tag;
    } else {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, 0) != cudaSuccess) {
            fprintf(stderr, "[StreamGC] no CUDA device\n");
            return 1;
        }
        hw = prop.name;
        std::replace(hw.begin(), hw.end(), ' ', '_');
    }
    printf("[StreamGC] Hardware: %s, GPUs: %u\n", hw.c_str(), num_gpus);
    cudaSetDevice(0);
    cudaFree(0);

    sgc_csr graph;
    OK(sgc_load_mtx(graph_file, &graph));
    printf("[StreamGC] Loaded: %u vertices, %llu edges (directed), %llu undirected\n", graph.n,
           (unsigned long long)graph.nnz, (unsigned long long)(graph.nnz / 2));
    StreamGCConfig cfg = sgc_default_config();
    cfg.num_gpus = 1;
    cfg.num_vertices = graph.n;
    cfg.num_edges = graph.nnz;
    cfg.epoch_size = epoch_size;
    cfg.histogram_threshold = histogram_threshold;
    printf("[StreamGC] Config: epoch_size=%u, histogram_threshold=%u, mode=%s\n", cfg.epoch_size,
           cfg.histogram_threshold, mode == SGC_MODE_DETERMINISTIC ? "det" : "conc");

    auto t_part = clk::now();
    sgc_handle* h = nullptr;
    OK(sgc_create_ex(&cfg, &opt, graph.row_ptr, graph.col_idx, graph.degree, &h));
    const double partition_time_ms = ms_since(t_part);
    sgc_stats st;
    sgc_get_stats(h, &st);
    printf("[StreamGC] GPU 0 partition allocated: %u owned, 0 ghost, %llu local edges, %u high-degree\n", graph.n,
           (unsigned long long)graph.nnz, st.num_high_degree);

    std::vector<uint32_t> init_pairs(graph.nnz);
    const uint64_t ninit = sgc_gen_init_stream(&graph, init_pairs.data());
    init_pairs.resize(2 * ninit);
    printf("[StreamGC] Init stream: %llu edges (degree-descending order)\n", (unsigned long long)ninit);
    std::vector<uint32_t> bench_pairs(2 * stream_size);
    std::vector<uint8_t> bench_types(stream_size);
    if (kcore_pct >= 0) {
        uint32_t k = 0, cs = 0;
        OK(sgc_gen_kcore_stream(&graph, stream_size, kcore_pct, seed, bench_pairs.data(), bench_types.data(), &k, &cs));
        printf("[StreamGC] Bench stream: %llu events (k-core %u, %u vertices, 2 inserts per delete, seed=%llu)\n",
               (unsigned long long)stream_size, k, cs, (unsigned long long)seed);
    } else {
        OK(sgc_gen_churn_stream(&graph, stream_size, insert_pct, seed, bench_pairs.data(), bench_types.data()));
        printf("[StreamGC] Bench stream: %llu events (%u%% insert, seed=%llu)\n", (unsigned long long)stream_size,
               insert_pct, (unsigned long long)seed);
    }
    const auto init_ups = to_updates(init_pairs, nullptr);
    const auto bench_ups = to_updates(bench_pairs, &bench_types);

    // process_stream (streamgc.cu:809-1053) with per-stage timing
    auto process = [&](const std::vector<EdgeUpdate>& ups, const char* phase, bool sample_queries, Prof& prof) -> int {
        std::mt19937 qrng((uint32_t)(seed + 999));
        const uint64_t total = ups.size();
        const uint64_t batch = mode == SGC_MODE_DETERMINISTIC ? SGC_HOST_BATCH_SIZE
                                                               : std::min<uint64_t>(epoch_size, opt.max_batch);
        uint64_t processed = 0, since = 0;
        auto t0 = clk::now();
        while (processed < total) {
            const uint32_t b = (uint32_t)std::min<uint64_t>(batch, total - processed);
            auto ts = clk::now();
            OK(sgc_apply(h, ups.data() + processed, b, mode));
            OK(sgc_synchronize(h));
            prof.local_kernel_ms += ms_since(ts);
            processed += b;
            since += b;
            if (since >= epoch_size) {
                auto te = clk::now();
                if (mode == SGC_MODE_DETERMINISTIC) OK(sgc_epoch(h));
                else OK(sgc_publish(h, nullptr));
                OK(sgc_synchronize(h));
                prof.epoch_ms += ms_since(te);
                if (sample_queries) {
                    std::uniform_int_distribution<uint32_t> qd(0, graph.n - 1);
                    for (int q = 0; q < 100; q++) {
                        const uint32_t v = qd(qrng);
                        uint16_t c = 0;
                        auto tq = clk::now();
                        OK(sgc_query(h, &v, &c, 1));
                        prof.query_total_us += ms_since(tq) * 1000.0;
                        prof.query_count++;
                    }
                }
                since = 0;
            }
            if (processed % (total / 10 + 1) < batch) {
                printf("[StreamGC] %s: %llu / %llu (%.0f%%)\n", phase, (unsigned long long)processed,
                       (unsigned long long)total, 100.0 * processed / total);
                fflush(stdout);
            }
        }
        prof.total_ms = ms_since(t0);
        return 0;
    };
    auto repair = [&](const char* phase) -> int {
        sgc_repair_report rep;
        auto t = clk::now();
        OK(sgc_repair(h, &rep));
        printf("[StreamGC] %s repair: tier-1 %u iteration(s), last %u conflicts; tier-2 %s fixed %u (%.2f ms)\n",
               phase, rep.tier1_iterations, rep.tier1_last_count, rep.tier2_ran ? "ran," : "skipped,",
               rep.tier2_fixed, ms_since(t));
        if (rep.drained)
            printf("[StreamGC] %s overflow drain: %u local attempted, %llu failed\n", phase, rep.drained,
                   (unsigned long long)rep.drain_failed);
        return 0;
    };

    printf("[StreamGC] Starting Phase 1: Init stream (%zu edges)...\n", init_ups.size());
    Prof init_prof;
    if (process(init_ups, "Init", false, init_prof)) return 1;
    const double init_time_ms = init_prof.total_ms;
    printf("[StreamGC] Init complete: %.2f ms\n", init_time_ms);
    if (repair("Init")) return 1;

    Prof bench_prof;
    double bench_stream_ms = 0, bench_total_ms = 0;
    if (!init_only) {
        printf("[StreamGC] Starting Phase 2: Bench stream (%zu events)...\n", bench_ups.size());
        auto tb = clk::now();
        if (process(bench_ups, "Bench", true, bench_prof)) return 1;
        bench_stream_ms = bench_prof.total_ms;
        printf("[StreamGC] Bench stream complete: %.2f ms\n", bench_stream_ms);
        if (repair("Bench")) return 1;
        bench_total_ms = ms_since(tb);
    }
    const double repair_ms = bench_total_ms - bench_stream_ms;
    printf("[StreamGC] Init time: %.2f ms\n", init_time_ms);
    printf("[StreamGC] Bench time: %.2f ms (stream: %.2f ms, repair: %.2f ms)\n", bench_total_ms, bench_stream_ms,
           repair_ms);
    const double raw_tp = bench_stream_ms > 0 ? bench_ups.size() / bench_stream_ms / 1000.0 : 0;
    const double eff_tp = bench_total_ms > 0 ? bench_ups.size() / bench_total_ms / 1000.0 : 0;
    printf("[StreamGC] Throughput: %.2f M updates/sec (effective: %.2f M updates/sec)\n", raw_tp, eff_tp);

    if (validate) {
        sgc_validation v;
        OK(sgc_validate(h, &v));
        if (v.violations)
            fprintf(stderr, "[StreamGC] COLORING INVALID: %llu violations, %llu uncolored-with-edges (edges: %llu)\n",
                    (unsigned long long)v.violations, (unsigned long long)v.uncolored_with_edges,
                    (unsigned long long)v.edges);
        else
            printf("[StreamGC] Coloring valid: 0 violations, %llu uncolored-with-edges (edges: %llu)\n",
                   (unsigned long long)v.uncolored_with_edges, (unsigned long long)v.edges);
        printf("[StreamGC] Colors used: %llu\n", (unsigned long long)v.max_color);
        if (v.violations) fprintf(stderr, "[StreamGC] VALIDATION FAILED\n");
    }

    if (output_dir) {
        ensure_dir(output_dir);
        std::string gp(graph_file);
        const size_t slash = gp.rfind('/');
        const size_t dot = gp.rfind('.');
        const std::string gname = gp.substr(slash == std::string::npos ? 0 : slash + 1,
                                            dot - (slash == std::string::npos ? 0 : slash + 1));
        char cpath[1024];
        snprintf(cpath, sizeof(cpath), "%s/streamgc_%ugpu_stream%llu_%upct.coloring", output_dir, num_gpus,
                 (unsigned long long)stream_size, insert_pct);
        std::vector<uint16_t> colors(graph.n);
        OK(sgc_download(h, SGC_DL_COLORS, colors.data(), colors.size() * 2));
        OK(sgc_write_coloring(cpath, colors.data(), graph.n));
        printf("[StreamGC] Coloring written: %s (%u vertices)\n", cpath, graph.n);
        const uint32_t greedy = sgc_static_greedy(&graph);
        printf("[StreamGC] Static greedy: %u colors\n", greedy);
        const uint16_t maxc = colors.empty() ? 0 : *std::max_element(colors.begin(), colors.end());
        const float ratio = greedy > 0 ? (float)maxc / greedy : 0.0f;
        char mpath[1100];
        snprintf(mpath, sizeof(mpath), "%s.meta", cpath);
        FILE* mf = fopen(mpath, "w");
        if (mf) {
            // key order and formats of streamgc.cu:1511-1570
            fprintf(mf, "{\n");
            fprintf(mf, "  \"algorithm\": \"streamgc\",\n");
            fprintf(mf, "  \"graph\": \"%s\",\n", gname.c_str());
            fprintf(mf, "  \"num_vertices\": %u,\n", graph.n);
            fprintf(mf, "  \"num_edges\": %lu,\n", (unsigned long)graph.nnz);
            fprintf(mf, "  \"num_colors_used\": %u,\n", maxc);
            fprintf(mf, "  \"static_greedy_colors\": %u,\n", greedy);
            fprintf(mf, "  \"color_ratio\": %.2f,\n", ratio);
            fprintf(mf, "  \"init_time_ms\": %.2f,\n", init_time_ms);
            fprintf(mf, "  \"bench_time_ms\": %.2f,\n", bench_total_ms);
            fprintf(mf, "  \"bench_stream_ms\": %.2f,\n", bench_stream_ms);
            fprintf(mf, "  \"repair_time_ms\": %.2f,\n", repair_ms);
            fprintf(mf, "  \"throughput_mups\": %.2f,\n", raw_tp);
            fprintf(mf, "  \"effective_throughput_mups\": %.2f,\n", eff_tp);
            fprintf(mf, "  \"classify_ms\": %.2f,\n", 0.0);
            fprintf(mf, "  \"local_kernel_ms\": %.2f,\n", bench_prof.local_kernel_ms);
            fprintf(mf, "  \"boundary_kernel_ms\": %.2f,\n", 0.0);
            fprintf(mf, "  \"gpu_sync_ms\": %.2f,\n", 0.0);
            fprintf(mf, "  \"ghost_sync_ms\": %.2f,\n", 0.0);
            fprintf(mf, "  \"epoch_maintenance_ms\": %.2f,\n", bench_prof.epoch_ms);
            fprintf(mf, "  \"memcpy_ms\": %.2f,\n", bench_prof.memcpy_ms);
            fprintf(mf, "  \"query_latency_us\": %.2f,\n",
                    bench_prof.query_count ? bench_prof.query_total_us / bench_prof.query_count : 0.0);
            fprintf(mf, "  \"query_count\": %lu,\n", (unsigned long)bench_prof.query_count);
            fprintf(mf, "  \"partition_time_ms\": %.2f,\n", partition_time_ms);
            fprintf(mf, "  \"partition_info\": [\n");
            fprintf(mf, "    {\"gpu\": %u, \"owned\": %u, \"ghost\": %u, \"edges\": %lu}\n", 0u, graph.n, 0u,
                    (unsigned long)graph.nnz);
            fprintf(mf, "  ],\n");
            fprintf(mf, "  \"stream_size\": %lu,\n", (unsigned long)stream_size);
            fprintf(mf, "  \"insert_pct\": %u,\n", insert_pct);
            fprintf(mf, "  \"seed\": %lu,\n", (unsigned long)seed);
            fprintf(mf, "  \"num_gpus\": %u,\n", num_gpus);
            fprintf(mf, "  \"hw_tag\": \"%s\"\n", hw.c_str());
            fprintf(mf, "}\n");
            fclose(mf);
            printf("[StreamGC] Meta written: %s (ratio: %.2f)\n", mpath, ratio);
        }
    }
    sgc_destroy(h);
    sgc_csr_free(&graph);
    printf("[StreamGC] Done.\n");
    return 0;
}
