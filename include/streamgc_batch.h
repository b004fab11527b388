/*
 * streamgc_batch.h -- many graphs on one GPU (libstreamgc_b200.so).
 *
 * The reference runs one graph per process (algorithms/streamgc/src/streamgc.cu
 * main(), process_stream at streamgc.cu:809-1053). This interface keeps the
 * same per-graph semantics -- updates in EdgeUpdate form, epochs of
 * `epoch_size` updates that end with a repaired, published snapshot -- for
 * many graphs of uneven sizes resident side by side on one GPU:
 *
 *   - the graphs' rows live in one slack CSR (each graph's vertices start at a
 *     multiple of 32); ids in the calls below are the graph's own;
 *   - sgc_batch_tick() applies every update submitted since the last tick in
 *     one persistent launch fed by a device work queue, repairs, and publishes
 *     a snapshot for each graph whose epoch closed;
 *   - the tick runs as a captured CUDA graph (its repair loop is a
 *     conditional while-node), so a tick costs one launch from the host;
 *   - per graph, the repair state (clean / mirror-complete / forced) is kept
 *     apart, so with SGC_BATCH_STREAM_ORDER a graph's colors do not depend on
 *     the other graphs in the batch.
 *
 * Colors are valid for the live edges of each graph; every published snapshot
 * of a tick whose report says `proper` is a proper coloring.
 */
#ifndef STREAMGC_BATCH_H
#define STREAMGC_BATCH_H

#include <stdint.h>

#include "streamgc_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sgc_batch sgc_batch;

/* One graph of a batch: its CSR (host memory, ids 0..num_vertices-1). */
typedef struct sgc_batch_graph {
    uint32_t num_vertices;
    uint32_t epoch_size;           /* updates per published epoch; 0 = chosen by the tuner */
    uint32_t histogram_threshold;  /* degree above which colors are chosen exactly from the row; 0 = 64 */
    uint32_t _reserved;
    const uint64_t* row_ptr;       /* num_vertices + 1 */
    const uint32_t* col_idx;       /* row_ptr[num_vertices] entries, each < num_vertices */
    const uint32_t* degree;        /* priorities' degrees; null = row lengths */
} sgc_batch_graph;

#define SGC_BATCH_CUDA_GRAPH   1u  /* run each tick as a captured CUDA graph */
#define SGC_BATCH_STREAM_ORDER 2u  /* each graph's updates in submission order (one warp per graph):
                                      a graph's colors do not depend on the other graphs */
#define SGC_BATCH_PROFILE      4u  /* time every tick with CUDA events */
#define SGC_BATCH_SORTED_ROWS  8u  /* compaction keeps rows as one sorted run (SGC_OPT_SORTED_ROWS) */

typedef struct sgc_batch_options {
    uint32_t struct_size;          /* sizeof(sgc_batch_options) */
    uint32_t slack_pct;            /* extra row capacity in percent; 300 = alpha 4 */
    uint32_t max_tick_updates;     /* updates one tick can hold (all graphs) */
    int32_t  device;
    uint32_t flags;                /* SGC_BATCH_* */
    uint32_t repair_tile;          /* slots per warp work item in repair sweeps (0 = 512) */
    uint32_t apply_blocks_per_sm;  /* resident 256-thread blocks of the persistent apply (0 = all that fit) */
    uint32_t _reserved;
} sgc_batch_options;

typedef struct sgc_batch_tick_report {
    uint32_t updates;              /* updates applied by this tick */
    uint32_t published;            /* graphs whose epoch closed: snapshot published */
    uint32_t tier1_iterations;     /* repair sweeps */
    uint32_t tier2_ran;            /* 1 when the sequential fallback had to run */
    uint32_t proper;               /* 1 when every graph's coloring is proper */
    uint32_t tier2_reason;         /* bit 0: some graph's rows may miss mirror entries; bit 1: the repair
                                      did not converge in 64 sweeps (Tier-2 visits only those graphs) */
    double   device_ms;            /* tick time on the device (SGC_BATCH_PROFILE), else 0 */
} sgc_batch_tick_report;

/* Knobs the tuner chooses; none changes how a color is chosen. */
typedef struct sgc_batch_tuning {
    uint32_t repair_tile;          /* 256 .. 2048 */
    uint32_t apply_blocks_per_sm;  /* 1 .. the occupancy limit */
} sgc_batch_tuning;

int sgc_batch_default_options(sgc_batch_options* opt);
int sgc_batch_create(const sgc_batch_graph* graphs, uint32_t count, const sgc_batch_options* opt, sgc_batch** out);
int sgc_batch_destroy(sgc_batch* b);
uint32_t sgc_batch_num_graphs(const sgc_batch* b);
uint32_t sgc_batch_epoch_size(const sgc_batch* b, uint32_t graph);

/* Stages updates of one graph for the next tick (host memory; ids local to the
 * graph; an id outside the graph makes the update a no-op, counted as skipped).
 * SGC_EINVAL when the tick buffer is full. Allowed while a tick runs (between
 * sgc_batch_tick_begin and _end): the staging buffer has two halves, so the
 * next tick's updates are staged while the current ones are applied. Calls
 * come from one thread (the one that ticks). */
int sgc_batch_submit(sgc_batch* b, uint32_t graph, const EdgeUpdate* ups, uint32_t n);
/* Updates staged and not yet applied, over all graphs. */
uint64_t sgc_batch_pending(const sgc_batch* b);
/* Applies everything staged, repairs, publishes the graphs whose epoch closed. */
int sgc_batch_tick(sgc_batch* b, sgc_batch_tick_report* rep);
/* The same in two halves: begin launches the tick on the batch's stream and
 * returns; end waits for it (ticks of several batches then overlap on the
 * device, and the next tick's submits overlap this one). */
int sgc_batch_tick_begin(sgc_batch* b);
int sgc_batch_tick_end(sgc_batch* b, sgc_batch_tick_report* rep);
/* Publishes every graph's current colors (closes all epochs) on the next tick. */
int sgc_batch_close_epochs(sgc_batch* b);
/* Closes one graph's epoch on the next tick. */
int sgc_batch_close_epoch(sgc_batch* b, uint32_t graph);
/* Snapshots the graph has published so far. */
uint64_t sgc_batch_publish_count(const sgc_batch* b, uint32_t graph);

/* Colors from the graph's last published snapshot (safe while a tick runs). */
int sgc_batch_query(sgc_batch* b, uint32_t graph, const uint32_t* v, uint16_t* out, uint32_t k);
int sgc_batch_snapshot(sgc_batch* b, uint32_t graph, uint16_t* out);  /* num_vertices entries */
/* The graph's live rows in its own ids: row_ptr (num_vertices + 1) and col
 * (row_ptr[num_vertices] entries) of the compacted rows; pass col = null to
 * read the size first. */
int sgc_batch_rows(sgc_batch* b, uint32_t graph, uint64_t* row_ptr, uint32_t* col, uint64_t col_cap);
/* Validator over all graphs (the reference's, streamgc.cu:448-556). */
int sgc_batch_validate(sgc_batch* b, sgc_validation* out);
/* sgc_color_core over every graph of the batch (graphs are disjoint, so each
 * one's colors are the same as alone); call before the first tick, which then
 * repairs every graph in full. */
int sgc_batch_color_core(sgc_batch* b, uint32_t min_degree, uint32_t* colored);
/* out[k] = 1 when graph k has dropped an entry since its creation: an
 * insert that found its row still full at the drain, or that arrived with the
 * overflow buffer full (the reference drops such entries too; the mirror
 * entry in the other row stays). Between ticks. */
int sgc_batch_dropped(sgc_batch* b, uint8_t* out);
/* Layout invariants of every graph's rows (sgc_check_state); between ticks. */
int sgc_batch_check_state(sgc_batch* b, sgc_state_report* out);

/* Histogram threshold of every graph created without one (32, 64 or 128 ...). */
int sgc_batch_set_thresholds(sgc_batch* b, uint32_t threshold);
int sgc_batch_get_tuning(sgc_batch* b, sgc_batch_tuning* t);
int sgc_batch_set_tuning(sgc_batch* b, const sgc_batch_tuning* t);
/* Online tuner: runs the next ticks (the caller keeps submitting) under
 * candidate settings, coordinate by coordinate, and keeps the fastest per
 * update. Returns once `ticks_per_candidate` ticks ran for each candidate. */
typedef int (*sgc_batch_feed_fn)(sgc_batch* b, void* ctx);  /* stages one tick's updates */
int sgc_batch_autotune(sgc_batch* b, sgc_batch_feed_fn feed, void* ctx, uint32_t ticks_per_candidate,
                       sgc_batch_tuning* chosen);

/* Counters of the union handle (updates, launches, bytes ...). */
int sgc_batch_stats(sgc_batch* b, sgc_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* STREAMGC_BATCH_H */
