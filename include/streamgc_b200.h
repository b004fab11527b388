/*
 * streamgc_b200.h -- C ABI of the B200 streaming graph-coloring library
 * (libstreamgc_b200.so). Plain pointers and sizes; no CUDA or C++ types.
 *
 * The reference exposes this path only as a program (algorithms/streamgc/src/
 * streamgc.cu main(), 654-1583) whose host loop calls device kernels. Each
 * entry point below replaces one piece of that loop; the comment on each names
 * the reference code it stands for. Every call returns 0 on success and a
 * negative SGC_E* code on failure (sgc_last_error() has the message); nothing
 * calls exit(). One handle owns all device memory of one graph and one CUDA
 * stream; handles are independent and may be driven from different threads
 * (one thread per handle at a time).
 */
#ifndef STREAMGC_B200_H
#define STREAMGC_B200_H

#include <stdint.h>
#include "streamgc_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sgc_handle sgc_handle;

/* status codes */
#define SGC_OK           0
#define SGC_EINVAL      -1   /* bad argument */
#define SGC_ECUDA       -2   /* CUDA runtime error */
#define SGC_ENOMEM      -3   /* device or host allocation failed */
#define SGC_EDEVICE     -4   /* device-side error word set (see sgc_stats.device_error) */
#define SGC_ENOTSUP     -5   /* request outside this library's single-GPU scope */

/* update-application modes */
#define SGC_MODE_DETERMINISTIC 0  /* stream order, one warp: bit-exact with the reference run as one warp */
#define SGC_MODE_CONCURRENT    1  /* one warp per update, same-edge updates kept in stream order */

/* sgc_options.flags */
#define SGC_OPT_PROFILE  1u       /* time sweeps with CUDA events (sgc_stats.sweep_*) */
/* Exact color selection above the histogram threshold: the first color no live
 * neighbor holds, from a bitset the warp builds in shared memory while it scans
 * the row, instead of the reference's global per-vertex histograms (which are
 * never rebuilt and drift, color_select.cuh:120-209). No histogram rows are
 * allocated. Bit-exact parity with the reference needs this flag off. */
#define SGC_OPT_EXACT_SELECT 2u
/* With SGC_OPT_EXACT_SELECT, a publish after concurrent batches replays one
 * captured CUDA graph (compaction, drain, the repair loop as a conditional
 * while-node, snapshot): one host synchronization per epoch instead of one per
 * sweep. Sweeps are not timed one by one (sgc_stats.sweep_ms stays 0). */
#define SGC_OPT_GRAPH_PUBLISH 4u
/* With SGC_OPT_EXACT_SELECT, compaction also sorts every row of at most 1024
 * live entries into one base run, and compacts a row whose unsorted tail (the
 * entries inserted since its last compaction) outgrows an eighth of it even
 * with few holes: searches stay 32-ary over long runs. Colors do not depend on
 * it. */
#define SGC_OPT_SORTED_ROWS 8u
/* The reference's ablation builds (Makefile abl-* targets), as options of the
 * reference rules (not with SGC_OPT_EXACT_SELECT):
 *   FORCE_BITMAP  every vertex picks its color from its neighbor bitmap
 *                 (STREAMGC_ABLATION_FORCE_BITMAP, color_select.cuh:98-100);
 *   NO_OVERFLOW   an insert into a full row is dropped, not buffered
 *                 (STREAMGC_ABLATION_NO_OVERFLOW, local_update.cu:28-38);
 *   LIVE_DEG      Tier-1 ranks a vertex by its live degree against its
 *                 neighbors' frozen priorities (STREAMGC_ABLATION_LIVE_DEG_PRIORITY,
 *                 conflict_repair.cu:46-57).
 * The reference's abl-force-histogram build compiles the same dispatch as its
 * default (color_select.cuh:101-107), so it has no option here. */
#define SGC_OPT_ABL_FORCE_BITMAP 16u
#define SGC_OPT_ABL_NO_OVERFLOW  32u
#define SGC_OPT_ABL_LIVE_DEG     64u

typedef struct sgc_options {
    uint32_t struct_size;      /* sizeof(sgc_options) */
    uint32_t slack_pct;        /* extra row capacity in percent (STREAMGC_CSR_EXTRA_SLACK_PCT, streamgc.cu:169-171); 300 = alpha 4 */
    uint32_t max_hist_colors;  /* histogram bins per high-degree vertex (STREAMGC_MAX_HISTOGRAM_COLORS, partition.cuh:6-9); multiple of 4 */
    uint32_t max_batch;        /* largest batch sgc_apply accepts (default 32768, the reference's host batch) */
    int32_t  device;           /* CUDA device ordinal */
    uint32_t flags;            /* SGC_OPT_* */
    uint32_t full_repair_every;/* exact selection: every Nth repair visits every vertex (0 = only when
                                  required, 1 = always); the others start from the touched vertices */
    uint32_t repair_tile;      /* slots per warp work item in repair sweeps (0 = 512; >= 256) */
} sgc_options;

/* What one repair (sgc_repair / sgc_publish) did. */
typedef struct sgc_repair_report {
    uint32_t tier1_iterations;   /* sweeps run (run_conflict_repair loop, streamgc.cu:1317-1393) */
    uint32_t tier1_last_count;   /* conflicts counted by the last sweep (0 = converged) */
    uint32_t tier2_ran;          /* 1 when Tier-2 had to run (it is a no-op after convergence on a symmetric CSR) */
    uint32_t tier2_fixed;        /* vertices Tier-2 recolored (cpu_serial_repair, streamgc.cu:1057-1240) */
    uint32_t tier2_gave_up;      /* 1 when Tier-2 stopped with conflicts left (30 passes or no free color) */
    uint32_t drained;            /* overflow entries re-inserted this call */
    uint64_t drain_failed;       /* overflow entries that still found no slot */
    uint32_t proper;             /* 1 when the result is a proper coloring of the live CSR */
    uint32_t incremental;        /* 1 when the first sweep visited only the vertices touched since the last repair */
} sgc_repair_report;

typedef struct sgc_stats {
    uint64_t updates_submitted;
    uint64_t updates_skipped;    /* endpoint outside [0, n): skipped like a hash miss */
    uint64_t epochs;             /* sgc_epoch + sgc_publish calls */
    uint64_t overflow_pending;   /* overflow counter (entries waiting for the next drain) */
    uint64_t overflow_lost;      /* overflows beyond the 262144-entry buffer (edge dropped) */
    uint64_t drain_failed;       /* cumulative */
    uint64_t tier1_sweeps;       /* cumulative */
    uint64_t tier2_runs;
    uint64_t tier2_fixed;
    uint32_t device_error;       /* bit 0: wait timeout, bit 1: bad update, bit 2: list overflow */
    uint32_t num_vertices;
    uint32_t num_high_degree;
    uint32_t max_hist_colors;    /* histogram bins per row kept on the device (0 with SGC_OPT_EXACT_SELECT) */
    uint64_t total_slots;        /* slack CSR slots */
    uint64_t device_bytes;       /* device memory held by the handle */
    double   sweep_ms;           /* SGC_OPT_PROFILE: summed device time of sweep edge passes */
    uint64_t sweep_count;        /* SGC_OPT_PROFILE: sweeps timed */
    uint64_t sweep_bytes;        /* algorithmic bytes of the timed sweeps: 8 per live entry + 28 per vertex */
    uint64_t live_entries;       /* live adjacency entries at the last sweep */
    uint64_t kernel_launches;    /* kernels launched by this handle */
    uint64_t h2d_bytes;          /* update bytes copied host -> device by sgc_apply */
    uint64_t d2h_bytes;          /* bytes the library read back (repair counters, stats) */
    double   sweep_phase_ms[4];  /* SGC_OPT_PROFILE: sweep_ms by phase: item build, long-row items,
                                    per-vertex finalize, color selection and commit */
    uint64_t hub_deferred;       /* row-scale operations of concurrent batches (color reductions and
                                    recolors of rows longer than 512 live entries) finished by the
                                    block-wide pass after the batch (cumulative) */
} sgc_stats;

typedef struct sgc_validation {
    uint64_t violations;            /* distinct live edges whose endpoints share a nonzero color */
    uint64_t uncolored_with_edges;  /* vertices with color 0 and a live row entry */
    uint64_t edges;                 /* distinct live undirected edges */
    uint64_t max_color;             /* "Colors used" of the reference validator */
    uint64_t out_of_range;          /* live entries naming a vertex >= n */
} sgc_validation;

/* Layout invariants of the rows (sgc_check_state). */
#define SGC_STATE_HW     0x1u   /* high-water mark beyond the row's capacity (or row offsets decreasing) */
#define SGC_STATE_TAIL   0x2u   /* a slot at or past the high-water mark that is not free */
#define SGC_STATE_ID     0x4u   /* an entry naming a vertex >= n */
#define SGC_STATE_RUN    0x8u   /* sorted prefix (base run / never-edited row) not strictly ascending */
#define SGC_STATE_HOLES  0x10u  /* live-entry count differs from the row's live slots */
#define SGC_STATE_COLOR  0x20u  /* a color above 2048 */

typedef struct sgc_state_report {
    uint64_t rows;        /* rows checked (the handle's vertices) */
    uint64_t bad_rows;    /* rows breaking at least one invariant */
    uint32_t flags;       /* SGC_STATE_* bits seen */
    uint32_t first_bad;   /* lowest such row, 0xFFFFFFFF when none */
} sgc_state_report;

/* sgc_download / sgc_upload targets */
#define SGC_DL_STATES    0   /* uint32[n] packed (color | version << 16) */
#define SGC_DL_COLORS    1   /* uint16[n] current colors */
#define SGC_DL_BITMAPS   2   /* uint64[n] */
#define SGC_DL_HIST      3   /* uint32[num_high_degree * max_hist_colors] */
#define SGC_DL_ROW_PTR   4   /* uint64[n + 1] logical row starts */
#define SGC_DL_COL       5   /* uint32[total_slots] */
#define SGC_DL_SNAPSHOT  6   /* uint16[n] last published snapshot */
#define SGC_DL_HIGHWATER 7   /* uint32[n] per-row high-water mark */
#define SGC_DL_HDMAP     8   /* uint32[n] histogram row or 0xFFFFFFFF */
#define SGC_DL_OVERFLOW  9   /* OverflowEdge[min(overflow_pending, 262144)] */
#define SGC_DL_BASE_RUN 10   /* uint32[n] length of each row's sorted base run (exact selection), else zeros */
#define SGC_DL_HOLES    11   /* uint32[n] free slots and tombstones below each row's mark (exact selection), else zeros */

/* Fills defaults: slack 300, 1024 histogram colors, batch 32768, device 0. */
int sgc_default_options(sgc_options* opt);

/* Builds the single-GPU partition from a base CSR: the work of
 * allocate_gpu_partition + the priority setup of main() (streamgc.cu:144-444,
 * 754-767). row_ptr has n+1 entries; rows are copied into the alpha slack CSR
 * in the given order; degree[v] sets the frozen priority (degree << 32 | v) and
 * histogram mode (degree > cfg->histogram_threshold). cfg->num_vertices = n. */
int sgc_create(const StreamGCConfig* cfg, const uint32_t* row_ptr, const uint32_t* col_idx,
               const uint32_t* degree, sgc_handle** out);
/* Same with 64-bit row offsets (graphs beyond 2^32 directed entries) and options. */
int sgc_create_ex(const StreamGCConfig* cfg, const sgc_options* opt, const uint64_t* row_ptr,
                  const uint32_t* col_idx, const uint32_t* degree, sgc_handle** out);
int sgc_destroy(sgc_handle* h);

/* Applies n <= max_batch updates (one host batch of process_stream,
 * streamgc.cu:828-856): local_update_kernel semantics per update. `updates`
 * may be host (pageable or pinned) or device memory. No epoch work. */
int sgc_apply(sgc_handle* h, const EdgeUpdate* updates, uint32_t n, int mode);
/* Stream ingest (the reference's feeder ring, feeder_thread.cpp:25-92, unused
 * there): sgc_stage copies a host batch (n <= max_batch) into the next of two
 * device staging slots on the handle's copy stream and returns without waiting
 * for the GPU; sgc_apply_staged applies the oldest staged batch on the handle's
 * stream once its copy is done. Staging batch k+1 before publishing batch k
 * overlaps the copy with the repair. Pageable input is copied into pinned
 * memory before sgc_stage returns; pinned or device input is copied as it is
 * and must not change until the batch is applied. At most two batches are
 * staged; SGC_EINVAL when both slots are full (stage) or none is (apply). */
int sgc_stage(sgc_handle* h, const EdgeUpdate* updates, uint32_t n);
int sgc_apply_staged(sgc_handle* h, int mode);

/* Ingest ring: the role of the reference's feeder thread and pinned ring,
 * which it declares but never calls (feeder_thread.cpp:25-92, streamgc.cu:285-292).
 * A pinned, device-mapped ring of 2^log2_slots update slots; one producer
 * thread appends with sgc_ring_push (no CUDA call: a copy into the ring and a
 * release of the new tail; *accepted may be below n when the ring is full),
 * and the stepping thread drains it with sgc_ring_apply: one kernel copies up
 * to max_updates published slots straight from host memory into the batch
 * buffer, then the batch is applied (no cudaMemcpy per batch). Slots return
 * to the producer once the GPU has read them (checked at the next
 * sgc_ring_apply). */
int sgc_ring_create(sgc_handle* h, uint32_t log2_slots);
int sgc_ring_push(sgc_handle* h, const EdgeUpdate* updates, uint32_t n, uint32_t* accepted);
int sgc_ring_apply(sgc_handle* h, uint32_t max_updates, int mode, uint32_t* applied);

/* Reference epoch boundary (streamgc.cu:949-1012): publish the snapshot of the
 * current colors, compact edited rows, drain overflow, rebuild bitmaps. */
int sgc_epoch(sgc_handle* h);
/* drain_and_compact (streamgc.cu:1243-1314). */
int sgc_drain_and_compact(sgc_handle* h, sgc_repair_report* rep);
/* Phase-end repair (streamgc.cu:1405-1408): drain_and_compact, Tier-1 loop,
 * Tier-2. The snapshot is not republished (as in the reference). */
int sgc_repair(sgc_handle* h, sgc_repair_report* rep);
/* Repaired epoch boundary: compact, drain, Tier-1 loop, Tier-2, then publish
 * the snapshot, so every published snapshot is proper. */
int sgc_publish(sgc_handle* h, sgc_repair_report* rep);

/* process_stream (streamgc.cu:809-1053) for one GPU. DETERMINISTIC: host
 * batches of 32768, sgc_epoch when updates_since_epoch >= epoch_size (checked
 * after each batch). CONCURRENT: batches of min(epoch_size, max_batch),
 * sgc_publish at each boundary. Returns the number of epoch boundaries in
 * *epochs (may be NULL). */
int sgc_process_stream(sgc_handle* h, const EdgeUpdate* updates, uint64_t n, int mode, uint32_t* epochs);

/* Point queries against the last published snapshot (host arrays). */
int sgc_query(sgc_handle* h, const uint32_t* vertices, uint16_t* colors, uint32_t n);

/* Point queries exactly like sgc_query, for callers that must not allocate
 * device memory: sgc_query takes scratch from the CUDA allocator on each call,
 * which a serving thread whose tenants already fill their HBM budget, or a
 * latency-bound path that must not enter the allocator, cannot afford. This
 * variant calls no cudaMalloc, cudaFree or allocating routine; it stages the
 * vertex ids and colors in a fixed scratch array compiled into the library
 * (384 KiB, held by every GPU that loads the library until the process exits).
 * At most SGC_QUERY_NOALLOC_MAX vertices per call; larger n is rejected with
 * SGC_EINVAL. The first call on a device looks up the scratch's device address
 * (once per device); make that first call before any CUDA stream capture. All
 * handles on a device share the one scratch, so calls whose GPU work overlaps
 * (different threads or streams) race on it; serialize them. Each call leaves
 * its data in the scratch; the next call overwrites what it uses.
 * No counterpart in the reference (it has no device query path). */
#define SGC_QUERY_NOALLOC_MAX 65536u
int sgc_query_noalloc(sgc_handle* h, const uint32_t* vertices, uint16_t* colors, uint32_t n);

int sgc_download(sgc_handle* h, int what, void* dst, uint64_t bytes);
int sgc_upload(sgc_handle* h, int what, const void* src, uint64_t bytes);   /* STATES, BITMAPS, HIST */
/* Colors the uncolored vertices of initial degree >= min_degree one at a time,
 * in descending degree order (ties by id), each with the first color in
 * 1..2047 that none of its live neighbors holds (version 1). For a large graph
 * loaded without an init stream: its dense high-degree core then needs no
 * long chain of independent-set sweeps; the next repair (sgc_publish) visits
 * every vertex and colors the rest. No reference counterpart (the reference
 * colors its graph with the init stream, streamgc.cu:1395-1408). */
int sgc_color_core(sgc_handle* h, uint32_t min_degree, uint32_t* colored);
/* FindAvailableColor(x) (color_select.cuh:93-115) on the current device state. */
int sgc_find_color(sgc_handle* h, uint32_t x, uint16_t* color);

/* check_coloring_valid, streamgc.cu:448-556. Slabs beyond 2^32 slots are
 * counted without the distinct-edge sort: each edge at its lower endpoint's
 * entry (the same counts when every entry has its mirror). */
int sgc_validate(sgc_handle* h, sgc_validation* out);
/* Checks every row's layout invariants on the device (a debugging aid with no
 * reference counterpart); call between batches. */
int sgc_check_state(sgc_handle* h, sgc_state_report* out);
int sgc_get_stats(sgc_handle* h, sgc_stats* out);
int sgc_synchronize(sgc_handle* h);
/* The handle's cudaStream_t, for callers that time or order work around it. */
void* sgc_cuda_stream(sgc_handle* h);
const char* sgc_last_error(void);
const char* sgc_version(void);

#ifdef __cplusplus
}
#endif
#endif /* STREAMGC_B200_H */
