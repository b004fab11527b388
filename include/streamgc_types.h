/*
 * streamgc_types.h -- record and struct layouts shared with the StreamGC
 * reference (C-compatible).
 *
 * Every struct here is byte-for-byte the layout the reference defines, so a
 * caller that builds these records with the reference headers can hand them to
 * this library unchanged:
 *   EdgeUpdate / UpdateType   algorithms/streamgc/include/types.h:8-21
 *   VertexState (packed word) algorithms/streamgc/include/vertex_state.cuh:8-27
 *   OverflowEdge              algorithms/streamgc/include/streamgc.cuh:17-23
 *   GPUPartition              algorithms/streamgc/include/streamgc.cuh:26-110
 *   StreamGCConfig            algorithms/streamgc/include/streamgc.cuh:113-135
 * The offsets are pinned by static_asserts at the end of this file (values
 * measured from the reference header compiled with nvcc 12.9, x86-64).
 */
#ifndef STREAMGC_TYPES_H
#define STREAMGC_TYPES_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Update kinds (types.h:8-13). Only ADD and DEL change state; the query kinds
 * are accepted and ignored by the update kernels exactly as the reference does. */
enum {
    SGC_UPDATE_ADD = 0,
    SGC_UPDATE_DEL = 1,
    SGC_UPDATE_QUERY_POINT = 2,
    SGC_UPDATE_QUERY_NEIGHBORHOOD = 3
};

/* 16-byte update record (types.h:16-21). `type` is the reference's
 * `UpdateType` enum class, whose underlying type is uint8_t. */
typedef struct __attribute__((aligned(16))) EdgeUpdate {
    uint32_t u;
    uint32_t v;
    uint8_t  type;
    uint8_t  _pad[7];
} EdgeUpdate;

/* Packed per-vertex word: color in bits 0..15, version in bits 16..31
 * (vertex_state.cuh:8-27). 0 = uncolored. */
typedef struct __attribute__((aligned(4))) VertexState {
    uint16_t color;
    uint16_t version;
} VertexState;

/* Overflow record for an insert that found its row full (streamgc.cuh:17-20). */
typedef struct OverflowEdge {
    uint32_t local_vertex_idx;
    uint32_t neighbor_global;
} OverflowEdge;

/* Opaque in this library: the multi-GPU partition map entry (partition.cuh:15-19). */
typedef struct PartitionEntry {
    uint8_t  current_owner;
    uint8_t  prev_owner;
    uint16_t migration_epoch;
} PartitionEntry;

/* Per-GPU partition state, every array in device memory (streamgc.cuh:26-110).
 * Used by the kernel-level drop-in entry points (streamgc_kernels.h), which take
 * a DEVICE copy of this struct exactly as the reference kernels do. */
typedef struct GPUPartition {
    VertexState* owned;
    uint32_t*    owned_to_global;
    VertexState* ghost;
    uint32_t*    ghost_to_global;
    uint32_t*    global_to_owned;
    uint32_t*    global_to_ghost;
    uint32_t     index_map_size;
    uint32_t     ghost_map_size;
    uint64_t*    neighbor_bitmap;
    uint32_t*    freq_histogram;
    uint32_t*    high_degree_map;
    uint32_t     num_high_degree;
    uint64_t*    init_priority;
    uint16_t*    epoch_snapshot;
    uint32_t*    row_ptr;
    uint32_t*    col_idx;
    uint32_t*    col_idx_capacity;
    uint32_t*    ghost_row_ptr;
    uint32_t*    ghost_col_idx;
    uint32_t*    ghost_col_idx_capacity;
    EdgeUpdate*  stream_buffer;
    uint32_t*    stream_head;
    uint32_t*    stream_tail;
    uint32_t     stream_mask;
    uint64_t*    update_counter;
    uint32_t*    epoch_ready_flag;
    uint32_t*    epoch_counter;
    PartitionEntry* d_partition_map;
    OverflowEdge* overflow_local;
    OverflowEdge* overflow_ghost;
    uint32_t*    overflow_local_count;
    uint32_t*    overflow_ghost_count;
    uint32_t     num_owned;
    uint32_t     num_ghost;
    uint32_t     num_edges_local;
    uint32_t     max_owned;
    uint32_t     max_ghost;
    uint32_t     gpu_id;
    int32_t*     phi_inflight;
    uint32_t*    phi_max;
    uint8_t*     is_boundary;
    uint8_t*     phi_dirty;
} GPUPartition;

/* System configuration (streamgc.cuh:113-122). `priority_refresh_interval`
 * and `rebalance_threshold` are carried but never read, as in the reference. */
typedef struct StreamGCConfig {
    uint32_t num_gpus;
    uint32_t num_vertices;
    uint64_t num_edges;
    uint32_t stream_buffer_size;
    uint32_t epoch_size;
    uint32_t priority_refresh_interval;
    uint32_t histogram_threshold;
    float    rebalance_threshold;
} StreamGCConfig;

/* Constants shared with the reference. */
#define SGC_HASH_EMPTY            0xFFFFFFFFu   /* types.h:24 */
#define SGC_CSR_INVALID           0xFFFFFFFFu   /* types.h:25 */
#define SGC_OVERFLOW_CAPACITY     262144u       /* streamgc.cuh:23 */
#define SGC_EPOCH_SIZE_DEFAULT    10000u        /* epoch.cuh:5 */
#define SGC_PRIORITY_REFRESH_DEFAULT 100u       /* epoch.cuh:6 */
#define SGC_REBALANCE_DEFAULT     0.2f          /* epoch.cuh:7 */
#define SGC_HISTOGRAM_THRESHOLD_DEFAULT 64u     /* partition.cuh:12 */
#define SGC_MAX_HISTOGRAM_COLORS_DEFAULT 1024u  /* partition.cuh:6-9 */
#define SGC_CSR_EXTRA_SLACK_PCT_DEFAULT 300u    /* streamgc.cu:169-171 */
#define SGC_HOST_BATCH_SIZE       32768u        /* streamgc.cu:785 */
#define SGC_BITMAP_COLORS         64u           /* color_select.cuh:5-8 */

/* default_config() of streamgc.cuh:124-135. */
static inline StreamGCConfig sgc_default_config(void) {
    StreamGCConfig c;
    c.num_gpus = 1;
    c.num_vertices = 0;
    c.num_edges = 0;
    c.stream_buffer_size = 1u << 20;
    c.epoch_size = SGC_EPOCH_SIZE_DEFAULT;
    c.priority_refresh_interval = SGC_PRIORITY_REFRESH_DEFAULT;
    c.histogram_threshold = SGC_HISTOGRAM_THRESHOLD_DEFAULT;
    c.rebalance_threshold = SGC_REBALANCE_DEFAULT;
    return c;
}

/* pack_state / unpack_* of vertex_state.cuh:17-27. */
static inline uint32_t sgc_pack_state(uint16_t color, uint16_t version) {
    return ((uint32_t)version << 16) | (uint32_t)color;
}
static inline uint16_t sgc_unpack_color(uint32_t packed) { return (uint16_t)(packed & 0xFFFFu); }
static inline uint16_t sgc_unpack_version(uint32_t packed) { return (uint16_t)(packed >> 16); }

/* compute_priority of priority.cuh:8-10: higher value keeps its color. */
static inline uint64_t sgc_compute_priority(uint32_t init_degree, uint32_t vertex_id) {
    return ((uint64_t)init_degree << 32) | (uint64_t)vertex_id;
}

#ifdef __cplusplus
} /* extern "C" */

static_assert(sizeof(EdgeUpdate) == 16 && offsetof(EdgeUpdate, type) == 8, "EdgeUpdate layout");
static_assert(sizeof(VertexState) == 4 && alignof(VertexState) == 4, "VertexState layout");
static_assert(sizeof(StreamGCConfig) == 40 && offsetof(StreamGCConfig, num_edges) == 8 &&
              offsetof(StreamGCConfig, histogram_threshold) == 28, "StreamGCConfig layout");
static_assert(sizeof(GPUPartition) == 304, "GPUPartition size");
static_assert(offsetof(GPUPartition, index_map_size) == 48 && offsetof(GPUPartition, neighbor_bitmap) == 56 &&
              offsetof(GPUPartition, num_high_degree) == 80 && offsetof(GPUPartition, init_priority) == 88 &&
              offsetof(GPUPartition, row_ptr) == 104 && offsetof(GPUPartition, col_idx) == 112 &&
              offsetof(GPUPartition, ghost_row_ptr) == 128 && offsetof(GPUPartition, stream_mask) == 176 &&
              offsetof(GPUPartition, overflow_local) == 216 && offsetof(GPUPartition, overflow_local_count) == 232 &&
              offsetof(GPUPartition, num_owned) == 248 && offsetof(GPUPartition, gpu_id) == 268 &&
              offsetof(GPUPartition, phi_inflight) == 272 && offsetof(GPUPartition, phi_dirty) == 296,
              "GPUPartition field offsets");
#endif

#endif /* STREAMGC_TYPES_H */
