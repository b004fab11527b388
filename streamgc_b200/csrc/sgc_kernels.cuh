// sgc_kernels.cuh -- kernel declarations and launch helpers of the handle API.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "sgc_device.cuh"

namespace sgc {

constexpr uint32_t SWEEP_CH = 512;       // default slots per warp work item in a sweep (repair tile width)
constexpr uint32_t SWEEP_CH_MIN = 256;   // smallest tile width (sizes the item list)
constexpr uint32_t SWEEP_TINY = 64;      // rows this short are swept by one thread (16-slot vector chunks)
constexpr uint32_t NONE32 = 0xFFFFFFFFu;
constexpr unsigned long long EMPTY64 = 0xFFFFFFFFFFFFFFFFull;

// Loop state of one repair, on the device (written by repair_begin_kernel and
// repair_step_kernel; fields marked host are set by the host before a repair).
struct RepairCtl {
    uint32_t mode;         // host: SWEEP_TIER1 or SWEEP_INDEP
    uint32_t max_sweeps;   // host
    uint32_t force_all;    // host: 1 = every graph is repaired in full
    uint32_t any_sym;      // some graph computes its mirror checksum in the first sweep
    uint32_t incr;         // some graph starts from its touched vertices only
    uint32_t list;         // the current sweep visits b.wl (else every vertex)
    uint32_t it;           // index of the current sweep
    uint32_t cont;         // another sweep runs
    uint32_t done;         // the last sweep left nothing to do
    uint32_t need;         // conflicted vertices counted by the last sweep
    uint32_t next;         // size of the next worklist
    uint32_t prev;         // reference rule: last count
    uint32_t plateau;      // reference rule: equal counts in a row
    uint32_t pad[3];
    unsigned long long sym;   // nonzero: some graph's first-sweep checksum was not 0
    unsigned long long live;  // first sweep's live entries
};

// Per-sweep work state: warp items for rows longer than SWEEP_TINY, per-vertex
// accumulators, the Jacobi pending list and the FAC work list.
struct SweepBufs {
    unsigned long long* items;   // x | chunk << 32
    uint32_t* item_count;
    uint32_t item_cap;
    uint32_t tile;               // slots per item (repair tile width, >= SWEEP_CH_MIN)
    uint32_t G;                  // graphs of the handle (entries of g.gctl)
    RepairCtl* rc;
    unsigned long long* acc_bm;  // OR of neighbor colors 1..64, per vertex
    uint32_t* acc_fl;            // bit0: a same-colored neighbor has higher priority
    uint32_t* pend_v;            // Jacobi commit list
    uint32_t* pend_w;
    uint32_t* pend_count;
    uint32_t* fac_v;             // vertices whose new color needs a warp (histogram or >64 scan)
    uint32_t* fac_count;
    unsigned long long* live;    // live entries seen by the sweep
    // worklist of the next sweep: vertices recolored by the last one and their neighbors
    uint32_t* wmark;             // bitmask
    uint32_t* wl;
    uint32_t* wl_count;
    unsigned long long* swept;   // [0] live entries, [1] vertices visited by the sweeps since reset
    // independent-set sweeps: conflicted vertices of the current sweep
    uint8_t* needf;              // per vertex: conflicted (or uncolored with neighbors) at the last visit
    uint32_t* need_v;
    uint32_t* need_count;
    uint32_t* rbits;             // bitmask: recolored by the last sweep (cleared with the worklist)
    uint32_t* hiused;            // exact selection: 64 words per histogram-class row, colors 64..2047
                                 // taken by its neighbors (filled and cleared within one sweep)
};

// Selection order of the independent-set rule: a 32-bit mix of (x, salt) with
// the id as tie-break. The mixer is the "lowbias32" function published in C.
// Wellons' hash-prospector; the salt changes with every sweep.
__host__ __device__ __forceinline__ unsigned long long sel_rank(uint32_t x, uint32_t salt) {
    uint32_t h = x ^ salt;
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return ((unsigned long long)h << 32) | x;
}
__host__ __device__ __forceinline__ uint32_t sweep_salt(uint32_t sweep) { return (sweep + 1u) * 0x9E3779B9u; }

// Same-edge ordering for a concurrently applied batch.
struct EdgeOrder {
    unsigned long long* tkey;  // open-addressed edge keys
    uint32_t* thead;           // per key: last update index pushed
    uint32_t* tslot;           // per update: its key slot (NONE32 = not an edge op)
    uint32_t* tnext;           // per update: next in the key's push list
    uint32_t* tprev;           // per update: previous update of the same edge (stream order)
    uint32_t* tsucc;           // per update: next update of the same edge (stream order)
    uint32_t* ticket;          // work ticket of the persistent apply kernel
    uint32_t tmask;            // table size - 1
};

// REBUILD: bitmaps only. TIER1: the reference rule (every conflicted vertex
// recolors from start-of-sweep state). INDEP: a conflicted vertex recolors only
// when no conflicted neighbor ranks above it (sel_rank of this sweep), so
// recolored vertices are never adjacent and a sweep creates no conflict.
enum SweepMode : int { SWEEP_REBUILD = 0, SWEEP_TIER1 = 1, SWEEP_INDEP = 2 };

// ---- launchers (sgc_kernels.cu) ----
void launch_det_apply(const Dev& g, const EdgeUpdate* ups, uint32_t n, cudaStream_t s);
void launch_ring_gather(const EdgeUpdate* ring, uint64_t mask, uint64_t head, uint32_t n, EdgeUpdate* out,
                        int num_sms, cudaStream_t s);
void launch_add_check(const Dev& g, const EdgeUpdate* ups, uint32_t n, const uint32_t* dyn, int num_sms,
                      cudaStream_t s);
void launch_conc_apply(const Dev& g, const EdgeUpdate* ups, uint32_t n, const EdgeOrder& eo, int num_sms,
                       cudaStream_t s);
// The same with the batch size read from the device word dyn[0] (replayable
// in a CUDA graph); fixed grids. blocks_per_sm <= 0:
// as many resident apply blocks as fit.
void launch_conc_apply_dyn(const Dev& g, const EdgeUpdate* ups, const uint32_t* dyn, const EdgeOrder& eo,
                           int num_sms, int blocks_per_sm, cudaStream_t s);
int conc_apply_occupancy();
// One warp per segment [segs[k], segs[k+1]), k < dyn[2]: each segment in stream order.
void launch_seg_apply(const Dev& g, const EdgeUpdate* ups, const uint32_t* segs, const uint32_t* dyn, uint32_t max_segs,
                      int num_sms, cudaStream_t s);
void launch_dirty_list(const Dev& g, uint32_t* list, uint32_t* count, cudaStream_t s);
// force: compact every listed row (else rows whose holes fill at most a quarter
// of their extent wait, under exact selection).
void launch_compact(const Dev& g, const uint32_t* list, const uint32_t* count, uint32_t max_rows, bool force,
                    cudaStream_t s, bool merge = false);
void launch_take_overflow(const Dev& g, uint32_t* drain_n, cudaStream_t s);
void launch_drain(const Dev& g, const uint32_t* drain_n, bool ordered, unsigned long long* failed, cudaStream_t s);
void launch_snapshot(const Dev& g, uint16_t* snap, cudaStream_t s);
// list_mode 0: every vertex; 1: the vertices in b.wl; 2: as b.rc->list says.
void launch_build_items(const Dev& g, const SweepBufs& b, int list_mode, int num_sms, cudaStream_t s);
// sym_mode 0: no mirror checksum; 2: in the first sweep of a repair, each graph
// repaired in full with asym set accumulates its checksum (sum over entries
// x->y, y != x, y < n, of H(x,y) - H(y,x)) in its GraphCtl. The sweep index
// (the independent-set order's salt) comes from b.rc.
// `phase` (optional): events recorded after the long-row items and after the
// per-vertex finalize.
void launch_sweep(const Dev& g, const SweepBufs& b, SweepMode mode, int list_mode, int sym_mode, int num_sms,
                  cudaStream_t s, cudaEvent_t* phase = nullptr);
// After a sweep: b.wl = the next worklist (reference rule: the vertices the
// sweep recolored and their neighbors; independent-set rule: the blocked and
// pushed vertices). Reads the sweep's items: call before the next
// launch_build_items.
void launch_next_worklist(const Dev& g, const SweepBufs& b, int num_sms, cudaStream_t s);
// The device-driven repair loop: begin (b.rc host fields set), then per sweep
// launch_repair_sweep + launch_repair_step; b.rc->cont says whether another
// sweep runs. With `cond`, the step also sets that graph conditional.
void launch_repair_begin(const Dev& g, const SweepBufs& b, SweepMode mode, int num_sms, cudaStream_t s);
// `phase` (optional): three events, recorded after the item build, the
// long-row items and the per-vertex finalize.
void launch_repair_sweep(const Dev& g, const SweepBufs& b, SweepMode mode, int num_sms, cudaStream_t s,
                         cudaEvent_t* phase = nullptr);
void launch_repair_step(const Dev& g, const SweepBufs& b, int num_sms, cudaStream_t s,
                        const cudaGraphConditionalHandle* cond);
void launch_query(const uint16_t* snap, uint32_t n, const uint32_t* v, uint16_t* out, uint32_t k, cudaStream_t s);
void launch_color_list(const Dev& g, const uint32_t* list, uint32_t m, uint32_t* colored, cudaStream_t s);
void launch_snapshot_changes(const Dev& g, uint32_t* prev, uint16_t* snap, cudaStream_t s);
void launch_colors(const Dev& g, uint16_t* out, cudaStream_t s);

// Tier-2 (sgc_tier2.cu)
struct Tier2Bufs {
    uint8_t* inU;
    uint8_t* inF;
    uint8_t* inL;
    uint8_t* done;
    uint32_t* list;        // current ordered list
    uint32_t* list2;
    uint32_t* count;       // [0] list count, [1] list2 count, [2] fixed, [3] rev count, [4] selected
    unsigned long long* rev_keys;   // (y << 32) | x for entries x -> y with inL[y]
    unsigned long long* rev_keys2;
    uint32_t rev_cap;
    uint32_t* rev_start;   // per list position: first index into sorted rev keys
    uint32_t* rev_end;
    void* cub_tmp;
    size_t cub_tmp_bytes;
    uint32_t* pend_v;
    uint32_t* pend_w;
};
// Runs the reference's Tier-2 (streamgc.cu:1057-1240) exactly; returns fixes.
// Readers skip holes and deleted run entries. `masked`: only the rows of graphs
// whose GraphCtl.t2 is set (every other graph converged on mirror-complete
// rows, so Tier-2 would change nothing there).
// Vertices [lo, hi) that a Tier-2 pass visits (whole graphs); masked: only
// graphs whose GraphCtl.t2 is set.
struct Tier2Span {
    uint32_t lo, hi;
    int masked;
};
uint32_t run_tier2(const Dev& g, Tier2Bufs& b, cudaStream_t s, uint32_t* host_scratch, bool* gave_up,
                   uint64_t* launches, bool masked = false, uint32_t lo = 0, uint32_t hi = 0xFFFFFFFFu);
// [first vertex, end) of the graphs whose GraphCtl.t2 is set, into span[0..1]
// ({n, 0} when none); one block.
void launch_t2_span(const Dev& g, uint32_t G, uint32_t* span, cudaStream_t s);
size_t tier2_cub_bytes(uint32_t n, uint32_t rev_cap);

// Validator (sgc_tier2.cu): [violations, uncolored_with_edges, distinct_edges, max_color, out_of_range]
int run_validate(const Dev& g, cudaStream_t s, uint64_t* out);
// Layout invariants of every row: out = {rows breaking one, SGC_STATE_* bits
// seen, lowest such row (~0 if none)}.
int run_check_state(const Dev& g, cudaStream_t s, uint64_t* out);

}  // namespace sgc
