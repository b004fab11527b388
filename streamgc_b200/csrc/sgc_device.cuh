// sgc_device.cuh -- warp-cooperative device primitives of the streaming
// coloring path (sm_100a).
//
// Semantics follow the reference's single-GPU path operation for operation:
//   row insert / delete          algorithms/streamgc/src/kernels/local_update.cu:12-56
//   FindAvailableColor           algorithms/streamgc/include/color_select.cuh:10-115
//   neighbor bitmap / histogram  algorithms/streamgc/include/color_select.cuh:120-209
//   recolor / color reduction    algorithms/streamgc/src/kernels/recolor.cu:49-163
//   ADD / DEL sequence           algorithms/streamgc/src/kernels/local_update.cu:61-147
// What changes is how each step maps onto the hardware: a whole warp scans a
// row with 16-byte loads (128 slots per warp-load, 2 in flight per lane) and a
// ballot picks the first candidate slot; color selection over a 1024-bin
// histogram row is a warp-wide load + ballot + min-reduction; the neighbor
// walk after a recolor spreads its bitmap/histogram atomics over 32 lanes.
// The per-vertex (color, version) word only changes through atomicCAS, so the
// same code is exact when one warp applies updates in stream order and safe
// when many warps apply a batch concurrently.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/streamgc_types.h"

namespace sgc {

constexpr uint32_t INV = SGC_CSR_INVALID;
constexpr uint32_t EMPTY = SGC_HASH_EMPTY;
constexpr uint32_t FULL = 0xFFFFFFFFu;
constexpr uint32_t OVF_CAP = SGC_OVERFLOW_CAPACITY;
constexpr uint32_t TOMB = 0x80000000u;  // tombstone bit of a deleted base-run entry (exact selection)

// Error bits written to the handle's device error word.
enum : uint32_t {
    ERR_RESERVED0 = 1u << 0,      // not set (formerly a same-edge wait timeout)
    ERR_BAD_UPDATE = 1u << 1,     // update endpoint outside [0, n)
    ERR_LIST_OVERFLOW = 1u << 2,  // a work list exceeded its capacity
    ERR_CHAIN = 1u << 3,          // same-edge ordering words inconsistent with the batch (chain past
                                  // the batch, or an update whose prep record does not match it)
    ERR_RETRY = 1u << 4,          // a color compare-and-swap kept failing past its retry bound
    ERR_ROW = 1u << 5,            // a row's high-water mark lay past its capacity (scans clamped)
};

// Ablations of the reference rules (Dev::abl), as its abl-* builds.
enum : uint32_t {
    ABL_FORCE_BITMAP = 1u << 0,  // every color choice from the bitmap (color_select.cuh:98-100)
    ABL_NO_OVERFLOW = 1u << 1,   // a full row drops the insert (local_update.cu:28-38)
    ABL_LIVE_DEG = 1u << 2,      // Tier-1: own live degree vs neighbors' frozen priority (conflict_repair.cu:46-57)
};

// Repair flags of one graph of a handle.
struct GraphCtl {
    uint32_t clean;   // the last repair ended proper and only updates changed colors since
    uint32_t asym;    // an entry may have lost its mirror since the rows were last found
                      // mirror-complete (set at creation, on every overflow, on a drain
                      // failure, and when an update found one direction only)
    uint32_t force;   // host: the next repair visits every vertex of the graph
    uint32_t full;    // the current repair visits every vertex of the graph
    unsigned long long sym;  // mirror checksum of the current repair (full repairs with asym set)
    uint32_t base;    // first vertex of the graph in the handle (ids minus base are the graph's own)
    uint32_t t2;      // the last repair left this graph to Tier-2 (rows missing mirrors, or not converged)
    uint32_t dropped; // an entry of this graph was dropped (a full row at drain, or the overflow buffer full)
};

// A row-scale operation of a concurrent batch left to the pass after it
// (exact selection): HUB_REDUCE moves x to color `freed` when that is below
// x's color and no live neighbor of x holds it; HUB_RECOLOR moves x to its
// first free color. The pass re-reads x's state word.
enum : uint32_t { HUB_REDUCE = 1u, HUB_RECOLOR = 2u };
struct HubOp {
    uint32_t x;
    uint32_t op;  // kind << 16 | freed
};
// Live slots a warp scans itself before it leaves the rest of a row to the
// pass, and the row length from which it does (shorter rows finish in the
// warp within a few rounds, sooner than a pass after the batch would).
constexpr uint32_t kHubScan = 512;
constexpr uint32_t kHubRow = 8192;

// Device view of one graph's state (handle layout). Row x owns logical slots
// [rp[x], rp[x+1]); hw[x] bounds the slots ever written since the row was last
// compacted (every slot at or past rp[x]+hw[x] holds INV), so after compaction
// the row's live entries are exactly [rp[x], rp[x]+hw[x]).
struct Dev {
    uint32_t n;
    uint32_t maxc;                 // histogram colors per row (multiple of 4)
    uint32_t exact;                // 1: colors above the threshold are chosen from the live
                                   // neighbors (no global histogram rows are kept)
    uint32_t abl;                  // ablations of the reference rules (ABL_* bits)
    const uint64_t* rp;            // n+1 row starts (64-bit: slabs beyond 2^32 slots)
    uint32_t* col;                 // slots, padded so 16-byte loads never leave the allocation
    uint32_t* st;                  // packed (color | version << 16)
    uint64_t* bm;                  // neighbor color bitmaps
    const uint32_t* hdmap;         // vertex -> histogram row, EMPTY for bitmap mode
    uint32_t* hist;                // num_hd * maxc counters
    const uint32_t* deg;           // frozen initial degree: priority = (deg << 32) | id
    uint32_t* hw;                  // per-row high-water mark (slots, relative to rp[x])
    uint32_t* live;                // lazy compaction (exact mode): live entries inside [rp, rp+hw) (the row's
                                   // holes, free slots and tombstones, are hw minus this count); else null
    uint32_t* dirty;               // bitmask of rows edited since their last compaction
    uint32_t* edited;              // bitmask of rows edited since creation (clear = pristine:
                                   // base entries sorted ascending in [rp, rp+hw), INV after)
    OverflowEdge* ovf;             // OVF_CAP entries
    uint32_t* ovf_count;           // counts every overflow, stored or not
    unsigned long long* ovf_lost;  // overflows beyond OVF_CAP (edge dropped, as the reference does)
    unsigned long long* nskip;     // updates skipped: an endpoint outside [0, n) (hash miss)
    uint32_t* err;
    uint32_t* blen;                // exact selection: per row, length of the base run [rp, rp+blen):
                                   // ids strictly ascending, deleted ones kept as id | TOMB (null otherwise)
    uint32_t* touched;             // exact selection: bitmask of the vertices the next incremental repair
                                   // starts from (null otherwise): every vertex whose color changed, every
                                   // bitmap-class endpoint of an update (its bitmap is rebuilt), and both
                                   // endpoints of an ADD whose colors are equal at the end of its batch
    uint32_t* chg;                 // single-graph handles under exact selection: bitmask of the vertices
                                   // whose color changed since the last snapshot (null otherwise)
    HubOp* hub_ops;                // concurrent batches under exact selection: row-scale operations left
    uint32_t* hub_count;           // to the pass after the batch (null: none are deferred); the count
    uint32_t hub_cap;              // runs past hub_cap when the list is full (those are done in place)
    unsigned long long* hub_total; // cumulative count of the operations the pass took
    GraphCtl* gctl;                // per graph: repair flags (one entry for a single-graph handle)
    const uint32_t* gidw;          // graph of each 32-vertex word (graphs start at multiples of 32);
                                   // null: one graph
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint16_t color_of(uint32_t w) { return (uint16_t)(w & 0xFFFFu); }
__device__ __forceinline__ uint16_t version_of(uint32_t w) { return (uint16_t)(w >> 16); }
__device__ __forceinline__ uint32_t pack(uint16_t c, uint16_t v) { return ((uint32_t)v << 16) | c; }

// priority(a) < priority(b) for priority = (deg << 32) | id (priority.cuh:8-23)
__device__ __forceinline__ bool prio_less(uint32_t da, uint32_t a, uint32_t db, uint32_t b) {
    return (da < db) || (da == db && a < b);
}

// Coherent (L1-bypassing) loads for words other warps may be changing.
__device__ __forceinline__ uint32_t ld_cg(const uint32_t* p) { return __ldcg(p); }
__device__ __forceinline__ uint64_t ld_cg(const uint64_t* p) { return __ldcg((const unsigned long long*)p); }
__device__ __forceinline__ uint4 ld_cg4(const uint32_t* p) { return __ldcg(reinterpret_cast<const uint4*>(p)); }

__device__ __forceinline__ uint32_t pick4(const uint4& q, int k) {
    return k == 0 ? q.x : (k == 1 ? q.y : (k == 2 ? q.z : q.w));
}

// Bit k of the result is set when slot i+k lies in [s, e) and pred(slot).
template <class P>
__device__ __forceinline__ uint32_t mask4(const uint4& q, uint64_t i, uint64_t s, uint64_t e, P pred) {
    uint32_t m = 0;
    m |= (i + 0 >= s && i + 0 < e && pred(q.x)) ? 1u : 0u;
    m |= (i + 1 >= s && i + 1 < e && pred(q.y)) ? 2u : 0u;
    m |= (i + 2 >= s && i + 2 < e && pred(q.z)) ? 4u : 0u;
    m |= (i + 3 >= s && i + 3 < e && pred(q.w)) ? 8u : 0u;
    return m;
}

// A lane group: the whole warp (W = 32) or one half of it (W = 16, lanes
// [base, base + 16)). Votes and shuffles stay inside the group, so the two
// halves of a warp can edit two different rows at once; every branch the
// group takes depends only on the group's own votes and shuffles.
template <int W>
struct Lanes {
    static_assert(W == 32 || W == 16, "a warp or half a warp");
    uint32_t base, lane, mask;
    __device__ __forceinline__ Lanes() {
        const uint32_t l = lane_id();
        base = W == 32 ? 0u : (l & 16u);
        lane = l - base;
        mask = W == 32 ? FULL : (0xFFFFu << base);
    }
    __device__ __forceinline__ bool leader() const { return lane == 0; }
    // bit k: the group's lane k
    __device__ __forceinline__ uint32_t ballot(bool p) const { return (__ballot_sync(mask, p) & mask) >> base; }
    template <class T>
    __device__ __forceinline__ T shfl(T v, int src) const { return __shfl_sync(mask, v, src, W); }
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
};

// Group-collective: first slot index p in [s, e) whose value satisfies pred,
// scanning in slot order exactly like the reference's serial loop. Loads are
// 16-byte aligned (col must be 16-byte aligned and padded past the last row
// to a multiple of 4 slots). Returns false when no slot matches.
template <int W, class P>
__device__ __forceinline__ bool grp_find(const Lanes<W>& L, const uint32_t* col, uint64_t s, uint64_t e, P pred,
                                         uint64_t& pos, uint32_t& val) {
    constexpr uint64_t R = 4ull * W;  // slots per group-wide 16-byte load
    for (uint64_t c = s & ~3ull; c < e; c += 4 * R) {  // four 16-byte loads per lane in flight
        uint4 q[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint64_t i = c + R * k + 4ull * L.lane;
            q[k] = make_uint4(INV, INV, INV, INV);
            if (i < e) q[k] = ld_cg4(col + i);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint64_t i = c + R * k + 4ull * L.lane;
            const uint32_t m = mask4(q[k], i, s, e, pred);
            const uint32_t b = L.ballot(m != 0);
            if (b) {
                const int src = __ffs(b) - 1;
                const int kk = __ffs(m) - 1;
                const uint32_t v = m ? pick4(q[k], kk) : 0u;
                const int ks = L.shfl(kk, src);
                val = L.shfl(v, src);
                pos = c + R * k + 4ull * src + ks;
                return true;
            }
        }
    }
    return false;
}
template <class P>
__device__ __forceinline__ bool warp_find(const uint32_t* col, uint64_t s, uint64_t e, P pred,
                                          uint64_t& pos, uint32_t& val) {
    return grp_find(Lanes<32>(), col, s, e, pred, pos, val);
}

// Warp-collective visit of every slot in [s, e): f(slot_index, value) runs on
// the lane that loaded the slot (each slot once).
template <class F>
__device__ __forceinline__ void warp_for_each(const uint32_t* col, uint64_t s, uint64_t e, F f) {
    const uint32_t lane = lane_id();
    for (uint64_t c = s & ~3ull; c < e; c += 512) {  // four 16-byte loads per lane in flight
        uint4 q[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint64_t i = c + 128ull * k + 4ull * lane;
            q[k] = make_uint4(INV, INV, INV, INV);
            if (i < e) q[k] = ld_cg4(col + i);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint64_t i = c + 128ull * k + 4ull * lane;
            if (i < e) {
                if (i + 0 >= s) f(i + 0, q[k].x);
                if (i + 1 >= s && i + 1 < e) f(i + 1, q[k].y);
                if (i + 2 >= s && i + 2 < e) f(i + 2, q[k].z);
                if (i + 3 >= s && i + 3 < e) f(i + 3, q[k].w);
            }
        }
    }
}

// Warp-collective visit of every slot of [s, e) holding a vertex id y < n,
// with arr[y] (a coherent load): a lane issues the loads of its 4K slots and
// their 4K gathers before it uses any of them (K 16-byte loads per lane per
// round). f(y, arr[y]) runs once per slot. With STOP, the scan ends after the
// first round in which f returned true on any lane (warp vote); the return
// value says whether that happened.
template <bool STOP, int K = 4, class F>
__device__ __forceinline__ bool warp_gather_each(const uint32_t* col, uint64_t s, uint64_t e, uint32_t n,
                                                 const uint32_t* arr, F f) {
    const uint32_t lane = lane_id();
    for (uint64_t c = s & ~3ull; c < e; c += 128 * K) {
        uint32_t y[4 * K], w[4 * K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const uint64_t i = c + 128ull * k + 4ull * lane;
            uint4 q = make_uint4(INV, INV, INV, INV);
            if (i < e) q = ld_cg4(col + i);
            y[4 * k + 0] = (i + 0 >= s && i + 0 < e) ? q.x : INV;
            y[4 * k + 1] = (i + 1 >= s && i + 1 < e) ? q.y : INV;
            y[4 * k + 2] = (i + 2 >= s && i + 2 < e) ? q.z : INV;
            y[4 * k + 3] = (i + 3 >= s && i + 3 < e) ? q.w : INV;
        }
#pragma unroll
        for (int t = 0; t < 4 * K; t++) w[t] = y[t] < n ? ld_cg(arr + y[t]) : 0u;
        bool hit = false;
#pragma unroll
        for (int t = 0; t < 4 * K; t++)
            if (y[t] < n) hit |= f(y[t], w[t]);
        if (STOP && __any_sync(FULL, hit)) return true;
    }
    return false;
}

// Marks are fire-and-forget reductions (their results unused): the warp does
// not wait for them on the update path.
__device__ __forceinline__ void mark_dirty(const Dev& g, uint32_t x) {
    atomicOr(g.dirty + (x >> 5), 1u << (x & 31));
    atomicOr(g.edited + (x >> 5), 1u << (x & 31));
}
__device__ __forceinline__ uint32_t graph_of(const Dev& g, uint32_t x) { return g.gidw ? __ldg(g.gidw + (x >> 5)) : 0u; }
// Row x's high-water mark, at most the row's capacity. The mark never
// exceeds it; the clamp keeps every scan and every compaction write inside the
// row whatever the word holds (sgc_check_state reports such a row).
__device__ __forceinline__ uint32_t row_len(const Dev& g, uint32_t x) {
    const uint32_t hw = g.hw[x];
    const uint64_t cap = g.rp[x + 1] - g.rp[x];
    return hw <= cap ? hw : (uint32_t)cap;
}

// End of the slots of row x that scans visit, [s, s + hw), clamped to the
// row's capacity (a larger mark sets ERR_ROW).
__device__ __forceinline__ uint64_t live_end(const Dev& g, uint32_t x, uint64_t s) {
    const uint64_t e = s + ld_cg(g.hw + x), cap = g.rp[x + 1];
    if (e <= cap) return e;
    if ((lane_id() & 15u) == 0) atomicOr(g.err, ERR_ROW);  // the first lane of each half-warp group
    return cap;
}

// Row x got an entry in slot q (relative to rp[x]): raise the high-water
// mark and count the entry live. Both are reductions the warp does not wait
// for, and they commute with every other row edit of the batch, so once the
// batch's edits have landed the mark minus the live count is exactly the
// row's free slots and tombstones inside the mark.
__device__ __forceinline__ void extend_row(const Dev& g, uint32_t x, uint32_t q) {
    atomicMax(g.hw + x, q + 1);
    if (g.live) atomicAdd(g.live + x, 1u);
}
// Holes of row x (free slots and tombstones inside the mark `hw`).
__device__ __forceinline__ uint32_t row_holes(const Dev& g, uint32_t x, uint32_t hw) {
    const uint32_t lv = g.live[x];
    return hw > lv ? hw - lv : 0u;
}

__device__ __forceinline__ void mark_touched(const Dev& g, uint32_t x) {
    if (g.touched) atomicOr(g.touched + (x >> 5), 1u << (x & 31));
}
// Every write of a state word notes the vertex for the next incremental snapshot.
__device__ __forceinline__ void note_color(const Dev& g, uint32_t x) {
    if (g.chg) atomicOr(g.chg + (x >> 5), 1u << (x & 31));
}

__device__ __forceinline__ void flag_asym(const Dev& g, uint32_t x) {
    uint32_t* a = &g.gctl[graph_of(g, x)].asym;
    if (!ld_cg(a)) atomicOr(a, 1u);
}
__device__ __forceinline__ bool pristine(const Dev& g, uint32_t x) {
    return !(ld_cg(g.edited + (x >> 5)) & (1u << (x & 31)));
}

// Group-collective W-ary search for `key` in the ascending run col[s, e):
// each round probes W evenly spaced slots and keeps the bucket holding the
// last probe <= key. Returns the slot index, or ~0 when key is absent.
template <int W>
__device__ __forceinline__ uint64_t grp_bsearch(const Lanes<W>& L, const uint32_t* col, uint64_t s, uint64_t e,
                                                uint32_t key) {
    uint64_t lo = s, hi = e;
    while (hi - lo > W) {
        const uint64_t step = (hi - lo) / W;
        const uint32_t v = ld_cg(col + lo + L.lane * step);
        const uint32_t b = L.ballot(v <= key);
        if (!b) return ~0ull;
        const uint32_t top = 31 - __clz(b);
        const uint64_t nlo = lo + top * step;
        hi = (top == W - 1) ? hi : nlo + step;
        lo = nlo;
    }
    const uint64_t i = lo + L.lane;
    const bool hit = i < hi && ld_cg(col + i) == key;
    const uint32_t b = L.ballot(hit);
    return b ? lo + (__ffs(b) - 1) : ~0ull;
}

// W-ary search by id in a base run (ascending ids, tombstones keep their id
// under TOMB). Returns the slot index, or ~0 when the id is absent; `val` gets
// the slot's value (the id, or id | TOMB).
template <int W>
__device__ __forceinline__ uint64_t grp_bsearch_key(const Lanes<W>& L, const uint32_t* col, uint64_t s, uint64_t e,
                                                    uint32_t key, uint32_t& val) {
    uint64_t lo = s, hi = e;
    while (hi - lo > W) {
        const uint64_t step = (hi - lo) / W;
        const uint32_t v = ld_cg(col + lo + L.lane * step) & ~TOMB;
        const uint32_t b = L.ballot(v <= key);
        if (!b) return ~0ull;
        const uint32_t top = 31 - __clz(b);
        const uint64_t nlo = lo + top * step;
        hi = (top == W - 1) ? hi : nlo + step;
        lo = nlo;
    }
    const uint64_t i = lo + L.lane;
    const uint32_t v = i < hi ? ld_cg(col + i) : INV;
    const uint32_t b = L.ballot(i < hi && (v & ~TOMB) == key);
    if (!b) return ~0ull;
    val = L.shfl(v, __ffs(b) - 1);
    return lo + (__ffs(b) - 1);
}

// ---------------- slack-CSR row edits (local_update.cu:12-56) ----------------

enum { ADD_INSERTED = 0, ADD_PRESENT = 1, ADD_OVERFLOW = 2 };

// Concurrent batches under exact selection: rows keep their base run sorted
// (a delete there leaves a tombstone, a re-insert of the same id revives it),
// so an update finds a base entry by a W-ary search; only entries inserted
// since the row's last compaction (its tail) are scanned. The updates of one
// edge are ordered, so no other warp touches the slot of `nbr` meanwhile.
// Add: returns ADD_PRESENT / ADD_INSERTED when the run holds nbr (live or
// tombstone), -1 when it does not.
template <int W>
__device__ __forceinline__ int grp_run_add(const Lanes<W>& L, const Dev& g, uint32_t x, uint32_t nbr, uint64_t s,
                                           uint32_t bl) {
    uint32_t val = 0;
    const uint64_t p = grp_bsearch_key(L, g.col, s, s + bl, nbr, val);
    if (p == ~0ull) return -1;
    if (val == nbr) return ADD_PRESENT;
    uint32_t old = 0;
    if (L.leader()) {
        old = atomicCAS(g.col + p, nbr | TOMB, nbr);
        if (old == (nbr | TOMB)) {
            atomicAdd(g.live + x, 1u);
            mark_dirty(g, x);
        }
    }
    old = L.shfl(old, 0);
    return old == nbr ? ADD_PRESENT : ADD_INSERTED;
}
__device__ __forceinline__ int warp_run_add(const Dev& g, uint32_t x, uint32_t nbr, uint64_t s, uint32_t bl) {
    return grp_run_add(Lanes<32>(), g, x, nbr, s, bl);
}
// Delete: true when the run held nbr live (now a tombstone).
template <int W>
__device__ __forceinline__ bool grp_run_remove(const Lanes<W>& L, const Dev& g, uint32_t x, uint32_t nbr, uint64_t s,
                                               uint32_t bl) {
    uint32_t val = 0;
    const uint64_t p = grp_bsearch_key(L, g.col, s, s + bl, nbr, val);
    if (p == ~0ull || val != nbr) return false;
    uint32_t old = 0;
    if (L.leader()) {
        old = atomicCAS(g.col + p, nbr, nbr | TOMB);
        if (old == nbr) {
            atomicSub(g.live + x, 1u);
            mark_dirty(g, x);
        }
    }
    old = L.shfl(old, 0);
    return old == nbr;
}

// add_local_neighbor: claim the first INV slot unless `nbr` shows up first;
// a full row appends to the overflow buffer (counter always advances, entry
// stored only below capacity). The row's bounds, base run and high-water
// mark are read together up front (a mark read early is only lower: the
// fallback scan to the row's end covers what it misses).
template <int W>
__device__ __forceinline__ int grp_add_slot(const Lanes<W>& L, const Dev& g, uint32_t x, uint32_t nbr, bool exact) {
    const uint64_t s = g.rp[x], e = g.rp[x + 1];
    const uint32_t bl = (!exact && g.blen) ? ld_cg(g.blen + x) : 0u;
    const uint32_t hw0 = ld_cg(g.hw + x);
    uint64_t from = s;
    if (!exact && g.blen) {
        if (bl) {
            const int r = grp_run_add(L, g, x, nbr, s, bl);
            if (r >= 0) return r;
        }
        from = s + bl;  // the tail: first INV or nbr
    } else if (pristine(g, x)) {
        // Sorted base entries, no holes: the scan would stop at nbr if present,
        // else at the first INV right after the base run.
        const uint64_t len = live_end(g, x, s) - s;
        if (grp_bsearch(L, g.col, s, s + len, nbr) != ~0ull) return ADD_PRESENT;
        // Past the sorted run: in stream order nothing else changes the row; in
        // a concurrent batch the updates of this edge are ordered, so nbr can
        // only be in the row through an earlier update of the edge, and that
        // one would have marked the row edited.
        from = s + len;
    }
    // The first free slot at or after `from` lies at or below the high-water
    // mark, so the first scan stops one slot past it (not at the end of the
    // row's slack); if a concurrent insert took those slots meanwhile, the
    // scan goes on to the end of the row.
    uint64_t lim = s + hw0 + 1;
    if (lim > e) lim = e;
    for (;;) {
        uint64_t p = 0;
        uint32_t v = 0;
        const bool hit =
            from < lim && grp_find(L, g.col, from, lim, [nbr](uint32_t t) { return t == INV || t == nbr; }, p, v);
        if (!hit && lim < e) {
            if (lim > from) from = lim;
            lim = e;
            continue;
        }
        if (!hit) {
            if (L.leader() && (g.abl & ABL_NO_OVERFLOW)) {  // the ablation drops the edge
                g.gctl[graph_of(g, x)].dropped = 1u;
                flag_asym(g, x);
            } else if (L.leader()) {
                const uint32_t pos = atomicAdd(g.ovf_count, 1u);
                if (pos < OVF_CAP) {
                    g.ovf[pos].local_vertex_idx = x;
                    g.ovf[pos].neighbor_global = nbr;
                } else {
                    atomicAdd(g.ovf_lost, 1ull);
                    g.gctl[graph_of(g, x)].dropped = 1u;
                }
                flag_asym(g, x);
            }
            L.sync();
            return ADD_OVERFLOW;
        }
        if (v == nbr) return ADD_PRESENT;
        uint32_t old = 0;
        if (L.leader()) {
            old = atomicCAS(g.col + p, INV, nbr);
            if (old == INV) {
                extend_row(g, x, (uint32_t)(p - s));
                mark_dirty(g, x);
            }
        }
        old = L.shfl(old, 0);
        if (old == INV) return ADD_INSERTED;
        if (old == nbr) return ADD_PRESENT;
        from = p + 1;  // lost the slot to a concurrent insert: keep scanning after it
    }
}
__device__ __forceinline__ int warp_add_slot(const Dev& g, uint32_t x, uint32_t nbr, bool exact) {
    return grp_add_slot(Lanes<32>(), g, x, nbr, exact);
}

// remove_local_neighbor: first slot equal to nbr becomes INV (lazy delete).
// Returns whether an entry was removed.
template <int W>
__device__ __forceinline__ bool grp_remove_slot(const Lanes<W>& L, const Dev& g, uint32_t x, uint32_t nbr,
                                                bool exact) {
    const uint64_t s = g.rp[x];
    const uint32_t bl = (!exact && g.blen) ? ld_cg(g.blen + x) : 0u;
    const uint64_t e = live_end(g, x, s);
    uint64_t from = s;
    if (!exact && g.blen) {
        if (bl && grp_run_remove(L, g, x, nbr, s, bl)) return true;
        from = s + bl;  // not live in the run: the tail
    } else if (pristine(g, x)) {
        const uint64_t p = grp_bsearch(L, g.col, s, e, nbr);
        if (p != ~0ull) {
            uint32_t old = 0;
            if (L.leader()) {
                old = atomicCAS(g.col + p, nbr, INV);
                if (old == nbr) {
                    mark_dirty(g, x);
                    if (g.live) atomicSub(g.live + x, 1u);
                    if (g.blen) g.blen[x] = 0;  // an INV inside the run ends it
                }
            }
            old = L.shfl(old, 0);
            if (old == nbr) return true;
        } else if (exact) {
            return false;  // absent from the sorted run and nothing after it
        }
    }
    for (;;) {
        uint64_t p = 0;
        uint32_t v = 0;
        if (!grp_find(L, g.col, from, e, [nbr](uint32_t t) { return t == nbr; }, p, v)) return false;
        uint32_t old = 0;
        if (L.leader()) {
            old = atomicCAS(g.col + p, nbr, INV);
            if (old == nbr) {
                mark_dirty(g, x);
                if (g.live) atomicSub(g.live + x, 1u);
                if (g.blen && p < s + ld_cg(g.blen + x)) g.blen[x] = 0;  // an INV inside the run ends it
            }
        }
        old = L.shfl(old, 0);
        if (old == nbr) return true;
        from = p + 1;
    }
}
__device__ __forceinline__ bool warp_remove_slot(const Dev& g, uint32_t x, uint32_t nbr, bool exact) {
    return grp_remove_slot(Lanes<32>(), g, x, nbr, exact);
}

// ---------------- color selection (color_select.cuh:10-115) ----------------

// Sets color c's bit (colors 1..64) in a 64-bit mask kept as two 32-bit words;
// c == 0 and c > 64 wrap out of both ranges.
__device__ __forceinline__ void add_color_bit(uint32_t c, uint32_t& lo, uint32_t& hi) {
    const uint32_t a = c - 1u, b = c - 33u;
    lo |= a < 32u ? 1u << a : 0u;
    hi |= b < 32u ? 1u << b : 0u;
}



// Histogram mode: first zero counter -> its color; else the first minimum.
// Whole row (maxc counters) is loaded warp-wide, 16 bytes per lane per step.
__device__ __forceinline__ uint16_t warp_fac_hist(const uint32_t* h, uint32_t maxc) {
    const uint32_t lane = lane_id();
    uint32_t best_v = FULL, best_i = FULL;  // lane-local first minimum
    for (uint32_t base = 0; base < maxc; base += 128) {
        const uint32_t i = base + 4 * lane;
        uint4 q = make_uint4(FULL, FULL, FULL, FULL);
        const bool ok = i < maxc;
        if (ok) q = ld_cg4(h + i);
        uint32_t zm = 0;
        if (ok) zm = (q.x == 0 ? 1u : 0u) | (q.y == 0 ? 2u : 0u) | (q.z == 0 ? 4u : 0u) | (q.w == 0 ? 8u : 0u);
        const uint32_t bz = __ballot_sync(FULL, zm != 0);
        if (bz) {
            const int src = __ffs(bz) - 1;
            const int k = __shfl_sync(FULL, __ffs(zm) - 1, src);
            return (uint16_t)(base + 4 * src + k + 1);
        }
        if (ok) {
            if (q.x < best_v) { best_v = q.x; best_i = i; }
            if (q.y < best_v) { best_v = q.y; best_i = i + 1; }
            if (q.z < best_v) { best_v = q.z; best_i = i + 2; }
            if (q.w < best_v) { best_v = q.w; best_i = i + 3; }
        }
    }
    // First minimum over the whole row: smallest value, ties to the smallest index.
    for (int off = 16; off > 0; off >>= 1) {
        const uint32_t ov = __shfl_xor_sync(FULL, best_v, off);
        const uint32_t oi = __shfl_xor_sync(FULL, best_i, off);
        if (ov < best_v || (ov == best_v && oi < best_i)) { best_v = ov; best_i = oi; }
    }
    return (uint16_t)(best_i + 1);
}

// Bitmap mode fallback when all 64 bits are set: first color in 1..255 no live
// neighbor holds (reading neighbor colors from `cols`), else 256.
__device__ __forceinline__ uint16_t warp_fac_scan(const Dev& g, uint32_t x, const uint32_t* cols) {
    const uint64_t s = g.rp[x], e = live_end(g, x, s);
    uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    warp_gather_each<false>(g.col, s, e, g.n, cols, [&](uint32_t, uint32_t sw) {
        const uint16_t c = color_of(sw);
        if (c > 0 && c < 256) {
#pragma unroll
            for (int k = 0; k < 8; k++)
                if ((c >> 5) == k) w[k] |= 1u << (c & 31);
        }
        return false;
    });
#pragma unroll
    for (int k = 0; k < 8; k++) w[k] = __reduce_or_sync(FULL, w[k]);
    w[0] |= 1u;  // color 0 is never a candidate
#pragma unroll
    for (int k = 0; k < 8; k++)
        if (~w[k]) return (uint16_t)(k * 32 + __ffs(~w[k]) - 1);
    return 256;
}

// Exact selection above the threshold: the first color no live neighbor holds.
// Colors 1..64 collect in a 64-bit lane mask, higher ones (up to 2047) in a
// 2048-bit set the warp fills in shared memory while it scans the row (the
// calling kernels run at most 8 warps per block).
__device__ __forceinline__ uint16_t warp_fac_exact(const Dev& g, uint32_t x, const uint32_t* cols) {
    __shared__ uint32_t s_used[8][64];
    uint32_t* used = s_used[(threadIdx.x >> 5) & 7];
    const uint32_t lane = lane_id();
    used[lane] = 0;
    used[lane + 32] = 0;
    __syncwarp();
    uint32_t lo = 0, hi = 0;
    const uint64_t s = g.rp[x], e = live_end(g, x, s);
    warp_gather_each<false>(g.col, s, e, g.n, cols, [&](uint32_t, uint32_t sw) {
        const uint16_t c = color_of(sw);
        add_color_bit(c, lo, hi);
        if (c > 64 && c < 2048) atomicOr(&used[c >> 5], 1u << (c & 31));
        return false;
    });
    lo = __reduce_or_sync(FULL, lo);
    hi = __reduce_or_sync(FULL, hi);
    const unsigned long long m = ((unsigned long long)hi << 32) | lo;
    __syncwarp();
    if (~m) return (uint16_t)__ffsll((long long)~m);
    uint32_t w0 = ~used[lane], w1 = ~used[lane + 32];
    if (lane < 2) w0 = 0;  // words 0-1 hold colors 0..64: settled by the lane masks
    if (lane == 2) w0 &= ~1u;  // color 64 sits in bit 0 of word 2 and is taken (mask was full)
    const uint32_t b0 = __ballot_sync(FULL, w0 != 0);
    if (b0) {
        const int src = __ffs(b0) - 1;
        return (uint16_t)(src * 32 + __shfl_sync(FULL, __ffs(w0) - 1, src));
    }
    const uint32_t b1 = __ballot_sync(FULL, w1 != 0);
    if (b1) {
        const int src = __ffs(b1) - 1;
        return (uint16_t)(1024 + src * 32 + __shfl_sync(FULL, __ffs(w1) - 1, src));
    }
    return 2048;
}

// FindAvailableColor: histogram row when the vertex has one, else bitmap.
__device__ __forceinline__ uint16_t warp_fac(const Dev& g, uint32_t x, const uint32_t* cols) {
    const uint32_t hd = __ldg(g.hdmap + x);
    if (hd != EMPTY && !(g.abl & ABL_FORCE_BITMAP))
        return g.exact ? warp_fac_exact(g, x, cols) : warp_fac_hist(g.hist + (uint64_t)hd * g.maxc, g.maxc);
    const uint64_t bmv = ld_cg(g.bm + x);
    if (~bmv) return (uint16_t)__ffsll((long long)~bmv);
    return warp_fac_scan(g, x, cols);
}

// ---------------- incremental bitmap / histogram (color_select.cuh:120-209) ----------------

// Sets color c's bit (1..64) of x's bitmap. With READ_FIRST a bit already set
// is left alone (bits are only cleared by rebuilds, which never overlap an
// apply): the recolor walk sets one bit in every neighbor's bitmap, most of
// them already set. Otherwise a fire-and-forget reduction: one vertex on the
// update path, where the warp should not wait.
template <bool READ_FIRST>
__device__ __forceinline__ void set_bm_bit(const Dev& g, uint32_t x, uint16_t c) {
    const unsigned long long bit = 1ull << (c - 1);
    if (!READ_FIRST || !(ld_cg(g.bm + x) & bit)) atomicOr((unsigned long long*)(g.bm + x), bit);
}

__device__ __forceinline__ void nbr_color_change(const Dev& g, uint32_t x, uint16_t oldc, uint16_t newc) {
    if (oldc == newc) return;
    if (newc != 0 && newc <= 64) set_bm_bit<true>(g, x, newc);
    if (g.exact) return;  // no histogram rows
    const uint32_t hd = __ldg(g.hdmap + x);
    if (hd != EMPTY) {
        uint32_t* h = g.hist + (uint64_t)hd * g.maxc;
        if (oldc != 0 && oldc <= g.maxc) atomicSub(h + oldc - 1, 1u);
        if (newc != 0 && newc <= g.maxc) atomicAdd(h + newc - 1, 1u);
    }
}
__device__ __forceinline__ void new_nbr(const Dev& g, uint32_t x, uint16_t c) {
    if (c == 0) return;
    if (c <= 64) set_bm_bit<false>(g, x, c);
    const uint32_t hd = __ldg(g.hdmap + x);
    if (hd != EMPTY && !g.exact && c <= g.maxc) atomicAdd(g.hist + (uint64_t)hd * g.maxc + c - 1, 1u);
}
__device__ __forceinline__ void removed_nbr(const Dev& g, uint32_t x, uint16_t c) {
    if (c == 0) return;
    const uint32_t hd = __ldg(g.hdmap + x);
    if (hd != EMPTY && !g.exact && c <= g.maxc) atomicSub(g.hist + (uint64_t)hd * g.maxc + c - 1, 1u);
}

// ---------------- recolor (recolor.cu:87-163) ----------------

__device__ __forceinline__ uint32_t warp_load_state(const Dev& g, uint32_t x) {
    uint32_t w = 0;
    if (lane_id() == 0) w = ld_cg(g.st + x);
    return __shfl_sync(FULL, w, 0);
}

// recolor_vertex: new = FAC(x); if different, CAS (new, version+1) in, retrying
// on a fresh word; the winner propagates old -> new to every live row entry.
// `chosen` (nonzero) is FAC(x) already computed on the current state by the
// caller; in stream order nothing changes in between, so it equals the call
// the reference makes here.
// warp_recolor_from: the same with x's state word `cur` as last read by the
// caller (a stale word fails the first compare-and-swap, which re-reads it).
__device__ __forceinline__ void warp_recolor_from(const Dev& g, uint32_t x, uint16_t chosen, uint32_t cur) {
    uint16_t newc = chosen ? chosen : warp_fac(g, x, g.st);
    if (newc == color_of(cur)) return;
    for (uint32_t tries = 0;; tries++) {
        const uint32_t want = pack(newc, (uint16_t)(version_of(cur) + 1));
        uint32_t got = 0;
        if (lane_id() == 0) got = atomicCAS(g.st + x, cur, want);
        got = __shfl_sync(FULL, got, 0);
        if (got == cur) break;
        if (tries >= (1u << 20)) {  // the repair after the batch settles x
            if (lane_id() == 0) atomicOr(g.err, ERR_RETRY);
            return;
        }
        cur = got;
        newc = warp_fac(g, x, g.st);
        if (newc == color_of(cur)) return;
    }
    if (lane_id() == 0) {
        mark_touched(g, x);
        note_color(g, x);
    }
    const uint16_t oldc = color_of(cur);
    const uint64_t s = g.rp[x], e = live_end(g, x, s);
    warp_for_each(g.col, s, e, [&](uint64_t, uint32_t ng) {
        if (ng == INV || ng >= g.n) return;
        nbr_color_change(g, ng, oldc, newc);
    });
    __syncwarp();
}
__device__ __forceinline__ void warp_recolor(const Dev& g, uint32_t x, uint16_t chosen = 0) {
    warp_recolor_from(g, x, chosen, warp_load_state(g, x));
}

// Warp-collective: does some live neighbor of x hold color c? Stops at the
// first round that finds one.
__device__ __forceinline__ bool warp_color_held(const Dev& g, uint32_t x, uint16_t c) {
    const uint64_t s = g.rp[x], e = live_end(g, x, s);
    // rounds of 128 slots: a holder is usually among the first neighbors
    return warp_gather_each<true, 1>(g.col, s, e, g.n, g.st, [c](uint32_t, uint32_t w) { return color_of(w) == c; });
}

// Does a live neighbor among the first `lim` live slots of x hold color c?
// `all`: those slots were the whole row.
__device__ __forceinline__ bool warp_color_held_first(const Dev& g, uint32_t x, uint16_t c, uint32_t lim, bool& all) {
    const uint64_t s = g.rp[x], e = live_end(g, x, s);
    const uint64_t e1 = e - s > lim ? s + lim : e;
    all = e1 == e;
    return warp_gather_each<true, 4>(g.col, s, e1, g.n, g.st, [c](uint32_t, uint32_t w) { return color_of(w) == c; });
}

// Appends a row-scale operation to the pass after the batch (lane 0).
// Warp-collective; false when nothing is deferred (no list, or it is full):
// the caller then does the work itself.
__device__ __forceinline__ bool warp_defer(const Dev& g, uint32_t x, uint32_t kind, uint16_t freed) {
    if (!g.hub_ops) return false;
    uint32_t ok = 0;
    if (lane_id() == 0) {
        const uint32_t pos = atomicAdd(g.hub_count, 1u);
        if (pos < g.hub_cap) {
            g.hub_ops[pos].x = x;
            g.hub_ops[pos].op = (kind << 16) | freed;
            ok = 1;
        }
    }
    return __shfl_sync(FULL, ok, 0) != 0;
}

// Both endpoints' state words in one round trip (lanes 0 and 1).
__device__ __forceinline__ void warp_load_states2(const Dev& g, uint32_t u, uint32_t v, uint32_t& su, uint32_t& sv) {
    const uint32_t lane = lane_id();
    uint32_t w = 0;
    if (lane < 2) w = ld_cg(g.st + (lane ? v : u));
    su = __shfl_sync(FULL, w, 0);
    sv = __shfl_sync(FULL, w, 1);
}

// try_color_reduction: after a delete freed `freed`, move to a lower color if one is open.
// `stream_order` false (a concurrent batch) with exact selection on a row above
// the threshold: instead of the full first-free scan, x moves to `freed` when no
// live neighbor holds it any more (an early-exit scan; the full scan of a
// high-degree row would almost always confirm the current color).
// `state` is x's state word as the caller last read it (in stream order
// nothing else changes it before this call; concurrently, a recolor re-reads it).
__device__ __forceinline__ void warp_try_reduce(const Dev& g, uint32_t x, uint16_t freed, bool stream_order,
                                                uint32_t state) {
    const uint16_t cur = color_of(state);
    if (cur == 0) return;
    if (freed >= cur) return;
    if (!stream_order && g.exact && __ldg(g.hdmap + x) != EMPTY) {
        if (freed == 0) return;
        if (g.hub_ops && row_len(g, x) > kHubRow) {
            // a holder is usually among the first neighbors; a hub row without
            // one there is finished (scan, move, walk) by the pass after the batch
            bool all = true;
            if (warp_color_held_first(g, x, freed, kHubScan, all)) return;
            if (warp_defer(g, x, HUB_REDUCE, freed) || warp_color_held(g, x, freed)) return;
        } else if (warp_color_held(g, x, freed)) {
            return;
        }
        warp_recolor(g, x, freed);
        return;
    }
    const uint16_t best = warp_fac(g, x, g.st);
    if (best < cur) warp_recolor(g, x, best);
}

// Colors x, read uncolored as state word `cur`, with FAC; version becomes 1
// (local_update.cu:90-101). Returns x's state word afterwards (another warp's
// color if it got there first).
__device__ __forceinline__ uint32_t warp_color_uncolored(const Dev& g, uint32_t x, uint32_t cur) {
    const uint16_t c = warp_fac(g, x, g.st);
    uint32_t got = 0;
    if (lane_id() == 0) {
        const uint32_t want = pack(c, 1);
        const uint32_t old = atomicCAS(g.st + x, cur, want);
        if (old == cur) {
            mark_touched(g, x);
            note_color(g, x);
            got = want;
        } else {
            got = old;
        }
    }
    return __shfl_sync(FULL, got, 0);
}

// ---------------- one update (local_update.cu:61-147) ----------------

// `exact`: the caller is the only warp touching the graph (stream order), so a
// pristine row's binary-search answer is final; concurrent callers fall back
// to the linear scan whenever the search does not find the key.
__device__ __forceinline__ void warp_apply(const Dev& g, uint32_t u, uint32_t v, uint8_t type, bool exact) {
    if (g.touched && lane_id() == 0 && (type == SGC_UPDATE_ADD || type == SGC_UPDATE_DEL)) {
        // bitmap-class rows are revisited (their bitmaps rebuilt); a row with a
        // histogram class takes exact colors from its live neighbors instead,
        // and is revisited only when its color changes or an ADD leaves a conflict
        if (__ldg(g.hdmap + u) == EMPTY) mark_touched(g, u);
        if (__ldg(g.hdmap + v) == EMPTY) mark_touched(g, v);
    }
    // The state words are read once, after the row edits, and kept: in stream
    // order only this warp changes them, so the reference's re-reads give the
    // same values; in a concurrent batch a later change by another warp is a
    // color change (marked) or leaves this ADD's endpoints equal (caught by
    // the check after the batch).
    // In a concurrent batch the two row edits of an edge (u != v) touch two
    // different rows and no other warp edits those slots of theirs, so the
    // two halves of the warp make them at once (lanes 0-15 row u, 16-31 row
    // v). In stream order they stay in order: the overflow buffer records
    // u's entry before v's, as the reference does.
    const bool halves = !exact && u != v;
    if (type == SGC_UPDATE_ADD) {
        int ru, rv;
        if (halves) {
            const Lanes<16> H;
            const uint32_t x = H.base ? v : u, y = H.base ? u : v;  // one call site: the halves stay converged
            const int r = grp_add_slot(H, g, x, y, false);
            __syncwarp();
            ru = __shfl_sync(FULL, r, 0);
            rv = __shfl_sync(FULL, r, 16);
        } else {
            ru = warp_add_slot(g, u, v, exact);
            rv = warp_add_slot(g, v, u, exact);
        }
        if (ru != rv && lane_id() == 0) flag_asym(g, u);
        uint32_t su, sv;
        warp_load_states2(g, u, v, su, sv);
        if (color_of(su) == 0) {
            su = warp_color_uncolored(g, u, su);
            if (v == u) sv = su;
        }
        if (color_of(sv) == 0) {
            if (lane_id() == 0) new_nbr(g, v, color_of(su));
            __syncwarp();
            sv = warp_color_uncolored(g, v, sv);
        }
        if (lane_id() == 0) new_nbr(g, u, color_of(sv));
        else if (lane_id() == 1) new_nbr(g, v, color_of(su));
        __syncwarp();
        const uint16_t cu = color_of(su), cv = color_of(sv);
        if (cu == cv && cu != 0) {
            const uint32_t loser = prio_less(__ldg(g.deg + u), u, __ldg(g.deg + v), v) ? u : v;
            // concurrent batches: a long histogram-class row's selection and
            // walk go to the pass after the batch
            const bool defer = !exact && g.hub_ops && __ldg(g.hdmap + loser) != EMPTY &&
                               row_len(g, loser) > kHubRow && warp_defer(g, loser, HUB_RECOLOR, 0);
            if (!defer) warp_recolor(g, loser);
        }
    } else if (type == SGC_UPDATE_DEL) {
        uint32_t su, sv;
        warp_load_states2(g, u, v, su, sv);
        const uint16_t fu = color_of(sv);
        const uint16_t fv = color_of(su);
        bool du, dv;
        if (halves) {
            const Lanes<16> H;
            const uint32_t x = H.base ? v : u, y = H.base ? u : v;
            const int d = grp_remove_slot(H, g, x, y, false) ? 1 : 0;
            __syncwarp();
            du = __shfl_sync(FULL, d, 0) != 0;
            dv = __shfl_sync(FULL, d, 16) != 0;
        } else {
            du = warp_remove_slot(g, u, v, exact);
            dv = warp_remove_slot(g, v, u, exact);
        }
        if (lane_id() == 0) {
            if (du != dv) flag_asym(g, u);
            removed_nbr(g, u, fu);
            removed_nbr(g, v, fv);
        }
        __syncwarp();
        warp_try_reduce(g, u, fu, exact, su);
        if (v == u) sv = warp_load_state(g, v);
        warp_try_reduce(g, v, fv, exact, sv);
    }
}

}  // namespace sgc
