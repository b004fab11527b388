// sgc_dropin.cu -- kernel-level drop-in: the reference's __global__ entry
// points with identical names and signatures (algorithms/streamgc/src/
// streamgc.cu:80-87), operating on a device copy of the reference's
// GPUPartition. Built as relocatable device code (libsgc_dropin.a) so a
// program written against the reference kernels -- e.g. the reference's
// algorithms/streamgc/test/integration/test_single_gpu.cu -- links unchanged.
//
// Each kernel keeps the reference's launch contract (warp per update for
// local_update_kernel, thread per vertex / per overflow entry for the rest):
// the set of rows or updates a launch covers is the one the caller's grid
// names. Inside, the lanes of each warp cooperate on the units their threads
// own, one unit at a time: row scans read 32 consecutive slots per step
// (coalesced) instead of one slot per serial iteration, and the neighbor walk
// of a recolor spreads its atomics over the warp. Ids go through the
// partition's hash maps exactly as the reference does (streamgc.cu:151-173);
// ghost rows are honoured where the reference reads them.
#include <cuda_runtime.h>

#include "../../include/streamgc_types.h"

namespace dropin {

constexpr uint32_t INV = SGC_CSR_INVALID;
constexpr uint32_t EMPTY = SGC_HASH_EMPTY;
constexpr uint32_t MAXC = SGC_MAX_HISTOGRAM_COLORS_DEFAULT;  // reference default build

// Cooperative group = the lanes of this warp that exist (blockDim need not be a
// multiple of 32). rank/width index them in lane order.
struct Grp {
    uint32_t mask, lane, rank, width;
};
__device__ __forceinline__ Grp grp() {
    Grp g;
    g.mask = __activemask();
    g.lane = threadIdx.x & 31u;
    g.rank = __popc(g.mask & ((1u << g.lane) - 1));
    g.width = __popc(g.mask);
    return g;
}
__device__ __forceinline__ uint32_t bcast(const Grp& g, uint32_t v, uint32_t src_lane) {
    return __shfl_sync(g.mask, v, src_lane);
}
__device__ __forceinline__ uint32_t leader(const Grp& g) { return __ffs(g.mask) - 1; }

__device__ __forceinline__ uint32_t hash_lookup(const uint32_t* map, uint32_t size, uint32_t key) {
    const uint32_t mask = size - 1;
    const uint32_t slot = (key * 2654435761u) & mask;
    for (uint32_t probe = 0; probe < size; probe++) {
        const uint32_t i = (slot + probe) & mask;
        const uint32_t k = map[2 * i];
        if (k == key) return map[2 * i + 1];
        if (k == EMPTY) return EMPTY;
    }
    return EMPTY;
}
__device__ __forceinline__ uint32_t owned_idx(const GPUPartition* p, uint32_t g) {
    return hash_lookup(p->global_to_owned, p->index_map_size, g);
}
__device__ __forceinline__ uint32_t ghost_idx(const GPUPartition* p, uint32_t g) {
    return hash_lookup(p->global_to_ghost, p->ghost_map_size, g);
}
__device__ __forceinline__ uint32_t ldv(const uint32_t* a) { return __ldcg(a); }
__device__ __forceinline__ uint32_t* stw(VertexState* s, uint32_t i) { return reinterpret_cast<uint32_t*>(s + i); }
__device__ __forceinline__ uint16_t colr(uint32_t w) { return (uint16_t)(w & 0xFFFFu); }
__device__ __forceinline__ uint16_t verr(uint32_t w) { return (uint16_t)(w >> 16); }
__device__ __forceinline__ uint32_t pk(uint16_t c, uint16_t v) { return ((uint32_t)v << 16) | c; }

// First slot j in [s, e) with pred(col[j]); returns e when none. Uniform result.
template <class P>
__device__ __forceinline__ uint32_t grp_find(const Grp& g, const uint32_t* col, uint32_t s, uint32_t e, P pred,
                                             uint32_t& val) {
    for (uint32_t c = s; c < e; c += g.width) {
        const uint32_t j = c + g.rank;
        uint32_t v = INV;
        bool hit = false;
        if (j < e) {
            v = ldv(col + j);
            hit = pred(v);
        }
        const uint32_t b = __ballot_sync(g.mask, hit);
        if (b) {
            const uint32_t src = __ffs(b) - 1;
            val = bcast(g, v, src);
            return c + __popc(g.mask & ((1u << src) - 1));
        }
    }
    return e;
}
template <class F>
__device__ __forceinline__ void grp_each(const Grp& g, const uint32_t* col, uint32_t s, uint32_t e, F f) {
    for (uint32_t j = s + g.rank; j < e; j += g.width) f(j, ldv(col + j));
}

// ---- color selection (color_select.cuh:10-115) ----
__device__ __forceinline__ uint16_t fac_hist(const Grp& g, const uint32_t* h) {
    uint32_t bv = 0xFFFFFFFFu, bi = 0xFFFFFFFFu;
    for (uint32_t c = 0; c < MAXC; c += g.width) {
        const uint32_t i = c + g.rank;
        uint32_t v = 0xFFFFFFFFu;
        if (i < MAXC) v = ldv(h + i);
        const uint32_t z = __ballot_sync(g.mask, i < MAXC && v == 0);
        if (z) {
            const uint32_t src = __ffs(z) - 1;
            return (uint16_t)(c + __popc(g.mask & ((1u << src) - 1)) + 1);
        }
        if (i < MAXC && v < bv) { bv = v; bi = i; }
    }
    // group minimum, ties to the smallest index
    uint32_t best_v = bv, best_i = bi;
    for (uint32_t m = g.mask; m; m &= m - 1) {
        const uint32_t src = __ffs(m) - 1;
        const uint32_t ov = bcast(g, bv, src), oi = bcast(g, bi, src);
        if (ov < best_v || (ov == best_v && oi < best_i)) { best_v = ov; best_i = oi; }
    }
    return (uint16_t)(best_i + 1);
}

__device__ __forceinline__ uint16_t fac_bitmap(const Grp& g, uint32_t x, const GPUPartition* p) {
    const uint64_t bm = __ldcg((const unsigned long long*)(p->neighbor_bitmap + x));
    if (~bm) return (uint16_t)__ffsll((long long)~bm);
    uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    auto mark = [&](uint16_t c) {
        if (c > 0 && c < 256) {
#pragma unroll
            for (int k = 0; k < 8; k++)
                if ((c >> 5) == k) w[k] |= 1u << (c & 31);
        }
    };
    grp_each(g, p->col_idx, p->row_ptr[x], p->row_ptr[x + 1], [&](uint32_t, uint32_t ng) {
        if (ng == INV) return;
        const uint32_t nl = owned_idx(p, ng);
        if (nl != EMPTY) mark(colr(ldv(stw(p->owned, nl))));
    });
    grp_each(g, p->ghost_col_idx, p->ghost_row_ptr[x], p->ghost_row_ptr[x + 1], [&](uint32_t, uint32_t gg) {
        if (gg == INV) return;
        const uint32_t gl = ghost_idx(p, gg);
        if (gl != EMPTY) mark(colr(ldv(stw(p->ghost, gl))));
    });
#pragma unroll
    for (int k = 0; k < 8; k++) {
        uint32_t acc = 0;
        for (uint32_t m = g.mask; m; m &= m - 1) acc |= bcast(g, w[k], __ffs(m) - 1);
        w[k] = acc;
    }
    w[0] |= 1u;
#pragma unroll
    for (int k = 0; k < 8; k++)
        if (~w[k]) return (uint16_t)(k * 32 + __ffs(~w[k]) - 1);
    return 256;
}

__device__ __forceinline__ uint16_t fac(const Grp& g, uint32_t x, const GPUPartition* p) {
    if (p->high_degree_map != nullptr) {
        const uint32_t hd = p->high_degree_map[x];
        if (hd != EMPTY) return fac_hist(g, p->freq_histogram + (uint64_t)hd * MAXC);
    }
    return fac_bitmap(g, x, p);
}

// ---- incremental bitmap / histogram (color_select.cuh:120-209), single thread ----
__device__ __forceinline__ uint32_t* hrow(const GPUPartition* p, uint32_t x) {
    if (!p->high_degree_map) return nullptr;
    const uint32_t hd = p->high_degree_map[x];
    return hd == EMPTY ? nullptr : p->freq_histogram + (uint64_t)hd * MAXC;
}
__device__ __forceinline__ void color_change(uint32_t x, uint16_t o, uint16_t nw, const GPUPartition* p) {
    if (o == nw) return;
    if (nw != 0 && nw <= 64) atomicOr((unsigned long long*)(p->neighbor_bitmap + x), 1ull << (nw - 1));
    uint32_t* h = hrow(p, x);
    if (h) {
        if (o != 0 && o <= MAXC) atomicSub(h + o - 1, 1u);
        if (nw != 0 && nw <= MAXC) atomicAdd(h + nw - 1, 1u);
    }
}
__device__ __forceinline__ void new_nbr(uint32_t x, uint16_t c, const GPUPartition* p) {
    if (c == 0) return;
    if (c <= 64) atomicOr((unsigned long long*)(p->neighbor_bitmap + x), 1ull << (c - 1));
    uint32_t* h = hrow(p, x);
    if (h && c <= MAXC) atomicAdd(h + c - 1, 1u);
}
__device__ __forceinline__ void removed_nbr(uint32_t x, uint16_t c, const GPUPartition* p) {
    if (c == 0) return;
    uint32_t* h = hrow(p, x);
    if (h && c <= MAXC) atomicSub(h + c - 1, 1u);
}

// ---- row edits (local_update.cu:12-56) ----
__device__ __forceinline__ void add_nbr(const Grp& g, uint32_t x, uint32_t nbr, const GPUPartition* p) {
    const uint32_t s = p->row_ptr[x], e = p->row_ptr[x + 1];
    uint32_t from = s;
    for (;;) {
        uint32_t v = 0;
        const uint32_t j = grp_find(g, p->col_idx, from, e, [nbr](uint32_t t) { return t == INV || t == nbr; }, v);
        if (j == e) break;
        if (v == nbr) return;
        uint32_t old = 0;
        if (g.lane == leader(g)) old = atomicCAS(p->col_idx + j, INV, nbr);
        old = bcast(g, old, leader(g));
        if (old == INV || old == nbr) return;
        from = j + 1;
    }
    if (g.lane == leader(g)) {
        const uint32_t pos = atomicAdd(p->overflow_local_count, 1u);
        if (pos < SGC_OVERFLOW_CAPACITY) {
            p->overflow_local[pos].local_vertex_idx = x;
            p->overflow_local[pos].neighbor_global = nbr;
        }
    }
    __syncwarp(g.mask);
}
__device__ __forceinline__ void remove_nbr(const Grp& g, uint32_t x, uint32_t nbr, const GPUPartition* p) {
    uint32_t v = 0;
    const uint32_t e = p->row_ptr[x + 1];
    const uint32_t j = grp_find(g, p->col_idx, p->row_ptr[x], e, [nbr](uint32_t t) { return t == nbr; }, v);
    if (j != e && g.lane == leader(g)) p->col_idx[j] = INV;
    __syncwarp(g.mask);
}

// ---- recolor (recolor.cu:87-163) ----
__device__ __forceinline__ uint32_t load_state(const Grp& g, const GPUPartition* p, uint32_t x) {
    uint32_t w = 0;
    if (g.lane == leader(g)) w = ldv(stw(p->owned, x));
    return bcast(g, w, leader(g));
}
__device__ __forceinline__ void recolor(const Grp& g, uint32_t x, const GPUPartition* p) {
    uint32_t cur = load_state(g, p, x);
    uint16_t nc = fac(g, x, p);
    if (nc == colr(cur)) return;
    for (;;) {
        uint32_t got = 0;
        if (g.lane == leader(g)) got = atomicCAS(stw(p->owned, x), cur, pk(nc, (uint16_t)(verr(cur) + 1)));
        got = bcast(g, got, leader(g));
        if (got == cur) break;
        cur = got;
        nc = fac(g, x, p);
        if (nc == colr(cur)) return;
    }
    const uint16_t oc = colr(cur);
    grp_each(g, p->col_idx, p->row_ptr[x], p->row_ptr[x + 1], [&](uint32_t, uint32_t ng) {
        if (ng == INV) return;
        const uint32_t nl = owned_idx(p, ng);
        if (nl != EMPTY) color_change(nl, oc, nc, p);
    });
    __syncwarp(g.mask);
}
__device__ __forceinline__ void try_reduce(const Grp& g, uint32_t x, uint16_t freed, const GPUPartition* p) {
    const uint16_t cur = colr(load_state(g, p, x));
    if (cur == 0 || freed >= cur) return;
    if (fac(g, x, p) < cur) recolor(g, x, p);
}
__device__ __forceinline__ void color_if_uncolored(const Grp& g, uint32_t x, const GPUPartition* p) {
    const uint32_t cur = load_state(g, p, x);
    if (colr(cur) != 0) return;
    const uint16_t c = fac(g, x, p);
    if (g.lane == leader(g)) atomicCAS(stw(p->owned, x), cur, pk(c, 1));
    __syncwarp(g.mask);
}

// Units [base, base + width) owned by this warp's lanes, one at a time.
template <class F>
__device__ __forceinline__ void per_lane_unit(const Grp& g, uint32_t my_unit, F f) {
    for (uint32_t m = g.mask; m; m &= m - 1) {
        const uint32_t src = __ffs(m) - 1;
        f(bcast(g, my_unit, src));
    }
}

}  // namespace dropin

using namespace dropin;

// local_update.cu:61-147 -- warp per update, grid-stride.
__global__ void local_update_kernel(EdgeUpdate* updates, uint32_t num_updates, GPUPartition* partition,
                                    uint32_t histogram_threshold) {
    (void)histogram_threshold;  // dispatch is fixed by high_degree_map, as in the reference
    const Grp g = grp();
    const GPUPartition* p = partition;
    const uint32_t warp_id = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    uint32_t total_warps = (gridDim.x * blockDim.x) / 32;
    if (total_warps == 0) total_warps = 1;
    for (uint32_t i = warp_id; i < num_updates; i += total_warps) {
        const EdgeUpdate e = updates[i];
        const uint32_t u = owned_idx(p, e.u), v = owned_idx(p, e.v);
        if (u == EMPTY || v == EMPTY) continue;
        if (e.type == SGC_UPDATE_ADD) {
            add_nbr(g, u, e.v, p);
            add_nbr(g, v, e.u, p);
            color_if_uncolored(g, u, p);
            if (colr(load_state(g, p, v)) == 0) {
                if (g.lane == leader(g)) new_nbr(v, colr(ldv(stw(p->owned, u))), p);
                __syncwarp(g.mask);
                color_if_uncolored(g, v, p);
            }
            if (g.lane == leader(g)) {
                new_nbr(u, colr(ldv(stw(p->owned, v))), p);
                new_nbr(v, colr(ldv(stw(p->owned, u))), p);
            }
            __syncwarp(g.mask);
            const uint16_t cu = colr(load_state(g, p, u)), cv = colr(load_state(g, p, v));
            const bool conflict = (cu == cv) && cu != 0;
            if (__ballot_sync(g.mask, conflict)) {
                const uint64_t pu = p->init_priority[p->owned_to_global[u]];
                const uint64_t pv = p->init_priority[p->owned_to_global[v]];
                recolor(g, pu < pv ? u : v, p);
            }
        } else if (e.type == SGC_UPDATE_DEL) {
            const uint16_t fu = colr(load_state(g, p, v)), fv = colr(load_state(g, p, u));
            remove_nbr(g, u, e.v, p);
            remove_nbr(g, v, e.u, p);
            if (g.lane == leader(g)) {
                removed_nbr(u, fu, p);
                removed_nbr(v, fv, p);
            }
            __syncwarp(g.mask);
            try_reduce(g, u, fu, p);
            try_reduce(g, v, fv, p);
        }
    }
}

// epoch_maintenance.cu:5-16
__global__ void epoch_snapshot_kernel(GPUPartition* partition, uint32_t num_vertices_global) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < partition->num_owned) {
        const uint32_t gid = partition->owned_to_global[t];
        if (gid < num_vertices_global) partition->epoch_snapshot[gid] = partition->owned[t].color;
    }
}

// Stable in-place compaction of one row by the group (INV tail).
__device__ __forceinline__ void compact_row(const Grp& g, uint32_t* col, uint32_t s, uint32_t e) {
    uint32_t w = s;
    for (uint32_t c = s; c < e; c += g.width) {
        const uint32_t j = c + g.rank;
        uint32_t v = INV;
        if (j < e) v = col[j];
        const bool keep = j < e && v != INV;
        const uint32_t b = __ballot_sync(g.mask, keep);
        __syncwarp(g.mask);
        if (keep) {
            const uint32_t dst = w + __popc(b & ((1u << g.lane) - 1));
            if (dst != j) col[dst] = v;
        }
        w += __popc(b);
        __syncwarp(g.mask);
    }
    for (uint32_t j = w + g.rank; j < e; j += g.width) col[j] = INV;
    __syncwarp(g.mask);
}

// epoch_maintenance.cu:20-61 -- the rows of this launch's thread ids.
__global__ void compact_csr_kernel(GPUPartition* partition) {
    const Grp g = grp();
    const GPUPartition* p = partition;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t mine = tid < p->num_owned ? tid : EMPTY;
    per_lane_unit(g, mine, [&](uint32_t x) {
        if (x == EMPTY) return;
        compact_row(g, p->col_idx, p->row_ptr[x], p->row_ptr[x + 1]);
        compact_row(g, p->ghost_col_idx, p->ghost_row_ptr[x], p->ghost_row_ptr[x + 1]);
    });
}

__device__ __forceinline__ bool drain_insert(const Grp& g, uint32_t* col, uint32_t s, uint32_t e, uint32_t nb) {
    uint32_t from = s;
    for (;;) {
        uint32_t v = 0;
        const uint32_t j = grp_find(g, col, from, e, [nb](uint32_t t) { return t == INV || t == nb; }, v);
        if (j == e) return false;
        if (v == nb) return true;
        uint32_t old = 0;
        if (g.lane == leader(g)) old = atomicCAS(col + j, INV, nb);
        old = bcast(g, old, leader(g));
        if (old == INV || old == nb) return true;
        from = j + 1;
    }
}

// epoch_maintenance.cu:66-87 -- thread per overflow entry.
__global__ void drain_overflow_local_kernel(GPUPartition* partition, uint32_t overflow_count, uint32_t* num_failed) {
    const Grp g = grp();
    const GPUPartition* p = partition;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    per_lane_unit(g, tid < overflow_count ? tid : EMPTY, [&](uint32_t k) {
        if (k == EMPTY) return;
        const OverflowEdge oe = p->overflow_local[k];
        const bool ok = drain_insert(g, p->col_idx, p->row_ptr[oe.local_vertex_idx],
                                     p->row_ptr[oe.local_vertex_idx + 1], oe.neighbor_global);
        if (!ok && num_failed && g.lane == leader(g)) atomicAdd(num_failed, 1u);
        __syncwarp(g.mask);
    });
}

// epoch_maintenance.cu:90-110
__global__ void drain_overflow_ghost_kernel(GPUPartition* partition, uint32_t overflow_count, uint32_t* num_failed) {
    const Grp g = grp();
    const GPUPartition* p = partition;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    per_lane_unit(g, tid < overflow_count ? tid : EMPTY, [&](uint32_t k) {
        if (k == EMPTY) return;
        const OverflowEdge oe = p->overflow_ghost[k];
        const bool ok = drain_insert(g, p->ghost_col_idx, p->ghost_row_ptr[oe.local_vertex_idx],
                                     p->ghost_row_ptr[oe.local_vertex_idx + 1], oe.neighbor_global);
        if (!ok && num_failed && g.lane == leader(g)) atomicAdd(num_failed, 1u);
        __syncwarp(g.mask);
    });
}

// OR of neighbor colors 1..64 (local + ghost rows), group-reduced.
__device__ __forceinline__ uint64_t nbr_bits(const Grp& g, uint32_t x, const GPUPartition* p) {
    unsigned long long bm = 0;
    grp_each(g, p->col_idx, p->row_ptr[x], p->row_ptr[x + 1], [&](uint32_t, uint32_t ng) {
        if (ng == INV) return;
        const uint32_t nl = owned_idx(p, ng);
        if (nl == EMPTY) return;
        const uint16_t c = colr(ldv(stw(p->owned, nl)));
        if (c != 0 && c <= 64) bm |= 1ull << (c - 1);
    });
    grp_each(g, p->ghost_col_idx, p->ghost_row_ptr[x], p->ghost_row_ptr[x + 1], [&](uint32_t, uint32_t gg) {
        if (gg == INV) return;
        const uint32_t gl = ghost_idx(p, gg);
        if (gl == EMPTY) return;
        const uint16_t c = colr(ldv(stw(p->ghost, gl)));
        if (c != 0 && c <= 64) bm |= 1ull << (c - 1);
    });
    unsigned long long acc = 0;
    for (uint32_t m = g.mask; m; m &= m - 1) {
        const uint32_t src = __ffs(m) - 1;
        acc |= ((unsigned long long)bcast(g, (uint32_t)(bm >> 32), src) << 32) | bcast(g, (uint32_t)bm, src);
    }
    return acc;
}

// epoch_maintenance.cu:113-128
__global__ void rebuild_bitmaps_kernel(GPUPartition* partition) {
    const Grp g = grp();
    const GPUPartition* p = partition;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    per_lane_unit(g, tid < p->num_owned ? tid : EMPTY, [&](uint32_t x) {
        if (x == EMPTY) return;
        if (p->high_degree_map != nullptr && p->high_degree_map[x] != EMPTY) return;
        const uint64_t bm = nbr_bits(g, x, p);
        if (g.lane == leader(g)) p->neighbor_bitmap[x] = bm;
        __syncwarp(g.mask);
    });
}

// conflict_repair.cu:10-114 -- thread-per-vertex contract. Like the reference's
// lockstep threads, every vertex of a warp decides from the colors and bitmaps
// as they stand before any vertex of the warp writes; the writes are plain
// stores, racy across warps exactly as in the reference.
__device__ __forceinline__ uint16_t fac_given_bitmap(const Grp& g, uint32_t x, const GPUPartition* p, uint64_t bm) {
    if (p->high_degree_map != nullptr) {
        const uint32_t hd = p->high_degree_map[x];
        if (hd != EMPTY) return fac_hist(g, p->freq_histogram + (uint64_t)hd * MAXC);
    }
    if (~bm) return (uint16_t)__ffsll((long long)~bm);
    return fac_bitmap(g, x, p);  // all 64 set: the neighbor scan does not read the bitmap
}

__global__ void conflict_repair_kernel(GPUPartition* partition, uint32_t histogram_threshold, uint32_t* num_conflicts) {
    (void)histogram_threshold;
    const Grp g = grp();
    const GPUPartition* p = partition;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    bool decide = false;
    uint64_t own_mask = 0;
    uint16_t new_color = 0;
    per_lane_unit(g, tid < p->num_owned ? tid : EMPTY, [&](uint32_t x) {
        if (x == EMPTY) return;
        const bool mine = x == tid;
        const uint16_t my = colr(load_state(g, p, x));
        uint32_t v = 0;
        bool has = grp_find(g, p->col_idx, p->row_ptr[x], p->row_ptr[x + 1], [](uint32_t t) { return t != INV; }, v) !=
                   p->row_ptr[x + 1];
        if (!has)
            has = grp_find(g, p->ghost_col_idx, p->ghost_row_ptr[x], p->ghost_row_ptr[x + 1],
                           [](uint32_t t) { return t != INV; }, v) != p->ghost_row_ptr[x + 1];
        const uint64_t bm = __ldcg((const unsigned long long*)(p->neighbor_bitmap + x));
        if (my == 0) {
            if (has) {
                const uint16_t c = fac_given_bitmap(g, x, p, bm);
                if (mine) { decide = true; new_color = c; }
            }
            return;
        }
        const uint64_t myp = p->init_priority[p->owned_to_global[x]];
        bool need = false;
        grp_each(g, p->col_idx, p->row_ptr[x], p->row_ptr[x + 1], [&](uint32_t, uint32_t ng) {
            if (ng == INV || need) return;
            const uint32_t nl = owned_idx(p, ng);
            if (nl == EMPTY) return;
            const uint16_t nc = colr(ldv(stw(p->owned, nl)));
            if (nc == my && nc != 0 && myp < p->init_priority[ng]) need = true;
        });
        need = __ballot_sync(g.mask, need) != 0;
        if (!need) {
            grp_each(g, p->ghost_col_idx, p->ghost_row_ptr[x], p->ghost_row_ptr[x + 1], [&](uint32_t, uint32_t gg) {
                if (gg == INV || need) return;
                const uint32_t gl = ghost_idx(p, gg);
                if (gl == EMPTY) return;
                const uint16_t gc = colr(ldv(stw(p->ghost, gl)));
                if (gc == my && gc != 0 && myp < p->init_priority[gg]) need = true;
            });
            need = __ballot_sync(g.mask, need) != 0;
        }
        if (need) {
            const uint64_t own = my <= 64 ? (1ull << (my - 1)) : 0ull;
            const uint16_t c = fac_given_bitmap(g, x, p, bm | own);
            if (mine) { decide = true; own_mask = own; new_color = c; }
        }
    });
    __syncwarp(g.mask);
    if (decide) {
        VertexState* s = p->owned + tid;
        if (own_mask) p->neighbor_bitmap[tid] |= own_mask;
        s->color = new_color;
        s->version += 1;
        atomicAdd(num_conflicts, 1u);
    }
}
