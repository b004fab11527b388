// sgc_kernels.cu -- kernels of the handle API (sm_100a).
//
//   det_apply_kernel      one warp applies a batch in stream order: the
//                         reference's local_update_kernel run as a single warp
//                         (local_update.cu:61-147), bit-exact.
//   conc_*                a batch applied by one warp per edge. A hash pre-pass
//                         links each update to the previous and the next update
//                         of the same edge in the batch; the persistent apply
//                         kernel hands out update tickets and the first update
//                         of each edge applies that edge's updates in stream
//                         order, so the edge set after a batch equals the
//                         sequential one; updates of different edges overlap.
//   dirty list + compact  stable per-row compaction (epoch_maintenance.cu:20-61)
//                         of only the rows edited since their last compaction
//                         (every other row is already compact, so compacting it
//                         is the identity); reads each row up to its high-water.
//   take_overflow/drain   streamgc.cu:967-995 + epoch_maintenance.cu:66-87.
//   sweep                 degree-balanced pass over every live adjacency entry:
//                         rebuild_bitmaps (epoch_maintenance.cu:113-128) and the
//                         Tier-1 decision (conflict_repair.cu:10-114) fused, as a
//                         Jacobi sweep (every decision reads start-of-sweep
//                         colors; new words are committed after the sweep).
#include <cuda_runtime.h>
#include <cuda/atomic>

#include "sgc_kernels.cuh"

namespace sgc {

// ---------------------------------------------------------------------------
// warp helpers
// ---------------------------------------------------------------------------

// One atomicAdd per warp; returns this lane's slot when pred, else NONE32.
__device__ __forceinline__ uint32_t warp_append(uint32_t* count, bool pred) {
    const uint32_t m = __ballot_sync(FULL, pred);
    if (!m) return NONE32;
    const uint32_t lane = lane_id();
    const int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(count, (uint32_t)__popc(m));
    base = __shfl_sync(FULL, base, leader);
    return pred ? base + __popc(m & ((1u << lane) - 1)) : NONE32;
}

// Exclusive warp prefix sum.
__device__ __forceinline__ uint32_t warp_excl_scan(uint32_t v, uint32_t& total) {
    const uint32_t lane = lane_id();
    uint32_t x = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, x, off);
        if (lane >= (uint32_t)off) x += y;
    }
    total = __shfl_sync(FULL, x, 31);
    return x - v;
}

// ---------------------------------------------------------------------------
// update kernels
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(32) det_apply_kernel(Dev g, const EdgeUpdate* __restrict__ ups, uint32_t n) {
    for (uint32_t i = 0; i < n; i++) {
        const uint4 r = ld_cg4(reinterpret_cast<const uint32_t*>(ups + i));
        const uint32_t u = r.x, v = r.y;
        const uint8_t type = (uint8_t)(r.z & 0xFFu);
        if (u >= g.n || v >= g.n) {
            if (lane_id() == 0) atomicAdd(g.nskip, 1ull);
            continue;  // get_owned_index miss: the reference skips the update
        }
        warp_apply(g, u, v, type, true);
    }
}

__device__ __forceinline__ unsigned long long edge_key(uint32_t u, uint32_t v) {
    const uint32_t a = u < v ? u : v, b = u < v ? v : u;
    return ((unsigned long long)a << 32) | b;
}
__device__ __forceinline__ uint32_t key_hash(unsigned long long k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return (uint32_t)k;
}

// `dyn` (device words, optional): [0] the batch size; it replaces the `n`
// argument so that a captured CUDA graph can replay the launches on every
// tick. Grid-stride loops.
__device__ __forceinline__ uint32_t batch_n(uint32_t n, const uint32_t* dyn) { return dyn ? ld_cg(dyn) : n; }

__global__ void conc_prep_insert(Dev g, const EdgeUpdate* __restrict__ ups, uint32_t n_arg, EdgeOrder eo,
                                 const uint32_t* dyn) {
    const uint32_t n = batch_n(n_arg, dyn);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *eo.ticket = 0;
        if (g.hub_count) *g.hub_count = 0;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint4 r = ld_cg4(reinterpret_cast<const uint32_t*>(ups + i));
        const uint32_t u = r.x, v = r.y;
        const uint8_t type = (uint8_t)(r.z & 0xFFu);
        if ((type != SGC_UPDATE_ADD && type != SGC_UPDATE_DEL) || u >= g.n || v >= g.n) {
            eo.tslot[i] = NONE32;
            continue;
        }
        const unsigned long long key = edge_key(u, v);
        uint32_t h = key_hash(key) & eo.tmask;
        for (uint32_t probe = 0; probe <= eo.tmask; probe++) {
            const unsigned long long k = atomicCAS(eo.tkey + h, EMPTY64, key);
            if (k == EMPTY64 || k == key) break;
            h = (h + 1) & eo.tmask;
        }
        eo.tslot[i] = h;
        eo.tnext[i] = atomicExch(eo.thead + h, i);
    }
}

// Per update: the previous and the next update of the same edge in stream
// order (NONE32 at the ends), from the slot's push list.
__global__ void conc_prep_prev(uint32_t n_arg, EdgeOrder eo, const uint32_t* dyn, uint32_t* err) {
    const uint32_t n = batch_n(n_arg, dyn);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t h = ld_cg(eo.tslot + i);
        uint32_t prev = NONE32, next = NONE32;
        if (h != NONE32) {
            // a list holds distinct positions of this batch: at most n links
            uint32_t links = 0;
            for (uint32_t j = ld_cg(eo.thead + h); j != NONE32; j = ld_cg(eo.tnext + j)) {
                if (j >= n || ++links > n) {
                    atomicOr(err, ERR_CHAIN);
                    break;
                }
                if (j < i && (prev == NONE32 || j > prev)) prev = j;
                if (j > i && (next == NONE32 || j < next)) next = j;
            }
        }
        eo.tprev[i] = prev;
        eo.tsucc[i] = next;
    }
}

// Warp per edge: a warp takes tickets (update positions) and, when the update
// is the first of its edge in the batch, applies every update of that edge in
// stream order; the later ones are skipped at their own tickets. So the
// updates of one edge never run concurrently and no warp waits for another.
// The batch and the ordering words were written by the copy and the prep
// kernels before this launch: L2-coherent loads. A warp takes its next ticket
// while it applies the current update, and reads a position's ordering words
// and record in one round (the next update of an edge's chain with them).
// Three blocks per SM: 80 registers (the budget the one-warp-per-update
// version ran fastest with; 64 registers spill the update path).
__global__ void __launch_bounds__(256, 3) conc_apply_kernel(Dev g, const EdgeUpdate* __restrict__ ups, uint32_t n_arg,
                                                            EdgeOrder eo, const uint32_t* dyn) {
    const uint32_t n = batch_n(n_arg, dyn);
    uint32_t i = 0;
    if (lane_id() == 0) i = atomicAdd(eo.ticket, 1u);
    i = __shfl_sync(FULL, i, 0);
    while (i < n) {
        uint32_t next = 0;
        if (lane_id() == 0) next = atomicAdd(eo.ticket, 1u);  // used after this update
        const uint32_t h = ld_cg(eo.tslot + i);
        const uint32_t prev = ld_cg(eo.tprev + i);
        uint32_t succ = ld_cg(eo.tsucc + i);
        uint4 r = ld_cg4(reinterpret_cast<const uint32_t*>(ups + i));
        if (h == NONE32) {
            if ((r.x >= g.n || r.y >= g.n) && lane_id() == 0) atomicAdd(g.nskip, 1ull);
        } else if (prev == NONE32) {  // the first update of its edge applies the whole chain
            uint32_t steps = 1;
            for (;;) {
                if (r.x >= g.n || r.y >= g.n) {
                    if (lane_id() == 0) atomicOr(g.err, ERR_CHAIN);
                    break;
                }
                warp_apply(g, r.x, r.y, (uint8_t)(r.z & 0xFFu), false);
                const uint32_t j = succ;
                if (j == NONE32) break;
                if (j >= n || j < i || ++steps > n) {  // ordering words inconsistent with the batch
                    if (lane_id() == 0) atomicOr(g.err, ERR_CHAIN);
                    break;
                }
                succ = ld_cg(eo.tsucc + j);
                r = ld_cg4(reinterpret_cast<const uint32_t*>(ups + j));
            }
            if (lane_id() == 0 && h <= eo.tmask) {  // no kernel reads the table during apply: reset it for the next batch
                eo.tkey[h] = EMPTY64;
                eo.thead[h] = NONE32;
            }
            __syncwarp();
        }
        i = __shfl_sync(FULL, next, 0);
    }
}

// ---------------------------------------------------------------------------
// The pass after a concurrent batch: row-scale operations the apply left
// (HubOp), one block of kHubThreads per operation. Each re-reads x's state
// word; the scans and the neighbor walk after a move take 8192 slots per
// round over the whole block. Decisions are made on words thread 0 read and
// shared, so every branch is block-uniform.
// ---------------------------------------------------------------------------
constexpr uint32_t kHubThreads = 1024;

// The ids of one round's slots: thread t loads the 16-byte chunks at
// c + 4t and c + 4t + 4096 (INV outside [s, e) and for ids >= n).
__device__ __forceinline__ void hub_round(const Dev& g, uint64_t c, uint64_t s, uint64_t e, uint32_t (&y)[8]) {
    const uint64_t i0 = c + 4ull * threadIdx.x, i1 = i0 + 4ull * kHubThreads;
    uint4 q0 = make_uint4(INV, INV, INV, INV), q1 = q0;
    if (i0 < e) q0 = ld_cg4(g.col + i0);
    if (i1 < e) q1 = ld_cg4(g.col + i1);
    const uint32_t v[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
    for (int t = 0; t < 8; t++) {
        const uint64_t p = (t < 4 ? i0 : i1) + (t & 3);
        y[t] = (p >= s && p < e && v[t] < g.n) ? v[t] : INV;
    }
}

// Does a live neighbor in [s, e) hold color c? Stops after the first round that finds one.
__device__ __forceinline__ bool block_color_held(const Dev& g, uint64_t s, uint64_t e, uint16_t c) {
    for (uint64_t r = s & ~3ull; r < e; r += 8ull * kHubThreads) {
        uint32_t y[8];
        hub_round(g, r, s, e, y);
        uint32_t w[8];
#pragma unroll
        for (int t = 0; t < 8; t++) w[t] = y[t] != INV ? ld_cg(g.st + y[t]) : 0u;
        bool hit = false;
#pragma unroll
        for (int t = 0; t < 8; t++) hit |= y[t] != INV && color_of(w[t]) == c;
        if (__syncthreads_or(hit)) return true;
    }
    return false;
}

// Exact selection: the first color no live neighbor in [s, e) holds (colors
// 1..2047, else 2048), as warp_fac_exact. `used`: 64 words of shared memory.
__device__ __forceinline__ uint16_t block_fac_exact(const Dev& g, uint64_t s, uint64_t e, uint32_t* used,
                                                    uint32_t* pick) {
    if (threadIdx.x < 64) used[threadIdx.x] = 0;
    __syncthreads();
    uint32_t lo = 0, hi = 0;  // colors 1..64 (bits 0..63 of a 64-bit mask)
    for (uint64_t r = s & ~3ull; r < e; r += 8ull * kHubThreads) {
        uint32_t y[8];
        hub_round(g, r, s, e, y);
        uint32_t w[8];
#pragma unroll
        for (int t = 0; t < 8; t++) w[t] = y[t] != INV ? ld_cg(g.st + y[t]) : 0u;
#pragma unroll
        for (int t = 0; t < 8; t++) {
            if (y[t] == INV) continue;
            const uint16_t c = color_of(w[t]);
            add_color_bit(c, lo, hi);
            if (c > 64 && c < 2048) atomicOr(&used[c >> 5], 1u << (c & 31));
        }
    }
    lo = __reduce_or_sync(FULL, lo);
    hi = __reduce_or_sync(FULL, hi);
    if (lane_id() == 0) {  // fold colors 1..64 into the same set (color c: word c >> 5, bit c & 31)
        if (lo) atomicOr(&used[0], lo << 1);
        if (lo >> 31) atomicOr(&used[1], 1u);
        if (hi) atomicOr(&used[1], hi << 1);
        if (hi >> 31) atomicOr(&used[2], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const uint32_t l = threadIdx.x;
        uint32_t w0 = ~used[l], w1 = ~used[l + 32];
        if (l == 0) w0 &= ~1u;  // color 0 is never a candidate
        const uint32_t b0 = __ballot_sync(FULL, w0 != 0), b1 = __ballot_sync(FULL, w1 != 0);
        if (l == 0) {
            uint32_t c = 2048;
            if (b0) {
                const int src = __ffs(b0) - 1;
                c = src * 32 + __ffs(~used[src] & (src == 0 ? ~1u : FULL)) - 1;
            } else if (b1) {
                const int src = __ffs(b1) - 1;
                c = 1024 + src * 32 + __ffs(~used[src + 32]) - 1;
            }
            *pick = c;
        }
    }
    __syncthreads();
    const uint16_t c = (uint16_t)*pick;
    __syncthreads();
    return c;
}

__global__ void __launch_bounds__(kHubThreads) hub_ops_kernel(Dev g) {
    __shared__ uint32_t used[64];
    __shared__ uint32_t word[2];
    const uint32_t total = ld_cg(g.hub_count);
    const uint32_t cnt = total < g.hub_cap ? total : g.hub_cap;
    if (blockIdx.x == 0 && threadIdx.x == 0 && cnt) atomicAdd(g.hub_total, (unsigned long long)cnt);
    for (uint32_t k = blockIdx.x; k < cnt; k += gridDim.x) {
        const HubOp op = g.hub_ops[k];
        const uint32_t x = op.x;
        if (x >= g.n) continue;  // block-uniform: every thread read the same record
        const uint32_t kind = op.op >> 16;
        const uint16_t freed = (uint16_t)(op.op & 0xFFFFu);
        const uint64_t s = g.rp[x], e = live_end(g, x, s);
        if (threadIdx.x == 0) word[0] = ld_cg(g.st + x);
        __syncthreads();
        uint32_t cur = word[0];
        __syncthreads();
        uint16_t newc;
        if (kind == HUB_REDUCE) {
            if (freed == 0 || freed >= color_of(cur) || block_color_held(g, s, e, freed)) continue;
            newc = freed;
        } else {
            newc = block_fac_exact(g, s, e, used, &word[1]);
        }
        // recolor_vertex: compare-and-swap (newc, version + 1) in; a changed word
        // re-selects from the live neighbors, as the warp's recolor does
        bool moved = false;
        for (uint32_t tries = 0;; tries++) {
            if (newc == color_of(cur)) break;
            if (threadIdx.x == 0) word[0] = atomicCAS(g.st + x, cur, pack(newc, (uint16_t)(version_of(cur) + 1)));
            __syncthreads();
            const uint32_t got = word[0];
            __syncthreads();
            if (got == cur) {
                moved = true;
                break;
            }
            if (tries >= 1024u) {  // the repair after the batch settles x
                if (threadIdx.x == 0) atomicOr(g.err, ERR_RETRY);
                break;
            }
            cur = got;
            newc = block_fac_exact(g, s, e, used, &word[1]);
        }
        if (!moved) continue;
        if (threadIdx.x == 0) {
            mark_touched(g, x);
            note_color(g, x);
        }
        const uint16_t oldc = color_of(cur);
        for (uint64_t r = s & ~3ull; r < e; r += 8ull * kHubThreads) {
            uint32_t y[8];
            hub_round(g, r, s, e, y);
#pragma unroll
            for (int t = 0; t < 8; t++)
                if (y[t] != INV) nbr_color_change(g, y[t], oldc, newc);
        }
    }
}

// After a batch (exact selection): both endpoints of every ADD whose colors
// are equal are marked for the next repair. Together with the marks of every
// color change, this makes every conflict of the rows have a marked endpoint
// once the last repair ended proper.
__global__ void add_check_kernel(Dev g, const EdgeUpdate* __restrict__ ups, uint32_t n, const uint32_t* dyn) {
    const uint32_t cnt = dyn ? ld_cg(dyn) : n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const uint4 r = ld_cg4(reinterpret_cast<const uint32_t*>(ups + i));
        if ((r.z & 0xFFu) != SGC_UPDATE_ADD || r.x >= g.n || r.y >= g.n || r.x == r.y) continue;
        const uint16_t a = color_of(ld_cg(g.st + r.x)), b = color_of(ld_cg(g.st + r.y));
        if (a == b && a != 0) {
            mark_touched(g, r.x);
            mark_touched(g, r.y);
        }
    }
}
void launch_add_check(const Dev& g, const EdgeUpdate* ups, uint32_t n, const uint32_t* dyn, int num_sms,
                      cudaStream_t s) {
    if (!g.touched || (!dyn && !n)) return;
    uint32_t blk = dyn ? (uint32_t)num_sms * 4 : (n + 255) / 256;
    if (blk > (uint32_t)num_sms * 4) blk = num_sms * 4;
    add_check_kernel<<<blk, 256, 0, s>>>(g, ups, n, dyn);
}

void launch_det_apply(const Dev& g, const EdgeUpdate* ups, uint32_t n, cudaStream_t s) {
    if (n) det_apply_kernel<<<1, 32, 0, s>>>(g, ups, n);
}

// The ingest ring's drain: positions [head, head + n) of a host ring of
// mask + 1 slots, read straight from pinned, device-mapped host memory (16
// bytes per thread, consecutive slots) into the batch buffer.
__global__ void ring_gather_kernel(const uint4* __restrict__ ring, unsigned long long mask, unsigned long long head,
                                   uint32_t n, uint4* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = ring[(head + i) & mask];
}
void launch_ring_gather(const EdgeUpdate* ring, uint64_t mask, uint64_t head, uint32_t n, EdgeUpdate* out,
                        int num_sms, cudaStream_t s) {
    if (!n) return;
    uint32_t blk = (n + 255) / 256;
    if (blk > (uint32_t)num_sms * 4) blk = num_sms * 4;
    ring_gather_kernel<<<blk, 256, 0, s>>>(reinterpret_cast<const uint4*>(ring), mask, head, n,
                                           reinterpret_cast<uint4*>(out));
}

int conc_apply_occupancy() {
    static int occ = 0;
    if (!occ) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, conc_apply_kernel, 256, 0);
        if (occ < 1) occ = 1;
    }
    return occ;
}

void launch_conc_apply(const Dev& g, const EdgeUpdate* ups, uint32_t n, const EdgeOrder& eo, int num_sms,
                       cudaStream_t s) {
    if (!n) return;
    uint32_t blk = (n + 255) / 256;
    if (blk > (uint32_t)num_sms * 16) blk = num_sms * 16;
    conc_prep_insert<<<blk, 256, 0, s>>>(g, ups, n, eo, nullptr);
    conc_prep_prev<<<blk, 256, 0, s>>>(n, eo, nullptr, g.err);
    uint32_t grid = (uint32_t)(num_sms * conc_apply_occupancy());
    const uint32_t need = (n + 7) / 8;  // 8 warps per block
    if (grid > need) grid = need;
    conc_apply_kernel<<<grid, 256, 0, s>>>(g, ups, n, eo, nullptr);
    if (g.hub_ops) hub_ops_kernel<<<num_sms, kHubThreads, 0, s>>>(g);
}

void launch_conc_apply_dyn(const Dev& g, const EdgeUpdate* ups, const uint32_t* dyn, const EdgeOrder& eo,
                           int num_sms, int blocks_per_sm, cudaStream_t s) {
    conc_prep_insert<<<num_sms * 16, 256, 0, s>>>(g, ups, 0, eo, dyn);
    conc_prep_prev<<<num_sms * 16, 256, 0, s>>>(0, eo, dyn, g.err);
    const int occ = conc_apply_occupancy();
    const int bps = (blocks_per_sm > 0 && blocks_per_sm < occ) ? blocks_per_sm : occ;
    conc_apply_kernel<<<num_sms * bps, 256, 0, s>>>(g, ups, 0, eo, dyn);
    if (g.hub_ops) hub_ops_kernel<<<num_sms, kHubThreads, 0, s>>>(g);
}

// Stream order per graph, graphs side by side: warp per segment
// [segs[k], segs[k+1]) of the batch (one graph's updates in submission order),
// so each graph's result does not depend on the others. The segment count
// comes from dyn[2].
__global__ void __launch_bounds__(256) seg_apply_kernel(Dev g, const EdgeUpdate* __restrict__ ups,
                                                        const uint32_t* __restrict__ segs, const uint32_t* dyn) {
    const uint32_t nseg = ld_cg(dyn + 2);
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < nseg; k += warps) {
        const uint32_t a = segs[k], e = segs[k + 1];
        for (uint32_t i = a; i < e; i++) {
            const uint4 r = ld_cg4(reinterpret_cast<const uint32_t*>(ups + i));
            const uint32_t u = r.x, v = r.y;
            const uint8_t type = (uint8_t)(r.z & 0xFFu);
            if (u >= g.n || v >= g.n) {
                if (lane_id() == 0) atomicAdd(g.nskip, 1ull);
                continue;
            }
            warp_apply(g, u, v, type, true);
        }
    }
}
void launch_seg_apply(const Dev& g, const EdgeUpdate* ups, const uint32_t* segs, const uint32_t* dyn, uint32_t max_segs,
                      int num_sms, cudaStream_t s) {
    uint32_t blocks = (max_segs + 7) / 8;
    if (blocks > (uint32_t)num_sms * 4) blocks = num_sms * 4;
    seg_apply_kernel<<<blocks ? blocks : 1, 256, 0, s>>>(g, ups, segs, dyn);
}

// ---------------------------------------------------------------------------
// compaction of edited rows
// ---------------------------------------------------------------------------

__global__ void dirty_list_kernel(Dev g, uint32_t* list, uint32_t* count) {
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nw = (g.n + 31) / 32;
    uint32_t bits = 0;
    if (w < nw) {
        bits = g.dirty[w];
        if (bits) g.dirty[w] = 0;
    }
    uint32_t total = 0;
    const uint32_t off = warp_excl_scan(__popc(bits), total);
    uint32_t base = 0;
    if (lane_id() == 0 && total) base = atomicAdd(count, total);
    base = __shfl_sync(FULL, base, 0);
    uint32_t k = base + off;
    while (bits) {
        const int b = __ffs(bits) - 1;
        bits &= bits - 1;
        list[k++] = w * 32 + b;
    }
}

void launch_dirty_list(const Dev& g, uint32_t* list, uint32_t* count, cudaStream_t s) {
    const uint32_t nw = (g.n + 31) / 32;
    dirty_list_kernel<<<(nw + 255) / 256, 256, 0, s>>>(g, list, count);
}

// Warp per edited row: stable in-place compaction of [rp, rp + hw), INV tail,
// hw = live count.
// Under exact selection a tombstone (id | TOMB) is a hole too, and the live
// entries of the base run, which stay in front and in order, form the new run.
// With `merge` (exact selection), a compacted row of at most kMergeMax live
// entries is also sorted into one base run (warp-wide bitonic sort in shared
// memory), so its later searches stay 32-ary instead of scanning a growing
// unsorted tail; and a row whose tail outgrows an eighth of it is compacted
// even with few holes.
constexpr uint32_t kMergeMax = 1024;

__device__ __forceinline__ void warp_sort_row(uint32_t* buf, uint32_t lane) {
    for (uint32_t k = 2; k <= kMergeMax; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = lane; i < kMergeMax; i += 32) {
                const uint32_t p = i ^ j;
                if (p > i) {
                    const uint32_t a = buf[i], b = buf[p];
                    if ((a > b) == ((i & k) == 0)) {
                        buf[i] = b;
                        buf[p] = a;
                    }
                }
            }
            __syncwarp();
        }
}

__global__ void __launch_bounds__(256) compact_kernel(Dev g, const uint32_t* __restrict__ list,
                                                      const uint32_t* __restrict__ count, int force, int merge) {
    extern __shared__ uint32_t sort_buf[];  // kMergeMax words per warp, only with `merge`
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t lane = lane_id();
    const uint32_t cnt = *count;
    merge = merge && g.blen;
    for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < cnt; k += warps) {
        const uint32_t x = list[k];
        const uint64_t s = g.rp[x];
        const uint32_t hwx = row_len(g, x);
        // Lazy mode: a row whose holes fill at most a quarter of its extent stays
        // as it is (every reader skips INV slots and tombstones); it is compacted later.
        const uint32_t run = merge ? min(g.blen[x], hwx) : 0u;
        const bool long_tail = merge && hwx - run > max(32u, hwx >> 3);
        const uint32_t holes = g.live ? row_holes(g, x, g.hw[x]) : 0u;
        if (!force && g.live && 4u * holes <= hwx && !long_tail) {
            if ((holes || (merge && run < hwx)) && lane == 0)  // still a candidate (holes, or a tail to merge)
                atomicOr(g.dirty + (x >> 5), 1u << (x & 31));
            continue;
        }
        const uint64_t e = s + hwx;
        const uint64_t run_end = s + (g.blen ? g.blen[x] : 0u);
        uint64_t w = s, run_live = 0;
        for (uint64_t c = s & ~3ull; c < e; c += 128) {
            const uint64_t i = c + 4ull * lane;
            uint4 q = make_uint4(INV, INV, INV, INV);
            if (i < e) q = ld_cg4(g.col + i);
            uint32_t vals[4] = {q.x, q.y, q.z, q.w};
            uint32_t m = 0, mr = 0;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const bool live = g.blen ? (vals[j] & TOMB) == 0 : vals[j] != INV;
                if (i + j >= s && i + j < e && live) {
                    m |= 1u << j;
                    if (i + j < run_end) mr |= 1u << j;
                }
            }
            run_live += __reduce_add_sync(FULL, (uint32_t)__popc(mr));
            uint32_t total = 0;
            const uint32_t pre = warp_excl_scan(__popc(m), total);
            __syncwarp();
            uint64_t dst = w + pre;
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (m & (1u << j)) {
                    if (dst != i + j) g.col[dst] = vals[j];
                    dst++;
                }
            w += total;
            __syncwarp();
        }
        for (uint64_t j = w + lane; j < e; j += 32) g.col[j] = INV;
        const uint32_t live = (uint32_t)(w - s);
        if (merge && live > run_live && live <= kMergeMax) {  // tail entries behind the run: one sorted run
            __syncwarp();
            uint32_t* buf = sort_buf + ((threadIdx.x >> 5) & 7) * kMergeMax;
            for (uint32_t i = lane; i < kMergeMax; i += 32) buf[i] = i < live ? g.col[s + i] : INV;
            __syncwarp();
            warp_sort_row(buf, lane);
            for (uint32_t i = lane; i < live; i += 32) g.col[s + i] = buf[i];
            run_live = live;
        }
        if (lane == 0) {
            g.hw[x] = live;
            if (g.live) g.live[x] = live;
            if (g.blen) g.blen[x] = (uint32_t)run_live;
        }
        __syncwarp();
    }
}

void launch_compact(const Dev& g, const uint32_t* list, const uint32_t* count, uint32_t max_rows, bool force,
                    cudaStream_t s, bool merge) {
    if (!max_rows) return;
    uint32_t blocks = (max_rows + 7) / 8;
    if (blocks > 148 * 16) blocks = 148 * 16;
    const size_t smem = merge && g.blen ? 8 * kMergeMax * sizeof(uint32_t) : 0;  // 32 KiB: under the 48 KiB default
    compact_kernel<<<blocks, 256, smem, s>>>(g, list, count, force ? 1 : 0, (merge && g.blen) ? 1 : 0);
}

// ---------------------------------------------------------------------------
// overflow drain (streamgc.cu:967-995, epoch_maintenance.cu:66-87)
// ---------------------------------------------------------------------------

__global__ void take_overflow_kernel(Dev g, uint32_t* drain_n) {
    const uint32_t c = *g.ovf_count;
    if (c) *g.ovf_count = 0;
    *drain_n = c < OVF_CAP ? c : OVF_CAP;
}
void launch_take_overflow(const Dev& g, uint32_t* drain_n, cudaStream_t s) {
    take_overflow_kernel<<<1, 1, 0, s>>>(g, drain_n);
}

// Re-insert without re-appending: first INV or equal slot; none -> failure.
// Unordered drains under exact selection look in the sorted base run first.
__device__ __forceinline__ bool warp_drain_insert(const Dev& g, uint32_t x, uint32_t nbr, bool ordered) {
    const uint64_t s = g.rp[x], e = g.rp[x + 1];
    uint64_t from = s;
    if (!ordered && g.blen) {
        const uint32_t bl = ld_cg(g.blen + x);
        if (bl && warp_run_add(g, x, nbr, s, bl) >= 0) return true;
        from = s + bl;
    }
    for (;;) {
        uint64_t p = 0;
        uint32_t v = 0;
        if (!warp_find(g.col, from, e, [nbr](uint32_t t) { return t == INV || t == nbr; }, p, v)) return false;
        if (v == nbr) return true;
        uint32_t old = 0;
        if (lane_id() == 0) {
            old = atomicCAS(g.col + p, INV, nbr);
            if (old == INV) {
                extend_row(g, x, (uint32_t)(p - s));
                mark_dirty(g, x);
            }
        }
        old = __shfl_sync(FULL, old, 0);
        if (old == INV || old == nbr) return true;
        from = p + 1;
    }
}

__global__ void drain_kernel(Dev g, const uint32_t* __restrict__ drain_n, int ordered, unsigned long long* failed) {
    const uint32_t cnt = *drain_n;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t step = ordered ? 1 : warps;
    if (ordered && w0 != 0) return;
    for (uint32_t k = w0; k < cnt; k += step) {
        const OverflowEdge oe = g.ovf[k];
        const bool ok = warp_drain_insert(g, oe.local_vertex_idx, oe.neighbor_global, ordered != 0);
        if (!ok && lane_id() == 0) {
            if (failed) atomicAdd(failed, 1ull);
            flag_asym(g, oe.local_vertex_idx);
            g.gctl[graph_of(g, oe.local_vertex_idx)].dropped = 1u;
        }
    }
}
void launch_drain(const Dev& g, const uint32_t* drain_n, bool ordered, unsigned long long* failed, cudaStream_t s) {
    if (ordered) drain_kernel<<<1, 32, 0, s>>>(g, drain_n, 1, failed);
    else drain_kernel<<<148 * 4, 256, 0, s>>>(g, drain_n, 0, failed);
}

// ---------------------------------------------------------------------------
// snapshot / query / colors
// ---------------------------------------------------------------------------

__global__ void snapshot_kernel(Dev g, uint16_t* snap) {
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < g.n; x += gridDim.x * blockDim.x)
        snap[x] = color_of(g.st[x]);
}
// Incremental snapshot into the back half, which was last written two
// snapshots ago: the colors of the vertices noted since then (`chg`, this
// epoch's, and `prev`, the epoch before) are copied from the state words;
// then this epoch's marks become `prev` and `chg` starts empty.
__global__ void snapshot_changes_kernel(Dev g, uint32_t* __restrict__ prev, uint16_t* __restrict__ snap) {
    const uint32_t nw = (g.n + 31) / 32;
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x) {
        const uint32_t cur = g.chg[w], old = prev[w];
        if (cur | old) {
            prev[w] = cur;
            if (cur) g.chg[w] = 0;
        }
        uint32_t bits = cur | old;
        while (bits) {
            const uint32_t x = w * 32 + (__ffs(bits) - 1);
            bits &= bits - 1;
            snap[x] = color_of(g.st[x]);
        }
    }
}
void launch_snapshot_changes(const Dev& g, uint32_t* prev, uint16_t* snap, cudaStream_t s) {
    const uint32_t nw = (g.n + 31) / 32;
    uint32_t blk = (nw + 255) / 256;
    if (blk > 148 * 8) blk = 148 * 8;
    snapshot_changes_kernel<<<blk, 256, 0, s>>>(g, prev, snap);
}

void launch_snapshot(const Dev& g, uint16_t* snap, cudaStream_t s) {
    snapshot_kernel<<<(g.n + 255) / 256 < 148 * 16 ? (g.n + 255) / 256 : 148 * 16, 256, 0, s>>>(g, snap);
}
void launch_colors(const Dev& g, uint16_t* out, cudaStream_t s) { launch_snapshot(g, out, s); }

// First-fit coloring of a vertex list in list order: one block walks the
// list, all its threads on the current vertex's row, which gathers the colors
// its live neighbors hold (colors given earlier in the walk included); the
// vertex takes the first color in 1..2047 none of them holds (2048 when all
// do), version 1. Vertices already colored are skipped.
__global__ void __launch_bounds__(1024) color_list_kernel(Dev g, const uint32_t* __restrict__ list, uint32_t m,
                                                          uint32_t* colored) {
    __shared__ uint32_t used[64];
    const uint32_t tid = threadIdx.x;
    uint32_t done = 0;
    for (uint32_t k = 0; k < m; k++) {
        const uint32_t v = list[k];
        if (color_of(ld_cg(g.st + v)) != 0) continue;  // the same word for every thread
        if (tid < 64) used[tid] = 0;
        __syncthreads();
        const uint64_t s = g.rp[v], e = s + row_len(g, v);
        for (uint64_t j = s + tid; j < e; j += blockDim.x) {
            const uint32_t y = g.col[j];
            if (y < g.n) {
                const uint32_t c = color_of(ld_cg(g.st + y));
                if (c != 0 && c < 2048) atomicOr(&used[c >> 5], 1u << (c & 31));
            }
        }
        __syncthreads();
        if (tid < 32) {
            uint32_t f0 = ~used[2 * tid], f1 = ~used[2 * tid + 1];
            if (tid == 0) f0 &= ~1u;  // color 0 is not a candidate
            const uint32_t any = __ballot_sync(FULL, (f0 | f1) != 0);
            uint32_t c = 2048;
            if (any) {
                const uint32_t src = __ffs(any) - 1;
                const uint32_t mine = f0 ? 64 * tid + __ffs(f0) - 1 : 64 * tid + 32 + __ffs(f1) - 1;
                c = __shfl_sync(FULL, (f0 | f1) ? mine : 0u, src);
            }
            if (tid == 0) {
                g.st[v] = pack((uint16_t)c, 1);
                note_color(g, v);
                done++;
            }
        }
        __syncthreads();  // the new color is visible to the next vertex's gathers
    }
    if (tid == 0) *colored = done;
}
void launch_color_list(const Dev& g, const uint32_t* list, uint32_t m, uint32_t* colored, cudaStream_t s) {
    color_list_kernel<<<1, 1024, 0, s>>>(g, list, m, colored);
}

__global__ void query_kernel(const uint16_t* __restrict__ snap, uint32_t n, const uint32_t* __restrict__ v,
                             uint16_t* __restrict__ out, uint32_t k) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) {
        const uint32_t x = v[i];
        out[i] = x < n ? snap[x] : 0;
    }
}
void launch_query(const uint16_t* snap, uint32_t n, const uint32_t* v, uint16_t* out, uint32_t k, cudaStream_t s) {
    if (k) query_kernel<<<(k + 255) / 256, 256, 0, s>>>(snap, n, v, out, k);
}

// ---------------------------------------------------------------------------
// degree-balanced sweeps and the device-driven repair loop
// ---------------------------------------------------------------------------
//
// A repair is a loop of sweeps whose state lives in the RepairCtl block on the
// device: repair_begin_kernel starts it, each sweep reads its index and its
// vertex set (every vertex, or the worklist b.wl) from there, and
// repair_step_kernel decides whether another sweep runs. The host either reads
// the block after each sweep (sgc_repair / sgc_publish) or lets a CUDA-graph
// while-node run the loop (the batched engine): the kernels are the same.

// list_mode of the per-vertex passes: 0 every vertex, 1 b.wl, 2 as RepairCtl says.
__device__ __forceinline__ bool use_list(const SweepBufs& b, int list_mode) {
    return list_mode == 2 ? ld_cg(&b.rc->list) != 0 : list_mode == 1;
}

__global__ void build_items_kernel(Dev g, SweepBufs b, int list_mode) {
    const bool list = use_list(b, list_mode);
    const uint32_t lim = list ? *b.wl_count : g.n;
    const uint32_t tile = b.tile;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < lim; base += stride) {  // warp-uniform trip count
        const uint32_t t = base + threadIdx.x;
        uint32_t k = 0, x = 0;
        if (t < lim) {
            x = list ? b.wl[t] : t;
            const uint32_t len = row_len(g, x);
            if (len > SWEEP_TINY) k = (len + tile - 1) / tile;
        }
        uint32_t total = 0;
        const uint32_t off = warp_excl_scan(k, total);
        uint32_t wbase = 0;
        if (lane_id() == 0 && total) wbase = atomicAdd(b.item_count, total);
        wbase = __shfl_sync(FULL, wbase, 0);
        if (wbase + off + k > b.item_cap) {
            if (k) atomicOr(g.err, ERR_LIST_OVERFLOW);
            continue;
        }
        for (uint32_t j = 0; j < k; j++) b.items[wbase + off + j] = (unsigned long long)x | ((unsigned long long)j << 32);
    }
}
void launch_build_items(const Dev& g, const SweepBufs& b, int list_mode, int num_sms, cudaStream_t s) {
    cudaMemsetAsync(b.item_count, 0, sizeof(uint32_t), s);
    uint32_t blocks = (g.n + 255) / 256;
    if (list_mode != 0 && blocks > (uint32_t)num_sms * 8) blocks = num_sms * 8;
    build_items_kernel<<<blocks ? blocks : 1, 256, 0, s>>>(g, b, list_mode);
}

// Ordered-pair hash for the symmetry checksum: the sum over all entries x->y
// of H(x,y) - H(y,x) is 0 when every entry has its mirror (and otherwise is 0
// only with probability ~2^-64).
__device__ __forceinline__ unsigned long long pair_hash(uint32_t x, uint32_t y) {
    const unsigned long long z = (((unsigned long long)x << 32) | y) * 0x9E3779B97F4A7C15ull;
    return z ^ (z >> 29);
}
__device__ __forceinline__ unsigned long long sym_term(uint32_t x, uint32_t y) {
    return pair_hash(x, y) - pair_hash(y, x);
}

// The bounds of item `it` (row x, chunk j) in slot space.
__device__ __forceinline__ void item_bounds(const Dev& g, const SweepBufs& b, unsigned long long it, uint32_t& x,
                                            uint64_t& s, uint64_t& e) {
    x = (uint32_t)it;
    const uint32_t j = (uint32_t)(it >> 32);
    const uint64_t rs = g.rp[x];
    s = rs + (uint64_t)j * b.tile;
    const uint64_t re = rs + row_len(g, x);
    e = s + b.tile < re ? s + b.tile : re;
}

// Warp per item: up to b.tile live slots of one row. Nothing in the graph
// changes during a sweep, so loads take the read-only path. Each lane keeps two
// 16-byte slot loads and their eight state gathers in flight per round.
// SYM: accumulate the mirror checksum of rows whose graph wants it. PUSH
// (independent-set rule): a same-colored neighbor that loses to x (lower
// priority) is marked for the next sweep, which decides it from its own row.
template <bool SYM, bool PUSH>
__device__ __forceinline__ void sweep_items_body(const Dev& g, const SweepBufs& b) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t lane = lane_id();
    const uint32_t cnt = *b.item_count;
    for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < cnt; k += warps) {
        uint32_t x;
        uint64_t s, e;
        item_bounds(g, b, b.items[k], x, s, e);
        GraphCtl* gc = SYM ? &g.gctl[graph_of(g, x)] : nullptr;
        const bool symx = SYM && gc->full && ld_cg(&gc->asym);
        const uint32_t myc = color_of(__ldg(g.st + x));
        const uint32_t mydeg = (g.abl & ABL_LIVE_DEG) ? row_len(g, x) : __ldg(g.deg + x);
        uint32_t lo = 0, hi = 0;
        unsigned long long sym = 0;
        bool conf = false;
        for (uint64_t c = s & ~3ull; c < e; c += 256) {
            const uint64_t i0 = c + 4ull * lane, i1 = i0 + 128;
            uint4 q0 = make_uint4(INV, INV, INV, INV), q1 = q0;
            if (i0 < e) q0 = __ldg(reinterpret_cast<const uint4*>(g.col + i0));
            if (i1 < e) q1 = __ldg(reinterpret_cast<const uint4*>(g.col + i1));
            uint32_t v[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
            uint32_t nc[8];
#pragma unroll
            for (int t = 0; t < 8; t++) {
                const uint64_t p = (t < 4 ? i0 : i1) + (t & 3);
                const bool in = p >= s && p < e && v[t] < g.n;
                v[t] = in ? v[t] : INV;
                nc[t] = in ? color_of(__ldg(g.st + v[t])) : 0u;
            }
#pragma unroll
            for (int t = 0; t < 8; t++) {
                add_color_bit(nc[t], lo, hi);
                if (nc[t] == myc && myc != 0) {
                    if (PUSH) {
                        if (prio_less(mydeg, x, __ldg(g.deg + v[t]), v[t])) conf = true;
                        else if (v[t] != x) atomicOr(b.wmark + (v[t] >> 5), 1u << (v[t] & 31));
                    } else if (!conf) {
                        conf = prio_less(mydeg, x, __ldg(g.deg + v[t]), v[t]);
                    }
                }
                if (SYM && symx && v[t] != INV && v[t] != x) sym += sym_term(x, v[t]);
            }
        }
        lo = __reduce_or_sync(FULL, lo);
        hi = __reduce_or_sync(FULL, hi);
        const bool anyc = __any_sync(FULL, conf);
        if (SYM)
            for (int off = 16; off > 0; off >>= 1) sym += __shfl_xor_sync(FULL, sym, off);
        if (lane == 0) {
            const unsigned long long m = ((unsigned long long)hi << 32) | lo;
            if (m) atomicOr(b.acc_bm + x, m);
            if (anyc) atomicOr(b.acc_fl + x, 1u);
            if (SYM && sym) atomicAdd(&gc->sym, sym);
        }
    }
}

// sym_mode 0: no checksum; 2: the first sweep of a repair accumulates it for
// the graphs of this repair that visit every vertex with asym set (RepairCtl).
__device__ __forceinline__ bool want_sym(const SweepBufs& b, int sym_mode) {
    return sym_mode == 2 && ld_cg(&b.rc->it) == 0 && ld_cg(&b.rc->any_sym) != 0;
}

__global__ void __launch_bounds__(256, 5) sweep_items_kernel(Dev g, SweepBufs b, int mode, int sym_mode) {
    const bool sym = want_sym(b, sym_mode);
    const bool push = mode == SWEEP_INDEP;
    if (push) {
        if (sym) sweep_items_body<true, true>(g, b);
        else sweep_items_body<false, true>(g, b);
    } else {
        if (sym) sweep_items_body<true, false>(g, b);
        else sweep_items_body<false, false>(g, b);
    }
}

// One vertex of the finalize pass (warp-collective: every lane calls it; `valid`
// lanes own a vertex). Short rows are swept here directly; long rows read the
// accumulators. REBUILD writes bitmaps; TIER1 and INDEP also decide.
// A thread sweeps a row of at most SWEEP_TINY live slots in pieces of
// kPiece slots: the vertex ids of slots [s, e) (any alignment; INV where no
// vertex) come from the covering 16-byte chunks, all loaded in one round
// (aligned, inside the slab: chunks past e are not loaded); the caller then
// gathers what it needs for all of them in a second round. One row of up to
// 64 entries costs a thread at most eight dependent round trips, instead of
// two per slot, and 32 rows share a warp.
constexpr uint32_t kPiece = 16;
constexpr int kPieceIds = 4 * ((kPiece + 3) / 4 + 1);
template <bool READONLY>
__device__ __forceinline__ void piece_ids(const Dev& g, uint64_t s, uint64_t e, uint32_t (&y)[kPieceIds]) {
    const uint64_t base = s & ~3ull;
#pragma unroll
    for (int c = 0; c < kPieceIds / 4; c++) {
        const uint64_t i = base + 4ull * c;
        uint4 q = make_uint4(INV, INV, INV, INV);
        if (i < e) q = READONLY ? __ldg(reinterpret_cast<const uint4*>(g.col + i)) : ld_cg4(g.col + i);
        const uint32_t v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const uint64_t p = i + t;
            y[4 * c + t] = (p >= s && p < e && v[t] < g.n) ? v[t] : INV;
        }
    }
}

__device__ __forceinline__ void finalize_one(const Dev& g, const SweepBufs& b, int mode, bool valid, uint32_t x,
                                             bool with_sym, bool push) {
    bool fac_needed = false, pend = false, need = false;
    uint32_t pend_word = 0;
    unsigned long long sym = 0, live = 0;
    if (valid) {
        if (with_sym) {
            const GraphCtl& gc = g.gctl[graph_of(g, x)];
            with_sym = gc.full && ld_cg(&gc.asym);
        }
        const uint32_t len = row_len(g, x);
        const uint32_t hd = __ldg(g.hdmap + x);
        const uint32_t w = __ldg(g.st + x);
        const uint16_t myc = color_of(w);
        unsigned long long bits = 0;
        bool conf = false;
        live = len;
        if (len <= SWEEP_TINY) {
            const uint32_t mydeg = (g.abl & ABL_LIVE_DEG) ? len : __ldg(g.deg + x);
            uint32_t lo = 0, hi = 0;
            const uint64_t s0 = g.rp[x], e0 = s0 + len;
            for (uint64_t s = s0; s < e0; s += kPiece) {
                uint32_t y[kPieceIds], sw[kPieceIds];
                piece_ids<true>(g, s, s + kPiece < e0 ? s + kPiece : e0, y);
#pragma unroll
                for (int t = 0; t < kPieceIds; t++) sw[t] = y[t] != INV ? __ldg(g.st + y[t]) : 0u;
#pragma unroll
                for (int t = 0; t < kPieceIds; t++) {
                    const uint32_t ng = y[t];
                    if (ng == INV) continue;
                    if (with_sym && ng != x) sym += sym_term(x, ng);
                    const uint32_t nc = color_of(sw[t]);
                    add_color_bit(nc, lo, hi);
                    if (nc == myc && nc != 0) {
                        if (prio_less(mydeg, x, __ldg(g.deg + ng), ng)) conf = true;
                        else if (push && ng != x) atomicOr(b.wmark + (ng >> 5), 1u << (ng & 31));
                    }
                }
            }
            bits = ((unsigned long long)hi << 32) | lo;
        } else {
            bits = b.acc_bm[x];
            conf = b.acc_fl[x] != 0;
            if (bits) b.acc_bm[x] = 0;
            if (conf) b.acc_fl[x] = 0;
        }
        if (mode == SWEEP_REBUILD) {
            if (hd == EMPTY) g.bm[x] = bits;
        } else {
            bool decide = false;
            const bool indep = mode == SWEEP_INDEP;
            if (myc == 0) {
                decide = len > (g.live ? row_holes(g, x, g.hw[x]) : 0u);  // has_neighbors: any non-INV slot
            } else if (conf) {
                decide = true;
                if (myc <= 64) bits |= 1ull << (myc - 1);
            }
            if (indep) {
                if (hd == EMPTY) g.bm[x] = bits;
                else if (decide && myc != 0 && myc <= 64) g.bm[x] |= 1ull << (myc - 1);
                if (decide) b.acc_bm[x] = bits;  // the selection step reads and clears it
                b.needf[x] = decide ? 1 : 0;
                need = decide;
            } else if (hd == EMPTY) {
                g.bm[x] = bits;
                if (decide) {
                    if (~bits) {
                        pend = true;
                        pend_word = pack((uint16_t)__ffsll((long long)~bits), (uint16_t)(version_of(w) + 1));
                    } else {
                        fac_needed = true;
                    }
                }
            } else if (decide) {
                if (myc != 0 && myc <= 64) g.bm[x] |= 1ull << (myc - 1);  // own bit on the (unused) bitmap
                fac_needed = true;
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1) live += __shfl_xor_sync(FULL, live, off);
    if (sym) atomicAdd(&g.gctl[graph_of(g, x)].sym, sym);  // per lane: the lanes' rows may sit in different graphs
    const unsigned long long nv = __popc(__ballot_sync(FULL, valid));
    if (lane_id() == 0) {
        if (live) {
            atomicAdd(b.live, live);
            atomicAdd(b.swept, live);
        }
        if (nv) atomicAdd(b.swept + 1, nv);
    }
    if (mode == SWEEP_INDEP) {
        const uint32_t ni = warp_append(b.need_count, need);
        if (need) b.need_v[ni] = x;
    }
    if (mode == SWEEP_TIER1) {
        const uint32_t pi = warp_append(b.pend_count, pend);
        if (pend) {
            b.pend_v[pi] = x;
            b.pend_w[pi] = pend_word;
        }
        const uint32_t fi = warp_append(b.fac_count, fac_needed);
        if (fac_needed) b.fac_v[fi] = x;
    }
}

// Thread per vertex (every vertex, or the worklist).
__global__ void __launch_bounds__(256, 3) sweep_finalize_kernel(Dev g, SweepBufs b, int mode, int list_mode,
                                                             int sym_mode) {
    const bool list = use_list(b, list_mode);
    const uint32_t lim = list ? *b.wl_count : g.n;
    const uint32_t stride = gridDim.x * blockDim.x;
    const bool sym = want_sym(b, sym_mode);
    const bool push = mode == SWEEP_INDEP;
    for (uint32_t base = blockIdx.x * blockDim.x; base < lim; base += stride) {  // warp-uniform trip count
        const uint32_t t = base + threadIdx.x;
        const bool valid = t < lim;
        finalize_one(g, b, mode, valid, valid ? (list ? b.wl[t] : t) : 0, sym, push);
    }
}

// Warp per vertex whose new color needs the histogram row or the >64 scan;
// colors read are the start-of-sweep ones (nothing is committed yet).
__global__ void __launch_bounds__(256) sweep_fac_kernel(Dev g, SweepBufs b) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t cnt = *b.fac_count;
    for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < cnt; k += warps) {
        const uint32_t x = b.fac_v[k];
        const uint32_t w = ld_cg(g.st + x);
        const uint16_t c = warp_fac(g, x, g.st);
        if (lane_id() == 0) {
            const uint32_t pi = atomicAdd(b.pend_count, 1u);
            b.pend_v[pi] = x;
            b.pend_w[pi] = pack(c, (uint16_t)(version_of(w) + 1));
        }
        __syncwarp();
    }
}

// Independent-set selection, step 1: warp per item (chunk) of a conflicted
// row. Sets the row's blocked flag (acc_fl) when a conflicted neighbor in the
// chunk ranks above it; for a histogram-class row whose neighbors take every
// color 1..64 (acc_bm, from the sweep) it also gathers the taken colors 65..2047
// into the row's words of b.hiused. Colors are the start-of-sweep ones.
__global__ void __launch_bounds__(256, 5) indep_items_kernel(Dev g, SweepBufs b) {
    __shared__ uint32_t s_used[8][64];
    uint32_t* used = s_used[threadIdx.x >> 5];
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t lane = lane_id();
    const uint32_t cnt = *b.item_count;
    const uint32_t salt = sweep_salt(ld_cg(&b.rc->it));
    used[lane] = 0;
    used[lane + 32] = 0;
    __syncwarp();
    for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < cnt; k += warps) {
        const unsigned long long it = b.items[k];
        if (!__ldg(b.needf + (uint32_t)it)) continue;
        if (ld_cg(b.acc_fl + (uint32_t)it)) continue;  // another chunk already found it blocked
        uint32_t x;
        uint64_t s, e;
        item_bounds(g, b, it, x, s, e);
        const uint32_t hd = __ldg(g.hdmap + x);
        const bool full = hd != EMPTY && g.exact && ~b.acc_bm[x] == 0ull;
        const uint32_t base = g.gctl[graph_of(g, x)].base;  // ranks use the graph's own ids
        const unsigned long long rx = sel_rank(x - base, salt);
        bool blocked = false;
        for (uint64_t c = s & ~3ull; c < e; c += 256) {
            const uint64_t i0 = c + 4ull * lane, i1 = i0 + 128;
            uint4 q0 = make_uint4(INV, INV, INV, INV), q1 = q0;
            if (i0 < e) q0 = __ldg(reinterpret_cast<const uint4*>(g.col + i0));
            if (i1 < e) q1 = __ldg(reinterpret_cast<const uint4*>(g.col + i1));
            uint32_t v[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
            uint8_t nf[8];
            uint32_t nc[8];
#pragma unroll
            for (int t = 0; t < 8; t++) {
                const uint64_t p = (t < 4 ? i0 : i1) + (t & 3);
                const bool in = p >= s && p < e && v[t] < g.n && v[t] != x;
                v[t] = in ? v[t] : INV;
                nf[t] = in ? __ldg(b.needf + v[t]) : (uint8_t)0;
                nc[t] = (in && full) ? color_of(__ldg(g.st + v[t])) : 0u;
            }
#pragma unroll
            for (int t = 0; t < 8; t++) {
                if (nf[t] && sel_rank(v[t] - base, salt) > rx) blocked = true;
                if (full && nc[t] > 64 && nc[t] < 2048) atomicOr(&used[nc[t] >> 5], 1u << (nc[t] & 31));
            }
            if (__any_sync(FULL, blocked)) break;  // a blocked row needs nothing more
        }
        blocked = __any_sync(FULL, blocked);
        if (lane == 0 && blocked) atomicOr(b.acc_fl + x, 1u);
        if (full) {
            __syncwarp();
            uint32_t* dst = b.hiused + (uint64_t)hd * 64;
            const uint32_t w0 = used[lane], w1 = used[lane + 32];
            if (w0) atomicOr(dst + lane, w0);
            if (w1) atomicOr(dst + lane + 32, w1);
            used[lane] = 0;
            used[lane + 32] = 0;
            __syncwarp();
        }
    }
}

// Independent-set selection, step 2: thread per conflicted vertex. A row of at
// most SWEEP_TINY slots checks its neighbors here; longer rows read step 1's
// flag. An unblocked vertex takes the first color its neighbors leave free:
// from the sweep's 64-bit mask, else from the gathered 65..2047 set
// (histogram-class rows), else through the warp scan of sweep_fac_kernel
// (bitmap rows whose 64 low colors are all taken). Blocked vertices are marked
// for the next sweep.
__global__ void __launch_bounds__(256) indep_decide_kernel(Dev g, SweepBufs b) {
    const uint32_t cnt = *b.need_count;
    const uint32_t salt = sweep_salt(ld_cg(&b.rc->it));
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const uint32_t x = b.need_v[t];
        const uint32_t len = row_len(g, x);
        bool blocked = false;
        if (len <= SWEEP_TINY) {
            const uint32_t base = g.gctl[graph_of(g, x)].base;  // ranks use the graph's own ids
            const unsigned long long rx = sel_rank(x - base, salt);
            const uint64_t s0 = g.rp[x], e0 = s0 + len;
            for (uint64_t s = s0; s < e0 && !blocked; s += kPiece) {
                uint32_t y[kPieceIds];
                uint8_t nf[kPieceIds];
                piece_ids<true>(g, s, s + kPiece < e0 ? s + kPiece : e0, y);
#pragma unroll
                for (int t = 0; t < kPieceIds; t++) nf[t] = (y[t] != INV && y[t] != x) ? __ldg(b.needf + y[t]) : 0;
#pragma unroll
                for (int t = 0; t < kPieceIds; t++)
                    if (nf[t] && sel_rank(y[t] - base, salt) > rx) blocked = true;
            }
        } else if (b.acc_fl[x]) {
            blocked = true;
            b.acc_fl[x] = 0;
        }
        if (blocked) atomicOr(b.wmark + (x >> 5), 1u << (x & 31));
        const unsigned long long mask = b.acc_bm[x];
        if (mask) b.acc_bm[x] = 0;
        const uint32_t hd = __ldg(g.hdmap + x);
        const bool full = ~mask == 0ull;
        uint32_t c = 0;
        if (full && hd != EMPTY && g.exact && len > SWEEP_TINY) {
            uint32_t* w = b.hiused + (uint64_t)hd * 64;
            c = 2048;
            for (uint32_t k = 2; k < 64; k++) {
                const uint32_t word = w[k];
                if (word) w[k] = 0;
                const uint32_t freew = ~word & (k == 2 ? ~1u : FULL);  // color 64 is taken (full mask)
                if (c == 2048 && freew) c = k * 32 + __ffs(freew) - 1;
            }
        }
        if (blocked) continue;
        if (!full) {
            c = __ffsll((long long)~mask);
        } else if (c == 0) {  // the scan over colors above 64 needs a warp
            b.fac_v[atomicAdd(b.fac_count, 1u)] = x;
            continue;
        }
        const uint32_t w = g.st[x];
        const uint32_t pi = atomicAdd(b.pend_count, 1u);
        b.pend_v[pi] = x;
        b.pend_w[pi] = pack((uint16_t)c, (uint16_t)(version_of(w) + 1));
    }
}

// Writes the chosen colors and clears the recolored vertices' conflict flags.
// Reference rule (TIER1): marks each recolored vertex and, for rows of at most
// SWEEP_TINY slots, its neighbors for the next worklist (longer rows: per item
// in mark_items_kernel). Independent-set rule: ORs the new color into the
// neighbors' bitmaps instead (the next sweep needs no neighbor of a recolored
// vertex: under that rule a recolor creates no conflict).
__global__ void sweep_commit_kernel(Dev g, SweepBufs b, int mode) {
    const uint32_t cnt = *b.pend_count;
    const bool incr = mode == SWEEP_INDEP;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
        const uint32_t x = b.pend_v[k];
        const uint32_t nw = b.pend_w[k];
        g.st[x] = nw;
        note_color(g, x);
        b.needf[x] = 0;
        atomicOr(b.rbits + (x >> 5), 1u << (x & 31));
        if (!incr) atomicOr(b.wmark + (x >> 5), 1u << (x & 31));
        const uint32_t len = row_len(g, x);
        if (len <= SWEEP_TINY) {
            const uint32_t c = color_of(nw);
            const uint64_t s0 = g.rp[x], e0 = s0 + len;
            for (uint64_t s = s0; s < e0; s += kPiece) {
                uint32_t y[kPieceIds];
                piece_ids<false>(g, s, s + kPiece < e0 ? s + kPiece : e0, y);
#pragma unroll
                for (int t = 0; t < kPieceIds; t++) {
                    if (y[t] == INV) continue;
                    if (!incr) atomicOr(b.wmark + (y[t] >> 5), 1u << (y[t] & 31));
                    else if (c != 0 && c <= 64) atomicOr((unsigned long long*)(g.bm + y[t]), 1ull << (c - 1));
                }
            }
        }
    }
}

// Warp per item of the last sweep whose row was recolored: marks the
// neighbors in the item's slots (reference rule) or ORs the row's new color
// into their bitmaps (independent-set rule).
__global__ void __launch_bounds__(256) mark_items_kernel(Dev g, SweepBufs b) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t lane = lane_id();
    const uint32_t cnt = *b.item_count;
    const bool incr = ld_cg(&b.rc->mode) == SWEEP_INDEP;
    for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < cnt; k += warps) {
        const unsigned long long it = b.items[k];
        const uint32_t x0 = (uint32_t)it;
        if (!(b.rbits[x0 >> 5] & (1u << (x0 & 31)))) continue;
        uint32_t x;
        uint64_t s, e;
        item_bounds(g, b, it, x, s, e);
        const uint32_t c = color_of(g.st[x]);
        const unsigned long long bit = (c != 0 && c <= 64) ? 1ull << (c - 1) : 0ull;
        if (incr && !bit) continue;
        for (uint64_t p = s + lane; p < e; p += 32) {
            const uint32_t y = g.col[p];
            if (y >= g.n) continue;
            if (incr) atomicOr((unsigned long long*)(g.bm + y), bit);
            else atomicOr(b.wmark + (y >> 5), 1u << (y & 31));
        }
    }
}

// Turns a bitmask into a list (appending at *count) and clears it; `clear2`
// (optional) is cleared alongside. With `keep` zero the bits are only cleared.
__global__ void collect_bits_kernel(uint32_t n, uint32_t* bits_arr, uint32_t* clear2, uint32_t* list, uint32_t* count,
                                    const uint32_t* keep) {
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nw = (n + 31) / 32;
    const bool k_on = keep == nullptr || ld_cg(keep) != 0;
    uint32_t bits = 0;
    if (w < nw) {
        bits = bits_arr[w];
        if (bits) bits_arr[w] = 0;
        if (clear2 && clear2[w]) clear2[w] = 0;
    }
    if (!k_on) bits = 0;
    uint32_t total = 0;
    const uint32_t off = warp_excl_scan(__popc(bits), total);
    uint32_t base = 0;
    if (lane_id() == 0 && total) base = atomicAdd(count, total);
    base = __shfl_sync(FULL, base, 0);
    uint32_t k = base + off;
    while (bits) {
        const int i = __ffs(bits) - 1;
        bits &= bits - 1;
        list[k++] = w * 32 + i;
    }
}

void launch_next_worklist(const Dev& g, const SweepBufs& b, int num_sms, cudaStream_t s) {
    mark_items_kernel<<<num_sms * 8, 256, 0, s>>>(g, b);
    cudaMemsetAsync(b.wl_count, 0, sizeof(uint32_t), s);
    const uint32_t nw = (g.n + 31) / 32;
    collect_bits_kernel<<<(nw + 255) / 256, 256, 0, s>>>(g.n, b.wmark, b.rbits, b.wl, b.wl_count, nullptr);
}

void launch_sweep(const Dev& g, const SweepBufs& b, SweepMode mode, int list_mode, int sym_mode, int num_sms,
                  cudaStream_t s, cudaEvent_t* phase) {
    if (mode != SWEEP_REBUILD) {
        cudaMemsetAsync(b.pend_count, 0, sizeof(uint32_t), s);
        cudaMemsetAsync(b.fac_count, 0, sizeof(uint32_t), s);
        cudaMemsetAsync(b.need_count, 0, sizeof(uint32_t), s);
    }
    sweep_items_kernel<<<num_sms * 5, 256, 0, s>>>(g, b, (int)mode, sym_mode);  // one wave: 5 blocks per SM
    if (phase) cudaEventRecord(phase[0], s);
    uint32_t fblocks = (g.n + 255) / 256;
    if (list_mode != 0 && fblocks > (uint32_t)num_sms * 3) fblocks = num_sms * 3;  // one wave: 3 blocks per SM
    sweep_finalize_kernel<<<fblocks ? fblocks : 1, 256, 0, s>>>(g, b, (int)mode, list_mode, sym_mode);
    if (phase) cudaEventRecord(phase[1], s);
    if (mode == SWEEP_INDEP) {
        indep_items_kernel<<<num_sms * 5, 256, 0, s>>>(g, b);
        indep_decide_kernel<<<num_sms * 2, 256, 0, s>>>(g, b);
    }
    if (mode != SWEEP_REBUILD) {
        sweep_fac_kernel<<<num_sms * 2, 256, 0, s>>>(g, b);
        sweep_commit_kernel<<<num_sms * 2, 256, 0, s>>>(g, b, (int)mode);
    }
}

// Starts a repair. Reference rule (TIER1, one graph): the first sweep visits
// every vertex. Independent-set rule: per graph, the first worklist is every
// vertex of the graph when it must be repaired in full (its last repair did
// not end proper, its rows may miss mirror entries, or the host forces it),
// else the vertices its updates touched since the last repair: every new
// conflict then has a touched endpoint. One block.
__global__ void repair_begin_kernel(Dev g, SweepBufs b) {
    RepairCtl& rc = *b.rc;
    const bool indep = rc.mode == SWEEP_INDEP;
    uint32_t any_sym = 0, any_incr = 0;
    for (uint32_t k = threadIdx.x; k < b.G; k += blockDim.x) {
        GraphCtl& c = g.gctl[k];
        const bool full = !indep || !c.clean || c.asym || c.force || rc.force_all || !g.touched;
        c.full = full ? 1u : 0u;
        c.force = 0;
        c.sym = 0;
        if (full && c.asym) any_sym = 1;
        if (!full) any_incr = 1;
    }
    any_sym = __syncthreads_or(any_sym);
    any_incr = __syncthreads_or(any_incr);
    if (threadIdx.x == 0) {
        rc.any_sym = any_sym;
        rc.incr = any_incr;
        rc.list = indep ? 1u : 0u;
        rc.it = 0;
        rc.cont = 1;
        rc.done = 0;
        rc.need = 0;
        rc.next = 0;
        rc.prev = 0xFFFFFFFFu;
        rc.plateau = 0;
        rc.sym = 0;
        rc.live = 0;
        *b.live = 0;
        *b.wl_count = 0;
        b.swept[0] = 0;
        b.swept[1] = 0;
    }
}

// First worklist of an independent-set repair: every vertex of the graphs
// repaired in full, the touched vertices of the others; clears the touched
// marks. Thread per 32-vertex word.
__global__ void seed_worklist_kernel(Dev g, SweepBufs b) {
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nw = (g.n + 31) / 32;
    uint32_t bits = 0;
    if (w < nw) {
        const uint32_t t = g.touched[w];
        if (t) g.touched[w] = 0;
        if (g.gctl[g.gidw ? g.gidw[w] : 0u].full) {
            const uint32_t left = g.n - w * 32;
            bits = left >= 32 ? FULL : (1u << left) - 1u;
        } else {
            bits = t;
        }
    }
    uint32_t total = 0;
    const uint32_t off = warp_excl_scan(__popc(bits), total);
    uint32_t base = 0;
    if (lane_id() == 0 && total) base = atomicAdd(b.wl_count, total);
    base = __shfl_sync(FULL, base, 0);
    uint32_t k = base + off;
    while (bits) {
        const int i = __ffs(bits) - 1;
        bits &= bits - 1;
        b.wl[k++] = w * 32 + i;
    }
}

// After each sweep: reads the counts, decides whether another sweep runs,
// advances the index. Reference rule (TIER1): stop at 0 conflicts, after 3
// equal counts, or at max_sweeps (streamgc.cu:1317-1393); later sweeps visit
// the worklist only when the first found the rows mirror-complete.
// Independent-set rule: stop when the next worklist is empty. After the first
// sweep a graph whose checksum came out 0 is known mirror-complete; when the
// loop ends every graph records whether it ended proper. `cond` (graph mode):
// the while-node's handle receives the decision. One block.
__global__ void repair_step_kernel(Dev g, SweepBufs b, cudaGraphConditionalHandle cond, int has_cond) {
    RepairCtl& rc = *b.rc;
    __shared__ uint32_t s_stop;
    const bool indep = rc.mode == SWEEP_INDEP;
    uint32_t sym_any = 0;
    if (rc.it == 0) {
        for (uint32_t k = threadIdx.x; k < b.G; k += blockDim.x) {
            GraphCtl& c = g.gctl[k];
            if (c.full && c.asym) {
                if (c.sym == 0) c.asym = 0;  // found mirror-complete
                else sym_any = 1;
            }
        }
    }
    sym_any = __syncthreads_or(sym_any);
    if (threadIdx.x == 0) {
        const uint32_t count = indep ? *b.need_count : *b.pend_count;
        const uint32_t next = *b.wl_count;
        if (rc.it == 0) {
            rc.sym = sym_any ? (g.gctl[0].sym ? g.gctl[0].sym : 1ull) : 0ull;
            rc.live = *b.live;
        }
        rc.need = count;
        rc.next = next;
        bool done, stop;
        if (indep) {
            done = next == 0;
            stop = done;
        } else {
            done = count == 0;
            stop = done;
            if (!done) {
                if (count == rc.prev) stop = ++rc.plateau >= 3;
                else rc.plateau = 0;
            }
            rc.prev = count;
        }
        rc.done = done ? 1u : 0u;
        rc.list = (indep || rc.sym == 0) ? 1u : 0u;
        rc.it += 1;
        rc.cont = (!stop && rc.it < rc.max_sweeps) ? 1u : 0u;
        s_stop = rc.cont ? 0u : 1u;
        if (has_cond) cudaGraphSetConditional(cond, rc.cont);
    }
    __syncthreads();
    if (s_stop) {
        const bool done = rc.done != 0;
        for (uint32_t k = threadIdx.x; k < b.G; k += blockDim.x) {
            GraphCtl& c = g.gctl[k];
            c.clean = (done && c.sym == 0) ? 1u : 0u;
            c.t2 = c.sym != 0 ? 1u : 0u;
        }
        __syncthreads();
        if (!done) {  // the graphs of the vertices still to visit hold the unresolved conflicts
            const uint32_t nx = *b.wl_count;
            for (uint32_t i = threadIdx.x; i < nx; i += blockDim.x) g.gctl[graph_of(g, b.wl[i])].t2 = 1;
        }
    }
}

void launch_repair_begin(const Dev& g, const SweepBufs& b, SweepMode mode, int num_sms, cudaStream_t s) {
    repair_begin_kernel<<<1, 256, 0, s>>>(g, b);
    if (mode == SWEEP_INDEP && g.touched) {
        const uint32_t nw = (g.n + 31) / 32;
        seed_worklist_kernel<<<(nw + 255) / 256, 256, 0, s>>>(g, b);
    }
    (void)num_sms;
}

void launch_repair_sweep(const Dev& g, const SweepBufs& b, SweepMode mode, int num_sms, cudaStream_t s,
                         cudaEvent_t* phase) {
    launch_build_items(g, b, 2, num_sms, s);
    if (phase) cudaEventRecord(phase[0], s);
    launch_sweep(g, b, mode, 2, 2, num_sms, s, phase ? phase + 1 : nullptr);
}

void launch_repair_step(const Dev& g, const SweepBufs& b, int num_sms, cudaStream_t s,
                        const cudaGraphConditionalHandle* cond) {
    launch_next_worklist(g, b, num_sms, s);
    repair_step_kernel<<<1, 256, 0, s>>>(g, b, cond ? *cond : (cudaGraphConditionalHandle)0, cond ? 1 : 0);
}

}  // namespace sgc
