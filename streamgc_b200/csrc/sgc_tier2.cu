// sgc_tier2.cu -- Tier-2 repair and the coloring validator on the GPU.
//
// Tier-2 restates cpu_serial_repair (algorithms/streamgc/src/streamgc.cu:1057-1240)
// exactly, without leaving the device:
//   adj(v)  = live row entries of v (!= v, < n)  union  {x : v in row(x), x != v}
//   step 1  uncolored vertices with a non-empty adj, in ascending id order,
//           take the first color in 1..1023 no neighbor holds;
//   step 2  up to 30 passes: detect every v with a lower-id neighbor of equal
//           nonzero color (on the colors at pass start), then greedy-recolor
//           those v in ascending id order; stop when nothing is found or fixed.
// A sequential ascending-order greedy over a list L is reproduced by rounds: a
// vertex of L runs once every lower-id L-neighbor has run, reading the current
// colors. No two adjacent L-vertices share a round, so every vertex sees
// exactly the colors the sequential loop would show it.
//
// The validator restates check_coloring_valid (streamgc.cu:448-556): distinct
// undirected edges of the live CSR with equal nonzero colors, vertices left
// uncolored with a live row entry, the distinct edge count and the max color.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <cuda_runtime.h>

#include <vector>

#include "../../include/streamgc_b200.h"
#include "sgc_kernels.cuh"

namespace sgc {

size_t tier2_cub_bytes(uint32_t n, uint32_t rev_cap);

namespace {

__device__ __forceinline__ uint64_t row_s(const Dev& g, uint32_t x) { return g.rp[x]; }
__device__ __forceinline__ uint64_t row_e(const Dev& g, uint32_t x) { return g.rp[x] + row_len(g, x); }

// Warp per vertex over the live rows of the vertices in [sp.lo, sp.hi): f(x, y)
// for every entry y != INV. With sp.masked only rows of graphs whose
// GraphCtl.t2 is set. A span always covers whole graphs, so every neighbor of
// a visited vertex lies inside it too.
template <class F>
__device__ __forceinline__ void for_all_entries(const Dev& g, Tier2Span sp, F f) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t x = sp.lo + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); x < sp.hi; x += warps) {
        if (sp.masked && !g.gctl[graph_of(g, x)].t2) continue;
        warp_for_each(g.col, row_s(g, x), row_e(g, x), [&](uint64_t, uint32_t y) {
            if (y != INV) f(x, y);
        });
    }
}

__global__ void mark_uncolored_kernel(Dev g, uint8_t* inU, Tier2Span sp) {
    for_all_entries(g, sp, [&](uint32_t x, uint32_t y) {
        if (y >= g.n || y == x) return;
        if (color_of(g.st[x]) == 0) inU[x] = 1;
        if (color_of(g.st[y]) == 0) inU[y] = 1;
    });
}

__global__ void mark_conflict_kernel(Dev g, uint8_t* inF, Tier2Span sp) {
    for_all_entries(g, sp, [&](uint32_t x, uint32_t y) {
        if (y >= g.n || y == x) return;
        const uint16_t a = color_of(g.st[x]), b = color_of(g.st[y]);
        if (a == b && a != 0) inF[x > y ? x : y] = 1;
    });
}

__global__ void set_flags_kernel(const uint32_t* list, const uint32_t* count, uint8_t* flags, uint8_t value) {
    const uint32_t c = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x)
        flags[list[i]] = value;
}

__global__ void iota_kernel(uint32_t* out, const uint32_t* count) {
    const uint32_t c = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) out[i] = i;
}

// Reverse entries into the list: (y << 32 | x) for x -> y with inL[y]. Counts
// every entry but stores only `cap`: the host grows the buffer to the count
// and collects again.
__global__ void rev_collect_kernel(Dev g, const uint8_t* inL, unsigned long long* keys, uint32_t* count,
                                   uint32_t cap, Tier2Span sp) {
    for_all_entries(g, sp, [&](uint32_t x, uint32_t y) {
        if (y >= g.n || y == x || !inL[y]) return;
        const uint32_t k = atomicAdd(count, 1u);
        if (k < cap) keys[k] = ((unsigned long long)y << 32) | x;
    });
}

__global__ void rev_bounds_kernel(const uint32_t* list, const uint32_t* count, const unsigned long long* keys,
                                  const uint32_t* nkeys, uint32_t* rs, uint32_t* re) {
    const uint32_t c = *count;
    const uint32_t nk = *nkeys;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
        const unsigned long long lo = (unsigned long long)list[i] << 32;
        const unsigned long long hi = lo | 0xFFFFFFFFull;
        uint32_t a = 0, b = nk;
        while (a < b) { const uint32_t m = (a + b) >> 1; if (keys[m] < lo) a = m + 1; else b = m; }
        uint32_t a2 = a, b2 = nk;
        while (a2 < b2) { const uint32_t m = (a2 + b2) >> 1; if (keys[m] <= hi) a2 = m + 1; else b2 = m; }
        rs[i] = a;
        re[i] = a2;
    }
}

// Greedy color of list vertex v from its row and its reverse entries
// rkeys[r0, r1): the smallest color in 1..1023 no neighbor holds (version + 1
// when it changes). Warp-collective; `used` is the warp's 32-word scratch.
__device__ __forceinline__ void greedy_color(const Dev& g, uint32_t v, const unsigned long long* rkeys, uint32_t r0,
                                             uint32_t r1, uint32_t* used, uint32_t* fixed) {
    const uint32_t lane = lane_id();
    used[lane] = 0;
    __syncwarp();
    auto mark = [&](uint32_t w) {
        if (w == INV || w >= g.n || w == v) return;
        const uint16_t nc = color_of(ld_cg(g.st + w));
        if (nc != 0 && nc < 1024) atomicOr(&used[nc >> 5], 1u << (nc & 31));
    };
    warp_for_each(g.col, row_s(g, v), row_e(g, v), [&](uint64_t, uint32_t w) { mark(w); });
    for (uint32_t t = r0 + lane; t < r1; t += 32) mark((uint32_t)rkeys[t]);
    __syncwarp();
    uint32_t freew = ~used[lane];
    if (lane == 0) freew &= ~1u;  // color 0 is not a candidate
    const uint32_t bal = __ballot_sync(FULL, freew != 0);
    uint32_t c = 0;
    if (bal) {
        const int src = __ffs(bal) - 1;
        const uint32_t bit = __shfl_sync(FULL, __ffs(freew) - 1, src);
        c = (uint32_t)src * 32 + bit;
    }
    if (lane == 0) {
        const uint32_t w = ld_cg(g.st + v);
        if (c != 0 && c != color_of(w)) {
            g.st[v] = pack((uint16_t)c, (uint16_t)(version_of(w) + 1));
            note_color(g, v);
            atomicAdd(fixed, 1u);
        }
    }
    __syncwarp();
}

// One round: warp per remaining list position. Ready vertices greedy-recolor
// in place and are listed as processed; the rest carry over.
__global__ void __launch_bounds__(256) greedy_round_kernel(Dev g, const uint32_t* L, const uint32_t* rem,
                                                           const uint32_t* rem_count, uint32_t* next,
                                                           uint32_t* next_count, uint32_t* proc, uint32_t* proc_count,
                                                           const uint8_t* inL, const uint8_t* done,
                                                           const unsigned long long* rkeys, const uint32_t* rs,
                                                           const uint32_t* re, uint32_t* fixed) {
    __shared__ uint32_t used_all[8][32];
    const uint32_t wib = threadIdx.x >> 5;
    uint32_t* used = used_all[wib];
    const uint32_t lane = lane_id();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t cnt = *rem_count;
    for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < cnt; k += warps) {
        const uint32_t pos = rem[k];
        const uint32_t v = L[pos];
        // ready: no lower-id L-neighbor still pending
        bool blocked = false;
        warp_for_each(g.col, row_s(g, v), row_e(g, v), [&](uint64_t, uint32_t w) {
            if (w != INV && w < v && inL[w] && !done[w]) blocked = true;
        });
        for (uint32_t t = rs[pos] + lane; t < re[pos]; t += 32) {
            const uint32_t w = (uint32_t)rkeys[t];
            if (w < v && inL[w] && !done[w]) blocked = true;
        }
        blocked = __any_sync(FULL, blocked);
        if (blocked) {
            if (lane == 0) next[atomicAdd(next_count, 1u)] = pos;
            __syncwarp();
            continue;
        }
        greedy_color(g, v, rkeys, rs[pos], re[pos], used, fixed);
        if (lane == 0) proc[atomicAdd(proc_count, 1u)] = v;
        __syncwarp();
    }
}

// One warp, after the round cap: the list positions still pending, in
// ascending order (every lower-id list neighbor is final when a vertex is
// reached, as in the rounds).
__global__ void __launch_bounds__(32) greedy_tail_kernel(Dev g, const uint32_t* L, uint32_t m, const uint8_t* done,
                                                         const unsigned long long* rkeys, const uint32_t* rs,
                                                         const uint32_t* re, uint32_t* fixed) {
    __shared__ uint32_t used[32];
    for (uint32_t pos = 0; pos < m; pos++) {
        const uint32_t v = L[pos];
        if (done[v]) continue;
        greedy_color(g, v, rkeys, rs[pos], re[pos], used, fixed);
    }
}

// Warp per vertex of the span, at most 8 blocks per SM.
uint32_t span_grid(Tier2Span sp) {
    const uint32_t b = (sp.hi - sp.lo + 7) / 8;
    return b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b);
}

// Host-synchronized rounds of the ordered greedy before the rest of the list
// goes to one warp in order (the same result, bounded time).
constexpr uint32_t kMaxRounds = 1024;

uint32_t grid_for(uint32_t items, uint32_t per_block) {
    uint32_t b = (items + per_block - 1) / per_block;
    if (b < 1) b = 1;
    if (b > 148 * 8) b = 148 * 8;
    return b;
}

// Sequential ascending greedy over the ordered list in b.list (count in b.count[4]).
uint32_t ordered_greedy(const Dev& g, Tier2Bufs& b, uint32_t m, cudaStream_t s, uint32_t* hs, uint64_t* nl,
                        Tier2Span sp) {
    uint32_t* cnt = b.count;  // [0] rem count, [1] next count, [2] fixed, [3] rev count, [4] list count, [5] proc count
    cudaMemsetAsync(b.inL + sp.lo, 0, sp.hi - sp.lo, s);
    cudaMemsetAsync(b.done + sp.lo, 0, sp.hi - sp.lo, s);
    set_flags_kernel<<<grid_for(m, 256), 256, 0, s>>>(b.list, cnt + 4, b.inL, 1);
    uint32_t nrev = 0;
    for (int attempt = 0; attempt < 2; attempt++) {
        cudaMemsetAsync(cnt + 3, 0, sizeof(uint32_t), s);
        rev_collect_kernel<<<span_grid(sp), 256, 0, s>>>(g, b.inL, b.rev_keys, cnt + 3, b.rev_cap, sp);
        cudaMemcpyAsync(hs, cnt + 3, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        nrev = hs[0];
        if (nrev <= b.rev_cap || attempt == 1) break;
        // more reverse entries than room: grow the buffers (and sort scratch) and collect again
        cudaFree(b.rev_keys);
        cudaFree(b.rev_keys2);
        cudaFree(b.cub_tmp);
        b.rev_keys = b.rev_keys2 = nullptr;
        b.cub_tmp = nullptr;
        b.rev_cap = nrev + nrev / 4;
        b.cub_tmp_bytes = tier2_cub_bytes(g.n, b.rev_cap);
        if (cudaMalloc(&b.rev_keys, (size_t)b.rev_cap * 8) || cudaMalloc(&b.rev_keys2, (size_t)b.rev_cap * 8) ||
            cudaMalloc(&b.cub_tmp, b.cub_tmp_bytes)) {
            cudaGetLastError();
            b.rev_cap = 0;
            return 0;
        }
        *nl += 1;
    }
    if (nrev > b.rev_cap) nrev = b.rev_cap;
    if (nrev) {
        size_t tb = b.cub_tmp_bytes;
        cub::DeviceRadixSort::SortKeys(b.cub_tmp, tb, b.rev_keys, b.rev_keys2, (int)nrev, 0, 64, s);
        cudaMemcpyAsync(b.rev_keys, b.rev_keys2, (size_t)nrev * 8, cudaMemcpyDeviceToDevice, s);
    }
    uint32_t nrev_h = nrev;
    cudaMemcpyAsync(cnt + 3, &nrev_h, sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    rev_bounds_kernel<<<grid_for(m, 256), 256, 0, s>>>(b.list, cnt + 4, b.rev_keys, cnt + 3, b.rev_start, b.rev_end);
    *nl += 5;
    // remaining positions 0..m-1
    uint32_t* rem = b.pend_v;
    uint32_t* nxt = b.pend_w;
    uint32_t* proc = b.list2;
    cudaMemcpyAsync(cnt + 0, cnt + 4, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    iota_kernel<<<grid_for(m, 256), 256, 0, s>>>(rem, cnt + 0);
    cudaMemsetAsync(cnt + 2, 0, sizeof(uint32_t), s);
    uint32_t left = m;
    for (uint32_t round = 0; round < m && round < kMaxRounds && left; round++) {
        cudaMemsetAsync(cnt + 1, 0, sizeof(uint32_t), s);
        cudaMemsetAsync(cnt + 5, 0, sizeof(uint32_t), s);
        greedy_round_kernel<<<grid_for(left, 8), 256, 0, s>>>(g, b.list, rem, cnt + 0, nxt, cnt + 1, proc, cnt + 5,
                                                             b.inL, b.done, b.rev_keys, b.rev_start, b.rev_end,
                                                             cnt + 2);
        set_flags_kernel<<<grid_for(left, 256), 256, 0, s>>>(proc, cnt + 5, b.done, 1);
        *nl += 2;
        cudaMemcpyAsync(cnt + 0, cnt + 1, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(hs, cnt + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        left = hs[0];
        uint32_t* t = rem;
        rem = nxt;
        nxt = t;
    }
    if (left) {  // round cap reached: the rest in order on one warp
        greedy_tail_kernel<<<1, 32, 0, s>>>(g, b.list, m, b.done, b.rev_keys, b.rev_start, b.rev_end, cnt + 2);
        *nl += 1;
    }
    cudaMemcpyAsync(hs, cnt + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return hs[0];
}

// Ordered selection of the flagged vertex ids of the span into b.list; count to b.count[4].
uint32_t select_flagged(Tier2Span sp, Tier2Bufs& b, const uint8_t* flags, cudaStream_t s, uint32_t* hs) {
    size_t tb = b.cub_tmp_bytes;
    thrust::counting_iterator<uint32_t> it(sp.lo);
    cub::DeviceSelect::Flagged(b.cub_tmp, tb, it, flags + sp.lo, b.list, b.count + 4, (int)(sp.hi - sp.lo), s);
    cudaMemcpyAsync(hs, b.count + 4, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return hs[0];
}

}  // namespace

namespace {

__global__ void t2_span_kernel(const GraphCtl* gc, uint32_t G, uint32_t n, uint32_t* span) {
    __shared__ uint32_t lo, hi;
    if (threadIdx.x == 0) {
        lo = n;
        hi = 0;
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < G; k += blockDim.x)
        if (gc[k].t2) {
            atomicMin(&lo, gc[k].base);
            atomicMax(&hi, k + 1 < G ? gc[k + 1].base : n);
        }
    __syncthreads();
    if (threadIdx.x == 0) {
        span[0] = lo;
        span[1] = hi;
    }
}

}  // namespace

void launch_t2_span(const Dev& g, uint32_t G, uint32_t* span, cudaStream_t s) {
    t2_span_kernel<<<1, 256, 0, s>>>(g.gctl, G, g.n, span);
}

size_t tier2_cub_bytes(uint32_t n, uint32_t rev_cap) {
    size_t a = 0, c = 0;
    thrust::counting_iterator<uint32_t> it(0);
    cub::DeviceSelect::Flagged(nullptr, a, it, (const uint8_t*)nullptr, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)n);
    cub::DeviceRadixSort::SortKeys(nullptr, c, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                   (int)(rev_cap ? rev_cap : 1), 0, 64);
    return a > c ? a : c;
}

uint32_t run_tier2(const Dev& g, Tier2Bufs& b, cudaStream_t s, uint32_t* hs, bool* gave_up, uint64_t* launches,
                   bool masked, uint32_t lo, uint32_t hi) {
    Tier2Span sp{lo, hi < g.n ? hi : g.n, masked ? 1 : 0};
    uint32_t total = 0;
    if (gave_up) *gave_up = false;
    if (sp.lo >= sp.hi) return 0;
    const uint32_t nsp = sp.hi - sp.lo;
    // step 1: uncolored vertices with a non-empty adjacency
    cudaMemsetAsync(b.inU + sp.lo, 0, nsp, s);
    mark_uncolored_kernel<<<span_grid(sp), 256, 0, s>>>(g, b.inU, sp);
    uint32_t m = select_flagged(sp, b, b.inU, s, hs);
    uint64_t nl = 2;
    if (m) total += ordered_greedy(g, b, m, s, hs, &nl, sp);
    // step 2: up to 30 detect / fix passes
    bool clean = false;
    for (int pass = 0; pass < 30; pass++) {
        cudaMemsetAsync(b.inF + sp.lo, 0, nsp, s);
        mark_conflict_kernel<<<span_grid(sp), 256, 0, s>>>(g, b.inF, sp);
        m = select_flagged(sp, b, b.inF, s, hs);
        nl += 2;
        if (!m) { clean = true; break; }
        const uint32_t fixed = ordered_greedy(g, b, m, s, hs, &nl, sp);
        total += fixed;
        if (!fixed) break;
    }
    if (gave_up) *gave_up = !clean;
    if (launches) *launches += nl;
    return total;
}

// ---------------------------------------------------------------------------
// validator
// ---------------------------------------------------------------------------

namespace {

__global__ void validate_kernel(Dev g, unsigned long long* ekeys, uint32_t* ecount, uint32_t ecap,
                                unsigned long long* vkeys, uint32_t* vcount, uint32_t vcap,
                                unsigned long long* stats /* [uncolored_with_edges, max_color, out_of_range] */) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; x < g.n; x += warps) {
        const uint16_t cx = color_of(g.st[x]);
        bool eff = false;
        unsigned long long oor = 0;
        warp_for_each(g.col, row_s(g, x), row_e(g, x), [&](uint64_t, uint32_t y) {
            if (y == INV || (g.blen && (y & TOMB))) return;  // free slot or deleted run entry
            if (y >= g.n) { oor++; return; }
            eff = true;
            const uint32_t a = x < y ? x : y, b2 = x < y ? y : x;
            const unsigned long long key = ((unsigned long long)a << 32) | b2;
            const uint32_t k = atomicAdd(ecount, 1u);
            if (k < ecap) ekeys[k] = key;
            if (cx == color_of(g.st[y]) && cx != 0) {
                const uint32_t kv = atomicAdd(vcount, 1u);
                if (kv < vcap) vkeys[kv] = key;
            }
        });
        eff = __any_sync(FULL, eff);
        for (int off = 16; off > 0; off >>= 1) oor += __shfl_xor_sync(FULL, oor, off);
        if (lane_id() == 0) {
            if (cx == 0 && eff) atomicAdd(stats + 0, 1ull);
            atomicMax(stats + 1, (unsigned long long)cx);
            if (oor) atomicAdd(stats + 2, oor);
        }
    }
}

__global__ void count_unique_kernel(const unsigned long long* keys, uint32_t n, unsigned long long* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (i == 0 || keys[i] != keys[i - 1]) atomicAdd(out, 1ull);
}

}  // namespace

namespace {

// Warp per row: the layout invariants every kernel relies on (see
// streamgc_b200.h, SGC_STATE_*). Reads stay inside [rp[x], rp[x+1]) whatever
// the row's other words say.
__global__ void check_state_kernel(Dev g, unsigned long long* out /* bad rows, flags, first bad */) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t lane = lane_id();
    for (uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; x < g.n; x += warps) {
        const uint64_t s = g.rp[x], e = g.rp[x + 1];
        uint32_t f = 0;
        if (e < s) f |= SGC_STATE_HW;
        const uint64_t cap = e >= s ? e - s : 0;
        const uint64_t hw = g.hw[x];
        if (hw > cap) f |= SGC_STATE_HW;
        const uint64_t he = s + (hw < cap ? hw : cap);
        const uint64_t bl = g.blen ? g.blen[x] : 0;
        if (bl > he - s) f |= SGC_STATE_RUN;
        // sorted prefix: the base run (exact selection) or a never-edited row
        const bool pristine = !(g.edited[x >> 5] & (1u << (x & 31)));
        const uint64_t se = g.blen ? s + (bl < he - s ? bl : he - s) : (pristine ? he : s);
        uint32_t holes_in = 0;
        for (uint64_t i = s + lane; i < e; i += 32) {
            const uint32_t v = g.col[i];
            if (i < he) {
                const bool tomb = g.blen && v != INV && (v & TOMB);
                const uint32_t id = tomb ? (v & ~TOMB) : v;
                if (v == INV || tomb) holes_in++;
                if (v != INV && id >= g.n) f |= SGC_STATE_ID;
                if (i > s && i < se) {
                    const uint32_t p = g.col[i - 1];
                    const uint32_t pid = g.blen ? (p & ~TOMB) : p;
                    if (v == INV || p == INV || pid >= id) f |= SGC_STATE_RUN;
                }
            } else if (v != INV) {
                f |= SGC_STATE_TAIL;
            }
        }
        f = __reduce_or_sync(FULL, f);
        holes_in = __reduce_add_sync(FULL, holes_in);
        if (lane == 0) {
            // the live count: exact between batches (mark minus free slots and tombstones)
            if (g.live && hw <= cap && g.live[x] != (he - s) - holes_in) f |= SGC_STATE_HOLES;
            if (color_of(g.st[x]) > 2048) f |= SGC_STATE_COLOR;
            if (f) {
                atomicAdd(out + 0, 1ull);
                atomicOr(out + 1, (unsigned long long)f);
                atomicMin(out + 2, (unsigned long long)x);
            }
        }
    }
}

}  // namespace

int run_check_state(const Dev& g, cudaStream_t s, uint64_t* out) {
    unsigned long long* d = nullptr;
    if (cudaMallocAsync(&d, 3 * 8, s) != cudaSuccess) return -2;
    const unsigned long long init[3] = {0, 0, ~0ull};
    cudaMemcpyAsync(d, init, sizeof(init), cudaMemcpyHostToDevice, s);
    check_state_kernel<<<148 * 8, 256, 0, s>>>(g, d);
    unsigned long long h[3];
    cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
    out[0] = h[0];
    out[1] = h[1];
    out[2] = h[2];
    return 0;
}

namespace {

// Validation without the distinct-edge sort, for slabs beyond 2^32 slots: an
// undirected edge is counted at its lower endpoint's entry (x < y), so the
// counts equal the distinct ones when every entry has its mirror.
__global__ void validate_count_kernel(Dev g, unsigned long long* stats /* uncolored, max color, oor, edges, violations */) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; x < g.n; x += warps) {
        const uint16_t cx = color_of(g.st[x]);
        bool eff = false;
        unsigned long long oor = 0, edges = 0, viol = 0;
        warp_for_each(g.col, row_s(g, x), row_e(g, x), [&](uint64_t, uint32_t y) {
            if (y == INV || (g.blen && (y & TOMB))) return;
            if (y >= g.n) { oor++; return; }
            eff = true;
            if (x < y) {
                edges++;
                if (cx != 0 && cx == color_of(g.st[y])) viol++;
            }
        });
        eff = __any_sync(FULL, eff);
        for (int off = 16; off > 0; off >>= 1) {
            oor += __shfl_xor_sync(FULL, oor, off);
            edges += __shfl_xor_sync(FULL, edges, off);
            viol += __shfl_xor_sync(FULL, viol, off);
        }
        if (lane_id() == 0) {
            if (cx == 0 && eff) atomicAdd(stats + 0, 1ull);
            atomicMax(stats + 1, (unsigned long long)cx);
            if (oor) atomicAdd(stats + 2, oor);
            if (edges) atomicAdd(stats + 3, edges);
            if (viol) atomicAdd(stats + 4, viol);
        }
    }
}

}  // namespace

int run_validate(const Dev& g, cudaStream_t s, uint64_t* out) {
    // capacity: every live slot
    std::vector<uint64_t> rp_last(1);
    cudaMemcpyAsync(rp_last.data(), g.rp + g.n, 8, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    const uint64_t slots = rp_last[0];
    if (slots > 0xF0000000ull) {  // the distinct-edge sort needs 32-bit key counts: count at the lower endpoint
        unsigned long long* st = nullptr;
        if (cudaMallocAsync(&st, 5 * 8, s) != cudaSuccess) return -2;
        cudaMemsetAsync(st, 0, 5 * 8, s);
        validate_count_kernel<<<148 * 8, 256, 0, s>>>(g, st);
        unsigned long long hs[5];
        cudaMemcpyAsync(hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s);
        cudaFreeAsync(st, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) return -3;
        out[0] = hs[4];
        out[1] = hs[0];
        out[2] = hs[3];
        out[3] = hs[1];
        out[4] = hs[2];
        return 0;
    }
    const uint32_t ecap = (uint32_t)(slots ? slots : 1);
    const uint32_t vcap = 1u << 22;
    unsigned long long *ekeys = nullptr, *ekeys2 = nullptr, *vkeys = nullptr, *vkeys2 = nullptr, *stats = nullptr;
    uint32_t* counts = nullptr;
    void* tmp = nullptr;
    size_t tb = 0, tb2 = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tb, ekeys, ekeys2, (int)ecap, 0, 64);
    cub::DeviceRadixSort::SortKeys(nullptr, tb2, vkeys, vkeys2, (int)vcap, 0, 64);
    if (tb2 > tb) tb = tb2;
    int rc = 0;
    if (cudaMalloc(&ekeys, (size_t)ecap * 8) || cudaMalloc(&ekeys2, (size_t)ecap * 8) ||
        cudaMalloc(&vkeys, (size_t)vcap * 8) || cudaMalloc(&vkeys2, (size_t)vcap * 8) ||
        cudaMalloc(&stats, 8 * 8) || cudaMalloc(&counts, 4 * 4) || cudaMalloc(&tmp, tb)) {
        rc = -2;
    } else {
        cudaMemsetAsync(stats, 0, 8 * 8, s);
        cudaMemsetAsync(counts, 0, 4 * 4, s);
        validate_kernel<<<148 * 8, 256, 0, s>>>(g, ekeys, counts, ecap, vkeys, counts + 1, vcap, stats);
        uint32_t hc[2];
        cudaMemcpyAsync(hc, counts, 8, cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        const uint32_t ne = hc[0] < ecap ? hc[0] : ecap;
        const uint32_t nv = hc[1] < vcap ? hc[1] : vcap;
        if (ne) {
            size_t t = tb;
            cub::DeviceRadixSort::SortKeys(tmp, t, ekeys, ekeys2, (int)ne, 0, 64, s);
            count_unique_kernel<<<148 * 8, 256, 0, s>>>(ekeys2, ne, stats + 3);
        }
        if (nv) {
            size_t t = tb;
            cub::DeviceRadixSort::SortKeys(tmp, t, vkeys, vkeys2, (int)nv, 0, 64, s);
            count_unique_kernel<<<148 * 8, 256, 0, s>>>(vkeys2, nv, stats + 4);
        }
        unsigned long long hs[8];
        cudaMemcpyAsync(hs, stats, 64, cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        out[0] = hs[4];  // violations (distinct edges)
        out[1] = hs[0];  // uncolored with edges
        out[2] = hs[3];  // distinct edges
        out[3] = hs[1];  // max color
        out[4] = hs[2];  // out-of-range entries
        if (hc[1] > vcap) rc = 1;  // violation list saturated: out[0] is a lower bound
    }
    cudaFree(ekeys);
    cudaFree(ekeys2);
    cudaFree(vkeys);
    cudaFree(vkeys2);
    cudaFree(stats);
    cudaFree(counts);
    cudaFree(tmp);
    if (cudaGetLastError() != cudaSuccess && rc == 0) rc = -3;
    return rc;
}

}  // namespace sgc
