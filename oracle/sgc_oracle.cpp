// sgc_oracle.cpp -- CPU ORACLE for the StreamGC single-GPU coloring path.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker: tests/, the smoke entry
// point and the bench's cpu_baseline leg may load it; the product library never
// does. It restates, in plain sequential C++17 (+OpenMP where the step is
// order-independent), what the reference computes on one GPU:
//
//   update rules       algorithms/streamgc/src/kernels/local_update.cu:12-147
//   recolor            algorithms/streamgc/src/kernels/recolor.cu:49-163
//   color selection    algorithms/streamgc/include/color_select.cuh:10-115
//   bitmap/histogram   algorithms/streamgc/include/color_select.cuh:120-251
//   epoch maintenance  algorithms/streamgc/src/kernels/epoch_maintenance.cu:5-128,
//                      driver algorithms/streamgc/src/streamgc.cu:949-1036
//   drain_and_compact  algorithms/streamgc/src/streamgc.cu:1243-1314
//   Tier-1 repair      algorithms/streamgc/src/kernels/conflict_repair.cu:10-114,
//                      loop algorithms/streamgc/src/streamgc.cu:1317-1393
//   Tier-2 repair      algorithms/streamgc/src/streamgc.cu:1057-1240
//   slack CSR build    algorithms/streamgc/src/streamgc.cu:350-433
//   validator          algorithms/streamgc/src/streamgc.cu:448-556
//   static greedy      algorithms/streamgc/src/streamgc.cu:559-592
//   stream generators  algorithms/streamgc/src/host/stream_gen.cpp:30-177
//   graph loader       algorithms/streamgc/src/host/graph_loader.cpp:29-169
//
// Deterministic choices where the reference GPU code is racy (documented):
//  * updates are applied strictly in stream order (the reference run with
//    local_update_kernel launched as a single warp);
//  * overflow drain re-inserts entries in buffer order;
//  * Tier-1 is a Jacobi sweep: every vertex decides on the colors as they were
//    at the start of the sweep (the reference thread-per-vertex kernel reads a
//    racy mix; its bitmaps are rebuilt before the sweep, which Jacobi keeps).
//
// Algorithmic byte counters count every array element each step touches
// (read + write for read-modify-write), at element granularity.

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <unordered_set>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/streamgc_types.h"

namespace {

constexpr uint32_t INV = SGC_CSR_INVALID;
constexpr uint32_t EMPTY = SGC_HASH_EMPTY;
constexpr uint32_t OVF_CAP = SGC_OVERFLOW_CAPACITY;
constexpr uint32_t TOMB = 0x80000000u;  // tombstone bit (concurrent-rules layout)

struct Bytes {
    uint64_t update = 0;   // local update path
    uint64_t epoch = 0;    // snapshot + compact + drain + rebuild
    uint64_t tier1 = 0;    // tier-1 sweeps (rebuild + detect)
    uint64_t tier2 = 0;
};

struct Oracle {
    uint32_t n = 0;
    uint32_t hist_thr = 64;
    uint32_t maxc = 1024;          // MAX_HISTOGRAM_COLORS
    bool exact = false;            // exact selection above the threshold + independent-set Tier-1
    // Concurrent rules (with exact): the row layout and update rules the
    // library's concurrent apply runs by, applied here in stream order. Rows
    // keep a sorted base run [rp, rp+mbl) searched 32-ary (a delete there
    // leaves id | TOMB, a re-insert of the id revives it); other inserts go to
    // the tail at the first free slot after the run; every reader stops at the
    // high-water mark rp+mhw; compaction is lazy (rows whose holes exceed a
    // quarter of the mark); a delete's color reduction on a row above the
    // threshold moves to the freed color only when no live neighbor holds it
    // (an early-exit scan). Colors and edge sets follow the same rules as the
    // library's concurrent configuration; byte counters count what those rules
    // read and write.
    bool conc = false;
    // The reference's ablation builds (reference rules only): every color
    // choice from the bitmap (color_select.cuh:98-100); a full row drops the
    // insert (local_update.cu:28-38); Tier-1 ranks a vertex by its live degree
    // against its neighbors' frozen priorities (conflict_repair.cu:46-57).
    bool abl_force_bitmap = false, abl_no_overflow = false, abl_live_deg = false;
    std::vector<uint32_t> mhw, mbl, mholes;
    std::vector<uint8_t> mdirty;
    std::vector<uint64_t> rp;      // logical row starts, rp[n] = total slots
    std::vector<uint32_t> col;     // slack CSR slots
    std::vector<uint32_t> st;      // packed (color | version << 16)
    std::vector<uint64_t> bm;      // neighbor bitmaps
    std::vector<uint32_t> hdmap;   // vertex -> histogram row or EMPTY
    std::vector<uint32_t> hist;    // num_hd * maxc
    uint32_t num_hd = 0;
    std::vector<uint32_t> deg;     // frozen init degree (priority = deg<<32 | id)
    std::vector<uint8_t> edited;   // row changed since creation; else its base run is sorted, hole-free
    std::vector<uint32_t> base_len;
    std::vector<uint16_t> snap;    // published snapshot
    std::vector<OverflowEdge> ovf; // OVF_CAP entries
    uint32_t ovf_count = 0;        // may exceed OVF_CAP (reference counts every overflow)
    uint64_t ovf_lost = 0;         // entries dropped because pos >= OVF_CAP
    uint64_t drain_failed = 0;
    uint64_t recolors = 0;
    uint64_t updates_applied = 0;
    uint64_t skipped_updates = 0;
    // repair bookkeeping of the exact-selection configuration (the library's
    // device flags): rows possibly not mirror-complete; last repair ended
    // proper; endpoints touched since the last repair; full-repair cadence
    bool asym = true;
    bool clean = false;
    std::vector<uint8_t> touched;
    uint32_t full_every = 16;
    uint64_t since_full = 0;
    Bytes bytes;
    std::string err;

    // -------- state helpers (vertex_state.cuh:17-27, priority.cuh:8-10) --------
    inline uint16_t color(uint32_t x) const { return (uint16_t)(st[x] & 0xFFFFu); }
    // end of the slots readers visit; a slot that holds no entry
    inline uint64_t re(uint32_t x) const { return conc ? rp[x] + mhw[x] : rp[x + 1]; }
    inline bool hole(uint32_t v) const { return v == INV || (conc && (v & TOMB)); }
    inline uint16_t ver(uint32_t x) const { return (uint16_t)(st[x] >> 16); }
    inline uint64_t prio(uint32_t x) const { return ((uint64_t)deg[x] << 32) | x; }
    inline uint32_t* hrow(uint32_t x) {
        uint32_t h = hdmap[x];
        return (h == EMPTY || exact) ? nullptr : &hist[(uint64_t)h * maxc];
    }

    // -------- color selection (color_select.cuh:10-115) --------
    // `cols` is the color source for the >64 fallback scan: live state in the
    // update path, the start-of-sweep copy in the Jacobi Tier-1 sweep.
    uint16_t fac_bitmap(uint32_t x, const std::vector<uint32_t>& cols, uint64_t& b) const {
        uint64_t bmv = bm[x];
        b += 8;
        if (~bmv != 0) return (uint16_t)(__builtin_ctzll(~bmv) + 1);
        bool used[256];
        std::memset(used, 0, sizeof(used));
        for (uint64_t j = rp[x]; j < re(x); j++) {
            uint32_t ng = col[j];
            b += 4;
            if (ng == INV) continue;
            if (ng >= n) continue;                 // not an owned vertex: hash miss
            uint16_t c = (uint16_t)(cols[ng] & 0xFFFFu);
            b += 4;
            if (c > 0 && c < 256) used[c] = true;
        }
        for (uint16_t c = 1; c < 256; c++)
            if (!used[c]) return c;
        return 256;
    }
    uint16_t fac_hist(uint32_t x, uint64_t& b) const {
        const uint32_t* h = &hist[(uint64_t)hdmap[x] * maxc];
        for (uint32_t c = 0; c < maxc; c++) {
            b += 4;
            if (h[c] == 0) return (uint16_t)(c + 1);
        }
        uint32_t mn = h[0], mc = 0;
        for (uint32_t c = 1; c < maxc; c++) {
            b += 4;
            if (h[c] < mn) { mn = h[c]; mc = c; }
        }
        return (uint16_t)(mc + 1);
    }
    // Exact selection: the first color (1..2047) no live neighbor holds, else 2048.
    uint16_t fac_exact(uint32_t x, const std::vector<uint32_t>& cols, uint64_t& b) const {
        std::vector<uint8_t> used(2048, 0);
        for (uint64_t j = rp[x]; j < re(x); j++) {
            uint32_t ng = col[j];
            b += 4;
            if (ng == INV || ng >= n) continue;
            uint16_t c = (uint16_t)(cols[ng] & 0xFFFFu);
            b += 4;
            if (c > 0 && c < 2048) used[c] = 1;
        }
        for (uint16_t c = 1; c < 2048; c++)
            if (!used[c]) return c;
        return 2048;
    }
    uint16_t fac(uint32_t x, const std::vector<uint32_t>& cols, uint64_t& b) const {
        b += 4;  // high_degree_map read
        if (hdmap[x] != EMPTY && !abl_force_bitmap) return exact ? fac_exact(x, cols, b) : fac_hist(x, b);
        return fac_bitmap(x, cols, b);
    }

    // -------- incremental bitmap/histogram maintenance (color_select.cuh:120-209) --------
    void nbr_color_change(uint32_t x, uint16_t oldc, uint16_t newc, uint64_t& b) {
        if (oldc == newc) return;
        if (oldc == 0 && newc == 0) return;
        if (newc != 0 && newc <= 64) { bm[x] |= 1ull << (newc - 1); b += 16; }
        b += 4;
        uint32_t* h = hrow(x);
        if (h) {
            if (oldc != 0 && oldc <= maxc) { h[oldc - 1] -= 1u; b += 8; }
            if (newc != 0 && newc <= maxc) { h[newc - 1] += 1u; b += 8; }
        }
    }
    void new_nbr(uint32_t x, uint16_t c, uint64_t& b) {
        if (c == 0) return;
        if (c <= 64) { bm[x] |= 1ull << (c - 1); b += 16; }
        b += 4;
        uint32_t* h = hrow(x);
        if (h && c <= maxc) { h[c - 1] += 1u; b += 8; }
    }
    void removed_nbr(uint32_t x, uint16_t c, uint64_t& b) {
        if (c == 0) return;
        b += 4;
        uint32_t* h = hrow(x);
        if (h && c <= maxc) { h[c - 1] -= 1u; b += 8; }
    }

    // Binary search of an unedited row's sorted base run; ~0 when absent.
    // Gives the slot the reference's linear scan stops at: the run holds no INV
    // and no duplicate, and only INV follows it.
    uint64_t pristine_find(uint32_t x, uint32_t nbr, uint64_t& b) const {
        uint64_t lo = rp[x], hi = rp[x] + base_len[x];
        while (lo < hi) {
            const uint64_t m = lo + (hi - lo) / 2;
            b += 4;
            if (col[m] < nbr) lo = m + 1;
            else hi = m;
        }
        if (lo < rp[x] + base_len[x] && col[lo] == nbr) return lo;
        return ~0ull;
    }

    // -------- concurrent-rules row edits (the library's warp_add_slot /
    // warp_remove_slot with a base run) --------
    // Slot of id `key` (live or tombstone) in the run, or ~0; counts one
    // 32-slot probe round per level of the 32-ary search.
    uint64_t run_find(uint32_t x, uint32_t key, uint64_t& b) const {
        uint64_t lo = rp[x], hi = rp[x] + mbl[x];
        if (lo == hi) return ~0ull;
        uint64_t len = hi - lo;
        for (; len > 32; len = len - 31 * (len / 32)) b += 128;  // 32 probes per round
        b += 4 * len;                                           // the last bucket, one slot per lane
        while (lo < hi) {
            const uint64_t m = lo + (hi - lo) / 2;
            if ((col[m] & ~TOMB) < key) lo = m + 1;
            else hi = m;
        }
        if (lo < rp[x] + mbl[x] && (col[lo] & ~TOMB) == key) return lo;
        return ~0ull;
    }
    void extend_row(uint32_t x, uint32_t q) {
        if (q < mhw[x]) mholes[x]--;
        else if (q > mhw[x]) mholes[x] += q - mhw[x];
        if (q + 1 > mhw[x]) mhw[x] = q + 1;
        mdirty[x] = 1;
    }
    int add_slot_conc(uint32_t x, uint32_t nbr, uint64_t& b) {
        b += 4;  // run length
        const uint64_t p = run_find(x, nbr, b);
        if (p != ~0ull) {
            if (col[p] == nbr) return 1;
            col[p] = nbr;  // revive the tombstone
            b += 8;
            mholes[x]--;
            mdirty[x] = 1;
            return 0;
        }
        for (uint64_t j = rp[x] + mbl[x]; j < rp[x + 1]; j++) {
            const uint32_t s = col[j];
            b += 4;
            if (s == INV) {
                col[j] = nbr;
                b += 12;  // slot, high-water mark, hole count
                extend_row(x, (uint32_t)(j - rp[x]));
                return 0;
            }
            if (s == nbr) return 1;
        }
        uint32_t pos = ovf_count++;
        if (pos < OVF_CAP) { ovf[pos].local_vertex_idx = x; ovf[pos].neighbor_global = nbr; b += 8; }
        else ovf_lost++;
        asym = true;
        return 2;
    }
    bool remove_slot_conc(uint32_t x, uint32_t nbr, uint64_t& b) {
        b += 8;  // run length, high-water mark
        const uint64_t p = run_find(x, nbr, b);
        if (p != ~0ull && col[p] == nbr) {
            col[p] = nbr | TOMB;
            b += 8;
            mholes[x]++;
            mdirty[x] = 1;
            return true;
        }
        for (uint64_t j = rp[x] + mbl[x]; j < re(x); j++) {
            b += 4;
            if (col[j] == nbr) {
                col[j] = INV;
                b += 8;
                mholes[x]++;
                mdirty[x] = 1;
                return true;
            }
        }
        return false;
    }
    // Lazy compaction of the rows edited since their last compaction: a row
    // whose holes fill more than a quarter of its mark (every row with
    // `force`) keeps its live run entries in front and in order, then its live
    // tail; the rest stay candidates while they hold holes.
    void compact_conc(bool force) {
        uint64_t b = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : b)
        for (int64_t xi = 0; xi < (int64_t)n; xi++) {
            const uint32_t x = (uint32_t)xi;
            if (!mdirty[x]) continue;
            b += 8;
            if (!force && 4ull * mholes[x] <= mhw[x]) {
                if (!mholes[x]) mdirty[x] = 0;
                continue;
            }
            const uint64_t s = rp[x], e = s + mhw[x], run_end = s + mbl[x];
            uint64_t w = s, run_live = 0;
            for (uint64_t j = s; j < e; j++) {
                const uint32_t v = col[j];
                b += 4;
                if (hole(v)) continue;
                if (j < run_end) run_live++;
                if (w != j) { col[w] = v; b += 4; }
                w++;
            }
            for (uint64_t j = w; j < e; j++) { col[j] = INV; b += 4; }
            mhw[x] = (uint32_t)(w - s);
            mbl[x] = (uint32_t)run_live;
            mholes[x] = 0;
            mdirty[x] = 0;
            b += 12;
        }
        bytes.epoch += b;
    }

    // -------- slack CSR row edits (local_update.cu:12-56) --------
    // Returns 0 inserted, 1 already present, 2 overflowed.
    int add_slot(uint32_t x, uint32_t nbr, uint64_t& b) {
        if (conc) return add_slot_conc(x, nbr, b);
        uint64_t from = rp[x];
        if (!edited[x]) {
            if (pristine_find(x, nbr, b) != ~0ull) return 1;
            from = rp[x] + base_len[x];
        }
        for (uint64_t j = from; j < rp[x + 1]; j++) {
            uint32_t s = col[j];
            b += 4;
            if (s == INV) { col[j] = nbr; b += 4; edited[x] = 1; return 0; }
            if (s == nbr) return 1;
        }
        asym = true;
        if (abl_no_overflow) return 2;  // dropped, nothing buffered
        uint32_t pos = ovf_count++;
        if (pos < OVF_CAP) { ovf[pos].local_vertex_idx = x; ovf[pos].neighbor_global = nbr; b += 8; }
        else ovf_lost++;
        return 2;
    }
    // Returns whether an entry was removed.
    bool remove_slot(uint32_t x, uint32_t nbr, uint64_t& b) {
        if (conc) return remove_slot_conc(x, nbr, b);
        if (!edited[x]) {
            const uint64_t p = pristine_find(x, nbr, b);
            if (p != ~0ull) { col[p] = INV; b += 4; edited[x] = 1; return true; }
            return false;
        }
        for (uint64_t j = rp[x]; j < rp[x + 1]; j++) {
            b += 4;
            if (col[j] == nbr) { col[j] = INV; b += 4; return true; }
        }
        return false;
    }

    // -------- recolor (recolor.cu:49-163) --------
    void recolor(uint32_t x, uint64_t& b, uint16_t chosen = 0) {
        uint16_t oldc = color(x);
        uint16_t newc = chosen ? chosen : fac(x, st, b);
        b += 4;
        if (newc == oldc) return;
        uint16_t nv = (uint16_t)(ver(x) + 1);
        st[x] = sgc_pack_state(newc, nv);
        b += 4;
        recolors++;
        if (exact) touched[x] = 1;  // a color change: the next repair starts from x
        // update_incremental_state: every live row entry, duplicates included.
        for (uint64_t j = rp[x]; j < re(x); j++) {
            uint32_t ng = col[j];
            b += 4;
            if (ng == INV || ng >= n) continue;
            nbr_color_change(ng, oldc, newc, b);
        }
    }
    void try_reduce(uint32_t x, uint16_t freed, uint64_t& b) {
        uint16_t cur = color(x);
        b += 4;
        if (cur == 0) return;
        if (freed >= cur) return;
        if (conc && hdmap[x] != EMPTY) {  // early-exit scan for a neighbor still holding `freed`
            b += 4;
            if (freed == 0) return;
            for (uint64_t j = rp[x]; j < re(x); j++) {
                const uint32_t ng = col[j];
                b += 4;
                if (ng >= n) continue;
                b += 4;
                if (color(ng) == freed) return;
            }
            recolor(x, b, freed);
            return;
        }
        uint16_t best = fac(x, st, b);
        if (best < cur) recolor(x, b, best);
    }

    // -------- one update (local_update.cu:61-147), stream order --------
    void apply_one(const EdgeUpdate& e) {
        uint64_t& b = bytes.update;
        b += 16;
        uint32_t u = e.u, v = e.v;
        if (u >= n || v >= n) { skipped_updates++; return; }  // hash miss -> continue
        updates_applied++;
        if (exact && (e.type == SGC_UPDATE_ADD || e.type == SGC_UPDATE_DEL)) {
            // bitmap-class rows are revisited (bitmaps rebuilt); histogram-class
            // rows only when their color changes or an ADD leaves a conflict
            if (hdmap[u] == EMPTY) touched[u] = 1;
            if (hdmap[v] == EMPTY) touched[v] = 1;
        }
        if (e.type == SGC_UPDATE_ADD) {
            if (add_slot(u, v, b) != add_slot(v, u, b)) asym = true;
            b += 4;
            if (color(u) == 0) {
                uint16_t c = fac(u, st, b);
                st[u] = sgc_pack_state(c, 1);
                b += 4;
                if (exact) touched[u] = 1;
            }
            b += 4;
            if (color(v) == 0) {
                new_nbr(v, color(u), b);
                uint16_t c = fac(v, st, b);
                st[v] = sgc_pack_state(c, 1);
                b += 4;
                if (exact) touched[v] = 1;
            }
            new_nbr(u, color(v), b);
            new_nbr(v, color(u), b);
            if (color(u) == color(v) && color(u) != 0) {
                b += 16;
                uint32_t loser = (prio(u) < prio(v)) ? u : v;
                recolor(loser, b);
            }
        } else if (e.type == SGC_UPDATE_DEL) {
            uint16_t fu = color(v);
            uint16_t fv = color(u);
            b += 8;
            const bool du = remove_slot(u, v, b);
            const bool dv = remove_slot(v, u, b);
            if (du != dv) asym = true;
            removed_nbr(u, fu, b);
            removed_nbr(v, fv, b);
            try_reduce(u, fu, b);
            try_reduce(v, fv, b);
        }
    }

    // End of a batch (exact selection): both endpoints of every ADD whose
    // colors are equal are marked for the next repair (the library's
    // add_check_kernel after each apply).
    void batch_end(const EdgeUpdate* ups, uint64_t cnt) {
        if (!exact) return;
        for (uint64_t i = 0; i < cnt; i++) {
            const EdgeUpdate& e = ups[i];
            if (e.type != SGC_UPDATE_ADD || e.u >= n || e.v >= n || e.u == e.v) continue;
            if (color(e.u) == color(e.v) && color(e.u) != 0) touched[e.u] = touched[e.v] = 1;
        }
    }

    // -------- epoch steps (epoch_maintenance.cu:5-128) --------
    void snapshot() {
        for (uint32_t x = 0; x < n; x++) snap[x] = color(x);
        bytes.epoch += (uint64_t)n * 6;
    }
    void compact_all() {
        if (conc) { compact_conc(false); return; }
        uint64_t b = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : b)
        for (int64_t xi = 0; xi < (int64_t)n; xi++) {
            uint32_t x = (uint32_t)xi;
            uint64_t w = rp[x];
            for (uint64_t j = rp[x]; j < rp[x + 1]; j++) {
                b += 4;
                if (col[j] != INV) {
                    if (w != j) { col[w] = col[j]; b += 4; }
                    w++;
                }
            }
            for (uint64_t j = w; j < rp[x + 1]; j++) { col[j] = INV; b += 4; }
        }
        bytes.epoch += b;
    }
    // drain_overflow_local_kernel, entries in buffer order; returns failures.
    uint64_t drain(uint32_t cnt) {
        uint64_t failed = 0;
        for (uint32_t i = 0; i < cnt; i++) {
            uint32_t x = ovf[i].local_vertex_idx, nb = ovf[i].neighbor_global;
            bool done = false;
            if (conc) {  // run revival, else the first free tail slot (the library's drain insert)
                uint64_t b = 0;
                const uint32_t keep = ovf_count;
                done = add_slot_conc(x, nb, b) != 2;
                if (!done) ovf_count = keep;  // a failed drain does not overflow again
                bytes.epoch += b;
                if (!done) { failed++; asym = true; }
                continue;
            }
            for (uint64_t j = rp[x]; j < rp[x + 1]; j++) {
                bytes.epoch += 4;
                uint32_t s = col[j];
                if (s == INV) { col[j] = nb; done = true; edited[x] = 1; break; }
                if (s == nb) { done = true; break; }
            }
            if (!done) { failed++; asym = true; }
        }
        drain_failed += failed;
        return failed;
    }
    uint64_t rebuild_one(uint32_t x, const std::vector<uint32_t>& cols, uint64_t& b) {
        uint64_t m = 0;
        for (uint64_t j = rp[x]; j < re(x); j++) {
            uint32_t ng = col[j];
            b += 4;
            if (ng == INV || ng >= n) continue;
            uint16_t c = (uint16_t)(cols[ng] & 0xFFFFu);
            b += 4;
            if (c != 0 && c <= 64) m |= 1ull << (c - 1);
        }
        return m;
    }
    void rebuild_all(uint64_t& bsum) {
        uint64_t b = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : b)
        for (int64_t xi = 0; xi < (int64_t)n; xi++) {
            uint32_t x = (uint32_t)xi;
            b += 4;
            if (hdmap[x] != EMPTY) continue;
            bm[x] = rebuild_one(x, st, b);
            b += 8;
        }
        bsum += b;
    }
    // Reads the overflow count, resets it, drains (streamgc.cu:967-995).
    uint64_t drain_pending() {
        uint32_t cnt = ovf_count;
        if (cnt == 0) return 0;
        ovf_count = 0;
        return drain(std::min(cnt, OVF_CAP));
    }
    // Reference epoch: snapshot, compact, drain, rebuild (streamgc.cu:949-1012).
    void epoch() {
        snapshot();
        compact_all();
        drain_pending();
        rebuild_all(bytes.epoch);
    }
    // drain_and_compact (streamgc.cu:1243-1314).
    uint64_t drain_and_compact() {
        if (conc) compact_conc(true);
        else compact_all();
        uint64_t f = drain_pending();
        rebuild_all(bytes.epoch);
        return f;
    }

    // -------- Tier-1 (conflict_repair.cu:10-114), Jacobi sweep --------
    uint32_t tier1_sweep() {
        std::vector<uint32_t> old = st;  // colors every decision reads
        uint32_t count = 0;
        uint64_t b = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : count, b)
        for (int64_t xi = 0; xi < (int64_t)n; xi++) {
            uint32_t x = (uint32_t)xi;
            uint16_t my = (uint16_t)(old[x] & 0xFFFFu);
            uint16_t myver = (uint16_t)(old[x] >> 16);
            b += 4 + 16;
            bool has = false;
            for (uint64_t j = rp[x]; j < rp[x + 1] && !has; j++) {
                b += 4;
                if (col[j] != INV) has = true;
            }
            if (my == 0) {
                if (has) {
                    uint16_t c = fac(x, old, b);
                    st[x] = sgc_pack_state(c, (uint16_t)(myver + 1));
                    b += 4;
                    count++;
                }
                continue;
            }
            uint64_t myp = prio(x);
            if (abl_live_deg) {  // live entries of the (compact) row
                uint32_t live = 0;
                for (uint64_t j = rp[x]; j < rp[x + 1]; j++) live += col[j] != INV;
                myp = ((uint64_t)live << 32) | x;
            }
            b += 4;
            bool need = false;
            for (uint64_t j = rp[x]; j < rp[x + 1]; j++) {
                uint32_t ng = col[j];
                b += 4;
                if (ng == INV || ng >= n) continue;
                uint16_t nc = (uint16_t)(old[ng] & 0xFFFFu);
                b += 4;
                if (nc == my && nc != 0) {
                    b += 4;
                    if (myp < prio(ng)) { need = true; break; }
                }
            }
            if (need) {
                count++;
                if (my <= 64) { bm[x] |= 1ull << (my - 1); b += 16; }
                uint16_t c = fac(x, old, b);
                st[x] = sgc_pack_state(c, (uint16_t)(myver + 1));
                b += 4;
            }
        }
        bytes.tier1 += b;
        return count;
    }
    // Independent-set sweep (exact selection): flag every vertex the reference
    // rule would recolor, then recolor only those with no flagged neighbor of
    // higher priority, each to the first color its neighbors leave free
    // (start-of-sweep colors). Returns the number flagged.
    // Selection order of the independent-set rule: the "lowbias32" mixer
    // (C. Wellons, hash-prospector) of x ^ salt, id as tie-break; the salt is
    // (sweep + 1) * 0x9E3779B9 for the sweep's index within its repair.
    static uint64_t sel_rank(uint32_t x, uint32_t salt) {
        uint32_t h = x ^ salt;
        h ^= h >> 16;
        h *= 0x7feb352du;
        h ^= h >> 15;
        h *= 0x846ca68bu;
        h ^= h >> 16;
        return ((uint64_t)h << 32) | x;
    }

    uint32_t tier1_indep_sweep(uint32_t sweep) {
        const uint32_t salt = (sweep + 1u) * 0x9E3779B9u;
        std::vector<uint32_t> old = st;
        std::vector<uint8_t> need(n, 0);
        uint32_t count = 0;
        uint64_t b = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : count, b)
        for (int64_t xi = 0; xi < (int64_t)n; xi++) {
            uint32_t x = (uint32_t)xi;
            uint16_t my = (uint16_t)(old[x] & 0xFFFFu);
            bool has = false, conf = false;
            for (uint64_t j = rp[x]; j < re(x); j++) {
                uint32_t ng = col[j];
                b += 4;
                if (hole(ng)) continue;
                has = true;
                if (my == 0 || ng >= n) continue;
                b += 4;
                if ((uint16_t)(old[ng] & 0xFFFFu) == my && prio(x) < prio(ng)) conf = true;
            }
            bool d = (my == 0) ? has : conf;
            if (d) {
                need[x] = 1;
                count++;
                if (my != 0 && my <= 64) { bm[x] |= 1ull << (my - 1); b += 16; }
            }
        }
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : b)
        for (int64_t xi = 0; xi < (int64_t)n; xi++) {
            uint32_t x = (uint32_t)xi;
            if (!need[x]) continue;
            bool blocked = false;
            for (uint64_t j = rp[x]; j < re(x) && !blocked; j++) {
                uint32_t y = col[j];
                b += 4;
                if (y == INV || y >= n || y == x) continue;
                if (need[y] && sel_rank(x, salt) < sel_rank(y, salt)) blocked = true;
            }
            if (blocked) continue;
            uint16_t c = fac(x, old, b);
            st[x] = sgc_pack_state(c, (uint16_t)((old[x] >> 16) + 1));
        }
        bytes.tier1 += b;
        return count;
    }

    // run_conflict_repair loop (streamgc.cu:1317-1393). Returns iterations run;
    // *last_count = conflicts counted by the last sweep.
    int tier1(uint32_t* history, int hist_cap, uint32_t* last_count) {
        if (exact) {  // independent-set rule: counts only fall; up to 64 sweeps
            uint32_t cnt = 0;
            for (int it = 0; it < 64; it++) {
                rebuild_all(bytes.tier1);
                cnt = tier1_indep_sweep((uint32_t)it);
                if (history && it < hist_cap) history[it] = cnt;
                if (cnt == 0) { if (last_count) *last_count = 0; return it + 1; }
            }
            if (last_count) *last_count = cnt;
            return 64;
        }
        uint32_t prev = UINT32_MAX;
        int plateau = 0;
        uint32_t cnt = 0;
        for (int it = 0; it < 20; it++) {
            rebuild_all(bytes.tier1);
            cnt = tier1_sweep();
            if (history && it < hist_cap) history[it] = cnt;
            if (cnt == 0) { if (last_count) *last_count = 0; return it + 1; }
            if (cnt == prev) {
                plateau++;
                if (plateau >= 3) { if (last_count) *last_count = cnt; return it + 1; }
            } else {
                plateau = 0;
            }
            prev = cnt;
        }
        if (last_count) *last_count = cnt;
        return 20;
    }

    // -------- mirror checksum and properness --------
    // Sum over live entries x->y (y < n, y != x) of H(x,y) - H(y,x): zero when
    // every entry has its mirror (the library's first-sweep checksum).
    static uint64_t pair_hash(uint32_t x, uint32_t y) {
        const uint64_t z = (((uint64_t)x << 32) | y) * 0x9E3779B97F4A7C15ull;
        return z ^ (z >> 29);
    }
    uint64_t mirror_sum() const {
        uint64_t sum = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : sum)
        for (int64_t xi = 0; xi < (int64_t)n; xi++) {
            const uint32_t x = (uint32_t)xi;
            for (uint64_t j = rp[x]; j < re(x); j++) {
                const uint32_t y = col[j];
                if (y >= n || y == x) continue;
                sum += pair_hash(x, y) - pair_hash(y, x);
            }
        }
        return sum;
    }
    // No live edge joins two equal nonzero colors and no vertex with a live
    // entry is uncolored.
    bool is_proper() const {
        for (uint32_t x = 0; x < n; x++)
            for (uint64_t j = rp[x]; j < re(x); j++) {
                const uint32_t y = col[j];
                if (hole(y)) continue;
                if (color(x) == 0) return false;
                if (y < n && y != x && color(y) == color(x)) return false;
            }
        return true;
    }

    // -------- independent-set repair (exact selection) --------
    // Starts from worklist W (every vertex for a full repair, else the vertices
    // touched by updates since the last repair). A sweep visits its worklist
    // only (start-of-sweep colors): it rebuilds their bitmaps and finds the
    // conflicted ones; a same-colored neighbor that loses to a visited vertex
    // joins the next worklist, as does every conflicted vertex the
    // independent-set rule blocks. A recolored vertex ORs its new color (1..64)
    // into its neighbors' bitmaps. Stops when the next worklist is empty (up to
    // 64 sweeps). Returns sweeps run.
    int tier1_worklist(std::vector<uint32_t> W, uint32_t* last_count, bool* done) {
        std::vector<uint8_t> needf(n, 0), nextf(n, 0);
        *done = false;
        uint32_t count = 0;
        for (int it = 0; it < 64; it++) {
            const std::vector<uint32_t> old = st;
            std::vector<uint32_t> need;
            for (uint32_t x : W) {
                const uint16_t my = (uint16_t)(old[x] & 0xFFFFu);
                uint64_t bits = 0;
                bool has = false, conf = false;
                for (uint64_t j = rp[x]; j < re(x); j++) {
                    const uint32_t ng = col[j];
                    if (hole(ng)) continue;
                    has = true;
                    if (ng >= n) continue;
                    const uint16_t c = (uint16_t)(old[ng] & 0xFFFFu);
                    if (c != 0 && c <= 64) bits |= 1ull << (c - 1);
                    if (my != 0 && c == my) {
                        if (prio(x) < prio(ng)) conf = true;
                        else if (ng != x) nextf[ng] = 1;
                    }
                }
                const bool d = (my == 0) ? has : conf;
                const uint64_t own = (d && my != 0 && my <= 64) ? 1ull << (my - 1) : 0ull;
                if (hdmap[x] == EMPTY) bm[x] = bits | own;
                else bm[x] |= own;
                needf[x] = d ? 1 : 0;
                if (d) need.push_back(x);
            }
            count = (uint32_t)need.size();
            const uint32_t salt = (uint32_t)(it + 1) * 0x9E3779B9u;
            std::vector<uint32_t> recolored;
            uint64_t b = 0;
            for (uint32_t x : need) {
                bool blocked = false;
                for (uint64_t j = rp[x]; j < re(x) && !blocked; j++) {
                    const uint32_t y = col[j];
                    if (y >= n || y == x) continue;
                    if (needf[y] && sel_rank(x, salt) < sel_rank(y, salt)) blocked = true;
                }
                if (blocked) { nextf[x] = 1; continue; }
                const uint16_t c = fac(x, old, b);
                st[x] = sgc_pack_state(c, (uint16_t)((old[x] >> 16) + 1));
                recolored.push_back(x);
            }
            bytes.tier1 += b;
            for (uint32_t x : recolored) {
                needf[x] = 0;
                const uint16_t c = color(x);
                if (c == 0 || c > 64) continue;
                for (uint64_t j = rp[x]; j < re(x); j++) {
                    const uint32_t y = col[j];
                    if (y < n) bm[y] |= 1ull << (c - 1);
                }
            }
            W.clear();
            for (uint32_t x = 0; x < n; x++)
                if (nextf[x]) { W.push_back(x); nextf[x] = 0; }
            if (W.empty()) {
                *done = true;
                if (last_count) *last_count = count;
                return it + 1;
            }
        }
        if (last_count) *last_count = count;
        return 64;
    }

    // One repair of the exact-selection configuration (the library's
    // sgc_publish / sgc_repair): incremental when the last repair ended proper,
    // the rows are known mirror-complete and no full repair is due or forced;
    // else full: the first sweep visits every vertex (and computes the mirror
    // checksum when the rows are not known mirror-complete). Tier-2 runs unless
    // the sweeps converged on mirror-complete rows. out: [sweeps, last count, incremental,
    // tier2 ran, proper, tier2 fixes].
    void repair_exact(bool force, uint32_t* out) {
        const bool incr = clean && !force && !asym && !(full_every && since_full + 1 >= full_every);
        uint32_t last = 0;
        int iters = 0;
        bool done = false, sym_bad = false;
        std::vector<uint32_t> W;
        for (uint32_t x = 0; x < n; x++)
            if (!incr || touched[x]) W.push_back(x);
        std::fill(touched.begin(), touched.end(), (uint8_t)0);
        if (!incr && asym) {
            sym_bad = mirror_sum() != 0;
            if (!sym_bad) asym = false;
        }
        iters = tier1_worklist(std::move(W), &last, &done);
        since_full = incr ? since_full + 1 : 0;
        bool proper = done && !sym_bad;
        bool t2 = false;
        uint32_t fixed = 0;
        if (!proper) {
            fixed = tier2();
            t2 = true;
            proper = is_proper();
        }
        clean = proper;
        if (out) {
            out[0] = (uint32_t)iters;
            out[1] = last;
            out[2] = incr ? 1 : 0;
            out[3] = t2 ? 1 : 0;
            out[4] = proper ? 1 : 0;
            out[5] = fixed;
        }
    }

    // -------- Tier-2 (streamgc.cu:1057-1240) --------
    uint32_t tier2() {
        std::vector<std::vector<uint32_t>> adj(n);
        {
            std::vector<uint32_t> d(n, 0);
            for (uint32_t x = 0; x < n; x++)
                for (uint64_t j = rp[x]; j < re(x); j++) {
                    uint32_t y = col[j];
                    if (y != INV && y < n && y != x) { d[x]++; d[y]++; }
                }
            for (uint32_t x = 0; x < n; x++) if (d[x]) adj[x].reserve(d[x]);
            for (uint32_t x = 0; x < n; x++)
                for (uint64_t j = rp[x]; j < re(x); j++) {
                    uint32_t y = col[j];
                    bytes.tier2 += 4;
                    if (y == INV || y >= n || y == x) continue;
                    adj[x].push_back(y);
                    adj[y].push_back(x);
                }
        }
        auto greedy = [&](uint32_t v) -> bool {
            bool used[1024];
            std::memset(used, 0, sizeof(used));
            for (uint32_t w : adj[v]) {
                uint16_t nc = color(w);
                bytes.tier2 += 4;
                if (nc != 0 && nc < 1024) used[nc] = true;
            }
            for (uint16_t c = 1; c < 1024; c++) {
                if (!used[c]) {
                    if (color(v) != c) {
                        st[v] = sgc_pack_state(c, (uint16_t)(ver(v) + 1));
                        bytes.tier2 += 4;
                        return true;
                    }
                    return false;
                }
            }
            return false;
        };
        uint32_t total = 0;
        for (uint32_t u = 0; u < n; u++) {
            if (color(u) != 0 || adj[u].empty()) continue;
            if (greedy(u)) total++;
        }
        for (int pass = 0; pass < 30; pass++) {
            std::vector<uint32_t> fix;
            for (uint32_t u = 0; u < n; u++)
                for (uint32_t v : adj[u]) {
                    if (v <= u) continue;
                    if (color(u) == color(v) && color(u) != 0) fix.push_back(v);
                }
            if (fix.empty()) break;
            std::sort(fix.begin(), fix.end());
            fix.erase(std::unique(fix.begin(), fix.end()), fix.end());
            uint32_t fixed = 0;
            for (uint32_t v : fix) if (greedy(v)) fixed++;
            total += fixed;
            if (fixed == 0) break;
        }
        return total;
    }
};

// ---------------- stream generators (stream_gen.cpp) ----------------
struct PairHash {
    size_t operator()(const std::pair<uint32_t, uint32_t>& p) const {
        return std::hash<uint64_t>()((uint64_t)p.first << 32 | p.second);
    }
};

}  // namespace

extern "C" {

// ---------------- lifecycle ----------------

// Builds the single-GPU slack CSR exactly as allocate_gpu_partition
// (streamgc.cu:350-433): cap = max(d + d*slack/100, 8), base edges first in
// loader order, the rest INVALID. High-degree rows: degree > threshold
// (streamgc.cu:225-250), histogram row index in vertex order.
void* og_create(uint32_t n, const uint64_t* row_ptr, const uint32_t* col_idx, const uint32_t* degree,
                uint32_t hist_thr, uint32_t slack_pct, uint32_t max_hist_colors, uint32_t flags) {
    Oracle* g = new Oracle();
    g->exact = (flags & 1u) != 0;
    g->conc = g->exact && (flags & 2u) != 0;
    g->abl_force_bitmap = (flags & 4u) != 0;
    g->abl_no_overflow = (flags & 8u) != 0;
    g->abl_live_deg = (flags & 16u) != 0;
    g->n = n;
    g->hist_thr = hist_thr;
    g->maxc = max_hist_colors ? max_hist_colors : SGC_MAX_HISTOGRAM_COLORS_DEFAULT;
    g->rp.assign((size_t)n + 1, 0);
    for (uint32_t x = 0; x < n; x++) {
        uint32_t cnt = (uint32_t)(row_ptr[x + 1] - row_ptr[x]);
        uint32_t extra = (uint32_t)(((uint64_t)cnt * slack_pct) / 100);
        uint32_t cap = std::max<uint32_t>(cnt + extra, 8u);
        g->rp[x + 1] = g->rp[x] + cap;
    }
    g->col.assign(g->rp[n], INV);
    for (uint32_t x = 0; x < n; x++) {
        uint64_t p = g->rp[x];
        for (uint64_t j = row_ptr[x]; j < row_ptr[x + 1]; j++) g->col[p++] = col_idx[j];
    }
    g->st.assign(n, 0);
    g->bm.assign(n, 0);
    g->edited.assign(n, 0);
    g->base_len.resize(n);
    for (uint32_t x = 0; x < n; x++) {
        g->base_len[x] = (uint32_t)(row_ptr[x + 1] - row_ptr[x]);
        for (uint64_t j = row_ptr[x] + 1; j < row_ptr[x + 1]; j++)
            if (col_idx[j - 1] >= col_idx[j]) { g->edited[x] = 1; break; }  // not strictly ascending: scan it
    }
    g->deg.assign(degree, degree + n);
    g->hdmap.assign(n, EMPTY);
    for (uint32_t x = 0; x < n; x++)
        if (degree[x] > hist_thr) g->hdmap[x] = g->num_hd++;
    g->hist.assign(g->exact ? 0 : (size_t)g->num_hd * g->maxc, 0);
    g->snap.assign(n, 0);
    g->ovf.resize(OVF_CAP);
    g->touched.assign(n, 0);
    if (g->conc) {  // marks at the base counts; sorted base rows are runs
        g->mhw.resize(n);
        g->mbl.resize(n);
        g->mholes.assign(n, 0);
        g->mdirty.assign(n, 0);
        for (uint32_t x = 0; x < n; x++) {
            g->mhw[x] = g->base_len[x];
            g->mbl[x] = g->edited[x] ? 0u : g->base_len[x];
        }
    }
    return g;
}

// Concurrent rules: per-row high-water marks, base-run lengths and hole
// counts taken from elsewhere (the library's state after load_state); rows
// with holes are compaction candidates.
void og_load_rows_model(void* h, const uint32_t* hw, const uint32_t* blen, const uint32_t* holes) {
    Oracle* g = (Oracle*)h;
    if (!g->conc) return;
    for (uint32_t x = 0; x < g->n; x++) {
        const uint32_t cap = (uint32_t)(g->rp[x + 1] - g->rp[x]);
        g->mhw[x] = hw[x] < cap ? hw[x] : cap;
        g->mbl[x] = blen[x] < g->mhw[x] ? blen[x] : g->mhw[x];
        g->mholes[x] = holes[x];
        g->mdirty[x] = holes[x] ? 1 : 0;
    }
}

void og_destroy(void* h) { delete (Oracle*)h; }

uint32_t og_num_vertices(void* h) { return ((Oracle*)h)->n; }
uint64_t og_total_slots(void* h) { return ((Oracle*)h)->rp.back(); }
uint32_t og_num_high_degree(void* h) { return ((Oracle*)h)->exact ? 0 : ((Oracle*)h)->num_hd; }
uint32_t og_max_hist_colors(void* h) { return ((Oracle*)h)->maxc; }

// ---------------- updates and epochs ----------------

void og_apply(void* h, const EdgeUpdate* ups, uint64_t n) {
    Oracle* g = (Oracle*)h;
    for (uint64_t i = 0; i < n; i++) g->apply_one(ups[i]);
    g->batch_end(ups, n);
}
void og_epoch(void* h) { ((Oracle*)h)->epoch(); }
uint64_t og_drain_and_compact(void* h) { return ((Oracle*)h)->drain_and_compact(); }
void og_snapshot(void* h) { ((Oracle*)h)->snapshot(); }
void og_compact(void* h) { ((Oracle*)h)->compact_all(); }
uint64_t og_drain_pending(void* h) { return ((Oracle*)h)->drain_pending(); }
void og_rebuild_bitmaps(void* h) { Oracle* g = (Oracle*)h; g->rebuild_all(g->bytes.epoch); }
uint32_t og_tier1_sweep(void* h) { return ((Oracle*)h)->tier1_sweep(); }
int og_tier1(void* h, uint32_t* history, int hist_cap, uint32_t* last_count) {
    return ((Oracle*)h)->tier1(history, hist_cap, last_count);
}
uint32_t og_tier2(void* h) { return ((Oracle*)h)->tier2(); }

// process_stream for one GPU (streamgc.cu:809-1053) in stream order: host
// batches of `batch` updates, epoch when updates_since_epoch >= epoch_size,
// checked after each batch. Returns the number of epoch boundaries.
uint32_t og_process_stream(void* h, const EdgeUpdate* ups, uint64_t n, uint32_t epoch_size, uint32_t batch) {
    Oracle* g = (Oracle*)h;
    uint64_t processed = 0, since = 0;
    uint32_t epochs = 0;
    if (batch == 0) batch = SGC_HOST_BATCH_SIZE;
    while (processed < n) {
        uint64_t b = std::min<uint64_t>(batch, n - processed);
        for (uint64_t i = 0; i < b; i++) g->apply_one(ups[processed + i]);
        g->batch_end(ups + processed, b);
        processed += b;
        since += b;
        if (since >= epoch_size) { g->epoch(); since = 0; epochs++; }
    }
    return epochs;
}

// Phase end exactly as main() does after each stream (streamgc.cu:1405-1408):
// drain_and_compact, Tier-1 loop, Tier-2. Returns tier-2 fixes; tier-1
// iterations and last count through the out pointers.
uint32_t og_phase_end(void* h, int* t1_iters, uint32_t* t1_last) {
    Oracle* g = (Oracle*)h;
    g->drain_and_compact();
    if (g->exact) {  // the library's phase end: a forced full repair
        uint32_t out[6];
        g->repair_exact(true, out);
        if (t1_iters) *t1_iters = (int)out[0];
        if (t1_last) *t1_last = out[1];
        return out[5];
    }
    uint32_t last = 0;
    int it = g->tier1(nullptr, 0, &last);
    if (t1_iters) *t1_iters = it;
    if (t1_last) *t1_last = last;
    return g->tier2();
}

// One repair as the library's sgc_publish does it (exact selection only):
// compact, drain, repair (incremental when allowed), snapshot. out: [sweeps,
// last count, incremental, tier2 ran, proper, tier2 fixes].
void og_publish_repair(void* h, int force_full, uint32_t* out) {
    Oracle* g = (Oracle*)h;
    g->compact_all();
    g->drain_pending();
    g->repair_exact(force_full != 0, out);
    g->snapshot();
}
void og_set_full_repair_every(void* h, uint32_t every) { ((Oracle*)h)->full_every = every; }
// Sets the repair bookkeeping (e.g. to continue from a state loaded with
// og_load_state that a proper repair produced on mirror-complete rows).
void og_set_repair_state(void* h, int clean, int asym) {
    Oracle* g = (Oracle*)h;
    g->clean = clean != 0;
    g->asym = asym != 0;
}

// Epoch with repair-before-publish (the concurrent mode's epoch): compact,
// drain, Tier-1 loop, Tier-2, then snapshot. Stream batches of min(E, batch).
uint32_t og_process_stream_repaired(void* h, const EdgeUpdate* ups, uint64_t n, uint32_t epoch_size,
                                    uint32_t batch) {
    Oracle* g = (Oracle*)h;
    if (batch == 0) batch = SGC_HOST_BATCH_SIZE;
    uint64_t step = std::min<uint64_t>(batch, epoch_size ? epoch_size : batch);
    uint64_t processed = 0, since = 0;
    uint32_t epochs = 0;
    while (processed < n) {
        uint64_t b = std::min<uint64_t>(step, n - processed);
        for (uint64_t i = 0; i < b; i++) g->apply_one(ups[processed + i]);
        g->batch_end(ups + processed, b);
        processed += b;
        since += b;
        if (since >= epoch_size) {
            g->compact_all();
            g->drain_pending();
            if (g->exact) {
                g->repair_exact(false, nullptr);
            } else {
                g->tier1(nullptr, 0, nullptr);
                g->tier2();
            }
            g->snapshot();
            since = 0;
            epochs++;
        }
    }
    return epochs;
}

// Overwrites slots, states, bitmaps and histograms with a state taken from
// elsewhere (same row layout). A row whose slots differ from the current ones
// is marked edited. Used to time the CPU path from the same starting state.
void og_load_state(void* h, const uint32_t* col, const uint32_t* states, const uint64_t* bitmaps,
                   const uint32_t* hist) {
    Oracle* g = (Oracle*)h;
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t xi = 0; xi < (int64_t)g->n; xi++) {
        const uint32_t x = (uint32_t)xi;
        if (std::memcmp(&g->col[g->rp[x]], col + g->rp[x], (g->rp[x + 1] - g->rp[x]) * 4)) g->edited[x] = 1;
    }
    std::memcpy(g->col.data(), col, g->col.size() * 4);
    std::memcpy(g->st.data(), states, g->n * 4ull);
    std::memcpy(g->bm.data(), bitmaps, g->n * 8ull);
    std::memcpy(g->hist.data(), hist, g->hist.size() * 4ull);
    g->clean = false;
    g->asym = true;
}

// The same for a state too large to hold twice in host memory: the caller
// first writes the slots straight into the oracle's slab (og_col_data, same
// row layout), then this marks as edited every row whose slots differ from
// its base row (row_ptr/col_idx, INV after it) and copies the rest.
uint32_t* og_col_data(void* h) { return ((Oracle*)h)->col.data(); }
void og_load_state_inplace(void* h, const uint64_t* row_ptr, const uint32_t* col_idx, const uint32_t* states,
                           const uint64_t* bitmaps, const uint32_t* hist) {
    Oracle* g = (Oracle*)h;
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t xi = 0; xi < (int64_t)g->n; xi++) {
        const uint32_t x = (uint32_t)xi;
        const uint64_t cnt = row_ptr[x + 1] - row_ptr[x], cap = g->rp[x + 1] - g->rp[x];
        const uint32_t* row = &g->col[g->rp[x]];
        bool same = std::memcmp(row, col_idx + row_ptr[x], cnt * 4) == 0;
        for (uint64_t j = cnt; same && j < cap; j++) same = row[j] == INV;
        if (!same) g->edited[x] = 1;
    }
    std::memcpy(g->st.data(), states, g->n * 4ull);
    std::memcpy(g->bm.data(), bitmaps, g->n * 8ull);
    if (hist) std::memcpy(g->hist.data(), hist, g->hist.size() * 4ull);
    g->clean = false;
    g->asym = true;
}

// ---------------- state access ----------------
void og_get_states(void* h, uint32_t* out) { Oracle* g = (Oracle*)h; std::memcpy(out, g->st.data(), g->n * 4ull); }
void og_set_states(void* h, const uint32_t* in) {
    Oracle* g = (Oracle*)h;
    std::memcpy(g->st.data(), in, g->n * 4ull);
    g->clean = false;  // colors from elsewhere: the next repair visits every vertex
}
void og_get_bitmaps(void* h, uint64_t* out) { Oracle* g = (Oracle*)h; std::memcpy(out, g->bm.data(), g->n * 8ull); }
void og_get_hdmap(void* h, uint32_t* out) { Oracle* g = (Oracle*)h; std::memcpy(out, g->hdmap.data(), g->n * 4ull); }
void og_get_hist(void* h, uint32_t* out) {
    Oracle* g = (Oracle*)h;
    std::memcpy(out, g->hist.data(), g->hist.size() * 4ull);
}
void og_get_row_ptr(void* h, uint64_t* out) { Oracle* g = (Oracle*)h; std::memcpy(out, g->rp.data(), (g->n + 1ull) * 8); }
void og_get_col(void* h, uint32_t* out) { Oracle* g = (Oracle*)h; std::memcpy(out, g->col.data(), g->col.size() * 4ull); }
void og_get_snapshot(void* h, uint16_t* out) { Oracle* g = (Oracle*)h; std::memcpy(out, g->snap.data(), g->n * 2ull); }
uint32_t og_overflow_count(void* h) { return ((Oracle*)h)->ovf_count; }
void og_get_overflow(void* h, uint32_t* out_pairs, uint32_t cnt) {
    Oracle* g = (Oracle*)h;
    for (uint32_t i = 0; i < cnt && i < OVF_CAP; i++) {
        out_pairs[2 * i] = g->ovf[i].local_vertex_idx;
        out_pairs[2 * i + 1] = g->ovf[i].neighbor_global;
    }
}
// counters: [updates_applied, skipped, recolors, ovf_lost, drain_failed,
//            bytes.update, bytes.epoch, bytes.tier1, bytes.tier2]
void og_counters(void* h, uint64_t* out) {
    Oracle* g = (Oracle*)h;
    out[0] = g->updates_applied; out[1] = g->skipped_updates; out[2] = g->recolors;
    out[3] = g->ovf_lost; out[4] = g->drain_failed;
    out[5] = g->bytes.update; out[6] = g->bytes.epoch; out[7] = g->bytes.tier1; out[8] = g->bytes.tier2;
}
void og_reset_bytes(void* h) { ((Oracle*)h)->bytes = Bytes(); }

// ---------------- color selection probe (known-answer tests) ----------------
// Sets vertex x's bitmap / histogram row and returns FindAvailableColor(x).
uint16_t og_fac(void* h, uint32_t x) {
    Oracle* g = (Oracle*)h;
    uint64_t b = 0;
    return g->fac(x, g->st, b);
}
void og_set_bitmap(void* h, uint32_t x, uint64_t v) { ((Oracle*)h)->bm[x] = v; }
void og_set_hist_row(void* h, uint32_t x, const uint32_t* vals, uint32_t cnt) {
    Oracle* g = (Oracle*)h;
    uint32_t* r = g->hrow(x);
    if (!r) return;
    for (uint32_t i = 0; i < cnt && i < g->maxc; i++) r[i] = vals[i];
}

// ---------------- validator (streamgc.cu:448-556) ----------------
// out: [violations, uncolored_with_edges, distinct_edges, max_color, entries_out_of_range]
void og_validate(void* h, uint64_t* out) {
    Oracle* g = (Oracle*)h;
    std::unordered_set<uint64_t> es;
    std::vector<uint32_t> eff(g->n, 0);
    uint64_t oor = 0;
    for (uint32_t x = 0; x < g->n; x++)
        for (uint64_t j = g->rp[x]; j < g->rp[x + 1]; j++) {
            uint32_t y = g->col[j];
            if (g->hole(y)) continue;
            if (y >= g->n) { oor++; continue; }
            eff[x]++;
            uint32_t lo = std::min(x, y), hi = std::max(x, y);
            es.insert(((uint64_t)lo << 32) | hi);
        }
    uint64_t viol = 0;
    for (uint64_t e : es) {
        uint32_t a = (uint32_t)(e >> 32), b = (uint32_t)e;
        if (g->color(a) == g->color(b) && g->color(a) != 0) viol++;
    }
    uint64_t unc = 0;
    uint16_t mx = 0;
    for (uint32_t x = 0; x < g->n; x++) {
        if (g->color(x) == 0 && eff[x] > 0) unc++;
        mx = std::max(mx, g->color(x));
    }
    out[0] = viol; out[1] = unc; out[2] = es.size(); out[3] = mx; out[4] = oor;
}

// Same checks for an arbitrary color vector against a base CSR (u64 offsets).
void og_validate_colors(uint32_t n, const uint64_t* rp, const uint32_t* col, const uint16_t* colors, uint64_t* out) {
    uint64_t viol = 0, unc = 0;
    uint16_t mx = 0;
    for (uint32_t x = 0; x < n; x++) {
        bool hasn = false;
        for (uint64_t j = rp[x]; j < rp[x + 1]; j++) {
            uint32_t y = col[j];
            if (y == INV || y >= n) continue;
            hasn = true;
            if (x <= y && colors[x] == colors[y] && colors[x] != 0) viol++;
        }
        if (colors[x] == 0 && hasn) unc++;
        mx = std::max(mx, colors[x]);
    }
    out[0] = viol; out[1] = unc; out[2] = mx;
}

// First-fit coloring of the live rows in id order (the static greedy of
// streamgc.cu:559-592 applied to the current rows), each color with version 1,
// then the bitmaps of the bitmap-mode rows rebuilt. The result is proper on
// mirror-complete rows, so the next repair may start from touched vertices.
// Returns the largest color.
uint16_t og_color_greedy(void* h) {
    Oracle* g = (Oracle*)h;
    const uint32_t n = g->n;
    std::vector<uint32_t> used(4096, 0);
    uint32_t stamp = 0;
    uint16_t mx = 0;
    for (uint32_t v = 0; v < n; v++) {
        stamp++;
        for (uint64_t j = g->rp[v]; j < g->re(v); j++) {
            const uint32_t y = g->col[j];
            if (y >= n) continue;
            const uint16_t c = g->color(y);
            if (c && c < used.size()) used[c] = stamp;
        }
        uint16_t k = 1;
        while (k < used.size() && used[k] == stamp) k++;
        g->st[v] = sgc_pack_state(k, 1);
        if (k > mx) mx = k;
    }
    uint64_t b = 0;
    g->rebuild_all(b);
    std::fill(g->touched.begin(), g->touched.end(), (uint8_t)0);
    g->clean = true;
    g->asym = false;
    return mx;
}

// The library's sgc_color_core: the uncolored vertices of initial degree >=
// min_degree one at a time in descending degree order (ties by id), each with
// the first color in 1..2047 none of its live neighbors holds (2048 when all
// do), version 1. Returns how many were colored.
uint32_t og_color_core(void* h, uint32_t min_degree) {
    Oracle* g = (Oracle*)h;
    std::vector<uint32_t> list;
    for (uint32_t x = 0; x < g->n; x++)
        if (g->deg[x] >= min_degree && g->deg[x] > 0) list.push_back(x);
    std::sort(list.begin(), list.end(), [&](uint32_t a, uint32_t b) {
        return g->deg[a] != g->deg[b] ? g->deg[a] > g->deg[b] : a < b;
    });
    uint32_t done = 0;
    std::vector<uint8_t> used(2048);
    for (uint32_t v : list) {
        if (g->color(v) != 0) continue;
        std::fill(used.begin(), used.end(), (uint8_t)0);
        for (uint64_t j = g->rp[v]; j < g->re(v); j++) {
            const uint32_t y = g->col[j];
            if (y >= g->n) continue;
            const uint16_t c = g->color(y);
            if (c != 0 && c < 2048) used[c] = 1;
        }
        uint16_t c = 1;
        while (c < 2048 && used[c]) c++;
        g->st[v] = sgc_pack_state(c, 1);
        done++;
    }
    g->clean = false;
    return done;
}

// ---------------- static greedy (streamgc.cu:559-592) ----------------
uint16_t og_static_greedy(uint32_t n, const uint64_t* rp, const uint32_t* col) {
    std::vector<uint16_t> c(n, 0);
    std::vector<bool> used((size_t)n + 1, false);
    for (uint32_t v = 0; v < n; v++) {
        for (uint64_t j = rp[v]; j < rp[v + 1]; j++) if (c[col[j]]) used[c[col[j]]] = true;
        uint16_t k = 1;
        while (used[k]) k++;
        c[v] = k;
        for (uint64_t j = rp[v]; j < rp[v + 1]; j++) if (c[col[j]]) used[c[col[j]]] = false;
    }
    uint16_t mx = 0;
    for (uint32_t v = 0; v < n; v++) mx = std::max(mx, c[v]);
    return mx;
}

// ---------------- stream generators (stream_gen.cpp:30-177) ----------------
// Init stream: u<v edges in CSR order, std::sort by (min deg desc, max deg desc).
// out must hold nnz/2 pairs; returns count.
uint64_t og_gen_init_stream(uint32_t n, const uint64_t* rp, const uint32_t* col, const uint32_t* degree,
                            uint32_t* out_pairs) {
    std::vector<std::pair<uint32_t, uint32_t>> edges;
    for (uint32_t u = 0; u < n; u++)
        for (uint64_t j = rp[u]; j < rp[u + 1]; j++)
            if (u < col[j]) edges.push_back({u, col[j]});
    std::sort(edges.begin(), edges.end(), [&degree](const auto& a, const auto& b) {
        uint32_t mina = std::min(degree[a.first], degree[a.second]);
        uint32_t minb = std::min(degree[b.first], degree[b.second]);
        if (mina != minb) return mina > minb;
        uint32_t maxa = std::max(degree[a.first], degree[a.second]);
        uint32_t maxb = std::max(degree[b.first], degree[b.second]);
        return maxa > maxb;
    });
    for (size_t i = 0; i < edges.size(); i++) { out_pairs[2 * i] = edges[i].first; out_pairs[2 * i + 1] = edges[i].second; }
    return edges.size();
}

// Churn bench stream (stream_gen.cpp:65-177) through libstdc++'s
// mt19937_64 / uniform_int_distribution. out_pairs: 2*stream_size, out_types: stream_size.
void og_gen_bench_stream(uint32_t n, const uint64_t* rp, const uint32_t* col, uint64_t stream_size,
                         uint32_t insert_pct, uint64_t seed, uint32_t* out_pairs, uint8_t* out_types) {
    std::mt19937_64 rng(seed);
    std::unordered_set<std::pair<uint32_t, uint32_t>, PairHash> live;
    std::vector<std::pair<uint32_t, uint32_t>> live_vec;
    for (uint32_t u = 0; u < n; u++)
        for (uint64_t j = rp[u]; j < rp[u + 1]; j++)
            if (u < col[j]) { live.insert({u, col[j]}); live_vec.push_back({u, col[j]}); }
    std::vector<std::pair<uint32_t, uint32_t>> pool;
    std::uniform_int_distribution<uint32_t> pct(0, 99);
    uint64_t k = 0;
    for (uint64_t i = 0; i < stream_size; i++) {
        bool ins = pct(rng) < insert_pct;
        if (ins) {
            if (!pool.empty()) {
                std::uniform_int_distribution<size_t> pd(0, pool.size() - 1);
                size_t idx = pd(rng);
                auto e = pool[idx];
                pool[idx] = pool.back();
                pool.pop_back();
                live.insert(e);
                live_vec.push_back(e);
                out_pairs[2 * k] = e.first; out_pairs[2 * k + 1] = e.second; out_types[k] = 0; k++;
            } else {
                std::uniform_int_distribution<uint32_t> vd(0, n - 1);
                uint32_t u = vd(rng), v = vd(rng);
                if (u == v) v = (v + 1) % n;
                uint32_t a = std::min(u, v), b = std::max(u, v);
                if (live.find({a, b}) == live.end()) {
                    live.insert({a, b});
                    live_vec.push_back({a, b});
                    out_pairs[2 * k] = a; out_pairs[2 * k + 1] = b; out_types[k] = 0; k++;
                } else {
                    i--;
                    continue;
                }
            }
        } else {
            if (live_vec.empty()) { i--; continue; }
            std::uniform_int_distribution<size_t> ed(0, live_vec.size() - 1);
            size_t idx = ed(rng);
            auto e = live_vec[idx];
            live.erase(e);
            live_vec[idx] = live_vec.back();
            live_vec.pop_back();
            pool.push_back(e);
            out_pairs[2 * k] = e.first; out_pairs[2 * k + 1] = e.second; out_types[k] = 1; k++;
        }
    }
}

// ---------------- graph loader (graph_loader.cpp:29-169) ----------------
// Two-call protocol: og_load_mtx returns a handle; og_loaded_* copy out.
struct Loaded {
    uint32_t n = 0;
    std::vector<uint64_t> rp;
    std::vector<uint32_t> col, deg;
};
void* og_load_mtx(const char* path) {
    FILE* f = fopen(path, "r");
    if (!f) return nullptr;
    char line[4096];
    bool pattern = false;
    if (fgets(line, sizeof(line), f) && strstr(line, "pattern")) pattern = true;
    while (fgets(line, sizeof(line), f)) if (line[0] != '%') break;
    unsigned rows = 0, cols = 0;
    unsigned long long nnz = 0;
    if (sscanf(line, "%u %u %llu", &rows, &cols, &nnz) != 3) { fclose(f); return nullptr; }
    uint32_t n = rows > cols ? rows : cols;
    std::vector<std::pair<uint32_t, uint32_t>> raw;
    raw.reserve(nnz);
    for (uint64_t i = 0; i < nnz; i++) {
        uint32_t u = 0, v = 0;
        if (fscanf(f, "%u %u", &u, &v) != 2) break;
        if (!pattern) { int c; while ((c = fgetc(f)) != '\n' && c != EOF) {} }
        u--; v--;
        if (u == v) continue;
        if (u > v) std::swap(u, v);
        raw.push_back({u, v});
    }
    fclose(f);
    std::sort(raw.begin(), raw.end());
    raw.erase(std::unique(raw.begin(), raw.end()), raw.end());
    Loaded* L = new Loaded();
    L->n = n;
    L->deg.assign(n, 0);
    for (auto& e : raw) { L->deg[e.first]++; L->deg[e.second]++; }
    L->rp.assign((size_t)n + 1, 0);
    for (uint32_t v = 0; v < n; v++) L->rp[v + 1] = L->rp[v] + L->deg[v];
    L->col.assign(raw.size() * 2, 0);
    std::vector<uint64_t> off(L->rp.begin(), L->rp.end() - 1);
    for (auto& e : raw) { L->col[off[e.first]++] = e.second; L->col[off[e.second]++] = e.first; }
    for (uint32_t v = 0; v < n; v++) std::sort(L->col.begin() + L->rp[v], L->col.begin() + L->rp[v + 1]);
    return L;
}
uint32_t og_loaded_n(void* h) { return ((Loaded*)h)->n; }
uint64_t og_loaded_nnz(void* h) { return ((Loaded*)h)->col.size(); }
void og_loaded_copy(void* h, uint64_t* rp, uint32_t* col, uint32_t* deg) {
    Loaded* L = (Loaded*)h;
    std::memcpy(rp, L->rp.data(), L->rp.size() * 8);
    std::memcpy(col, L->col.data(), L->col.size() * 4);
    std::memcpy(deg, L->deg.data(), L->deg.size() * 4);
}
void og_loaded_free(void* h) { delete (Loaded*)h; }

int og_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Threads of the order-independent passes (compaction, rebuild, repair
// decisions, validation); updates stay in stream order on one thread.
void og_set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

}  // extern "C"
