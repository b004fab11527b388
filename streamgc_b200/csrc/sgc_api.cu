// sgc_api.cu -- the C ABI (include/streamgc_b200.h): one handle per graph,
// owning its device state and one CUDA stream. The host side is a thin
// sequencer; every step on the graph runs as a kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/streamgc_b200.h"
#include "sgc_internal.h"

using namespace sgc;

namespace sgci {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

// Scatters the base CSR into the slack layout: warp per row.
__global__ void scatter_base_kernel(uint32_t n, const uint64_t* __restrict__ brp, const uint32_t* __restrict__ bcol,
                                    const uint64_t* __restrict__ rp, uint32_t* __restrict__ col) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; x < n; x += warps) {
        const uint64_t s = brp[x], e = brp[x + 1], d = rp[x];
        for (uint64_t j = s + (threadIdx.x & 31); j < e; j += 32) col[d + (j - s)] = bcol[j];
    }
}

__global__ void find_color_kernel(Dev g, uint32_t x, uint16_t* out) {
    const uint16_t c = warp_fac(g, x, g.st);
    if (lane_id() == 0) *out = c;
}

int check_cuda(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(SGC_ECUDA, "%s: %s", where, cudaGetErrorString(e));
    return SGC_OK;
}

cudaEvent_t take_event(sgc_handle* h) {
    if (!h->ev_pool.empty()) {
        cudaEvent_t e = h->ev_pool.back();
        h->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Gathers the elapsed time of recorded sweeps, whole and per phase (stream must be idle).
void collect_events(sgc_handle* h) {
    for (auto& se : h->ev_pending) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, se.ev[0], se.ev[4]) == cudaSuccess) {
            h->sweep_ms += ms;
            h->sweep_count++;
            for (int k = 0; k < 4; k++)
                if (cudaEventElapsedTime(&ms, se.ev[k], se.ev[k + 1]) == cudaSuccess) h->sweep_phase_ms[k] += ms;
        }
        for (int k = 0; k < 5; k++) h->ev_pool.push_back(se.ev[k]);
    }
    h->ev_pending.clear();
}

int sync(sgc_handle* h) {
    CK(cudaStreamSynchronize(h->stream));
    collect_events(h);
    return SGC_OK;
}

// ---- epoch building blocks ----

// force: compact every edited row (epoch maintenance and phase end, as the
// reference does); publishes under exact selection leave rows with few holes.
int compact_dirty(sgc_handle* h, bool force) {
    CK(cudaMemsetAsync(&h->ctl->dirty_count, 0, 4, h->stream));
    launch_dirty_list(h->g, h->dirty_list, &h->ctl->dirty_count, h->stream);
    launch_compact(h->g, h->dirty_list, &h->ctl->dirty_count, h->n, force, h->stream,
                   (h->opt.flags & SGC_OPT_SORTED_ROWS) != 0);
    h->launches += 2;
    return check_cuda("compact");
}

int drain(sgc_handle* h, bool ordered, unsigned long long* failed_counter) {
    launch_take_overflow(h->g, &h->ctl->drain_n, h->stream);
    launch_drain(h->g, &h->ctl->drain_n, ordered, failed_counter, h->stream);
    h->launches += 2;
    return check_cuda("drain");
}

// A REBUILD sweep over every vertex (epoch maintenance), with optional event
// timing.
int rebuild_sweep(sgc_handle* h) {
    launch_build_items(h->g, h->sb, 0, h->num_sms, h->stream);
    launch_sweep(h->g, h->sb, SWEEP_REBUILD, 0, 0, h->num_sms, h->stream);
    h->launches += 3;
    return check_cuda("rebuild");
}

// The control block's `clean` flag: whether the next repair may start from the
// touched vertices (the current colors are a proper coloring of the rows).
int set_clean(sgc_handle* h, uint32_t v) {
    CK(cudaMemsetAsync(&h->g.gctl->clean, 0, 4, h->stream));
    if (v) CK(cudaMemsetAsync(&h->g.gctl->clean, 1, 1, h->stream));
    return SGC_OK;
}

// Writes the back half of the snapshot and makes it the front. With
// incremental snapshots only the colors changed in the last two epochs are
// copied (plus a full copy while snap_full says so).
void publish_snapshot(sgc_handle* h) {
    const int back = 1 - h->front;
    if (h->g.chg) {
        launch_snapshot_changes(h->g, h->chg_prev, h->snap[back], h->stream);
        h->launches += 1;
    }
    if (!h->g.chg || h->snap_full > 0) {
        launch_snapshot(h->g, h->snap[back], h->stream);
        h->launches += 1;
        if (h->snap_full > 0) h->snap_full--;
    }
    h->front = back;
}

// Tier-1 loop of run_conflict_repair (streamgc.cu:1317-1393) on compact rows,
// driven by the device control block: the host starts it and reads the block
// after each sweep. Tier-2 runs unless convergence on a mirror-complete CSR
// proves it a no-op.
//   Reference rule (deterministic parity): at most 20 sweeps, stop at 0 or after
//   3 equal counts. Independent-set rule (exact color selection): each sweep
//   resolves at least the highest-ranked conflict and creates none; up to 64
//   sweeps. Under it a repair is incremental -- its first sweep visits only the
//   vertices touched by updates since the last repair -- when that repair ended
//   proper, the rows are mirror-complete and `force_full` is off: every new
//   conflict then has an endpoint among the touched vertices.
int repair_loop(sgc_handle* h, sgc_repair_report* rep, bool force_full) {
    const bool indep = h->g.exact != 0;
    const SweepMode mode = indep ? SWEEP_INDEP : SWEEP_TIER1;
    const uint32_t every = h->opt.full_repair_every;
    if (every && h->repairs_since_full + 1 >= every) force_full = true;
    RepairCtl* hin = h->h_rc_in;
    hin->mode = (uint32_t)mode;
    hin->max_sweeps = indep ? 64u : 20u;
    hin->force_all = force_full ? 1u : 0u;
    CK(cudaMemcpyAsync(h->sb.rc, hin, 12, cudaMemcpyHostToDevice, h->stream));
    const size_t mwords = ((h->n + 31) / 32) * 4;
    CK(cudaMemsetAsync(h->sb.wmark, 0, mwords, h->stream));
    CK(cudaMemsetAsync(h->sb.rbits, 0, mwords, h->stream));
    CK(cudaMemsetAsync(h->sb.needf, 0, h->n, h->stream));  // no vertex starts conflicted
    launch_repair_begin(h->g, h->sb, mode, h->num_sms, h->stream);
    h->launches += (mode == SWEEP_INDEP && h->g.touched) ? 2 : 1;
    const bool prof = (h->opt.flags & SGC_OPT_PROFILE) != 0;
    RepairCtl* rc = h->h_rc_out;
    for (uint32_t sweeps = 0;; sweeps++) {
        if (sweeps > hin->max_sweeps) return fail(SGC_EDEVICE, "repair loop ran past %u sweeps", hin->max_sweeps);
        sgc_handle::SweepEvents se{};
        if (prof) {
            for (int k = 0; k < 5; k++) se.ev[k] = take_event(h);
            cudaEventRecord(se.ev[0], h->stream);
        }
        launch_repair_sweep(h->g, h->sb, mode, h->num_sms, h->stream, prof ? se.ev + 1 : nullptr);
        if (prof) {
            cudaEventRecord(se.ev[4], h->stream);
            h->ev_pending.push_back(se);
        }
        launch_repair_step(h->g, h->sb, h->num_sms, h->stream, nullptr);
        h->launches += 1 + (mode == SWEEP_INDEP ? 6 : 4) + 3;
        CK(cudaMemcpyAsync(rc, h->sb.rc, sizeof(RepairCtl), cudaMemcpyDeviceToHost, h->stream));
        h->d2h_bytes += sizeof(RepairCtl);
        TRY(sync(h));
        if (!rc->cont) break;
    }
    TRY(check_cuda("repair"));
    if (prof) {
        unsigned long long sw[2];
        CK(cudaMemcpyAsync(sw, h->sb.swept, 16, cudaMemcpyDeviceToHost, h->stream));
        TRY(sync(h));
        h->sweep_bytes += 8ull * sw[0] + 28ull * sw[1];
    }
    return finish_repair(h, rep);
}

// After the Tier-1 loop (its control block read back into h_rc_out): the
// counters, and Tier-2 when the loop did not leave a proper coloring.
int finish_repair(sgc_handle* h, sgc_repair_report* rep) {
    const RepairCtl* rc = h->h_rc_out;
    h->tier1_sweeps += rc->it;
    if (!rc->incr) h->live_entries = rc->live;
    h->repairs_since_full = rc->incr ? h->repairs_since_full + 1 : 0;
    sgc_repair_report r{};
    r.tier1_iterations = rc->it;
    r.tier1_last_count = rc->need;
    r.incremental = rc->incr;
    bool proper = rc->done && rc->sym == 0;
    if (!proper) {
        bool gave_up = false;
        const uint32_t fixed = run_tier2(h->g, h->t2, h->stream, h->h_small, &gave_up, &h->launches);
        TRY(check_cuda("tier2"));
        r.tier2_ran = 1;
        r.tier2_fixed = fixed;
        r.tier2_gave_up = gave_up ? 1 : 0;
        h->tier2_runs++;
        h->tier2_fixed += fixed;
        proper = !gave_up;
        if (proper) TRY(set_clean(h, 1));
    }
    r.proper = proper ? 1 : 0;
    if (rep) {
        r.drained = rep->drained;
        r.drain_failed = rep->drain_failed;
        *rep = r;
    }
    return SGC_OK;
}

// ---- applying a batch that is already on the device ----

int apply_device(sgc_handle* h, const EdgeUpdate* src, uint32_t n, int mode) {
    if (mode == SGC_MODE_DETERMINISTIC) {
        launch_det_apply(h->g, src, n, h->stream);
        h->launches += 1;
    } else {
        launch_conc_apply(h->g, src, n, h->eo, h->num_sms, h->stream);
        h->launches += 3;
    }
    if (h->g.touched) {
        launch_add_check(h->g, src, n, nullptr, h->num_sms, h->stream);
        h->launches += 1;
    }
    h->last_mode = mode;
    h->updates += n;
    return check_cuda("apply");
}

// The ingest slots, made on first use: two device batches of max_batch
// updates, their pinned host images, a copy stream and the events that order
// a slot's copy before its apply and its apply before its next copy.
int ensure_ingest(sgc_handle* h) {
    if (h->copy_stream) return SGC_OK;
    const size_t bytes = (size_t)h->opt.max_batch * sizeof(EdgeUpdate);
    for (int k = 0; k < 2; k++) {
        int r = dalloc(h, &h->slot_dev[k], h->opt.max_batch);
        if (r) return r;
        if (cudaHostAlloc(&h->slot_host[k], bytes, cudaHostAllocDefault) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->copy_done[k], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->slot_free[k], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return fail(SGC_ENOMEM, "ingest slot allocation failed");
        }
    }
    CK(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    return SGC_OK;
}

// ---- the concurrent configuration's publish as a CUDA graph ----
//
// compaction of edited rows, overflow drain, the repair's start, a
// conditional while-node { sweep, step } and the snapshot into one half of
// the double buffer, captured once per half; the repair's host fields (mode,
// sweep cap, full repair) reach the device through the graph's first copy,
// from pinned memory written before each launch. One host synchronization per
// epoch instead of one per sweep.

void enqueue_publish_head(sgc_handle* h, cudaStream_t s) {
    cudaMemsetAsync(&h->ctl->dirty_count, 0, 4, s);
    launch_dirty_list(h->g, h->dirty_list, &h->ctl->dirty_count, s);
    launch_compact(h->g, h->dirty_list, &h->ctl->dirty_count, h->n, false, s, (h->opt.flags & SGC_OPT_SORTED_ROWS) != 0);
    launch_take_overflow(h->g, &h->ctl->drain_n, s);
    launch_drain(h->g, &h->ctl->drain_n, false, &h->ctl->drain_failed, s);
    cudaMemcpyAsync(h->sb.rc, h->h_rc_in, 12, cudaMemcpyHostToDevice, s);
    const size_t mwords = ((h->n + 31) / 32) * 4;
    cudaMemsetAsync(h->sb.wmark, 0, mwords, s);
    cudaMemsetAsync(h->sb.rbits, 0, mwords, s);
    cudaMemsetAsync(h->sb.needf, 0, h->n, s);
    launch_repair_begin(h->g, h->sb, SWEEP_INDEP, h->num_sms, s);
}

void drop_publish_graphs(sgc_handle* h) {
    for (int k = 0; k < 2; k++) {
        if (h->pub_exec[k]) cudaGraphExecDestroy(h->pub_exec[k]);
        if (h->pub_graph[k]) cudaGraphDestroy(h->pub_graph[k]);
        h->pub_exec[k] = nullptr;
        h->pub_graph[k] = nullptr;
    }
}

int capture_publish_impl(sgc_handle* h, int back) {
    cudaStream_t s = h->stream;
    cudaGraph_t& graph = h->pub_graph[back];
    CK(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault));
    CK(cudaStreamBeginCaptureToGraph(s, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_publish_head(h, s);
    cudaStreamCaptureStatus st;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    CK(cudaStreamGetCaptureInfo(s, &st, nullptr, nullptr, &deps, &ndeps));
    std::vector<cudaGraphNode_t> head_tail(deps, deps + ndeps);
    cudaGraph_t g0 = nullptr;
    CK(cudaStreamEndCapture(s, &g0));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    CK(cudaGraphAddNode(&cnode, graph, head_tail.data(), head_tail.size(), &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    launch_repair_sweep(h->g, h->sb, SWEEP_INDEP, h->num_sms, s);
    launch_repair_step(h->g, h->sb, h->num_sms, s, &cond);
    cudaGraph_t g1 = nullptr;
    CK(cudaStreamEndCapture(s, &g1));
    CK(cudaStreamBeginCaptureToGraph(s, graph, &cnode, nullptr, 1, cudaStreamCaptureModeThreadLocal));
    if (h->g.chg) launch_snapshot_changes(h->g, h->chg_prev, h->snap[back], s);
    else launch_snapshot(h->g, h->snap[back], s);
    cudaMemcpyAsync(h->h_rc_out, h->sb.rc, sizeof(RepairCtl), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h->h_small + 32, h->sb.swept, 16, cudaMemcpyDeviceToHost, s);
    cudaGraph_t g2 = nullptr;
    CK(cudaStreamEndCapture(s, &g2));
    CK(cudaGraphInstantiate(&h->pub_exec[back], graph, 0));
    return SGC_OK;
}

int capture_publish(sgc_handle* h, int back) {
    const int r = capture_publish_impl(h, back);
    if (r != SGC_OK) {  // leave the stream out of capture mode; the eager publish takes over
        cudaStreamCaptureStatus st;
        if (cudaStreamIsCapturing(h->stream, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(h->stream, &g);
            if (g) cudaGraphDestroy(g);
        }
        cudaGetLastError();
        drop_publish_graphs(h);
        h->pub_graph_failed = true;
    }
    return r;
}

int publish_graph(sgc_handle* h, sgc_repair_report* rep) {
    const int back = 1 - h->front;
    const uint32_t every = h->opt.full_repair_every;
    RepairCtl* hin = h->h_rc_in;  // read by the graph's first copy
    hin->mode = (uint32_t)SWEEP_INDEP;
    hin->max_sweeps = 64u;
    hin->force_all = (every && h->repairs_since_full + 1 >= every) ? 1u : 0u;
    CK(cudaGraphLaunch(h->pub_exec[back], h->stream));
    TRY(sync(h));
    TRY(check_cuda("publish graph"));
    const RepairCtl* rc = h->h_rc_out;
    const unsigned long long* sw = (const unsigned long long*)(h->h_small + 32);
    h->sweep_bytes += 8ull * sw[0] + 28ull * sw[1];
    h->launches += (h->g.touched ? 6 : 5) + 10ull * rc->it + 1;
    h->d2h_bytes += sizeof(RepairCtl) + 16;
    sgc_repair_report r{};
    TRY(finish_repair(h, &r));
    if (r.tier2_ran || (h->g.chg && h->snap_full > 0)) {  // Tier-2 changed colors after the graph's
        launch_snapshot(h->g, h->snap[back], h->stream);      // snapshot, or a full one is due: take it again
        h->launches += 1;
        if (h->snap_full > 0) h->snap_full--;
    }
    h->front = back;
    h->epochs++;
    if (rep) *rep = r;
    return check_cuda("publish");
}

int read_drain(sgc_handle* h, sgc_repair_report* rep, unsigned long long before_failed) {
    CK(cudaMemcpyAsync(h->h_small, &h->ctl->drain_n, 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(h->h_small + 2, &h->ctl->drain_failed, 8, cudaMemcpyDeviceToHost, h->stream));
    h->d2h_bytes += 12;
    TRY(sync(h));
    if (rep) {
        rep->drained = h->h_small[0];
        rep->drain_failed = *(unsigned long long*)(h->h_small + 2) - before_failed;
    }
    return SGC_OK;
}

}  // namespace sgci

using namespace sgci;

extern "C" {

int sgc_default_options(sgc_options* o) {
    if (!o) return fail(SGC_EINVAL, "null options");
    std::memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(sgc_options);
    o->slack_pct = SGC_CSR_EXTRA_SLACK_PCT_DEFAULT;
    o->max_hist_colors = SGC_MAX_HISTOGRAM_COLORS_DEFAULT;
    o->max_batch = SGC_HOST_BATCH_SIZE;
    o->device = 0;
    o->flags = 0;
    o->full_repair_every = 16;
    o->repair_tile = SWEEP_CH;
    return SGC_OK;
}

int sgc_destroy(sgc_handle* h) {
    if (!h) return SGC_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    drop_publish_graphs(h);
    if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
    for (int k = 0; k < 2; k++) {
        if (h->slot_host[k]) cudaFreeHost(h->slot_host[k]);
        if (h->copy_done[k]) cudaEventDestroy(h->copy_done[k]);
        if (h->slot_free[k]) cudaEventDestroy(h->slot_free[k]);
    }
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    if (h->ring_host) cudaFreeHost(h->ring_host);
    if (h->ring_done) cudaEventDestroy(h->ring_done);
    for (void* p : h->allocs) cudaFree(p);
    if (h->h_stage) cudaFreeHost(h->h_stage);
    if (h->h_small) cudaFreeHost(h->h_small);
    if (h->h_rc_in) cudaFreeHost(h->h_rc_in);
    if (h->h_rc_out) cudaFreeHost(h->h_rc_out);
    if (h->stage_free) cudaEventDestroy(h->stage_free);
    for (auto& se : h->ev_pending)
        for (int k = 0; k < 5; k++) cudaEventDestroy(se.ev[k]);
    for (auto e : h->ev_pool) cudaEventDestroy(e);
    if (h->t2.rev_keys) cudaFree(h->t2.rev_keys);
    if (h->t2.rev_keys2) cudaFree(h->t2.rev_keys2);
    if (h->t2.cub_tmp) cudaFree(h->t2.cub_tmp);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return SGC_OK;
}

}  // extern "C"

int sgci::create_internal(const StreamGCConfig* cfg, const sgc_options* opt_in, const uint64_t* row_ptr,
                          const uint32_t* col_idx, const uint32_t* degree, const CreateExtra* ex, sgc_handle** out) {
    if (!cfg || !row_ptr || !degree || !out) return fail(SGC_EINVAL, "null argument");
    *out = nullptr;
    sgc_options opt;
    sgc_default_options(&opt);
    if (opt_in) {
        if (opt_in->struct_size != sizeof(sgc_options)) return fail(SGC_EINVAL, "sgc_options.struct_size mismatch");
        opt = *opt_in;
    }
    if (cfg->num_gpus > 1) return fail(SGC_ENOTSUP, "num_gpus=%u: this library runs the single-GPU path", cfg->num_gpus);
    if (opt.max_hist_colors == 0 || opt.max_hist_colors % 4 || opt.max_hist_colors > 65535)
        return fail(SGC_EINVAL, "max_hist_colors must be a positive multiple of 4");
    if (opt.max_batch == 0) return fail(SGC_EINVAL, "max_batch must be positive");
    if (opt.repair_tile == 0) opt.repair_tile = SWEEP_CH;
    if (opt.repair_tile < SWEEP_CH_MIN || opt.repair_tile % 32 || opt.repair_tile > (1u << 20))
        return fail(SGC_EINVAL, "repair_tile must be a multiple of 32 in [%u, 2^20]", SWEEP_CH_MIN);
    const uint32_t n = cfg->num_vertices;
    if (n == 0) return fail(SGC_EINVAL, "num_vertices is 0");
    if (row_ptr[0] != 0) return fail(SGC_EINVAL, "row_ptr[0] must be 0");
    const uint64_t nnz = row_ptr[n];
    if (nnz && !col_idx) return fail(SGC_EINVAL, "col_idx is null");
    // host-side layout: capacity max(d + d*slack/100, 8) (streamgc.cu:373-378)
    std::vector<uint64_t> rp((size_t)n + 1, 0);
    std::vector<uint32_t> hdmap(n, EMPTY);
    std::vector<uint32_t> hw(n, 0);
    uint32_t num_hd = 0;
    for (uint32_t x = 0; x < n; x++) {
        if (row_ptr[x + 1] < row_ptr[x]) return fail(SGC_EINVAL, "row_ptr not monotone at %u", x);
        const uint64_t cnt64 = row_ptr[x + 1] - row_ptr[x];
        if (cnt64 > 0x3FFFFFFFull) return fail(SGC_EINVAL, "row %u too long", x);
        const uint32_t cnt = (uint32_t)cnt64;
        const uint32_t extra = (uint32_t)(((uint64_t)cnt * opt.slack_pct) / 100);
        const uint32_t cap = std::max<uint32_t>(cnt + extra, 8u);
        rp[x + 1] = rp[x] + cap;
        hw[x] = cnt;
        const uint32_t thr = (ex && ex->thr_word) ? ex->thr_word[x >> 5] : cfg->histogram_threshold;
        if (degree[x] > thr) hdmap[x] = num_hd++;
    }
    const bool exact_sel = (opt.flags & SGC_OPT_EXACT_SELECT) != 0;
    if (exact_sel && (opt.flags & (SGC_OPT_ABL_FORCE_BITMAP | SGC_OPT_ABL_NO_OVERFLOW | SGC_OPT_ABL_LIVE_DEG)))
        return fail(SGC_EINVAL, "the ablation options apply to the reference rules, not to SGC_OPT_EXACT_SELECT");
    for (uint64_t j = 0; j < nnz; j++) {
        if (col_idx[j] == INV) return fail(SGC_EINVAL, "col_idx holds the INVALID sentinel at %llu", (unsigned long long)j);
        if (exact_sel && (col_idx[j] & TOMB))  // the top bit marks deleted entries under exact selection
            return fail(SGC_EINVAL, "col_idx[%llu] >= 2^31 (exact selection)", (unsigned long long)j);
    }
    if (exact_sel && n >= TOMB) return fail(SGC_EINVAL, "num_vertices >= 2^31 (exact selection)");
    // rows whose base entries are not strictly ascending start "edited": the
    // binary-search fast path only serves sorted, duplicate-free rows
    std::vector<uint32_t> edited((n + 31) / 32 + 1, 0);
    for (uint32_t x = 0; x < n; x++)
        for (uint64_t j = row_ptr[x] + 1; j < row_ptr[x + 1]; j++)
            if (col_idx[j - 1] >= col_idx[j]) { edited[x >> 5] |= 1u << (x & 31); break; }

    sgc_handle* h = new sgc_handle();
    h->opt = opt;
    h->cfg = *cfg;
    h->device = opt.device;
    h->n = n;
    h->num_hd = num_hd;
    h->maxc = opt.max_hist_colors;
    h->total_slots = rp[n];
    auto bail = [&](int code) { sgc_destroy(h); return code; };
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return bail(fail(SGC_ECUDA, "cudaSetDevice(%d) failed", h->device)); }
    cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(fail(SGC_ECUDA, "stream create failed"));

    int r = SGC_OK;
#define A(...) do { r = dalloc(h, __VA_ARGS__); if (r) return bail(r); } while (0)
    Dev& g = h->g;
    g.n = n;
    g.maxc = h->maxc;
    g.exact = (opt.flags & SGC_OPT_EXACT_SELECT) ? 1u : 0u;
    g.abl = ((opt.flags & SGC_OPT_ABL_FORCE_BITMAP) ? ABL_FORCE_BITMAP : 0u) |
            ((opt.flags & SGC_OPT_ABL_NO_OVERFLOW) ? ABL_NO_OVERFLOW : 0u) |
            ((opt.flags & SGC_OPT_ABL_LIVE_DEG) ? ABL_LIVE_DEG : 0u);
    const uint32_t hist_rows = g.exact ? 0u : num_hd;  // exact selection keeps no histogram rows
    uint64_t* d_rp; A(&d_rp, (size_t)n + 1);
    const uint64_t padded = ((h->total_slots + 3) & ~3ull) + 8;  // 16-byte loads stay inside
    uint32_t* d_col; A(&d_col, padded, 0xFF);
    A(&g.st, n, 0);
    A(&g.bm, n, 0);
    uint32_t* d_hdmap; A(&d_hdmap, n);
    A(&g.hist, (size_t)hist_rows * h->maxc, 0);
    h->hist_rows = hist_rows;
    uint32_t* d_deg; A(&d_deg, n);
    A(&g.hw, n);
    if (g.exact) A(&g.live, n);  // lazy compaction goes with the concurrent configuration
    else g.live = nullptr;
    A(&g.dirty, (n + 31) / 32 + 1, 0);
    A(&g.edited, (n + 31) / 32 + 1, 0);
    A(&g.ovf, OVF_CAP);
    A(&h->ctl, 1, 0);
    A(&h->snap[0], n, 0);
    A(&h->snap[1], n, 0);
    g.rp = d_rp;
    g.col = d_col;
    g.hdmap = d_hdmap;
    g.deg = d_deg;
    g.ovf_count = &h->ctl->ovf_count;
    g.ovf_lost = &h->ctl->ovf_lost;
    g.nskip = &h->ctl->nskip;
    g.err = &h->ctl->err;
    const uint32_t G = (ex && ex->G) ? ex->G : 1u;
    {
        std::vector<GraphCtl> gc(G);
        for (uint32_t k = 0; k < G; k++) {
            std::memset(&gc[k], 0, sizeof(GraphCtl));
            gc[k].asym = 1;  // nothing known about the mirrors yet
            gc[k].base = (ex && ex->base) ? ex->base[k] : 0u;
        }
        A(&g.gctl, G);
        if (cudaMemcpyAsync(g.gctl, gc.data(), G * sizeof(GraphCtl), cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
            cudaStreamSynchronize(h->stream) != cudaSuccess)
            return bail(fail(SGC_ECUDA, "control block init failed"));
    }
    g.gidw = nullptr;
    if (ex && ex->gidw) {
        uint32_t* d_gidw;
        A(&d_gidw, (n + 31) / 32);
        if (cudaMemcpyAsync(d_gidw, ex->gidw, ((n + 31) / 32) * 4ull, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
            cudaStreamSynchronize(h->stream) != cudaSuccess)
            return bail(fail(SGC_ECUDA, "graph map upload failed"));
        g.gidw = d_gidw;
    }
    if (cudaMemcpyAsync(d_rp, rp.data(), rp.size() * 8, cudaMemcpyHostToDevice, h->stream) ||
        cudaMemcpyAsync(d_hdmap, hdmap.data(), (size_t)n * 4, cudaMemcpyHostToDevice, h->stream) ||
        cudaMemcpyAsync(d_deg, degree, (size_t)n * 4, cudaMemcpyHostToDevice, h->stream) ||
        cudaMemcpyAsync(g.hw, hw.data(), (size_t)n * 4, cudaMemcpyHostToDevice, h->stream) ||
        (g.live && cudaMemcpyAsync(g.live, hw.data(), (size_t)n * 4, cudaMemcpyHostToDevice, h->stream)) ||
        cudaMemcpyAsync(g.edited, edited.data(), edited.size() * 4, cudaMemcpyHostToDevice, h->stream))
        return bail(fail(SGC_ECUDA, "upload failed"));
    // base entries: staged through a temporary device copy of the base CSR
    if (nnz) {
        uint64_t* d_brp = nullptr;
        uint32_t* d_bcol = nullptr;
        if (cudaMalloc(&d_brp, ((size_t)n + 1) * 8) || cudaMalloc(&d_bcol, nnz * 4)) {
            cudaFree(d_brp);
            cudaGetLastError();
            return bail(fail(SGC_ENOMEM, "base CSR staging allocation failed"));
        }
        cudaMemcpyAsync(d_brp, row_ptr, ((size_t)n + 1) * 8, cudaMemcpyHostToDevice, h->stream);
        cudaMemcpyAsync(d_bcol, col_idx, nnz * 4, cudaMemcpyHostToDevice, h->stream);
        scatter_base_kernel<<<h->num_sms * 8, 256, 0, h->stream>>>(n, d_brp, d_bcol, d_rp, d_col);
        cudaStreamSynchronize(h->stream);
        cudaFree(d_brp);
        cudaFree(d_bcol);
        if ((r = check_cuda("scatter_base"))) return bail(r);
    }
    // update staging + same-edge ordering
    const uint32_t mb = opt.max_batch;
    A(&h->d_batch, mb);
    if (cudaHostAlloc(&h->h_stage, (size_t)mb * sizeof(EdgeUpdate), cudaHostAllocDefault) != cudaSuccess)
        return bail(fail(SGC_ENOMEM, "pinned staging allocation failed"));
    if (cudaHostAlloc(&h->h_small, 256, cudaHostAllocDefault) != cudaSuccess)
        return bail(fail(SGC_ENOMEM, "pinned scratch allocation failed"));
    cudaEventCreateWithFlags(&h->stage_free, cudaEventDisableTiming);
    uint32_t tsize = 1;
    while (tsize < 2 * mb) tsize <<= 1;
    EdgeOrder& eo = h->eo;
    A(&eo.tkey, tsize, 0xFF);
    A(&eo.thead, tsize, 0xFF);
    A(&eo.tslot, mb);
    A(&eo.tnext, mb);
    A(&eo.tprev, mb);
    A(&eo.tsucc, mb);
    eo.ticket = &h->ctl->ticket;
    eo.tmask = tsize - 1;
    if (g.exact) {  // row-scale operations of concurrent batches: the pass after the batch
        A(&g.hub_ops, 2ull * mb);
        g.hub_count = &h->ctl->hub_count;
        g.hub_cap = 2 * mb;
        g.hub_total = &h->ctl->hub_total;
    }
    // sweep buffers
    SweepBufs& sb = h->sb;
    const uint64_t icap = h->total_slots / SWEEP_CH_MIN + (uint64_t)n + 1;
    if (icap > 0xFFFFFFF0ull) return bail(fail(SGC_ENOTSUP, "sweep item list beyond 2^32 entries"));
    sb.item_cap = (uint32_t)icap;
    A(&sb.items, icap);
    sb.item_count = &h->ctl->item_count;
    A(&sb.acc_bm, n, 0);
    A(&sb.acc_fl, n, 0);
    A(&sb.pend_v, n);
    A(&sb.pend_w, n);
    sb.pend_count = &h->ctl->pend_count;
    A(&sb.fac_v, n);
    sb.fac_count = &h->ctl->fac_count;
    sb.live = &h->ctl->live;
    A(&sb.wmark, (n + 31) / 32 + 1, 0);
    A(&sb.wl, n);
    A(&sb.wl_count, 4, 0);
    A(&sb.swept, 2, 0);
    A(&sb.needf, n, 0);
    A(&sb.need_v, n);
    A(&sb.need_count, 4, 0);
    A(&sb.rbits, (n + 31) / 32 + 1, 0);
    A(&sb.rc, 1, 0);
    sb.tile = opt.repair_tile;
    sb.G = G;
    if (g.exact) A(&g.touched, (n + 31) / 32 + 1, 0);
    else g.touched = nullptr;
    if (g.exact && G == 1) {  // incremental snapshots (a batched handle publishes per graph)
        A(&g.chg, (n + 31) / 32 + 1, 0);
        A(&h->chg_prev, (n + 31) / 32 + 1, 0);
    } else {
        g.chg = nullptr;
    }
    if (g.exact) {  // base runs: rows whose base entries are strictly ascending
        std::vector<uint32_t> bl(n);
        for (uint32_t x = 0; x < n; x++) bl[x] = (edited[x >> 5] >> (x & 31)) & 1u ? 0u : hw[x];
        A(&g.blen, n);
        if (cudaMemcpyAsync(g.blen, bl.data(), (size_t)n * 4, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
            cudaStreamSynchronize(h->stream) != cudaSuccess)
            return bail(fail(SGC_ECUDA, "base run upload failed"));
    } else {
        g.blen = nullptr;
    }
    if (cudaHostAlloc(&h->h_rc_in, sizeof(RepairCtl), cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc(&h->h_rc_out, sizeof(RepairCtl), cudaHostAllocDefault) != cudaSuccess)
        return bail(fail(SGC_ENOMEM, "pinned control block allocation failed"));
    std::memset(h->h_rc_in, 0, sizeof(RepairCtl));
    std::memset(h->h_rc_out, 0, sizeof(RepairCtl));
    if (g.exact) A(&sb.hiused, (size_t)num_hd * 64, 0);
    else sb.hiused = nullptr;
    A(&h->dirty_list, n);
    // tier-2 buffers
    Tier2Bufs& t2 = h->t2;
    A(&t2.inU, n);
    A(&t2.inF, n);
    A(&t2.inL, n);
    A(&t2.done, n);
    A(&t2.list, n);
    A(&t2.list2, n);
    A(&t2.count, 16, 0);
    A(&t2.rev_start, n);
    A(&t2.rev_end, n);
    A(&t2.pend_v, n);
    A(&t2.pend_w, n);
    t2.rev_cap = 1u << 20;
    if (cudaMalloc(&t2.rev_keys, (size_t)t2.rev_cap * 8) || cudaMalloc(&t2.rev_keys2, (size_t)t2.rev_cap * 8))
        return bail(fail(SGC_ENOMEM, "tier-2 reverse buffer allocation failed"));
    t2.cub_tmp_bytes = tier2_cub_bytes(n, t2.rev_cap);
    if (cudaMalloc(&t2.cub_tmp, t2.cub_tmp_bytes)) return bail(fail(SGC_ENOMEM, "tier-2 scratch allocation failed"));
#undef A
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bail(fail(SGC_ECUDA, "create sync failed"));
    if ((r = check_cuda("create"))) return bail(r);
    *out = h;
    return SGC_OK;
}

extern "C" {

int sgc_create_ex(const StreamGCConfig* cfg, const sgc_options* opt_in, const uint64_t* row_ptr,
                  const uint32_t* col_idx, const uint32_t* degree, sgc_handle** out) {
    return create_internal(cfg, opt_in, row_ptr, col_idx, degree, nullptr, out);
}

int sgc_create(const StreamGCConfig* cfg, const uint32_t* row_ptr, const uint32_t* col_idx, const uint32_t* degree,
               sgc_handle** out) {
    if (!cfg || !row_ptr) return fail(SGC_EINVAL, "null argument");
    std::vector<uint64_t> rp((size_t)cfg->num_vertices + 1);
    for (size_t i = 0; i < rp.size(); i++) rp[i] = row_ptr[i];
    return sgc_create_ex(cfg, nullptr, rp.data(), col_idx, degree, out);
}

int sgc_apply(sgc_handle* h, const EdgeUpdate* ups, uint32_t n, int mode) {
    if (!h) return fail(SGC_EINVAL, "null handle");
    if (n == 0) return SGC_OK;
    if (!ups) return fail(SGC_EINVAL, "null updates");
    if (n > h->opt.max_batch) return fail(SGC_EINVAL, "batch %u exceeds max_batch %u", n, h->opt.max_batch);
    if (mode != SGC_MODE_DETERMINISTIC && mode != SGC_MODE_CONCURRENT) return fail(SGC_EINVAL, "bad mode %d", mode);
    CK(cudaSetDevice(h->device));
    const EdgeUpdate* src = ups;
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, ups) != cudaSuccess) cudaGetLastError();
    if (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) {
        src = ups;  // caller keeps it alive until the stream passes this point
    } else if (attr.type == cudaMemoryTypeHost) {
        CK(cudaMemcpyAsync(h->d_batch, ups, (size_t)n * sizeof(EdgeUpdate), cudaMemcpyHostToDevice, h->stream));
        h->h2d_bytes += (uint64_t)n * sizeof(EdgeUpdate);
        src = h->d_batch;
    } else {
        CK(cudaEventSynchronize(h->stage_free));
        std::memcpy(h->h_stage, ups, (size_t)n * sizeof(EdgeUpdate));
        CK(cudaMemcpyAsync(h->d_batch, h->h_stage, (size_t)n * sizeof(EdgeUpdate), cudaMemcpyHostToDevice, h->stream));
        CK(cudaEventRecord(h->stage_free, h->stream));
        h->h2d_bytes += (uint64_t)n * sizeof(EdgeUpdate);
        src = h->d_batch;
    }
    return apply_device(h, src, n, mode);
}

int sgc_stage(sgc_handle* h, const EdgeUpdate* ups, uint32_t n) {
    if (!h) return fail(SGC_EINVAL, "null handle");
    if (n == 0) return SGC_OK;
    if (!ups) return fail(SGC_EINVAL, "null updates");
    if (n > h->opt.max_batch) return fail(SGC_EINVAL, "batch %u exceeds max_batch %u", n, h->opt.max_batch);
    if (h->staged == 2) return fail(SGC_EINVAL, "both staging slots hold a batch");
    CK(cudaSetDevice(h->device));
    TRY(ensure_ingest(h));
    const uint32_t k = h->stage_next;
    CK(cudaEventSynchronize(h->slot_free[k]));  // the apply that read this slot (and its copy) finished
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, ups) != cudaSuccess) cudaGetLastError();
    const size_t bytes = (size_t)n * sizeof(EdgeUpdate);
    if (attr.type == cudaMemoryTypeHost || attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) {
        // pinned or device memory: copied as it is (it must not change until the copy is done)
        CK(cudaMemcpyAsync(h->slot_dev[k], ups, bytes, cudaMemcpyDefault, h->copy_stream));
    } else {
        std::memcpy(h->slot_host[k], ups, bytes);
        CK(cudaMemcpyAsync(h->slot_dev[k], h->slot_host[k], bytes, cudaMemcpyHostToDevice, h->copy_stream));
    }
    CK(cudaEventRecord(h->copy_done[k], h->copy_stream));
    h->h2d_bytes += (uint64_t)n * sizeof(EdgeUpdate);
    h->slot_n[k] = n;
    h->stage_next = 1 - k;
    h->staged++;
    return SGC_OK;
}

int sgc_apply_staged(sgc_handle* h, int mode) {
    if (!h) return fail(SGC_EINVAL, "null handle");
    if (h->staged == 0) return fail(SGC_EINVAL, "no staged batch");
    if (mode != SGC_MODE_DETERMINISTIC && mode != SGC_MODE_CONCURRENT) return fail(SGC_EINVAL, "bad mode %d", mode);
    CK(cudaSetDevice(h->device));
    const uint32_t k = h->staged == 2 ? h->stage_next : 1 - h->stage_next;  // the oldest staged slot
    CK(cudaStreamWaitEvent(h->stream, h->copy_done[k], 0));
    TRY(apply_device(h, h->slot_dev[k], h->slot_n[k], mode));
    CK(cudaEventRecord(h->slot_free[k], h->stream));
    h->staged--;
    return SGC_OK;
}

int sgc_ring_create(sgc_handle* h, uint32_t log2_slots) {
    if (!h) return fail(SGC_EINVAL, "null handle");
    if (h->ring_host) return fail(SGC_EINVAL, "the handle already has a ring");
    if (log2_slots < 10 || log2_slots > 28) return fail(SGC_EINVAL, "log2_slots must be in [10, 28]");
    CK(cudaSetDevice(h->device));
    const uint64_t slots = 1ull << log2_slots;
    void* p = nullptr;
    if (cudaHostAlloc(&p, slots * sizeof(EdgeUpdate), cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return fail(SGC_ENOMEM, "pinned mapped ring of %llu slots", (unsigned long long)slots);
    }
    void* d = nullptr;
    if (cudaHostGetDevicePointer(&d, p, 0) != cudaSuccess || cudaEventCreateWithFlags(&h->ring_done, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeHost(p);
        return fail(SGC_ECUDA, "ring mapping failed");
    }
    h->ring_host = static_cast<EdgeUpdate*>(p);
    h->ring_dev = static_cast<EdgeUpdate*>(d);
    h->ring_mask = slots - 1;
    return SGC_OK;
}

int sgc_ring_push(sgc_handle* h, const EdgeUpdate* ups, uint32_t n, uint32_t* accepted) {
    if (!h || (n && !ups)) return fail(SGC_EINVAL, "null argument");
    if (!h->ring_host) return fail(SGC_EINVAL, "no ring (sgc_ring_create)");
    const uint64_t tail = h->ring_tail.load(std::memory_order_relaxed);
    const uint64_t free_slots = h->ring_mask + 1 - (tail - h->ring_released.load(std::memory_order_acquire));
    const uint32_t k = (uint32_t)std::min<uint64_t>(n, free_slots);
    for (uint32_t i = 0; i < k;) {  // at most two runs of consecutive slots
        const uint64_t pos = (tail + i) & h->ring_mask;
        const uint32_t run = (uint32_t)std::min<uint64_t>(k - i, h->ring_mask + 1 - pos);
        std::memcpy(h->ring_host + pos, ups + i, (size_t)run * sizeof(EdgeUpdate));
        i += run;
    }
    h->ring_tail.store(tail + k, std::memory_order_release);  // the slots are written before they are published
    if (accepted) *accepted = k;
    return SGC_OK;
}

int sgc_ring_apply(sgc_handle* h, uint32_t max_updates, int mode, uint32_t* applied) {
    if (!h) return fail(SGC_EINVAL, "null handle");
    if (!h->ring_host) return fail(SGC_EINVAL, "no ring (sgc_ring_create)");
    if (mode != SGC_MODE_DETERMINISTIC && mode != SGC_MODE_CONCURRENT) return fail(SGC_EINVAL, "bad mode %d", mode);
    CK(cudaSetDevice(h->device));
    // slots of the previous gather go back to the producer once it has finished
    if (h->ring_inflight > h->ring_released.load(std::memory_order_relaxed)) {
        const cudaError_t q = cudaEventQuery(h->ring_done);
        if (q == cudaSuccess) h->ring_released.store(h->ring_inflight, std::memory_order_release);
        else if (q != cudaErrorNotReady) return fail(SGC_ECUDA, "ring: %s", cudaGetErrorString(q));
    }
    const uint64_t tail = h->ring_tail.load(std::memory_order_acquire);
    const uint32_t k = (uint32_t)std::min<uint64_t>({tail - h->ring_head, (uint64_t)max_updates,
                                                    (uint64_t)h->opt.max_batch});
    if (applied) *applied = k;
    if (!k) return SGC_OK;
    launch_ring_gather(h->ring_dev, h->ring_mask, h->ring_head, k, h->d_batch, h->num_sms, h->stream);
    h->launches += 1;
    h->h2d_bytes += (uint64_t)k * sizeof(EdgeUpdate);
    h->ring_head += k;
    h->ring_inflight = h->ring_head;
    CK(cudaEventRecord(h->ring_done, h->stream));
    return apply_device(h, h->d_batch, k, mode);
}

int sgc_epoch(sgc_handle* h) {
    if (!h) return fail(SGC_EINVAL, "null handle");
    CK(cudaSetDevice(h->device));
    publish_snapshot(h);
    TRY(compact_dirty(h, true));
    TRY(drain(h, h->last_mode == SGC_MODE_DETERMINISTIC, nullptr));
    TRY(rebuild_sweep(h));
    h->epochs++;
    return SGC_OK;
}

int sgc_drain_and_compact(sgc_handle* h, sgc_repair_report* rep) {
    if (!h) return fail(SGC_EINVAL, "null handle");
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(h->h_small + 8, &h->ctl->drain_failed, 8, cudaMemcpyDeviceToHost, h->stream));
    TRY(sync(h));
    const unsigned long long before = *(unsigned long long*)(h->h_small + 8);
    TRY(compact_dirty(h, true));
    TRY(drain(h, h->last_mode == SGC_MODE_DETERMINISTIC, &h->ctl->drain_failed));
    TRY(rebuild_sweep(h));
    return read_drain(h, rep, before);
}

int sgc_repair(sgc_handle* h, sgc_repair_report* rep) {
    if (!h) return fail(SGC_EINVAL, "null handle");
    CK(cudaSetDevice(h->device));
    sgc_repair_report r{};
    CK(cudaMemcpyAsync(h->h_small + 8, &h->ctl->drain_failed, 8, cudaMemcpyDeviceToHost, h->stream));
    TRY(sync(h));
    const unsigned long long before = *(unsigned long long*)(h->h_small + 8);
    TRY(compact_dirty(h, true));
    TRY(drain(h, h->last_mode == SGC_MODE_DETERMINISTIC, &h->ctl->drain_failed));
    // drain_and_compact's rebuild is subsumed: the first (full) sweep rebuilds every bitmap first.
    TRY(read_drain(h, &r, before));
    TRY(repair_loop(h, &r, true));
    if (rep) *rep = r;
    return SGC_OK;
}

int sgc_publish(sgc_handle* h, sgc_repair_report* rep) {
    if (!h) return fail(SGC_EINVAL, "null handle");
    CK(cudaSetDevice(h->device));
    if ((h->opt.flags & SGC_OPT_GRAPH_PUBLISH) && h->g.exact && h->last_mode == SGC_MODE_CONCURRENT &&
        !h->pub_graph_failed) {
        const int back = 1 - h->front;
        if (h->pub_exec[back] || capture_publish(h, back) == SGC_OK) return publish_graph(h, rep);
    }
    sgc_repair_report r{};
    TRY(compact_dirty(h, false));
    TRY(drain(h, h->last_mode == SGC_MODE_DETERMINISTIC, &h->ctl->drain_failed));
    TRY(repair_loop(h, &r, false));
    publish_snapshot(h);
    h->epochs++;
    if (rep) *rep = r;
    return check_cuda("publish");
}

int sgc_process_stream(sgc_handle* h, const EdgeUpdate* ups, uint64_t n, int mode, uint32_t* epochs) {
    if (!h) return fail(SGC_EINVAL, "null handle");
    const uint32_t E = h->cfg.epoch_size;
    uint64_t batch = mode == SGC_MODE_DETERMINISTIC ? SGC_HOST_BATCH_SIZE
                                                     : std::min<uint64_t>(E ? E : SGC_HOST_BATCH_SIZE, h->opt.max_batch);
    batch = std::min<uint64_t>(batch, h->opt.max_batch);
    uint64_t processed = 0, since = 0;
    uint32_t ne = 0;
    while (processed < n) {
        const uint32_t b = (uint32_t)std::min<uint64_t>(batch, n - processed);
        TRY(sgc_apply(h, ups + processed, b, mode));
        processed += b;
        since += b;
        if (since >= E) {
            if (mode == SGC_MODE_DETERMINISTIC) TRY(sgc_epoch(h));
            else TRY(sgc_publish(h, nullptr));
            since = 0;
            ne++;
        }
    }
    if (epochs) *epochs = ne;
    return SGC_OK;
}

int sgc_query(sgc_handle* h, const uint32_t* v, uint16_t* out, uint32_t k) {
    if (!h || (k && (!v || !out))) return fail(SGC_EINVAL, "null argument");
    if (!k) return SGC_OK;
    CK(cudaSetDevice(h->device));
    uint32_t* dv = nullptr;
    uint16_t* dout = nullptr;
    CK(cudaMallocAsync(&dv, (size_t)k * 4, h->stream));
    CK(cudaMallocAsync(&dout, (size_t)k * 2, h->stream));
    CK(cudaMemcpyAsync(dv, v, (size_t)k * 4, cudaMemcpyHostToDevice, h->stream));
    launch_query(h->snap[h->front], h->n, dv, dout, k, h->stream);
    CK(cudaMemcpyAsync(out, dout, (size_t)k * 2, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaFreeAsync(dv, h->stream));
    CK(cudaFreeAsync(dout, h->stream));
    return sync(h);
}

}  // extern "C"

// ---- point queries that allocate nothing ----
// sgc_query takes its device scratch from the stream-ordered allocator on every
// call. A serving thread that answers queries while its tenants already fill
// their HBM budget, or one that must not enter the allocator on a latency-bound
// path, cannot do that; it queries through this fixed scratch compiled into the
// library instead: one static array per GPU that loads the library, held until
// the process exits. Vertex ids occupy words [0, MAX); the uint16 colors are
// packed after them.
namespace {
constexpr uint32_t QUERY_NOALLOC_MAX = SGC_QUERY_NOALLOC_MAX;
static __device__ __align__(256) uint32_t g_query_scratch[QUERY_NOALLOC_MAX + QUERY_NOALLOC_MAX / 2];
constexpr int MAX_DEVICES = 256;
std::mutex g_query_scratch_mu;
uint32_t* g_query_scratch_addr[MAX_DEVICES] = {};  // device address of the array, per device ordinal

// Device address of the scratch on the current device (set-up once per device,
// with that device current). In host code the array's name is only a host-side
// stand-in, so kernels get this address, never &g_query_scratch.
int query_scratch(int device, uint32_t** out) {
    if (device < 0 || device >= MAX_DEVICES) return fail(SGC_EINVAL, "device ordinal %d out of range", device);
    std::lock_guard<std::mutex> lock(g_query_scratch_mu);
    if (!g_query_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_query_scratch);
        if (e != cudaSuccess || !p)
            return fail(SGC_ECUDA, "cudaGetSymbolAddress(query scratch) on device %d: %s", device,
                        cudaGetErrorString(e));
        g_query_scratch_addr[device] = static_cast<uint32_t*>(p);
    }
    *out = g_query_scratch_addr[device];
    return SGC_OK;
}
}  // namespace

extern "C" {

int sgc_query_noalloc(sgc_handle* h, const uint32_t* v, uint16_t* out, uint32_t k) {
    if (!h || (k && (!v || !out))) return fail(SGC_EINVAL, "null argument");
    if (k > QUERY_NOALLOC_MAX)
        return fail(SGC_EINVAL, "sgc_query_noalloc: %u queries exceed its fixed scratch of %u; split the call", k,
                    QUERY_NOALLOC_MAX);
    if (!k) return SGC_OK;
    CK(cudaSetDevice(h->device));
    uint32_t* base = nullptr;
    TRY(query_scratch(h->device, &base));
    uint32_t* dv = base;
    uint16_t* dout = reinterpret_cast<uint16_t*>(base + QUERY_NOALLOC_MAX);
    CK(cudaMemcpyAsync(dv, v, (size_t)k * 4, cudaMemcpyHostToDevice, h->stream));
    launch_query(h->snap[h->front], h->n, dv, dout, k, h->stream);  // not counted in launches, as in sgc_query
    CK(cudaMemcpyAsync(out, dout, (size_t)k * 2, cudaMemcpyDeviceToHost, h->stream));
    return sync(h);
}

int sgc_download(sgc_handle* h, int what, void* dst, uint64_t bytes) {
    if (!h || !dst) return fail(SGC_EINVAL, "null argument");
    CK(cudaSetDevice(h->device));
    const void* src = nullptr;
    uint64_t need = 0;
    uint16_t* tmp = nullptr;
    switch (what) {
        case SGC_DL_STATES: src = h->g.st; need = h->n * 4ull; break;
        case SGC_DL_BITMAPS: src = h->g.bm; need = h->n * 8ull; break;
        case SGC_DL_HIST: src = h->g.hist; need = (uint64_t)h->hist_rows * h->maxc * 4; break;
        case SGC_DL_ROW_PTR: src = h->g.rp; need = (h->n + 1ull) * 8; break;
        case SGC_DL_COL: src = h->g.col; need = h->total_slots * 4; break;
        case SGC_DL_SNAPSHOT: src = h->snap[h->front]; need = h->n * 2ull; break;
        case SGC_DL_HIGHWATER: src = h->g.hw; need = h->n * 4ull; break;
        case SGC_DL_HDMAP: src = h->g.hdmap; need = h->n * 4ull; break;
        case SGC_DL_BASE_RUN: {
            need = h->n * 4ull;
            if (bytes < need) return fail(SGC_EINVAL, "download target %d needs %llu bytes", what, (unsigned long long)need);
            if (!h->g.blen) {
                std::memset(dst, 0, need);
                return SGC_OK;
            }
            src = h->g.blen;
            break;
        }
        case SGC_DL_HOLES: {  // each row's mark minus its live count
            need = h->n * 4ull;
            if (bytes < need) return fail(SGC_EINVAL, "download target %d needs %llu bytes", what, (unsigned long long)need);
            if (!h->g.live) {
                std::memset(dst, 0, need);
                return SGC_OK;
            }
            std::vector<uint32_t> lv(h->n);
            uint32_t* out = static_cast<uint32_t*>(dst);
            CK(cudaMemcpyAsync(out, h->g.hw, need, cudaMemcpyDeviceToHost, h->stream));
            CK(cudaMemcpyAsync(lv.data(), h->g.live, need, cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            for (uint32_t x = 0; x < h->n; x++) out[x] = out[x] > lv[x] ? out[x] - lv[x] : 0u;
            return SGC_OK;
        }
        case SGC_DL_COLORS: {
            CK(cudaMallocAsync(&tmp, h->n * 2ull, h->stream));
            launch_colors(h->g, tmp, h->stream);
            src = tmp;
            need = h->n * 2ull;
            break;
        }
        case SGC_DL_OVERFLOW: {
            CK(cudaMemcpyAsync(h->h_small, &h->ctl->ovf_count, 4, cudaMemcpyDeviceToHost, h->stream));
            TRY(sync(h));
            const uint32_t c = std::min<uint32_t>(h->h_small[0], OVF_CAP);
            src = h->g.ovf;
            need = c * 8ull;
            break;
        }
        default: return fail(SGC_EINVAL, "bad download target %d", what);
    }
    if (bytes < need) {
        if (tmp) cudaFreeAsync(tmp, h->stream);
        return fail(SGC_EINVAL, "download target %d needs %llu bytes", what, (unsigned long long)need);
    }
    if (need) CK(cudaMemcpyAsync(dst, src, need, cudaMemcpyDeviceToHost, h->stream));
    if (tmp) CK(cudaFreeAsync(tmp, h->stream));
    return sync(h);
}

int sgc_upload(sgc_handle* h, int what, const void* src, uint64_t bytes) {
    if (!h || !src) return fail(SGC_EINVAL, "null argument");
    CK(cudaSetDevice(h->device));
    void* dst = nullptr;
    uint64_t need = 0;
    switch (what) {
        case SGC_DL_STATES: dst = h->g.st; need = h->n * 4ull; h->snap_full = 2; break;
        case SGC_DL_BITMAPS: dst = h->g.bm; need = h->n * 8ull; break;
        case SGC_DL_HIST: dst = h->g.hist; need = (uint64_t)h->hist_rows * h->maxc * 4; break;
        default: return fail(SGC_EINVAL, "upload target %d not writable", what);
    }
    if (bytes != need) return fail(SGC_EINVAL, "upload target %d needs exactly %llu bytes", what, (unsigned long long)need);
    CK(cudaMemcpyAsync(dst, src, need, cudaMemcpyHostToDevice, h->stream));
    TRY(set_clean(h, 0));  // colors from elsewhere: the next repair visits every vertex
    return sync(h);
}

int sgc_color_core(sgc_handle* h, uint32_t min_degree, uint32_t* colored) {
    if (!h) return fail(SGC_EINVAL, "null handle");
    CK(cudaSetDevice(h->device));
    std::vector<uint32_t> deg(h->n);
    CK(cudaMemcpyAsync(deg.data(), h->g.deg, (size_t)h->n * 4, cudaMemcpyDeviceToHost, h->stream));
    TRY(sync(h));
    std::vector<uint32_t> list;
    for (uint32_t x = 0; x < h->n; x++)
        if (deg[x] >= min_degree && deg[x] > 0) list.push_back(x);
    std::sort(list.begin(), list.end(), [&](uint32_t a, uint32_t b) { return deg[a] != deg[b] ? deg[a] > deg[b] : a < b; });
    uint32_t done = 0;
    if (!list.empty()) {
        uint32_t* d = nullptr;
        CK(cudaMallocAsync(&d, (list.size() + 1) * 4, h->stream));
        CK(cudaMemcpyAsync(d, list.data(), list.size() * 4, cudaMemcpyHostToDevice, h->stream));
        launch_color_list(h->g, d, (uint32_t)list.size(), d + list.size(), h->stream);
        h->launches += 1;
        CK(cudaMemcpyAsync(h->h_small, d + list.size(), 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaFreeAsync(d, h->stream));
        for (uint32_t k = 0; k < std::max<uint32_t>(h->sb.G, 1u); k++)  // every graph's next repair is full
            CK(cudaMemsetAsync(&h->g.gctl[k].clean, 0, 4, h->stream));
        TRY(sync(h));
        TRY(check_cuda("color_core"));
        done = h->h_small[0];
    }
    if (colored) *colored = done;
    return SGC_OK;
}

int sgc_find_color(sgc_handle* h, uint32_t x, uint16_t* color) {
    if (!h || !color) return fail(SGC_EINVAL, "null argument");
    if (x >= h->n) return fail(SGC_EINVAL, "vertex %u out of range", x);
    CK(cudaSetDevice(h->device));
    uint16_t* d = nullptr;
    CK(cudaMallocAsync(&d, 2, h->stream));
    find_color_kernel<<<1, 32, 0, h->stream>>>(h->g, x, d);
    CK(cudaMemcpyAsync(color, d, 2, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaFreeAsync(d, h->stream));
    return sync(h);
}

int sgc_validate(sgc_handle* h, sgc_validation* out) {
    if (!h || !out) return fail(SGC_EINVAL, "null argument");
    CK(cudaSetDevice(h->device));
    uint64_t v[5] = {0, 0, 0, 0, 0};
    const int r = run_validate(h->g, h->stream, v);
    if (r < 0) return fail(SGC_ECUDA, "validator failed (%d)", r);
    out->violations = v[0];
    out->uncolored_with_edges = v[1];
    out->edges = v[2];
    out->max_color = v[3];
    out->out_of_range = v[4];
    return SGC_OK;
}

int sgc_check_state(sgc_handle* h, sgc_state_report* out) {
    if (!h || !out) return fail(SGC_EINVAL, "null argument");
    CK(cudaSetDevice(h->device));
    uint64_t v[3] = {0, 0, 0};
    if (run_check_state(h->g, h->stream, v) < 0) return fail(SGC_ECUDA, "state check failed: %s", cudaGetErrorString(cudaGetLastError()));
    out->rows = h->n;
    out->bad_rows = v[0];
    out->flags = (uint32_t)v[1];
    out->first_bad = v[0] ? (uint32_t)v[2] : 0xFFFFFFFFu;
    return SGC_OK;
}

int sgc_get_stats(sgc_handle* h, sgc_stats* o) {
    if (!h || !o) return fail(SGC_EINVAL, "null argument");
    CK(cudaSetDevice(h->device));
    Ctl c;
    CK(cudaMemcpyAsync(&c, h->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
    h->d2h_bytes += sizeof(Ctl);
    TRY(sync(h));
    std::memset(o, 0, sizeof(*o));
    o->updates_submitted = h->updates;
    o->updates_skipped = c.nskip;
    o->epochs = h->epochs;
    o->overflow_pending = c.ovf_count;
    o->overflow_lost = c.ovf_lost;
    o->drain_failed = c.drain_failed;
    o->tier1_sweeps = h->tier1_sweeps;
    o->tier2_runs = h->tier2_runs;
    o->tier2_fixed = h->tier2_fixed;
    o->device_error = c.err;
    o->num_vertices = h->n;
    o->num_high_degree = h->num_hd;
    o->max_hist_colors = h->hist_rows ? h->maxc : 0;
    o->total_slots = h->total_slots;
    o->device_bytes = h->device_bytes;
    o->sweep_ms = h->sweep_ms;
    o->sweep_count = h->sweep_count;
    o->sweep_bytes = h->sweep_bytes;
    o->live_entries = h->live_entries;
    o->kernel_launches = h->launches;
    o->h2d_bytes = h->h2d_bytes;
    o->d2h_bytes = h->d2h_bytes;
    for (int k = 0; k < 4; k++) o->sweep_phase_ms[k] = h->sweep_phase_ms[k];
    o->hub_deferred = c.hub_total;
    return c.err ? fail(SGC_EDEVICE, "device error word 0x%x", c.err) : SGC_OK;
}

int sgc_synchronize(sgc_handle* h) {
    if (!h) return fail(SGC_EINVAL, "null handle");
    CK(cudaSetDevice(h->device));
    return sync(h);
}

void* sgc_cuda_stream(sgc_handle* h) { return h ? (void*)h->stream : nullptr; }

const char* sgc_last_error(void) { return g_err.c_str(); }

const char* sgc_version(void) { return "streamgc_b200 0.1 (sm_100a)"; }

}  // extern "C"
