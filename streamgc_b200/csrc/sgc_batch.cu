// sgc_batch.cu -- many graphs on one GPU (include/streamgc_batch.h).
//
// The graphs share one handle: their rows sit side by side in one slack CSR
// (graph k's vertex ids are offset by voff[k], a multiple of 32, so every
// 32-vertex word belongs to one graph and gidw maps words to graphs). A tick
//   1. applies the staged updates in one persistent launch fed by the device
//      ticket queue, a warp per edge (or, in stream-order mode, one warp per
//      graph walks that graph's updates in order);
//   2. compacts edited rows and drains the overflow buffer;
//   3. repairs with the independent-set rule, each graph starting from its
//      touched vertices (or from all of them when its repair must be full);
//      the loop is a conditional while-node of the captured CUDA graph;
//   4. publishes a snapshot for each graph whose epoch closed (double buffer
//      per graph: queries read the other half while the tick writes);
//   5. copies the loop state back for the host.
// A tick whose repair did not converge runs the sequential fallback (Tier-2)
// on the host's side of the stream and publishes again.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/streamgc_batch.h"
#include "sgc_internal.h"

using namespace sgc;
using namespace sgci;

namespace {

// Writes the colors of every graph whose target is 0 or 1 into that half of
// the snapshot double buffer. Thread per vertex.
__global__ void publish_graphs_kernel(Dev g, uint16_t* snap0, uint16_t* snap1, const uint8_t* __restrict__ target) {
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < g.n; x += gridDim.x * blockDim.x) {
        const uint8_t t = target[graph_of(g, x)];
        if (t < 2) (t ? snap1 : snap0)[x] = color_of(g.st[x]);
    }
}

__global__ void set_clean_all_kernel(GraphCtl* gc, uint32_t G) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < G; k += gridDim.x * blockDim.x) gc[k].clean = 1;
}

// Histogram-class rows of each graph: degree above the graph's threshold.
// hdidx holds the row index assigned for the lowest threshold on offer.
__global__ void rethreshold_kernel(Dev g, uint32_t* hdmap, const uint32_t* __restrict__ hdidx,
                                   const uint32_t* __restrict__ thr) {
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < g.n; x += gridDim.x * blockDim.x)
        hdmap[x] = g.deg[x] > thr[graph_of(g, x)] ? hdidx[x] : EMPTY;
}

constexpr uint32_t kMinThreshold = 32;  // lowest histogram threshold the tuner offers
constexpr uint32_t kQueryCap = 1u << 16;

}  // namespace

struct sgc_batch {
    sgc_handle* h = nullptr;
    uint32_t G = 0;
    uint32_t flags = 0;
    std::vector<uint32_t> voff, nv, epoch, since, pending, thr;
    std::vector<uint8_t> auto_thr;
    uint32_t cap = 0;
    // staging
    std::vector<std::vector<EdgeUpdate>> per_graph;  // stream-order mode: grouped by graph
    EdgeUpdate* h_stage = nullptr;                   // pinned, cap entries: the half being filled
    EdgeUpdate* h_stage_buf[2] = {nullptr, nullptr}; // two halves: the next tick's updates are staged
    uint32_t fill = 0;                               // while the current tick's are copied and applied
    uint32_t staged = 0;
    bool close_all = false;
    // per-tick control (device + pinned mirrors)
    uint32_t* d_dyn = nullptr;   // [0] updates, [2] segments, [4..5] Tier-2 span
    uint32_t* h_dyn = nullptr;
    uint32_t* d_segs = nullptr;  // G + 1
    uint32_t* h_segs = nullptr;
    uint8_t* d_target = nullptr; // per graph: snapshot half to write, 2 = none
    uint8_t* h_target = nullptr;
    uint32_t* d_thr = nullptr;
    uint32_t* d_hdidx = nullptr;
    std::vector<uint8_t> front;
    std::mutex front_mu;
    // captured tick
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // tuning
    uint32_t tile = SWEEP_CH;
    uint32_t bps = 0;
    // queries (own stream, fixed scratch)
    cudaStream_t qstream = nullptr;
    uint32_t* d_qv = nullptr;
    uint16_t* d_qout = nullptr;
    std::mutex qmu;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint64_t ticks = 0, tier2_ticks = 0;
    // tick in flight (begin .. end)
    bool in_tick = false;
    uint32_t tick_updates = 0, tick_published = 0;
    std::vector<uint8_t> close_one;    // per graph: close its epoch at the next tick
    std::vector<uint64_t> publishes;   // per graph: snapshots published so far
};

namespace {

uint32_t default_epoch(uint64_t nnz) {
    // staleness vs repair amortization: small graphs publish often
    if (nnz < (1ull << 16)) return 1024;
    if (nnz < (1ull << 22)) return 8192;
    return 32768;
}

void drop_graph(sgc_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// Everything of a tick before the repair loop.
void enqueue_head(sgc_batch* b, cudaStream_t s) {
    sgc_handle* h = b->h;
    if (b->flags & SGC_BATCH_STREAM_ORDER)
        launch_seg_apply(h->g, h->d_batch, b->d_segs, b->d_dyn, b->G, h->num_sms, s);
    else
        launch_conc_apply_dyn(h->g, h->d_batch, b->d_dyn, h->eo, h->num_sms, (int)b->bps, s);
    launch_add_check(h->g, h->d_batch, 0, b->d_dyn, h->num_sms, s);
    cudaMemsetAsync(&h->ctl->dirty_count, 0, 4, s);
    launch_dirty_list(h->g, h->dirty_list, &h->ctl->dirty_count, s);
    launch_compact(h->g, h->dirty_list, &h->ctl->dirty_count, h->n, false, s, (h->opt.flags & SGC_OPT_SORTED_ROWS) != 0);
    launch_take_overflow(h->g, &h->ctl->drain_n, s);
    launch_drain(h->g, &h->ctl->drain_n, (b->flags & SGC_BATCH_STREAM_ORDER) != 0, &h->ctl->drain_failed, s);
    const size_t mwords = ((h->n + 31) / 32) * 4;
    cudaMemsetAsync(h->sb.wmark, 0, mwords, s);
    cudaMemsetAsync(h->sb.rbits, 0, mwords, s);
    cudaMemsetAsync(h->sb.needf, 0, h->n, s);
    launch_repair_begin(h->g, h->sb, SWEEP_INDEP, h->num_sms, s);
}

void enqueue_tail(sgc_batch* b, cudaStream_t s) {
    sgc_handle* h = b->h;
    publish_graphs_kernel<<<h->num_sms * 8, 256, 0, s>>>(h->g, h->snap[0], h->snap[1], b->d_target);
    cudaMemcpyAsync(h->h_rc_out, h->sb.rc, sizeof(RepairCtl), cudaMemcpyDeviceToHost, s);
}

// Captures the whole tick: head, while-node { sweep, step }, tail.
int capture_tick_impl(sgc_batch* b);
int capture_tick(sgc_batch* b) {
    const int r = capture_tick_impl(b);
    if (r != SGC_OK) {  // leave the stream out of capture mode
        cudaStreamCaptureStatus st;
        if (cudaStreamIsCapturing(b->h->stream, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(b->h->stream, &g);
        }
        cudaGetLastError();
        drop_graph(b);
    }
    return r;
}
int capture_tick_impl(sgc_batch* b) {
    sgc_handle* h = b->h;
    cudaStream_t s = h->stream;
    drop_graph(b);
    CK(cudaGraphCreate(&b->graph, 0));
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, b->graph, 1, cudaGraphCondAssignDefault));
    CK(cudaStreamBeginCaptureToGraph(s, b->graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_head(b, s);
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
    CK(cudaGraphAddNode(&cnode, b->graph, head_tail.data(), head_tail.size(), &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    launch_repair_sweep(h->g, h->sb, SWEEP_INDEP, h->num_sms, s);
    launch_repair_step(h->g, h->sb, h->num_sms, s, &cond);
    cudaGraph_t g1 = nullptr;
    CK(cudaStreamEndCapture(s, &g1));
    CK(cudaStreamBeginCaptureToGraph(s, b->graph, &cnode, nullptr, 1, cudaStreamCaptureModeThreadLocal));
    enqueue_tail(b, s);
    cudaGraph_t g2 = nullptr;
    CK(cudaStreamEndCapture(s, &g2));
    CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
    return SGC_OK;
}

// Eager tick (no CUDA graph): the same kernels, the loop read back per sweep.
int run_tick_eager(sgc_batch* b) {
    sgc_handle* h = b->h;
    cudaStream_t s = h->stream;
    enqueue_head(b, s);
    for (;;) {
        launch_repair_sweep(h->g, h->sb, SWEEP_INDEP, h->num_sms, s);
        launch_repair_step(h->g, h->sb, h->num_sms, s, nullptr);
        CK(cudaMemcpyAsync(h->h_rc_out, h->sb.rc, sizeof(RepairCtl), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (!h->h_rc_out->cont) break;
    }
    enqueue_tail(b, s);
    return check_cuda("batch tick");
}

}  // namespace

extern "C" {

int sgc_batch_default_options(sgc_batch_options* o) {
    if (!o) return fail(SGC_EINVAL, "null options");
    std::memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(sgc_batch_options);
    o->slack_pct = SGC_CSR_EXTRA_SLACK_PCT_DEFAULT;
    o->max_tick_updates = 1u << 20;
    o->flags = SGC_BATCH_CUDA_GRAPH;
    o->repair_tile = SWEEP_CH;
    return SGC_OK;
}

int sgc_batch_destroy(sgc_batch* b) {
    if (!b) return SGC_OK;
    if (b->h) cudaSetDevice(b->h->device);
    drop_graph(b);
    for (EdgeUpdate* p : b->h_stage_buf)
        if (p) cudaFreeHost(p);
    if (b->h_dyn) cudaFreeHost(b->h_dyn);
    if (b->h_segs) cudaFreeHost(b->h_segs);
    if (b->h_target) cudaFreeHost(b->h_target);
    for (void* p : {(void*)b->d_dyn, (void*)b->d_segs, (void*)b->d_target, (void*)b->d_thr, (void*)b->d_hdidx,
                    (void*)b->d_qv, (void*)b->d_qout})
        if (p) cudaFree(p);
    if (b->qstream) cudaStreamDestroy(b->qstream);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->h) sgc_destroy(b->h);
    delete b;
    return SGC_OK;
}

int sgc_batch_create(const sgc_batch_graph* graphs, uint32_t count, const sgc_batch_options* opt_in, sgc_batch** out) {
    if (!graphs || !count || !out) return fail(SGC_EINVAL, "null argument");
    *out = nullptr;
    sgc_batch_options opt;
    sgc_batch_default_options(&opt);
    if (opt_in) {
        if (opt_in->struct_size != sizeof(sgc_batch_options)) return fail(SGC_EINVAL, "sgc_batch_options.struct_size mismatch");
        opt = *opt_in;
    }
    if (opt.max_tick_updates == 0) return fail(SGC_EINVAL, "max_tick_updates must be positive");
    // union layout
    std::vector<uint32_t> voff(count), nv(count);
    uint64_t N = 0, nnz = 0;
    for (uint32_t k = 0; k < count; k++) {
        const sgc_batch_graph& gr = graphs[k];
        if (!gr.row_ptr || (gr.row_ptr[gr.num_vertices] && !gr.col_idx)) return fail(SGC_EINVAL, "graph %u: null CSR", k);
        if (gr.num_vertices == 0) return fail(SGC_EINVAL, "graph %u: no vertices", k);
        voff[k] = (uint32_t)N;
        nv[k] = gr.num_vertices;
        N += ((uint64_t)gr.num_vertices + 31) & ~31ull;
        nnz += gr.row_ptr[gr.num_vertices];
        if (N >= (1ull << 31)) return fail(SGC_EINVAL, "batch holds 2^31 vertices or more");
    }
    const uint32_t n = (uint32_t)N;
    std::vector<uint64_t> rp((size_t)n + 1, 0);
    std::vector<uint32_t> deg(n, 0), gidw(n / 32), thr_word(n / 32);
    std::vector<uint64_t> base(count);
    for (uint32_t k = 0; k < count; k++) {
        const sgc_batch_graph& gr = graphs[k];
        base[k] = rp[voff[k]];
        for (uint32_t x = 0; x < gr.num_vertices; x++) {
            const uint64_t len = gr.row_ptr[x + 1] - gr.row_ptr[x];
            rp[voff[k] + x + 1] = rp[voff[k] + x] + len;
            deg[voff[k] + x] = gr.degree ? gr.degree[x] : (uint32_t)len;
        }
        const uint32_t end = voff[k] + ((gr.num_vertices + 31) & ~31u);
        for (uint32_t x = voff[k] + gr.num_vertices; x < end; x++) rp[x + 1] = rp[x];
        for (uint32_t w = voff[k] / 32; w < end / 32; w++) {
            gidw[w] = k;
            thr_word[w] = gr.histogram_threshold ? gr.histogram_threshold : kMinThreshold;
        }
    }
    std::vector<uint32_t> col(nnz);
    int bad = 0;
    for (uint32_t k = 0; k < count; k++) {
        const sgc_batch_graph& gr = graphs[k];
        const uint64_t m = gr.row_ptr[gr.num_vertices];
        const uint32_t off = voff[k], lim = gr.num_vertices;
        uint32_t* dst = col.data() + base[k];
#pragma omp parallel for schedule(static) reduction(| : bad)
        for (int64_t j = 0; j < (int64_t)m; j++) {
            const uint32_t y = gr.col_idx[j];
            if (y >= lim) bad |= 1;
            dst[j] = y + off;
        }
        if (bad) return fail(SGC_EINVAL, "graph %u: col_idx entry >= num_vertices", k);
    }
    StreamGCConfig cfg = sgc_default_config();
    cfg.num_vertices = n;
    cfg.num_edges = nnz;
    cfg.epoch_size = 32768;
    cfg.histogram_threshold = 64;
    sgc_options hopt;
    sgc_default_options(&hopt);
    hopt.slack_pct = opt.slack_pct;
    hopt.max_batch = opt.max_tick_updates;
    hopt.device = opt.device;
    hopt.flags = SGC_OPT_EXACT_SELECT | ((opt.flags & SGC_BATCH_SORTED_ROWS) ? SGC_OPT_SORTED_ROWS : 0u);
    hopt.full_repair_every = 0;  // a graph is repaired in full only when it needs it
    hopt.repair_tile = opt.repair_tile ? opt.repair_tile : SWEEP_CH;
    CreateExtra ex{thr_word.data(), gidw.data(), count, voff.data()};
    sgc_batch* b = new sgc_batch();
    int r = create_internal(&cfg, &hopt, rp.data(), col.data(), deg.data(), &ex, &b->h);
    if (r != SGC_OK) {
        delete b;
        return r;
    }
    auto bail = [&](int code) { sgc_batch_destroy(b); return code; };
    sgc_handle* h = b->h;
    b->G = count;
    b->flags = opt.flags;
    b->voff = voff;
    b->nv = nv;
    b->cap = opt.max_tick_updates;
    b->tile = h->sb.tile;
    b->bps = opt.apply_blocks_per_sm;
    b->epoch.resize(count);
    b->thr.resize(count);
    b->auto_thr.resize(count);
    for (uint32_t k = 0; k < count; k++) {
        b->epoch[k] = graphs[k].epoch_size ? graphs[k].epoch_size : default_epoch(graphs[k].row_ptr[graphs[k].num_vertices]);
        b->auto_thr[k] = graphs[k].histogram_threshold ? 0 : 1;
        b->thr[k] = graphs[k].histogram_threshold ? graphs[k].histogram_threshold : 64;
    }
    b->since.assign(count, 0);
    b->pending.assign(count, 0);
    b->front.assign(count, 0);
    b->close_one.assign(count, 0);
    b->publishes.assign(count, 0);
    b->per_graph.resize(count);
    // hdmap as created (threshold 32 where tunable) is the index source for re-thresholding
    if (cudaMalloc(&b->d_hdidx, (size_t)n * 4) || cudaMalloc(&b->d_thr, (size_t)count * 4) ||
        cudaMalloc(&b->d_dyn, 32) || cudaMalloc(&b->d_segs, ((size_t)count + 1) * 4) || cudaMalloc(&b->d_target, count) ||
        cudaMalloc(&b->d_qv, kQueryCap * 4) || cudaMalloc(&b->d_qout, kQueryCap * 2)) {
        cudaGetLastError();
        return bail(fail(SGC_ENOMEM, "batch control allocation failed"));
    }
    if (cudaHostAlloc(&b->h_stage_buf[0], (size_t)b->cap * sizeof(EdgeUpdate), cudaHostAllocDefault) ||
        cudaHostAlloc(&b->h_stage_buf[1], (size_t)b->cap * sizeof(EdgeUpdate), cudaHostAllocDefault) ||
        cudaHostAlloc(&b->h_dyn, 16, cudaHostAllocDefault) ||
        cudaHostAlloc(&b->h_segs, ((size_t)count + 1) * 4, cudaHostAllocDefault) ||
        cudaHostAlloc(&b->h_target, count, cudaHostAllocDefault)) {
        cudaGetLastError();
        return bail(fail(SGC_ENOMEM, "batch staging allocation failed"));
    }
    b->h_stage = b->h_stage_buf[0];
    CK(cudaMemcpyAsync(b->d_hdidx, h->g.hdmap, (size_t)n * 4, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(b->d_thr, b->thr.data(), (size_t)count * 4, cudaMemcpyHostToDevice, h->stream));
    rethreshold_kernel<<<h->num_sms * 8, 256, 0, h->stream>>>(h->g, const_cast<uint32_t*>(h->g.hdmap), b->d_hdidx,
                                                               b->d_thr);
    CK(cudaMemsetAsync(b->d_dyn, 0, 16, h->stream));
    // repair control: host fields stay fixed for the batch
    RepairCtl* hin = h->h_rc_in;
    hin->mode = SWEEP_INDEP;
    hin->max_sweeps = 64;
    hin->force_all = 0;
    CK(cudaMemcpyAsync(h->sb.rc, hin, 12, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamCreateWithFlags(&b->qstream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&b->ev0));
    CK(cudaEventCreate(&b->ev1));
    CK(cudaStreamSynchronize(h->stream));
    if ((r = check_cuda("batch create"))) return bail(r);
    *out = b;
    return SGC_OK;
}

uint32_t sgc_batch_num_graphs(const sgc_batch* b) { return b ? b->G : 0; }
uint32_t sgc_batch_epoch_size(const sgc_batch* b, uint32_t graph) {
    return (b && graph < b->G) ? b->epoch[graph] : 0;
}
uint64_t sgc_batch_pending(const sgc_batch* b) { return b ? b->staged : 0; }

int sgc_batch_submit(sgc_batch* b, uint32_t graph, const EdgeUpdate* ups, uint32_t n) {
    if (!b || (n && !ups)) return fail(SGC_EINVAL, "null argument");
    if (graph >= b->G) return fail(SGC_EINVAL, "graph %u out of range", graph);
    if ((uint64_t)b->staged + n > b->cap) return fail(SGC_EINVAL, "tick buffer full (%u updates)", b->cap);
    const uint32_t off = b->voff[graph], lim = b->nv[graph];
    auto translate = [&](const EdgeUpdate& e) {
        EdgeUpdate t = e;
        t.u = e.u < lim ? e.u + off : SGC_CSR_INVALID;  // outside the graph: skipped on the device
        t.v = e.v < lim ? e.v + off : SGC_CSR_INVALID;
        return t;
    };
    if (b->flags & SGC_BATCH_STREAM_ORDER) {
        auto& q = b->per_graph[graph];
        for (uint32_t i = 0; i < n; i++) q.push_back(translate(ups[i]));
    } else {
        EdgeUpdate* dst = b->h_stage + b->staged;
        for (uint32_t i = 0; i < n; i++) dst[i] = translate(ups[i]);
    }
    b->staged += n;
    b->pending[graph] += n;
    return SGC_OK;
}

int sgc_batch_close_epochs(sgc_batch* b) {
    if (!b) return fail(SGC_EINVAL, "null batch");
    b->close_all = true;
    return SGC_OK;
}

int sgc_batch_close_epoch(sgc_batch* b, uint32_t graph) {
    if (!b) return fail(SGC_EINVAL, "null batch");
    if (graph >= b->G) return fail(SGC_EINVAL, "graph %u out of range", graph);
    b->close_one[graph] = 1;
    return SGC_OK;
}

uint64_t sgc_batch_publish_count(const sgc_batch* b, uint32_t graph) {
    return (b && graph < b->G) ? b->publishes[graph] : 0;
}

int sgc_batch_tick(sgc_batch* b, sgc_batch_tick_report* rep) {
    TRY(sgc_batch_tick_begin(b));
    return sgc_batch_tick_end(b, rep);
}

int sgc_batch_tick_begin(sgc_batch* b) {
    if (!b) return fail(SGC_EINVAL, "null batch");
    if (b->in_tick) return fail(SGC_EINVAL, "a tick is already running");
    sgc_handle* h = b->h;
    CK(cudaSetDevice(h->device));
    const uint32_t G = b->G;
    uint32_t published = 0;
    for (uint32_t k = 0; k < G; k++) {
        b->since[k] += b->pending[k];
        const bool pub = b->close_all || b->close_one[k] || b->since[k] >= b->epoch[k];
        b->h_target[k] = pub ? (uint8_t)(1 - b->front[k]) : 2;
        b->close_one[k] = 0;
        if (pub) {
            b->since[k] = 0;
            published++;
        }
    }
    b->close_all = false;
    b->tick_published = published;
    uint32_t nup = b->staged;
    if (b->flags & SGC_BATCH_STREAM_ORDER) {
        uint32_t pos = 0;
        for (uint32_t k = 0; k < G; k++) {
            b->h_segs[k] = pos;
            auto& q = b->per_graph[k];
            if (!q.empty()) std::memcpy(b->h_stage + pos, q.data(), q.size() * sizeof(EdgeUpdate));
            pos += (uint32_t)q.size();
            q.clear();
        }
        b->h_segs[G] = pos;
        CK(cudaMemcpyAsync(b->d_segs, b->h_segs, ((size_t)G + 1) * 4, cudaMemcpyHostToDevice, h->stream));
    }
    b->h_dyn[0] = nup;
    b->h_dyn[2] = G;
    CK(cudaMemcpyAsync(b->d_dyn, b->h_dyn, 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(b->d_dyn + 2, b->h_dyn + 2, 4, cudaMemcpyHostToDevice, h->stream));
    if (nup) CK(cudaMemcpyAsync(h->d_batch, b->h_stage, (size_t)nup * sizeof(EdgeUpdate), cudaMemcpyHostToDevice, h->stream));
    // the staged updates are consumed: the next tick's go to the other half (its
    // copy belonged to the previous tick, which has ended)
    for (uint32_t k = 0; k < G; k++) b->pending[k] = 0;
    b->staged = 0;
    b->fill ^= 1u;
    b->h_stage = b->h_stage_buf[b->fill];
    CK(cudaMemcpyAsync(b->d_target, b->h_target, G, cudaMemcpyHostToDevice, h->stream));
    h->h2d_bytes += (uint64_t)nup * sizeof(EdgeUpdate) + G + 8;
    const bool prof = (b->flags & SGC_BATCH_PROFILE) != 0;
    if (prof) CK(cudaEventRecord(b->ev0, h->stream));
    if (b->flags & SGC_BATCH_CUDA_GRAPH) {
        if (!b->exec) TRY(capture_tick(b));
        CK(cudaGraphLaunch(b->exec, h->stream));
    } else {
        TRY(run_tick_eager(b));
    }
    if (prof) CK(cudaEventRecord(b->ev1, h->stream));
    b->tick_updates = nup;
    b->in_tick = true;
    return SGC_OK;
}

int sgc_batch_tick_end(sgc_batch* b, sgc_batch_tick_report* rep) {
    if (!b) return fail(SGC_EINVAL, "null batch");
    if (!b->in_tick) return fail(SGC_EINVAL, "no tick is running");
    b->in_tick = false;
    sgc_handle* h = b->h;
    CK(cudaSetDevice(h->device));
    const uint32_t G = b->G;
    const uint32_t nup = b->tick_updates, published = b->tick_published;
    const bool prof = (b->flags & SGC_BATCH_PROFILE) != 0;
    CK(cudaStreamSynchronize(h->stream));
    TRY(check_cuda("batch tick"));
    const RepairCtl rc = *h->h_rc_out;
    h->d2h_bytes += sizeof(RepairCtl);
    bool proper = rc.done && rc.sym == 0;
    uint32_t t2 = 0;
    if (!proper) {  // sequential fallback, then publish again
        bool gave_up = false;
        // only the graphs the repair left unresolved (repair_step_kernel sets GraphCtl.t2),
        // over the vertex span from the first to the last of them
        launch_t2_span(h->g, G, b->d_dyn + 4, h->stream);
        h->launches++;
        CK(cudaMemcpyAsync(h->h_small, b->d_dyn + 4, 8, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        const uint32_t lo = h->h_small[0], hi = h->h_small[1];
        const uint32_t fixed = run_tier2(h->g, h->t2, h->stream, h->h_small, &gave_up, &h->launches, true, lo, hi);
        TRY(check_cuda("batch tier2"));
        h->tier2_runs++;
        h->tier2_fixed += fixed;
        t2 = 1;
        proper = !gave_up;
        if (proper) set_clean_all_kernel<<<(G + 255) / 256, 256, 0, h->stream>>>(h->g.gctl, G);
        publish_graphs_kernel<<<h->num_sms * 8, 256, 0, h->stream>>>(h->g, h->snap[0], h->snap[1], b->d_target);
        CK(cudaStreamSynchronize(h->stream));
        TRY(check_cuda("batch republish"));
        b->tier2_ticks++;
    }
    {
        std::lock_guard<std::mutex> lk(b->front_mu);
        for (uint32_t k = 0; k < G; k++)
            if (b->h_target[k] < 2) {
                b->front[k] = b->h_target[k];
                b->publishes[k]++;
            }
    }
    h->updates += nup;
    h->tier1_sweeps += rc.it;
    h->epochs += published;
    b->ticks++;
    if (rep) {
        std::memset(rep, 0, sizeof(*rep));
        rep->updates = nup;
        rep->published = published;
        rep->tier1_iterations = rc.it;
        rep->tier2_ran = t2;
        rep->tier2_reason = (rc.sym != 0 ? 1u : 0u) | (rc.done ? 0u : 2u);
        rep->proper = proper ? 1 : 0;
        if (prof) {
            float ms = 0;
            cudaEventElapsedTime(&ms, b->ev0, b->ev1);
            rep->device_ms = ms;
        }
    }
    return SGC_OK;
}

int sgc_batch_query(sgc_batch* b, uint32_t graph, const uint32_t* v, uint16_t* out, uint32_t k) {
    if (!b || (k && (!v || !out))) return fail(SGC_EINVAL, "null argument");
    if (graph >= b->G) return fail(SGC_EINVAL, "graph %u out of range", graph);
    if (!k) return SGC_OK;
    std::lock_guard<std::mutex> lk(b->qmu);
    CK(cudaSetDevice(b->h->device));
    const uint16_t* snap;
    {
        std::lock_guard<std::mutex> lf(b->front_mu);
        snap = b->h->snap[b->front[graph]] + b->voff[graph];
    }
    for (uint32_t s = 0; s < k; s += kQueryCap) {
        const uint32_t m = std::min(kQueryCap, k - s);
        CK(cudaMemcpyAsync(b->d_qv, v + s, (size_t)m * 4, cudaMemcpyHostToDevice, b->qstream));
        launch_query(snap, b->nv[graph], b->d_qv, b->d_qout, m, b->qstream);
        CK(cudaMemcpyAsync(out + s, b->d_qout, (size_t)m * 2, cudaMemcpyDeviceToHost, b->qstream));
    }
    CK(cudaStreamSynchronize(b->qstream));
    return check_cuda("batch query");
}

int sgc_batch_snapshot(sgc_batch* b, uint32_t graph, uint16_t* out) {
    if (!b || !out) return fail(SGC_EINVAL, "null argument");
    if (graph >= b->G) return fail(SGC_EINVAL, "graph %u out of range", graph);
    std::lock_guard<std::mutex> lk(b->qmu);
    CK(cudaSetDevice(b->h->device));
    const uint16_t* snap;
    {
        std::lock_guard<std::mutex> lf(b->front_mu);
        snap = b->h->snap[b->front[graph]] + b->voff[graph];
    }
    CK(cudaMemcpyAsync(out, snap, (size_t)b->nv[graph] * 2, cudaMemcpyDeviceToHost, b->qstream));
    CK(cudaStreamSynchronize(b->qstream));
    return SGC_OK;
}

int sgc_batch_rows(sgc_batch* b, uint32_t graph, uint64_t* row_ptr, uint32_t* col, uint64_t col_cap) {
    if (!b || !row_ptr) return fail(SGC_EINVAL, "null argument");
    if (graph >= b->G) return fail(SGC_EINVAL, "graph %u out of range", graph);
    sgc_handle* h = b->h;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    const uint32_t off = b->voff[graph], nvx = b->nv[graph];
    std::vector<uint64_t> rp((size_t)nvx + 1);
    std::vector<uint32_t> hw(nvx);
    CK(cudaMemcpy(rp.data(), h->g.rp + off, ((size_t)nvx + 1) * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hw.data(), h->g.hw + off, (size_t)nvx * 4, cudaMemcpyDeviceToHost));
    const uint64_t s0 = rp[0], s1 = rp[nvx];
    std::vector<uint32_t> slots(s1 - s0);
    if (s1 > s0) CK(cudaMemcpy(slots.data(), h->g.col + s0, (s1 - s0) * 4, cudaMemcpyDeviceToHost));
    uint64_t pos = 0;
    row_ptr[0] = 0;
    for (uint32_t x = 0; x < nvx; x++) {
        const uint64_t len = std::min<uint64_t>(hw[x], rp[x + 1] - rp[x]);  // a mark never exceeds the row
        for (uint64_t j = rp[x] - s0; j < rp[x] - s0 + len; j++) {
            const uint32_t y = slots[j];
            if (y >= off && y < off + nvx) {  // live entries only (INV and deleted run entries are >= 2^31)
                if (col) {
                    if (pos >= col_cap) return fail(SGC_EINVAL, "col_cap too small");
                    col[pos] = y - off;
                }
                pos++;
            }
        }
        row_ptr[x + 1] = pos;
    }
    return SGC_OK;
}

int sgc_batch_color_core(sgc_batch* b, uint32_t min_degree, uint32_t* colored) {
    if (!b) return fail(SGC_EINVAL, "null batch");
    return sgc_color_core(b->h, min_degree, colored);
}

int sgc_batch_validate(sgc_batch* b, sgc_validation* out) {
    if (!b) return fail(SGC_EINVAL, "null batch");
    return sgc_validate(b->h, out);
}

int sgc_batch_dropped(sgc_batch* b, uint8_t* out) {
    if (!b || !out) return fail(SGC_EINVAL, "null argument");
    if (b->in_tick) return fail(SGC_EINVAL, "a tick is running");
    sgc_handle* h = b->h;
    CK(cudaSetDevice(h->device));
    std::vector<GraphCtl> gc(b->G);
    CK(cudaMemcpyAsync(gc.data(), h->g.gctl, (size_t)b->G * sizeof(GraphCtl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->d2h_bytes += (uint64_t)b->G * sizeof(GraphCtl);
    for (uint32_t k = 0; k < b->G; k++) out[k] = gc[k].dropped ? 1 : 0;
    return SGC_OK;
}

int sgc_batch_check_state(sgc_batch* b, sgc_state_report* out) {
    if (!b) return fail(SGC_EINVAL, "null batch");
    if (b->in_tick) return fail(SGC_EINVAL, "a tick is running");
    return sgc_check_state(b->h, out);
}

int sgc_batch_stats(sgc_batch* b, sgc_stats* out) {
    if (!b) return fail(SGC_EINVAL, "null batch");
    return sgc_get_stats(b->h, out);
}

int sgc_batch_get_tuning(sgc_batch* b, sgc_batch_tuning* t) {
    if (!b || !t) return fail(SGC_EINVAL, "null argument");
    t->repair_tile = b->tile;
    t->apply_blocks_per_sm = b->bps ? b->bps : (uint32_t)conc_apply_occupancy();
    return SGC_OK;
}

int sgc_batch_set_tuning(sgc_batch* b, const sgc_batch_tuning* t) {
    if (!b || !t) return fail(SGC_EINVAL, "null argument");
    if (t->repair_tile < SWEEP_CH_MIN || t->repair_tile > 2048 || t->repair_tile % 32)
        return fail(SGC_EINVAL, "repair_tile must be a multiple of 32 in [%u, 2048]", SWEEP_CH_MIN);
    b->tile = t->repair_tile;
    b->h->sb.tile = t->repair_tile;
    b->bps = t->apply_blocks_per_sm;
    drop_graph(b);  // launch shapes and kernel arguments changed: capture again
    return SGC_OK;
}

int sgc_batch_set_thresholds(sgc_batch* b, uint32_t threshold);

int sgc_batch_autotune(sgc_batch* b, sgc_batch_feed_fn feed, void* ctx, uint32_t ticks_per_candidate,
                       sgc_batch_tuning* chosen) {
    if (!b || !feed) return fail(SGC_EINVAL, "null argument");
    if (!ticks_per_candidate) ticks_per_candidate = 2;
    const uint32_t saved_flags = b->flags;
    b->flags |= SGC_BATCH_PROFILE;
    auto trial = [&](double* ms_per_update) -> int {
        double ms = 0;
        uint64_t ups = 0;
        for (uint32_t t = 0; t < ticks_per_candidate; t++) {
            TRY(feed(b, ctx));
            sgc_batch_tick_report r;
            TRY(sgc_batch_tick(b, &r));
            if (t > 0 || ticks_per_candidate == 1) {  // the first tick of a candidate also captures its graph
                ms += r.device_ms;
                ups += r.updates;
            }
        }
        *ms_per_update = ups ? ms / (double)ups : 1e30;
        return SGC_OK;
    };
    sgc_batch_tuning best;
    sgc_batch_get_tuning(b, &best);
    double best_cost = 1e30;
    // coordinate 1: repair tile width
    for (uint32_t tile : {256u, 512u, 1024u, 2048u}) {
        sgc_batch_tuning t = best;
        t.repair_tile = tile;
        TRY(sgc_batch_set_tuning(b, &t));
        double c;
        TRY(trial(&c));
        if (c < best_cost) {
            best_cost = c;
            best = t;
        }
    }
    // coordinate 2: resident apply warps (blocks of 8 warps per SM)
    const uint32_t occ = (uint32_t)conc_apply_occupancy();
    const uint32_t start_bps = best.apply_blocks_per_sm;
    for (uint32_t bps = 1; bps <= occ; bps++) {
        if (bps == start_bps) continue;
        sgc_batch_tuning t = best;
        t.apply_blocks_per_sm = bps;
        TRY(sgc_batch_set_tuning(b, &t));
        double c;
        TRY(trial(&c));
        if (c < best_cost) {
            best_cost = c;
            best = t;
        }
    }
    // coordinate 3: histogram threshold of the graphs created without one
    uint32_t best_thr = 0;
    for (uint32_t thr : {32u, 64u, 128u}) {
        TRY(sgc_batch_set_tuning(b, &best));
        TRY(sgc_batch_set_thresholds(b, thr));
        double c;
        TRY(trial(&c));
        if (c < best_cost || best_thr == 0) {
            if (c < best_cost) best_cost = c;
            best_thr = thr;
        }
    }
    TRY(sgc_batch_set_thresholds(b, best_thr));
    TRY(sgc_batch_set_tuning(b, &best));
    b->flags = saved_flags;
    drop_graph(b);
    if (chosen) *chosen = best;
    return SGC_OK;
}

// Histogram threshold of every graph created without one (tuned); rows keep
// the index they were given for the lowest threshold on offer.
int sgc_batch_set_thresholds(sgc_batch* b, uint32_t threshold) {
    if (!b) return fail(SGC_EINVAL, "null batch");
    if (threshold < kMinThreshold) return fail(SGC_EINVAL, "threshold below %u", kMinThreshold);
    sgc_handle* h = b->h;
    for (uint32_t k = 0; k < b->G; k++)
        if (b->auto_thr[k]) b->thr[k] = threshold;
    CK(cudaMemcpyAsync(b->d_thr, b->thr.data(), (size_t)b->G * 4, cudaMemcpyHostToDevice, h->stream));
    rethreshold_kernel<<<h->num_sms * 8, 256, 0, h->stream>>>(h->g, const_cast<uint32_t*>(h->g.hdmap), b->d_hdidx,
                                                               b->d_thr);
    CK(cudaStreamSynchronize(h->stream));
    return check_cuda("rethreshold");
}

}  // extern "C"
