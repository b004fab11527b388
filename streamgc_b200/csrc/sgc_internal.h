// sgc_internal.h -- internals shared by the handle API (sgc_api.cu) and the
// batched engine (sgc_batch.cu): the handle layout and the host-side building
// blocks of an epoch. Not part of the public interface.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <utility>
#include <atomic>
#include <vector>

#include "../../include/streamgc_b200.h"
#include "sgc_kernels.cuh"

namespace sgci {
using namespace sgc;

// Records the message returned by sgc_last_error(); returns `code`.
int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));

#define CK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fail(SGC_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
    } while (0)

// Control block on the device: counters every kernel family writes.
struct Ctl {
    uint32_t ovf_count;
    uint32_t err;
    uint32_t drain_n;
    uint32_t dirty_count;
    uint32_t item_count;
    uint32_t pend_count;
    uint32_t fac_count;
    uint32_t ticket;
    uint32_t hub_count;  // row-scale operations deferred by the last concurrent batch
    uint32_t hub_pad;
    unsigned long long ovf_lost;
    unsigned long long nskip;
    unsigned long long drain_failed;
    unsigned long long symsum;
    unsigned long long live;
    unsigned long long hub_total;  // cumulative: operations the pass after concurrent batches finished
    unsigned long long pad[2];
};

}  // namespace sgci

// One handle: a graph (or several, side by side) resident on one GPU.
struct sgc_handle {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    sgc_options opt{};
    StreamGCConfig cfg{};
    uint32_t n = 0, num_hd = 0, maxc = 1024, hist_rows = 0;
    uint64_t total_slots = 0;
    uint64_t device_bytes = 0;
    sgc::Dev g{};
    // owned device buffers
    std::vector<void*> allocs;
    sgci::Ctl* ctl = nullptr;
    uint16_t* snap[2] = {nullptr, nullptr};
    int front = 0;
    // incremental snapshots (g.chg set): the marks of the epoch before, and how
    // many more snapshots must be written in full (both halves once at first,
    // again after states were uploaded)
    uint32_t* chg_prev = nullptr;
    int snap_full = 2;
    EdgeUpdate* d_batch = nullptr;
    EdgeUpdate* h_stage = nullptr;  // pinned staging for pageable inputs
    cudaEvent_t stage_free = nullptr;
    sgc::EdgeOrder eo{};
    sgc::SweepBufs sb{};
    uint32_t* dirty_list = nullptr;
    sgc::Tier2Bufs t2{};
    uint32_t* h_small = nullptr;         // pinned readback scratch
    sgc::RepairCtl* h_rc_in = nullptr;   // pinned: host fields of the repair control block
    sgc::RepairCtl* h_rc_out = nullptr;  // pinned: its readback
    uint64_t repairs_since_full = 0;
    int last_mode = SGC_MODE_DETERMINISTIC;
    // host counters
    uint64_t updates = 0, epochs = 0, tier1_sweeps = 0, tier2_runs = 0, tier2_fixed = 0;
    // profiling
    std::vector<cudaEvent_t> ev_pool;
    struct SweepEvents {
        cudaEvent_t ev[5];  // start, after the item build, the long-row items, the finalize; end
    };
    std::vector<SweepEvents> ev_pending;
    double sweep_ms = 0;
    double sweep_phase_ms[4] = {0, 0, 0, 0};  // item build, long-row items, finalize, selection + commit
    uint64_t sweep_count = 0, sweep_bytes = 0, live_entries = 0;
    // stream ingest: two device slots filled on a copy stream (allocated on first use)
    cudaStream_t copy_stream = nullptr;
    EdgeUpdate* slot_dev[2] = {nullptr, nullptr};
    EdgeUpdate* slot_host[2] = {nullptr, nullptr};  // pinned
    cudaEvent_t copy_done[2] = {nullptr, nullptr};
    cudaEvent_t slot_free[2] = {nullptr, nullptr};
    uint32_t slot_n[2] = {0, 0};
    uint32_t stage_next = 0, staged = 0;  // next slot to fill; slots holding a batch (oldest first from stage_next - staged)
    // ingest ring (sgc_ring_*): pinned, device-mapped slots the GPU copies from itself.
    // Positions count updates since creation; slot = position & ring_mask.
    EdgeUpdate* ring_host = nullptr;     // 2^k slots, written by the producer
    EdgeUpdate* ring_dev = nullptr;      // the same memory as the GPU addresses it
    uint64_t ring_mask = 0;
    std::atomic<uint64_t> ring_tail{0};      // producer: positions published (slots written)
    std::atomic<uint64_t> ring_released{0};  // consumer: positions whose gather has finished
    uint64_t ring_head = 0;              // consumer: positions gathered (launched)
    uint64_t ring_inflight = 0;          // consumer: end of the last launched gather
    cudaEvent_t ring_done = nullptr;     // recorded after the last gather
    // SGC_OPT_GRAPH_PUBLISH: the publish captured once per snapshot half
    cudaGraph_t pub_graph[2] = {nullptr, nullptr};
    cudaGraphExec_t pub_exec[2] = {nullptr, nullptr};
    bool pub_graph_failed = false;  // capture failed: the eager publish
    uint64_t launches = 0;          // kernels this handle launched
    uint64_t h2d_bytes = 0, d2h_bytes = 0;  // bytes the library moved across PCIe / C2C
};

namespace sgci {

template <class T>
int dalloc(sgc_handle* h, T** p, size_t count, int fill = -1) {
    const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(SGC_ENOMEM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    }
    h->allocs.push_back(q);
    h->device_bytes += bytes;
    if (fill >= 0) CK(cudaMemsetAsync(q, fill, bytes, h->stream));
    *p = (T*)q;
    return SGC_OK;
}

#define TRY(x)                   \
    do {                         \
        int r_ = (x);            \
        if (r_ != SGC_OK) return r_; \
    } while (0)


int check_cuda(const char* where);
cudaEvent_t take_event(sgc_handle* h);
int sync(sgc_handle* h);
int compact_dirty(sgc_handle* h, bool force);
int drain(sgc_handle* h, bool ordered, unsigned long long* failed_counter);
int set_clean(sgc_handle* h, uint32_t v);
int repair_loop(sgc_handle* h, sgc_repair_report* rep, bool force_full);
int finish_repair(sgc_handle* h, sgc_repair_report* rep);
int apply_device(sgc_handle* h, const EdgeUpdate* src, uint32_t n, int mode);
int ensure_ingest(sgc_handle* h);
void drop_publish_graphs(sgc_handle* h);
// Extra layout of a handle that holds several graphs (the batched engine).
struct CreateExtra {
    const uint32_t* thr_word;  // per 32-vertex word: histogram threshold (null: cfg->histogram_threshold)
    const uint32_t* gidw;      // per 32-vertex word: graph id (null: one graph)
    uint32_t G;                // graphs
    const uint32_t* base;      // per graph: first vertex (null: 0)
};
int create_internal(const StreamGCConfig* cfg, const sgc_options* opt_in, const uint64_t* row_ptr,
                    const uint32_t* col_idx, const uint32_t* degree, const CreateExtra* ex, sgc_handle** out);

}  // namespace sgci

