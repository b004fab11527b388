// sgc_server.cpp -- the request loop of the served form (include/streamgc_server.h).
//
// Host-side scheduling only: tenants live in groups, each group one batched
// engine (sgc_batch) holding the tenants admitted together. Submissions are
// held on the host per tenant; a step frees the groups whose tenants all left,
// admits queued tenants that fit the HBM budget (one new group per step),
// forwards the held requests to their groups, closes the epochs that reached
// their staleness deadline, and ticks every group with work: all ticks are
// launched first and waited for afterwards (with the lock released, so
// queries and submits go on), so the groups' kernels overlap on the device.
// Lock order: `life` (group lifetime) before `mu` (tables). Tenants removed
// while their group is being created end when the creation is done.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <mutex>
#include <shared_mutex>
#include <unordered_set>
#include <vector>

#include "../../include/streamgc_server.h"
#include "sgc_host.h"

namespace sgci {
int fail(int code, const char* fmt, ...);  // sgc_api.cu: sets the message sgc_last_error() returns
}

namespace {

int bad(const char* what) { return sgci::fail(SGC_EINVAL, "%s", what); }

using clk = std::chrono::steady_clock;

double ms_since(clk::time_point t0, clk::time_point t1) {
    return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

// Device bytes of a handle per vertex (row offsets, states, bitmaps, maps,
// sweep and fallback work arrays, two snapshot halves) and per slot, and of a
// group per update of its tick capacity (staging and same-edge tables).
constexpr uint64_t kBytesPerVertex = 176;
constexpr uint64_t kBytesPerSlot = 4;
constexpr uint64_t kBytesPerTickUpdate = 64;
// Vertices of at least this degree in a newly admitted group are colored one
// at a time (descending degree) before its first repair (sgc_color_core).
constexpr uint32_t kCoreMinDegree = 256;

struct Request {
    uint64_t id;
    clk::time_point arrival;
    uint32_t n;  // updates
};

struct Tenant {
    int state = SGC_TENANT_QUEUED;
    uint32_t n = 0;
    uint32_t epoch = 0, threshold = 0;
    std::vector<uint64_t> rp;  // the CSR until the tenant is resident
    std::vector<uint32_t> col, deg;
    uint64_t footprint = 0;
    int group = -1;
    uint32_t local = 0;
    std::vector<EdgeUpdate> held;    // submitted, not yet forwarded to the group
    std::deque<Request> held_reqs;
    std::deque<Request> waiting;     // forwarded to the group, not yet visible
    uint64_t seen_publishes = 0;
    bool admitting = false;          // its group is being created (its CSR is in use)
    bool remove_pending = false;     // removed while admitting: ends once admission is done
    bool regrow_wanted = false;      // its rows dropped an entry (options.regrow): re-admit at the next step
    bool regrowing = false;          // its rows are being rebuilt: requests wait, queries read its old group
    bool requeued = false;           // ... and it waits in the queue (its old group counts it until it is resident again)
    // options.regrow: edges whose last forwarded update since the tenant's
    // last admission was an insert, as (min << 32 | max). An insert whose two
    // directions were both dropped on full rows is in no row; re-admission
    // merges these edges back into the rows it reads.
    std::unordered_set<uint64_t> inserted;
};

struct Group {
    sgc_batch* b = nullptr;
    std::vector<uint32_t> tenants;   // by local index
    uint64_t bytes = 0;
    uint32_t alive = 0;
    bool has_work = false;
    bool retired = false;            // all tenants removed: freed at the next step
    sgc_stats last{};                // the batch's counters after its last tick
    bool last_ok = true;
};

// The most recent latency samples of one kind (a bounded ring): a long-running
// server reports percentiles over its last kMax requests.
struct LatencyWindow {
    static constexpr size_t kMax = size_t(1) << 20;
    std::vector<double> v;
    size_t next = 0;
    uint64_t total = 0;
    void add(double ms) {
        if (v.size() < kMax) {
            v.push_back(ms);
        } else {
            v[next] = ms;
            next = (next + 1) % kMax;
        }
        total++;
    }
};

double pct(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    const size_t i = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5));
    std::nth_element(v.begin(), v.begin() + (ptrdiff_t)i, v.end());
    return v[i];
}

}  // namespace

struct sgc_server {
    sgc_server_options opt{};
    std::shared_mutex life;  // queries read a group under it; freeing a group excludes them
    std::mutex mu;
    std::vector<Tenant> tenants;
    std::vector<Group> groups;
    std::deque<uint32_t> queue;      // tenants waiting for admission, in arrival order
    uint64_t resident_bytes = 0;
    uint64_t next_request = 1;
    // Request states from the oldest one not yet resolved (0 pending, 1 visible,
    // 2 dropped with its tenant); older ids are visible unless in `dropped`.
    std::deque<uint8_t> req_state;
    uint64_t req_base = 1;
    // Ids of the most recent kMaxDropped requests dropped with their tenants
    // (in the order they were dropped); an id at or below `forgotten` that is
    // not among them may have been dropped earlier and is reported unknown.
    static constexpr size_t kMaxDropped = size_t(1) << 20;
    std::unordered_set<uint64_t> dropped;
    std::deque<uint64_t> dropped_order;
    uint64_t forgotten = 0;
    uint64_t dropped_total = 0;
    LatencyWindow vis_ms, query_ms;
    uint64_t update_requests = 0, updates_applied = 0, queries = 0, query_vertices = 0;
    uint64_t ticks = 0, tier1_sweeps = 0, tier2_ticks = 0, tier2_mirror_ticks = 0, regrown = 0;
    double tick_device_ms = 0;
};

// Drops the resolved requests at the front of the state window (under mu).
void trim_requests(sgc_server* s) {
    while (!s->req_state.empty() && s->req_state.front() != 0) {
        s->req_state.pop_front();
        s->req_base++;
    }
}

// A tenant leaves for good (under mu): its held and forwarded requests will
// never be visible. They are resolved as dropped, so the state window can
// move past them, and the tenant's host buffers are released.
void end_tenant(sgc_server* s, Tenant& t) {
    t.state = SGC_TENANT_REMOVED;
    t.regrowing = t.requeued = false;
    for (const auto* reqs : {&t.held_reqs, &t.waiting})
        for (const Request& q : *reqs) {
            s->req_state[q.id - s->req_base] = 2;
            if (s->dropped.insert(q.id).second) {
                s->dropped_order.push_back(q.id);
                s->dropped_total++;
            }
        }
    while (s->dropped_order.size() > sgc_server::kMaxDropped) {
        const uint64_t id = s->dropped_order.front();
        s->dropped_order.pop_front();
        s->dropped.erase(id);
        if (id > s->forgotten) s->forgotten = id;
    }
    trim_requests(s);
    std::vector<uint64_t>().swap(t.rp);
    std::vector<uint32_t>().swap(t.col);
    std::vector<uint32_t>().swap(t.deg);
    std::vector<EdgeUpdate>().swap(t.held);
    t.held_reqs.clear();
    t.waiting.clear();
    std::unordered_set<uint64_t>().swap(t.inserted);
}

namespace {

}  // namespace

extern "C" {

uint64_t sgc_tenant_footprint(uint32_t num_vertices, uint64_t num_entries, uint32_t slack_pct) {
    // rows get max(d + d*slack/100, 8) slots: at least 8 per vertex
    const uint64_t slots = std::max<uint64_t>(num_entries + num_entries * slack_pct / 100, 8ull * num_vertices);
    const uint64_t nv = ((uint64_t)num_vertices + 31) & ~31ull;
    return slots * kBytesPerSlot + nv * kBytesPerVertex + (slots / 256) * 8;
}

int sgc_server_default_options(sgc_server_options* o) {
    if (!o) return SGC_EINVAL;
    std::memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(sgc_server_options);
    o->flags = SGC_BATCH_CUDA_GRAPH;
    o->hbm_budget_bytes = 150ull << 30;
    o->max_tick_updates = 1u << 20;
    o->slack_pct = SGC_CSR_EXTRA_SLACK_PCT_DEFAULT;
    return SGC_OK;
}

int sgc_server_create(const sgc_server_options* opt, sgc_server** out) {
    if (!out) return bad("null argument");
    if (opt && opt->struct_size != sizeof(sgc_server_options)) return bad("sgc_server_options.struct_size mismatch");
    sgc_server* s = new sgc_server();
    sgc_server_default_options(&s->opt);
    if (opt) s->opt = *opt;
    *out = s;
    return SGC_OK;
}

int sgc_server_destroy(sgc_server* s) {
    if (!s) return SGC_OK;
    for (auto& g : s->groups)
        if (g.b) sgc_batch_destroy(g.b);
    delete s;
    return SGC_OK;
}

int sgc_server_add_tenant(sgc_server* s, const sgc_batch_graph* g, uint32_t* tenant) {
    if (!s || !g || !tenant || !g->row_ptr || !g->num_vertices) return bad("null argument or empty graph");
    const uint64_t m = g->row_ptr[g->num_vertices];
    if (m && !g->col_idx) return bad("col_idx is null");
    Tenant t;
    t.n = g->num_vertices;
    t.epoch = g->epoch_size;
    t.threshold = g->histogram_threshold;
    t.rp.assign(g->row_ptr, g->row_ptr + (size_t)g->num_vertices + 1);
    if (m) t.col.assign(g->col_idx, g->col_idx + m);
    if (g->degree) t.deg.assign(g->degree, g->degree + g->num_vertices);
    std::lock_guard<std::mutex> lk(s->mu);
    t.footprint = sgc_tenant_footprint(t.n, m, s->opt.slack_pct);
    *tenant = (uint32_t)s->tenants.size();
    s->tenants.push_back(std::move(t));
    s->queue.push_back(*tenant);
    return SGC_OK;
}

int sgc_server_tenant_state(sgc_server* s, uint32_t tenant) {
    if (!s) return SGC_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    if (tenant >= s->tenants.size()) return bad("tenant out of range");
    return s->tenants[tenant].state;
}

int sgc_server_remove_tenant(sgc_server* s, uint32_t tenant) {
    if (!s) return SGC_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    if (tenant >= s->tenants.size()) return bad("tenant out of range");
    Tenant& t = s->tenants[tenant];
    if (t.state == SGC_TENANT_REMOVED) return SGC_OK;
    if (t.admitting) {  // the step creating its group ends it afterwards
        t.remove_pending = true;
        return SGC_OK;
    }
    if (t.state == SGC_TENANT_QUEUED || t.requeued)
        s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), tenant), s->queue.end());
    if (t.state == SGC_TENANT_RESIDENT) {  // a requeued tenant still counts in its old group
        Group& g = s->groups[t.group];
        if (--g.alive == 0) g.retired = true;  // its memory goes back to the budget at the next step
    }
    end_tenant(s, t);
    return SGC_OK;
}

int sgc_server_submit(sgc_server* s, uint32_t tenant, const EdgeUpdate* ups, uint32_t n, uint64_t* request) {
    if (!s || (n && !ups)) return bad("null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    if (tenant >= s->tenants.size()) return bad("tenant out of range");
    Tenant& t = s->tenants[tenant];
    if (t.state == SGC_TENANT_REMOVED) return bad("tenant was removed");
    if (n > s->opt.max_tick_updates) return bad("request larger than max_tick_updates");
    Request r{s->next_request++, clk::now(), n};
    s->req_state.push_back(0);
    s->update_requests++;
    // held on the host until the next step forwards it (a step may be running)
    t.held.insert(t.held.end(), ups, ups + n);
    t.held_reqs.push_back(r);
    if (request) *request = r.id;
    return SGC_OK;
}

int sgc_server_query(sgc_server* s, uint32_t tenant, const uint32_t* v, uint16_t* out, uint32_t k) {
    if (!s || (k && (!v || !out))) return bad("null argument");
    const auto t0 = clk::now();
    sgc_batch* b = nullptr;
    uint32_t local = 0;
    std::shared_lock<std::shared_mutex> sl(s->life);  // the group stays alive until the answer is back
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (tenant >= s->tenants.size()) return bad("tenant out of range");
        Tenant& t = s->tenants[tenant];
        if (t.state == SGC_TENANT_RESIDENT && s->groups[t.group].b) {
            b = s->groups[t.group].b;
            local = t.local;
        }
    }
    int rc = SGC_OK;
    if (b) rc = sgc_batch_query(b, local, v, out, k);
    else std::memset(out, 0, (size_t)k * 2);  // nothing published yet
    sl.unlock();
    const double ms = ms_since(t0, clk::now());
    std::lock_guard<std::mutex> lk(s->mu);
    s->queries++;
    s->query_vertices += k;
    s->query_ms.add(ms);
    return rc;
}

namespace {

// Tenants whose rows dropped entries (options.regrow): their live rows are
// read back, every entry's mirror restored (an edge is kept when either
// direction survived), and the tenant is queued again at the front with rows
// sized from its new degrees. Until its new group is resident, queries read
// its old group (which keeps counting it) and its requests wait; the updates
// already forwarded are in the rows read, so they become visible at the new
// group's first publish.
int regrow_tenants(sgc_server* s) {
    struct Job {
        uint32_t tid;
        sgc_batch* b;
        uint32_t local, n;
    };
    std::vector<Job> jobs;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (uint32_t tid = 0; tid < (uint32_t)s->tenants.size(); tid++) {
            Tenant& t = s->tenants[tid];
            if (!t.regrow_wanted) continue;
            t.regrow_wanted = false;
            if (t.state != SGC_TENANT_RESIDENT || t.regrowing || t.admitting || !s->groups[t.group].b) continue;
            t.regrowing = true;  // from here its requests are held
            jobs.push_back({tid, s->groups[t.group].b, t.local, t.n});
        }
    }
    for (const Job& j : jobs) {
        // the live rows (the groups' ticks are done: the step is single-threaded)
        std::vector<uint64_t> rp((size_t)j.n + 1);
        int rc = sgc_batch_rows(j.b, j.local, rp.data(), nullptr, 0);
        std::vector<uint32_t> col(std::max<uint64_t>(rp[j.n], 1));
        if (rc == SGC_OK) rc = sgc_batch_rows(j.b, j.local, rp.data(), col.data(), col.size());
        // inserts that are in no row (both directions dropped): appended to
        // their lower endpoint's row before the mirrors are restored
        if (rc == SGC_OK) {
            std::vector<uint64_t> extra;
            {
                std::lock_guard<std::mutex> lk(s->mu);
                const Tenant& t = s->tenants[j.tid];
                extra.assign(t.inserted.begin(), t.inserted.end());
            }
            if (!extra.empty()) {
                std::sort(extra.begin(), extra.end());
                std::vector<uint64_t> add((size_t)j.n + 1, 0);
                for (uint64_t e : extra) add[(e >> 32) + 1]++;
                for (uint32_t x = 0; x < j.n; x++) add[x + 1] += add[x];
                std::vector<uint64_t> rp2((size_t)j.n + 1, 0);
                std::vector<uint32_t> col2(std::max<uint64_t>(rp[j.n] + extra.size(), 1));
                size_t k = 0;
                for (uint32_t x = 0; x < j.n; x++) {
                    uint64_t w = rp[x] + add[x];
                    rp2[x] = w;
                    for (uint64_t i = rp[x]; i < rp[x + 1]; i++) col2[w++] = col[i];
                    for (; k < extra.size() && (extra[k] >> 32) == x; k++) col2[w++] = (uint32_t)extra[k];
                }
                rp2[j.n] = rp[j.n] + extra.size();
                rp.swap(rp2);
                col.swap(col2);
            }
        }
        // undirected edges from either direction, then both directions, rows ascending
        std::vector<uint64_t> nrp;
        std::vector<uint32_t> ncol, ndeg;
        if (rc == SGC_OK) {
            sgc_csr sym{};
            if (sgc_csr_symmetrize(j.n, rp.data(), col.data(), &sym) != 0) {
                rc = SGC_ENOMEM;
            } else {
                nrp.assign(sym.row_ptr, sym.row_ptr + (size_t)j.n + 1);
                ncol.assign(sym.col_idx, sym.col_idx + sym.nnz);
                ndeg.assign(sym.degree, sym.degree + j.n);
            }
            sgc_csr_free(&sym);
        }
        std::lock_guard<std::mutex> lk(s->mu);
        Tenant& t = s->tenants[j.tid];
        if (t.state != SGC_TENANT_RESIDENT || rc != SGC_OK) {  // removed meanwhile (it left its group then)
            t.regrowing = false;
            if (rc != SGC_OK) return rc;
            continue;
        }
        t.rp.swap(nrp);
        t.col.swap(ncol);
        t.deg.swap(ndeg);
        t.footprint = sgc_tenant_footprint(t.n, t.rp[t.n], s->opt.slack_pct);
        t.requeued = true;
        s->queue.push_front(j.tid);
        s->regrown++;
    }
    return SGC_OK;
}

// One tenant's requests moved out of its held buffer by a step.
struct Forward {
    sgc_batch* b;
    uint32_t local;
    std::vector<EdgeUpdate> ups;
};

}  // namespace

// The table lock (`mu`) is held only for bookkeeping: creating a group,
// copying updates into the groups' staging and the ticks themselves run
// without it. Batches are touched by the stepping thread only (and, for
// snapshot reads, by queries under `life`).
int sgc_server_step(sgc_server* s, sgc_server_step_report* rep) {
    if (!s) return SGC_EINVAL;
    const auto t0 = clk::now();
    {  // 0. groups whose tenants all left: free them (lock order: life, then mu)
        std::unique_lock<std::shared_mutex> xl(s->life);
        std::lock_guard<std::mutex> lk0(s->mu);
        for (auto& g : s->groups) {
            if (!g.retired || !g.b) continue;
            sgc_batch_destroy(g.b);
            g.b = nullptr;
            s->resident_bytes -= g.bytes;
        }
    }
    sgc_server_step_report r{};
    r.proper = 1;
    if (s->opt.regrow) {
        const int rc = regrow_tenants(s);
        if (rc != SGC_OK) return rc;
    }
    // 1. admission: first come first served against the budget
    std::vector<uint32_t> admit;
    uint64_t add_bytes = (uint64_t)s->opt.max_tick_updates * kBytesPerTickUpdate;
    std::vector<sgc_batch_graph> gs;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        while (!s->queue.empty()) {
            Tenant& t = s->tenants[s->queue.front()];
            if (s->resident_bytes + add_bytes + t.footprint > s->opt.hbm_budget_bytes) break;
            add_bytes += t.footprint;
            t.admitting = true;
            admit.push_back(s->queue.front());
            s->queue.pop_front();
        }
        for (uint32_t tid : admit) {
            Tenant& t = s->tenants[tid];
            gs.push_back(sgc_batch_graph{t.n, t.epoch, t.threshold, 0, t.rp.data(),
                                         t.col.empty() ? nullptr : t.col.data(), t.deg.empty() ? nullptr : t.deg.data()});
        }
        if (!admit.empty()) s->resident_bytes += add_bytes;  // reserved while the group is built
    }
    if (!admit.empty()) {
        sgc_batch_options bo;
        sgc_batch_default_options(&bo);
        bo.slack_pct = s->opt.slack_pct;
        bo.max_tick_updates = s->opt.max_tick_updates;
        bo.device = s->opt.device;
        bo.flags = s->opt.flags;
        Group g;
        int rc = sgc_batch_create(gs.data(), (uint32_t)gs.size(), &bo, &g.b);
        // the first tick colors the new tenants' graphs and publishes them; their
        // dense cores (degree >= kCoreMinDegree) are colored one vertex at a time
        // first (outside the table lock)
        if (rc == SGC_OK && (rc = sgc_batch_color_core(g.b, kCoreMinDegree, nullptr)) != SGC_OK) {
            sgc_batch_destroy(g.b);
            g.b = nullptr;
        }
        std::lock_guard<std::mutex> lk(s->mu);
        if (rc != SGC_OK) {  // back to the head of the queue
            s->resident_bytes -= add_bytes;
            for (auto it = admit.rbegin(); it != admit.rend(); ++it) {
                Tenant& t = s->tenants[*it];
                t.admitting = false;
                if (t.remove_pending) {
                    if (t.requeued) {  // it still counted in its old group
                        Group& og = s->groups[t.group];
                        if (--og.alive == 0) og.retired = true;
                    }
                    end_tenant(s, t);
                    continue;
                }
                s->queue.push_front(*it);
            }
            return rc;
        }
        sgc_batch_close_epochs(g.b);
        g.tenants = admit;
        g.bytes = add_bytes;
        g.has_work = true;
        const int gi = (int)s->groups.size();
        for (size_t i = 0; i < admit.size(); i++) {
            Tenant& t = s->tenants[admit[i]];
            t.admitting = false;
            if (t.requeued) {  // re-admitted with rebuilt rows: it leaves its old group now
                Group& og = s->groups[t.group];
                if (--og.alive == 0) og.retired = true;
            }
            t.regrowing = t.requeued = false;
            t.group = gi;
            t.local = (uint32_t)i;
            t.seen_publishes = 0;  // the new group's publish count starts at 0
            std::vector<uint64_t>().swap(t.rp);  // the CSR lives on the device now
            std::vector<uint32_t>().swap(t.col);
            std::vector<uint32_t>().swap(t.deg);
            std::unordered_set<uint64_t>().swap(t.inserted);  // the rows just admitted hold them
            if (t.remove_pending) {
                end_tenant(s, t);
            } else {
                t.state = SGC_TENANT_RESIDENT;
                g.alive++;
            }
        }
        if (g.alive == 0) g.retired = true;
        s->groups.push_back(g);
        r.admitted = (uint32_t)admit.size();
    }
    // 2. requests submitted since the last step: whole and in order, as far as
    //    each group's tick capacity allows (the rest waits for the next step)
    std::vector<Forward> fw;
    std::vector<sgc_batch*> closes_b;
    std::vector<uint32_t> closes_l;
    std::vector<int> ticking;
    std::vector<sgc_batch*> tb;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        std::vector<uint64_t> room(s->groups.size());
        for (size_t gi = 0; gi < s->groups.size(); gi++)
            if (s->groups[gi].b) room[gi] = s->opt.max_tick_updates - sgc_batch_pending(s->groups[gi].b);
        const auto now = clk::now();
        for (auto& t : s->tenants) {
            if (t.state != SGC_TENANT_RESIDENT || t.regrowing) continue;  // a regrowing tenant's requests wait
            Group& g = s->groups[t.group];
            if (!t.held_reqs.empty()) {
                uint64_t take = 0;
                size_t k = 0;
                while (k < t.held_reqs.size() && take + t.held_reqs[k].n <= room[t.group]) take += t.held_reqs[k++].n;
                if (k) {
                    Forward f{g.b, t.local, {}};
                    if (take == t.held.size()) {
                        f.ups.swap(t.held);
                    } else {
                        f.ups.assign(t.held.begin(), t.held.begin() + (ptrdiff_t)take);
                        t.held.erase(t.held.begin(), t.held.begin() + (ptrdiff_t)take);
                    }
                    room[t.group] -= take;
                    s->updates_applied += take;
                    if (s->opt.regrow)
                        for (const EdgeUpdate& e : f.ups) {
                            if (e.u == e.v || e.u >= t.n || e.v >= t.n) continue;  // skipped on the device too
                            const uint64_t key = e.u < e.v ? ((uint64_t)e.u << 32) | e.v : ((uint64_t)e.v << 32) | e.u;
                            if (e.type == SGC_UPDATE_ADD) t.inserted.insert(key);
                            else t.inserted.erase(key);
                        }
                    for (size_t i = 0; i < k; i++) t.waiting.push_back(t.held_reqs[i]);
                    t.held_reqs.erase(t.held_reqs.begin(), t.held_reqs.begin() + (ptrdiff_t)k);
                    g.has_work = true;
                    if (!f.ups.empty()) fw.push_back(std::move(f));
                }
            }
            // 3. staleness deadline
            if (s->opt.max_staleness_us && !t.waiting.empty() &&
                1e3 * ms_since(t.waiting.front().arrival, now) >= (double)s->opt.max_staleness_us) {
                closes_b.push_back(g.b);
                closes_l.push_back(t.local);
                g.has_work = true;
            }
        }
        for (size_t gi = 0; gi < s->groups.size(); gi++) {
            Group& g = s->groups[gi];
            if (!g.b || !g.has_work) continue;
            ticking.push_back((int)gi);
            tb.push_back(g.b);
            g.has_work = false;
        }
    }
    // 4. staging copies and ticks without the lock: launch all, then wait for all
    for (auto& f : fw) {
        const int rc = sgc_batch_submit(f.b, f.local, f.ups.data(), (uint32_t)f.ups.size());
        if (rc != SGC_OK) return rc;
    }
    for (size_t i = 0; i < closes_b.size(); i++) sgc_batch_close_epoch(closes_b[i], closes_l[i]);
    for (sgc_batch* b : tb) {
        const int rc = sgc_batch_tick_begin(b);
        if (rc != SGC_OK) return rc;
    }
    std::vector<sgc_batch_tick_report> trs(tb.size());
    int end_rc = SGC_OK;
    for (size_t i = 0; i < tb.size(); i++) {
        const int rc = sgc_batch_tick_end(tb[i], &trs[i]);
        if (rc != SGC_OK && end_rc == SGC_OK) end_rc = rc;
    }
    if (end_rc != SGC_OK) return end_rc;
    // counters of the ticked groups while their streams are idle (the stats
    // call reads them without waiting on a running tick)
    std::vector<sgc_stats> bst(tb.size());
    std::vector<int> brc(tb.size());
    std::vector<std::vector<uint8_t>> dropped(tb.size());
    for (size_t i = 0; i < tb.size(); i++) {
        brc[i] = sgc_batch_stats(tb[i], &bst[i]);
        if (s->opt.regrow && bst[i].drain_failed + bst[i].overflow_lost > 0) {  // which graphs dropped entries
            dropped[i].resize(sgc_batch_num_graphs(tb[i]));
            if (sgc_batch_dropped(tb[i], dropped[i].data()) != SGC_OK) dropped[i].clear();
        }
    }
    std::lock_guard<std::mutex> lk(s->mu);
    const auto now = clk::now();
    for (size_t i = 0; i < ticking.size(); i++) {
        Group& g = s->groups[ticking[i]];
        g.last = bst[i];
        g.last_ok = brc[i] == SGC_OK;
        const sgc_batch_tick_report& tr = trs[i];
        r.groups_ticked++;
        r.updates += tr.updates;
        r.published += tr.published;
        s->ticks++;
        s->tier1_sweeps += tr.tier1_iterations;
        s->tier2_ticks += tr.tier2_ran;
        s->tier2_mirror_ticks += (tr.tier2_reason & 1u) ? 1 : 0;
        s->tick_device_ms += tr.device_ms;
        if (!tr.proper) r.proper = 0;
        for (uint32_t tid : g.tenants) {
            Tenant& t = s->tenants[tid];
            if (t.state != SGC_TENANT_RESIDENT || t.group != ticking[i]) continue;  // moved tenants left this group
            if (!dropped[i].empty() && dropped[i][t.local] && !t.regrowing) t.regrow_wanted = true;
            const uint64_t p = sgc_batch_publish_count(g.b, t.local);
            if (p != t.seen_publishes) {  // everything forwarded so far is in this snapshot
                t.seen_publishes = p;
                for (auto& q : t.waiting) {
                    s->req_state[q.id - s->req_base] = 1;
                    s->vis_ms.add(ms_since(q.arrival, now));
                    r.requests_visible++;
                }
                t.waiting.clear();
            }
            // a deadline still to come, or requests held back by the capacity, need another tick
            if ((!t.waiting.empty() && s->opt.max_staleness_us) || !t.held_reqs.empty()) g.has_work = true;
        }
    }
    trim_requests(s);
    r.step_ms = ms_since(t0, clk::now());
    if (rep) *rep = r;
    return SGC_OK;
}

int sgc_server_request_visible(sgc_server* s, uint64_t request) {
    if (!s) return SGC_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    if (request == 0 || request >= s->next_request) return 0;
    if (request < s->req_base) {
        if (s->dropped.count(request)) return 0;
        if (request <= s->forgotten)
            return sgci::fail(SGC_EINVAL, "request %llu is older than the dropped requests the server remembers",
                              (unsigned long long)request);
        return 1;
    }
    return s->req_state[request - s->req_base] == 1 ? 1 : 0;
}

int sgc_server_snapshot(sgc_server* s, uint32_t tenant, uint16_t* out) {
    if (!s || !out) return SGC_EINVAL;
    sgc_batch* b = nullptr;
    uint32_t local = 0, n = 0;
    std::shared_lock<std::shared_mutex> sl(s->life);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (tenant >= s->tenants.size()) return bad("tenant out of range");
        Tenant& t = s->tenants[tenant];
        n = t.n;
        if (t.state == SGC_TENANT_RESIDENT && s->groups[t.group].b) {
            b = s->groups[t.group].b;
            local = t.local;
        }
    }
    if (!b) {
        std::memset(out, 0, (size_t)n * 2);
        return SGC_OK;
    }
    return sgc_batch_snapshot(b, local, out);
}

int sgc_server_rows(sgc_server* s, uint32_t tenant, uint64_t* row_ptr, uint32_t* col, uint64_t col_cap) {
    if (!s || !row_ptr) return bad("null argument");
    std::lock_guard<std::mutex> lk(s->mu);  // excludes steps' bookkeeping; the rows are read between ticks
    if (tenant >= s->tenants.size()) return bad("tenant out of range");
    Tenant& t = s->tenants[tenant];
    if (t.state != SGC_TENANT_RESIDENT || !s->groups[t.group].b) return bad("tenant is not resident");
    return sgc_batch_rows(s->groups[t.group].b, t.local, row_ptr, col, col_cap);
}

int sgc_server_get_stats(sgc_server* s, sgc_server_stats* o) {
    if (!s || !o) return SGC_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(o, 0, sizeof(*o));
    for (auto& t : s->tenants) {
        if (t.state == SGC_TENANT_RESIDENT) o->tenants_resident++;
        if (t.state == SGC_TENANT_QUEUED) o->tenants_queued++;
    }
    for (auto& g : s->groups) {
        if (!g.b) continue;
        o->groups++;
        o->overflows += g.last.overflow_pending + g.last.overflow_lost;
        o->drain_failed += g.last.drain_failed;
        if (!g.last_ok || g.last.device_error) o->device_errors++;
    }
    o->resident_bytes = s->resident_bytes;
    o->budget_bytes = s->opt.hbm_budget_bytes;
    o->update_requests = s->update_requests;
    o->updates_applied = s->updates_applied;
    o->requests_visible = s->vis_ms.total;
    o->queries = s->queries;
    o->query_vertices = s->query_vertices;
    o->visible_p50_ms = pct(s->vis_ms.v, 0.50);
    o->visible_p99_ms = pct(s->vis_ms.v, 0.99);
    o->query_p50_ms = pct(s->query_ms.v, 0.50);
    o->query_p99_ms = pct(s->query_ms.v, 0.99);
    o->ticks = s->ticks;
    o->tier1_sweeps = s->tier1_sweeps;
    o->tier2_ticks = s->tier2_ticks;
    o->tier2_mirror_ticks = s->tier2_mirror_ticks;
    o->tick_device_ms = s->tick_device_ms;
    o->tenants_regrown = s->regrown;
    o->requests_tracked = s->req_state.size();
    o->requests_dropped = s->dropped_total;
    return SGC_OK;
}

}  // extern "C"
