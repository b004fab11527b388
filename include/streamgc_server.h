/*
 * streamgc_server.h -- a request loop serving many tenant graphs from one GPU
 * (libstreamgc_b200.so), on top of the batched engine (streamgc_batch.h).
 *
 *   - Tenants are admitted against an HBM budget computed from their
 *     alpha-slack CSR footprint (sgc_tenant_footprint); a tenant that does not
 *     fit waits, first come first served, until removals free enough memory.
 *     Tenants admitted at the same step become resident together as one group;
 *     the first tick of a group colors its tenants' graphs from scratch.
 *   - Update batches and color queries are accepted at any time, from any
 *     thread (continuous batching): a step applies everything submitted since
 *     the previous step, for every resident group at once -- the groups' ticks
 *     run on their own streams and overlap on the device. Queries answer
 *     immediately from the tenant's last published snapshot, also while a step
 *     runs.
 *   - Epochs close per tenant: after `epoch_size` updates, or once its oldest
 *     unpublished update is `max_staleness_us` old.
 *   - Update-to-visible latency (submit -> the publish that includes it) and
 *     query latency are recorded per request.
 * With SGC_BATCH_STREAM_ORDER a tenant's colors do not depend on the other
 * tenants (for the same submissions and steps).
 * The reference serves one graph per process; this interface has no
 * counterpart there.
 */
#ifndef STREAMGC_SERVER_H
#define STREAMGC_SERVER_H

#include <stdint.h>

#include "streamgc_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sgc_server sgc_server;

typedef struct sgc_server_options {
    uint32_t struct_size;        /* sizeof(sgc_server_options) */
    uint32_t flags;              /* SGC_BATCH_* for every group (SGC_BATCH_CUDA_GRAPH by default) */
    uint64_t hbm_budget_bytes;   /* admission budget over the resident tenants' footprints */
    uint32_t max_tick_updates;   /* per group and step */
    uint32_t max_staleness_us;   /* 0: epochs close by update count only */
    int32_t  device;
    uint32_t slack_pct;          /* 300 = alpha 4 */
    uint32_t regrow;             /* 1: a tenant whose rows dropped an entry (a row still full at the
                                    drain) is re-admitted with rows sized from its current degrees: every
                                    surviving entry's mirror is restored, and every edge whose last
                                    forwarded update since its last admission was an insert is put back
                                    (the server keeps those edges per tenant while this is on);
                                    0 (default): kept as is */
} sgc_server_options;

enum { SGC_TENANT_QUEUED = 0, SGC_TENANT_RESIDENT = 1, SGC_TENANT_REMOVED = 2 };

typedef struct sgc_server_step_report {
    uint32_t admitted;           /* tenants that became resident this step */
    uint32_t groups_ticked;
    uint32_t updates;            /* updates applied */
    uint32_t published;          /* tenant snapshots published */
    uint32_t requests_visible;   /* update requests that became visible */
    uint32_t proper;             /* 1 when every ticked group's coloring is proper */
    double   step_ms;            /* wall time of the step */
} sgc_server_step_report;

typedef struct sgc_server_stats {
    uint64_t tenants_resident, tenants_queued, groups;
    uint64_t resident_bytes, budget_bytes;
    uint64_t update_requests, updates_applied, requests_visible, queries, query_vertices;
    double   visible_p50_ms, visible_p99_ms;  /* update-to-visible, over the last 2^20 requests */
    double   query_p50_ms, query_p99_ms;      /* over the last 2^20 queries */
    uint64_t ticks, tier1_sweeps, tier2_ticks;  /* group ticks, their repair sweeps, ticks that needed Tier-2 */
    uint64_t tier2_mirror_ticks;                /* ... of which because some tenant's rows may miss mirror entries */
    double   tick_device_ms;                    /* device time of the ticks (SGC_BATCH_PROFILE groups), else 0 */
    uint64_t overflows, drain_failed;           /* row overflows (pending + lost) and failed drains, all groups */
    uint64_t device_errors;                     /* groups whose device error word is set */
    uint64_t tenants_regrown;                   /* re-admissions with rebuilt rows (options.regrow) */
    uint64_t requests_tracked;                  /* request states kept: from the oldest unresolved request on */
    uint64_t requests_dropped;                  /* requests dropped with removed tenants, all time */
} sgc_server_stats;

int sgc_server_default_options(sgc_server_options* opt);
int sgc_server_create(const sgc_server_options* opt, sgc_server** out);
int sgc_server_destroy(sgc_server* s);
/* Resident bytes of a tenant: its slack CSR (max(d + d*slack/100, 8) slots per
 * row, 4 bytes each) and its per-vertex state. */
uint64_t sgc_tenant_footprint(uint32_t num_vertices, uint64_t num_entries, uint32_t slack_pct);
/* Queues a tenant (the CSR is copied); it becomes resident at a later step. */
int sgc_server_add_tenant(sgc_server* s, const sgc_batch_graph* g, uint32_t* tenant);
/* Ends a tenant; its group's memory is released at the step after all its tenants ended. */
int sgc_server_remove_tenant(sgc_server* s, uint32_t tenant);
int sgc_server_tenant_state(sgc_server* s, uint32_t tenant);
/* An update request (tenant's ids), at most max_tick_updates updates. Its
 * arrival is stamped now. */
int sgc_server_submit(sgc_server* s, uint32_t tenant, const EdgeUpdate* ups, uint32_t n, uint64_t* request);
/* Colors from the tenant's last published snapshot (0 before its first publish). */
int sgc_server_query(sgc_server* s, uint32_t tenant, const uint32_t* v, uint16_t* out, uint32_t k);
/* One scheduling round: admit, tick every group with work, publish, record
 * latencies. Steps must not overlap each other (one stepping thread). */
int sgc_server_step(sgc_server* s, sgc_server_step_report* rep);
/* 1 once the request's updates are in a published snapshot; 0 while pending
 * or when it was dropped with its removed tenant. The server remembers the
 * ids of the last 2^20 dropped requests: for an older resolved request that
 * may have been among earlier drops the answer is SGC_EINVAL (unknown). */
int sgc_server_request_visible(sgc_server* s, uint64_t request);
int sgc_server_snapshot(sgc_server* s, uint32_t tenant, uint16_t* out);
/* A resident tenant's live rows in its own ids (as sgc_batch_rows); call
 * between steps. */
int sgc_server_rows(sgc_server* s, uint32_t tenant, uint64_t* row_ptr, uint32_t* col, uint64_t col_cap);
int sgc_server_get_stats(sgc_server* s, sgc_server_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* STREAMGC_SERVER_H */
