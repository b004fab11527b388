// sgc_host.cpp -- host helpers: graph input, update streams, output files.
#include "sgc_host.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <unordered_set>
#include <utility>
#include <vector>

#include <omp.h>
#include <parallel/algorithm>

namespace {

constexpr uint32_t INV = SGC_CSR_INVALID;

inline uint64_t key_of(uint32_t a, uint32_t b) { return ((uint64_t)a << 32) | b; }

// Open-addressing set of u64 edge keys (a << 32 | b, a < b, so ~0 and ~0-1 are
// never keys: they mark empty and deleted slots). Membership only.
struct KeySet {
    static constexpr uint64_t EMPTY = ~0ull, DEAD = ~0ull - 1;
    std::vector<uint64_t> t;
    uint64_t mask = 0, used = 0;
    explicit KeySet(uint64_t expect = 1024) {
        uint64_t cap = 1024;
        while (cap < 2 * expect + 16) cap <<= 1;
        t.assign(cap, EMPTY);
        mask = cap - 1;
    }
    static uint64_t mix(uint64_t k) {
        k ^= k >> 33; k *= 0xff51afd7ed558ccdull; k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ull; return k ^ (k >> 33);
    }
    bool has(uint64_t k) const {
        for (uint64_t i = mix(k) & mask;; i = (i + 1) & mask) {
            if (t[i] == k) return true;
            if (t[i] == EMPTY) return false;
        }
    }
    void grow() {
        std::vector<uint64_t> old;
        old.swap(t);
        t.assign(old.size() * 2, EMPTY);
        mask = t.size() - 1;
        used = 0;
        for (uint64_t k : old)
            if (k != EMPTY && k != DEAD) add(k);
    }
    void add(uint64_t k) {
        if (2 * (used + 1) > t.size()) grow();
        uint64_t dead = EMPTY;
        for (uint64_t i = mix(k) & mask;; i = (i + 1) & mask) {
            if (t[i] == k) return;
            if (t[i] == DEAD && dead == EMPTY) dead = i;
            if (t[i] == EMPTY) {
                if (dead != EMPTY) t[dead] = k;
                else { t[i] = k; used++; }
                return;
            }
        }
    }
    void del(uint64_t k) {
        for (uint64_t i = mix(k) & mask;; i = (i + 1) & mask) {
            if (t[i] == k) { t[i] = DEAD; return; }
            if (t[i] == EMPTY) return;
        }
    }
};

// Whether every row holds strictly ascending neighbor ids.
bool rows_sorted(const sgc_csr* g) {
    bool ok = true;
#pragma omp parallel for reduction(&& : ok) schedule(static)
    for (int64_t u = 0; u < (int64_t)g->n; u++)
        for (uint64_t j = g->row_ptr[u] + 1; j < g->row_ptr[u + 1]; j++)
            if (g->col_idx[j - 1] >= g->col_idx[j]) ok = false;
    return ok;
}

// The live edge set of a churn. With sorted rows: the base graph's edges
// (binary search in the row) plus the changes since (base edges now gone, new
// edges now live), so it grows with the stream, not with the graph; else
// every live edge in one KeySet.
struct LiveEdges {
    const sgc_csr* g;
    bool sorted;
    KeySet full, gone, extra;
    LiveEdges(const sgc_csr* g_, uint64_t stream)
        : g(g_), sorted(rows_sorted(g_)), full(sorted ? 1 : g_->nnz / 2 + stream), gone(sorted ? stream : 1),
          extra(sorted ? stream : 1) {
        if (!sorted)
            for (uint32_t u = 0; u < g->n; u++)
                for (uint64_t j = g->row_ptr[u]; j < g->row_ptr[u + 1]; j++)
                    if (u < g->col_idx[j]) full.add(key_of(u, g->col_idx[j]));
    }
    bool in_base(uint64_t e) const {
        const uint32_t a = (uint32_t)(e >> 32), b = (uint32_t)e;
        const uint32_t* lo = g->col_idx + g->row_ptr[a];
        const uint32_t* hi = g->col_idx + g->row_ptr[a + 1];
        return std::binary_search(lo, hi, b);
    }
    bool has(uint64_t e) const {
        if (!sorted) return full.has(e);
        return in_base(e) ? !gone.has(e) : extra.has(e);
    }
    void add(uint64_t e) {
        if (!sorted) full.add(e);
        else if (in_base(e)) gone.del(e);
        else extra.add(e);
    }
    void del(uint64_t e) {
        if (!sorted) full.del(e);
        else if (in_base(e)) gone.add(e);
        else extra.del(e);
    }
};

// Symmetric CSR from normalised (min, max) keys, sorted and unique.
int csr_from_sorted_keys(uint32_t n, const std::vector<uint64_t>& keys, sgc_csr* out) {
    std::memset(out, 0, sizeof(*out));
    out->n = n;
    out->nnz = keys.size() * 2;
    out->row_ptr = (uint64_t*)calloc((size_t)n + 1, 8);
    out->degree = (uint32_t*)calloc(n ? n : 1, 4);
    out->col_idx = (uint32_t*)malloc(std::max<size_t>(out->nnz, 1) * 4);
    if (!out->row_ptr || !out->degree || !out->col_idx) return -3;
    for (uint64_t k : keys) {
        out->degree[k >> 32]++;
        out->degree[(uint32_t)k]++;
    }
    for (uint32_t v = 0; v < n; v++) out->row_ptr[v + 1] = out->row_ptr[v] + out->degree[v];
    std::vector<uint64_t> fill(out->row_ptr, out->row_ptr + n);
    // Keys ascend by (a, b), so row x first receives every a < x (keys (a, x),
    // in ascending a) and then every b > x (keys (x, b), ascending b): each
    // row comes out sorted without a per-row sort.
    for (uint64_t k : keys) {
        const uint32_t a = (uint32_t)(k >> 32), b = (uint32_t)k;
        out->col_idx[fill[a]++] = b;
        out->col_idx[fill[b]++] = a;
    }
    return 0;
}

int csr_from_pairs(uint32_t n, std::vector<uint64_t>& keys, sgc_csr* out) {
    __gnu_parallel::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    return csr_from_sorted_keys(n, keys, out);
}

}  // namespace

extern "C" {

void sgc_csr_free(sgc_csr* g) {
    if (!g) return;
    free(g->row_ptr);
    free(g->col_idx);
    free(g->degree);
    std::memset(g, 0, sizeof(*g));
}

int sgc_csr_from_edges(uint32_t n, const uint32_t* pairs, uint64_t m, sgc_csr* out) {
    if (!out || (m && !pairs)) return -1;
    std::vector<uint64_t> keys;
    keys.reserve(m);
    for (uint64_t i = 0; i < m; i++) {
        uint32_t u = pairs[2 * i], v = pairs[2 * i + 1];
        if (u >= n || v >= n) return -1;
        if (u == v) continue;
        if (u > v) std::swap(u, v);
        keys.push_back(key_of(u, v));
    }
    return csr_from_pairs(n, keys, out);
}

int sgc_csr_symmetrize(uint32_t n, const uint64_t* row_ptr, const uint32_t* col_idx, sgc_csr* out) {
    if (!out || !row_ptr || (row_ptr[n] && !col_idx)) return -1;
    std::vector<uint64_t> keys;
    keys.reserve(row_ptr[n]);
    for (uint32_t x = 0; x < n; x++)
        for (uint64_t e = row_ptr[x]; e < row_ptr[x + 1]; e++) {
            const uint32_t y = col_idx[e];
            if (y == x || y >= n) continue;
            keys.push_back(x < y ? key_of(x, y) : key_of(y, x));
        }
    return csr_from_pairs(n, keys, out);
}

int sgc_load_mtx(const char* path, sgc_csr* out) {
    if (!path || !out) return -1;
    FILE* f = fopen(path, "r");
    if (!f) return -2;
    char line[4096];
    bool pattern = false;
    if (fgets(line, sizeof(line), f) && strstr(line, "pattern")) pattern = true;
    bool have = false;
    while (fgets(line, sizeof(line), f)) {
        if (line[0] != '%') { have = true; break; }
    }
    unsigned rows = 0, cols = 0;
    unsigned long long nnz = 0;
    if (!have || sscanf(line, "%u %u %llu", &rows, &cols, &nnz) != 3) {
        fclose(f);
        return -4;
    }
    const uint32_t n = rows > cols ? rows : cols;
    std::vector<uint64_t> keys;
    keys.reserve(nnz);
    for (unsigned long long i = 0; i < nnz; i++) {
        unsigned u = 0, v = 0;
        if (fscanf(f, "%u %u", &u, &v) != 2) break;  // truncated file: keep what was read
        if (!pattern) {
            int c;
            while ((c = fgetc(f)) != '\n' && c != EOF) {}
        }
        if (u == 0 || v == 0 || u > n || v > n) {  // outside the declared 1-based range
            fclose(f);
            return -5;
        }
        u--; v--;
        if (u == v) continue;
        if (u > v) std::swap(u, v);
        keys.push_back(key_of(u, v));
    }
    fclose(f);
    return csr_from_pairs(n, keys, out);
}

int sgc_write_mtx(const char* path, const sgc_csr* g) {
    FILE* f = fopen(path, "w");
    if (!f) return -2;
    fprintf(f, "%%%%MatrixMarket matrix coordinate pattern symmetric\n");
    fprintf(f, "%u %u %llu\n", g->n, g->n, (unsigned long long)(g->nnz / 2));
    for (uint32_t u = 0; u < g->n; u++)
        for (uint64_t j = g->row_ptr[u]; j < g->row_ptr[u + 1]; j++)
            if (g->col_idx[j] < u) fprintf(f, "%u %u\n", u + 1, g->col_idx[j] + 1);
    fclose(f);
    return 0;
}

uint64_t sgc_gen_init_stream(const sgc_csr* g, uint32_t* out) {
    // Order of generate_init_stream: by (min degree desc, max degree desc) with
    // std::sort. Each edge carries key = ~min << 32 | ~max, so `key <` gives
    // exactly the reference comparator's answer for every pair and std::sort
    // takes the same path (same output, ties included) without re-reading degrees.
    struct E {
        uint64_t key;
        uint32_t u, v;
    };
    std::vector<E> e;
    e.reserve(g->nnz / 2);
    const uint32_t* d = g->degree;
    for (uint32_t u = 0; u < g->n; u++)
        for (uint64_t j = g->row_ptr[u]; j < g->row_ptr[u + 1]; j++) {
            const uint32_t v = g->col_idx[j];
            if (u < v) {
                const uint32_t lo = std::min(d[u], d[v]), hi = std::max(d[u], d[v]);
                e.push_back({((uint64_t)(~lo) << 32) | (uint32_t)(~hi), u, v});
            }
        }
    std::sort(e.begin(), e.end(), [](const E& p, const E& q) { return p.key < q.key; });
    for (size_t i = 0; i < e.size(); i++) {
        out[2 * i] = e[i].u;
        out[2 * i + 1] = e[i].v;
    }
    return e.size();
}

int sgc_gen_churn_stream(const sgc_csr* g, uint64_t size, uint32_t insert_pct, uint64_t seed, uint32_t* out,
                         uint8_t* types) {
    if (!g || g->n == 0) return -1;
    std::mt19937_64 rng(seed);
    LiveEdges live(g, size);
    std::vector<uint64_t> live_vec;  // (a << 32 | b), a < b, in the order the reference keeps
    live_vec.reserve(g->nnz / 2 + size);
    for (uint32_t u = 0; u < g->n; u++)
        for (uint64_t j = g->row_ptr[u]; j < g->row_ptr[u + 1]; j++)
            if (u < g->col_idx[j]) live_vec.push_back(key_of(u, g->col_idx[j]));
    std::vector<uint64_t> pool;  // deleted edges available for re-insertion
    uint64_t k = 0;
    auto emit = [&](uint64_t e, uint8_t t) {
        out[2 * k] = (uint32_t)(e >> 32);
        out[2 * k + 1] = (uint32_t)e;
        types[k] = t;
        k++;
    };
    while (k < size) {
        const bool insert = std::uniform_int_distribution<uint32_t>(0, 99)(rng) < insert_pct;
        if (insert) {
            if (!pool.empty()) {
                const size_t idx = std::uniform_int_distribution<size_t>(0, pool.size() - 1)(rng);
                const uint64_t e = pool[idx];
                pool[idx] = pool.back();
                pool.pop_back();
                live.add(e);
                live_vec.push_back(e);
                emit(e, SGC_UPDATE_ADD);
            } else {
                std::uniform_int_distribution<uint32_t> vd(0, g->n - 1);
                const uint32_t u = vd(rng);
                uint32_t v = vd(rng);
                if (u == v) v = (v + 1) % g->n;
                const uint64_t e = key_of(std::min(u, v), std::max(u, v));
                if (live.has(e)) continue;  // present: draw again (no event)
                live.add(e);
                live_vec.push_back(e);
                emit(e, SGC_UPDATE_ADD);
            }
        } else {
            if (live_vec.empty()) continue;
            const size_t idx = std::uniform_int_distribution<size_t>(0, live_vec.size() - 1)(rng);
            const uint64_t e = live_vec[idx];
            live.del(e);
            live_vec[idx] = live_vec.back();
            live_vec.pop_back();
            pool.push_back(e);
            emit(e, SGC_UPDATE_DEL);
        }
    }
    return 0;
}

int sgc_core_numbers(const sgc_csr* g, uint32_t* core) {
    const uint32_t n = g->n;
    uint32_t maxd = 0;
    for (uint32_t v = 0; v < n; v++) maxd = std::max(maxd, g->degree[v]);
    std::vector<uint32_t> deg(g->degree, g->degree + n), bin((size_t)maxd + 2, 0), pos(n), vert(n);
    for (uint32_t v = 0; v < n; v++) bin[deg[v]]++;
    uint32_t start = 0;
    for (uint32_t d = 0; d <= maxd; d++) {
        const uint32_t c = bin[d];
        bin[d] = start;
        start += c;
    }
    for (uint32_t v = 0; v < n; v++) {
        pos[v] = bin[deg[v]]++;
        vert[pos[v]] = v;
    }
    for (uint32_t d = maxd; d > 0; d--) bin[d] = bin[d - 1];
    bin[0] = 0;
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t v = vert[i];
        for (uint64_t j = g->row_ptr[v]; j < g->row_ptr[v + 1]; j++) {
            const uint32_t u = g->col_idx[j];
            if (deg[u] > deg[v]) {
                const uint32_t du = deg[u], pu = pos[u], pw = bin[du], w = vert[pw];
                if (u != w) {
                    pos[u] = pw; vert[pu] = w;
                    pos[w] = pu; vert[pw] = u;
                }
                bin[du]++;
                deg[u]--;
            }
        }
    }
    for (uint32_t v = 0; v < n; v++) core[v] = deg[v];
    return 0;
}

int sgc_gen_kcore_stream(const sgc_csr* g, uint64_t size, double pct, uint64_t seed, uint32_t* out, uint8_t* types,
                         uint32_t* core_k, uint32_t* core_size) {
    if (!g || g->n < 2 || pct < 0 || pct > 100) return -1;
    std::vector<uint32_t> core(g->n);
    sgc_core_numbers(g, core.data());
    std::vector<uint32_t> sorted(core);
    std::sort(sorted.begin(), sorted.end());
    size_t idx = (size_t)std::ceil(pct / 100.0 * g->n);
    idx = idx ? idx - 1 : 0;
    if (idx >= g->n) idx = g->n - 1;
    const uint32_t k = sorted[idx];
    std::vector<uint32_t> C;
    std::vector<uint8_t> in(g->n, 0);
    for (uint32_t v = 0; v < g->n; v++)
        if (core[v] >= k) { C.push_back(v); in[v] = 1; }
    if (core_k) *core_k = k;
    if (core_size) *core_size = (uint32_t)C.size();
    if (C.size() < 2) return -2;
    uint64_t core_entries = 0;
    for (uint32_t u : C) core_entries += g->row_ptr[u + 1] - g->row_ptr[u];
    KeySet live(core_entries / 2 + size);
    std::vector<uint64_t> live_vec;
    for (uint32_t u : C)
        for (uint64_t j = g->row_ptr[u]; j < g->row_ptr[u + 1]; j++) {
            const uint32_t v = g->col_idx[j];
            if (u < v && in[v]) {
                live.add(key_of(u, v));
                live_vec.push_back(key_of(u, v));
            }
        }
    const uint64_t csz = C.size();
    if (live_vec.size() + size >= csz * (csz - 1) / 2) return -3;  // core too small to keep inserting
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<uint64_t> pick(0, csz - 1);
    for (uint64_t i = 0; i < size; i++) {
        const bool del = (i % 3 == 2) && !live_vec.empty();
        if (del) {
            const uint64_t j = std::uniform_int_distribution<uint64_t>(0, live_vec.size() - 1)(rng);
            const uint64_t e = live_vec[j];
            live.del(e);
            live_vec[j] = live_vec.back();
            live_vec.pop_back();
            out[2 * i] = (uint32_t)(e >> 32);
            out[2 * i + 1] = (uint32_t)e;
            types[i] = SGC_UPDATE_DEL;
        } else {
            for (;;) {
                const uint32_t a = C[pick(rng)], b = C[pick(rng)];
                if (a == b) continue;
                const uint64_t e = key_of(std::min(a, b), std::max(a, b));
                if (live.has(e)) continue;
                live.add(e);
                live_vec.push_back(e);
                out[2 * i] = (uint32_t)(e >> 32);
                out[2 * i + 1] = (uint32_t)e;
                types[i] = SGC_UPDATE_ADD;
                break;
            }
        }
    }
    return 0;
}

int sgc_gen_rmat(uint32_t scale, uint32_t ef, double a, double b, double c, uint64_t seed, sgc_csr* out) {
    if (scale == 0 || scale > 31 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return -1;
    const uint32_t n = 1u << scale;
    const uint64_t m = (uint64_t)ef * n;
    // Draws come in chunks of 2^20; chunk c uses mt19937_64(seed + c * golden)
    // so the graph does not depend on the thread count.
    const uint64_t CH = 1ull << 20;
    const uint64_t nch = (m + CH - 1) / CH;
    std::vector<std::vector<uint64_t>> parts(nch);
    const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t ci = 0; ci < (int64_t)nch; ci++) {
        std::mt19937_64 rng(seed + (uint64_t)ci * 0x9E3779B97F4A7C15ull);
        const uint64_t lo = (uint64_t)ci * CH, hi = std::min(m, lo + CH);
        auto& out_keys = parts[ci];
        out_keys.reserve(hi - lo);
        for (uint64_t i = lo; i < hi; i++) {
            uint32_t u = 0, v = 0;
            for (uint32_t lvl = 0; lvl < scale; lvl++) {
                const double r = (double)(rng() >> 11) * (1.0 / 9007199254740992.0);
                const uint32_t bit = 1u << (scale - 1 - lvl);
                if (r < a) {
                } else if (r < ab) {
                    v |= bit;
                } else if (r < abc) {
                    u |= bit;
                } else {
                    u |= bit;
                    v |= bit;
                }
            }
            if (u != v) out_keys.push_back(key_of(std::min(u, v), std::max(u, v)));
        }
    }
    std::vector<uint64_t> keys;
    {
        uint64_t tot = 0;
        for (auto& p : parts) tot += p.size();
        keys.reserve(tot);
        for (auto& p : parts) {
            keys.insert(keys.end(), p.begin(), p.end());
            std::vector<uint64_t>().swap(p);
        }
    }
    return csr_from_pairs(n, keys, out);
}

int sgc_gen_chung_lu(uint32_t n, double exponent, double avg, double maxd, uint64_t seed, sgc_csr* out) {
    if (n < 2 || exponent <= 1.0 || avg <= 0) return -1;
    // w_i ~ (i + 1)^(-1/(exponent-1)), scaled to mean `avg`, capped at maxd
    std::vector<double> w(n);
    const double p = 1.0 / (exponent - 1.0);
    double sum = 0;
    for (uint32_t i = 0; i < n; i++) sum += (w[i] = std::pow((double)i + 1.0, -p));
    double scale = avg * n / sum;
    for (int iter = 0; iter < 50; iter++) {  // re-scale after capping
        double s2 = 0;
        for (uint32_t i = 0; i < n; i++) s2 += std::min(w[i] * scale, maxd);
        const double ratio = avg * n / s2;
        scale *= ratio;
        if (std::fabs(ratio - 1.0) < 1e-9) break;
    }
    double acc = 0;
    for (uint32_t i = 0; i < n; i++) acc += (w[i] = std::min(w[i] * scale, maxd));
    const uint64_t m = (uint64_t)std::llround(acc / 2.0);
    // Endpoints drawn with probability w_i / sum w from an alias table (Vose's
    // construction of Walker's alias method): one uniform slot and one coin per
    // draw instead of a binary search.
    std::vector<float> prob(n);
    std::vector<uint32_t> alias(n);
    {
        std::vector<double> q(n);
        std::vector<uint32_t> small, large;
        for (uint32_t i = 0; i < n; i++) {
            q[i] = w[i] * (double)n / acc;
            (q[i] < 1.0 ? small : large).push_back(i);
        }
        while (!small.empty() && !large.empty()) {
            const uint32_t l = small.back(), g = large.back();
            small.pop_back();
            large.pop_back();
            prob[l] = (float)q[l];
            alias[l] = g;
            q[g] = (q[g] + q[l]) - 1.0;
            (q[g] < 1.0 ? small : large).push_back(g);
        }
        for (uint32_t i : large) prob[i] = 1.0f, alias[i] = i;
        for (uint32_t i : small) prob[i] = 1.0f, alias[i] = i;  // rounding leftovers
    }
    std::vector<double>().swap(w);
    // Fixed chunks of draws, each from its own generator seeded by (seed,
    // chunk): the graph does not depend on the number of threads.
    const uint64_t chunk = 1ull << 22;
    const uint64_t nchunks = (m + chunk - 1) / chunk;
    std::vector<std::vector<uint64_t>> parts(nchunks);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t c = 0; c < (int64_t)nchunks; c++) {
        std::mt19937_64 rng(seed ^ (0x9E3779B97F4A7C15ull * (uint64_t)(c + 1)));
        auto draw = [&]() -> uint32_t {
            const uint64_t r = rng();
            const uint32_t i = (uint32_t)(((r >> 32) * (uint64_t)n) >> 32);
            const double coin = (double)(uint32_t)r * (1.0 / 4294967296.0);  // in [0, 1)
            return coin < (double)prob[i] ? i : alias[i];
        };
        const uint64_t lo = (uint64_t)c * chunk, hi = std::min(m, lo + chunk);
        std::vector<uint64_t>& out_c = parts[c];
        out_c.reserve(hi - lo);
        for (uint64_t k = lo; k < hi; k++) {
            const uint32_t u = draw(), v = draw();
            if (u == v) continue;
            out_c.push_back(key_of(std::min(u, v), std::max(u, v)));
        }
    }
    std::vector<uint64_t> keys;
    {
        uint64_t total = 0;
        for (auto& p : parts) total += p.size();
        keys.reserve(total);
        for (auto& p : parts) {
            keys.insert(keys.end(), p.begin(), p.end());
            std::vector<uint64_t>().swap(p);
        }
    }
    return csr_from_pairs(n, keys, out);
}

uint32_t sgc_static_greedy(const sgc_csr* g) {
    std::vector<uint32_t> color(g->n, 0);
    std::vector<uint32_t> mark((size_t)g->n + 2, 0xFFFFFFFFu);
    uint32_t mx = 0;
    for (uint32_t v = 0; v < g->n; v++) {
        for (uint64_t j = g->row_ptr[v]; j < g->row_ptr[v + 1]; j++) {
            const uint32_t c = color[g->col_idx[j]];
            if (c) mark[c] = v;
        }
        uint32_t c = 1;
        while (mark[c] == v) c++;
        color[v] = c;
        mx = std::max(mx, c);
    }
    return mx;
}

int sgc_write_coloring(const char* path, const uint16_t* colors, uint32_t n) {
    FILE* f = fopen(path, "wb");
    if (!f) return -2;
    const size_t w = fwrite(colors, sizeof(uint16_t), n, f);
    fclose(f);
    if (w != n) return -2;
    std::string txt = std::string(path) + ".txt";
    FILE* t = fopen(txt.c_str(), "w");
    if (!t) return -2;
    uint16_t mx = 0;
    for (uint32_t i = 0; i < n; i++) mx = std::max(mx, colors[i]);
    fprintf(t, "# vertices: %u\n# colors: %u\n# algorithm: streamgc\n", n, mx);
    for (uint32_t i = 0; i < n; i++) fprintf(t, "%u %u\n", i, colors[i]);
    fclose(t);
    return 0;
}

}  // extern "C"
