// Frequent-pattern mining over a graph database (transaction setting: the
// support of a pattern is the number of graphs holding at least one
// embedding), built on the batched matcher.
//
// The reference matches one given pattern per process (src/gpumine.cpp:866);
// it has no pattern generation.  Here patterns grow level by level:
//   level 1   every (vertex label, edge label, vertex label) edge pattern
//   level k+1 each frequent k-edge pattern plus one edge, either between two
//             of its vertices (backward) or to a new vertex (forward), using
//             only frequent edge types; duplicates removed by a canonical
//             code; a candidate is kept only if every connected k-edge
//             sub-pattern is frequent (anti-monotone support)
// and each level's candidates are matched in one gva_batch_count-style run
// (shared step prefixes, per-graph bitmaps) whose supports decide the next
// level.  Each candidate is matched with the planner's own plan for its
// query text, so embedding counts are the reference's row counts.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <array>
#include <atomic>
#include <chrono>
#include <cstring>
#include <functional>
#include <future>
#include <memory>
#include <thread>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <unordered_set>
#include <vector>

#include "../../include/geneva.h"
#include "gva_engine.cuh"
#include "gva_internal.h"

namespace gva {

namespace {

constexpr uint32_t kMaxPatEdges = GVA_MAX_QUERY_VERTICES - 1;  // mining keeps max_edges + 1 <= 32 vertices
constexpr uint32_t kMaxCode = 1 + GVA_MAX_QUERY_VERTICES + GVA_MAX_QUERY_VERTICES * (GVA_MAX_QUERY_VERTICES - 1) / 2;

struct PEdge {
    uint8_t u, v;  // u < v
    uint16_t el;   // edge label (partition id)
    bool operator<(const PEdge& o) const {
        return u != o.u ? u < o.u : (v != o.v ? v < o.v : el < o.el);
    }
};

// A pattern with dense vertex labels (indices into the database's sorted
// label list) and no heap storage.
struct Pattern {
    uint32_t n = 0, ne = 0;
    uint32_t vl[GVA_MAX_QUERY_VERTICES];
    PEdge edges[kMaxPatEdges];
    uint32_t el(uint32_t a, uint32_t b) const {
        for (uint32_t i = 0; i < ne; ++i)
            if ((edges[i].u == a && edges[i].v == b) || (edges[i].u == b && edges[i].v == a)) return edges[i].el;
        return 0;
    }
    void add_edge(uint32_t a, uint32_t b, uint32_t l) {
        edges[ne++] = {(uint8_t)std::min(a, b), (uint8_t)std::max(a, b), (uint16_t)l};
    }
};

// Canonical code of a pattern as bytes: the lexicographically smallest
// (n, vertex labels, upper-triangle edge labels) over vertex orders that sort
// vertices by an isomorphism-invariant key (label, degree, hash of the sorted
// (edge label, neighbour label) list); only orders within equal-key cells are
// tried.  Equal keys of non-equivalent vertices only enlarge a cell, which
// costs time, not correctness.  Values are written `width` bytes each (1 when
// labels and edge labels fit a byte).
struct CodeBuf {
    uint32_t len = 0;  // bytes
    uint8_t b[kMaxCode * 4];
};

uint64_t code_hash(const uint8_t* b, uint32_t len) {
    uint64_t h = 1469598103934665603ull;
    for (uint32_t i = 0; i < len; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h ^ (h >> 29);
}

// Insertion sort: patterns have at most a few dozen vertices, where it beats
// std::sort; ties never occur (the comparators are total), so the order is
// the same.
template <typename T, typename Less>
inline void small_sort(T* a, uint32_t n, Less less) {
    for (uint32_t i = 1; i < n; ++i) {
        const T x = a[i];
        uint32_t j = i;
        while (j > 0 && less(x, a[j - 1])) {
            a[j] = a[j - 1];
            --j;
        }
        a[j] = x;
    }
}

void canonical(const Pattern& p, uint32_t width, CodeBuf& out, uint32_t* order_out = nullptr) {
    const uint32_t n = p.n;
    uint32_t adj[GVA_MAX_QUERY_VERTICES][GVA_MAX_QUERY_VERTICES];
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = 0; j < n; ++j) adj[i][j] = 0;
    for (uint32_t i = 0; i < p.ne; ++i) adj[p.edges[i].u][p.edges[i].v] = adj[p.edges[i].v][p.edges[i].u] = p.edges[i].el;
    uint64_t key[GVA_MAX_QUERY_VERTICES];
    for (uint32_t v = 0; v < n; ++v) {
        uint64_t nb[GVA_MAX_QUERY_VERTICES];
        uint32_t d = 0;
        for (uint32_t u = 0; u < n; ++u)
            if (adj[v][u]) nb[d++] = ((uint64_t)adj[v][u] << 32) | p.vl[u];
        small_sort(nb, d, [](uint64_t a, uint64_t b) { return a < b; });
        uint64_t h = 1469598103934665603ull;
        for (uint32_t i = 0; i < d; ++i) h = (h ^ nb[i]) * 1099511628211ull;
        key[v] = ((uint64_t)(p.vl[v] & 0xffffu) << 48) | ((uint64_t)d << 40) | (h & 0xffffffffffull);
    }
    uint32_t ord[GVA_MAX_QUERY_VERTICES];
    for (uint32_t i = 0; i < n; ++i) ord[i] = i;
    small_sort(ord, n, [&](uint32_t a, uint32_t b) { return key[a] != key[b] ? key[a] < key[b] : a < b; });
    uint32_t cb[GVA_MAX_QUERY_VERTICES], ce[GVA_MAX_QUERY_VERTICES], nc = 0;  // cells [cb, ce)
    bool trivial = true;
    for (uint32_t i = 0; i < n;) {
        uint32_t j = i + 1;
        while (j < n && key[ord[j]] == key[ord[i]]) ++j;
        trivial &= (j == i + 1);
        cb[nc] = i;
        ce[nc++] = j;
        i = j;
    }
    const uint32_t len = 1 + n + n * (n - 1) / 2;
    uint32_t best[kMaxCode], cur[kMaxCode];
    uint32_t best_ord[GVA_MAX_QUERY_VERTICES];
    bool have = false;
    for (;;) {
        // build the code, giving up as soon as it exceeds the best one
        cur[0] = n;
        int cmp = have ? 0 : -1;
        uint32_t k = 1;
        for (uint32_t i = 0; i < n && cmp <= 0; ++i, ++k) {
            cur[k] = p.vl[ord[i]];
            if (cmp == 0 && cur[k] != best[k]) cmp = cur[k] < best[k] ? -1 : 1;
        }
        for (uint32_t i = 0; i < n && cmp <= 0; ++i)
            for (uint32_t j = i + 1; j < n && cmp <= 0; ++j, ++k) {
                cur[k] = adj[ord[i]][ord[j]];
                if (cmp == 0 && cur[k] != best[k]) cmp = cur[k] < best[k] ? -1 : 1;
            }
        if (cmp < 0) {
            std::memcpy(best, cur, sizeof(uint32_t) * len);
            std::memcpy(best_ord, ord, sizeof(uint32_t) * n);
            have = true;
        }
        if (trivial) break;
        int c = (int)nc - 1;
        for (; c >= 0; --c)
            if (std::next_permutation(ord + cb[c], ord + ce[c])) break;
        if (c < 0) break;
    }
    if (order_out) std::memcpy(order_out, best_ord, sizeof(uint32_t) * n);
    out.len = len * width;
    if (width == 1) {
        for (uint32_t i = 0; i < len; ++i) out.b[i] = (uint8_t)best[i];
    } else {
        for (uint32_t i = 0; i < len; ++i)
            for (uint32_t w = 0; w < width; ++w) out.b[i * width + w] = (uint8_t)(best[i] >> (8 * w));
    }
}

// Open-addressing set of byte codes; codes are kept in one arena, so
// inserting and probing allocate nothing per code.
struct CodeSet {
    struct Slot {
        uint64_t hash;
        uint32_t off, len;  // len 0: empty
    };
    std::vector<uint8_t> arena;
    std::vector<Slot> table;
    size_t count = 0;
    CodeSet() : table(1024, Slot{0, 0, 0}) {}
    const uint8_t* at(uint32_t off) const { return arena.data() + off; }
    // true when the code was not present; *off_out = its arena offset
    bool insert(const uint8_t* b, uint32_t len, uint64_t h, uint32_t* off_out = nullptr) {
        if (2 * (count + 1) > table.size()) grow();
        const size_t m = table.size() - 1;
        for (size_t i = h & m;; i = (i + 1) & m) {
            Slot& s = table[i];
            if (s.len == 0) {
                s.hash = h;
                s.off = (uint32_t)arena.size();
                s.len = len;
                arena.insert(arena.end(), b, b + len);
                ++count;
                if (off_out) *off_out = s.off;
                return true;
            }
            if (s.hash == h && s.len == len && std::memcmp(arena.data() + s.off, b, len) == 0) {
                if (off_out) *off_out = s.off;
                return false;
            }
        }
    }
    bool contains(const uint8_t* b, uint32_t len, uint64_t h) const {
        const size_t m = table.size() - 1;
        for (size_t i = h & m;; i = (i + 1) & m) {
            const Slot& s = table[i];
            if (s.len == 0) return false;
            if (s.hash == h && s.len == len && std::memcmp(arena.data() + s.off, b, len) == 0) return true;
        }
    }
    void grow() {
        std::vector<Slot> old(table.size() * 2, Slot{0, 0, 0});
        old.swap(table);
        const size_t m = table.size() - 1;
        for (const Slot& s : old) {
            if (s.len == 0) continue;
            size_t i = s.hash & m;
            while (table[i].len) i = (i + 1) & m;
            table[i] = s;
        }
    }
};

Pattern relabel(const Pattern& p, const uint32_t* ord) {
    Pattern q;
    q.n = p.n;
    uint32_t pos[GVA_MAX_QUERY_VERTICES];
    for (uint32_t i = 0; i < p.n; ++i) {
        pos[ord[i]] = i;
        q.vl[i] = p.vl[ord[i]];
    }
    for (uint32_t i = 0; i < p.ne; ++i) q.add_edge(pos[p.edges[i].u], pos[p.edges[i].v], p.edges[i].el);
    std::sort(q.edges, q.edges + q.ne);
    return q;
}

std::string query_text(const Pattern& p, const std::vector<uint32_t>& labels) {
    std::string o;
    o.reserve(16 * (p.n + p.ne));
    for (uint32_t i = 0; i < p.n; ++i)
        o += "v " + std::to_string(i) + " " + std::to_string(labels[p.vl[i]]) + "\n";
    for (uint32_t i = 0; i < p.ne; ++i)
        o += "e " + std::to_string(p.edges[i].u) + " " + std::to_string(p.edges[i].v) + " " +
             std::to_string(p.edges[i].el) + "\n";
    return o;
}

// Connectivity of the edge set minus edge `skip`; reports the vertex left
// without edges (pendant removal) in `isolated`, or kNone.
bool connected_without(const Pattern& p, uint32_t skip, uint32_t& isolated) {
    uint32_t deg[GVA_MAX_QUERY_VERTICES] = {0};
    for (uint32_t i = 0; i < p.ne; ++i)
        if (i != skip) deg[p.edges[i].u]++, deg[p.edges[i].v]++;
    isolated = kNone;
    uint32_t iso_count = 0, start = kNone;
    for (uint32_t v = 0; v < p.n; ++v) {
        if (deg[v] == 0)
            isolated = v, ++iso_count;
        else if (start == kNone)
            start = v;
    }
    if (iso_count > 1 || start == kNone) return false;
    uint32_t seen = 1u << start, frontier = 1u << start;
    while (frontier) {
        uint32_t nxt = 0;
        for (uint32_t i = 0; i < p.ne; ++i) {
            if (i == skip) continue;
            const uint32_t a = p.edges[i].u, b = p.edges[i].v;
            if (frontier >> a & 1) nxt |= 1u << b;
            if (frontier >> b & 1) nxt |= 1u << a;
        }
        frontier = nxt & ~seen;
        seen |= nxt;
    }
    for (uint32_t v = 0; v < p.n; ++v)
        if (deg[v] && !(seen >> v & 1)) return false;
    return true;
}

Pattern remove_edge(const Pattern& p, uint32_t skip, uint32_t isolated) {
    Pattern q;
    uint32_t map[GVA_MAX_QUERY_VERTICES];
    for (uint32_t v = 0; v < p.n; ++v)
        if (v != isolated) map[v] = q.n, q.vl[q.n++] = p.vl[v];
    for (uint32_t i = 0; i < p.ne; ++i)
        if (i != skip) q.add_edge(map[p.edges[i].u], map[p.edges[i].v], p.edges[i].el);
    return q;
}

// One generated extension: parent pattern + one edge, with its canonical
// code (bytes in the generating thread's CodeSet arena).
struct Ext {
    uint64_t hash;
    uint32_t parent;
    uint32_t code_off;
    uint16_t code_len;
    uint8_t thread;
    uint8_t u, v;  // v == 0xff: forward edge to a new vertex labelled `lab`
    uint8_t pad;
    uint16_t el;
    uint32_t lab;
};

Pattern apply_ext(const Pattern& p, const Ext& x) {
    Pattern c = p;
    if (x.v == 0xff) {
        c.vl[c.n] = x.lab;
        c.add_edge(x.u, c.n, x.el);
        c.n += 1;
    } else {
        c.add_edge(x.u, x.v, x.el);
    }
    return c;
}

constexpr uint32_t kBuckets = 256;  // candidate partitions by code hash (fixed: output order is machine-independent)

}  // namespace

int run_mine(DevDB& db, cudaStream_t s, uint64_t budget, uint32_t max_edges, uint32_t min_support,
             uint32_t batch_limit, bool profile, ReduceFn reduce, void* reduce_user, uint32_t support_mode,
             uint32_t mni_cap, std::vector<MinedPattern>& out, MineStats& st, const volatile int* cancel,
             uint32_t sm_percent, uint32_t host_threads) {
    out.clear();
    st = MineStats();
    const bool mni = support_mode == GVA_SUPPORT_MNI;
    if (support_mode != GVA_SUPPORT_GRAPHS && !mni) return fail(GVA_ERR_ARG, "unknown support mode");
    if (mni) {
        if (reduce) return fail(GVA_ERR_UNSUPPORTED, "MNI supports of graph shards do not add up; mine one graph per process");
        if (max_edges == 0 || max_edges + 1 > (uint32_t)kMniMaxVertices)
            return fail(GVA_ERR_ARG, "MNI mining handles max_edges 1..7");
        if (mni_cap == 0) mni_cap = min_support;
    } else {
        if (!db.vgraph || db.num_graphs == 0) return fail(GVA_ERR_ARG, "mining needs graph ids (gva_db_set_graphs)");
        if (max_edges == 0 || max_edges + 1 > GVA_MAX_QUERY_VERTICES) return fail(GVA_ERR_ARG, "max_edges out of range");
    }
    if (batch_limit == 0) batch_limit = mni ? 65536 : 32768;
    const uint32_t P = (uint32_t)db.parts.size();
    const std::vector<uint32_t>& labels = db.labels;
    auto t_host0 = std::chrono::steady_clock::now();
    double gpu_ms = 0.0;
    const unsigned nthreads =
        std::max(1u, std::min(64u, host_threads ? host_threads : std::thread::hardware_concurrency()));

    // plan + lower candidates [b0, b1) on the worker threads; a failure's
    // message (thread-local) is carried back in `msg`
    auto plan_range = [&](const std::vector<Pattern>& cands, size_t b0, size_t b1,
                          std::vector<std::vector<Step>>& steps, std::string& msg) -> int {
        auto t0 = std::chrono::steady_clock::now();
        steps.assign(b1 - b0, {});
        std::vector<int> rcs(nthreads, GVA_OK);
        std::vector<std::string> msgs(nthreads);
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nthreads; ++t)
            pool.emplace_back([&, t]() {
                for (size_t i = b0 + t; i < b1; i += nthreads) {
                    Plan plan;
                    int r = plan_from_text(query_text(cands[i], labels), GVA_MODE_DV, plan);
                    if (!r) r = lower_plan(plan, db.meta, steps[i - b0], true);
                    if (r) {
                        rcs[t] = r;
                        msgs[t] = last_error_cstr();
                        return;
                    }
                }
            });
        for (auto& th : pool) th.join();
        st.plan_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        for (unsigned t = 0; t < nthreads; ++t)
            if (rcs[t]) {
                msg = msgs[t];
                return rcs[t];
            }
        return GVA_OK;
    };

    // evaluate a candidate list: supports + embeddings.  All candidates are
    // planned first and ordered by their step sequences, so that candidates
    // sharing plan prefixes land in the same batch (one trie: a shared prefix
    // is matched once); then they run in bounded batches.
    // MNI: image-set supports of every candidate on the one data graph, in
    // batches of batch_limit patterns (no embedding counts)
    auto evaluate_mni = [&](const std::vector<Pattern>& cands, std::vector<uint32_t>& sup,
                            std::vector<uint64_t>& emb) -> int {
        const size_t n = cands.size();
        sup.assign(n, 0);
        emb.assign(n, 0);
        std::vector<uint32_t> bsup;
        // batch b + 1's search tasks are built on a helper thread while batch
        // b's rounds run on the device
        const size_t nbatch = (n + batch_limit - 1) / batch_limit;
        auto prepare = [&](size_t b) {
            const size_t b0 = b * batch_limit, b1 = std::min(n, b0 + (size_t)batch_limit);
            std::vector<MniPattern> mp(b1 - b0);
            for (size_t i = b0; i < b1; ++i) {
                const Pattern& c = cands[i];
                MniPattern& m = mp[i - b0];
                m.n = c.n;
                for (uint32_t v = 0; v < c.n; ++v) m.vl[v] = c.vl[v];
                for (uint32_t e = 0; e < c.ne; ++e)
                    m.el[c.edges[e].u][c.edges[e].v] = m.el[c.edges[e].v][c.edges[e].u] = (uint8_t)c.edges[e].el;
            }
            return mni_prepare(db, mp, {}, nthreads);
        };
        std::future<std::shared_ptr<MniPrepared>> next =
            nbatch ? std::async(std::launch::async, prepare, (size_t)0) : std::future<std::shared_ptr<MniPrepared>>();
        for (size_t b = 0; b < nbatch; ++b) {
            const size_t b0 = b * batch_limit, b1 = std::min(n, b0 + (size_t)batch_limit);
            std::shared_ptr<MniPrepared> cur = next.get();
            if (b + 1 < nbatch) next = std::async(std::launch::async, prepare, b + 1);
            MniStats ms;
            int rc = mni_run_prepared(db, *cur, mni_cap, false, profile, s, bsup, ms, cancel, sm_percent);
            if (rc) return rc;
            for (size_t i = b0; i < b1; ++i) sup[i] = bsup[i - b0];
            gpu_ms += ms.gpu_ms;
            st.wait_ms += ms.wait_ms;
            st.mni_tasks += ms.tasks;
            st.mni_rounds += ms.rounds;
            st.mni_found += ms.found;
            st.kstat[K_MNI].launches += ms.kstat.launches;
            st.kstat[K_MNI].ms += ms.kstat.ms;
            st.kstat[K_MNI].bytes += ms.kstat.bytes;
            st.kstat[K_MNI].rows += ms.kstat.rows;
        }
        st.candidates += n;
        return GVA_OK;
    };

    auto evaluate = [&](const std::vector<Pattern>& cands, std::vector<uint32_t>& sup, std::vector<uint64_t>& emb) -> int {
        const size_t n = cands.size();
        if (mni) return evaluate_mni(cands, sup, emb);
        sup.assign(n, 0);
        emb.assign(n, 0);
        if (n == 0) return GVA_OK;
        std::vector<std::vector<Step>> all;
        std::string msg;
        int prc = plan_range(cands, 0, n, all, msg);
        if (prc) return fail(prc, msg);
        auto t_order = std::chrono::steady_clock::now();
        size_t width_k = 0;
        for (auto& v : all) width_k = std::max(width_k, v.size());
        std::vector<uint64_t> key(n * width_k, 0);
        {
            std::vector<std::thread> pool;
            for (unsigned t = 0; t < nthreads; ++t)
                pool.emplace_back([&, t]() {
                    uint8_t kb[512];
                    for (size_t i = t; i < n; i += nthreads)
                        for (size_t j = 0; j < all[i].size(); ++j) {
                            const size_t len = step_key_bytes(all[i][j], kb);
                            key[i * width_k + j] = code_hash(kb, (uint32_t)len) | 1;  // 0 marks the end
                        }
                });
            for (auto& th : pool) th.join();
        }
        std::vector<uint32_t> order(n);
        for (size_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
            const uint64_t* ka = key.data() + (size_t)a * width_k;
            const uint64_t* kb = key.data() + (size_t)b * width_k;
            for (size_t j = 0; j < width_k; ++j)
                if (ka[j] != kb[j]) return ka[j] < kb[j];
            return a < b;
        });
        st.plan_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_order).count();
        std::vector<uint32_t> bsup;
        std::vector<uint64_t> bemb;
        // batch b + 1's session (device set-up, step trie) is built on a
        // helper thread while batch b's rounds run
        struct Prep {
            PreparedBatch pb;
            int rc = GVA_OK;
            std::string err;
        };
        const size_t nbatch = (n + batch_limit - 1) / batch_limit;
        auto prepare = [&](size_t b) {
            std::unique_ptr<Prep> p(new Prep());
            const size_t b0 = b * batch_limit, b1 = std::min(n, b0 + batch_limit);
            std::vector<std::vector<Step>> cur(b1 - b0);
            for (size_t i = b0; i < b1; ++i) cur[i - b0] = std::move(all[order[i]]);
            p->rc = prepare_batch(db, cur, s, budget, true, false, profile, p->pb);
            if (p->rc) p->err = last_error_cstr();
            return p;
        };
        std::future<std::unique_ptr<Prep>> next = std::async(std::launch::async, prepare, (size_t)0);
        for (size_t b = 0; b < nbatch; ++b) {
            const size_t b0 = b * batch_limit, b1 = std::min(n, b0 + batch_limit);
            std::unique_ptr<Prep> cur = next.get();
            if (b + 1 < nbatch) next = std::async(std::launch::async, prepare, b + 1);
            if (cur->rc) return fail(cur->rc, cur->err);
            bsup.assign(b1 - b0, 0);
            bemb.assign(b1 - b0, 0);
            BatchStats bs;
            int rc = finish_batch(db, cur->pb, bemb.data(), nullptr, bsup.data(), &bs, cancel);
            if (rc) return rc;
            for (size_t i = b0; i < b1; ++i) {
                sup[order[i]] = bsup[i - b0];
                emb[order[i]] = bemb[i - b0];
            }
            gpu_ms += bs.gpu_ms;
            st.submit_ms += bs.submit_ms;
            st.round_host_ms += bs.round_host_ms;
            st.wait_ms += bs.wait_ms;
            st.session_ms += bs.session_ms;
            for (int i = 0; i < 5; ++i) st.phase_ms[i] += bs.phase_ms[i];
            for (int kk = 0; kk < K_NUM; ++kk) {
                st.kstat[kk].launches += bs.kstat[kk].launches;
                st.kstat[kk].ms += bs.kstat[kk].ms;
                st.kstat[kk].bytes += bs.kstat[kk].bytes;
                st.kstat[kk].rows += bs.kstat[kk].rows;
            }
        }
        st.candidates += n;
        for (uint64_t e : emb) st.embeddings += e;  // this process's share
        if (reduce && reduce(sup.data(), emb.data(), n, reduce_user))
            return fail(GVA_ERR_ARG, "support reduction across processes failed");
        return GVA_OK;
    };

    // ---- level 1: every edge type
    const uint32_t L = (uint32_t)labels.size();
    const uint32_t width = (L <= 256 && P <= 255) ? 1 : (L <= 65536 ? 2 : 4);
    std::vector<Pattern> cands;
    for (uint32_t a = 0; a < L; ++a)
        for (uint32_t b = a; b < L; ++b)
            for (uint32_t el = 1; el <= P; ++el) {
                if (!db.parts[el - 1].off) continue;
                Pattern p;
                p.n = 2;
                p.vl[0] = a;
                p.vl[1] = b;
                p.add_edge(0, 1, el);
                cands.push_back(p);
            }
    std::vector<uint32_t> sup;
    std::vector<uint64_t> emb;
    int rc = evaluate(cands, sup, emb);
    if (rc) return rc;
    std::vector<char> freq_tab((size_t)L * L * (P + 1), 0);  // frequent edge types (a, b, el), both orientations
    auto freq = [&](uint32_t a, uint32_t el, uint32_t b) { return freq_tab[((size_t)a * L + b) * (P + 1) + el] != 0; };
    std::vector<Pattern> level;
    CodeSet level_codes;
    CodeBuf cbuf;
    for (size_t i = 0; i < cands.size(); ++i) {
        if (sup[i] < min_support) continue;
        const Pattern& p = cands[i];
        const uint32_t el = p.edges[0].el;
        freq_tab[((size_t)p.vl[0] * L + p.vl[1]) * (P + 1) + el] = 1;
        freq_tab[((size_t)p.vl[1] * L + p.vl[0]) * (P + 1) + el] = 1;
        uint32_t ord[GVA_MAX_QUERY_VERTICES];
        canonical(p, width, cbuf, ord);
        Pattern q = relabel(p, ord);
        level.push_back(q);
        level_codes.insert(cbuf.b, cbuf.len, code_hash(cbuf.b, cbuf.len));
        out.push_back({query_text(q, labels), 1, sup[i], emb[i]});
    }
    st.levels = 1;

    // ---- levels 2..max_edges
    for (uint32_t k = 1; k < max_edges && !level.empty(); ++k) {
        if (cancel && *cancel) return fail(GVA_ERR_CANCELLED, "cancelled");
        auto t_gen = std::chrono::steady_clock::now();
        // (1) each thread extends every nthreads-th pattern by one frequent
        // edge type, keeps the extensions whose canonical code it has not seen
        // yet and files them by code hash into kBuckets partitions
        std::vector<CodeSet> seen(nthreads);
        std::vector<std::vector<std::vector<Ext>>> exts(nthreads, std::vector<std::vector<Ext>>(kBuckets));
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nthreads; ++t)
            pool.emplace_back([&, t]() {
                CodeBuf cb;
                auto consider = [&](uint32_t parent, const Pattern& c, const Ext& x) {
                    canonical(c, width, cb);
                    const uint64_t h = code_hash(cb.b, cb.len);
                    uint32_t off;
                    if (!seen[t].insert(cb.b, cb.len, h, &off)) return;
                    Ext e = x;
                    e.hash = h;
                    e.parent = parent;
                    e.code_off = off;
                    e.code_len = (uint16_t)cb.len;
                    e.thread = (uint8_t)t;
                    exts[t][h % kBuckets].push_back(e);
                };
                for (size_t i = t; i < level.size(); i += nthreads) {
                    const Pattern& p = level[i];
                    Ext x{};
                    for (uint32_t u = 0; u < p.n; ++u) {
                        x.u = (uint8_t)u;
                        for (uint32_t v = u + 1; v < p.n; ++v) {  // backward edges
                            if (p.el(u, v)) continue;
                            x.v = (uint8_t)v;
                            for (uint32_t el = 1; el <= P; ++el) {
                                if (!freq(p.vl[u], el, p.vl[v])) continue;
                                x.el = (uint16_t)el;
                                consider((uint32_t)i, apply_ext(p, x), x);
                            }
                        }
                        if (p.n + 1 > max_edges + 1 || p.n + 1 > GVA_MAX_QUERY_VERTICES) continue;
                        x.v = 0xff;
                        for (uint32_t el = 1; el <= P; ++el) {  // forward edges
                            x.el = (uint16_t)el;
                            for (uint32_t l = 0; l < L; ++l) {
                                if (!freq(p.vl[u], el, l)) continue;
                                x.lab = l;
                                consider((uint32_t)i, apply_ext(p, x), x);
                            }
                        }
                    }
                }
            });
        for (auto& th : pool) th.join();
        // (2) each partition is deduplicated across threads (sorted by code, so
        // the level's order depends on the codes only), and each distinct
        // candidate is kept only if every connected k-edge sub-pattern other
        // than its parent is frequent (anti-monotone support); survivors are
        // stored in canonical vertex order
        auto t_merge = std::chrono::steady_clock::now();
        std::vector<std::vector<Pattern>> buckets(kBuckets);
        std::vector<uint64_t> pruned(kBuckets, 0);
        std::atomic<uint32_t> next_bucket{0};
        pool.clear();
        for (unsigned t = 0; t < nthreads; ++t)
            pool.emplace_back([&]() {
                std::vector<const Ext*> all;
                CodeBuf sb;
                for (uint32_t b; (b = next_bucket.fetch_add(1)) < kBuckets;) {
                    all.clear();
                    for (unsigned w = 0; w < nthreads; ++w)
                        for (const Ext& x : exts[w][b]) all.push_back(&x);
                    auto bytes = [&](const Ext* x) { return seen[x->thread].at(x->code_off); };
                    auto less = [&](const Ext* a, const Ext* c) {
                        if (a->hash != c->hash) return a->hash < c->hash;
                        if (a->code_len != c->code_len) return a->code_len < c->code_len;
                        return std::memcmp(bytes(a), bytes(c), a->code_len) < 0;
                    };
                    std::sort(all.begin(), all.end(), less);
                    for (size_t i = 0; i < all.size(); ++i) {
                        if (i > 0 && !less(all[i - 1], all[i])) continue;  // same code as the previous one
                        const Ext& x = *all[i];
                        Pattern c = apply_ext(level[x.parent], x);
                        bool ok = true;
                        for (uint32_t e = 0; e + 1 < c.ne && ok; ++e) {  // edge c.ne - 1 is the parent's extension
                            uint32_t iso;
                            if (!connected_without(c, e, iso)) continue;
                            canonical(remove_edge(c, e, iso), width, sb);
                            ok = level_codes.contains(sb.b, sb.len, code_hash(sb.b, sb.len));
                        }
                        if (!ok) {
                            pruned[b]++;
                            continue;
                        }
                        uint32_t ord[GVA_MAX_QUERY_VERTICES];
                        canonical(c, width, sb, ord);
                        buckets[b].push_back(relabel(c, ord));
                    }
                }
            });
        for (auto& th : pool) th.join();
        std::vector<Pattern> next;
        for (uint32_t b = 0; b < kBuckets; ++b) {
            st.pruned += pruned[b];
            next.insert(next.end(), buckets[b].begin(), buckets[b].end());
        }
        exts.clear();
        seen.clear();
        st.merge_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_merge).count();
        st.gen_ms += std::chrono::duration<double, std::milli>(t_merge - t_gen).count();
        auto t_eval = std::chrono::steady_clock::now();
        rc = evaluate(next, sup, emb);
        if (rc) return rc;
        st.eval_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_eval).count();
        level.clear();
        level_codes = CodeSet();
        for (size_t i = 0; i < next.size(); ++i) {
            if (sup[i] < min_support) continue;
            level.push_back(next[i]);
            canonical(next[i], width, cbuf);
            level_codes.insert(cbuf.b, cbuf.len, code_hash(cbuf.b, cbuf.len));
            out.push_back({query_text(next[i], labels), k + 1, sup[i], emb[i]});
        }
        st.levels = k + 1;
    }
    st.frequent = out.size();
    st.gpu_ms = gpu_ms;
    st.host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_host0).count();
    if (getenv("GVA_TRACE"))  // host-time split, for tuning
        fprintf(stderr,
                "gva_mine: host %.1f ms: gen %.1f merge %.1f plan %.1f eval %.1f (submit %.1f session %.1f rounds %.1f "
                "[scan %.1f count %.1f choose %.1f write %.1f next %.1f] wait %.1f) gpu %.1f\n",
                st.host_ms, st.gen_ms, st.merge_ms, st.plan_ms, st.eval_ms, st.submit_ms, st.session_ms,
                st.round_host_ms, st.phase_ms[0], st.phase_ms[1], st.phase_ms[2], st.phase_ms[3], st.phase_ms[4],
                st.wait_ms, st.gpu_ms);
    return GVA_OK;
}

}  // namespace gva
