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
#include <array>
#include <chrono>
#include <cstring>
#include <functional>
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

struct Pattern {
    uint32_t n = 0;
    uint32_t vl[GVA_MAX_QUERY_VERTICES];
    std::vector<std::array<uint32_t, 3>> edges;  // (u, v, edge label), u < v
    uint32_t el(uint32_t a, uint32_t b) const {
        for (auto& e : edges)
            if ((e[0] == a && e[1] == b) || (e[0] == b && e[1] == a)) return e[2];
        return 0;
    }
};

using Code = std::vector<uint32_t>;

struct CodeHash {
    size_t operator()(const Code& c) const {
        size_t h = 1469598103934665603ull;
        for (uint32_t x : c) h = (h ^ x) * 1099511628211ull;
        return h;
    }
};

// Canonical code: the lexicographically smallest (n, labels, upper-triangle
// edge labels) over vertex orders that sort vertices by an isomorphism-
// invariant key (label, degree, hash of the sorted (edge label, neighbour
// label) list); only orders within equal-key cells are tried.  Equal keys of
// non-equivalent vertices only enlarge a cell, which costs time, not
// correctness.  Work arrays live on the stack (patterns have <= 32 vertices).
Code canonical(const Pattern& p, std::vector<uint32_t>* order_out = nullptr) {
    const uint32_t n = p.n;
    uint32_t adj[GVA_MAX_QUERY_VERTICES][GVA_MAX_QUERY_VERTICES];
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = 0; j < n; ++j) adj[i][j] = 0;
    for (auto& e : p.edges) adj[e[0]][e[1]] = adj[e[1]][e[0]] = e[2];
    uint64_t key[GVA_MAX_QUERY_VERTICES];
    for (uint32_t v = 0; v < n; ++v) {
        uint64_t nb[GVA_MAX_QUERY_VERTICES];
        uint32_t d = 0;
        for (uint32_t u = 0; u < n; ++u)
            if (adj[v][u]) nb[d++] = ((uint64_t)adj[v][u] << 32) | p.vl[u];
        std::sort(nb, nb + d);
        uint64_t h = 1469598103934665603ull;
        for (uint32_t i = 0; i < d; ++i) h = (h ^ nb[i]) * 1099511628211ull;
        key[v] = ((uint64_t)(p.vl[v] & 0xffffu) << 48) | ((uint64_t)d << 40) | (h & 0xffffffffffull);
    }
    uint32_t ord[GVA_MAX_QUERY_VERTICES];
    for (uint32_t i = 0; i < n; ++i) ord[i] = i;
    std::sort(ord, ord + n, [&](uint32_t a, uint32_t b) { return key[a] != key[b] ? key[a] < key[b] : a < b; });
    uint32_t cb[GVA_MAX_QUERY_VERTICES], ce[GVA_MAX_QUERY_VERTICES], nc = 0;  // cells [cb, ce)
    for (uint32_t i = 0; i < n;) {
        uint32_t j = i + 1;
        while (j < n && key[ord[j]] == key[ord[i]]) ++j;
        cb[nc] = i;
        ce[nc++] = j;
        i = j;
    }
    const size_t len = 1 + n + (size_t)n * (n - 1) / 2;
    Code best(len), cur(len);
    uint32_t best_ord[GVA_MAX_QUERY_VERTICES];
    bool have = false;
    for (;;) {
        // build the code, giving up as soon as it exceeds the best one
        cur[0] = n;
        int cmp = have ? 0 : -1;
        size_t k = 1;
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
            best.swap(cur);
            for (uint32_t i = 0; i < n; ++i) best_ord[i] = ord[i];
            have = true;
        }
        int c = (int)nc - 1;
        for (; c >= 0; --c)
            if (std::next_permutation(ord + cb[c], ord + ce[c])) break;
        if (c < 0) break;
    }
    if (order_out) order_out->assign(best_ord, best_ord + n);
    return best;
}

Pattern relabel(const Pattern& p, const std::vector<uint32_t>& ord) {
    Pattern q;
    q.n = p.n;
    std::vector<uint32_t> pos(p.n);
    for (uint32_t i = 0; i < p.n; ++i) {
        pos[ord[i]] = i;
        q.vl[i] = p.vl[ord[i]];
    }
    for (auto& e : p.edges) {
        uint32_t a = pos[e[0]], b = pos[e[1]];
        q.edges.push_back({std::min(a, b), std::max(a, b), e[2]});
    }
    std::sort(q.edges.begin(), q.edges.end());
    return q;
}

std::string query_text(const Pattern& p) {
    std::ostringstream o;
    for (uint32_t i = 0; i < p.n; ++i) o << "v " << i << " " << p.vl[i] << "\n";
    for (auto& e : p.edges) o << "e " << e[0] << " " << e[1] << " " << e[2] << "\n";
    return o.str();
}

bool connected_without(const Pattern& p, size_t skip, uint32_t& isolated) {
    // connectivity of the edge set minus edge `skip`; reports a vertex left
    // without edges (pendant removal), or kNone
    std::vector<uint32_t> deg(p.n, 0);
    for (size_t i = 0; i < p.edges.size(); ++i)
        if (i != skip) deg[p.edges[i][0]]++, deg[p.edges[i][1]]++;
    isolated = kNone;
    uint32_t iso_count = 0;
    for (uint32_t v = 0; v < p.n; ++v)
        if (deg[v] == 0) isolated = v, ++iso_count;
    if (iso_count > 1) return false;
    uint32_t start = kNone;
    for (uint32_t v = 0; v < p.n; ++v)
        if (deg[v]) { start = v; break; }
    if (start == kNone) return false;
    std::vector<char> seen(p.n, 0);
    std::vector<uint32_t> st{start};
    seen[start] = 1;
    while (!st.empty()) {
        uint32_t v = st.back();
        st.pop_back();
        for (size_t i = 0; i < p.edges.size(); ++i) {
            if (i == skip) continue;
            uint32_t a = p.edges[i][0], b = p.edges[i][1];
            uint32_t o = a == v ? b : (b == v ? a : kNone);
            if (o != kNone && !seen[o]) seen[o] = 1, st.push_back(o);
        }
    }
    for (uint32_t v = 0; v < p.n; ++v)
        if (deg[v] && !seen[v]) return false;
    return true;
}

Pattern remove_edge(const Pattern& p, size_t skip, uint32_t isolated) {
    Pattern q;
    std::vector<uint32_t> map(p.n, kNone);
    for (uint32_t v = 0; v < p.n; ++v)
        if (v != isolated) map[v] = q.n, q.vl[q.n++] = p.vl[v];
    for (size_t i = 0; i < p.edges.size(); ++i)
        if (i != skip) {
            uint32_t a = map[p.edges[i][0]], b = map[p.edges[i][1]];
            q.edges.push_back({std::min(a, b), std::max(a, b), p.edges[i][2]});
        }
    return q;
}

}  // namespace

int run_mine(DevDB& db, cudaStream_t s, uint64_t budget, uint32_t max_edges, uint32_t min_support,
             uint32_t batch_limit, bool profile, ReduceFn reduce, void* reduce_user, std::vector<MinedPattern>& out,
             MineStats& st) {
    out.clear();
    st = MineStats();
    if (!db.vgraph || db.num_graphs == 0) return fail(GVA_ERR_ARG, "mining needs graph ids (gva_db_set_graphs)");
    if (max_edges == 0 || max_edges + 1 > GVA_MAX_QUERY_VERTICES) return fail(GVA_ERR_ARG, "max_edges out of range");
    if (batch_limit == 0) batch_limit = 8192;
    const uint32_t P = (uint32_t)db.parts.size();
    const std::vector<uint32_t>& labels = db.labels;
    auto t_host0 = std::chrono::steady_clock::now();
    double gpu_ms = 0.0;
    const unsigned nthreads = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));

    // evaluate a candidate list: supports + embeddings, in bounded batches
    auto evaluate = [&](const std::vector<Pattern>& cands, std::vector<uint32_t>& sup, std::vector<uint64_t>& emb) -> int {
        sup.assign(cands.size(), 0);
        emb.assign(cands.size(), 0);
        for (size_t b0 = 0; b0 < cands.size(); b0 += batch_limit) {
            const size_t b1 = std::min(cands.size(), b0 + batch_limit);
            std::vector<std::vector<Step>> steps(b1 - b0);
            auto t0 = std::chrono::steady_clock::now();
            std::vector<int> rcs(nthreads, GVA_OK);
            std::vector<std::thread> pool;
            for (unsigned t = 0; t < nthreads; ++t)
                pool.emplace_back([&, t]() {
                    for (size_t i = b0 + t; i < b1; i += nthreads) {
                        Plan plan;
                        int r = plan_from_text(query_text(cands[i]), GVA_MODE_DV, plan);
                        if (!r) r = lower_plan(plan, db.meta, steps[i - b0], true);
                        if (r) {
                            rcs[t] = r;
                            return;
                        }
                    }
                });
            for (auto& th : pool) th.join();
            for (int r : rcs)
                if (r) return r;
            st.plan_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            BatchStats bs;
            int rc = run_batch(db, steps, s, budget, db.vgraph, db.num_graphs, emb.data() + b0, nullptr,
                               sup.data() + b0, profile, &bs);
            if (rc) return rc;
            gpu_ms += bs.gpu_ms;
            st.submit_ms += bs.submit_ms;
            st.round_host_ms += bs.round_host_ms;
            st.wait_ms += bs.wait_ms;
            for (int kk = 0; kk < K_NUM; ++kk) {
                st.kstat[kk].launches += bs.kstat[kk].launches;
                st.kstat[kk].ms += bs.kstat[kk].ms;
                st.kstat[kk].bytes += bs.kstat[kk].bytes;
                st.kstat[kk].rows += bs.kstat[kk].rows;
            }
        }
        st.candidates += cands.size();
        for (uint64_t e : emb) st.embeddings += e;  // this process's share
        if (reduce && !cands.empty() && reduce(sup.data(), emb.data(), cands.size(), reduce_user))
            return fail(GVA_ERR_ARG, "support reduction across processes failed");
        return GVA_OK;
    };

    // ---- level 1: every edge type
    std::vector<Pattern> cands;
    for (uint32_t a = 0; a < labels.size(); ++a)
        for (uint32_t b = a; b < labels.size(); ++b)
            for (uint32_t el = 1; el <= P; ++el) {
                if (!db.parts[el - 1].off) continue;
                Pattern p;
                p.n = 2;
                p.vl[0] = labels[a];
                p.vl[1] = labels[b];
                p.edges.push_back({0, 1, el});
                cands.push_back(p);
            }
    std::vector<uint32_t> sup;
    std::vector<uint64_t> emb;
    int rc = evaluate(cands, sup, emb);
    if (rc) return rc;
    std::set<std::array<uint32_t, 3>> freq_edge;  // (min label, edge label, max label)
    std::vector<Pattern> level;
    std::unordered_set<Code, CodeHash> level_codes;
    for (size_t i = 0; i < cands.size(); ++i) {
        if (sup[i] < min_support) continue;
        const Pattern& p = cands[i];
        freq_edge.insert({std::min(p.vl[0], p.vl[1]), p.edges[0][2], std::max(p.vl[0], p.vl[1])});
        std::vector<uint32_t> ord;
        Code c = canonical(p, &ord);
        Pattern q = relabel(p, ord);
        level.push_back(q);
        level_codes.insert(c);
        out.push_back({query_text(q), 1, sup[i], emb[i]});
    }
    st.levels = 1;

    // ---- levels 2..max_edges
    for (uint32_t k = 1; k < max_edges && !level.empty(); ++k) {
        auto t_gen = std::chrono::steady_clock::now();
        auto freq = [&](uint32_t a, uint32_t el, uint32_t b) {
            return freq_edge.count({std::min(a, b), el, std::max(a, b)}) != 0;
        };
        // each thread extends every nthreads-th pattern; candidates are merged
        // by canonical code and sorted so the level is deterministic
        std::vector<std::vector<std::pair<Code, Pattern>>> found(nthreads);
        std::vector<uint64_t> pruned(nthreads, 0);
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nthreads; ++t)
            pool.emplace_back([&, t]() {
                std::unordered_set<Code, CodeHash> seen;
                auto consider = [&](const Pattern& c) {
                    std::vector<uint32_t> ord;
                    Code code = canonical(c, &ord);
                    if (!seen.insert(code).second) return;
                    // every connected k-edge sub-pattern must be frequent
                    for (size_t e = 0; e < c.edges.size(); ++e) {
                        uint32_t iso;
                        if (!connected_without(c, e, iso)) continue;
                        if (!level_codes.count(canonical(remove_edge(c, e, iso)))) {
                            pruned[t]++;
                            return;
                        }
                    }
                    found[t].push_back({std::move(code), relabel(c, ord)});
                };
                for (size_t i = t; i < level.size(); i += nthreads) {
                    const Pattern& p = level[i];
                    for (uint32_t u = 0; u < p.n; ++u) {
                        for (uint32_t v = u + 1; v < p.n; ++v) {  // backward edges
                            if (p.el(u, v)) continue;
                            for (uint32_t el = 1; el <= P; ++el) {
                                if (!freq(p.vl[u], el, p.vl[v])) continue;
                                Pattern c = p;
                                c.edges.push_back({u, v, el});
                                consider(c);
                            }
                        }
                        if (p.n + 1 > max_edges + 1 || p.n + 1 > GVA_MAX_QUERY_VERTICES) continue;
                        for (uint32_t el = 1; el <= P; ++el) {  // forward edges
                            for (uint32_t l : labels) {
                                if (!freq(p.vl[u], el, l)) continue;
                                Pattern c = p;
                                c.vl[c.n] = l;
                                c.edges.push_back({u, c.n, el});
                                c.n += 1;
                                consider(c);
                            }
                        }
                    }
                }
            });
        for (auto& th : pool) th.join();
        // merge: bucket candidates by code hash, dedupe and sort each bucket on
        // its own thread, concatenate the buckets in order (deterministic)
        auto t_merge = std::chrono::steady_clock::now();
        for (unsigned t = 0; t < nthreads; ++t) st.pruned += pruned[t];
        std::vector<std::vector<Pattern>> buckets(nthreads);
        {
            CodeHash hasher;
            std::vector<std::vector<size_t>> hs(nthreads);
            std::vector<std::thread> hp;
            for (unsigned t = 0; t < nthreads; ++t)
                hp.emplace_back([&, t]() {
                    hs[t].reserve(found[t].size());
                    for (auto& x : found[t]) hs[t].push_back(hasher(x.first) % nthreads);
                });
            for (auto& th : hp) th.join();
            std::vector<std::thread> bp;
            for (unsigned b = 0; b < nthreads; ++b)
                bp.emplace_back([&, b]() {
                    std::vector<std::pair<Code, Pattern>*> mine;
                    for (unsigned t = 0; t < nthreads; ++t)
                        for (size_t i = 0; i < found[t].size(); ++i)
                            if (hs[t][i] == b) mine.push_back(&found[t][i]);
                    std::sort(mine.begin(), mine.end(), [](const auto* a, const auto* c) { return a->first < c->first; });
                    for (size_t i = 0; i < mine.size(); ++i)
                        if (i == 0 || mine[i]->first != mine[i - 1]->first) buckets[b].push_back(std::move(mine[i]->second));
                });
            for (auto& th : bp) th.join();
        }
        std::vector<Pattern> next;
        for (auto& bk : buckets)
            for (auto& pt : bk) next.push_back(std::move(pt));
        st.merge_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_merge).count();
        st.gen_ms += std::chrono::duration<double, std::milli>(t_merge - t_gen).count();
        auto t_eval = std::chrono::steady_clock::now();
        rc = evaluate(next, sup, emb);
        if (rc) return rc;
        st.eval_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_eval).count();
        level.clear();
        level_codes.clear();
        for (size_t i = 0; i < next.size(); ++i) {
            if (sup[i] < min_support) continue;
            level.push_back(next[i]);
            level_codes.insert(canonical(next[i]));
            out.push_back({query_text(next[i]), k + 1, sup[i], emb[i]});
        }
        st.levels = k + 1;
    }
    st.frequent = out.size();
    st.gpu_ms = gpu_ms;
    st.host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_host0).count();
    return GVA_OK;
}

}  // namespace gva
