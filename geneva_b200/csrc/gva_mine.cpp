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
// query text (computed from the pattern by the heap-free planner, gva_dplan.h,
// or the host planner for the queries it leaves), so embedding counts are the
// reference's row counts.  The level loop is mine_levels (gva_grow.h); this
// file supplies its evaluators (graph supports, MNI supports).
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
#include "gva_dplan.h"
#include "gva_grow.h"
#include "gva_pool.h"

namespace gva {

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
        const unsigned pt = std::max(1u, std::min<unsigned>(nthreads, (unsigned)((b1 - b0) / 64 + 1)));
        std::vector<int> rcs(pt, GVA_OK);
        std::vector<std::string> msgs(pt);
        pool_run(pt, [&](unsigned t) {
                uint32_t sdl[3 * kMaxPatEdges];
                std::unique_ptr<DPlanQuery> dq(new DPlanQuery());
                std::unique_ptr<DPlan> dp(new DPlan());
                for (size_t i = b0 + t; i < b1; i += pt) {
                    // the plan of the candidate's query text, built from the
                    // pattern by the heap-free planner, else by the host planner
                    const Pattern& c = cands[i];
                    dq->n = c.n;
                    dq->lines = c.ne;
                    for (uint32_t v = 0; v < c.n; ++v) dq->label[v] = labels[c.vl[v]];
                    for (uint32_t e = 0; e < c.ne; ++e) {
                        dq->s[e] = sdl[3 * e] = c.edges[e].u;
                        dq->d[e] = sdl[3 * e + 1] = c.edges[e].v;
                        dq->l[e] = sdl[3 * e + 2] = c.edges[e].el;
                    }
                    dplan(*dq, *dp);
                    int r;
                    if (dp->status == DPLAN_OK) {
                        r = lower_dplan(*dp, dq->label, db.meta, steps[i - b0], true);
                    } else {
                        Plan plan;
                        r = plan_from_query(c.n, dq->label, sdl, c.ne, GVA_MODE_DV, plan);
                        if (!r) r = lower_plan(plan, db.meta, steps[i - b0], true);
                    }
                    if (r) {
                        rcs[t] = r;
                        msgs[t] = last_error_cstr();
                        return;
                    }
                }
            });
        st.plan_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        for (unsigned t = 0; t < pt; ++t)
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
            const unsigned kt = std::max(1u, std::min<unsigned>(nthreads, (unsigned)(n / 256 + 1)));
            pool_run(kt, [&](unsigned t) {
                for (size_t i = t; i < n; i += kt)
                    for (size_t j = 0; j < all[i].size(); ++j)
                        key[i * width_k + j] = step_key_hash(all[i][j]);  // never 0: 0 marks the end
            });
        }
        std::vector<uint32_t> order(n);
        for (size_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
        parallel_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
            const uint64_t* ka = key.data() + (size_t)a * width_k;
            const uint64_t* kb = key.data() + (size_t)b * width_k;
            for (size_t j = 0; j < width_k; ++j)
                if (ka[j] != kb[j]) return ka[j] < kb[j];
            return a < b;
        }, nthreads);
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
            p->rc = prepare_batch(db, std::move(cur), s, budget, true, false, profile, p->pb, true);  // ordered by step keys
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

    std::vector<char> has_part(P + 1, 0);
    for (uint32_t el = 1; el <= P; ++el) has_part[el] = db.parts[el - 1].off != nullptr;
    LevelStats ls;
    int rc = mine_levels((uint32_t)labels.size(), P, has_part, labels, max_edges, min_support, nthreads, cancel,
                         evaluate, out, ls);
    st.pruned = ls.pruned;
    st.gen_ms = ls.gen_ms;
    st.merge_ms = ls.merge_ms;
    st.eval_ms = ls.eval_ms;
    st.levels = ls.levels;
    if (rc == GVA_ERR_CANCELLED) return fail(rc, "cancelled");
    if (rc) return rc;
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

int run_mine_host(const std::vector<uint32_t>& labels, uint32_t num_edge_labels, const uint8_t* has_edge_label,
                  uint32_t max_edges, uint32_t min_support, uint32_t host_threads, TextEvalFn evaluate,
                  void* eval_user, ReduceFn reduce, void* reduce_user, std::vector<MinedPattern>& out, MineStats& st) {
    out.clear();
    st = MineStats();
    if (!evaluate) return fail(GVA_ERR_ARG, "no evaluator");
    if (labels.empty() || num_edge_labels == 0 || !has_edge_label) return fail(GVA_ERR_ARG, "no labels");
    for (size_t i = 1; i < labels.size(); ++i)
        if (labels[i] <= labels[i - 1]) return fail(GVA_ERR_ARG, "vertex labels must be ascending and distinct");
    if (max_edges == 0 || max_edges + 1 > (uint32_t)GVA_MAX_QUERY_VERTICES)
        return fail(GVA_ERR_ARG, "max_edges out of range");
    const auto t0 = std::chrono::steady_clock::now();
    const unsigned nthreads =
        host_threads ? host_threads : std::max(1u, (unsigned)std::thread::hardware_concurrency());
    std::vector<char> has_part(num_edge_labels + 1, 0);
    for (uint32_t el = 1; el <= num_edge_labels; ++el) has_part[el] = has_edge_label[el] != 0;
    std::string blob;
    std::vector<uint64_t> offsets;
    auto eval = [&](const std::vector<Pattern>& cands, std::vector<uint32_t>& sup, std::vector<uint64_t>& emb) -> int {
        const size_t n = cands.size();
        sup.assign(n, 0);
        emb.assign(n, 0);
        if (n == 0) return GVA_OK;
        blob.clear();
        offsets.resize(n);
        for (size_t i = 0; i < n; ++i) {
            offsets[i] = blob.size();
            blob += query_text(cands[i], labels);
            blob.push_back('\0');
        }
        if (evaluate(blob.data(), offsets.data(), n, sup.data(), emb.data(), eval_user))
            return fail(GVA_ERR_ARG, "candidate evaluation failed");
        st.candidates += n;
        for (uint64_t e : emb) st.embeddings += e;  // this process's share
        if (reduce && reduce(sup.data(), emb.data(), n, reduce_user))
            return fail(GVA_ERR_ARG, "support reduction across processes failed");
        return GVA_OK;
    };
    LevelStats ls;
    int rc = mine_levels((uint32_t)labels.size(), num_edge_labels, has_part, labels, max_edges, min_support, nthreads,
                         nullptr, eval, out, ls);
    if (rc) return rc;
    st.pruned = ls.pruned;
    st.gen_ms = ls.gen_ms;
    st.merge_ms = ls.merge_ms;
    st.eval_ms = ls.eval_ms;
    st.levels = ls.levels;
    st.frequent = out.size();
    st.host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return GVA_OK;
}

}  // namespace gva
