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
#include "gva_grow.h"

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
        std::vector<int> rcs(nthreads, GVA_OK);
        std::vector<std::string> msgs(nthreads);
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nthreads; ++t)
            pool.emplace_back([&, t]() {
                uint32_t ql[GVA_MAX_QUERY_VERTICES], sdl[3 * kMaxPatEdges];
                for (size_t i = b0 + t; i < b1; i += nthreads) {
                    // the plan of the candidate's query text, built from the pattern
                    const Pattern& c = cands[i];
                    for (uint32_t v = 0; v < c.n; ++v) ql[v] = labels[c.vl[v]];
                    for (uint32_t e = 0; e < c.ne; ++e) {
                        sdl[3 * e] = c.edges[e].u;
                        sdl[3 * e + 1] = c.edges[e].v;
                        sdl[3 * e + 2] = c.edges[e].el;
                    }
                    Plan plan;
                    int r = plan_from_query(c.n, ql, sdl, c.ne, GVA_MODE_DV, plan);
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
            p->rc = prepare_batch(db, cur, s, budget, true, false, profile, p->pb, true);  // ordered by step keys
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
    WedgeTab wedges;
    for (uint32_t k = 1; k < max_edges && !level.empty(); ++k) {
        if (cancel && *cancel) return fail(GVA_ERR_CANCELLED, "cancelled");
        GrowStats gt;
        std::vector<Pattern> next;
        if (k == 2 && WedgeTab::fits(L, P)) wedges.build(level, L, P);  // `level` holds the 2-edge patterns
        grow_level(level, level_codes, freq, L, P, width, max_edges, nthreads, wedges.bits.empty() ? nullptr : &wedges,
                   next, gt);
        st.pruned += gt.pruned;
        st.gen_ms += gt.gen_ms;
        st.merge_ms += gt.merge_ms;
        auto t_eval = std::chrono::steady_clock::now();
        rc = evaluate(next, sup, emb);
        if (rc) return rc;
        st.eval_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_eval).count();
        // the frequent ones: codes and query texts on the worker threads,
        // then filed in candidate order
        std::vector<uint32_t> fi;
        for (size_t i = 0; i < next.size(); ++i)
            if (sup[i] >= min_support) fi.push_back((uint32_t)i);
        std::vector<std::string> texts(fi.size());
        std::vector<std::vector<uint8_t>> code_arena(nthreads);
        std::vector<uint32_t> code_at(fi.size()), code_len(fi.size());
        std::vector<uint8_t> code_thread(fi.size());
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nthreads; ++t)
            pool.emplace_back([&, t]() {
                CodeBuf cb;
                for (size_t j = t; j < fi.size(); j += nthreads) {
                    canonical(next[fi[j]], width, cb);
                    code_at[j] = (uint32_t)code_arena[t].size();
                    code_len[j] = cb.len;
                    code_thread[j] = (uint8_t)t;
                    code_arena[t].insert(code_arena[t].end(), cb.b, cb.b + cb.len);
                    texts[j] = query_text(next[fi[j]], labels);
                }
            });
        for (auto& th : pool) th.join();
        level.clear();
        level_codes = CodeSet();
        for (size_t j = 0; j < fi.size(); ++j) {
            const uint32_t i = fi[j];
            level.push_back(next[i]);
            const uint8_t* code = code_arena[code_thread[j]].data() + code_at[j];
            level_codes.insert(code, code_len[j], code_hash(code, code_len[j]));
            out.push_back({std::move(texts[j]), k + 1, sup[i], emb[i]});
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
