// Test driver (host only, no device needed): the batched engine's step trie
// (BatchSession::submit) on seeded random plans.  A session that is never
// initialised touches no device memory while plans are submitted.
//
// Checks, for the plans in the miner's order (sorted by step keys) built with
// and without the presorted shortcut, and for the same plans shuffled:
//   * every plan's root-to-terminal path reproduces its own steps (by the
//     step key bytes that decide a step's output) and the plan is on its
//     terminal's list exactly once;
//   * the presorted trie has as many nodes as the indexed one, and the
//     shuffled (indexed) trie as many as the sorted one: shared prefixes are
//     matched once whatever the order.
//
// usage: batch_trie_check plans seed
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../geneva_b200/csrc/gva_engine.cuh"
#include "../include/geneva.h"

using namespace gva;

namespace {

uint64_t fnv(const uint8_t* b, size_t n) {
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}

int check(BatchSession& ses, const std::vector<std::vector<Step>>& plans, const std::vector<int>& ids, const char* what) {
    uint8_t ka[512], kb[512];
    std::vector<int> listed(plans.size(), 0);
    for (size_t n = 0; n < ses.num_nodes(); ++n)
        for (int q = ses.node((int)n).first_term; q >= 0; q = ses.plan(q).next_term) {
            if (q < 0 || q >= (int)listed.size()) {
                printf("%s: bad plan id %d on a terminal list\n", what, q);
                return 1;
            }
            listed[q]++;
        }
    for (size_t q = 0; q < plans.size(); ++q) {
        if (listed[ids[q]] != 1) {
            printf("%s: plan %zu listed %d times\n", what, q, listed[ids[q]]);
            return 1;
        }
        int nd = ses.plan(ids[q]).terminal;
        for (size_t d = plans[q].size(); d-- > 0;) {
            if (nd < 0 || ses.node(nd).depth != (int)d) {
                printf("%s: plan %zu: path shorter than its steps\n", what, q);
                return 1;
            }
            const size_t la = step_key_bytes(ses.node_step(nd), ka), lb = step_key_bytes(plans[q][d], kb);
            if (la != lb || std::memcmp(ka, kb, la) != 0) {
                printf("%s: plan %zu: step %zu differs on its path\n", what, q, d);
                return 1;
            }
            nd = ses.node(nd).parent;
        }
        if (nd != -1) {
            printf("%s: plan %zu: path longer than its steps\n", what, q);
            return 1;
        }
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    const int nplans = atoi(argv[1]);
    std::mt19937_64 rng(atoi(argv[2]));
    // database: labels 1..3, partitions 1..2 (for lowering and seed groups)
    HostGraph g;
    {
        std::vector<uint32_t> vl(10), sv, dv, el;
        for (uint32_t v = 1; v <= 9; ++v) vl[v] = 1 + (v - 1) % 3;
        for (uint32_t v = 1; v <= 9; ++v)
            for (uint32_t u = v + 1; u <= 9; ++u) sv.push_back(v), dv.push_back(u), el.push_back(1 + (u + v) % 2);
        if (graph_from_edges(vl.data(), 9, sv.data(), dv.data(), el.data(), sv.size(), g)) return 2;
    }
    DevDB db;  // host fields only: the session reads the seed groups' sizes
    db.L = g.num_labels();
    db.seed_off.assign(db.L + 1, 0);
    for (uint32_t l = 0; l < db.L; ++l) db.seed_off[l + 1] = db.seed_off[l] + 3;
    // random small connected queries over few labels, so plans share prefixes
    std::vector<std::vector<Step>> plans;
    while ((int)plans.size() < nplans) {
        const uint32_t n = 2 + rng() % 5;
        std::string t;
        for (uint32_t v = 0; v < n; ++v) t += "v " + std::to_string(v) + " " + std::to_string(1 + rng() % 3) + "\n";
        for (uint32_t v = 1; v < n; ++v)
            t += "e " + std::to_string(rng() % v) + " " + std::to_string(v) + " " + std::to_string(1 + rng() % 2) + "\n";
        if (rng() % 3 == 0 && n > 2) t += "e 0 " + std::to_string(n - 1) + " 1\n";
        Plan p;
        std::vector<Step> st;
        if (plan_from_text(t, rng() % 4 ? GVA_MODE_DV : GVA_MODE_SV, p) || lower_plan(p, g, st, true)) continue;
        plans.push_back(st);
    }
    // the miner's order: by the hashes of the steps' key bytes, ties by index
    const size_t n = plans.size();
    std::vector<std::vector<uint64_t>> key(n);
    uint8_t kb[512];
    for (size_t i = 0; i < n; ++i)
        for (const Step& s : plans[i]) key[i].push_back(fnv(kb, step_key_bytes(s, kb)) | 1);
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return key[a] != key[b] ? key[a] < key[b] : a < b; });
    std::vector<std::vector<Step>> sorted(n), shuffled;
    for (size_t i = 0; i < n; ++i) sorted[i] = plans[order[i]];
    shuffled = sorted;
    std::shuffle(shuffled.begin(), shuffled.end(), rng);
    size_t nodes[3];
    const std::vector<std::vector<Step>>* input[3] = {&sorted, &sorted, &shuffled};
    const char* name[3] = {"sorted, indexed", "sorted, presorted", "shuffled, indexed"};
    for (int m = 0; m < 3; ++m) {
        BatchSession ses(db, nullptr, 1ull << 30, 0, false, false);
        std::vector<int> ids;
        if (ses.submit(*input[m], {}, &ids, m == 1)) {
            printf("%s: submit failed: %s\n", name[m], last_error_cstr());
            return 1;
        }
        if (ids.size() != n || check(ses, *input[m], ids, name[m])) return 1;
        nodes[m] = ses.num_nodes();
    }
    if (nodes[0] != nodes[1] || nodes[0] != nodes[2]) {
        printf("node counts differ: %zu %zu %zu\n", nodes[0], nodes[1], nodes[2]);
        return 1;
    }
    printf("ok %zu plans, %zu trie nodes\n", n, nodes[0]);
    return 0;
}
