// Test driver (CPU only): the host database build (graph_from_edges) and the
// init-phase seed groups (seed_groups) against their definitions on seeded
// random graphs with repeated edges, self-loop-free pairs in both
// directions, edge-label gaps and hub vertices:
//   * per edge label, vertex v's neighbours with dense label l are
//     adj[off[v*L + l] .. off[v*L + l + 1]), ascending ids, no repeats, and
//     they are exactly the distinct neighbours of v over edges of that label;
//   * offsets never decrease and end at the list length;
//   * seed_verts holds each label's vertices in ascending id order, and
//     seed_by_degree the same vertices by total degree (largest first), ties
//     by id.
//
// usage: graph_build_check graphs seed max_vertices
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <set>
#include <vector>

#include "../geneva_b200/csrc/gva_internal.h"

using namespace gva;

int main(int argc, char** argv) {
    if (argc < 4) return 2;
    const int graphs = atoi(argv[1]);
    std::mt19937 rng(atoi(argv[2]));
    const uint32_t maxv = (uint32_t)atoi(argv[3]);
    for (int t = 0; t < graphs; ++t) {
        const uint32_t n = 1 + rng() % maxv, L = 1 + rng() % 12, P = 1 + rng() % 4;
        std::vector<uint32_t> vl(n + 1), s, d, e;
        for (uint32_t v = 1; v <= n; ++v) vl[v] = 10 + 3 * (rng() % L);
        const uint64_t m = rng() % (4ull * n + 1);
        const uint32_t hub = 1 + rng() % n;
        for (uint64_t i = 0; i < m; ++i) {
            uint32_t a = 1 + rng() % n, b = (rng() % 5 == 0) ? hub : 1 + rng() % n;
            if (a == b) continue;
            const uint32_t l = (rng() % 4 == 0) ? P : 1 + rng() % P;  // labels below P may be missing
            s.push_back(a), d.push_back(b), e.push_back(l);
            if (rng() % 6 == 0) s.push_back(b), d.push_back(a), e.push_back(l);  // repeated, reversed
        }
        HostGraph g;
        if (graph_from_edges(vl.data(), n, s.data(), d.data(), e.data(), s.size(), g)) {
            printf("graph %d: build failed: %s\n", t, last_error_cstr());
            return 1;
        }
        const uint32_t Lg = g.num_labels();
        // expected neighbour sets per (label, vertex)
        uint32_t Pmax = 0;
        for (uint32_t x : e) Pmax = std::max(Pmax, x);
        std::vector<std::vector<std::set<uint32_t>>> want(Pmax, std::vector<std::set<uint32_t>>(n + 1));
        for (size_t i = 0; i < s.size(); ++i) want[e[i] - 1][s[i]].insert(d[i]), want[e[i] - 1][d[i]].insert(s[i]);
        if (Pmax && g.parts.size() != Pmax) {
            printf("graph %d: %zu partitions, expected %u\n", t, g.parts.size(), Pmax);
            return 1;
        }
        std::vector<uint32_t> deg(n + 1, 0);
        for (uint32_t p = 0; p < Pmax; ++p) {
            const HostPartition& hp = g.parts[p];
            const uint64_t entries = (uint64_t)(n + 1) * Lg + 1;
            if (hp.off.size() != entries || hp.off[0] != 0 || hp.off[entries - 1] != hp.adj.size()) {
                printf("graph %d label %u: bad offset table\n", t, p + 1);
                return 1;
            }
            for (uint64_t i = 1; i < entries; ++i)
                if (hp.off[i] < hp.off[i - 1]) {
                    printf("graph %d label %u: offsets decrease\n", t, p + 1);
                    return 1;
                }
            for (uint32_t v = 0; v <= n; ++v) {
                std::vector<uint32_t> got;
                for (uint32_t l = 0; l < Lg; ++l)
                    for (uint32_t k = hp.off[(uint64_t)v * Lg + l]; k < hp.off[(uint64_t)v * Lg + l + 1]; ++k) {
                        const uint32_t u = hp.adj[k];
                        if (u == 0 || u > n || g.dlabel[u] != l || (!got.empty() && g.dlabel[got.back()] == l && got.back() >= u)) {
                            printf("graph %d label %u vertex %u: list out of order\n", t, p + 1, v);
                            return 1;
                        }
                        got.push_back(u);
                    }
                std::vector<uint32_t> w(want[p][v].begin(), want[p][v].end());
                std::sort(got.begin(), got.end());
                if (got != w) {
                    printf("graph %d label %u vertex %u: %zu neighbours, expected %zu\n", t, p + 1, v, got.size(), w.size());
                    return 1;
                }
                deg[v] += (uint32_t)got.size();
            }
        }
        std::vector<uint32_t> so, sv, sd;
        seed_groups(g, so, sv, sd);
        if (so.size() != Lg + 1 || so[Lg] != n || sv.size() != n || sd.size() != n) {
            printf("graph %d: bad seed groups\n", t);
            return 1;
        }
        for (uint32_t l = 0; l < Lg; ++l) {
            for (uint32_t i = so[l]; i < so[l + 1]; ++i) {
                if (g.dlabel[sv[i]] != l || (i > so[l] && sv[i - 1] >= sv[i])) {
                    printf("graph %d: seed group %u not by ascending id\n", t, l);
                    return 1;
                }
                if (i > so[l] && (deg[sd[i - 1]] < deg[sd[i]] || (deg[sd[i - 1]] == deg[sd[i]] && sd[i - 1] >= sd[i]))) {
                    printf("graph %d: seed group %u not by degree\n", t, l);
                    return 1;
                }
            }
            std::vector<uint32_t> a(sv.begin() + so[l], sv.begin() + so[l + 1]), b(sd.begin() + so[l], sd.begin() + so[l + 1]);
            std::sort(b.begin(), b.end());
            if (a != b) {
                printf("graph %d: seed group %u by degree is not the same vertices\n", t, l);
                return 1;
            }
        }
    }
    printf("ok %d graphs\n", graphs);
    return 0;
}
