// Brute-force frequent-pattern miner for graph databases (test oracle).
//
// The same definition as tests/brute_miner.py, in C++ so that it finishes on
// the 1,000-graph database in seconds: in every graph, every connected edge
// subset of up to K edges becomes a pattern (vertex labels, edge labels),
// canonicalised by trying every vertex permutation (smallest code of labels
// in position order followed by the upper triangle of edge labels, 0 = no
// edge); a pattern's support is the number of graphs holding it.  It shares
// no code with the product's pattern growth or canonical codes.
//
//   brute_mine <input> <max_edges> <min_support>
//
// input (text): "V E G", V vertex labels (ids 1..V), E lines "src dst elabel",
// G + 1 graph boundaries (graph g owns ids [first[g], first[g+1])).
// output: one line per frequent pattern: "support n code..." where code is
// the n labels then the n(n-1)/2 edge labels, as in brute_miner.canon.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <map>
#include <set>
#include <unordered_set>
#include <vector>

struct Edge {
    uint32_t a, b, l;
};

static std::vector<uint32_t> canon(const std::vector<uint32_t>& vl, const std::vector<Edge>& es) {
    const int n = (int)vl.size();
    std::vector<uint32_t> adj((size_t)n * n, 0);
    for (const Edge& e : es) adj[e.a * n + e.b] = adj[e.b * n + e.a] = e.l;
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    std::vector<uint32_t> best, code(n + n * (n - 1) / 2);
    do {
        size_t k = 0;
        for (int i = 0; i < n; ++i) code[k++] = vl[perm[i]];
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) code[k++] = adj[perm[i] * n + perm[j]];
        if (best.empty() || code < best) best = code;
    } while (std::next_permutation(perm.begin(), perm.end()));
    best.insert(best.begin(), (uint32_t)n);
    return best;
}

int main(int argc, char** argv) {
    if (argc != 4) {
        fprintf(stderr, "usage: brute_mine <input> <max_edges> <min_support>\n");
        return 2;
    }
    FILE* f = fopen(argv[1], "r");
    if (!f) return 2;
    const int K = atoi(argv[2]);
    const unsigned minsup = (unsigned)atoi(argv[3]);
    unsigned V, E, G;
    if (fscanf(f, "%u %u %u", &V, &E, &G) != 3) return 2;
    std::vector<uint32_t> vlabel(V + 1, 0);
    for (unsigned i = 1; i <= V; ++i)
        if (fscanf(f, "%u", &vlabel[i]) != 1) return 2;
    std::vector<Edge> edges(E);
    for (auto& e : edges)
        if (fscanf(f, "%u %u %u", &e.a, &e.b, &e.l) != 3) return 2;
    std::vector<long long> first(G + 1);
    for (auto& x : first)
        if (fscanf(f, "%lld", &x) != 1) return 2;
    fclose(f);
    // edges of each graph, in input order
    std::vector<std::vector<Edge>> by_graph(G);
    for (const Edge& e : edges) {
        const long long g = std::upper_bound(first.begin(), first.end(), (long long)e.a) - first.begin() - 1;
        if (g >= 0 && g < (long long)G) by_graph[g].push_back(e);
    }
    std::map<std::vector<uint32_t>, unsigned> support;
    for (unsigned g = 0; g < G; ++g) {
        const std::vector<Edge>& ge = by_graph[g];
        if (ge.size() > 64) {
            fprintf(stderr, "graph %u has more than 64 edges\n", g);
            return 2;
        }
        std::map<uint32_t, std::vector<int>> inc;
        for (int i = 0; i < (int)ge.size(); ++i) {
            inc[ge[i].a].push_back(i);
            inc[ge[i].b].push_back(i);
        }
        std::set<std::vector<uint32_t>> found;
        std::unordered_set<uint64_t> seen;
        std::vector<uint64_t> frontier;
        for (int i = 0; i < (int)ge.size(); ++i) frontier.push_back(1ull << i);
        for (int k = 1; k <= K; ++k) {
            for (uint64_t m : frontier) {
                std::vector<uint32_t> vs;
                for (int i = 0; i < (int)ge.size(); ++i)
                    if (m >> i & 1) {
                        vs.push_back(ge[i].a);
                        vs.push_back(ge[i].b);
                    }
                std::sort(vs.begin(), vs.end());
                vs.erase(std::unique(vs.begin(), vs.end()), vs.end());
                std::vector<uint32_t> labels(vs.size());
                for (size_t j = 0; j < vs.size(); ++j) labels[j] = vlabel[vs[j]];
                std::vector<Edge> pe;
                for (int i = 0; i < (int)ge.size(); ++i)
                    if (m >> i & 1) {
                        const uint32_t a = (uint32_t)(std::lower_bound(vs.begin(), vs.end(), ge[i].a) - vs.begin());
                        const uint32_t b = (uint32_t)(std::lower_bound(vs.begin(), vs.end(), ge[i].b) - vs.begin());
                        pe.push_back({a, b, ge[i].l});
                    }
                found.insert(canon(labels, pe));
            }
            if (k == K) break;
            std::vector<uint64_t> next;
            for (uint64_t m : frontier) {
                std::set<uint32_t> vs;
                for (int i = 0; i < (int)ge.size(); ++i)
                    if (m >> i & 1) {
                        vs.insert(ge[i].a);
                        vs.insert(ge[i].b);
                    }
                for (uint32_t v : vs)
                    for (int i : inc[v]) {
                        if (m >> i & 1) continue;
                        const uint64_t nm = m | (1ull << i);
                        if (seen.insert(nm).second) next.push_back(nm);
                    }
            }
            frontier.swap(next);
        }
        for (const auto& c : found) ++support[c];
    }
    for (const auto& kv : support) {
        if (kv.second < minsup) continue;
        printf("%u", kv.second);
        for (uint32_t x : kv.first) printf(" %u", x);
        printf("\n");
    }
    return 0;
}
