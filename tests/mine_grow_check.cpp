// Test driver (CPU only): one mining run's candidate levels from grow_level,
// the miner's level step, against a brute-force generator that shares no code
// with it.  Supports are a seeded anti-monotone stand-in (a product of per
// edge-type weights, degree and cycle factors), so the frequent sets have the
// downward closure real supports have.
//
// Brute force, per level k -> k + 1: every frequent k-edge pattern plus every
// edge (between two of its vertices, or to a new vertex of any label) of a
// frequent edge type; kept when every connected sub-pattern with one edge
// less is frequent.  Patterns are compared by a canonical code taken as the
// minimum over ALL vertex orders.  grow_level must return exactly that set,
// each pattern once, in its own canonical vertex order.  Then the miner's
// whole host level loop (mine_levels: level 1, frequent edge types, wedge
// table, growth, filing of frequent patterns as query texts) runs with the
// same supports as its evaluator and must evaluate exactly the brute-force
// candidates of every level and return exactly its frequent patterns, with
// their supports, over the original labels.
//
// usage: mine_grow_check L P max_edges seed threshold threads
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <random>
#include <set>

#include "../geneva_b200/csrc/gva_grow.h"

using namespace gva;

namespace {

using Code = std::vector<uint32_t>;

// minimum over all vertex orders of (n, labels, upper-triangle edge labels)
Code brute_code(const Pattern& p) {
    std::vector<uint32_t> adj(p.n * p.n, 0), ord(p.n);
    for (uint32_t e = 0; e < p.ne; ++e)
        adj[p.edges[e].u * p.n + p.edges[e].v] = adj[p.edges[e].v * p.n + p.edges[e].u] = p.edges[e].el;
    for (uint32_t i = 0; i < p.n; ++i) ord[i] = i;
    Code best;
    do {
        Code c;
        c.push_back(p.n);
        for (uint32_t i = 0; i < p.n; ++i) c.push_back(p.vl[ord[i]]);
        for (uint32_t i = 0; i < p.n; ++i)
            for (uint32_t j = i + 1; j < p.n; ++j) c.push_back(adj[ord[i] * p.n + ord[j]]);
        if (best.empty() || c < best) best = c;
    } while (std::next_permutation(ord.begin(), ord.end()));
    return best;
}

bool connected(const Pattern& p) {
    if (p.n == 0) return false;
    std::vector<int> seen(p.n, 0);
    std::vector<uint32_t> stack{0};
    seen[0] = 1;
    while (!stack.empty()) {
        uint32_t v = stack.back();
        stack.pop_back();
        for (uint32_t e = 0; e < p.ne; ++e) {
            uint32_t a = p.edges[e].u, b = p.edges[e].v, w = a == v ? b : (b == v ? a : kNone);
            if (w != kNone && !seen[w]) seen[w] = 1, stack.push_back(w);
        }
    }
    for (uint32_t v = 0; v < p.n; ++v)
        if (!seen[v]) return false;
    return true;
}

// p without edge `skip`, vertices left without edges dropped
Pattern without(const Pattern& p, uint32_t skip) {
    std::vector<uint32_t> deg(p.n, 0), map(p.n, kNone);
    for (uint32_t e = 0; e < p.ne; ++e)
        if (e != skip) deg[p.edges[e].u]++, deg[p.edges[e].v]++;
    Pattern q;
    for (uint32_t v = 0; v < p.n; ++v)
        if (deg[v]) map[v] = q.n, q.vl[q.n++] = p.vl[v];
    for (uint32_t e = 0; e < p.ne; ++e)
        if (e != skip) q.add_edge(map[p.edges[e].u], map[p.edges[e].v], p.edges[e].el);
    return q;
}

}  // namespace

// Canonical codes of large symmetric patterns (stars and cliques beyond what
// the brute force can enumerate, a double star) must not depend on the
// vertex numbering.  Twins make stars and cliques fast; equivalent vertices
// that are not twins (the two leaf sets of a double star) are still searched
// over all their arrangements.
int symmetric_check(std::mt19937& rng) {
    auto shuffled = [&](const Pattern& p) {
        uint32_t perm[GVA_MAX_QUERY_VERTICES];
        for (uint32_t i = 0; i < p.n; ++i) perm[i] = i;
        std::shuffle(perm, perm + p.n, rng);
        Pattern q;
        q.n = p.n;
        for (uint32_t v = 0; v < p.n; ++v) q.vl[perm[v]] = p.vl[v];
        for (uint32_t e = 0; e < p.ne; ++e) q.add_edge(perm[p.edges[e].u], perm[p.edges[e].v], p.edges[e].el);
        return q;
    };
    std::vector<Pattern> pats;
    for (uint32_t k : {8u, 16u, 24u, 31u}) {  // stars, one leaf label or two
        for (uint32_t two = 0; two < 2; ++two) {
            Pattern p;
            p.n = k + 1;
            p.vl[0] = 0;
            for (uint32_t v = 1; v <= k; ++v) p.vl[v] = two ? v % 2 : 0, p.add_edge(0, v, 1);
            pats.push_back(p);
        }
    }
    for (uint32_t k : {6u, 8u}) {  // cliques (k(k-1)/2 <= 31 edges)
        Pattern p;
        p.n = k;
        for (uint32_t v = 0; v < k; ++v) p.vl[v] = 0;
        for (uint32_t a = 0; a < k; ++a)
            for (uint32_t b = a + 1; b < k; ++b) p.add_edge(a, b, 1);
        pats.push_back(p);
    }
    {  // double star: two centres, 6 equal leaves each (leaves of different
       // centres share a cell but are not twins: C(12, 6) arrangements)
        Pattern p;
        p.n = 14;
        for (uint32_t v = 0; v < 14; ++v) p.vl[v] = 0;
        p.add_edge(0, 1, 2);
        for (uint32_t v = 2; v < 14; ++v) p.add_edge(v < 8 ? 0 : 1, v, 1);
        pats.push_back(p);
    }
    CodeBuf a, b;
    for (const Pattern& p : pats) {
        canonical(p, 1, a);
        for (int r = 0; r < 5; ++r) {
            canonical(shuffled(p), 1, b);
            if (a.len != b.len || std::memcmp(a.b, b.b, a.len) != 0) {
                printf("symmetric pattern of %u vertices: code depends on the numbering\n", p.n);
                return 1;
            }
        }
    }
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 7) return 2;
    const uint32_t L = atoi(argv[1]), P = atoi(argv[2]), max_edges = atoi(argv[3]);
    const uint32_t seed = atoi(argv[4]);
    const double thr = atof(argv[5]);
    const unsigned nthreads = atoi(argv[6]);
    {
        std::mt19937 srng(seed + 1000);  // its own stream: the supports below stay the same
        if (symmetric_check(srng)) return 1;
    }
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> uni(0.3, 1.0);
    std::vector<double> w((size_t)L * L * (P + 1));
    for (uint32_t a = 0; a < L; ++a)
        for (uint32_t b = a; b < L; ++b)
            for (uint32_t el = 1; el <= P; ++el)
                w[((size_t)a * L + b) * (P + 1) + el] = w[((size_t)b * L + a) * (P + 1) + el] = uni(rng);
    auto support = [&](const Pattern& p) {
        double v = 1.0;
        std::vector<uint32_t> deg(p.n, 0);
        for (uint32_t e = 0; e < p.ne; ++e) {
            v *= w[((size_t)p.vl[p.edges[e].u] * L + p.vl[p.edges[e].v]) * (P + 1) + p.edges[e].el];
            deg[p.edges[e].u]++, deg[p.edges[e].v]++;
        }
        for (uint32_t d : deg) v *= d <= 2 ? 1.0 : 0.8;
        for (int c = (int)p.ne - (int)p.n + 1; c > 0; --c) v *= 0.7;
        return v;
    };
    // supports as the miner sees them: integers, frequent when >= minsup
    auto isup = [&](const Pattern& p) { return (uint32_t)(support(p) * 1e6); };
    const uint32_t minsup = (uint32_t)(thr * 1e6);
    const uint32_t width = (L <= 256 && P <= 255) ? 1 : (L <= 65536 ? 2 : 4);
    std::vector<char> freq_tab((size_t)L * L * (P + 1), 0);
    auto freq = [&](uint32_t a, uint32_t el, uint32_t b) { return freq_tab[((size_t)a * L + b) * (P + 1) + el] != 0; };
    std::vector<Pattern> level;
    CodeSet level_codes;
    CodeBuf cb;
    std::set<Code> level_brute;
    for (uint32_t a = 0; a < L; ++a)
        for (uint32_t b = a; b < L; ++b)
            for (uint32_t el = 1; el <= P; ++el) {
                Pattern p;
                p.n = 2, p.vl[0] = a, p.vl[1] = b;
                p.add_edge(0, 1, el);
                if (isup(p) < minsup) continue;
                freq_tab[((size_t)a * L + b) * (P + 1) + el] = freq_tab[((size_t)b * L + a) * (P + 1) + el] = 1;
                uint32_t ord[GVA_MAX_QUERY_VERTICES];
                canonical(p, width, cb, ord);
                level.push_back(relabel(p, ord));
                level_codes.insert(cb.b, cb.len, code_hash(cb.b, cb.len));
                level_brute.insert(brute_code(p));
            }
    size_t total = 0;
    std::vector<std::set<Code>> brute_cands(1), brute_freq{level_brute};  // per level (index = edges - 1)
    WedgeTab wedges;
    for (uint32_t k = 1; k < max_edges && !level.empty(); ++k) {
        // brute force
        std::set<Code> want;
        for (const Pattern& p : level) {
            std::vector<Pattern> ext;
            for (uint32_t u = 0; u < p.n; ++u) {
                for (uint32_t v = u + 1; v < p.n; ++v) {
                    if (p.el(u, v)) continue;
                    for (uint32_t el = 1; el <= P; ++el)
                        if (freq(p.vl[u], el, p.vl[v])) {
                            Pattern c = p;
                            c.add_edge(u, v, el);
                            ext.push_back(c);
                        }
                }
                if (p.n + 1 > max_edges + 1) continue;
                for (uint32_t el = 1; el <= P; ++el)
                    for (uint32_t l = 0; l < L; ++l)
                        if (freq(p.vl[u], el, l)) {
                            Pattern c = p;
                            c.vl[c.n] = l;
                            c.add_edge(u, c.n, el);
                            c.n += 1;
                            ext.push_back(c);
                        }
            }
            for (const Pattern& c : ext) {
                bool ok = true;
                for (uint32_t e = 0; e < c.ne && ok; ++e) {
                    Pattern s = without(c, e);
                    if (s.n + 1 < c.n || !connected(s)) continue;  // two vertices lost or split
                    ok = level_brute.count(brute_code(s)) != 0;
                }
                if (ok) want.insert(brute_code(c));
            }
        }
        // the miner's level step, as the miner calls it
        if (k == 2 && WedgeTab::fits(L, P)) wedges.build(level, L, P);
        GrowStats gt;
        std::vector<Pattern> next;
        grow_level(level, level_codes, freq, L, P, width, max_edges, nthreads, wedges.bits.empty() ? nullptr : &wedges,
                   next, gt);
        std::set<Code> got;
        for (const Pattern& c : next) {
            if (!got.insert(brute_code(c)).second) {
                printf("level %u: a candidate appears twice\n", k + 1);
                return 1;
            }
            uint32_t ord[GVA_MAX_QUERY_VERTICES];
            canonical(c, width, cb, ord);
            for (uint32_t i = 0; i < c.n; ++i)
                if (ord[i] != i) {
                    printf("level %u: a candidate is not in canonical vertex order\n", k + 1);
                    return 1;
                }
        }
        brute_cands.push_back(want);
        if (got != want) {
            size_t miss = 0, extra = 0;
            for (auto& c : want) miss += !got.count(c);
            for (auto& c : got) extra += !want.count(c);
            printf("level %u: %zu candidates, brute force %zu: %zu missing, %zu extra\n", k + 1, got.size(), want.size(),
                   miss, extra);
            return 1;
        }
        total += next.size();
        // frequent ones become the next level
        level.clear();
        level_codes = CodeSet();
        level_brute.clear();
        for (const Pattern& c : next) {
            if (isup(c) < minsup) continue;
            level.push_back(c);
            canonical(c, width, cb);
            level_codes.insert(cb.b, cb.len, code_hash(cb.b, cb.len));
            level_brute.insert(brute_code(c));
        }
        brute_freq.push_back(level_brute);
        printf("level %u: %zu candidates (%llu pruned), %zu frequent\n", k + 1, next.size(),
               (unsigned long long)gt.pruned, level.size());
    }

    // the miner's whole host level loop (mine_levels) with the same supports:
    // every level's evaluated candidates and the frequent patterns it returns
    // (query texts over original labels) against the brute force
    std::vector<uint32_t> labels(L);
    for (uint32_t l = 0; l < L; ++l) labels[l] = 100 + 3 * l;
    std::vector<char> has_part(P + 1, 1);
    std::vector<std::set<Code>> evaluated;
    auto evaluate = [&](const std::vector<Pattern>& cands, std::vector<uint32_t>& sup, std::vector<uint64_t>& emb) {
        std::set<Code> s;
        sup.assign(cands.size(), 0);
        emb.assign(cands.size(), 0);
        for (size_t i = 0; i < cands.size(); ++i) {
            s.insert(brute_code(cands[i]));
            sup[i] = isup(cands[i]);
            emb[i] = cands[i].ne * 1000ull + cands[i].n;
        }
        evaluated.push_back(s);
        return 0;
    };
    std::vector<MinedPattern> out;
    LevelStats ls;
    if (mine_levels(L, P, has_part, labels, max_edges, minsup, nthreads, nullptr, evaluate, out, ls)) {
        printf("mine_levels failed\n");
        return 1;
    }
    if (evaluated.empty() || evaluated[0].size() != (size_t)L * (L + 1) / 2 * P) {
        printf("level 1: wrong edge types evaluated\n");
        return 1;
    }
    if (evaluated.size() != brute_freq.size() && !(evaluated.size() == brute_freq.size() - 1 && brute_freq.back().empty())) {
        printf("mine_levels evaluated %zu levels, brute force %zu\n", evaluated.size(), brute_freq.size());
        return 1;
    }
    for (size_t lv = 1; lv < evaluated.size(); ++lv)
        if (evaluated[lv] != brute_cands[lv]) {
            printf("mine_levels level %zu: evaluated candidates differ from the brute force\n", lv + 1);
            return 1;
        }
    std::vector<std::set<Code>> mined(brute_freq.size());
    for (const MinedPattern& m : out) {
        Pattern p;
        const char* c = m.text.c_str();
        while (*c) {
            unsigned a, b, l;
            int used = 0;
            if (sscanf(c, "v %u %u\n%n", &a, &l, &used) == 2 && used) {
                if ((l - 100) % 3 || (l - 100) / 3 >= L || a != p.n) {
                    printf("bad vertex line in %s\n", m.text.c_str());
                    return 1;
                }
                p.vl[p.n++] = (l - 100) / 3;
            } else if (sscanf(c, "e %u %u %u\n%n", &a, &b, &l, &used) == 3 && used) {
                p.add_edge(a, b, l);
            } else {
                printf("unparsable pattern text %s\n", m.text.c_str());
                return 1;
            }
            c += used;
        }
        if (m.edges != p.ne || m.edges == 0 || m.edges > mined.size() || m.support != isup(p) ||
            m.embeddings != p.ne * 1000ull + p.n || !connected(p)) {
            printf("mined pattern with wrong edges/support/embeddings: %s\n", m.text.c_str());
            return 1;
        }
        if (!mined[m.edges - 1].insert(brute_code(p)).second) {
            printf("pattern mined twice: %s\n", m.text.c_str());
            return 1;
        }
    }
    for (size_t lv = 0; lv < mined.size(); ++lv)
        if (mined[lv] != brute_freq[lv]) {
            printf("mine_levels level %zu: %zu frequent patterns, brute force %zu\n", lv + 1, mined[lv].size(),
                   brute_freq[lv].size());
            return 1;
        }
    printf("ok %zu candidates, %zu frequent\n", total, out.size());
    return 0;
}
