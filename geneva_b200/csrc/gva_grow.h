// Pattern growth for level-wise mining, host only: labelled patterns,
// canonical codes, code sets, one level of candidate generation with its
// anti-monotone pruning (grow_level) and the level loop around it with the
// evaluator as a callback (mine_levels).  Shared by the miner (gva_mine.cpp,
// whose evaluator runs the batched matcher) and a CPU test that checks both
// against a brute-force miner.
#pragma once

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/geneva.h"
#include "gva_internal.h"
#include "gva_pool.h"

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
// tried, and twins (interchangeable by an automorphism) in one fixed order.
// Equal keys of non-equivalent vertices only enlarge a cell, which costs
// time, not correctness.  Values are written `width` bytes each (1 when
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
    // twins (same label, same edge label to every other vertex) can be
    // swapped by an automorphism, which leaves every code unchanged: orders
    // that differ only in how twins are placed give the same code, so cells
    // are permuted as multisets of twin classes, each class filled with its
    // vertices in ascending id (a star's k equal leaves: one order, not k!)
    uint32_t cls[GVA_MAX_QUERY_VERTICES];      // twin class at each position
    uint32_t members[GVA_MAX_QUERY_VERTICES];  // class c: members[mat[c] .. mat[c] + mcnt[c]), ascending id
    uint32_t mat[GVA_MAX_QUERY_VERTICES], mcnt[GVA_MAX_QUERY_VERTICES], ncls = 0;
    if (!trivial) {
        uint32_t vcls[GVA_MAX_QUERY_VERTICES], rep[GVA_MAX_QUERY_VERTICES];  // rep: a class's first vertex
        for (uint32_t c = 0; c < nc; ++c) {
            const uint32_t first = ncls;
            for (uint32_t i = cb[c]; i < ce[c]; ++i) {  // ascending id within the cell
                const uint32_t v = ord[i];
                uint32_t k = first;
                for (; k < ncls; ++k) {
                    const uint32_t u = rep[k];
                    bool twin = p.vl[u] == p.vl[v];
                    for (uint32_t w = 0; w < n && twin; ++w)
                        if (w != u && w != v) twin = adj[u][w] == adj[v][w];
                    if (twin) break;
                }
                if (k == ncls) {
                    rep[k] = v;
                    mcnt[k] = 0;
                    ++ncls;
                }
                vcls[i] = k;
            }
            // lay the cell's classes out contiguously, members in ascending id
            uint32_t at = cb[c];
            for (uint32_t k = first; k < ncls; ++k) {
                mat[k] = at;
                for (uint32_t i = cb[c]; i < ce[c]; ++i)
                    if (vcls[i] == k) members[at++] = ord[i], mcnt[k]++;
            }
            for (uint32_t k = first, i = cb[c]; k < ncls; ++k)
                for (uint32_t m = 0; m < mcnt[k]; ++m) cls[i++] = k;  // ascending: the first arrangement
        }
    }
    auto arrange = [&]() {  // ord from the class arrangement
        uint32_t used_of[GVA_MAX_QUERY_VERTICES];
        for (uint32_t k = 0; k < ncls; ++k) used_of[k] = 0;
        for (uint32_t i = 0; i < n; ++i) ord[i] = members[mat[cls[i]] + used_of[cls[i]]++];
    };
    if (!trivial) arrange();
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
            if (std::next_permutation(cls + cb[c], cls + ce[c])) break;
        if (c < 0) break;
        arrange();
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
    uint8_t next_edge;  // first edge whose removal is still to be checked
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

// std::sort on `nthreads` threads: sorted chunks merged pairwise.  With a
// total order (no two elements equivalent) the result is std::sort's.
template <typename It, typename Less>
void parallel_sort(It first, It last, Less less, unsigned nthreads) {
    const size_t n = (size_t)(last - first);
    if (nthreads <= 1 || n < (1u << 14)) {
        std::sort(first, last, less);
        return;
    }
    size_t chunks = 1;
    while (chunks * 2 <= nthreads && chunks < 64) chunks *= 2;
    std::vector<size_t> cut(chunks + 1);
    for (size_t c = 0; c <= chunks; ++c) cut[c] = n * c / chunks;
    pool_run((unsigned)chunks, [&](unsigned c) { std::sort(first + cut[c], first + cut[c + 1], less); });
    for (size_t width = 1; width < chunks; width *= 2) {
        const unsigned jobs = (unsigned)((chunks + 2 * width - 1) / (2 * width));
        pool_run(jobs, [&](unsigned m) {
            const size_t c = (size_t)m * 2 * width;
            if (c + width >= chunks) return;
            const size_t lo = cut[c], mid = cut[c + width], hi = cut[std::min(chunks, c + 2 * width)];
            std::inplace_merge(first + lo, first + mid, first + hi, less);
        });
    }
}

constexpr uint32_t kBuckets = 256;  // candidate partitions by code hash (fixed: output order is machine-independent)

struct GrowStats {
    uint64_t pruned = 0;
    double gen_ms = 0.0, merge_ms = 0.0;
};

// Order-free invariant of a pattern: the sum of a 64-bit mix of every edge's
// type (end labels unordered, edge label) and of every vertex label.
// Isomorphic patterns have equal sums, so a sub-pattern whose sum is not
// among the frequent patterns' sums is not frequent; the sum of a parent
// plus one edge minus another is found without building the sub-pattern.
inline uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}
inline uint64_t edge_inv(uint32_t a, uint32_t b, uint32_t el) {
    if (a > b) std::swap(a, b);
    return mix64((((uint64_t)a << 32) | b) ^ mix64(el + 0x51ed27ull));
}
inline uint64_t vertex_inv(uint32_t l) { return mix64(l ^ 0xa0761d6478bd642full); }
uint64_t pattern_inv(const Pattern& p) {
    uint64_t h = 0;
    for (uint32_t v = 0; v < p.n; ++v) h += vertex_inv(p.vl[v]);
    for (uint32_t e = 0; e < p.ne; ++e) h += edge_inv(p.vl[p.edges[e].u], p.vl[p.edges[e].v], p.edges[e].el);
    return h;
}

// Open-addressing set of 64-bit values (invariants of one level's patterns).
struct InvSet {
    std::vector<uint64_t> table;  // 0 = empty; a value 0 is stored as 1
    uint64_t mask = 0;
    void build(const std::vector<uint64_t>& vals) {
        size_t cap = 16;
        while (cap < 2 * vals.size() + 2) cap <<= 1;
        table.assign(cap, 0);
        mask = cap - 1;
        for (uint64_t v : vals) {
            v = v ? v : 1;
            size_t i = mix64(v) & mask;
            while (table[i] && table[i] != v) i = (i + 1) & mask;
            table[i] = v;
        }
    }
    bool contains(uint64_t v) const {
        v = v ? v : 1;
        for (size_t i = mix64(v) & mask;; i = (i + 1) & mask) {
            if (table[i] == v) return true;
            if (!table[i]) return false;
        }
    }
};

// Frequent wedges: 2-edge patterns a -el1- c -el2- b, filed under both end
// orders.  Every connected sub-pattern of a kept candidate is frequent, so an
// extension of a pattern with two or more edges whose new edge makes an
// infrequent wedge with an edge already there would be pruned: it is dropped
// before its canonical code is computed (same candidate set, less work).
struct WedgeTab {
    uint32_t L = 0, P = 0;
    std::vector<uint8_t> bits;
    static bool fits(uint32_t L, uint32_t P) {
        return (uint64_t)L * L * L * (P + 1) * (P + 1) <= (1ull << 26);
    }
    size_t idx(uint32_t a, uint32_t el1, uint32_t c, uint32_t el2, uint32_t b) const {
        return ((((size_t)c * L + a) * L + b) * (P + 1) + el1) * (P + 1) + el2;
    }
    bool has(uint32_t a, uint32_t el1, uint32_t c, uint32_t el2, uint32_t b) const {
        return bits[idx(a, el1, c, el2, b)] != 0;
    }
    // from the frequent 2-edge patterns
    void build(const std::vector<Pattern>& level2, uint32_t L_, uint32_t P_) {
        L = L_, P = P_;
        bits.assign((size_t)L * L * L * (P + 1) * (P + 1), 0);
        for (const Pattern& w : level2) {
            const PEdge& x = w.edges[0];
            const PEdge& y = w.edges[1];
            const uint32_t c = (x.u == y.u || x.u == y.v) ? x.u : x.v;  // shared vertex
            const uint32_t a = x.u == c ? x.v : x.u, b = y.u == c ? y.v : y.u;
            bits[idx(w.vl[a], x.el, w.vl[c], y.el, w.vl[b])] = 1;
            bits[idx(w.vl[b], y.el, w.vl[c], x.el, w.vl[a])] = 1;
        }
    }
};

// One mining level: every extension of `level` by one frequent edge type
// (freq(a, el, b)), deduplicated by canonical code and kept only when every
// connected sub-pattern with one edge less is in `level_codes`; survivors in
// canonical vertex order, ordered by code hash partition then code.
// `wedges` (patterns of two or more edges only, or null) drops extensions
// that make an infrequent wedge before their codes are computed.
template <typename Freq>
void grow_level(const std::vector<Pattern>& level, const CodeSet& level_codes, Freq freq, uint32_t L, uint32_t P,
                uint32_t width, uint32_t max_edges, unsigned nthreads, const WedgeTab* wedges,
                std::vector<Pattern>& next, GrowStats& gt) {
    // small levels on few threads: starting a thread costs more than a few patterns
    nthreads = std::max(1u, std::min<unsigned>(nthreads, (unsigned)((level.size() + 15) / 16)));
    auto t_gen = std::chrono::steady_clock::now();
    std::vector<uint64_t> pinv(level.size());
    for (size_t i = 0; i < level.size(); ++i) pinv[i] = pattern_inv(level[i]);
    InvSet level_inv;
    level_inv.build(pinv);
    // (1) each thread extends every nthreads-th pattern by one frequent
    // edge type, drops the extensions that fail the wedge check or the first
    // sub-pattern check, keeps those whose canonical code it has not seen yet
    // and files them by code hash into kBuckets partitions
    std::vector<CodeSet> seen(nthreads);
    std::vector<uint64_t> dropped(nthreads, 0);  // extensions dropped before their codes
    std::vector<std::vector<std::vector<Ext>>> exts(nthreads, std::vector<std::vector<Ext>>(kBuckets));
    pool_run(nthreads, [&](unsigned t) {
            CodeBuf cb;
            // per parent edge e: what removing it leaves, so that the
            // connectivity of (parent + x) - e is known without building it:
            // R_CONN connected; R_LEAF connected but for the leaf vertex
            // rm_w[e]; R_BRIDGE two parts with edges, rm_mask[e] one of them;
            // R_SINGLE the parent's only edge
            enum : uint8_t { R_CONN, R_LEAF, R_BRIDGE, R_SINGLE };
            uint8_t rm_kind[kMaxPatEdges], rm_w[kMaxPatEdges];
            uint32_t rm_mask[kMaxPatEdges];
            uint64_t rm_inv[kMaxPatEdges];  // parent invariant minus edge e
            uint64_t vinv[GVA_MAX_QUERY_VERTICES];
            uint8_t nb[GVA_MAX_QUERY_VERTICES][GVA_MAX_QUERY_VERTICES];  // neighbour vertices
            uint16_t nbl[GVA_MAX_QUERY_VERTICES][GVA_MAX_QUERY_VERTICES];  // their edge labels
            uint32_t deg[GVA_MAX_QUERY_VERTICES];
            // the new edge u -el- (vertex labelled lb) makes a frequent wedge
            // with every edge at u
            auto wedges_ok = [&](const Pattern& p, uint32_t u, uint32_t el, uint32_t lb) {
                for (uint32_t j = 0; j < deg[u]; ++j)
                    if (!wedges->has(p.vl[nb[u][j]], nbl[u][j], p.vl[u], el, lb)) return false;
                return true;
            };
            // parent p + extension x (x.v == 0xff: forward from x.u).  The
            // sub-patterns without one of p's edges are checked before the
            // extension's own code: by invariant each, then the first
            // connected one exactly (nearly every extension that gets pruned
            // fails one of these)
            auto consider = [&](uint32_t parent, const Pattern& p, const Ext& x) {
                const bool fwd = x.v == 0xff;
                const uint64_t xinv =
                    edge_inv(p.vl[x.u], fwd ? x.lab : p.vl[x.v], x.el) + (fwd ? vertex_inv(x.lab) : 0);
                uint32_t first = kNone, first_iso = kNone;
                for (uint32_t e = 0; e < p.ne; ++e) {
                    uint32_t iso = kNone;
                    switch (rm_kind[e]) {
                        case R_CONN:
                            break;
                        case R_LEAF:
                            if (fwd) {
                                if (x.u == rm_w[e]) continue;  // leaf + new vertex apart from the rest
                                iso = rm_w[e];
                            } else if (x.u != rm_w[e] && x.v != rm_w[e]) {
                                iso = rm_w[e];
                            }
                            break;
                        case R_BRIDGE:
                            if (fwd || ((rm_mask[e] >> x.u & 1) == (rm_mask[e] >> x.v & 1))) continue;
                            break;
                        default:  // R_SINGLE: only x is left; its other end is gone
                            iso = p.edges[e].u == x.u ? p.edges[e].v : p.edges[e].u;
                            break;
                    }
                    const uint64_t sinv = rm_inv[e] + xinv - (iso != kNone ? vinv[iso] : 0);
                    if (!level_inv.contains(sinv)) {
                        ++dropped[t];
                        return;
                    }
                    if (first == kNone) first = e, first_iso = iso;
                }
                const Pattern c = apply_ext(p, x);
                if (first != kNone) {
                    canonical(remove_edge(c, first, first_iso), width, cb);
                    if (!level_codes.contains(cb.b, cb.len, code_hash(cb.b, cb.len))) {
                        ++dropped[t];
                        return;
                    }
                }
                canonical(c, width, cb);
                const uint64_t h = code_hash(cb.b, cb.len);
                uint32_t off;
                if (!seen[t].insert(cb.b, cb.len, h, &off)) return;
                Ext r = x;
                r.hash = h;
                r.parent = parent;
                r.code_off = off;
                r.code_len = (uint16_t)cb.len;
                r.thread = (uint8_t)t;
                r.next_edge = (uint8_t)(first == kNone ? c.ne : first + 1);  // sub-patterns left to check
                exts[t][h % kBuckets].push_back(r);
            };
            for (size_t i = t; i < level.size(); i += nthreads) {
                const Pattern& p = level[i];
                for (uint32_t v = 0; v < p.n; ++v) deg[v] = 0, vinv[v] = vertex_inv(p.vl[v]);
                for (uint32_t e = 0; e < p.ne; ++e) {
                    const PEdge& pe = p.edges[e];
                    nb[pe.u][deg[pe.u]] = pe.v, nbl[pe.u][deg[pe.u]++] = pe.el;
                    nb[pe.v][deg[pe.v]] = pe.u, nbl[pe.v][deg[pe.v]++] = pe.el;
                }
                for (uint32_t e = 0; e < p.ne; ++e) {
                    const PEdge& pe = p.edges[e];
                    rm_inv[e] = pinv[i] - edge_inv(p.vl[pe.u], p.vl[pe.v], pe.el);
                    uint32_t iso;
                    if (p.ne == 1) {
                        rm_kind[e] = R_SINGLE;
                    } else if (connected_without(p, e, iso)) {
                        rm_kind[e] = iso == kNone ? R_CONN : R_LEAF;
                        rm_w[e] = (uint8_t)(iso == kNone ? 0 : iso);
                    } else {
                        // the part holding pe.u, by edges other than e
                        uint32_t seen_m = 1u << pe.u, frontier = seen_m;
                        while (frontier) {
                            uint32_t nxt = 0;
                            for (uint32_t f = 0; f < p.ne; ++f) {
                                if (f == e) continue;
                                if (frontier >> p.edges[f].u & 1) nxt |= 1u << p.edges[f].v;
                                if (frontier >> p.edges[f].v & 1) nxt |= 1u << p.edges[f].u;
                            }
                            frontier = nxt & ~seen_m;
                            seen_m |= nxt;
                        }
                        rm_kind[e] = R_BRIDGE;
                        rm_mask[e] = seen_m;
                    }
                }
                Ext x{};
                for (uint32_t u = 0; u < p.n; ++u) {
                    x.u = (uint8_t)u;
                    for (uint32_t v = u + 1; v < p.n; ++v) {  // backward edges
                        if (p.el(u, v)) continue;
                        x.v = (uint8_t)v;
                        for (uint32_t el = 1; el <= P; ++el) {
                            if (!freq(p.vl[u], el, p.vl[v])) continue;
                            if (wedges && !(wedges_ok(p, u, el, p.vl[v]) && wedges_ok(p, v, el, p.vl[u]))) {
                                ++dropped[t];
                                continue;
                            }
                            x.el = (uint16_t)el;
                            consider((uint32_t)i, p, x);
                        }
                    }
                    if (p.n + 1 > max_edges + 1 || p.n + 1 > GVA_MAX_QUERY_VERTICES) continue;
                    x.v = 0xff;
                    for (uint32_t el = 1; el <= P; ++el) {  // forward edges
                        x.el = (uint16_t)el;
                        for (uint32_t l = 0; l < L; ++l) {
                            if (!freq(p.vl[u], el, l)) continue;
                            if (wedges && !wedges_ok(p, u, el, l)) {
                                ++dropped[t];
                                continue;
                            }
                            x.lab = l;
                            consider((uint32_t)i, p, x);
                        }
                    }
                }
            }
        });
    // (2) each partition is deduplicated across threads (sorted by code, so
    // the level's order depends on the codes only), and each distinct
    // candidate is kept only if every connected k-edge sub-pattern other
    // than its parent is frequent (anti-monotone support); survivors are
    // stored in canonical vertex order
    auto t_merge = std::chrono::steady_clock::now();
    std::vector<std::vector<Pattern>> buckets(kBuckets);
    std::vector<uint64_t> pruned(kBuckets, 0);
    std::atomic<uint32_t> next_bucket{0};
    pool_run(nthreads, [&](unsigned) {
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
                    for (uint32_t e = x.next_edge; e + 1 < c.ne && ok; ++e) {  // edge c.ne - 1 is the parent's extension
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
    for (unsigned t = 0; t < nthreads; ++t) gt.pruned += dropped[t];
    std::vector<size_t> at(kBuckets + 1, 0);
    for (uint32_t b = 0; b < kBuckets; ++b) {
        gt.pruned += pruned[b];
        at[b + 1] = at[b] + buckets[b].size();
    }
    next.clear();
    next.resize(at[kBuckets]);
    pool_run(nthreads, [&](unsigned t) {
        for (uint32_t b = t; b < kBuckets; b += nthreads) {
            std::copy(buckets[b].begin(), buckets[b].end(), next.begin() + at[b]);
            std::vector<Pattern>().swap(buckets[b]);
        }
    });
    exts.clear();
    seen.clear();
    gt.merge_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_merge).count();
    gt.gen_ms += std::chrono::duration<double, std::milli>(t_merge - t_gen).count();
}

struct LevelStats {  // host split of a level-wise run
    uint64_t pruned = 0, levels = 0;
    double gen_ms = 0.0, merge_ms = 0.0, eval_ms = 0.0;
};

// Level-wise mining over dense vertex labels 0..L-1 and edge labels 1..P
// (edge label el absent when has_part[el] == 0): level 1 is every edge type,
// level k + 1 is grow_level of the frequent k-edge patterns.  evaluate(cands,
// sup, emb) gives each candidate's support and embedding count (non-zero
// return: that status is returned).  The frequent patterns (support >=
// min_support) are appended to `out` level by level in candidate order, as
// query texts over the original labels labels[dense].  GVA_ERR_CANCELLED when
// *cancel is set before a level.
template <typename Eval>
int mine_levels(uint32_t L, uint32_t P, const std::vector<char>& has_part, const std::vector<uint32_t>& labels,
                uint32_t max_edges, uint32_t min_support, unsigned nthreads, const volatile int* cancel,
                Eval&& evaluate, std::vector<MinedPattern>& out, LevelStats& ls) {
    const uint32_t width = (L <= 256 && P <= 255) ? 1 : (L <= 65536 ? 2 : 4);
    // ---- level 1: every edge type
    std::vector<Pattern> cands;
    for (uint32_t a = 0; a < L; ++a)
        for (uint32_t b = a; b < L; ++b)
            for (uint32_t el = 1; el <= P; ++el) {
                if (!has_part[el]) continue;
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
    ls.levels = 1;

    // ---- levels 2..max_edges
    WedgeTab wedges;
    for (uint32_t k = 1; k < max_edges && !level.empty(); ++k) {
        if (cancel && *cancel) return GVA_ERR_CANCELLED;
        GrowStats gt;
        std::vector<Pattern> next;
        if (k == 2 && WedgeTab::fits(L, P)) wedges.build(level, L, P);  // `level` holds the 2-edge patterns
        grow_level(level, level_codes, freq, L, P, width, max_edges, nthreads, wedges.bits.empty() ? nullptr : &wedges,
                   next, gt);
        ls.pruned += gt.pruned;
        ls.gen_ms += gt.gen_ms;
        ls.merge_ms += gt.merge_ms;
        auto t_eval = std::chrono::steady_clock::now();
        rc = evaluate(next, sup, emb);
        if (rc) return rc;
        ls.eval_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_eval).count();
        // the frequent ones: codes and query texts on the worker threads,
        // then filed in candidate order
        std::vector<uint32_t> fi;
        for (size_t i = 0; i < next.size(); ++i)
            if (sup[i] >= min_support) fi.push_back((uint32_t)i);
        std::vector<std::string> texts(fi.size());
        const unsigned pt = std::max(1u, std::min<unsigned>(nthreads, (unsigned)(fi.size() / 256 + 1)));
        std::vector<std::vector<uint8_t>> code_arena(pt);
        std::vector<uint32_t> code_at(fi.size()), code_len(fi.size());
        std::vector<uint8_t> code_thread(fi.size());
        pool_run(pt, [&](unsigned t) {
            CodeBuf cb;
            for (size_t j = t; j < fi.size(); j += pt) {
                canonical(next[fi[j]], width, cb);
                code_at[j] = (uint32_t)code_arena[t].size();
                code_len[j] = cb.len;
                code_thread[j] = (uint8_t)t;
                code_arena[t].insert(code_arena[t].end(), cb.b, cb.b + cb.len);
                texts[j] = query_text(next[fi[j]], labels);
            }
        });
        level.clear();
        level_codes = CodeSet();
        for (size_t j = 0; j < fi.size(); ++j) {
            const uint32_t i = fi[j];
            level.push_back(next[i]);
            const uint8_t* code = code_arena[code_thread[j]].data() + code_at[j];
            level_codes.insert(code, code_len[j], code_hash(code, code_len[j]));
            out.push_back({std::move(texts[j]), k + 1, sup[i], emb[i]});
        }
        ls.levels = k + 1;
    }
    return GVA_OK;
}

}  // namespace
}  // namespace gva
