// Match-order planner: phases, pair orientation, automorphism restrictions
// and repeat flags for one query pattern.
//
// Restates the reference planner src/genMatchOrderCPU.cpp:670-983 (identical
// in semantics to src/genMatchOrder.cpp) with bitmask state instead of maps
// where iteration order does not matter.  Where the reference sorts with
// std::sort the same comparators are applied to the same input sequence, so
// equal-key ties resolve identically (libstdc++ introsort is deterministic).
// The single-vertex mode (src/genMatchOrderSingleV.cpp) is the same plan with
// every 2-vertex extension split into two 1-vertex phases and every
// multi-pair reduction split into 1-pair phases.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <list>
#include <sstream>

#include "../../include/geneva.h"
#include "gva_dplan.h"
#include "gva_internal.h"

namespace gva {
namespace {

inline uint32_t bit(uint32_t v) { return 1u << v; }
inline int popc(uint32_t x) { return __builtin_popcount(x); }

// ---- query text ------------------------------------------------------------
// The reference reads vertices character by character: 'v' starts "vid label",
// '#' skips the rest of the line, the first 'e' ends the vertex section
// (src/genMatchOrderCPU.cpp:679-696).  Edges: every 'e' starts
// "svid evid label"; all other characters are ignored (:708-743).
struct Cursor {
    const std::string& s;
    size_t i = 0;
    bool ok = true;
    explicit Cursor(const std::string& t) : s(t) {}
    bool get(char& c) {
        if (!ok || i >= s.size()) return false;
        c = s[i++];
        return true;
    }
    bool read_uint(uint32_t& v) {  // istream >> unsigned: skip spaces, digits
        while (i < s.size() && isspace((unsigned char)s[i])) ++i;
        if (i >= s.size() || !isdigit((unsigned char)s[i])) { ok = false; return false; }
        uint64_t x = 0;
        while (i < s.size() && isdigit((unsigned char)s[i])) {
            x = x * 10 + (uint64_t)(s[i] - '0');
            if (x > 0xffffffffull) { ok = false; return false; }
            ++i;
        }
        v = (uint32_t)x;
        return true;
    }
    void skip_line() {
        while (i < s.size() && s[i] != '\n') ++i;
        if (i < s.size()) ++i;
    }
};

// Stable sort without a heap buffer for the planner's short lists (the
// order std::stable_sort gives); long lists go to std::stable_sort.
template <typename T, typename Less>
void stable_sort_small(T* a, size_t n, Less less) {
    if (n > 64) {
        std::stable_sort(a, a + n, less);
        return;
    }
    for (size_t i = 1; i < n; ++i) {
        T x = a[i];
        size_t j = i;
        while (j > 0 && less(x, a[j - 1])) {
            a[j] = a[j - 1];
            --j;
        }
        a[j] = x;
    }
}

// The planner's key -> value maps hold a few keys per query: a vector kept in
// ascending key order walks like std::map without a node per key.
template <typename V>
struct FlatMap {
    std::vector<std::pair<uint64_t, V>> items;
    V& operator[](uint64_t k) {
        auto it = std::lower_bound(items.begin(), items.end(), k,
                                   [](const std::pair<uint64_t, V>& a, uint64_t b) { return a.first < b; });
        if (it == items.end() || it->first != k) it = items.insert(it, {k, V()});
        return it->second;
    }
};

struct LabelGroup {  // query[v].edgeLabelNeigs[label] = {count, neighbour mask}
    uint32_t count = 0;
    uint32_t mask = 0;
};

struct NeigInfo {  // one candidate (partial vertex, neighbour) pair
    uint32_t commonVNum, svid, evid, edgeLabel, evLabel, evNum;
};

// src/genMatchOrderCPU.cpp:125-149
bool neig_order(const NeigInfo& a, const NeigInfo& b) {
    if (a.commonVNum != b.commonVNum) return a.commonVNum > b.commonVNum;
    if (a.evNum != b.evNum) return a.evNum > b.evNum;
    if (a.edgeLabel != b.edgeLabel) return a.edgeLabel < b.edgeLabel;
    if (a.svid != b.svid) return a.svid < b.svid;
    return a.evLabel < b.evLabel;
}

struct TriInfo {
    uint32_t edgeIndex = 0, triCount = 0, triScore = 0, maxScoreVID = 0;
};

struct ReduceKey {  // reducePhaseKeyCount entry
    uint32_t count = 0;
    std::vector<uint64_t> partners;
    std::vector<std::pair<uint32_t, uint32_t>> where;  // (phase index, pair index)
};

class Planner {
public:
    uint32_t n = 0;
    std::vector<uint32_t> qlabel;
    std::vector<uint32_t> adj;                       // n*n edge label, kNone = no edge
    std::vector<uint32_t> nbr_full;                  // all neighbours (never consumed)
    // query[v].edgeLabelNeigs as one flat list: vertex v's groups are
    // groups[group_off[v] .. group_off[v + 1]), ascending edge label
    struct LabelEntry {
        uint32_t v, label;
        LabelGroup g;
    };
    std::vector<LabelEntry> groups;
    std::vector<uint32_t> group_off;
    std::vector<uint32_t> live;                      // neighbours whose edge is not planned yet
    struct QEdge { uint32_t s, e, l; };
    std::vector<QEdge> edges;

    std::vector<uint32_t> order;  // matched query vertices in match order
    uint32_t visited = 0;
    std::vector<Phase> phases;
    FlatMap<uint32_t> ext_keys, other_keys;
    FlatMap<ReduceKey> red_keys;
    std::vector<uint32_t> auts;  // automorphisms, n entries each
    uint32_t eqmask[32] = {};    // eqmask[a] bit b: equivalent(a, b)
    uint64_t aut_steps = 0;      // vertex tries of the automorphism search
    bool aut_over = false;       // the search passed its bounds

    uint32_t E(uint32_t a, uint32_t b) const { return adj[(size_t)a * n + b]; }
    static uint64_t key(uint32_t el, uint32_t vl) { return ((uint64_t)el << 32) | vl; }

    const LabelGroup& group(uint32_t v, uint32_t label) const {
        for (uint32_t i = group_off[v]; i < group_off[v + 1]; ++i)
            if (groups[i].label == label) return groups[i].g;
        static const LabelGroup none;
        return none;
    }
    int parse(const std::string& text);
    int set_vertices(uint32_t nv, const uint32_t* labels);  // vertex v labelled labels[v]
    int set_edges(const uint32_t* sdl, size_t ne);  // (svid, evid, label) triples in query order
    void count_triangle(uint32_t i, TriInfo& t) const;
    void seed_without_triangle(uint32_t& s, uint32_t& e1, uint32_t& e2) const;
    void add_ext(uint32_t s1, uint32_t e1, uint32_t s2, uint32_t e2, int num);
    void add_reduce(const std::vector<uint32_t>& pairs);
    bool equivalent(uint32_t a, uint32_t b) const;
    bool possible(const std::vector<uint32_t>& cand, uint32_t nid) const;
    void automorphisms(std::vector<uint32_t>& cand, bool identity);
    void rearrange(Plan& out);
    void restrictions(Plan& out) const;
    int run(Plan& out);
};

int Planner::parse(const std::string& text) {
    std::vector<uint32_t> labels, sdl;
    int st = read_query_text(text, labels, sdl);
    if (st) return st;
    st = set_vertices((uint32_t)labels.size(), labels.data());
    if (st) return st;
    return set_edges(sdl.data(), sdl.size() / 3);
}

int Planner::set_vertices(uint32_t nv, const uint32_t* labels) {
    n = nv;
    if (n == 0) return fail(GVA_ERR_FORMAT, "query has no vertices");
    if (n > GVA_MAX_QUERY_VERTICES) return fail(GVA_ERR_UNSUPPORTED, "query has more than 32 vertices");
    qlabel.assign(labels, labels + n);
    return GVA_OK;
}

// Edges in query order; errors at the first offending edge.
int Planner::set_edges(const uint32_t* sdl, size_t ne) {
    adj.assign((size_t)n * n, kNone);
    nbr_full.assign(n, 0);
    live.assign(n, 0);
    groups.clear();
    groups.reserve(2 * ne);
    edges.reserve(ne);
    for (size_t i = 0; i < ne; ++i) {
        const uint32_t s = sdl[3 * i], d = sdl[3 * i + 1], l = sdl[3 * i + 2];
        if (s >= n || d >= n) return fail(GVA_ERR_FORMAT, "query edge names an undefined vertex");
        if (s == d) return fail(GVA_ERR_UNSUPPORTED, "query self-loop");
        for (int dir = 0; dir < 2; ++dir) {  // addToQueryGraph both ways (:69-85)
            uint32_t a = dir ? d : s, b = dir ? s : d;
            nbr_full[a] |= bit(b);
            groups.push_back({a, l, {1, bit(b)}});
        }
        if (E(s, d) == kNone) {  // first label of a vertex pair wins (:729-737)
            edges.push_back({std::min(s, d), std::max(s, d), l});
            adj[(size_t)s * n + d] = l;
            adj[(size_t)d * n + s] = l;
        }
        live[s] |= bit(d);
        live[d] |= bit(s);
    }
    // one group per (vertex, edge label): counts add up, masks join
    stable_sort_small(groups.data(), groups.size(), [](const LabelEntry& x, const LabelEntry& y) {
        return x.v != y.v ? x.v < y.v : x.label < y.label;
    });
    size_t k = 0;
    for (size_t i = 0; i < groups.size(); ++i) {
        if (k > 0 && groups[k - 1].v == groups[i].v && groups[k - 1].label == groups[i].label) {
            groups[k - 1].g.count += 1;
            groups[k - 1].g.mask |= groups[i].g.mask;
        } else {
            groups[k++] = groups[i];
        }
    }
    groups.resize(k);
    group_off.assign(n + 1, 0);
    for (const LabelEntry& x : groups) group_off[x.v + 1]++;
    for (uint32_t v = 0; v < n; ++v) group_off[v + 1] += group_off[v];
    if (edges.empty()) return fail(GVA_ERR_FORMAT, "query has no edges");
    // connectivity: the reference loops forever on a disconnected pattern
    uint32_t reach = 1, frontier = 1;
    while (frontier) {
        uint32_t next = 0;
        for (uint32_t v = 0; v < n; ++v)
            if (frontier & bit(v)) next |= nbr_full[v];
        frontier = next & ~reach;
        reach |= next;
    }
    if (reach != (n == 32 ? 0xffffffffu : (bit(n) - 1)))
        return fail(GVA_ERR_UNSUPPORTED, "query pattern is not connected");
    return GVA_OK;
}

// src/genMatchOrderCPU.cpp:88-115
void Planner::count_triangle(uint32_t i, TriInfo& t) const {
    const QEdge& ed = edges[i];
    uint32_t tri = live[ed.s] & live[ed.e];
    t.edgeIndex = i;
    t.triCount = (uint32_t)popc(tri);
    if (!tri) return;
    int best = -1;
    int best_v = -1;
    for (uint32_t rest = tri; rest; rest &= rest - 1) {
        const uint32_t v = (uint32_t)__builtin_ctz(rest);
        uint32_t l1 = E(ed.s, v), l2 = E(ed.e, v), l3 = ed.l;
        int score = 10 * ((l1 == l2) + (l1 == l3) + (l2 == l3));
        score += (qlabel[ed.s] == qlabel[ed.e]) + (qlabel[ed.s] == qlabel[v]) + (qlabel[ed.e] == qlabel[v]);
        if (score > best) {
            best = score;
            best_v = (int)v;
        }
    }
    t.triScore = (uint32_t)best;
    t.maxScoreVID = (uint32_t)best_v;
}

// src/genMatchOrderCPU.cpp:176-285: a source whose neighbours best share edge
// and vertex labels, preferring high-degree end vertices.
void Planner::seed_without_triangle(uint32_t& s_out, uint32_t& e1_out, uint32_t& e2_out) const {
    // the reference's three maps (same edge and end label; same edge label;
    // same source), as (key, members) lists in key order.  Keys are unique
    // but for same_el_vl keys of edge labels >= 2^20, where the map keeps the
    // first entry: a stable sort and keeping the first of equal keys does too.
    struct Entry {
        uint64_t key;
        uint32_t at, len;  // members[at .. at + len)
    };
    // sized for the worst case: every group's members, at most one entry per
    // member (repeated edge lines with distinct labels make more groups than
    // there are edges)
    size_t cap = 0;
    for (const LabelEntry& x : groups) cap += (size_t)popc(x.g.mask);
    thread_local std::vector<uint32_t> members[3];
    thread_local std::vector<Entry> list[3];
    for (int i = 0; i < 3; ++i) {
        if (members[i].size() < cap) members[i].resize(cap);
        if (list[i].size() < cap + n) list[i].resize(cap + n);
    }
    uint32_t used[3] = {0, 0, 0};
    uint32_t cnt[3] = {0, 0, 0};
    enum { SAME_EL_VL = 0, SAME_EL = 1, SAME_SRC = 2 };
    for (uint32_t v = 0; v < n; ++v) {
        const uint32_t src_at = used[SAME_SRC];
        for (uint32_t gi = group_off[v]; gi < group_off[v + 1]; ++gi) {
            const uint64_t k_sv_el = ((uint64_t)groups[gi].label << 20) | v;
            const uint32_t mask = groups[gi].g.mask;
            if (popc(mask) >= 2) {
                // end vertices by label: ascending label, ascending id within
                uint32_t ends[32], ne = 0;
                for (uint32_t rest = mask; rest; rest &= rest - 1) ends[ne++] = (uint32_t)__builtin_ctz(rest);
                stable_sort_small(ends, ne, [&](uint32_t x, uint32_t y) { return qlabel[x] < qlabel[y]; });
                const uint32_t el_at = used[SAME_EL];
                for (uint32_t i = 0; i < ne;) {
                    uint32_t j = i + 1;
                    while (j < ne && qlabel[ends[j]] == qlabel[ends[i]]) ++j;
                    if (j - i >= 2) {
                        Entry& x = list[SAME_EL_VL][cnt[SAME_EL_VL]++];
                        x.key = ((uint64_t)qlabel[ends[i]] << 40) | k_sv_el;
                        x.at = used[SAME_EL_VL];
                        x.len = j - i;
                        for (uint32_t t = i; t < j; ++t) members[SAME_EL_VL][used[SAME_EL_VL]++] = ends[t];
                    } else {
                        members[SAME_EL][used[SAME_EL]++] = ends[i];
                    }
                    i = j;
                }
                if (used[SAME_EL] > el_at) list[SAME_EL][cnt[SAME_EL]++] = {k_sv_el, el_at, used[SAME_EL] - el_at};
            } else {
                for (uint32_t rest = mask; rest; rest &= rest - 1)
                    members[SAME_SRC][used[SAME_SRC]++] = (uint32_t)__builtin_ctz(rest);
            }
        }
        if (used[SAME_SRC] > src_at) list[SAME_SRC][cnt[SAME_SRC]++] = {(uint64_t)v, src_at, used[SAME_SRC] - src_at};
    }
    const bool pairwise = cnt[SAME_EL_VL] || cnt[SAME_EL];
    const int which = cnt[SAME_EL_VL] ? SAME_EL_VL : (cnt[SAME_EL] ? SAME_EL : SAME_SRC);
    Entry* pool = list[which].data();
    uint32_t np = cnt[which];
    stable_sort_small(pool, np, [](const Entry& x, const Entry& y) { return x.key < y.key; });
    uint32_t gs = kNone, g1 = 0, g2 = 0, gv1 = kNone, gv2 = kNone;
    for (uint32_t pi = 0; pi < np; ++pi) {
        if (pi > 0 && pool[pi].key == pool[pi - 1].key) continue;  // map::emplace keeps the first
        uint32_t m1 = 0, m2 = 0, v1 = kNone, v2 = kNone;
        for (uint32_t t = 0; t < pool[pi].len; ++t) {
            const uint32_t u = members[which][pool[pi].at + t];
            uint32_t deg = (uint32_t)popc(nbr_full[u]);
            if (deg > m1) {
                m2 = m1; v2 = v1;
                m1 = deg; v1 = u;
            } else if (deg > m2) {
                m2 = deg; v2 = u;
            }
        }
        if (pairwise) {
            if (m1 + m2 > g1 + g2) {
                g1 = m1; gv1 = v1; g2 = m2; gv2 = v2;
                gs = (uint32_t)(pool[pi].key & 0xfffffu);
            }
        } else if (m1 > g1) {
            g1 = m1; gv1 = v1;
            gs = (uint32_t)(pool[pi].key & 0xfffffu);
        }
    }
    s_out = gs;
    e1_out = gv1;
    e2_out = gv2;
}

// src/genMatchOrderCPU.cpp:287-333
void Planner::add_ext(uint32_t s1, uint32_t e1, uint32_t s2, uint32_t e2, int num) {
    if (num == 2 && qlabel[e2] < qlabel[e1]) {
        std::swap(s1, s2);
        std::swap(e1, e2);
    }
    Phase ph;
    ph.type = 'E';
    ph.pairs = {s1, e1};
    ph.edge_label = E(s1, e1);
    auto take = [&](uint32_t s, uint32_t e) {
        ext_keys[key(E(s, e), qlabel[e])] += 1;
        visited |= bit(e);
        order.push_back(e);
        live[s] &= ~bit(e);
        live[e] &= ~bit(s);
    };
    take(s1, e1);
    if (num == 2) {
        ph.pairs.push_back(s2);
        ph.pairs.push_back(e2);
        take(s2, e2);
    }
    phases.push_back(std::move(ph));
}

// src/genMatchOrderCPU.cpp:334-394
void Planner::add_reduce(const std::vector<uint32_t>& pairs) {
    Phase ph;
    ph.type = 'R';
    const uint32_t idx = (uint32_t)phases.size();
    for (size_t i = 0; i < pairs.size() / 2; ++i) {
        uint32_t a = pairs[2 * i], b = pairs[2 * i + 1];
        ph.pairs.push_back(a);
        ph.pairs.push_back(b);
        live[a] &= ~bit(b);
        live[b] &= ~bit(a);
        ph.edge_label = E(a, b);
        uint64_t kb = key(E(a, b), qlabel[b]), ka = key(E(a, b), qlabel[a]);
        if (kb == ka) {
            other_keys[kb] += 1;
        } else {
            ReduceKey& x = red_keys[kb];
            x.count += 1;
            x.partners.push_back(ka);
            x.where.push_back({idx, (uint32_t)i});
            ReduceKey& y = red_keys[ka];
            y.count += 1;
            y.partners.push_back(kb);
            y.where.push_back({idx, (uint32_t)i});
        }
    }
    phases.push_back(std::move(ph));
}

// src/genMatchOrderCPU.cpp:396-431
bool Planner::equivalent(uint32_t a, uint32_t b) const {
    if (a == b) return true;
    if (qlabel[a] != qlabel[b]) return false;
    const uint32_t na = group_off[a + 1] - group_off[a], nb = group_off[b + 1] - group_off[b];
    if (na != nb) return false;
    for (uint32_t i = 0; i < na; ++i) {
        const LabelEntry& x = groups[group_off[a] + i];
        const LabelEntry& y = groups[group_off[b] + i];
        if (x.label != y.label || x.g.count != y.g.count) return false;
    }
    return true;
}

bool Planner::possible(const std::vector<uint32_t>& cand, uint32_t nid) const {
    uint32_t ori = (uint32_t)cand.size();
    if (!(eqmask[ori] >> nid & 1)) return false;  // equivalent(ori, nid)
    for (uint32_t i = 0; i < cand.size(); ++i)
        if (E(i, ori) != E(cand[i], nid)) return false;
    return true;
}

// src/genMatchOrderCPU.cpp:433-462: every non-identity automorphism.
// The reference enumerates without bound; here a query whose search passes
// kMaxAutSteps vertex tries or kMaxAuts automorphisms is rejected instead of
// holding the caller (and memory) indefinitely.
constexpr uint64_t kMaxAutSteps = 1ull << 27, kMaxAuts = 1ull << 20;

void Planner::automorphisms(std::vector<uint32_t>& cand, bool identity) {
    if (aut_over) return;
    uint32_t used = 0;
    for (uint32_t v : cand) used |= bit(v);
    if (cand.size() + 1 == n) {
        for (uint32_t v = 0; v < n; ++v) {
            if (used & bit(v)) continue;
            if (identity && v == cand.size()) return;
            if (possible(cand, v)) {
                if (auts.size() / n >= kMaxAuts) {
                    aut_over = true;
                    return;
                }
                cand.push_back(v);
                auts.insert(auts.end(), cand.begin(), cand.end());
                cand.pop_back();
            }
            break;
        }
        return;
    }
    for (uint32_t v = 0; v < n && !aut_over; ++v) {
        if (used & bit(v)) continue;
        if (++aut_steps > kMaxAutSteps) {
            aut_over = true;
            return;
        }
        if (!possible(cand, v)) continue;
        bool id = identity && v == cand.size();
        cand.push_back(v);
        automorphisms(cand, id);
        cand.pop_back();
    }
}

// src/genMatchOrderCPU.cpp:508-667.  The reference's key-selection loop never
// raises its running maximum, so each round takes the largest remaining key;
// its count is then driven to zero by decrementing once per partner.
void Planner::rearrange(Plan& out) {
    auto note_stat = [&](uint64_t k) {
        uint32_t el = (uint32_t)(k >> 32), vl = (uint32_t)(k & 0xffffffffu);
        auto& v = out.record_stat[el];
        if (std::find(v.begin(), v.end(), vl) == v.end()) {
            v.push_back(vl);
            std::sort(v.begin(), v.end());
        }
    };
    for (size_t ri = red_keys.items.size(); ri-- > 0;) {  // largest key first
        const uint64_t k = red_keys.items[ri].first;
        ReduceKey& rk = red_keys.items[ri].second;
        for (size_t i = 0; i < rk.partners.size(); ++i)
            if (rk.count > 0) rk.count -= 1;
        for (auto& w : rk.where) {
            std::vector<uint32_t>& pr = phases[w.first].pairs;
            if (qlabel[pr[2 * w.second]] == (uint32_t)(k & 0xffffffffu))
                std::swap(pr[2 * w.second], pr[2 * w.second + 1]);
        }
        out.repeat_flag[k] = (rk.count << 16) | rk.count;
        if (rk.count > 1) note_stat(k);
    }
    red_keys.items.clear();
    for (auto* m : {&ext_keys, &other_keys}) {
        for (auto& kv : m->items) {
            auto f = out.repeat_flag.find(kv.first);
            if (f == out.repeat_flag.end()) {
                out.repeat_flag[kv.first] = (kv.second << 16) | kv.second;
                if (kv.second > 1) note_stat(kv.first);
            } else {
                f->second += kv.second;
                if (f->second > 1) note_stat(kv.first);
            }
        }
    }
}

// src/genMatchOrderCPU.cpp:467-506: walk the matched vertices in plan order;
// each automorphism that moves v forces aut(v) < v, then only the stabiliser
// of v is kept.  Per vertex the reference keeps the largest bounding id.
void Planner::restrictions(Plan& out) const {
    std::vector<uint32_t> cur = auts;  // the stabiliser so far, n entries per automorphism
    size_t m = n ? cur.size() / n : 0;
    out.restricts.assign(n + 1, kNone);
    uint32_t seen = 0;
    for (const Phase& ph : phases) {
        if (ph.type == 'R') continue;
        for (uint32_t v : ph.pairs) {
            if (seen & bit(v)) continue;
            seen |= bit(v);
            size_t keep = 0;
            for (size_t i = 0; i < m; ++i) {
                const uint32_t* a = cur.data() + i * n;
                if (a[v] == v) {
                    if (keep != i) std::copy(a, a + n, cur.begin() + keep * n);
                    ++keep;
                } else {
                    uint32_t& r = out.restricts[a[v]];
                    if (r == kNone || r < v) r = v;
                }
            }
            m = keep;
        }
    }
}

int Planner::run(Plan& out) {
    std::vector<TriInfo> tris(edges.size());
    for (uint32_t i = 0; i < edges.size(); ++i) count_triangle(i, tris[i]);
    std::sort(tris.begin(), tris.end(), [](const TriInfo& a, const TriInfo& b) { return a.triCount > b.triCount; });
    if (tris[0].triCount == 0) {
        uint32_t s, e1, e2;
        seed_without_triangle(s, e1, e2);
        if (s == kNone || e1 == kNone) return fail(GVA_ERR_FORMAT, "planner found no seed edge");
        visited |= bit(s);
        order.push_back(s);
        add_ext(s, e1, s, e2, e2 == kNone ? 1 : 2);
    } else {
        // src/genMatchOrderCPU.cpp:768-819: seed with the best triangle
        uint32_t best = 0;
        for (uint32_t i = 1; i < tris.size() && tris[i].triCount == tris[0].triCount; ++i)
            if (tris[i].triScore > tris[best].triScore) best = i;
        const uint32_t score = tris[best].triScore;
        const QEdge& ed = edges[tris[best].edgeIndex];
        uint32_t s = ed.s, e1 = ed.e, e2 = tris[best].maxScoreVID;
        if (score == 33 || score == 31 || score == 30 || (score >= 10 && score <= 13)) {
            if (score == 31) {
                const uint32_t a = ed.s, b = ed.e, c = tris[best].maxScoreVID;
                if (qlabel[a] == qlabel[b]) { s = c; e1 = a; e2 = b; }
                else if (qlabel[a] == qlabel[c]) { s = b; e1 = a; e2 = c; }
                else if (qlabel[b] == qlabel[c]) { s = a; e1 = b; e2 = c; }
            } else if (score >= 10 && score <= 13) {
                const uint32_t a = ed.s, b = ed.e, c = tris[best].maxScoreVID;
                uint32_t l1 = E(a, c), l2 = E(b, c), l3 = ed.l;
                if (l1 == l2) { s = c; e1 = a; e2 = b; }
                else if (l1 == l3) { s = a; e1 = b; e2 = c; }
                else if (l2 == l3) { s = b; e1 = a; e2 = c; }
            }
            visited |= bit(s);
            order.push_back(s);
            add_ext(s, e1, s, e2, 2);
            add_reduce({e1, e2});
        } else if (score <= 3) {
            visited |= bit(s);
            order.push_back(s);
            add_ext(s, e1, s, e2, 1);
            add_ext(s, e2, s, e2, 1);
            add_reduce({e1, e2});
        } else {
            return fail(GVA_ERR_FORMAT, "planner: unexpected triangle score");
        }
    }

    // src/genMatchOrderCPU.cpp:823-963: grow one or two vertices at a time
    // by_el: (edge label, svid, evid) of the edges to unmatched vertices, in
    // discovery order; stably sorted by label it is the reference's
    // label -> pairs map walked in key order
    struct ElPair {
        uint32_t el, s, u;
    };
    std::vector<NeigInfo> infos, back;
    std::vector<ElPair> by_el;
    std::vector<uint32_t> red_pairs;
    infos.reserve(64);
    by_el.reserve(64);
    phases.reserve(2 * n);
    while (order.size() < n) {
        infos.clear();
        by_el.clear();
        for (uint32_t s : order) {
            const uint32_t nb = live[s];
            for (uint32_t rest = nb; rest; rest &= rest - 1) {
                const uint32_t u = (uint32_t)__builtin_ctz(rest);
                NeigInfo ni;
                ni.svid = s;
                ni.evid = u;
                ni.edgeLabel = E(s, u);
                ni.commonVNum = (uint32_t)popc(live[u] & visited) - 1u;
                ni.evLabel = qlabel[u];
                ni.evNum = (uint32_t)popc(nb & group(s, ni.edgeLabel).mask);
                infos.push_back(ni);
                if (!(visited & bit(u))) by_el.push_back({ni.edgeLabel, s, u});
            }
        }
        if (infos.empty()) return fail(GVA_ERR_UNSUPPORTED, "planner: no edge leaves the matched set");
        std::sort(infos.begin(), infos.end(), neig_order);
        if (infos[0].commonVNum > 0) {
            const uint32_t e = infos[0].evid;
            add_ext(infos[0].svid, e, 0, 0, 1);
            back.clear();
            const uint32_t m = live[e] & visited;
            for (uint32_t rest = m; rest; rest &= rest - 1) {
                const uint32_t u = (uint32_t)__builtin_ctz(rest);
                NeigInfo ni{};
                ni.svid = e;
                ni.evid = u;
                ni.edgeLabel = E(e, u);
                ni.evLabel = qlabel[u];
                back.push_back(ni);
            }
            std::sort(back.begin(), back.end(), [](const NeigInfo& a, const NeigInfo& b) {
                if (a.edgeLabel != b.edgeLabel) return a.edgeLabel < b.edgeLabel;
                return a.evLabel < b.evLabel;
            });
            red_pairs.clear();
            for (size_t i = 0; i < back.size(); ++i) {
                if (i > 0 && back[i].edgeLabel != back[i - 1].edgeLabel) {
                    add_reduce(red_pairs);
                    red_pairs.clear();
                }
                red_pairs.push_back(back[i].svid);
                red_pairs.push_back(back[i].evid);
            }
            add_reduce(red_pairs);
            continue;
        }
        // no back edge: two same-edge-label candidates that are adjacent?
        bool found = false;
        stable_sort_small(by_el.data(), by_el.size(), [](const ElPair& a, const ElPair& b) { return a.el < b.el; });
        for (size_t g0 = 0; g0 < by_el.size() && !found;) {
            size_t g1 = g0 + 1;
            while (g1 < by_el.size() && by_el[g1].el == by_el[g0].el) ++g1;
            const ElPair* v = by_el.data() + g0;
            const size_t cnt = g1 - g0;
            for (size_t i = 0; i < cnt && !found; ++i) {
                for (size_t j = i + 1; j < cnt; ++j) {
                    if (E(v[i].u, v[j].u) != kNone) {
                        add_ext(v[i].s, v[i].u, v[j].s, v[j].u, 2);
                        add_reduce({v[i].u, v[j].u});
                        found = true;
                        break;
                    }
                }
            }
            g0 = g1;
        }
        if (found) continue;
        if (infos[0].evNum > 1) {
            add_ext(infos[0].svid, infos[0].evid, infos[1].svid, infos[1].evid, 2);
            continue;
        }
        bool paired = false;
        for (size_t i = 0; i + 1 < infos.size(); ++i) {
            if (infos[i].edgeLabel == infos[i + 1].edgeLabel) {
                add_ext(infos[i].svid, infos[i].evid, infos[i + 1].svid, infos[i + 1].evid, 2);
                paired = true;
                break;
            }
        }
        if (!paired) add_ext(infos[0].svid, infos[0].evid, 0, 0, 1);
    }

    for (uint32_t a = 0; a < n; ++a) {
        eqmask[a] = 0;
        for (uint32_t b = 0; b < n; ++b)
            if (equivalent(a, b)) eqmask[a] |= bit(b);
    }
    std::vector<uint32_t> cand;
    cand.reserve(n);
    automorphisms(cand, true);
    if (aut_over) return fail(GVA_ERR_UNSUPPORTED, "query has too many symmetric vertex maps to enumerate");
    rearrange(out);
    restrictions(out);
    return GVA_OK;
}

}  // namespace

std::string Plan::describe() const {
    std::ostringstream o;
    o << "vnum " << vnum << "\n";
    for (size_t i = 0; i < phases.size(); ++i) {
        const Phase& p = phases[i];
        o << "phase " << i << " " << p.type << " " << p.edge_label << " " << p.pairs.size() / 2;
        for (uint32_t v : p.pairs) o << " " << v;
        o << "\n";
    }
    for (size_t v = 0; v < restricts.size(); ++v) o << "restrict " << v << " " << restricts[v] << "\n";
    char buf[64];
    for (auto& kv : repeat_flag) {
        std::snprintf(buf, sizeof buf, "%x", kv.second);
        o << "repeat " << (uint32_t)(kv.first >> 32) << " " << (uint32_t)(kv.first & 0xffffffffu) << " " << buf << "\n";
    }
    for (auto& kv : record_stat)
        for (uint32_t vl : kv.second) o << "stat " << kv.first << " " << vl << "\n";
    return o.str();
}

namespace {

int finish_plan(Planner& p, int mode, Plan& out) {
    Plan plan;
    plan.mode = mode;
    plan.vnum = p.n;
    plan.qlabel = p.qlabel;
    int st = p.run(plan);
    if (st) return st;
    // output columns: the first phase's source, then every extended vertex
    plan.columns.push_back(p.phases[0].pairs[0]);
    for (const Phase& ph : p.phases)
        if (ph.type == 'E')
            for (size_t i = 1; i < ph.pairs.size(); i += 2) plan.columns.push_back(ph.pairs[i]);
    if (mode == GVA_MODE_DV) {
        plan.phases = std::move(p.phases);
    } else {
        // single-vertex phases (src/genMatchOrderSingleV.cpp:288-401)
        for (const Phase& ph : p.phases) {
            for (size_t i = 0; i < ph.pairs.size(); i += 2) {
                Phase q;
                q.type = ph.type;
                q.edge_label = ph.type == 'E' ? ph.edge_label : p.E(ph.pairs[i], ph.pairs[i + 1]);
                q.pairs = {ph.pairs[i], ph.pairs[i + 1]};
                plan.phases.push_back(q);
            }
        }
    }
    out = std::move(plan);
    return GVA_OK;
}

}  // namespace

int read_query_text(const std::string& text, std::vector<uint32_t>& labels_out, std::vector<uint32_t>& sdl) {
    Cursor c(text);
    // vid -> label, first definition wins, kept in vid order (insertion into
    // a short sorted array; past GVA_MAX_QUERY_VERTICES distinct ids the
    // query is refused anyway, so one more entry marks that)
    constexpr uint32_t kCap = GVA_MAX_QUERY_VERTICES + 1;
    uint32_t vids[kCap], labs[kCap];
    uint32_t n = 0;
    char ch;
    bool in_edges = false;
    while (c.get(ch)) {
        if (ch == 'v') {
            uint32_t vid, lab;
            if (!c.read_uint(vid) || !c.read_uint(lab)) break;
            uint32_t at = n;
            while (at > 0 && vids[at - 1] > vid) --at;
            if (at > 0 && vids[at - 1] == vid) continue;  // defined before: the first definition stands
            if (n == kCap) continue;                      // too many already (refused below)
            for (uint32_t j = n; j > at; --j) {
                vids[j] = vids[j - 1];
                labs[j] = labs[j - 1];
            }
            vids[at] = vid;
            labs[at] = lab;
            ++n;
        } else if (ch == 'e') {
            --c.i;
            in_edges = true;
            break;
        } else if (ch == '#') {
            c.skip_line();
        }
    }
    if (n == 0) return fail(GVA_ERR_FORMAT, "query has no vertices");
    if (n > GVA_MAX_QUERY_VERTICES) return fail(GVA_ERR_UNSUPPORTED, "query has more than 32 vertices");
    labels_out.clear();
    for (uint32_t i = 0; i < n; ++i) {
        if (vids[i] != i) return fail(GVA_ERR_FORMAT, "query vertex ids must be 0..n-1");
        labels_out.push_back(labs[i]);
    }
    if (!in_edges) return fail(GVA_ERR_FORMAT, "query has no edges");
    sdl.clear();
    while (c.ok && c.get(ch)) {
        if (ch != 'e') continue;
        uint32_t s, d, l;
        if (!c.read_uint(s) || !c.read_uint(d) || !c.read_uint(l)) break;
        sdl.push_back(s);
        sdl.push_back(d);
        sdl.push_back(l);
    }
    return GVA_OK;
}

int plan_from_text(const std::string& text, int mode, Plan& out) {
    if (mode != GVA_MODE_DV && mode != GVA_MODE_SV) return fail(GVA_ERR_ARG, "mode must be GVA_MODE_DV or GVA_MODE_SV");
    Planner p;
    int st = p.parse(text);
    if (st) return st;
    return finish_plan(p, mode, out);
}

int plan_from_dplan(const DPlan& d, const uint32_t* labels, Plan& out) {
    if (d.status != DPLAN_OK) return fail(GVA_ERR_ARG, "query was left to the host planner");
    Plan plan;
    plan.mode = GVA_MODE_DV;
    plan.vnum = d.vnum;
    plan.qlabel.assign(labels, labels + d.vnum);
    plan.phases.resize(d.nphase);
    for (uint32_t p = 0; p < d.nphase; ++p) {
        Phase& ph = plan.phases[p];
        ph.type = (char)d.ph_type[p];
        ph.edge_label = d.ph_el[p];
        ph.pairs.assign(d.pairs + d.ph_at[p], d.pairs + d.ph_at[p] + 2 * d.ph_np[p]);
    }
    plan.restricts.assign(d.restricts, d.restricts + d.vnum + 1);
    for (uint32_t i = 0; i < d.nrep; ++i) plan.repeat_flag.emplace_hint(plan.repeat_flag.end(), d.rep_key[i], d.rep_val[i]);
    for (uint32_t i = 0; i < d.nstat; ++i) plan.record_stat[d.stat_el[i]].push_back(d.stat_vl[i]);
    plan.columns.assign(d.columns, d.columns + d.ncol);
    out = std::move(plan);
    return GVA_OK;
}

int plan_from_query(uint32_t n, const uint32_t* labels, const uint32_t* sdl, size_t ne, int mode, Plan& out) {
    if (mode != GVA_MODE_DV && mode != GVA_MODE_SV) return fail(GVA_ERR_ARG, "mode must be GVA_MODE_DV or GVA_MODE_SV");
    Planner p;
    int st = p.set_vertices(n, labels);
    if (!st) st = p.set_edges(sdl, ne);
    if (st) return st;
    return finish_plan(p, mode, out);
}

}  // namespace gva
