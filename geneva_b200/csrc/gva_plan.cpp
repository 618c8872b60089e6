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
    std::vector<std::map<uint32_t, LabelGroup>> by_label;
    std::vector<uint32_t> live;                      // neighbours whose edge is not planned yet
    struct QEdge { uint32_t s, e, l; };
    std::vector<QEdge> edges;

    std::vector<uint32_t> order;  // matched query vertices in match order
    uint32_t visited = 0;
    std::vector<Phase> phases;
    std::map<uint64_t, uint32_t> ext_keys, other_keys;
    std::map<uint64_t, ReduceKey> red_keys;
    std::vector<std::vector<uint32_t>> auts;

    uint32_t E(uint32_t a, uint32_t b) const { return adj[(size_t)a * n + b]; }
    static uint64_t key(uint32_t el, uint32_t vl) { return ((uint64_t)el << 32) | vl; }

    int parse(const std::string& text);
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
    Cursor c(text);
    std::map<uint32_t, uint32_t> labels;  // vid -> label, first definition wins
    char ch;
    bool in_edges = false;
    while (c.get(ch)) {
        if (ch == 'v') {
            uint32_t vid, lab;
            if (!c.read_uint(vid) || !c.read_uint(lab)) break;
            labels.emplace(vid, lab);
        } else if (ch == 'e') {
            --c.i;
            in_edges = true;
            break;
        } else if (ch == '#') {
            c.skip_line();
        }
    }
    n = (uint32_t)labels.size();
    if (n == 0) return fail(GVA_ERR_FORMAT, "query has no vertices");
    if (n > GVA_MAX_QUERY_VERTICES) return fail(GVA_ERR_UNSUPPORTED, "query has more than 32 vertices");
    uint32_t expect = 0;
    for (auto& kv : labels) {
        if (kv.first != expect++) return fail(GVA_ERR_FORMAT, "query vertex ids must be 0..n-1");
        qlabel.push_back(kv.second);
    }
    adj.assign((size_t)n * n, kNone);
    nbr_full.assign(n, 0);
    by_label.assign(n, {});
    live.assign(n, 0);
    if (!in_edges) return fail(GVA_ERR_FORMAT, "query has no edges");
    while (c.ok && c.get(ch)) {
        if (ch != 'e') continue;
        uint32_t s, d, l;
        if (!c.read_uint(s) || !c.read_uint(d) || !c.read_uint(l)) break;
        if (s >= n || d >= n) return fail(GVA_ERR_FORMAT, "query edge names an undefined vertex");
        if (s == d) return fail(GVA_ERR_UNSUPPORTED, "query self-loop");
        for (int dir = 0; dir < 2; ++dir) {  // addToQueryGraph both ways (:69-85)
            uint32_t a = dir ? d : s, b = dir ? s : d;
            nbr_full[a] |= bit(b);
            LabelGroup& g = by_label[a][l];
            g.count += 1;
            g.mask |= bit(b);
        }
        if (E(s, d) == kNone) {  // first label of a vertex pair wins (:729-737)
            edges.push_back({std::min(s, d), std::max(s, d), l});
            adj[(size_t)s * n + d] = l;
            adj[(size_t)d * n + s] = l;
        }
        live[s] |= bit(d);
        live[d] |= bit(s);
    }
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
    for (uint32_t v = 0; v < 32; ++v) {
        if (!(tri & bit(v))) continue;
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
    std::map<uint64_t, std::vector<uint32_t>> same_el_vl, same_el, same_src;
    for (uint32_t v = 0; v < n; ++v) {
        for (auto& kv : by_label[v]) {
            uint64_t k_sv_el = ((uint64_t)kv.first << 20) | v;
            uint32_t mask = kv.second.mask;
            if (popc(mask) >= 2) {
                std::map<uint32_t, std::vector<uint32_t>> by_vl;
                for (uint32_t u = 0; u < 32; ++u)
                    if (mask & bit(u)) by_vl[qlabel[u]].push_back(u);
                for (auto& g : by_vl) {
                    if (g.second.size() >= 2) {
                        same_el_vl.emplace(((uint64_t)g.first << 40) | k_sv_el, g.second);
                    } else {
                        auto& dst = same_el[k_sv_el];
                        dst.insert(dst.end(), g.second.begin(), g.second.end());
                    }
                }
            } else {
                for (uint32_t u = 0; u < 32; ++u)
                    if (mask & bit(u)) same_src[(uint64_t)v].push_back(u);
            }
        }
    }
    const bool pairwise = !same_el_vl.empty() || !same_el.empty();
    const auto& pool = !same_el_vl.empty() ? same_el_vl : (!same_el.empty() ? same_el : same_src);
    uint32_t gs = kNone, g1 = 0, g2 = 0, gv1 = kNone, gv2 = kNone;
    for (auto& kv : pool) {
        uint32_t m1 = 0, m2 = 0, v1 = kNone, v2 = kNone;
        for (uint32_t u : kv.second) {
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
                gs = (uint32_t)(kv.first & 0xfffffu);
            }
        } else if (m1 > g1) {
            g1 = m1; gv1 = v1;
            gs = (uint32_t)(kv.first & 0xfffffu);
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
    phases.push_back(ph);
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
    phases.push_back(ph);
}

// src/genMatchOrderCPU.cpp:396-431
bool Planner::equivalent(uint32_t a, uint32_t b) const {
    if (a == b) return true;
    if (qlabel[a] != qlabel[b]) return false;
    const auto& ga = by_label[a];
    const auto& gb = by_label[b];
    if (ga.size() != gb.size()) return false;
    for (auto ia = ga.begin(), ib = gb.begin(); ia != ga.end(); ++ia, ++ib)
        if (ia->first != ib->first || ia->second.count != ib->second.count) return false;
    return true;
}

bool Planner::possible(const std::vector<uint32_t>& cand, uint32_t nid) const {
    uint32_t ori = (uint32_t)cand.size();
    if (!equivalent(ori, nid)) return false;
    for (uint32_t i = 0; i < cand.size(); ++i)
        if (E(i, ori) != E(cand[i], nid)) return false;
    return true;
}

// src/genMatchOrderCPU.cpp:433-462: every non-identity automorphism.
void Planner::automorphisms(std::vector<uint32_t>& cand, bool identity) {
    uint32_t used = 0;
    for (uint32_t v : cand) used |= bit(v);
    if (cand.size() + 1 == n) {
        for (uint32_t v = 0; v < n; ++v) {
            if (used & bit(v)) continue;
            if (identity && v == cand.size()) return;
            if (possible(cand, v)) {
                cand.push_back(v);
                auts.push_back(cand);
                cand.pop_back();
            }
            break;
        }
        return;
    }
    for (uint32_t v = 0; v < n; ++v) {
        if (used & bit(v)) continue;
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
    while (!red_keys.empty()) {
        auto it = std::prev(red_keys.end());
        const uint64_t k = it->first;
        ReduceKey& rk = it->second;
        for (size_t i = 0; i < rk.partners.size(); ++i)
            if (rk.count > 0) rk.count -= 1;
        for (auto& w : rk.where) {
            std::vector<uint32_t>& pr = phases[w.first].pairs;
            if (qlabel[pr[2 * w.second]] == (uint32_t)(k & 0xffffffffu))
                std::swap(pr[2 * w.second], pr[2 * w.second + 1]);
        }
        out.repeat_flag[k] = (rk.count << 16) | rk.count;
        if (rk.count > 1) note_stat(k);
        red_keys.erase(it);
    }
    for (auto* m : {&ext_keys, &other_keys}) {
        for (auto& kv : *m) {
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
    std::vector<std::vector<uint32_t>> cur = auts;
    out.restricts.assign(n + 1, kNone);
    uint32_t seen = 0;
    for (const Phase& ph : phases) {
        if (ph.type == 'R') continue;
        for (uint32_t v : ph.pairs) {
            if (seen & bit(v)) continue;
            seen |= bit(v);
            std::vector<std::vector<uint32_t>> stab;
            for (auto& a : cur) {
                if (a[v] == v) {
                    stab.push_back(a);
                } else {
                    uint32_t& r = out.restricts[a[v]];
                    if (r == kNone || r < v) r = v;
                }
            }
            cur.swap(stab);
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
    while (order.size() < n) {
        std::vector<NeigInfo> infos;
        std::map<uint32_t, std::vector<uint32_t>> by_el;  // edge label -> (svid, evid) pairs
        for (uint32_t s : order) {
            const uint32_t nb = live[s];
            for (uint32_t u = 0; u < 32; ++u) {
                if (!(nb & bit(u))) continue;
                NeigInfo ni;
                ni.svid = s;
                ni.evid = u;
                ni.edgeLabel = E(s, u);
                ni.commonVNum = (uint32_t)popc(live[u] & visited) - 1u;
                ni.evLabel = qlabel[u];
                ni.evNum = (uint32_t)popc(nb & by_label[s].at(ni.edgeLabel).mask);
                infos.push_back(ni);
                if (!(visited & bit(u))) {
                    auto& v = by_el[ni.edgeLabel];
                    v.push_back(s);
                    v.push_back(u);
                }
            }
        }
        if (infos.empty()) return fail(GVA_ERR_UNSUPPORTED, "planner: no edge leaves the matched set");
        std::sort(infos.begin(), infos.end(), neig_order);
        if (infos[0].commonVNum > 0) {
            const uint32_t e = infos[0].evid;
            add_ext(infos[0].svid, e, 0, 0, 1);
            std::vector<NeigInfo> back;
            const uint32_t m = live[e] & visited;
            for (uint32_t u = 0; u < 32; ++u) {
                if (!(m & bit(u))) continue;
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
            std::vector<uint32_t> group;
            for (size_t i = 0; i < back.size(); ++i) {
                if (i > 0 && back[i].edgeLabel != back[i - 1].edgeLabel) {
                    add_reduce(group);
                    group.clear();
                }
                group.push_back(back[i].svid);
                group.push_back(back[i].evid);
            }
            add_reduce(group);
            continue;
        }
        // no back edge: two same-edge-label candidates that are adjacent?
        bool found = false;
        for (auto& kv : by_el) {
            const std::vector<uint32_t>& v = kv.second;
            const size_t cnt = v.size() / 2;
            for (size_t i = 0; i < cnt && !found; ++i) {
                for (size_t j = i + 1; j < cnt; ++j) {
                    if (E(v[2 * i + 1], v[2 * j + 1]) != kNone) {
                        add_ext(v[2 * i], v[2 * i + 1], v[2 * j], v[2 * j + 1], 2);
                        add_reduce({v[2 * i + 1], v[2 * j + 1]});
                        found = true;
                        break;
                    }
                }
            }
            if (found) break;
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

    std::vector<uint32_t> cand;
    automorphisms(cand, true);
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

int plan_from_text(const std::string& text, int mode, Plan& out) {
    if (mode != GVA_MODE_DV && mode != GVA_MODE_SV) return fail(GVA_ERR_ARG, "mode must be GVA_MODE_DV or GVA_MODE_SV");
    Planner p;
    int st = p.parse(text);
    if (st) return st;
    Plan plan;
    plan.mode = mode;
    plan.vnum = p.n;
    plan.qlabel = p.qlabel;
    st = p.run(plan);
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

}  // namespace gva
