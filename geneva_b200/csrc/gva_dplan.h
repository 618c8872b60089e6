// Match-order planner without heap storage, compilable for the host and the
// device (one query per thread): the same plan as the host planner
// (gva_plan.cpp, itself a restatement of src/genMatchOrderCPU.cpp:670-983)
// for every query it accepts, DV mode.
//
// Where the host planner sorts with std::sort, this sorts with a stable
// insertion sort, which is what libstdc++'s std::sort does for 16 entries or
// fewer; a query whose edge, neighbour or back-edge lists grow longer, or
// that exceeds a fixed capacity below, is answered with DPLAN_HOST and left
// to the host planner, as is one whose automorphism search grows past fixed
// bounds (so that a call's time is bounded).  Restrictions are gathered
// while automorphisms are enumerated: an automorphism contributes only at the
// first vertex (in plan order) that it moves, so none has to be stored.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define GVA_HD __host__ __device__
#else
#define GVA_HD
#endif

namespace gva {

constexpr uint32_t kDpNone = 0xffffffffu;
constexpr int kDpV = 32;          // query vertices
constexpr int kDpLines = 64;      // edge lines of the query
constexpr int kDpPhases = 96;     // E phases <= vertices, R phases <= edges
constexpr int kDpPairs = 256;     // vertex ids over all phases
constexpr int kDpKeys = 256;      // (edge label, vertex label) keys
constexpr int kDpSort = 16;       // longest list sorted as std::sort would
constexpr uint64_t kDpMaxAut = 1u << 20;    // automorphisms enumerated at most
constexpr uint64_t kDpMaxSearch = 1u << 22;  // partial maps tried at most (bounds the search's time)

enum : uint32_t { DPLAN_OK = 0, DPLAN_HOST = 1 };

struct DPlanQuery {
    uint32_t n = 0, lines = 0;
    uint32_t label[kDpV];
    uint32_t s[kDpLines], d[kDpLines], l[kDpLines];  // edge lines in query order
};

struct DPlan {
    uint32_t status = DPLAN_HOST;
    uint32_t vnum = 0, nphase = 0, npair = 0, nrep = 0, nstat = 0, ncol = 0;
    uint8_t ph_type[kDpPhases];  // 'E' / 'R'
    uint32_t ph_el[kDpPhases];
    uint16_t ph_at[kDpPhases], ph_np[kDpPhases];  // pairs[ph_at .. ph_at + 2 * ph_np)
    uint8_t pairs[kDpPairs];
    uint32_t restricts[kDpV + 1];
    uint64_t rep_key[kDpKeys];  // repeat flags, ascending key (edge label << 32 | vertex label)
    uint32_t rep_val[kDpKeys];
    uint32_t stat_el[kDpKeys], stat_vl[kDpKeys];  // record stats, ascending (edge label, vertex label)
    uint8_t columns[kDpV];
};

namespace dplan_detail {

GVA_HD inline uint32_t bit(uint32_t v) { return 1u << v; }
GVA_HD inline uint32_t popc(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return (uint32_t)__popc(x);
#else
    return (uint32_t)__builtin_popcount(x);
#endif
}
GVA_HD inline uint32_t ctz(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return (uint32_t)(__ffs((int)x) - 1);
#else
    return (uint32_t)__builtin_ctz(x);
#endif
}
template <typename T>
GVA_HD inline void swap_(T& a, T& b) {
    T t = a;
    a = b;
    b = t;
}
// stable insertion sort (std::sort's order for up to 16 entries)
template <typename T, typename Less>
GVA_HD inline void isort(T* a, uint32_t n, Less less) {
    for (uint32_t i = 1; i < n; ++i) {
        T x = a[i];
        uint32_t j = i;
        while (j > 0 && less(x, a[j - 1])) {
            a[j] = a[j - 1];
            --j;
        }
        a[j] = x;
    }
}

struct Info {  // one (matched vertex, neighbour) candidate
    uint32_t commonVNum, svid, evid, edgeLabel, evLabel, evNum;
};
GVA_HD inline bool info_less(const Info& a, const Info& b) {  // src/genMatchOrderCPU.cpp:125-149
    if (a.commonVNum != b.commonVNum) return a.commonVNum > b.commonVNum;
    if (a.evNum != b.evNum) return a.evNum > b.evNum;
    if (a.edgeLabel != b.edgeLabel) return a.edgeLabel < b.edgeLabel;
    if (a.svid != b.svid) return a.svid < b.svid;
    return a.evLabel < b.evLabel;
}
struct Tri {
    uint32_t edgeIndex, triCount, triScore, maxScoreVID;
};
struct Group {  // query[v].edgeLabelNeigs[label]
    uint32_t v, label, count, mask;
};
struct KeyCount {
    uint64_t key;
    uint32_t count;
};
struct RedRef {  // one side of a reduce pair: its key and where the pair is
    uint64_t key;
    uint32_t phase, pair;
};
struct SeedEntry {  // one entry of the seed selection's maps
    uint64_t key;
    uint32_t at, len;
};

struct DPlanner {
    const DPlanQuery& q;
    DPlan& out;
    uint32_t n = 0;
    uint8_t adj[kDpV][kDpV];  // index of the distinct edge (es, ee, el), 0xff: none
    uint32_t nbr_full[kDpV], live[kDpV];
    Group groups[2 * kDpLines];
    uint32_t ngroups = 0, goff[kDpV + 1];
    uint32_t es[kDpLines], ee[kDpLines], el[kDpLines], nedges = 0;  // distinct edges, first label wins
    uint32_t order[kDpV], norder = 0, visited = 0;
    KeyCount ext_keys[kDpV], other_keys[kDpLines];  // one per matched vertex / planned edge at most
    uint32_t next_keys = 0, nother_keys = 0;
    RedRef red[2 * kDpLines];  // two per reduce pair; a pair is a planned edge
    uint32_t nred = 0;

    GVA_HD DPlanner(const DPlanQuery& q_, DPlan& out_) : q(q_), out(out_) {}

    GVA_HD uint32_t E(uint32_t a, uint32_t b) const { return adj[a][b] == 0xff ? kDpNone : el[adj[a][b]]; }
    GVA_HD uint32_t ql(uint32_t v) const { return q.label[v]; }
    GVA_HD static uint64_t key(uint32_t e, uint32_t v) { return ((uint64_t)e << 32) | v; }
    GVA_HD uint32_t group_mask(uint32_t v, uint32_t label) const {
        for (uint32_t i = goff[v]; i < goff[v + 1]; ++i)
            if (groups[i].label == label) return groups[i].mask;
        return 0;
    }

    GVA_HD bool setup() {
        n = q.n;
        if (n == 0 || n > (uint32_t)kDpV || q.lines == 0 || q.lines > (uint32_t)kDpLines) return false;
        for (uint32_t a = 0; a < n; ++a) {
            nbr_full[a] = live[a] = 0;
            for (uint32_t b = 0; b < n; ++b) adj[a][b] = 0xff;
        }
        for (uint32_t i = 0; i < q.lines; ++i) {
            const uint32_t s = q.s[i], d = q.d[i], l = q.l[i];
            if (s >= n || d >= n || s == d) return false;  // the host planner reports these
            nbr_full[s] |= bit(d);
            nbr_full[d] |= bit(s);
            groups[ngroups++] = {s, l, 1, bit(d)};
            groups[ngroups++] = {d, l, 1, bit(s)};
            if (adj[s][d] == 0xff) {
                es[nedges] = s < d ? s : d;
                ee[nedges] = s < d ? d : s;
                el[nedges] = l;
                adj[s][d] = adj[d][s] = (uint8_t)nedges;
                ++nedges;
            }
            live[s] |= bit(d);
            live[d] |= bit(s);
        }
        isort(groups, ngroups, [](const Group& x, const Group& y) {
            return x.v != y.v ? x.v < y.v : x.label < y.label;
        });
        uint32_t k = 0;
        for (uint32_t i = 0; i < ngroups; ++i) {
            if (k > 0 && groups[k - 1].v == groups[i].v && groups[k - 1].label == groups[i].label) {
                groups[k - 1].count += 1;
                groups[k - 1].mask |= groups[i].mask;
            } else {
                groups[k++] = groups[i];
            }
        }
        ngroups = k;
        for (uint32_t v = 0; v <= n; ++v) goff[v] = 0;
        for (uint32_t i = 0; i < ngroups; ++i) goff[groups[i].v + 1]++;
        for (uint32_t v = 0; v < n; ++v) goff[v + 1] += goff[v];
        uint32_t reach = 1, frontier = 1;
        while (frontier) {
            uint32_t nx = 0;
            for (uint32_t rest = frontier; rest; rest &= rest - 1) nx |= nbr_full[ctz(rest)];
            frontier = nx & ~reach;
            reach |= nx;
        }
        return reach == (n == 32 ? 0xffffffffu : (bit(n) - 1));
    }

    GVA_HD bool push_order(uint32_t v) {
        if (norder >= (uint32_t)kDpV) return false;
        order[norder++] = v;
        return true;
    }
    GVA_HD bool add_key(KeyCount* keys, uint32_t& nk, uint64_t k, uint32_t cap) {  // keys[k] += 1, ascending
        uint32_t i = 0;
        while (i < nk && keys[i].key < k) ++i;
        if (i < nk && keys[i].key == k) {
            keys[i].count += 1;
            return true;
        }
        if (nk >= cap) return false;
        for (uint32_t j = nk; j > i; --j) keys[j] = keys[j - 1];
        keys[i] = {k, 1};
        ++nk;
        return true;
    }
    GVA_HD bool new_phase(uint8_t type, uint32_t edge_label) {
        if (out.nphase >= (uint32_t)kDpPhases) return false;
        const uint32_t p = out.nphase++;
        out.ph_type[p] = type;
        out.ph_el[p] = edge_label;
        out.ph_at[p] = (uint16_t)out.npair;
        out.ph_np[p] = 0;
        return true;
    }
    GVA_HD bool add_pair(uint32_t a, uint32_t b) {
        if (out.npair + 2 > (uint32_t)kDpPairs) return false;
        out.pairs[out.npair++] = (uint8_t)a;
        out.pairs[out.npair++] = (uint8_t)b;
        out.ph_np[out.nphase - 1]++;
        return true;
    }

    // src/genMatchOrderCPU.cpp:287-333
    GVA_HD bool add_ext(uint32_t s1, uint32_t e1, uint32_t s2, uint32_t e2, int num) {
        if (num == 2 && ql(e2) < ql(e1)) {
            swap_(s1, s2);
            swap_(e1, e2);
        }
        if (!new_phase('E', E(s1, e1))) return false;
        auto take = [&](uint32_t s, uint32_t e) {
            if (!add_pair(s, e) || !add_key(ext_keys, next_keys, key(E(s, e), ql(e)), kDpV)) return false;
            visited |= bit(e);
            if (!push_order(e)) return false;
            live[s] &= ~bit(e);
            live[e] &= ~bit(s);
            return true;
        };
        if (!take(s1, e1)) return false;
        if (num == 2 && !take(s2, e2)) return false;
        return true;
    }

    // src/genMatchOrderCPU.cpp:334-394; pairs a0 b0 a1 b1 ...
    GVA_HD bool add_reduce(const uint32_t* pr, uint32_t np) {
        const uint32_t idx = out.nphase;
        if (!new_phase('R', 0)) return false;
        for (uint32_t i = 0; i < np; ++i) {
            const uint32_t a = pr[2 * i], b = pr[2 * i + 1];
            if (!add_pair(a, b)) return false;
            live[a] &= ~bit(b);
            live[b] &= ~bit(a);
            out.ph_el[idx] = E(a, b);
            const uint64_t kb = key(E(a, b), ql(b)), ka = key(E(a, b), ql(a));
            if (kb == ka) {
                if (!add_key(other_keys, nother_keys, kb, kDpLines)) return false;
            } else {
                if (nred + 2 > (uint32_t)(2 * kDpLines)) return false;
                red[nred++] = {kb, idx, i};
                red[nred++] = {ka, idx, i};
            }
        }
        return true;
    }

    // src/genMatchOrderCPU.cpp:88-115
    GVA_HD void count_triangle(uint32_t i, Tri& t) const {
        const uint32_t tri = live[es[i]] & live[ee[i]];
        t.edgeIndex = i;
        t.triCount = popc(tri);
        t.triScore = 0;
        t.maxScoreVID = 0;
        if (!tri) return;
        int best = -1, best_v = -1;
        for (uint32_t rest = tri; rest; rest &= rest - 1) {
            const uint32_t v = ctz(rest);
            const uint32_t l1 = E(es[i], v), l2 = E(ee[i], v), l3 = el[i];
            int score = 10 * ((l1 == l2) + (l1 == l3) + (l2 == l3));
            score += (ql(es[i]) == ql(ee[i])) + (ql(es[i]) == ql(v)) + (ql(ee[i]) == ql(v));
            if (score > best) {
                best = score;
                best_v = (int)v;
            }
        }
        t.triScore = (uint32_t)best;
        t.maxScoreVID = (uint32_t)best_v;
    }

    // src/genMatchOrderCPU.cpp:176-285: the reference's three maps as
    // (key, members) lists in key order; for same-edge-and-end-label keys the
    // first entry of equal keys is kept, as map::emplace does
    GVA_HD void seed_without_triangle(uint32_t& s_out, uint32_t& e1_out, uint32_t& e2_out) const {
        // a group's members are its mask bits: at most two per edge line in all
        constexpr uint32_t kCap = 2 * kDpLines;
        // entries: a same-edge-and-end-label list has two or more members,
        // a same-edge-label list one per group, a same-source list one per vertex
        const uint32_t list_cap[3] = {kCap / 2, kCap, (uint32_t)kDpV};
        uint32_t members[3][kCap];
        SeedEntry list0[kCap / 2], list1[kCap], list2[kDpV];
        SeedEntry* list[3] = {list0, list1, list2};
        uint32_t used[3] = {0, 0, 0}, cnt[3] = {0, 0, 0};
        enum { SAME_EL_VL = 0, SAME_EL = 1, SAME_SRC = 2 };
        bool overflow = false;
        for (uint32_t v = 0; v < n && !overflow; ++v) {
            const uint32_t src_at = used[SAME_SRC];
            for (uint32_t gi = goff[v]; gi < goff[v + 1]; ++gi) {
                const uint64_t k_sv_el = ((uint64_t)groups[gi].label << 20) | v;
                const uint32_t mask = groups[gi].mask;
                const uint32_t pm = popc(mask);
                if (used[SAME_EL_VL] + pm > kCap || used[SAME_EL] + pm > kCap || used[SAME_SRC] + pm > kCap ||
                    cnt[SAME_EL_VL] + pm / 2 > list_cap[SAME_EL_VL] || cnt[SAME_EL] + 1 > list_cap[SAME_EL] ||
                    cnt[SAME_SRC] + 1 > list_cap[SAME_SRC]) {
                    overflow = true;
                    break;
                }
                if (pm >= 2) {
                    uint32_t ends[kDpV], ne = 0;
                    for (uint32_t rest = mask; rest; rest &= rest - 1) ends[ne++] = ctz(rest);
                    const DPlanQuery& qq = q;
                    isort(ends, ne, [&qq](uint32_t x, uint32_t y) { return qq.label[x] < qq.label[y]; });
                    const uint32_t el_at = used[SAME_EL];
                    for (uint32_t i = 0; i < ne;) {
                        uint32_t j = i + 1;
                        while (j < ne && ql(ends[j]) == ql(ends[i])) ++j;
                        if (j - i >= 2) {
                            SeedEntry& x = list[SAME_EL_VL][cnt[SAME_EL_VL]++];
                            x.key = ((uint64_t)ql(ends[i]) << 40) | k_sv_el;
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
                    for (uint32_t rest = mask; rest; rest &= rest - 1) members[SAME_SRC][used[SAME_SRC]++] = ctz(rest);
                }
            }
            if (!overflow && used[SAME_SRC] > src_at)
                list[SAME_SRC][cnt[SAME_SRC]++] = {(uint64_t)v, src_at, used[SAME_SRC] - src_at};
        }
        s_out = e1_out = e2_out = kDpNone;
        if (overflow) return;
        const bool pairwise = cnt[SAME_EL_VL] || cnt[SAME_EL];
        const int which = cnt[SAME_EL_VL] ? SAME_EL_VL : (cnt[SAME_EL] ? SAME_EL : SAME_SRC);
        SeedEntry* pool = list[which];
        const uint32_t np = cnt[which];
        isort(pool, np, [](const SeedEntry& x, const SeedEntry& y) { return x.key < y.key; });
        uint32_t gs = kDpNone, g1 = 0, g2 = 0, gv1 = kDpNone, gv2 = kDpNone;
        for (uint32_t pi = 0; pi < np; ++pi) {
            if (pi > 0 && pool[pi].key == pool[pi - 1].key) continue;
            uint32_t m1 = 0, m2 = 0, v1 = kDpNone, v2 = kDpNone;
            for (uint32_t t = 0; t < pool[pi].len; ++t) {
                const uint32_t u = members[which][pool[pi].at + t];
                const uint32_t deg = popc(nbr_full[u]);
                if (deg > m1) {
                    m2 = m1;
                    v2 = v1;
                    m1 = deg;
                    v1 = u;
                } else if (deg > m2) {
                    m2 = deg;
                    v2 = u;
                }
            }
            if (pairwise) {
                if (m1 + m2 > g1 + g2) {
                    g1 = m1;
                    gv1 = v1;
                    g2 = m2;
                    gv2 = v2;
                    gs = (uint32_t)(pool[pi].key & 0xfffffu);
                }
            } else if (m1 > g1) {
                g1 = m1;
                gv1 = v1;
                gs = (uint32_t)(pool[pi].key & 0xfffffu);
            }
        }
        s_out = gs;
        e1_out = gv1;
        e2_out = gv2;
    }

    // the first phases: seed edge(s), src/genMatchOrderCPU.cpp:747-819
    GVA_HD bool seed() {
        if (nedges > (uint32_t)kDpSort) return false;
        Tri tris[kDpSort];
        for (uint32_t i = 0; i < nedges; ++i) count_triangle(i, tris[i]);
        isort(tris, nedges, [](const Tri& a, const Tri& b) { return a.triCount > b.triCount; });
        if (tris[0].triCount == 0) {
            uint32_t s, e1, e2;
            seed_without_triangle(s, e1, e2);
            if (s == kDpNone || e1 == kDpNone) return false;
            visited |= bit(s);
            if (!push_order(s)) return false;
            return add_ext(s, e1, s, e2, e2 == kDpNone ? 1 : 2);
        }
        uint32_t best = 0;
        for (uint32_t i = 1; i < nedges && tris[i].triCount == tris[0].triCount; ++i)
            if (tris[i].triScore > tris[best].triScore) best = i;
        const uint32_t score = tris[best].triScore;
        const uint32_t ei = tris[best].edgeIndex;
        uint32_t s = es[ei], e1 = ee[ei], e2 = tris[best].maxScoreVID;
        if (score == 33 || score == 31 || score == 30 || (score >= 10 && score <= 13)) {
            const uint32_t a = es[ei], b = ee[ei], c = tris[best].maxScoreVID;
            if (score == 31) {
                if (ql(a) == ql(b)) {
                    s = c, e1 = a, e2 = b;
                } else if (ql(a) == ql(c)) {
                    s = b, e1 = a, e2 = c;
                } else if (ql(b) == ql(c)) {
                    s = a, e1 = b, e2 = c;
                }
            } else if (score >= 10 && score <= 13) {
                const uint32_t l1 = E(a, c), l2 = E(b, c), l3 = el[ei];
                if (l1 == l2) {
                    s = c, e1 = a, e2 = b;
                } else if (l1 == l3) {
                    s = a, e1 = b, e2 = c;
                } else if (l2 == l3) {
                    s = b, e1 = a, e2 = c;
                }
            }
            visited |= bit(s);
            if (!push_order(s) || !add_ext(s, e1, s, e2, 2)) return false;
            const uint32_t pr[2] = {e1, e2};
            return add_reduce(pr, 1);
        }
        if (score <= 3) {
            visited |= bit(s);
            if (!push_order(s) || !add_ext(s, e1, s, e2, 1) || !add_ext(s, e2, s, e2, 1)) return false;
            const uint32_t pr[2] = {e1, e2};
            return add_reduce(pr, 1);
        }
        return false;
    }

    // src/genMatchOrderCPU.cpp:823-963: grow one or two vertices at a time
    GVA_HD bool grow() {
        Info infos[kDpSort];
        struct ElPair {
            uint32_t el, s, u;
        };
        ElPair by_el[kDpSort];  // a subset of the candidates
        while (norder < n) {
            uint32_t ni = 0, nb_el = 0;
            for (uint32_t oi = 0; oi < norder; ++oi) {
                const uint32_t s = order[oi];
                const uint32_t nb = live[s];
                for (uint32_t rest = nb; rest; rest &= rest - 1) {
                    const uint32_t u = ctz(rest);
                    if (ni >= (uint32_t)kDpSort) return false;
                    Info& x = infos[ni++];
                    x.svid = s;
                    x.evid = u;
                    x.edgeLabel = E(s, u);
                    x.commonVNum = popc(live[u] & visited) - 1u;
                    x.evLabel = ql(u);
                    x.evNum = popc(nb & group_mask(s, x.edgeLabel));
                    if (!(visited & bit(u))) by_el[nb_el++] = {x.edgeLabel, s, u};
                }
            }
            if (ni == 0) return false;
            isort(infos, ni, info_less);
            if (infos[0].commonVNum > 0) {
                const uint32_t e = infos[0].evid;
                if (!add_ext(infos[0].svid, e, 0, 0, 1)) return false;
                Info back[kDpSort];
                uint32_t nback = 0;
                const uint32_t m = live[e] & visited;
                for (uint32_t rest = m; rest; rest &= rest - 1) {
                    const uint32_t u = ctz(rest);
                    if (nback >= (uint32_t)kDpSort) return false;
                    Info& x = back[nback++];
                    x = Info{0, e, u, E(e, u), ql(u), 0};
                }
                isort(back, nback, [](const Info& a, const Info& b) {
                    if (a.edgeLabel != b.edgeLabel) return a.edgeLabel < b.edgeLabel;
                    return a.evLabel < b.evLabel;
                });
                uint32_t pr[2 * kDpSort], np = 0;
                for (uint32_t i = 0; i < nback; ++i) {
                    if (i > 0 && back[i].edgeLabel != back[i - 1].edgeLabel) {
                        if (!add_reduce(pr, np)) return false;
                        np = 0;
                    }
                    pr[2 * np] = back[i].svid;
                    pr[2 * np + 1] = back[i].evid;
                    ++np;
                }
                if (!add_reduce(pr, np)) return false;
                continue;
            }
            // no back edge: two same-edge-label candidates that are adjacent?
            isort(by_el, nb_el, [](const ElPair& a, const ElPair& b) { return a.el < b.el; });
            bool found = false;
            for (uint32_t g0 = 0; g0 < nb_el && !found;) {
                uint32_t g1 = g0 + 1;
                while (g1 < nb_el && by_el[g1].el == by_el[g0].el) ++g1;
                const ElPair* v = by_el + g0;
                const uint32_t c = g1 - g0;
                for (uint32_t i = 0; i < c && !found; ++i)
                    for (uint32_t j = i + 1; j < c; ++j)
                        if (E(v[i].u, v[j].u) != kDpNone) {
                            if (!add_ext(v[i].s, v[i].u, v[j].s, v[j].u, 2)) return false;
                            const uint32_t pr[2] = {v[i].u, v[j].u};
                            if (!add_reduce(pr, 1)) return false;
                            found = true;
                            break;
                        }
                g0 = g1;
            }
            if (found) continue;
            if (infos[0].evNum > 1) {
                if (ni < 2 || !add_ext(infos[0].svid, infos[0].evid, infos[1].svid, infos[1].evid, 2)) return false;
                continue;
            }
            bool paired = false;
            for (uint32_t i = 0; i + 1 < ni; ++i)
                if (infos[i].edgeLabel == infos[i + 1].edgeLabel) {
                    if (!add_ext(infos[i].svid, infos[i].evid, infos[i + 1].svid, infos[i + 1].evid, 2)) return false;
                    paired = true;
                    break;
                }
            if (!paired && !add_ext(infos[0].svid, infos[0].evid, 0, 0, 1)) return false;
        }
        return true;
    }

    // src/genMatchOrderCPU.cpp:433-506: every non-identity automorphism;
    // each one bounds aut(v) < v at the first vertex v it moves, walking the
    // matched vertices in plan order, and a vertex keeps its largest bound
    GVA_HD bool restrictions() {
        uint32_t eq[kDpV];  // eq[a] bit b: a and b are equivalent
        for (uint32_t a = 0; a < n; ++a) {
            eq[a] = 0;
            for (uint32_t b = 0; b < n; ++b) {
                bool same = a == b;
                if (!same && ql(a) == ql(b) && goff[a + 1] - goff[a] == goff[b + 1] - goff[b]) {
                    same = true;
                    for (uint32_t i = 0; i < goff[a + 1] - goff[a] && same; ++i)
                        same = groups[goff[a] + i].label == groups[goff[b] + i].label &&
                               groups[goff[a] + i].count == groups[goff[b] + i].count;
                }
                if (same) eq[a] |= bit(b);
            }
        }
        uint32_t porder[kDpV], np = 0, seen = 0;  // matched vertices in plan order
        for (uint32_t p = 0; p < out.nphase; ++p) {
            if (out.ph_type[p] == 'R') continue;
            for (uint32_t i = 0; i < 2u * out.ph_np[p]; ++i) {
                const uint32_t v = out.pairs[out.ph_at[p] + i];
                if (seen & bit(v)) continue;
                seen |= bit(v);
                porder[np++] = v;
            }
        }
        for (uint32_t v = 0; v <= n; ++v) out.restricts[v] = kDpNone;
        // depth-first over partial maps cand[0..depth) (vertex i -> cand[i])
        uint32_t cand[kDpV], nextv[kDpV], used = 0;
        uint64_t found = 0, tried = 0;
        uint32_t depth = 0;
        nextv[0] = 0;
        bool identity[kDpV + 1];  // the map so far is the identity
        identity[0] = true;
        while (true) {
            if (nextv[depth] >= n) {  // this level is exhausted: back up
                if (depth == 0) break;
                --depth;
                used &= ~bit(cand[depth]);
                nextv[depth] = cand[depth] + 1;
                continue;
            }
            const uint32_t v = nextv[depth];
            if (used & bit(v)) {
                nextv[depth] = v + 1;
                continue;
            }
            if (++tried > kDpMaxSearch) return false;
            bool ok = (eq[depth] >> v) & 1;
            for (uint32_t i = 0; i < depth && ok; ++i) ok = E(i, depth) == E(cand[i], v);
            if (depth + 1 == n) {
                // the last vertex: only the single unused one is tried
                if (!(identity[depth] && v == depth) && ok) {
                    cand[depth] = v;
                    if (++found > kDpMaxAut) return false;
                    for (uint32_t i = 0; i < np; ++i) {
                        const uint32_t w = porder[i];
                        if (cand[w] != w) {
                            uint32_t& r = out.restricts[cand[w]];
                            if (r == kDpNone || r < w) r = w;
                            break;
                        }
                    }
                }
                nextv[depth] = n;  // as the reference, stop after the first unused vertex
                continue;
            }
            if (!ok) {
                nextv[depth] = v + 1;
                continue;
            }
            cand[depth] = v;
            used |= bit(v);
            identity[depth + 1] = identity[depth] && v == depth;
            ++depth;
            nextv[depth] = 0;
        }
        return true;
    }

    // src/genMatchOrderCPU.cpp:508-667
    GVA_HD bool rearrange() {
        // reduce keys, largest first; entries of one key in insertion order
        for (uint32_t i = 1; i < nred; ++i) {  // stable, descending key
            RedRef x = red[i];
            uint32_t j = i;
            while (j > 0 && red[j - 1].key < x.key) {
                red[j] = red[j - 1];
                --j;
            }
            red[j] = x;
        }
        out.nrep = out.nstat = 0;
        auto rep_find = [&](uint64_t k) -> int {
            for (uint32_t i = 0; i < out.nrep; ++i)
                if (out.rep_key[i] == k) return (int)i;
            return -1;
        };
        auto rep_set = [&](uint64_t k, uint32_t v) -> bool {  // ascending key
            int at = rep_find(k);
            if (at >= 0) {
                out.rep_val[at] = v;
                return true;
            }
            if (out.nrep >= (uint32_t)kDpKeys) return false;
            uint32_t i = out.nrep;
            while (i > 0 && out.rep_key[i - 1] > k) {
                out.rep_key[i] = out.rep_key[i - 1];
                out.rep_val[i] = out.rep_val[i - 1];
                --i;
            }
            out.rep_key[i] = k;
            out.rep_val[i] = v;
            out.nrep++;
            return true;
        };
        auto note_stat = [&](uint64_t k) -> bool {
            const uint32_t e = (uint32_t)(k >> 32), v = (uint32_t)(k & 0xffffffffu);
            for (uint32_t i = 0; i < out.nstat; ++i)
                if (out.stat_el[i] == e && out.stat_vl[i] == v) return true;
            if (out.nstat >= (uint32_t)kDpKeys) return false;
            uint32_t i = out.nstat;
            while (i > 0 && (out.stat_el[i - 1] > e || (out.stat_el[i - 1] == e && out.stat_vl[i - 1] > v))) {
                out.stat_el[i] = out.stat_el[i - 1];
                out.stat_vl[i] = out.stat_vl[i - 1];
                --i;
            }
            out.stat_el[i] = e;
            out.stat_vl[i] = v;
            out.nstat++;
            return true;
        };
        for (uint32_t i = 0; i < nred;) {
            uint32_t j = i;
            const uint64_t k = red[i].key;
            for (; j < nred && red[j].key == k; ++j) {
                uint8_t* pr = out.pairs + out.ph_at[red[j].phase];
                if (ql(pr[2 * red[j].pair]) == (uint32_t)(k & 0xffffffffu)) swap_(pr[2 * red[j].pair], pr[2 * red[j].pair + 1]);
            }
            // the count is driven to zero, once per partner
            if (!rep_set(k, 0)) return false;
            i = j;
        }
        for (int m = 0; m < 2; ++m) {
            const KeyCount* keys = m == 0 ? ext_keys : other_keys;
            const uint32_t nk = m == 0 ? next_keys : nother_keys;
            for (uint32_t i = 0; i < nk; ++i) {
                const int at = rep_find(keys[i].key);
                if (at < 0) {
                    if (!rep_set(keys[i].key, (keys[i].count << 16) | keys[i].count)) return false;
                    if (keys[i].count > 1 && !note_stat(keys[i].key)) return false;
                } else {
                    out.rep_val[at] += keys[i].count;
                    if (out.rep_val[at] > 1 && !note_stat(keys[i].key)) return false;
                }
            }
        }
        return true;
    }

    GVA_HD void run() {
        out.status = DPLAN_HOST;
        out.vnum = q.n;
        out.nphase = out.npair = out.nrep = out.nstat = out.ncol = 0;
        if (!setup() || !seed() || !grow() || !restrictions() || !rearrange()) return;
        // output columns: the first phase's source, then every extended vertex
        out.columns[out.ncol++] = out.pairs[out.ph_at[0]];
        for (uint32_t p = 0; p < out.nphase; ++p) {
            if (out.ph_type[p] != 'E') continue;
            for (uint32_t i = 1; i < 2u * out.ph_np[p]; i += 2) {
                if (out.ncol >= (uint32_t)kDpV) return;
                out.columns[out.ncol++] = out.pairs[out.ph_at[p] + i];
            }
        }
        out.status = DPLAN_OK;
    }
};

}  // namespace dplan_detail

// Plans one query (DV mode); out.status DPLAN_HOST when it is left to the
// host planner.
GVA_HD inline void dplan(const DPlanQuery& q, DPlan& out) {
    dplan_detail::DPlanner p(q, out);
    p.run();
}

}  // namespace gva
