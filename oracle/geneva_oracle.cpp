// Test infrastructure only: the CPU oracle (see geneva_oracle.h).
//
// Restates, in memory and single-threaded:
//   planner   src/genMatchOrderCPU.cpp:69-983  (query parse, triangle seed,
//             growth loop, automorphisms, restrictions, reduce-pair orientation)
//   matcher   src/cpumine.cpp:54-196  genInit
//             src/cpumine.cpp:198-439 genExtEmb
//             src/cpumine.cpp:486-584 reduction
// State lives in one object per call instead of the reference's globals.
#include "geneva_oracle.h"

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <list>
#include <map>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

typedef uint32_t uint;
static const uint NONE = 0xffffffffu;
static thread_local std::string g_err;

struct oracle_graph {
    // parts[edge label][svid][vertex label] = ascending neighbour ids
    std::vector<std::unordered_map<uint, std::map<uint, std::vector<uint>>>> parts;
    std::vector<uint> vlabel;  // index = vertex id
};

namespace {

// ------------------------------------------------------------------ graph --
int fail(const std::string& m) {
    g_err = m;
    return 1;
}

int load_graph(const char* mygraph, const char* metadata, oracle_graph& g) {
    std::ifstream mf(metadata);
    if (!mf) return fail("metadata missing");
    uint nid, lab, oid, maxid = 0;
    std::vector<std::pair<uint, uint>> v;
    while (mf >> nid >> lab >> oid) {
        v.push_back({nid, lab});
        maxid = std::max(maxid, nid);
    }
    g.vlabel.assign(maxid + 1, NONE);
    for (auto& p : v)
        if (g.vlabel[p.first] == NONE) g.vlabel[p.first] = p.second;
    std::ifstream f(mygraph, std::ios::binary);
    if (!f) return fail("graph missing");
    uint P;
    f.read((char*)&P, 4);
    g.parts.assign(1, {});
    for (uint key = 1; key <= P; ++key) {
        uint tot;
        if (!f.read((char*)&tot, 4)) break;  // header may overstate the partition count
        std::vector<uint> a(tot);
        a[0] = tot;
        f.read((char*)&a[1], (std::streamsize)(tot - 1) * 4);
        const uint nint = a[2];
        const uint slot0 = 5 + 2 * nint + 2;
        const uint nbr0 = 5 + a[4];
        g.parts.push_back({});
        auto& part = g.parts.back();
        uint prev = 0;
        for (uint i = 0; i < nint; ++i) {
            const uint start = a[5 + i], cum = a[5 + nint + 1 + i];
            for (uint s = prev; s < cum; ++s) {
                const uint vid = start + (s - prev);
                const uint b = a[slot0 + s], e = a[slot0 + s + 1];
                auto& byl = part[vid];
                // group by end-vertex label, dropping genDatabase's index vertices
                // (tools/genDatabase.cpp:415-436; decode as src/loadDataBase.cpp:71-98)
                uint j = b;
                while (j < e) {
                    const uint l = g.vlabel[a[nbr0 + j]];
                    uint k = j;
                    while (k < e && g.vlabel[a[nbr0 + k]] == l) ++k;
                    const uint n = k - j;
                    const uint idx = n <= 128 ? 0 : (n <= 4128 ? (n + 128) / 129 : 32);
                    auto& lst = byl[l];
                    for (uint t = j + idx; t < k; ++t) lst.push_back(a[nbr0 + t]);
                    j = k;
                }
            }
            prev = cum;
        }
    }
    return 0;
}

int graph_from_edges(const uint* vl, uint maxid, const uint* src, const uint* dst, const uint* el, uint64_t ne,
                     oracle_graph& g) {
    g.vlabel.assign(vl, vl + maxid + 1);
    g.vlabel[0] = NONE;
    uint P = 0;
    for (uint64_t i = 0; i < ne; ++i) P = std::max(P, el[i]);
    g.parts.assign(P + 1, {});
    for (uint64_t i = 0; i < ne; ++i) {
        auto& part = g.parts[el[i]];
        // both directions, duplicates ignored (tools/genDatabase.cpp:600-667)
        for (int d = 0; d < 2; ++d) {
            const uint s = d ? dst[i] : src[i], t = d ? src[i] : dst[i];
            auto& lst = part[s][g.vlabel[t]];
            if (std::find(lst.begin(), lst.end(), t) == lst.end()) lst.push_back(t);
        }
    }
    for (auto& part : g.parts)
        for (auto& kv : part)
            for (auto& kv2 : kv.second) std::sort(kv2.second.begin(), kv2.second.end());
    return 0;
}

// ---------------------------------------------------------------- planner --
struct Phase {
    char phaseType;
    uint edgeLabel;
    std::vector<uint> pairs;
};

struct QNeig {  // queryNeigInfo
    uint neigs = 0;
    std::map<uint, std::vector<uint>> edgeLabelNeigs;  // label -> {count, mask}
};
struct QEdge {
    uint svid, evid, edgeLabel;
};
struct Tri {
    uint edgeIndex, triCount, triScore, maxScoreVID;
};
struct NInfo {
    uint commonVNum, svid, evid, edgeLabel, evLabel, evNum;
};
struct KeyCount {
    uint64_t key = 0;
    uint count = 0;
    std::vector<uint64_t> keyList;
    std::vector<uint> phaseList;
};

struct Planner {
    uint partialQueryVidMap = 0;
    std::list<uint> partialQueryVid;
    std::vector<uint> vertexNeig, adjMatrix;
    uint vnum = 0;
    std::map<uint, uint> queryLabel;
    std::vector<QNeig> query;
    std::vector<QEdge> edges;
    std::vector<Phase> matchOrder;
    std::map<uint64_t, uint> repeatFlag;
    std::map<uint, uint> restricts;
    std::map<uint, std::map<uint, bool>> stat;
    std::map<uint64_t, uint> extKC, othersKC;
    std::map<uint64_t, KeyCount> redKC;
    bool ok = true;

    void addToQueryGraph(uint s, uint e, uint el) {
        query[s].neigs |= (1u << e);
        auto it = query[s].edgeLabelNeigs.find(el);
        if (it != query[s].edgeLabelNeigs.end()) {
            it->second[0] += 1;
            it->second[1] |= (1u << e);
        } else {
            query[s].edgeLabelNeigs[el] = {1u, 1u << e};
        }
    }

    void countTriangle(uint ei, std::vector<Tri>& r) {
        QEdge& ed = edges[ei];
        uint tri = vertexNeig[ed.svid] & vertexNeig[ed.evid];
        r[ei].edgeIndex = ei;
        r[ei].triCount = __builtin_popcount(tri);
        if (!tri) return;
        int prei = -1, prescore = -1;
        for (uint i = 0; i < 32; ++i) {
            if (!((1u << i) & tri)) continue;
            uint e1l = adjMatrix[ed.svid * vnum + i], e2l = adjMatrix[ed.evid * vnum + i], e3l = ed.edgeLabel;
            int es = ((e1l == e2l) + (e1l == e3l) + (e2l == e3l)) * 10;
            uint v1 = queryLabel[ed.svid], v2 = queryLabel[ed.evid], v3 = queryLabel[i];
            int vs = (v1 == v2) + (v1 == v3) + (v2 == v3);
            if (vs + es > prescore) {
                prescore = vs + es;
                prei = (int)i;
            }
        }
        r[ei].triScore = (uint)prescore;
        r[ei].maxScoreVID = (uint)prei;
    }

    void initNoTriangle(uint& svid, uint& e1, uint& e2) {
        uint gS = NONE, gF = 0, gS2 = 0, gFE = NONE, gSE = NONE;
        std::map<uint64_t, std::vector<uint>> A, B, C;
        for (uint i = 0; i < vnum; ++i) {
            for (auto& kv : query[i].edgeLabelNeigs) {
                uint64_t ksve = ((uint64_t)kv.first << 20) | i;
                uint neigs = kv.second[1];
                if (__builtin_popcount(neigs) >= 2) {
                    std::map<uint, std::vector<uint>> t;
                    for (uint k = 0; k < 32; ++k)
                        if (neigs & (1u << k)) t[queryLabel[k]].push_back(k);
                    for (auto& g : t) {
                        uint64_t k3 = ((uint64_t)g.first << 40) | ksve;
                        if (g.second.size() >= 2)
                            A.insert({k3, g.second});
                        else {
                            auto& v = B[ksve];
                            v.insert(v.end(), g.second.begin(), g.second.end());
                        }
                    }
                } else {
                    for (uint k = 0; k < 32; ++k)
                        if (neigs & (1u << k)) C[(uint64_t)i].push_back(k);
                }
            }
        }
        std::map<uint64_t, std::vector<uint>>& T = A.size() ? A : (B.size() ? B : C);
        for (auto& kv : T) {
            uint f = 0, s = 0, fe = NONE, se = NONE;
            for (uint ev : kv.second) {
                uint tn = __builtin_popcount(query[ev].neigs);
                if (tn > f) {
                    s = f;
                    se = fe;
                    f = tn;
                    fe = ev;
                } else if (tn > s) {
                    s = tn;
                    se = ev;
                }
            }
            if (A.size() || B.size()) {
                if (f + s > gF + gS2) {
                    gF = f;
                    gFE = fe;
                    gS2 = s;
                    gSE = se;
                    gS = (uint)(kv.first & 0xfffff);
                }
            } else if (f > gF) {
                gF = f;
                gFE = fe;
                gS = (uint)(kv.first & 0xfffff);
            }
        }
        svid = gS;
        e1 = gFE;
        e2 = gSE;
    }

    void addExt(uint s1, uint x1, uint s2, uint x2, uint num) {
        if (num == 2 && queryLabel[x2] < queryLabel[x1]) {
            std::swap(s1, s2);
            std::swap(x1, x2);
        }
        Phase p{'E', adjMatrix[s1 * vnum + x1], {s1, x1}};
        extKC[((uint64_t)p.edgeLabel << 32) | queryLabel[x1]] += 1;
        partialQueryVidMap |= (1u << x1);
        partialQueryVid.push_back(x1);
        vertexNeig[s1] &= ~(1u << x1);
        vertexNeig[x1] &= ~(1u << s1);
        if (num == 2) {
            p.pairs.push_back(s2);
            p.pairs.push_back(x2);
            extKC[((uint64_t)adjMatrix[s2 * vnum + x2] << 32) | queryLabel[x2]] += 1;
            partialQueryVidMap |= (1u << x2);
            partialQueryVid.push_back(x2);
            vertexNeig[s2] &= ~(1u << x2);
            vertexNeig[x2] &= ~(1u << s2);
        }
        matchOrder.push_back(p);
    }

    void addReduce(const std::vector<uint>& pairs) {
        Phase p{'R', 0, {}};
        for (uint i = 0; i < pairs.size() / 2; ++i) {
            uint a = pairs[2 * i], b = pairs[2 * i + 1];
            p.pairs.push_back(a);
            p.pairs.push_back(b);
            vertexNeig[a] &= ~(1u << b);
            vertexNeig[b] &= ~(1u << a);
            p.edgeLabel = adjMatrix[a * vnum + b];
            uint64_t key = ((uint64_t)p.edgeLabel << 32) | queryLabel[b];
            uint64_t key1 = ((uint64_t)adjMatrix[a * vnum + b] << 32) | queryLabel[a];
            if (key == key1) {
                othersKC[key] += 1;
            } else {
                for (int t = 0; t < 2; ++t) {
                    uint64_t k = t ? key1 : key, other = t ? key : key1;
                    KeyCount& kc = redKC[k];
                    kc.key = k;
                    kc.count += 1;
                    kc.keyList.push_back(other);
                    kc.phaseList.push_back((uint)matchOrder.size());
                    kc.phaseList.push_back(i);
                }
            }
        }
        matchOrder.push_back(p);
    }

    bool isEquivalent(uint a, uint b) {
        if (a == b) return true;
        if (queryLabel[a] != queryLabel[b]) return false;
        auto& na = query[a].edgeLabelNeigs;
        auto& nb = query[b].edgeLabelNeigs;
        if (na.size() != nb.size()) return false;
        for (auto i = na.begin(), j = nb.begin(); i != na.end(); ++i, ++j)
            if (i->first != j->first || i->second[0] != j->second[0]) return false;
        return true;
    }
    bool isPossibleAut(std::vector<uint>& c, uint nid) {
        uint ori = (uint)c.size();
        if (!isEquivalent(ori, nid)) return false;
        for (uint i = 0; i < c.size(); ++i)
            if (adjMatrix[i * vnum + ori] != adjMatrix[c[i] * vnum + nid]) return false;
        return true;
    }
    void genAut(std::vector<uint> c, bool isId, std::vector<std::vector<uint>>& out) {
        if (c.size() == vnum - 1) {
            for (uint i = 0; i < vnum; ++i) {
                if (std::find(c.begin(), c.end(), i) != c.end()) continue;
                if (isId && i == c.size()) return;
                if (isPossibleAut(c, i)) {
                    c.push_back(i);
                    out.push_back(c);
                }
                break;
            }
        } else {
            for (uint i = 0; i < vnum; ++i) {
                if (std::find(c.begin(), c.end(), i) != c.end()) continue;
                if (isPossibleAut(c, i)) {
                    c.push_back(i);
                    genAut(c, isId && (i == c.size() - 1), out);
                    c.pop_back();
                }
            }
        }
    }
    void genRestriction(std::vector<std::vector<uint>> auts) {
        std::vector<bool> vis(vnum, false);
        for (auto& ph : matchOrder) {
            if (ph.phaseType == 'R') continue;
            for (uint v : ph.pairs) {
                if (vis[v]) continue;
                vis[v] = true;
                std::vector<std::vector<uint>> st;
                for (auto& a : auts) {
                    if (a[v] == v)
                        st.push_back(a);
                    else {
                        auto it = restricts.find(a[v]);
                        if (it == restricts.end())
                            restricts[a[v]] = v;
                        else if (it->second < v)
                            it->second = v;
                    }
                }
                auts = st;
            }
        }
        for (uint i = 0; i <= vnum; ++i)
            if (!restricts.count(i)) restricts[i] = NONE;
    }
    void noteStat(uint64_t key) { stat[(uint)(key >> 32)][(uint)(key & 0xffffffffu)] = true; }
    void rearrange() {
        uint iters = (uint)redKC.size();
        for (uint j = 0; j < iters; ++j) {
            // the reference's selection never raises its running maximum: last key wins
            auto maxite = redKC.begin();
            uint pre = 0;
            for (auto it = redKC.begin(); it != redKC.end(); ++it) {
                uint c = (extKC.count(it->first) ? extKC[it->first] : 0) +
                         (othersKC.count(it->first) ? othersKC[it->first] : 0) + it->second.count;
                if (c > pre) maxite = it;
            }
            uint64_t key = maxite->first;
            KeyCount& kc = maxite->second;
            for (size_t i = 0; i < kc.keyList.size(); ++i)
                if (kc.count > 0) kc.count -= 1;
            for (size_t i = 0; i < kc.phaseList.size() / 2; ++i) {
                auto& pr = matchOrder[kc.phaseList[2 * i]].pairs;
                uint pi = kc.phaseList[2 * i + 1];
                if (queryLabel[pr[2 * pi]] == (uint)(key & 0xffffffffu)) std::swap(pr[2 * pi], pr[2 * pi + 1]);
            }
            repeatFlag[key] = (kc.count << 16) | kc.count;
            if (kc.count > 1) noteStat(key);
            redKC.erase(key);
        }
        for (auto* m : {&extKC, &othersKC})
            for (auto& kv : *m) {
                auto it = repeatFlag.find(kv.first);
                if (it == repeatFlag.end()) {
                    repeatFlag[kv.first] = (kv.second << 16) | kv.second;
                    if (kv.second > 1) noteStat(kv.first);
                } else {
                    it->second += kv.second;
                    if (it->second > 1) noteStat(kv.first);
                }
            }
    }

    bool parse(const std::string& text) {
        std::istringstream q(text);
        char type;
        while (q.get(type)) {
            if (type == 'v') {
                uint vid, vl;
                q >> vid >> vl;
                if (!queryLabel.count(vid)) queryLabel[vid] = vl;
            } else if (type == 'e') {
                break;
            } else if (type == '#') {
                std::string dummy;
                std::getline(q, dummy);
            }
        }
        q.unget();
        vnum = (uint)queryLabel.size();
        query.assign(vnum, QNeig());
        adjMatrix.assign(vnum * vnum, NONE);
        vertexNeig.assign(vnum, 0);
        while (q.get(type)) {
            if (type != 'e') continue;
            uint s, e, l;
            if (!(q >> s >> e >> l)) break;
            addToQueryGraph(s, e, l);
            addToQueryGraph(e, s, l);
            if (adjMatrix[s * vnum + e] == NONE) {
                edges.push_back({std::min(s, e), std::max(s, e), l});
                adjMatrix[s * vnum + e] = l;
                adjMatrix[e * vnum + s] = l;
            }
            vertexNeig[s] |= 1u << e;
            vertexNeig[e] |= 1u << s;
        }
        return vnum > 0 && !edges.empty();
    }

    bool plan(const std::string& text) {
        if (!parse(text)) return false;
        std::vector<Tri> tc(edges.size(), Tri{0, 0, 0, 0});
        for (uint i = 0; i < edges.size(); ++i) countTriangle(i, tc);
        std::sort(tc.begin(), tc.end(), [](const Tri& a, const Tri& b) { return a.triCount > b.triCount; });
        if (tc[0].triCount == 0) {
            uint s, x1, x2;
            initNoTriangle(s, x1, x2);
            partialQueryVid.push_back(s);
            partialQueryVidMap |= 1u << s;
            addExt(s, x1, s, x2, x2 == NONE ? 1 : 2);
        } else {
            uint tcnt = tc[0].triCount, i = 1, prei = 0;
            while (i < tc.size() && tc[i].triCount == tcnt) {
                if (tc[i].triScore > tc[prei].triScore) prei = i;
                ++i;
            }
            uint score = tc[prei].triScore;
            QEdge& ed = edges[tc[prei].edgeIndex];
            uint sv = ed.svid, ev = ed.evid, th = tc[prei].maxScoreVID;
            if (score == 33 || score == 31 || score == 30 || (score >= 10 && score <= 13)) {
                uint so = sv, x1 = ev, x2 = th;
                if (score == 31) {
                    if (queryLabel[sv] == queryLabel[ev]) { so = th; x1 = sv; x2 = ev; }
                    else if (queryLabel[sv] == queryLabel[th]) { so = ev; x1 = sv; x2 = th; }
                    else if (queryLabel[ev] == queryLabel[th]) { so = sv; x1 = ev; x2 = th; }
                } else if (score >= 10 && score <= 13) {
                    uint e1l = adjMatrix[sv * vnum + th], e2l = adjMatrix[ev * vnum + th], e3l = ed.edgeLabel;
                    if (e1l == e2l) { so = th; x1 = sv; x2 = ev; }
                    else if (e1l == e3l) { so = sv; x1 = ev; x2 = th; }
                    else if (e2l == e3l) { so = ev; x1 = sv; x2 = th; }
                }
                partialQueryVid.push_back(so);
                partialQueryVidMap |= 1u << so;
                addExt(so, x1, so, x2, 2);
                addReduce({x1, x2});
            } else if (score <= 3) {
                partialQueryVid.push_back(sv);
                partialQueryVidMap |= 1u << sv;
                addExt(sv, ev, sv, th, 1);
                addExt(sv, th, sv, th, 1);
                addReduce({ev, th});
            } else {
                return false;
            }
        }
        int guard = 0;
        while (partialQueryVid.size() < vnum) {
            if (++guard > 64) return false;  // disconnected pattern
            std::vector<NInfo> info;
            std::map<uint, std::vector<uint>> same;
            for (uint s : partialQueryVid) {
                uint neigs = vertexNeig[s];
                for (uint i = 0; i < 32; ++i) {
                    if (!(neigs & (1u << i))) continue;
                    NInfo n;
                    n.svid = s;
                    n.evid = i;
                    n.edgeLabel = adjMatrix[s * vnum + i];
                    n.commonVNum = (uint)__builtin_popcount(vertexNeig[i] & partialQueryVidMap) - 1;
                    n.evLabel = queryLabel[i];
                    n.evNum = __builtin_popcount(neigs & query[s].edgeLabelNeigs[n.edgeLabel][1]);
                    info.push_back(n);
                    if (!((1u << i) & partialQueryVidMap)) {
                        same[n.edgeLabel].push_back(s);
                        same[n.edgeLabel].push_back(i);
                    }
                }
            }
            if (info.empty()) return false;
            std::sort(info.begin(), info.end(), [](const NInfo& a, const NInfo& b) {
                if (a.commonVNum > b.commonVNum) return true;
                if (a.commonVNum == b.commonVNum) {
                    if (a.evNum > b.evNum) return true;
                    if (a.evNum == b.evNum) {
                        if (a.edgeLabel < b.edgeLabel) return true;
                        if (a.edgeLabel == b.edgeLabel) {
                            if (a.svid < b.svid) return true;
                            if (a.svid == b.svid && a.evLabel < b.evLabel) return true;
                        }
                    }
                }
                return false;
            });
            if (info[0].commonVNum > 0) {
                uint so = info[0].svid, x1 = info[0].evid;
                addExt(so, x1, 0, 0, 1);
                std::vector<NInfo> back;
                uint np = vertexNeig[x1] & partialQueryVidMap;
                for (uint i = 0; i < 32; ++i)
                    if (np & (1u << i)) back.push_back(NInfo{0, x1, i, adjMatrix[x1 * vnum + i], queryLabel[i], 0});
                std::sort(back.begin(), back.end(), [](const NInfo& a, const NInfo& b) {
                    if (a.edgeLabel < b.edgeLabel) return true;
                    if (a.edgeLabel == b.edgeLabel) return a.evLabel < b.evLabel;
                    return false;
                });
                uint prei = 0;
                std::vector<uint> prev;
                for (uint i = 0; i < back.size(); ++i) {
                    if (back[i].edgeLabel == back[prei].edgeLabel) {
                        prev.push_back(back[i].svid);
                        prev.push_back(back[i].evid);
                    } else {
                        addReduce(prev);
                        prev.clear();
                        prei = i;
                        --i;
                    }
                }
                addReduce(prev);
            } else {
                bool found = false;
                for (auto& kv : same) {
                    auto& ev = kv.second;
                    for (uint i = 0; i < ev.size() / 2 && !found; ++i)
                        for (uint j = i + 1; j < ev.size() / 2; ++j)
                            if (adjMatrix[ev[2 * i + 1] * vnum + ev[2 * j + 1]] != NONE) {
                                found = true;
                                addExt(ev[2 * i], ev[2 * i + 1], ev[2 * j], ev[2 * j + 1], 2);
                                addReduce({ev[2 * i + 1], ev[2 * j + 1]});
                                break;
                            }
                    if (found) break;
                }
                if (!found) {
                    if (info[0].evNum > 1) {
                        addExt(info[0].svid, info[0].evid, info[1].svid, info[1].evid, 2);
                    } else {
                        bool f2 = false;
                        for (uint i = 0; i + 1 < info.size(); ++i)
                            if (info[i].edgeLabel == info[i + 1].edgeLabel) {
                                addExt(info[i].svid, info[i].evid, info[i + 1].svid, info[i + 1].evid, 2);
                                f2 = true;
                                break;
                            }
                        if (!f2) addExt(info[0].svid, info[0].evid, 0, 0, 1);
                    }
                }
            }
        }
        std::vector<std::vector<uint>> auts;
        genAut({}, true, auts);
        rearrange();
        genRestriction(auts);
        return true;
    }

    std::string describe() {
        std::ostringstream o;
        o << "vnum " << vnum << "\n";
        for (size_t i = 0; i < matchOrder.size(); ++i) {
            auto& p = matchOrder[i];
            o << "phase " << i << " " << p.phaseType << " " << p.edgeLabel << " " << p.pairs.size() / 2;
            for (uint v : p.pairs) o << " " << v;
            o << "\n";
        }
        for (auto& kv : restricts) o << "restrict " << kv.first << " " << kv.second << "\n";
        char b[32];
        for (auto& kv : repeatFlag) {
            snprintf(b, sizeof b, "%x", kv.second);
            o << "repeat " << (uint)(kv.first >> 32) << " " << (uint)(kv.first & 0xffffffffu) << " " << b << "\n";
        }
        for (auto& kv : stat)
            for (auto& kv2 : kv.second) o << "stat " << kv.first << " " << kv2.first << "\n";
        return o.str();
    }
};

// ---------------------------------------------------------------- matcher --
struct CapExceeded {};

struct Matcher {
    const oracle_graph& g;
    Planner& P;
    uint64_t cap_words = 0;  // 0 = unlimited; else abort when a frontier grows past it
    void check(const std::vector<uint>& out) const {
        if (cap_words && out.size() > cap_words) throw CapExceeded();
    }
    std::map<uint, uint> pos;               // posOfVisitedV
    std::map<uint, std::vector<uint>> eq;   // equalPos
    std::vector<uint> cur;                  // current frontier, row-major
    uint width = 0;

    Matcher(const oracle_graph& gg, Planner& pp) : g(gg), P(pp) {}

    const std::vector<uint>* nbrs(uint el, uint v, uint vl) const {
        if (el >= g.parts.size()) return nullptr;
        auto it = g.parts[el].find(v);
        if (it == g.parts[el].end()) return nullptr;
        auto jt = it->second.find(vl);
        return jt == it->second.end() ? nullptr : &jt->second;
    }
    uint lab(uint v) const { return v < g.vlabel.size() ? g.vlabel[v] : NONE; }

    // src/cpumine.cpp:54-196
    void init(Phase& ph) {
        const uint el = ph.edgeLabel;
        std::vector<uint> out;
        if (el >= g.parts.size()) { cur.clear(); width = ph.pairs.size() == 2 ? 2 : 3; return; }
        if (ph.pairs.size() == 2) {
            uint s = ph.pairs[0], e = ph.pairs[1];
            pos[s] = 0;
            pos[e] = 1;
            uint sl = P.queryLabel[s], elb = P.queryLabel[e];
            bool restrict_ = P.restricts[e] == s;
            if (sl == elb) eq[sl] = {0, 1};
            else { eq[sl] = {0}; eq[elb] = {1}; }
            for (auto& kv : g.parts[el]) {
                uint v = kv.first;
                if (lab(v) != sl) continue;
                auto it = kv.second.find(elb);
                if (it == kv.second.end()) continue;
                for (uint u : it->second)
                    if (!restrict_ || v > u) { out.push_back(v); out.push_back(u); }
            }
            width = 2;
        } else {
            uint s = ph.pairs[0], e1 = ph.pairs[1], e2 = ph.pairs[3];
            uint sl = P.queryLabel[s], l1 = P.queryLabel[e1], l2 = P.queryLabel[e2];
            pos[s] = 0; pos[e1] = 1; pos[e2] = 2;
            bool r1 = P.restricts[e1] != NONE;
            bool r12 = P.restricts[e2] != NONE ? P.restricts[e2] == e1 : false;
            bool r2 = r12 ? false : P.restricts[e2] != NONE;
            if (sl == l1 && sl == l2) eq[sl] = {0, 1, 2};
            else if (sl == l1) { eq[sl] = {0, 1}; eq[l2] = {2}; }
            else if (sl == l2) { eq[sl] = {0, 2}; eq[l1] = {1}; }
            else if (l1 == l2) { eq[sl] = {0}; eq[l1] = {1, 2}; }
            else { eq[sl] = {0}; eq[l1] = {1}; eq[l2] = {2}; }
            for (auto& kv : g.parts[el]) {
                uint v = kv.first;
                if (lab(v) != sl) continue;
                auto a = kv.second.find(l1), b = kv.second.find(l2);
                if (a == kv.second.end() || b == kv.second.end()) continue;
                for (uint x : a->second)
                    for (uint y : b->second) {
                        if (y == x) continue;
                        if (r1 && v < x) continue;
                        if (r2 && v < y) continue;
                        if (r12 && x < y) continue;
                        out.push_back(v); out.push_back(x); out.push_back(y);
                    }
                check(out);
            }
            width = 3;
        }
        cur.swap(out);
    }

    // src/cpumine.cpp:198-439
    void extend(Phase& ph) {
        const uint el = ph.edgeLabel;
        const uint pre = width;
        std::vector<uint> out;
        if (ph.pairs.size() == 2) {
            uint s = ph.pairs[0], e = ph.pairs[1];
            pos[e] = (uint)pos.size();
            uint elb = P.queryLabel[e];
            bool rs = P.restricts[e] != NONE;
            if (eq.count(elb)) eq[elb].push_back(pos[e]);
            else eq[elb] = {pos[e]};
            const uint sp = pos[s];
            const uint rp = rs ? pos[P.restricts[e]] : 0;
            for (size_t r = 0; r + pre <= cur.size() && pre; r += pre) {
                const uint* row = &cur[r];
                auto* nb = nbrs(el, row[sp], elb);
                if (!nb) continue;
                for (uint u : *nb) {
                    bool found = false;
                    for (uint k = 0; k < pre; ++k) found |= (row[k] == u);
                    if (found) continue;
                    if (rs && !(row[rp] > u)) continue;
                    out.insert(out.end(), row, row + pre);
                    out.push_back(u);
                }
                check(out);
            }
            width = pre + 1;
        } else {
            uint s1 = ph.pairs[0], e1 = ph.pairs[1], s2 = ph.pairs[2], e2 = ph.pairs[3];
            uint idx = (uint)pos.size();
            pos[e1] = idx;
            pos[e2] = idx + 1;
            uint l1 = P.queryLabel[e1], l2 = P.queryLabel[e2];
            bool r1 = P.restricts[e1] != NONE;
            bool r12 = P.restricts[e2] != NONE ? P.restricts[e2] == e1 : false;
            bool r2 = r12 ? false : P.restricts[e2] != NONE;
            eq[l1].push_back(pos[e1]);
            eq[l2].push_back(pos[e2]);
            const uint p1 = pos[s1], p2 = pos[s2];
            const uint rp1 = r1 ? pos[P.restricts[e1]] : 0, rp2 = r2 ? pos[P.restricts[e2]] : 0;
            for (size_t r = 0; r + pre <= cur.size() && pre; r += pre) {
                const uint* row = &cur[r];
                auto* n1 = nbrs(el, row[p1], l1);
                auto* n2 = nbrs(el, row[p2], l2);
                if (!n1 || !n2) continue;
                for (uint x : *n1) {
                    bool found = false;
                    for (uint k = 0; k < pre; ++k) found |= (row[k] == x);
                    if (found) continue;
                    if (r1 && x > row[rp1]) continue;
                    for (uint y : *n2) {
                        bool f2 = false;
                        for (uint k = 0; k < pre; ++k) f2 |= (row[k] == y);
                        if (f2 || y == x) continue;
                        if (r2 && y > row[rp2]) continue;
                        if (r12 && y > x) continue;
                        out.insert(out.end(), row, row + pre);
                        out.push_back(x);
                        out.push_back(y);
                    }
                    check(out);
                }
            }
            width = pre + 2;
        }
        cur.swap(out);
    }

    // src/cpumine.cpp:486-584 (more than 16 pairs: the reference emits nothing)
    void reduce(Phase& ph) {
        if (ph.pairs.size() > 32) { cur.clear(); return; }
        const uint el = ph.edgeLabel;
        std::vector<uint> out;
        for (size_t r = 0; r + width <= cur.size() && width; r += width) {
            const uint* row = &cur[r];
            bool all = true;
            for (size_t j = 0; j < ph.pairs.size() / 2 && all; ++j) {
                uint a = ph.pairs[2 * j], b = ph.pairs[2 * j + 1];
                auto* nb = nbrs(el, row[pos[a]], P.queryLabel[b]);
                all = nb && std::find(nb->begin(), nb->end(), row[pos[b]]) != nb->end();
            }
            if (all) out.insert(out.end(), row, row + width);
        }
        cur.swap(out);
    }

    std::vector<uint64_t> run() {
        std::vector<uint64_t> counts;
        for (size_t i = 0; i < P.matchOrder.size(); ++i) {
            Phase& ph = P.matchOrder[i];
            if (i == 0) init(ph);
            else if (ph.phaseType == 'E') extend(ph);
            else reduce(ph);
            counts.push_back(width ? cur.size() / width : 0);
            if (cur.empty()) {
                // later phases still widen the rows but stay empty
                for (size_t j = i + 1; j < P.matchOrder.size(); ++j) {
                    counts.push_back(0);
                    if (P.matchOrder[j].phaseType == 'E') width += (uint)P.matchOrder[j].pairs.size() / 2;
                }
                break;
            }
        }
        return counts;
    }
};

}  // namespace

extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

int oracle_graph_load(const char* mygraph, const char* metadata, oracle_graph** out) {
    oracle_graph* g = new oracle_graph();
    if (load_graph(mygraph, metadata, *g)) {
        delete g;
        return 1;
    }
    *out = g;
    return 0;
}

int oracle_graph_from_edges(const uint32_t* vl, uint32_t maxid, const uint32_t* src, const uint32_t* dst,
                            const uint32_t* el, uint64_t ne, oracle_graph** out) {
    oracle_graph* g = new oracle_graph();
    graph_from_edges(vl, maxid, src, dst, el, ne, *g);
    *out = g;
    return 0;
}

void oracle_graph_free(oracle_graph* g) { delete g; }

size_t oracle_plan(const char* text, char* buf, size_t cap) {
    Planner p;
    if (!p.plan(text)) return 0;
    std::string s = p.describe();
    if (buf && cap) {
        size_t n = std::min(cap - 1, s.size());
        memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return s.size();
}

int oracle_match(const oracle_graph* g, const char* text, uint32_t** rows, uint64_t* nrows, int* width,
                 uint64_t* phase_rows, int cap, int* nphases) {
    Planner p;
    if (!p.plan(text)) return fail("planner failed");
    Matcher m(*g, p);
    std::vector<uint64_t> c = m.run();
    *width = (int)m.width;
    *nrows = m.width ? m.cur.size() / m.width : 0;
    *rows = (uint32_t*)malloc(std::max<size_t>(1, m.cur.size()) * 4);
    if (!m.cur.empty()) memcpy(*rows, m.cur.data(), m.cur.size() * 4);
    for (int i = 0; i < (int)c.size() && i < cap; ++i) phase_rows[i] = c[i];
    if (nphases) *nphases = (int)c.size();
    return 0;
}

int oracle_count(const oracle_graph* g, const char* text, uint64_t* nrows) {
    return oracle_count_capped(g, text, 0, nrows);
}

int oracle_count_capped(const oracle_graph* g, const char* text, uint64_t cap_rows, uint64_t* nrows) {
    Planner p;
    if (!p.plan(text)) return fail("planner failed");
    Matcher m(*g, p);
    m.cap_words = cap_rows * 32;
    try {
        m.run();
    } catch (const CapExceeded&) {
        *nrows = 0;
        return 2;
    }
    *nrows = m.width ? m.cur.size() / m.width : 0;
    return 0;
}

int oracle_graph_counts(const oracle_graph* g, const char* text, const int64_t* first, uint32_t G, uint64_t* counts,
                        uint64_t* nrows) {
    Planner p;
    if (!p.plan(text)) return fail("planner failed");
    Matcher m(*g, p);
    m.run();
    for (uint32_t i = 0; i < G; ++i) counts[i] = 0;
    const uint64_t n = m.width ? m.cur.size() / m.width : 0;
    *nrows = n;
    for (uint64_t r = 0; r < n; ++r) {
        const int64_t v = m.cur[r * m.width];
        // graph of v: the last i with first[i] <= v
        const int64_t* it = std::upper_bound(first, first + G + 1, v);
        const int64_t i = (it - first) - 1;
        if (i >= 0 && i < (int64_t)G) ++counts[i];
    }
    return 0;
}

void oracle_free(void* p) { free(p); }

}  // extern "C"

// ---------------------------------------------------------------- MNI ------
// Test infrastructure: the CPU statement of minimum image-based support.
struct oracle_mni_graph {
    uint n = 0;
    std::vector<uint> vlabel;                 // original label per id (0..n)
    std::vector<std::vector<uint>> by_label;  // original label -> vertex ids (ascending)
    // adjacency per edge label: adj[el][v] = neighbours sorted by (label, id)
    std::vector<std::vector<std::vector<uint>>> adj;
};

namespace {

struct MniPat {
    uint n = 0;
    uint vl[8];
    uint el[8][8];
};

bool parse_mni_pattern(const char* text, MniPat& p) {
    std::istringstream in(text);
    std::string t;
    std::vector<std::pair<uint, uint>> vs;
    std::vector<std::array<uint, 3>> es;
    while (in >> t) {
        if (t == "v") {
            uint a, b;
            in >> a >> b;
            vs.push_back({a, b});
        } else if (t == "e") {
            uint a, b, c;
            in >> a >> b >> c;
            es.push_back({a, b, c});
        } else {
            return false;
        }
    }
    if (vs.empty() || vs.size() > 8) return false;
    p.n = (uint)vs.size();
    memset(p.el, 0, sizeof p.el);
    for (auto& v : vs) {
        if (v.first >= p.n) return false;
        p.vl[v.first] = v.second;
    }
    for (auto& e : es) {
        if (e[0] >= p.n || e[1] >= p.n) return false;
        p.el[e[0]][e[1]] = p.el[e[1]][e[0]] = e[2];
    }
    return true;
}

// all vertex permutations that keep labels and edges; orbit[v] = min image
void mni_orbits(const MniPat& p, uint* orbit) {
    uint perm[8];
    for (uint i = 0; i < p.n; ++i) perm[i] = i, orbit[i] = i;
    do {
        bool ok = true;
        for (uint i = 0; i < p.n && ok; ++i) ok = p.vl[perm[i]] == p.vl[i];
        for (uint i = 0; i < p.n && ok; ++i)
            for (uint j = 0; j < p.n && ok; ++j) ok = p.el[perm[i]][perm[j]] == p.el[i][j];
        if (ok)
            for (uint i = 0; i < p.n; ++i) orbit[i] = std::min(orbit[i], perm[i]);
    } while (std::next_permutation(perm, perm + p.n));
    for (int it = 0; it < 8; ++it)
        for (uint i = 0; i < p.n; ++i) orbit[i] = orbit[orbit[i]];
}

struct MniSearch {
    const oracle_mni_graph& g;
    const MniPat& p;
    uint order[8];
    uint f[8];
    // neighbours of v (edge label el) with vertex label lab
    std::pair<const uint*, const uint*> seg(uint v, uint el, uint lab) const {
        if (el >= g.adj.size() || g.adj[el].empty()) return {nullptr, nullptr};
        const std::vector<uint>& a = g.adj[el][v];
        auto lo = std::lower_bound(a.begin(), a.end(), lab, [&](uint w, uint l) { return g.vlabel[w] < l; });
        auto hi = std::upper_bound(lo, a.end(), lab, [&](uint l, uint w) { return l < g.vlabel[w]; });
        return {a.data() + (lo - a.begin()), a.data() + (hi - a.begin())};
    }
    bool extend(uint k) {
        if (k == p.n) return true;
        const uint u = order[k];
        // candidates: neighbours of the first matched neighbour of u
        uint j0 = 8;
        for (uint j = 0; j < k && j0 == 8; ++j)
            if (p.el[u][order[j]]) j0 = j;
        auto s = seg(f[j0], p.el[u][order[j0]], p.vl[u]);
        for (const uint* c = s.first; c != s.second; ++c) {
            bool ok = true;
            for (uint j = 0; j < k && ok; ++j) {
                if (f[j] == *c) ok = false;
                else if (j != j0 && p.el[u][order[j]]) {
                    auto t = seg(f[j], p.el[u][order[j]], p.vl[u]);
                    ok = std::binary_search(t.first, t.second, *c,
                                            [&](uint a, uint b) { return g.vlabel[a] != g.vlabel[b] ? g.vlabel[a] < g.vlabel[b] : a < b; });
                }
            }
            if (!ok) continue;
            f[k] = *c;
            if (extend(k + 1)) return true;
        }
        return false;
    }
};

}  // namespace

extern "C" {

int oracle_mni_graph_from_edges(const uint32_t* vl, uint32_t maxid, const uint32_t* src, const uint32_t* dst,
                                const uint32_t* el, uint64_t ne, oracle_mni_graph** out) {
    oracle_mni_graph* g = new oracle_mni_graph();
    g->n = maxid;
    g->vlabel.assign(vl, vl + maxid + 1);
    uint maxl = 0, P = 0;
    for (uint v = 1; v <= maxid; ++v) maxl = std::max(maxl, g->vlabel[v]);
    g->by_label.assign(maxl + 1, {});
    for (uint v = 1; v <= maxid; ++v) g->by_label[g->vlabel[v]].push_back(v);
    for (uint64_t i = 0; i < ne; ++i) P = std::max(P, el[i]);
    g->adj.assign(P + 1, {});
    for (uint l = 1; l <= P; ++l) g->adj[l].assign(maxid + 1, {});
    for (uint64_t i = 0; i < ne; ++i) {
        g->adj[el[i]][src[i]].push_back(dst[i]);
        g->adj[el[i]][dst[i]].push_back(src[i]);
    }
    for (auto& part : g->adj)
        for (auto& l : part) {
            std::sort(l.begin(), l.end(), [&](uint a, uint b) {
                return g->vlabel[a] != g->vlabel[b] ? g->vlabel[a] < g->vlabel[b] : a < b;
            });
            l.erase(std::unique(l.begin(), l.end()), l.end());
        }
    *out = g;
    return 0;
}

void oracle_mni_graph_free(oracle_mni_graph* g) { delete g; }

int oracle_mni(const oracle_mni_graph* g, const char* text, uint32_t cap, uint32_t* support, uint64_t* searches) {
    MniPat p;
    if (!parse_mni_pattern(text, p)) return fail("bad pattern text");
    if (cap == 0) cap = NONE;
    uint orbit[8];
    mni_orbits(p, orbit);
    uint best = cap;
    uint64_t ns = 0;
    for (uint r = 0; r < p.n; ++r) {
        if (orbit[r] != r) continue;
        MniSearch s{*g, p, {}, {}};
        // search order: breadth-first from r, pattern vertex ids ascending
        uint seen = 1u << r, k = 1;
        s.order[0] = r;
        for (uint h = 0; h < k; ++h)
            for (uint w = 0; w < p.n; ++w)
                if (p.el[s.order[h]][w] && !(seen >> w & 1)) {
                    seen |= 1u << w;
                    s.order[k++] = w;
                }
        if (k != p.n) return fail("pattern is not connected");
        uint count = 0;
        if (p.vl[r] < g->by_label.size())
            for (uint v : g->by_label[p.vl[r]]) {
                if (count >= best) break;
                s.f[0] = v;
                ++ns;
                if (s.extend(1)) ++count;
            }
        best = std::min(best, count);
    }
    *support = best;
    if (searches) *searches = ns;
    return 0;
}

}  // extern "C"
