// Host side of the database: .mygraph/.metadata parsing, edge-list builder,
// and the lowering of a plan to engine steps.
#include <algorithm>
#include <atomic>
#include <thread>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

#include "../../include/geneva.h"
#include "gva_dplan.h"
#include "gva_internal.h"

namespace gva {

static thread_local std::string g_err = "no error";

void set_error(int status, const std::string& msg) {
    (void)status;
    g_err = msg;
}
int fail(int status, const std::string& msg) {
    set_error(status, msg);
    return status;
}
const char* last_error_cstr() { return g_err.c_str(); }

uint32_t HostGraph::dense_label(uint32_t orig) const {
    auto it = std::lower_bound(labels.begin(), labels.end(), orig);
    if (it == labels.end() || *it != orig) return kNone;
    return (uint32_t)(it - labels.begin());
}

namespace {

// Sorted distinct labels and each vertex's dense label.  Labels are few
// against vertices: they are collected in an open-addressing table (label ->
// dense index, filled in once the distinct labels are sorted).
void finish_labels(HostGraph& g) {
    std::vector<uint64_t> tab(64, ~0ull);  // label << 32 | dense index; ~0: empty
    size_t count = 0;
    auto slot = [&](uint32_t l) -> uint64_t& {
        const size_t m = tab.size() - 1;
        size_t i = (size_t)((l * 0x9e3779b97f4a7c15ull) >> 32) & m;
        while (tab[i] != ~0ull && (uint32_t)(tab[i] >> 32) != l) i = (i + 1) & m;
        return tab[i];
    };
    std::vector<uint32_t> ls;
    uint32_t last = kNone;
    for (uint32_t v = 1; v <= g.max_id; ++v) {
        const uint32_t l = g.vlabel[v];
        if (l == kNone || l == last) continue;
        last = l;
        uint64_t& t = slot(l);
        if (t != ~0ull) continue;
        t = (uint64_t)l << 32;
        ls.push_back(l);
        if (2 * ++count > tab.size()) {  // grow: re-file the labels seen so far
            tab.assign(tab.size() * 2, ~0ull);
            for (uint32_t x : ls) slot(x) = (uint64_t)x << 32;
        }
    }
    std::sort(ls.begin(), ls.end());
    for (size_t i = 0; i < ls.size(); ++i) slot(ls[i]) = ((uint64_t)ls[i] << 32) | i;
    g.labels = ls;
    g.dlabel.assign(g.max_id + 1, kNone);
    last = kNone;
    uint32_t last_dense = kNone;
    for (uint32_t v = 1; v <= g.max_id; ++v) {
        const uint32_t l = g.vlabel[v];
        if (l == kNone) continue;
        if (l != last) last = l, last_dense = (uint32_t)(slot(l) & 0xffffffffu);
        g.dlabel[v] = last_dense;
    }
}

// Number of index vertices genDatabase prepends to a label group of raw
// length n (tools/genDatabase.cpp:415-436, decoded as src/loadDataBase.cpp:71-98).
uint32_t index_prefix(uint32_t n) {
    if (n <= 128) return 0;
    if (n <= 32 * 128 + 32) return (n + 128) / 129;
    return 32;
}

}  // namespace

namespace {

// istream >> uint32_t on text held in memory: leading white space, an
// optional sign ('-' negates modulo 2^32), at least one digit; false where
// the stream would fail (no digit, or a value above 2^32 - 1).
bool read_u32(const char*& p, const char* end, uint32_t& out) {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r' || *p == '\v' || *p == '\f')) ++p;
    if (p == end) return false;
    bool neg = false;
    if (*p == '+' || *p == '-') neg = *p++ == '-';
    if (p == end || *p < '0' || *p > '9') return false;
    uint64_t x = 0;
    while (p < end && *p >= '0' && *p <= '9') {
        x = x * 10 + (uint64_t)(*p++ - '0');
        if (x > 0xffffffffull) return false;
    }
    out = neg ? (uint32_t)(0u - (uint32_t)x) : (uint32_t)x;
    return true;
}

}  // namespace

int load_mygraph(const std::string& mygraph, const std::string& metadata, HostGraph& g, std::string* warnings) {
    // ---- .metadata: "newid label oldid" (src/loadDataBase.cpp:320-340) ----
    std::ifstream mf(metadata, std::ios::binary | std::ios::ate);
    if (!mf.is_open()) return fail(GVA_ERR_IO, "cannot open metadata file " + metadata);
    std::string text;
    {
        const std::streamoff size = mf.tellg();
        text.resize(size > 0 ? (size_t)size : 0);
        mf.seekg(0);
        if (size > 0 && !mf.read(&text[0], size)) return fail(GVA_ERR_IO, "cannot read metadata file " + metadata);
    }
    std::vector<std::pair<uint32_t, uint32_t>> vl;
    uint32_t maxid = 0;
    {
        const char* p = text.data();
        const char* end = p + text.size();
        uint32_t nid, lab, oid;
        while (read_u32(p, end, nid) && read_u32(p, end, lab) && read_u32(p, end, oid)) {
            vl.push_back({nid, lab});
            maxid = std::max(maxid, nid);
        }
    }
    if (vl.empty()) return fail(GVA_ERR_FORMAT, "metadata file has no vertices");
    g = HostGraph();
    g.max_id = maxid;
    g.vlabel.assign(maxid + 1, kNone);
    for (auto& p : vl)
        if (p.first != 0 && g.vlabel[p.first] == kNone) g.vlabel[p.first] = p.second;  // first wins
    finish_labels(g);

    // ---- .mygraph: uint32 P, then P partitions (tools/genDatabase.cpp:856-869) ----
    std::ifstream gf(mygraph, std::ios::binary);
    if (!gf.is_open()) return fail(GVA_ERR_IO, "cannot open graph file " + mygraph);
    uint32_t P = 0;
    if (!gf.read((char*)&P, 4)) return fail(GVA_ERR_FORMAT, "graph file is empty");
    const uint64_t V = (uint64_t)maxid + 1, L = g.num_labels();
    const unsigned nth = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<uint32_t> part;
    std::vector<uint64_t> cnt(V), start(V + 1);
    std::vector<uint32_t> last(V);
    for (uint32_t key = 1; key <= P; ++key) {
        uint32_t tot = 0;
        if (!gf.read((char*)&tot, 4)) {
            // The shipped Enron.mygraph declares 4 partitions and holds 3.
            if (warnings) *warnings += "graph header declares " + std::to_string(P) + " partitions, file holds " +
                                       std::to_string(key - 1) + "\n";
            break;
        }
        if (tot < 5) return fail(GVA_ERR_FORMAT, "partition shorter than its header");
        part.resize(tot);
        part[0] = tot;
        if (!gf.read((char*)&part[1], (std::streamsize)(tot - 1) * 4)) return fail(GVA_ERR_FORMAT, "truncated partition");
        // header: [1] source slots, [2] intervals, [3]/[4] hash/neighbour offsets from word 5
        const uint64_t nslot = part[1], nint = part[2];
        const uint64_t slots_at = 5 + 2 * nint + 2, nbr_at = 5 + (uint64_t)part[4];
        if (part[3] != part[4]) return fail(GVA_ERR_UNSUPPORTED, "hash-indexed partitions are not supported");
        if (slots_at + nslot + 1 > tot || nbr_at > tot || 5 + 2 * nint + 1 > tot)
            return fail(GVA_ERR_FORMAT, "partition offsets out of range");
        const uint64_t nnbr = tot - nbr_at;
        const uint32_t* start_v = &part[5];
        const uint32_t* cum = &part[5 + nint + 1];
        const uint32_t* soff = &part[slots_at];
        const uint32_t* nbr = &part[nbr_at];
        if (soff[nslot] > nnbr) return fail(GVA_ERR_FORMAT, "neighbour offsets beyond partition");
        if (soff[nslot] < nnbr && warnings)
            *warnings += "partition " + std::to_string(key) +
                         " holds neighbours of sources beyond its 256 intervals (dropped, as the reference)\n";
        // every source slot's neighbours, split into vertex-label groups, each
        // group without its index prefix; `visit(v, x)` gets them in order
        auto walk = [&](bool check, auto&& visit) -> int {
            uint32_t prev = 0;
            for (uint64_t i = 0; i < nint; ++i) {
                if (check && (cum[i] < prev || cum[i] > nslot)) return fail(GVA_ERR_FORMAT, "interval lengths not cumulative");
                for (uint32_t s = prev; s < cum[i]; ++s) {
                    const uint64_t v = (uint64_t)start_v[i] + (s - prev);
                    if (check && (v == 0 || v > maxid)) return fail(GVA_ERR_FORMAT, "source vertex id outside metadata");
                    const uint32_t b = soff[s], e = soff[s + 1];
                    if (check && (b > e || e > nnbr)) return fail(GVA_ERR_FORMAT, "bad neighbour range");
                    uint32_t j = b;
                    while (j < e) {
                        const uint32_t u0 = nbr[j];
                        if (check && (u0 == 0 || u0 > maxid || g.vlabel[u0] == kNone))
                            return fail(GVA_ERR_FORMAT, "neighbour id outside metadata");
                        uint32_t k = j;
                        while (k < e && nbr[k] != 0 && nbr[k] <= maxid && g.vlabel[nbr[k]] == g.vlabel[u0]) ++k;
                        for (uint32_t t = j + index_prefix(k - j); t < k; ++t)
                            if (int rc = visit(v, nbr[t])) return rc;
                        j = k;
                    }
                }
                prev = cum[i];
            }
            return GVA_OK;
        };
        // pass 1: checks and list lengths (a list's groups must ascend
        // strictly within a label, as the lists are appended slot by slot)
        std::fill(cnt.begin(), cnt.end(), 0);
        std::fill(last.begin(), last.end(), 0);
        int rc = walk(true, [&](uint64_t v, uint32_t x) -> int {
            const uint32_t b = last[v];
            if (b != 0 && g.dlabel[b] == g.dlabel[x] && b >= x)
                return fail(GVA_ERR_FORMAT, "neighbour group not strictly ascending");
            last[v] = x;
            cnt[v]++;
            return GVA_OK;
        });
        if (rc) return rc;
        start[0] = 0;
        for (uint64_t v = 0; v < V; ++v) start[v + 1] = start[v] + cnt[v];
        const uint64_t total = start[V];
        const uint64_t entries = V * L + 1;
        if (entries >= 0xffffffffull) return fail(GVA_ERR_UNSUPPORTED, "vertex count x label count exceeds 2^32");
        if (total >= 0xffffffffull) return fail(GVA_ERR_UNSUPPORTED, "partition has 2^32 or more adjacency entries");
        HostPartition hp;
        hp.edge_label = key;
        hp.adj.resize(total);
        // pass 2: the lists, flat in vertex order
        std::fill(cnt.begin(), cnt.end(), 0);
        walk(false, [&](uint64_t v, uint32_t x) -> int {
            hp.adj[start[v] + cnt[v]++] = x;
            return GVA_OK;
        });
        // (vertex, label) offsets by vertex ranges; a list must be grouped by
        // non-decreasing dense label
        hp.off.resize(entries);
        std::atomic<bool> ungrouped{false};
        auto fill_range = [&](uint64_t v0, uint64_t v1) {
            for (uint64_t v = v0; v < v1; ++v) {
                const uint64_t at = start[v], n = start[v + 1] - at;
                uint64_t j = 0;
                for (uint64_t l = 0; l < L; ++l) {
                    hp.off[v * L + l] = (uint32_t)(at + j);
                    while (j < n && g.dlabel[hp.adj[at + j]] == l) ++j;
                }
                if (j != n) ungrouped = true;
            }
        };
        if (nth == 1 || V < (1u << 16)) {
            fill_range(0, V);
        } else {
            std::vector<std::thread> pool;
            for (unsigned t = 0; t < nth; ++t) pool.emplace_back(fill_range, V * t / nth, V * (t + 1) / nth);
            for (auto& th : pool) th.join();
        }
        if (ungrouped) return fail(GVA_ERR_FORMAT, "neighbour list is not grouped by vertex label");
        hp.off[entries - 1] = (uint32_t)total;
        if (g.parts.size() < key) g.parts.resize(key);
        g.parts[key - 1] = std::move(hp);
    }
    if (g.parts.empty()) return fail(GVA_ERR_FORMAT, "graph file holds no partition");
    return GVA_OK;
}

void seed_groups(const HostGraph& g, std::vector<uint32_t>& seed_off, std::vector<uint32_t>& seed_verts,
                 std::vector<uint32_t>& seed_by_degree) {
    const uint32_t L = g.num_labels();
    seed_off.assign(L + 1, 0);
    for (uint32_t v = 1; v <= g.max_id; ++v)
        if (g.dlabel[v] != kNone) seed_off[g.dlabel[v] + 1]++;
    for (uint32_t l = 0; l < L; ++l) seed_off[l + 1] += seed_off[l];
    seed_verts.resize(seed_off[L]);
    {
        std::vector<uint32_t> fill(seed_off.begin(), seed_off.end() - 1);
        for (uint32_t v = 1; v <= g.max_id; ++v)
            if (g.dlabel[v] != kNone) seed_verts[fill[g.dlabel[v]]++] = v;
    }
    // total degree over all edge labels; within a label group the vertices
    // are in ascending id, so a stable counting sort by degree (largest
    // first) gives (degree descending, id ascending)
    std::vector<uint32_t> deg(g.max_id + 1, 0);
    for (auto& p : g.parts)
        if (!p.off.empty())
            for (uint32_t v = 0; v <= g.max_id; ++v) deg[v] += p.off[(uint64_t)(v + 1) * L] - p.off[(uint64_t)v * L];
    seed_by_degree.resize(seed_verts.size());
    std::vector<uint32_t> cnt;
    for (uint32_t l = 0; l < L; ++l) {
        const uint32_t b = seed_off[l], e = seed_off[l + 1];
        uint32_t dmax = 0;
        for (uint32_t i = b; i < e; ++i) dmax = std::max(dmax, deg[seed_verts[i]]);
        cnt.assign((size_t)dmax + 2, 0);
        for (uint32_t i = b; i < e; ++i) cnt[dmax - deg[seed_verts[i]] + 1]++;  // rank 0 = largest degree
        for (size_t r = 1; r < cnt.size(); ++r) cnt[r] += cnt[r - 1];
        for (uint32_t i = b; i < e; ++i) seed_by_degree[b + cnt[dmax - deg[seed_verts[i]]]++] = seed_verts[i];
    }
}

int graph_from_edges(const uint32_t* vlabels, uint32_t max_id, const uint32_t* src, const uint32_t* dst,
                     const uint32_t* elabel, uint64_t ne, HostGraph& g) {
    if (!vlabels || (ne && (!src || !dst || !elabel))) return fail(GVA_ERR_ARG, "null array");
    if (max_id == 0) return fail(GVA_ERR_ARG, "max_vertex_id must be >= 1");
    g = HostGraph();
    g.max_id = max_id;
    g.vlabel.assign(vlabels, vlabels + max_id + 1);
    g.vlabel[0] = kNone;
    finish_labels(g);
    uint32_t P = 0;
    for (uint64_t i = 0; i < ne; ++i) {
        if (elabel[i] == 0) return fail(GVA_ERR_ARG, "edge labels must be >= 1");
        if (src[i] == 0 || dst[i] == 0 || src[i] > max_id || dst[i] > max_id)
            return fail(GVA_ERR_ARG, "edge endpoint outside 1..max_vertex_id");
        P = std::max(P, elabel[i]);
    }
    for (uint64_t i = 0; i < ne; ++i)  // every endpoint is some vertex's neighbour
        if (g.dlabel[src[i]] == kNone || g.dlabel[dst[i]] == kNone)
            return fail(GVA_ERR_ARG, "edge endpoint without a vertex label");
    const uint64_t L = g.num_labels();
    const uint64_t entries = (uint64_t)(max_id + 1) * L + 1;
    if (P && entries >= 0xffffffffull) return fail(GVA_ERR_UNSUPPORTED, "vertex count x label count exceeds 2^32");
    // Per edge label: both directions of every edge bucketed by source
    // (counting sort), each source's neighbours sorted by (dense label, id)
    // with repeated edges removed, on the host's cores; then the (vertex,
    // label) offsets.  Same arrays as sorting all entries at once.
    const unsigned nth = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    const uint64_t V = (uint64_t)max_id + 1;
    g.parts.resize(P);
    // Edge labels in groups whose bucket tables and entries stay within a
    // memory bound; each group's entries are bucketed by source in one
    // counting and one scatter pass over the edges: pos_all[p - p0][v] is
    // where vertex v's bucket starts in keys_all[p - p0]
    std::vector<uint64_t> per_label(P + 1, 0);
    for (uint64_t i = 0; i < ne; ++i) per_label[elabel[i]]++;
    constexpr uint64_t kGroupBytes = 1ull << 30;
    std::vector<uint64_t> len(V), start(V);
    for (uint32_t p0 = 1, p1; p0 <= P; p0 = p1 + 1) {
        uint64_t bytes = (V + 1) * 8 + 16 * per_label[p0];
        for (p1 = p0; p1 < P && bytes + (V + 1) * 8 + 16 * per_label[p1 + 1] <= kGroupBytes; ++p1)
            bytes += (V + 1) * 8 + 16 * per_label[p1 + 1];
        const uint32_t G = p1 - p0 + 1;
        std::vector<std::vector<uint64_t>> pos_all(G, std::vector<uint64_t>(V + 1, 0)), keys_all(G);
        for (uint64_t i = 0; i < ne; ++i) {
            if (elabel[i] < p0 || elabel[i] > p1) continue;
            std::vector<uint64_t>& c = pos_all[elabel[i] - p0];
            c[src[i] + 1]++, c[dst[i] + 1]++;
        }
        for (uint32_t q = 0; q < G; ++q) {
            std::vector<uint64_t>& c = pos_all[q];
            for (uint64_t v = 0; v < V; ++v) c[v + 1] += c[v];
            keys_all[q].resize(c[V]);
        }
        {
            std::vector<std::vector<uint64_t>> cur(G);
            for (uint32_t q = 0; q < G; ++q) cur[q].assign(pos_all[q].begin(), pos_all[q].end() - 1);
            for (uint64_t i = 0; i < ne; ++i) {  // (dense label << 32) | neighbour
                if (elabel[i] < p0 || elabel[i] > p1) continue;
                const uint32_t q = elabel[i] - p0;
                keys_all[q][cur[q][src[i]]++] = ((uint64_t)g.dlabel[dst[i]] << 32) | dst[i];
                keys_all[q][cur[q][dst[i]]++] = ((uint64_t)g.dlabel[src[i]] << 32) | src[i];
            }
        }
        for (uint32_t p = p0; p <= p1; ++p) {
            const std::vector<uint64_t>& pos = pos_all[p - p0];
            std::vector<uint64_t> keys;
            keys.swap(keys_all[p - p0]);
            auto sort_range = [&](uint64_t v0, uint64_t v1) {
                for (uint64_t v = v0; v < v1; ++v) {
                    uint64_t* a = keys.data() + pos[v];
                    uint64_t* b = keys.data() + pos[v + 1];
                    std::sort(a, b);
                    len[v] = (uint64_t)(std::unique(a, b) - a);
                }
            };
            if (nth == 1 || keys.size() < (1u << 16)) {
                sort_range(0, V);
            } else {
                // vertex ranges of about equal entry counts
                std::vector<std::thread> pool;
                uint64_t v0 = 0;
                for (unsigned t = 0; t < nth; ++t) {
                    const uint64_t target = pos[V] * (t + 1) / nth;
                    uint64_t v1 = t + 1 == nth ? V : (uint64_t)(std::lower_bound(pos.begin(), pos.end(), target) - pos.begin());
                    v1 = std::min(std::max(v1, v0), V);
                    pool.emplace_back(sort_range, v0, v1);
                    v0 = v1;
                }
                for (auto& th : pool) th.join();
            }
            uint64_t total = 0;  // start[v]: where vertex v's list starts in adj
            for (uint64_t v = 0; v < V; ++v) {
                const uint64_t l = len[v];
                start[v] = total;
                total += l;
            }
            if (total >= 0xffffffffull) return fail(GVA_ERR_UNSUPPORTED, "partition has 2^32 or more adjacency entries");
            HostPartition& part = g.parts[p - 1];
            part.edge_label = p;
            part.off.resize(entries);  // group (v, l) starts at off[v * L + l]
            part.adj.resize(total);
            // each vertex's offsets and list, written by vertex ranges: its list
            // is sorted by label, so group l starts after the entries of labels < l
            auto fill_range = [&](uint64_t v0, uint64_t v1) {
                for (uint64_t v = v0; v < v1; ++v) {
                    const uint64_t* a = keys.data() + pos[v];
                    const uint64_t at = start[v], n = len[v];
                    uint64_t j = 0;
                    for (uint64_t l = 0; l < L; ++l) {
                        part.off[v * L + l] = (uint32_t)(at + j);
                        while (j < n && (a[j] >> 32) == l) {
                            part.adj[at + j] = (uint32_t)a[j];
                            ++j;
                        }
                    }
                }
            };
            if (nth == 1 || V < (1u << 16)) {
                fill_range(0, V);
            } else {
                std::vector<std::thread> pool;
                for (unsigned t = 0; t < nth; ++t) pool.emplace_back(fill_range, V * t / nth, V * (t + 1) / nth);
                for (auto& th : pool) th.join();
            }
            part.off[entries - 1] = (uint32_t)total;
        }
    }
    if (g.parts.empty()) g.parts.resize(1);
    return GVA_OK;
}

// ---------------------------------------------------------------------------
// Plan -> steps.  Column c of a row holds plan.columns[c].
//   init, one pair (s,e)      : seed(label s) + ext(s->e, e < s iff restricted to s)
//                               (cpumine genInit 2V, src/cpumine.cpp:60-119: no injectivity test)
//   init, two pairs (s,e1,e2) : seed + ext(s->e1, e1 <= s) + ext(s->e2, e2 < e1 or e2 <= s,
//                               e2 != e1) (src/cpumine.cpp:120-194)
//   E, one pair               : ext(s->e, injective against same-label columns, e < row[restrict])
//   E, two pairs              : two such exts; the second also avoids the first
//                               (src/cpumine.cpp:298-435)
//   R                         : reduce over all pairs (src/cpumine.cpp:486-584); more than
//                               16 pairs empties the frontier as the reference does (:499-502)
// The plan read through a small view, so that host plans and plans from the
// heap-free planner (gva_dplan.h) lower through the same code.
struct PlanView {
    const Plan& p;
    struct Ph {
        const Phase& ph;
        char type() const { return ph.type; }
        uint32_t edge_label() const { return ph.edge_label; }
        size_t npairs() const { return ph.pairs.size() / 2; }
        uint32_t pair(size_t k) const { return ph.pairs[k]; }
    };
    uint32_t vnum() const { return p.vnum; }
    int mode() const { return p.mode; }
    uint32_t qlabel(uint32_t v) const { return p.qlabel[v]; }
    uint32_t restrict_of(uint32_t v) const { return p.restricts[v]; }
    size_t nphase() const { return p.phases.size(); }
    Ph phase(size_t i) const { return Ph{p.phases[i]}; }
};

struct DPlanView {
    const DPlan& d;
    const uint32_t* labels;
    struct Ph {
        const DPlan& d;
        size_t i;
        char type() const { return (char)d.ph_type[i]; }
        uint32_t edge_label() const { return d.ph_el[i]; }
        size_t npairs() const { return d.ph_np[i]; }
        uint32_t pair(size_t k) const { return d.pairs[d.ph_at[i] + k]; }
    };
    uint32_t vnum() const { return d.vnum; }
    int mode() const { return GVA_MODE_DV; }
    uint32_t qlabel(uint32_t v) const { return labels[v]; }
    uint32_t restrict_of(uint32_t v) const { return d.restricts[v]; }
    size_t nphase() const { return d.nphase; }
    Ph phase(size_t i) const { return Ph{d, i}; }
};

template <typename View>
int lower_core(const View& plan, const HostGraph& g, std::vector<Step>& steps, bool fuse_reductions) {
    steps.clear();
    steps.reserve(2 * plan.nphase() + 1);  // a phase lowers to at most two steps, the first one plus a seed
    int newest = -1;  // query vertex added by the last extension step
    const uint32_t P = (uint32_t)g.parts.size();
    if (plan.vnum() > (uint32_t)kMaxCols) return fail(GVA_ERR_UNSUPPORTED, "query has more than 32 vertices");
    int col[kMaxCols];
    for (uint32_t v = 0; v < plan.vnum(); ++v) col[v] = -1;
    int width = 0;
    auto part_of = [&](uint32_t el) -> uint32_t { return (el >= 1 && el <= P && !g.parts[el - 1].off.empty()) ? el : 0; };
    struct EqCols {  // columns of matched vertices with the new vertex's label, ascending
        uint32_t n = 0;
        int c[kMaxCols];
    };
    auto ext = [&](uint32_t el, uint32_t s, uint32_t e, int bound_col, bool incl, const EqCols& eq) {
        Step st;
        st.kind = STEP_EXT;
        st.width_in = (uint32_t)width;
        st.part = part_of(el);
        st.label = g.dense_label(plan.qlabel(e));
        st.src_col = col[s];
        st.bound_col = bound_col;
        st.bound_inclusive = incl ? 1 : 0;
        st.n_eq = eq.n;
        for (uint32_t i = 0; i < eq.n; ++i) st.eq_cols[i] = (uint8_t)eq.c[i];
        st.always_empty = (st.part == 0 || st.label == kNone) ? 1 : 0;
        steps.push_back(st);
        col[e] = width++;
        newest = (int)e;
    };
    auto same_label_cols = [&](uint32_t e) {
        EqCols eq;
        for (uint32_t v = 0; v < plan.vnum(); ++v)
            if (col[v] >= 0 && plan.qlabel(v) == plan.qlabel(e)) eq.c[eq.n++] = col[v];
        std::sort(eq.c, eq.c + eq.n);
        return eq;
    };
    for (size_t pi = 0; pi < plan.nphase(); ++pi) {
        const auto ph = plan.phase(pi);
        const size_t np = ph.npairs();
        if (pi == 0) {
            if (ph.type() != 'E' || np < 1 || np > 2) return fail(GVA_ERR_FORMAT, "first phase must extend 1 or 2 vertices");
            const uint32_t s = ph.pair(0);
            Step seed;
            seed.kind = STEP_SEED;
            seed.width_in = 0;
            seed.part = part_of(ph.edge_label());
            seed.label = g.dense_label(plan.qlabel(s));
            seed.always_empty = (seed.part == 0 || seed.label == kNone) ? 1 : 0;
            steps.push_back(seed);
            col[s] = width++;
            if (np == 1 || plan.mode() == GVA_MODE_SV) {
                const uint32_t e = ph.pair(1);
                ext(ph.edge_label(), s, e, plan.restrict_of(e) == s ? 0 : -1, false, EqCols());
            } else {
                const uint32_t e1 = ph.pair(1), e2 = ph.pair(3);
                ext(ph.edge_label(), s, e1, plan.restrict_of(e1) != kNone ? 0 : -1, true, EqCols());
                EqCols eq;
                if (plan.qlabel(e2) == plan.qlabel(e1)) eq.c[eq.n++] = col[e1];
                if (plan.restrict_of(e2) == e1)
                    ext(ph.edge_label(), s, e2, col[e1], false, eq);
                else
                    ext(ph.edge_label(), s, e2, plan.restrict_of(e2) != kNone ? 0 : -1, true, eq);
            }
            steps.back().phase_end = 0;
            continue;
        }
        if (ph.type() == 'E') {
            for (size_t i = 0; i < np; ++i) {
                const uint32_t s = ph.pair(2 * i), e = ph.pair(2 * i + 1);
                if (col[s] < 0) return fail(GVA_ERR_FORMAT, "extension from an unmatched vertex");
                int bc = -1;
                if (plan.restrict_of(e) != kNone) {
                    bc = col[plan.restrict_of(e)];
                    if (bc < 0) return fail(GVA_ERR_FORMAT, "restriction names an unmatched vertex");
                }
                ext(ph.edge_label(), s, e, bc, false, same_label_cols(e));
            }
        } else {
            // fold into the previous extension when every pair touches its new vertex
            if (fuse_reductions && !steps.empty() && steps.back().kind == STEP_EXT && newest >= 0 &&
                !steps.back().always_empty && np <= 8 - steps.back().n_chk && np <= GVA_MAX_REDUCE_PAIRS) {
                bool ok = true;
                for (size_t i = 0; i < np && ok; ++i)
                    ok = (int)ph.pair(2 * i) == newest || (int)ph.pair(2 * i + 1) == newest;
                if (ok) {
                    Step& st = steps.back();
                    const uint32_t part = part_of(ph.edge_label());
                    if (part == 0) st.always_empty = 1;
                    for (size_t i = 0; i < np; ++i) {
                        const uint32_t a = ph.pair(2 * i), b = ph.pair(2 * i + 1);
                        const bool new_is_b = (int)b == newest;  // pair checks b in adj(a) with label(b)
                        const uint32_t other = new_is_b ? a : b;
                        st.chk_col[st.n_chk] = (uint8_t)col[other];
                        st.chk_dir[st.n_chk] = new_is_b ? 0 : 1;
                        st.chk_part[st.n_chk] = part;
                        st.chk_lab[st.n_chk] = g.dense_label(plan.qlabel(b));
                        if (st.chk_lab[st.n_chk] == kNone) st.always_empty = 1;
                        st.n_chk++;
                    }
                    st.phase_end = (int)pi;
                    continue;
                }
            }
            Step st;
            st.kind = STEP_REDUCE;
            st.width_in = (uint32_t)width;
            st.part = part_of(ph.edge_label());
            if (np > GVA_MAX_REDUCE_PAIRS) {
                st.always_empty = 1;
            } else {
                st.n_pairs = (uint32_t)np;
                for (size_t i = 0; i < np; ++i) {
                    const uint32_t a = ph.pair(2 * i), b = ph.pair(2 * i + 1);
                    if (col[a] < 0 || col[b] < 0) return fail(GVA_ERR_FORMAT, "reduction over an unmatched vertex");
                    st.rs_col[i] = (uint8_t)col[a];
                    st.re_col[i] = (uint8_t)col[b];
                    st.re_label[i] = g.dense_label(plan.qlabel(b));
                    if (st.re_label[i] == kNone) st.always_empty = 1;
                }
                if (st.part == 0) st.always_empty = 1;
            }
            steps.push_back(st);
        }
        steps.back().phase_end = (int)pi;
    }
    return GVA_OK;
}

int lower_plan(const Plan& plan, const HostGraph& g, std::vector<Step>& steps, bool fuse_reductions) {
    return lower_core(PlanView{plan}, g, steps, fuse_reductions);
}

int lower_dplan(const DPlan& plan, const uint32_t* labels, const HostGraph& g, std::vector<Step>& steps,
                bool fuse_reductions) {
    if (plan.status != DPLAN_OK) return fail(GVA_ERR_ARG, "query was left to the host planner");
    return lower_core(DPlanView{plan, labels}, g, steps, fuse_reductions);
}

}  // namespace gva
