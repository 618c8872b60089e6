// .g -> .mygraph / .metadata / .reorder converter, byte-identical to the
// reference converter tools/genDatabase.cpp on the same input.
//
// The output depends on the reference's vertex renumbering
// (genReorderMap, tools/genDatabase.cpp:259-413): vertices are numbered so
// that each edge-label partition covers few contiguous id runs (the
// .mygraph interval index holds at most 256 runs, :454-460).  Its steps are
// restated here with sorted vectors in place of std::map/std::list where only
// the iteration order matters:
//   1. partitions (sets of source vertices per edge label) are ordered by
//      size, largest first, stable for equal sizes;
//   2. the largest partition B is split into sub-parts by every other
//      partition (vertices shared with it vs not), each sub-part keeping its
//      order, shared vertices leaving B;
//   3. sub-parts are numbered from the top of B's id range downwards, grouped
//      by the partitions they overlap (each group narrowed by the later
//      partitions until one sub-part remains), vertices left in B take the
//      lowest ids, ascending;
//   4. numbered vertices leave every other partition, B is dropped, repeat.
// Neighbour lists are then renumbered, sorted, and lists longer than 128 get
// the index-vertex prefix (:415-436); partitions are written as in
// writeHybridDataStructure (:451-580).  The adjacency is held as one flat
// array of (source, neighbour label, neighbour) per edge label, sorted on all
// host cores (repeated edges removed after sorting), in place of the
// reference's nested maps; the renumbering keeps ordered sets.
#include <algorithm>
#include <array>
#include <thread>
#include <unordered_map>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <list>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/geneva.h"
#include "gva_internal.h"

namespace gva {
namespace {

// first three unsigned integers of a line (tools/genDatabase.cpp:69-92)
int parse_uints(const char* line, size_t len, uint32_t* out, int want) {
    int n = 0;
    size_t i = 0;
    while (i < len && n < want) {
        if (line[i] >= '0' && line[i] <= '9') {
            uint64_t x = 0;
            while (i < len && line[i] >= '0' && line[i] <= '9') x = x * 10 + (uint64_t)(line[i++] - '0');
            out[n++] = (uint32_t)x;
        } else {
            ++i;
        }
    }
    return n;
}

// A partition's set of source vertices during the renumbering, over ranks
// of the source ids (rank order = id order): the ranks it ever held,
// ascending, and a bitset of those it still holds.  Iteration visits the
// held ranks in ascending order, as std::set would.
struct RankSet {
    std::vector<uint32_t> items;
    std::vector<uint64_t> bits;
    size_t count = 0;
    bool has(uint32_t r) const { return bits[r >> 6] >> (r & 63) & 1; }
    void erase(uint32_t r) {
        if (has(r)) bits[r >> 6] &= ~(1ull << (r & 63)), --count;
    }
};

// Step 2 of the renumbering for one other partition `cur`.
void split_by(RankSet& base, const RankSet& cur, std::vector<std::vector<uint32_t>>& subs) {
    std::vector<uint32_t> common;
    for (uint32_t v : base.items)
        if (base.has(v) && cur.has(v)) common.push_back(v);
    const size_t before = subs.size();
    for (size_t i = 0; i < before; ++i) {
        std::vector<uint32_t> in, out;
        for (uint32_t v : subs[i]) (cur.has(v) ? in : out).push_back(v);
        if (in.size() == subs[i].size() || out.size() == subs[i].size()) continue;
        subs[i] = out;
        subs.push_back(in);
    }
    if (!common.empty()) subs.push_back(common);
    for (uint32_t v : common) base.erase(v);
}

// The new id of every source vertex, as (old id, new id) by ascending old id.
std::vector<std::pair<uint32_t, uint32_t>> renumber(const std::vector<std::vector<uint32_t>>& sources) {
    // ranks: the sorted union of all partitions' (sorted) source ids
    std::vector<uint32_t> ids;
    for (const std::vector<uint32_t>& src : sources) ids.insert(ids.end(), src.begin(), src.end());
    std::sort(ids.begin(), ids.end());
    ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
    const size_t nr = ids.size(), words = (nr + 63) / 64;
    std::vector<RankSet> parts(sources.size());
    for (size_t p = 0; p < sources.size(); ++p) {
        RankSet& rs = parts[p];
        rs.bits.assign(words, 0);
        rs.items.reserve(sources[p].size());
        size_t k = 0;  // sources[p] is sorted: a merge walk gives the ranks
        for (uint32_t v : sources[p]) {
            while (ids[k] < v) ++k;
            if (rs.items.empty() || rs.items.back() != k) {
                rs.items.push_back((uint32_t)k);
                rs.bits[k >> 6] |= 1ull << (k & 63);
                ++rs.count;
            }
        }
    }
    auto by_size = [](const RankSet& a, const RankSet& b) { return a.count > b.count; };
    std::stable_sort(parts.begin(), parts.end(), by_size);
    std::vector<uint32_t> newid(nr, 0);  // by rank; 0: not numbered yet (ids start at 1)
    auto assign = [&](uint32_t r, uint32_t id) {
        if (!newid[r]) newid[r] = id;  // first one wins, as map::emplace
    };
    uint32_t numbered = 0;
    const size_t rounds = parts.size();
    for (size_t r = 0; r < rounds; ++r) {
        RankSet& base = parts[0];
        uint32_t top = numbered + (uint32_t)base.count;
        numbered += (uint32_t)base.count;
        std::vector<std::vector<uint32_t>> subs;
        for (size_t i = 1; i < parts.size(); ++i) split_by(base, parts[i], subs);
        std::map<size_t, std::set<size_t>> overlaps;  // other partition -> sub-parts it touches
        for (size_t i = 0; i < subs.size(); ++i) {
            const uint32_t probe = subs[i][0];
            for (size_t j = 1; j < parts.size(); ++j)
                if (parts[j].has(probe)) overlaps[j].insert(i);
            for (uint32_t v : subs[i])
                for (size_t k = 1; k < parts.size(); ++k) parts[k].erase(v);
        }
        std::vector<char> done(subs.size(), 0);
        for (auto it = overlaps.begin(); it != overlaps.end(); ++it) {
            std::vector<size_t> todo;
            for (size_t sid : it->second)
                if (!done[sid]) todo.push_back(sid), done[sid] = 1;
            std::vector<std::pair<std::vector<size_t>, uint32_t>> groups;  // (sub-parts, first id from the top)
            while (!todo.empty()) {
                std::vector<size_t> grp = todo;
                for (auto jt = std::next(it); jt != overlaps.end(); ++jt) {
                    std::vector<size_t> keep;
                    for (size_t sid : grp)
                        if (jt->second.count(sid)) keep.push_back(sid);
                    if (!keep.empty()) grp = keep;
                    if (grp.size() == 1) break;
                }
                groups.push_back({grp, top});
                uint32_t tot = 0;
                for (size_t sid : grp) tot += (uint32_t)subs[sid].size();
                top -= tot;
                std::vector<size_t> rest;
                for (size_t sid : todo)
                    if (std::find(grp.begin(), grp.end(), sid) == grp.end()) rest.push_back(sid);
                todo.swap(rest);
            }
            for (auto& gr : groups) {
                uint32_t id = gr.second;
                for (size_t sid : gr.first)
                    for (uint32_t v : subs[sid]) assign(v, id--);
            }
        }
        uint32_t id = top - (uint32_t)base.count + 1;
        for (uint32_t v : base.items)
            if (base.has(v)) assign(v, id++);
        parts.erase(parts.begin());
        std::stable_sort(parts.begin(), parts.end(), by_size);
    }
    std::vector<std::pair<uint32_t, uint32_t>> out;
    out.reserve(nr);
    for (size_t k = 0; k < nr; ++k)
        if (newid[k]) out.push_back({ids[k], newid[k]});
    return out;
}

// tools/genDatabase.cpp:415-436
void add_index_prefix(std::vector<uint32_t>& v) {
    std::vector<uint32_t> idx;
    if (v.size() <= 32 * 128) {
        const size_t blocks = v.size() / 128;
        for (size_t i = 1; i <= blocks; ++i) idx.push_back(v[i * 128 - 1]);
        if (v.size() % 128) idx.push_back(v.back());
    } else {
        const size_t blk = v.size() / 32;
        for (size_t i = 1; i <= 31; ++i) idx.push_back(v[i * blk - 1]);
        idx.push_back(v.back());
    }
    v.insert(v.begin(), idx.begin(), idx.end());
}


// One directed adjacency entry: source, label of the neighbour, neighbour.
struct Half {
    uint32_t a, lb, b;
    bool operator<(const Half& o) const { return a != o.a ? a < o.a : (lb != o.lb ? lb < o.lb : b < o.b); }
    bool operator==(const Half& o) const { return a == o.a && lb == o.lb && b == o.b; }
};

// Sorts on the host's cores: chunks sorted in parallel, then merged pairwise.
void parallel_sort(std::vector<Half>& v) {
    const size_t n = v.size();
    const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    if (n < (1u << 20) || hw == 1) {
        std::sort(v.begin(), v.end());
        return;
    }
    size_t chunks = 1;
    while (chunks * 2 <= hw) chunks *= 2;
    std::vector<size_t> cut(chunks + 1);
    for (size_t c = 0; c <= chunks; ++c) cut[c] = n * c / chunks;
    std::vector<std::thread> pool;
    for (size_t c = 0; c < chunks; ++c)
        pool.emplace_back([&, c]() { std::sort(v.begin() + cut[c], v.begin() + cut[c + 1]); });
    for (auto& t : pool) t.join();
    for (size_t width = 1; width < chunks; width *= 2) {
        pool.clear();
        for (size_t c = 0; c + width < chunks; c += 2 * width) {
            const size_t lo = cut[c], mid = cut[c + width], hi = cut[std::min(chunks, c + 2 * width)];
            pool.emplace_back([&v, lo, mid, hi]() { std::inplace_merge(v.begin() + lo, v.begin() + mid, v.begin() + hi); });
        }
        for (auto& t : pool) t.join();
    }
}

// Growing text output with a decimal formatter (the .reorder file is large).
struct Out {
    std::string s;
    void u(uint64_t x) {
        char b[24];
        int k = 0;
        do {
            b[k++] = (char)('0' + x % 10);
            x /= 10;
        } while (x);
        while (k) s.push_back(b[--k]);
    }
    void c(char ch) { s.push_back(ch); }
};

bool write_file(const std::string& path, const void* data, size_t n) {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = fwrite(data, 1, n, f) == n;
    return fclose(f) == 0 && ok;
}

}  // namespace

int convert_g(const std::string& g_path, const std::string& mygraph, const std::string& metadata,
              const std::string& reorder) {
    std::string text;
    {
        FILE* f = fopen(g_path.c_str(), "rb");
        if (!f) return fail(GVA_ERR_IO, "cannot open " + g_path);
        char buf[1 << 16];
        size_t k;
        while ((k = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, k);
        fclose(f);
    }
    std::unordered_map<uint32_t, uint32_t> vlabel;  // first definition wins; only looked up
    uint32_t x[3];
    size_t pos = 0;
    const char* line = nullptr;  // the current line, [line, line + len), in `text`
    size_t len = 0;
    auto next_line = [&]() {
        if (pos >= text.size()) return false;
        const char* b = text.data() + pos;
        const void* nl = std::memchr(b, '\n', text.size() - pos);
        const size_t e = nl ? (size_t)((const char*)nl - text.data()) : text.size();
        line = b;
        len = e - pos;
        pos = e + 1;
        return true;
    };
    // vertex section (tools/genDatabase.cpp:769-778): up to the first `e` line
    bool have_edge = false;
    vlabel.reserve(text.size() / 16);
    while (next_line()) {
        if (len == 0 || line[0] == 't') continue;
        if (line[0] == 'v') {
            if (parse_uints(line, len, x, 2) == 2) vlabel.emplace(x[0], x[1]);
        } else if (line[0] == 'e') {
            have_edge = true;
            break;
        }
    }
    std::vector<std::array<uint32_t, 3>> edges;  // (label, src, dst)
    size_t P = 0;
    uint32_t max_id = 0;
    while (have_edge) {
        if (len != 0 && line[0] == 'e') {
            if (parse_uints(line, len, x, 3) < 3)
                return fail(GVA_ERR_FORMAT, "malformed edge line: " + std::string(line, len));
            P = std::max<size_t>(P, (size_t)x[2] + 1);
            max_id = std::max(max_id, std::max(x[0], x[1]));
            edges.push_back({x[2], x[0], x[1]});
        }
        if (!next_line()) break;
    }
    text.clear();
    text.shrink_to_fit();
    if (edges.empty()) return fail(GVA_ERR_FORMAT, "no edges in " + g_path);
    // neighbour labels: a vertex without a `v` line has label 0
    const bool dense = max_id < (1u << 28);
    std::vector<uint32_t> lab_of;
    if (dense) {
        lab_of.assign((size_t)max_id + 1, 0);
        for (auto& kv : vlabel)
            if (kv.first <= max_id) lab_of[kv.first] = kv.second;
    }
    auto label = [&](uint32_t v) -> uint32_t {
        if (dense) return lab_of[v];
        auto it = vlabel.find(v);
        return it == vlabel.end() ? 0u : it->second;
    };
    // per edge label both directions, sorted by (source, neighbour label,
    // neighbour) with repeats removed
    std::vector<std::vector<Half>> part(P);
    {
        std::vector<size_t> cnt(P, 0);
        for (auto& e : edges) cnt[e[0]] += 2;
        for (size_t p = 0; p < P; ++p) part[p].reserve(cnt[p]);
        for (auto& e : edges) {
            part[e[0]].push_back({e[1], label(e[2]), e[2]});
            part[e[0]].push_back({e[2], label(e[1]), e[1]});
        }
        edges.clear();
        edges.shrink_to_fit();
    }
    std::vector<std::vector<uint32_t>> sources(P);
    for (size_t p = 0; p < P; ++p) {
        parallel_sort(part[p]);
        part[p].erase(std::unique(part[p].begin(), part[p].end()), part[p].end());
        for (const Half& h : part[p])
            if (sources[p].empty() || sources[p].back() != h.a) sources[p].push_back(h.a);
    }
    const std::vector<std::pair<uint32_t, uint32_t>> newid = renumber(sources);  // by old id
    std::vector<uint32_t> nid_dense;
    std::unordered_map<uint32_t, uint32_t> nid_hash;
    if (dense) {
        nid_dense.assign((size_t)max_id + 1, 0);
        for (auto& kv : newid) nid_dense[kv.first] = kv.second;
    } else {
        nid_hash.reserve(newid.size() * 2);
        for (auto& kv : newid) nid_hash.emplace(kv.first, kv.second);
    }
    auto nid = [&](uint32_t v) { return dense ? nid_dense[v] : nid_hash.at(v); };
    // renumbered partitions, sorted by (new source, label, new neighbour)
    for (size_t p = 0; p < P; ++p) {
        for (Half& h : part[p]) {
            h.a = nid(h.a);
            h.b = nid(h.b);
        }
        parallel_sort(part[p]);
    }
    // One pass per partition over its (source, label) groups: the written
    // neighbour list of a group is its sorted ids, with the index-vertex
    // prefix when longer than 128 (tools/genDatabase.cpp:415-436).
    Out ro;
    ro.u(P);
    ro.c('\n');
    std::vector<uint32_t> words;
    words.push_back((uint32_t)(P - 1));  // .mygraph header counts label 0 out (:856-869)
    std::vector<uint32_t> nv;
    for (size_t p = 0; p < P; ++p) {
        const std::vector<Half>& H = part[p];
        // group boundaries: sources, then (source, label) runs
        std::vector<size_t> src_at, grp_at;
        for (size_t i = 0; i < H.size(); ++i) {
            if (i == 0 || H[i].a != H[i - 1].a) src_at.push_back(i);
            if (i == 0 || H[i].a != H[i - 1].a || H[i].lb != H[i - 1].lb) grp_at.push_back(i);
        }
        src_at.push_back(H.size());
        grp_at.push_back(H.size());
        // lists with prefixes, and each source's total written length
        std::vector<std::vector<uint32_t>> lists(grp_at.size() - 1);
        for (size_t g = 0; g + 1 < grp_at.size(); ++g) {
            nv.clear();
            for (size_t i = grp_at[g]; i < grp_at[g + 1]; ++i) nv.push_back(H[i].b);
            if (nv.size() > 128) add_index_prefix(nv);
            lists[g] = nv;
        }
        // .reorder (tools/genDatabase.cpp:826-846)
        ro.u(src_at.size() - 1);
        ro.c('\n');
        size_t g = 0;
        std::vector<uint64_t> src_len(src_at.size() - 1, 0);
        for (size_t si = 0; si + 1 < src_at.size(); ++si) {
            size_t ng = 0;
            for (size_t k = g; k + 1 < grp_at.size() && grp_at[k] < src_at[si + 1]; ++k) ++ng;
            ro.u(H[src_at[si]].a);
            ro.c(' ');
            ro.u(ng);
            ro.c('\n');
            for (size_t k = 0; k < ng; ++k, ++g) {
                ro.u(H[grp_at[g]].lb);
                ro.c(' ');
                ro.u(lists[g].size());
                ro.c('\n');
                for (uint32_t u : lists[g]) {
                    ro.u(u);
                    ro.c(' ');
                }
                ro.c('\n');
                src_len[si] += lists[g].size();
            }
        }
        if (H.empty()) continue;
        // .mygraph partition (tools/genDatabase.cpp:451-580; the hash section is always empty)
        struct Run { uint32_t s, e; };
        std::vector<Run> runs;
        uint64_t nbrs = 0;
        for (size_t si = 0; si + 1 < src_at.size(); ++si) {
            const uint32_t v = H[src_at[si]].a;
            nbrs += src_len[si];
            if (!runs.empty() && v == runs.back().e + 1)
                runs.back().e = v;
            else
                runs.push_back({v, v});
        }
        const size_t nint = std::min<size_t>(runs.size(), 256);
        uint64_t slots = 0;
        for (size_t i = 0; i < nint; ++i) slots += runs[i].e - runs[i].s + 1;
        const uint64_t tot = 5 + nint * 2 + 2 + slots + 1 + nbrs;
        std::vector<uint32_t> w(tot, 0);
        w[0] = (uint32_t)tot;
        w[1] = (uint32_t)slots;
        w[2] = (uint32_t)nint;
        w[3] = (uint32_t)(nint * 2 + 2 + slots + 1);
        w[4] = w[3];
        const uint64_t slot_at = 5 + nint * 2 + 2, nbr_at = slot_at + slots + 1;
        uint64_t si_w = slot_at, nb = nbr_at, cum = 0;
        size_t si = 0, gi = 0;
        for (size_t i = 0; i < nint; ++i) {
            w[5 + i] = runs[i].s;
            cum += runs[i].e - runs[i].s + 1;
            w[5 + i + nint + 1] = (uint32_t)cum;
            for (uint32_t v = runs[i].s; v <= runs[i].e; ++v, ++si) {
                w[si_w++] = (uint32_t)(nb - nbr_at);
                while (gi + 1 < grp_at.size() && grp_at[gi] < src_at[si + 1]) {
                    for (uint32_t u : lists[gi]) w[nb++] = u;
                    ++gi;
                }
            }
        }
        w[si_w] = (uint32_t)(nb - nbr_at);
        words.insert(words.end(), w.begin(), w.end());
    }
    if (!write_file(reorder, ro.s.data(), ro.s.size())) return fail(GVA_ERR_IO, "cannot write " + reorder);
    if (!write_file(mygraph, words.data(), words.size() * 4)) return fail(GVA_ERR_IO, "cannot write " + mygraph);
    // .metadata (tools/genDatabase.cpp:873-879): "new label old", by old id
    Out md;
    for (auto& kv : newid) {
        auto it = vlabel.find(kv.first);
        md.u(kv.second);
        md.c(' ');
        md.u(it == vlabel.end() ? 0u : it->second);
        md.c(' ');
        md.u(kv.first);
        md.c('\n');
    }
    if (!write_file(metadata, md.s.data(), md.s.size())) return fail(GVA_ERR_IO, "cannot write " + metadata);
    return GVA_OK;
}

}  // namespace gva
