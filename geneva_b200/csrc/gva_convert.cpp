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
// writeHybridDataStructure (:451-580).
#include <algorithm>
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

using Adj = std::map<uint32_t, std::map<uint32_t, std::vector<uint32_t>>>;  // svid -> vlabel -> nbrs

// first three unsigned integers of a line (tools/genDatabase.cpp:69-92)
int parse_uints(const std::string& line, uint32_t* out, int want) {
    int n = 0;
    size_t i = 0;
    while (i < line.size() && n < want) {
        if (line[i] >= '0' && line[i] <= '9') {
            uint64_t x = 0;
            while (i < line.size() && line[i] >= '0' && line[i] <= '9') x = x * 10 + (uint64_t)(line[i++] - '0');
            out[n++] = (uint32_t)x;
        } else {
            ++i;
        }
    }
    return n;
}

// Appends both directions; repeated edges are removed when the lists are
// sorted after renumbering (the reference skips them on insertion, which
// gives the same sets: the written lists are sorted either way, and a linear
// duplicate check per insertion is quadratic in a hub's degree).
void add_edge(std::vector<Adj>& g, std::map<uint32_t, uint32_t>& vlabel, uint32_t s, uint32_t d, uint32_t el) {
    Adj& part = g[el];
    for (int dir = 0; dir < 2; ++dir) {
        const uint32_t a = dir ? d : s, b = dir ? s : d;
        const uint32_t lb = vlabel[b];  // a vertex without a `v` line has label 0
        part[a][lb].push_back(b);
    }
}

// Step 2 of the renumbering for one other partition `cur`.
void split_by(std::set<uint32_t>& base, const std::set<uint32_t>& cur, std::vector<std::vector<uint32_t>>& subs) {
    std::vector<uint32_t> common;
    for (uint32_t v : base)
        if (cur.count(v)) common.push_back(v);
    const size_t before = subs.size();
    for (size_t i = 0; i < before; ++i) {
        std::vector<uint32_t> in, out;
        for (uint32_t v : subs[i]) (cur.count(v) ? in : out).push_back(v);
        if (in.size() == subs[i].size() || out.size() == subs[i].size()) continue;
        subs[i] = out;
        subs.push_back(in);
    }
    if (!common.empty()) subs.push_back(common);
    for (uint32_t v : common) base.erase(v);
}

std::map<uint32_t, uint32_t> renumber(const std::vector<Adj>& g) {
    std::vector<std::set<uint32_t>> parts;
    for (const Adj& p : g) {
        std::set<uint32_t> s;
        for (auto& kv : p) s.insert(kv.first);
        parts.push_back(std::move(s));
    }
    auto by_size = [](const std::set<uint32_t>& a, const std::set<uint32_t>& b) { return a.size() > b.size(); };
    std::stable_sort(parts.begin(), parts.end(), by_size);
    std::map<uint32_t, uint32_t> newid;  // old -> new
    uint32_t numbered = 0;
    const size_t rounds = parts.size();
    for (size_t r = 0; r < rounds; ++r) {
        std::set<uint32_t>& base = parts[0];
        uint32_t top = numbered + (uint32_t)base.size();
        numbered += (uint32_t)base.size();
        std::vector<std::vector<uint32_t>> subs;
        for (size_t i = 1; i < parts.size(); ++i) split_by(base, parts[i], subs);
        std::map<size_t, std::set<size_t>> overlaps;  // other partition -> sub-parts it touches
        for (size_t i = 0; i < subs.size(); ++i) {
            const uint32_t probe = subs[i][0];
            for (size_t j = 1; j < parts.size(); ++j)
                if (parts[j].count(probe)) overlaps[j].insert(i);
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
                    for (uint32_t v : subs[sid]) newid.emplace(v, id--);
            }
        }
        uint32_t id = top - (uint32_t)base.size() + 1;
        for (uint32_t v : base) newid.emplace(v, id++);
        parts.erase(parts.begin());
        std::stable_sort(parts.begin(), parts.end(), by_size);
    }
    return newid;
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

// tools/genDatabase.cpp:451-580 (the hash section is always empty)
void write_partition(const Adj& part, std::vector<uint32_t>& out) {
    struct Run { uint32_t s, e; };
    std::vector<Run> runs;
    uint64_t nbrs = 0;
    for (auto it = part.begin(); it != part.end(); ++it) {
        for (auto& kv : it->second) nbrs += kv.second.size();
        if (!runs.empty() && it->first == runs.back().e + 1)
            runs.back().e = it->first;
        else
            runs.push_back({it->first, it->first});
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
    uint64_t si = slot_at, nb = nbr_at, cum = 0;
    for (size_t i = 0; i < nint; ++i) {
        w[5 + i] = runs[i].s;
        cum += runs[i].e - runs[i].s + 1;
        w[5 + i + nint + 1] = (uint32_t)cum;
        for (uint32_t v = runs[i].s; v <= runs[i].e; ++v) {
            w[si++] = (uint32_t)(nb - nbr_at);
            for (auto& kv : part.at(v))
                for (uint32_t u : kv.second) w[nb++] = u;
        }
    }
    w[si] = (uint32_t)(nb - nbr_at);
    out.insert(out.end(), w.begin(), w.end());
}

}  // namespace

int convert_g(const std::string& g_path, const std::string& mygraph, const std::string& metadata,
              const std::string& reorder) {
    std::ifstream in(g_path);
    if (!in.is_open()) return fail(GVA_ERR_IO, "cannot open " + g_path);
    std::map<uint32_t, uint32_t> vlabel;
    std::string line;
    uint32_t x[3];
    // vertex section (tools/genDatabase.cpp:769-778): up to the first `e` line
    bool have_edge = false;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == 't') continue;
        if (line[0] == 'v') {
            if (parse_uints(line, x, 2) == 2) vlabel.emplace(x[0], x[1]);
        } else if (line[0] == 'e') {
            have_edge = true;
            break;
        }
    }
    std::vector<Adj> g;
    while (have_edge) {
        if (!line.empty() && line[0] == 'e') {
            if (parse_uints(line, x, 3) < 3) return fail(GVA_ERR_FORMAT, "malformed edge line: " + line);
            if (x[2] + 1 > g.size()) g.resize(x[2] + 1);
            add_edge(g, vlabel, x[0], x[1], x[2]);
        }
        if (!std::getline(in, line)) break;
    }
    if (g.empty()) return fail(GVA_ERR_FORMAT, "no edges in " + g_path);
    const std::map<uint32_t, uint32_t> newid = renumber(g);
    // renumbered partitions: new svid -> label -> sorted new neighbour ids
    std::vector<Adj> rg(g.size());
    for (size_t p = 0; p < g.size(); ++p) {
        for (auto& sv : g[p]) {
            auto& dst = rg[p][newid.at(sv.first)];
            for (auto& lv : sv.second) {
                std::vector<uint32_t> nv;
                for (uint32_t u : lv.second) nv.push_back(newid.at(u));
                std::sort(nv.begin(), nv.end());
                nv.erase(std::unique(nv.begin(), nv.end()), nv.end());
                if (nv.size() > 128) add_index_prefix(nv);
                dst[lv.first] = std::move(nv);
            }
        }
    }
    // .reorder (tools/genDatabase.cpp:826-846)
    {
        std::ofstream f(reorder);
        if (!f.is_open()) return fail(GVA_ERR_IO, "cannot write " + reorder);
        f << rg.size() << "\n";
        for (const Adj& part : rg) {
            f << part.size() << "\n";
            for (auto& sv : part) {
                f << sv.first << " " << sv.second.size() << "\n";
                for (auto& lv : sv.second) {
                    f << lv.first << " " << lv.second.size() << "\n";
                    for (uint32_t u : lv.second) f << u << " ";
                    f << "\n";
                }
            }
        }
    }
    // .mygraph (tools/genDatabase.cpp:856-869): header counts label 0 out
    {
        std::vector<uint32_t> words;
        words.push_back((uint32_t)(rg.size() - 1));
        for (const Adj& part : rg)
            if (!part.empty()) write_partition(part, words);
        std::ofstream f(mygraph, std::ios::binary);
        if (!f.is_open()) return fail(GVA_ERR_IO, "cannot write " + mygraph);
        f.write((const char*)words.data(), (std::streamsize)words.size() * 4);
    }
    // .metadata (tools/genDatabase.cpp:873-879): "new label old", by old id
    {
        std::ofstream f(metadata);
        if (!f.is_open()) return fail(GVA_ERR_IO, "cannot write " + metadata);
        for (auto& kv : newid) {
            auto it = vlabel.find(kv.first);
            f << kv.second << " " << (it == vlabel.end() ? 0u : it->second) << " " << kv.first << "\n";
        }
    }
    return GVA_OK;
}

}  // namespace gva
