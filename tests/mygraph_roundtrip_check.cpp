// Test driver (CPU only): .g -> converter (convert_g, byte-identical to the
// reference genDatabase) -> .mygraph / .metadata -> loader (load_mygraph)
// must give the same database as building it from the edge list directly
// (graph_from_edges) after the converter's renumbering, read back from the
// .metadata lines "new id, label, old id".  Random graphs with repeated
// edges and hub vertices whose lists pass 128 entries (the converter then
// writes index vertices, which the loader drops).
//
// usage: mygraph_roundtrip_check graphs seed workdir
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "../geneva_b200/csrc/gva_internal.h"

using namespace gva;

int main(int argc, char** argv) {
    if (argc < 4) return 2;
    const int graphs = atoi(argv[1]);
    std::mt19937 rng(atoi(argv[2]));
    const std::string dir = argv[3];
    for (int t = 0; t < graphs; ++t) {
        const uint32_t n = 2 + rng() % 3000, L = 1 + rng() % 6, P = 1 + rng() % 3;
        std::vector<uint32_t> vl(n);
        for (uint32_t v = 0; v < n; ++v) vl[v] = 1 + rng() % L;
        std::vector<uint32_t> s, d, e;
        const uint32_t hub = rng() % n;
        const uint64_t m = n + rng() % (3ull * n);
        for (uint64_t i = 0; i < m; ++i) {
            const uint32_t a = rng() % 4 == 0 ? hub : rng() % n, b = rng() % n;
            if (a == b) continue;
            s.push_back(a), d.push_back(b), e.push_back(1 + rng() % P);
            if (rng() % 8 == 0) s.push_back(b), d.push_back(a), e.push_back(e.back());  // repeated
        }
        for (uint32_t l = 1; l <= P; ++l) {  // every edge label 1..P occurs
            s.push_back(0), d.push_back(1), e.push_back(l);
        }
        const std::string g = dir + "/t.g";
        {
            std::ofstream out(g);
            for (uint32_t v = 0; v < n; ++v) out << "v " << v << " " << vl[v] << "\n";
            for (size_t i = 0; i < s.size(); ++i) out << "e " << s[i] << " " << d[i] << " " << e[i] << "\n";
        }
        if (convert_g(g, dir + "/t.mygraph", dir + "/t.metadata", dir + "/t.reorder")) {
            printf("graph %d: conversion failed: %s\n", t, last_error_cstr());
            return 1;
        }
        HostGraph got;
        std::string warn;
        if (load_mygraph(dir + "/t.mygraph", dir + "/t.metadata", got, &warn) || !warn.empty()) {
            printf("graph %d: load failed: %s %s\n", t, last_error_cstr(), warn.c_str());
            return 1;
        }
        // the renumbering, from the metadata
        std::vector<uint32_t> new_of(n, 0);
        uint32_t max_new = 0;
        {
            std::ifstream mf(dir + "/t.metadata");
            uint32_t nid, lab, oid;
            while (mf >> nid >> lab >> oid) {
                if (oid >= n || lab != vl[oid]) {
                    printf("graph %d: metadata line %u %u %u does not match the .g\n", t, nid, lab, oid);
                    return 1;
                }
                new_of[oid] = nid;
                max_new = std::max(max_new, nid);
            }
        }
        std::vector<uint32_t> vlab(max_new + 1, 0), ns, nd;
        for (uint32_t v = 0; v < n; ++v)
            if (new_of[v]) vlab[new_of[v]] = vl[v];
        for (size_t i = 0; i < s.size(); ++i) {
            if (!new_of[s[i]] || !new_of[d[i]]) {
                printf("graph %d: an edge endpoint has no new id\n", t);
                return 1;
            }
            ns.push_back(new_of[s[i]]), nd.push_back(new_of[d[i]]);
        }
        HostGraph want;
        if (graph_from_edges(vlab.data(), max_new, ns.data(), nd.data(), e.data(), ns.size(), want)) {
            printf("graph %d: build failed: %s\n", t, last_error_cstr());
            return 1;
        }
        bool same = got.max_id == want.max_id && got.labels == want.labels && got.dlabel == want.dlabel &&
                    got.parts.size() == want.parts.size();
        for (size_t p = 0; same && p < got.parts.size(); ++p)
            same = got.parts[p].off == want.parts[p].off && got.parts[p].adj == want.parts[p].adj;
        if (!same) {
            printf("graph %d (%u vertices, %zu edges): loaded database differs from the edge-list build\n", t, n, s.size());
            return 1;
        }
    }
    printf("ok %d graphs\n", graphs);
    return 0;
}
