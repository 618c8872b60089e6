// Test driver (CPU only): the heap-free planner (dplan, gva_dplan.h, written
// to run on the device as well) against the host planner (plan_from_query,
// pinned to the reference's plans) on seeded random connected queries: every
// query dplan accepts must get the host planner's plan (phases, pair
// orientation, restrictions, repeat flags, record stats, columns); the others
// must be ones it may leave to the host (a list longer than 16 entries, a
// capacity, or a query the host planner rejects).  Its plans lowered
// directly (lower_dplan) must give the host plan's steps.
//
// usage: dplan_check queries seed max_vertices
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../geneva_b200/csrc/gva_dplan.h"
#include "../geneva_b200/csrc/gva_internal.h"
#include "../include/geneva.h"

using namespace gva;

int main(int argc, char** argv) {
    if (argc < 4) return 2;
    const int nq = atoi(argv[1]);
    const uint32_t maxv = (uint32_t)atoi(argv[3]);
    uint64_t x = 0x9e3779b97f4a7c15ull * (uint64_t)(atoi(argv[2]) + 7);
    auto rnd = [&]() {
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        return x;
    };
    static DPlanQuery dq;
    static DPlan dp;
    // a database with labels 1..4 and partitions 1..3, for lowering
    HostGraph g;
    {
        std::vector<uint32_t> vl(13), sv, dv, el;
        for (uint32_t v = 1; v <= 12; ++v) vl[v] = 1 + (v - 1) % 4;
        for (uint32_t v = 1; v <= 12; ++v)
            for (uint32_t u = v + 1; u <= 12; ++u) sv.push_back(v), dv.push_back(u), el.push_back(1 + (u + v) % 3);
        if (graph_from_edges(vl.data(), 12, sv.data(), dv.data(), el.data(), sv.size(), g)) return 2;
    }
    int accepted = 0, host_only = 0;
    for (int qi = 0; qi < nq; ++qi) {
        const uint32_t n = 2 + rnd() % (maxv - 1), nl = 1 + rnd() % 4, nel = 1 + rnd() % 3;
        dq.n = n;
        for (uint32_t v = 0; v < n; ++v) dq.label[v] = 1 + rnd() % nl;
        std::vector<std::pair<uint32_t, uint32_t>> es;
        for (uint32_t v = 1; v < n; ++v) es.push_back({(uint32_t)(rnd() % v), v});
        const uint32_t extra = rnd() % (n + 2);
        for (uint32_t k = 0; k < extra; ++k) {
            uint32_t a = rnd() % n, b = rnd() % n;
            if (a != b) es.push_back({a, b});
        }
        if (rnd() % 2) std::swap(es.front(), es.back());
        if (es.size() > (size_t)kDpLines) es.resize(kDpLines);
        std::vector<uint32_t> sdl;
        dq.lines = (uint32_t)es.size();
        for (size_t i = 0; i < es.size(); ++i) {
            const uint32_t l = 1 + rnd() % nel;
            dq.s[i] = es[i].first, dq.d[i] = es[i].second, dq.l[i] = l;
            sdl.push_back(es[i].first);
            sdl.push_back(es[i].second);
            sdl.push_back(l);
        }
        dplan(dq, dp);
        Plan want;
        const int rc = plan_from_query(n, dq.label, sdl.data(), es.size(), GVA_MODE_DV, want);
        if (dp.status != DPLAN_OK) {
            ++host_only;
            continue;
        }
        if (rc) {
            printf("query %d: accepted by dplan, rejected by the host planner (%s)\n", qi, last_error_cstr());
            return 1;
        }
        Plan got;
        if (plan_from_dplan(dp, dq.label, got)) {
            printf("query %d: conversion failed\n", qi);
            return 1;
        }
        if (got.describe() != want.describe() || got.columns != want.columns || got.qlabel != want.qlabel ||
            got.vnum != want.vnum) {
            std::string t;
            for (uint32_t v = 0; v < n; ++v) t += "v " + std::to_string(v) + " " + std::to_string(dq.label[v]) + "\n";
            for (size_t i = 0; i < es.size(); ++i)
                t += "e " + std::to_string(dq.s[i]) + " " + std::to_string(dq.d[i]) + " " + std::to_string(dq.l[i]) + "\n";
            printf("query %d: plans differ\n%s--- host\n%s--- dplan\n%s", qi, t.c_str(), want.describe().c_str(),
                   got.describe().c_str());
            return 1;
        }
        std::vector<Step> sa, sb;
        if (lower_plan(want, g, sa, true) || lower_dplan(dp, dq.label, g, sb, true) || sa.size() != sb.size() ||
            (!sa.empty() && std::memcmp(sa.data(), sb.data(), sa.size() * sizeof(Step)) != 0)) {
            printf("query %d: lowered steps differ\n", qi);
            return 1;
        }
        ++accepted;
    }
    printf("ok %d accepted, %d left to the host\n", accepted, host_only);
    return 0;
}
