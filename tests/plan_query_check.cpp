// Test driver (CPU only): the planner's entry from a pattern's arrays
// (plan_from_query, used by the miner) against its entry from query text
// (plan_from_text, the reference's input) on seeded random connected queries
// with cycles, repeated labels and repeated edge lines: plans, output
// columns and lowered steps must be identical.  The query reader of the
// texts path (read_query_text) must give back the arrays each text was made
// from, and its rules (first definition of a vertex wins, ids 0..n-1, at
// most 32 vertices, comments skipped) hold on hand-made texts.
//
// usage: plan_query_check queries seed
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../geneva_b200/csrc/gva_internal.h"
#include "../include/geneva.h"

using namespace gva;

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    const int nq = atoi(argv[1]);
    uint64_t x = 0x9e3779b97f4a7c15ull * (uint64_t)(atoi(argv[2]) + 1);
    auto rnd = [&]() {
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        return x;
    };
    // a database with labels 1..4 and partitions 1..3 for lowering
    HostGraph g;
    {
        std::vector<uint32_t> vl(13), sv, dv, el;
        for (uint32_t v = 1; v <= 12; ++v) vl[v] = 1 + (v - 1) % 4;
        for (uint32_t v = 1; v <= 12; ++v)
            for (uint32_t u = v + 1; u <= 12; ++u) sv.push_back(v), dv.push_back(u), el.push_back(1 + (u + v) % 3);
        if (graph_from_edges(vl.data(), 12, sv.data(), dv.data(), el.data(), sv.size(), g)) return 2;
    }
    int planned = 0;
    for (int q = 0; q < nq; ++q) {
        const uint32_t n = 2 + rnd() % 11, nl = 1 + rnd() % 4, nel = 1 + rnd() % 3;
        std::vector<uint32_t> labels(n), sdl;
        std::string text;
        for (uint32_t v = 0; v < n; ++v) {
            labels[v] = 1 + rnd() % nl;
            text += "v " + std::to_string(v) + " " + std::to_string(labels[v]) + "\n";
        }
        std::vector<std::pair<uint32_t, uint32_t>> es;
        for (uint32_t v = 1; v < n; ++v) es.push_back({(uint32_t)(rnd() % v), v});
        const uint32_t extra = rnd() % (n + 2);
        for (uint32_t k = 0; k < extra; ++k) {
            uint32_t a = rnd() % n, b = rnd() % n;
            if (a != b) es.push_back({a, b});
        }
        if (rnd() % 2) std::swap(es.front(), es.back());
        for (auto& e : es) {
            const uint32_t l = 1 + rnd() % nel;
            sdl.push_back(e.first);
            sdl.push_back(e.second);
            sdl.push_back(l);
            text += "e " + std::to_string(e.first) + " " + std::to_string(e.second) + " " + std::to_string(l) + "\n";
        }
        {
            std::vector<uint32_t> rl, rs;
            if (read_query_text(text, rl, rs) || rl != labels || rs != sdl) {
                printf("query %d: the query reader gives other arrays\n%s", q, text.c_str());
                return 1;
            }
        }
        for (int mode : {GVA_MODE_DV, GVA_MODE_SV}) {
            Plan a, b;
            const int ra = plan_from_text(text, mode, a);
            const int rb = plan_from_query(n, labels.data(), sdl.data(), sdl.size() / 3, mode, b);
            if (ra != rb) {
                printf("query %d: status %d from text, %d from arrays\n%s", q, ra, rb, text.c_str());
                return 1;
            }
            if (ra) continue;
            if (a.describe() != b.describe() || a.columns != b.columns || a.qlabel != b.qlabel || a.vnum != b.vnum) {
                printf("query %d mode %d: plans differ\n%s", q, mode, text.c_str());
                return 1;
            }
            std::vector<Step> sa, sb;
            if (lower_plan(a, g, sa, true) || lower_plan(b, g, sb, true) || sa.size() != sb.size() ||
                (sa.size() && std::memcmp(sa.data(), sb.data(), sa.size() * sizeof(Step)) != 0)) {
                printf("query %d mode %d: lowered steps differ\n%s", q, mode, text.c_str());
                return 1;
            }
            ++planned;
        }
    }
    // the reader's rules on hand-made texts
    struct Case {
        std::string text;
        int status;
        std::vector<uint32_t> labels;
    };
    std::string big;
    for (int v = 0; v < 33; ++v) big += "v " + std::to_string(v) + " 1\n";
    big += "e 0 1 1\n";
    const Case cases[] = {
        {"v 0 1\nv 0 2\nv 1 3\ne 0 1 1\n", GVA_OK, {1, 3}},        // first definition wins
        {"v 1 3\nv 0 1\ne 0 1 1\n", GVA_OK, {1, 3}},                // ids in any order
        {"# a comment\nv 0 1\n# another\nv 1 2\ne 0 1 1\n", GVA_OK, {1, 2}},
        {"v 1 1\nv 2 1\ne 1 2 1\n", GVA_ERR_FORMAT, {}},            // ids not 0..n-1
        {"v 0 1\nv 1 1\n", GVA_ERR_FORMAT, {}},                     // no edges
        {"e 0 1 1\n", GVA_ERR_FORMAT, {}},                           // no vertices
        {big, GVA_ERR_UNSUPPORTED, {}},                               // 33 vertices
    };
    for (const Case& c : cases) {
        std::vector<uint32_t> rl, rs;
        const int r = read_query_text(c.text, rl, rs);
        if (r != c.status || (r == GVA_OK && rl != c.labels)) {
            printf("query reader: status %d on\n%s", r, c.text.c_str());
            return 1;
        }
    }
    printf("ok %d plans\n", planned);
    return 0;
}
