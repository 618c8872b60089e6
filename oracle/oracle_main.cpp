// Test infrastructure only: command-line front end of the CPU oracle.
//
//   oracle_cpumine <db>.mygraph <db>.metadata <q>.query [out.txt]
//
// Prints "rows <n>" and "phase <i> <rows>" lines; with out.txt also writes
// the rows one per line like partialResultsCPU.txt (src/cpumine.cpp:587-601).
#include <chrono>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>

#include "geneva_oracle.h"

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s <mygraph> <metadata> <query> [out]\n", argv[0]);
        return 2;
    }
    oracle_graph* g = nullptr;
    if (oracle_graph_load(argv[1], argv[2], &g)) {
        std::fprintf(stderr, "load failed: %s\n", oracle_last_error());
        return 1;
    }
    std::ifstream qf(argv[3]);
    std::stringstream ss;
    ss << qf.rdbuf();
    uint32_t* rows = nullptr;
    uint64_t n = 0, ph[64];
    int w = 0, np = 0;
    auto t0 = std::chrono::steady_clock::now();
    if (oracle_match(g, ss.str().c_str(), &rows, &n, &w, ph, 64, &np)) {
        std::fprintf(stderr, "match failed: %s\n", oracle_last_error());
        return 1;
    }
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::printf("rows %llu\nwidth %d\nms %.3f\n", (unsigned long long)n, w, ms);
    for (int i = 0; i < np && i < 64; ++i) std::printf("phase %d %llu\n", i, (unsigned long long)ph[i]);
    if (argc > 4) {
        FILE* f = std::fopen(argv[4], "w");
        for (uint64_t r = 0; r < n; ++r) {
            for (int c = 0; c < w; ++c) std::fprintf(f, c ? " %u" : "%u", rows[r * w + c]);
            std::fprintf(f, "\n");
        }
        std::fclose(f);
    }
    oracle_free(rows);
    oracle_graph_free(g);
    return 0;
}
