// Test infrastructure only (the checker, never shipped): a main() of our own
// around the reference planner, compiled from the reference's unmodified
// source src/genMatchOrderCPU.cpp by oracle/Makefile into oracle/_ref/plandump.
//
//   plandump <query file> <out file>
//
// Runs genMatchOrder (src/genMatchOrderCPU.cpp:670-983) on one query and writes
// the plan in the canonical text form that the product planner
// (gva_plan_describe) and the oracle's own restatement both print:
//
//   vnum <n>
//   phase <i> <E|R> <edge label> <npairs> <s0> <e0> [<s1> <e1> ...]
//   restrict <query vertex> <bound vertex | 4294967295>
//   repeat <edge label> <vertex label> <hex value>
//   stat <edge label> <vertex label>
//
// The reference planner keeps its state in globals, so one process plans one
// query (the reference drivers do the same).
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "genMatchOrderCPU.h"

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: plandump <query> <out>\n");
        return 2;
    }
    std::vector<Phase> order;
    std::map<uint64_t, uint> repeatFlag;
    std::map<uint, uint> restricts;
    std::map<uint, std::map<uint, bool>> stat;
    std::map<uint, uint> qlabel;
    // The reference planner prints progress to std::cout; silence it.
    std::ostringstream sink;
    std::streambuf* saved = std::cout.rdbuf(sink.rdbuf());
    genMatchOrder(argv[1], order, repeatFlag, restricts, stat, qlabel);
    std::cout.rdbuf(saved);

    FILE* f = std::fopen(argv[2], "w");
    if (!f) return 3;
    std::fprintf(f, "vnum %zu\n", qlabel.size());
    for (size_t i = 0; i < order.size(); ++i) {
        const Phase& p = order[i];
        std::fprintf(f, "phase %zu %c %u %zu", i, p.phaseType, p.edgeLabel, p.pairs.size() / 2);
        for (uint v : p.pairs) std::fprintf(f, " %u", v);
        std::fprintf(f, "\n");
    }
    for (auto& kv : restricts) std::fprintf(f, "restrict %u %u\n", kv.first, kv.second);
    for (auto& kv : repeatFlag)
        std::fprintf(f, "repeat %u %u %x\n", (uint)(kv.first >> 32), (uint)(kv.first & 0xffffffffu), kv.second);
    for (auto& kv : stat)
        for (auto& kv2 : kv.second) std::fprintf(f, "stat %u %u\n", kv.first, kv2.first);
    std::fclose(f);
    return 0;
}
