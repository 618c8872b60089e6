// gpumine / gpumineSV command line (built twice, GVA_CLI_MODE = 0 / 1).
//
//   gpumine   <db>.mygraph <db>.metadata <q>.query
//   gpumineSV <db>.mygraph <db>.metadata <q>.query
//
// Same arguments, stdout lines and output file as the reference drivers
// (src/gpumine.cpp:866-1072, src/gpumine_singleV.cpp:722-928): the phase list,
// "time: <ms>", "Result: <rows> extra size0", "PartialRowNum: <rows> embLen:  <k>"
// and ./partialResultsGPU.txt with one match-ordered row per line.
// Differences: "time" is wall-clock milliseconds of planning + matching (the
// reference prints process CPU time), and a failure exits with status 1 and
// an "error:" line instead of printing and exiting 0.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/geneva.h"

#ifndef GVA_CLI_MODE
#define GVA_CLI_MODE GVA_MODE_DV
#endif

static int die(int st) {
    std::printf("error: %s (%s)\n", gva_last_error(), gva_status_string(st));
    return 1;
}

int main(int argc, char** argv) {
    if (argc != 4) {
        std::printf("usage: %s <db>.mygraph <db>.metadata <query>.query\n", argv[0]);
        return 1;
    }
    std::printf("loading database\n");
    gva_db* db = nullptr;
    int st = gva_db_load(argv[1], argv[2], 0, &db);
    if (st) return die(st);
    gva_db_info info;
    gva_db_get_info(db, &info);
    std::printf("maxid=%u\n", info.max_vertex_id);
    const char* w = gva_db_warnings(db);
    if (w && *w) std::printf("%s", w);

    auto t0 = std::chrono::steady_clock::now();
    gva_plan* plan = nullptr;
    st = gva_plan_from_file(argv[3], GVA_CLI_MODE, &plan);
    if (st) return die(st);
    std::string desc(gva_plan_describe(plan, nullptr, 0) + 1, '\0');
    gva_plan_describe(plan, &desc[0], desc.size());
    // phase list in the reference's wording (src/gpumine.cpp:923-931)
    {
        size_t pos = 0;
        while (pos < desc.size()) {
            size_t nl = desc.find('\n', pos);
            if (nl == std::string::npos) break;
            std::string line = desc.substr(pos, nl - pos);
            pos = nl + 1;
            unsigned idx, el, np;
            char type;
            int consumed = 0;
            if (std::sscanf(line.c_str(), "phase %u %c %u %u%n", &idx, &type, &el, &np, &consumed) == 4) {
                std::printf("phase %u type %c edge label:%u\n", idx, type, el);
                const char* p = line.c_str() + consumed;
                for (unsigned j = 0; j < np; ++j) {
                    unsigned a, b;
                    int used = 0;
                    if (std::sscanf(p, " %u %u%n", &a, &b, &used) != 2) break;
                    p += used;
                    std::printf("svid:%u evid:%u ", a, b);
                }
                std::printf("\n");
            }
        }
    }
    gva_result* res = nullptr;
    gva_match_opts opts;
    std::memset(&opts, 0, sizeof opts);
    st = gva_match(db, plan, &opts, &res);
    if (st) return die(st);
    auto t1 = std::chrono::steady_clock::now();
    double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    std::printf("time: %g\n", ms);
    std::printf("no error\n");
    const unsigned long long rows = (unsigned long long)gva_result_num_rows(res);
    const int width = gva_result_num_columns(res);
    std::printf("Result: %llu extra size0\n", rows);
    std::printf("PartialRowNum: %llu embLen:  %d\n", rows, width);
    st = gva_result_write_text(res, "partialResultsGPU.txt");
    if (st) return die(st);
    gva_result_free(res);
    gva_plan_free(plan);
    gva_db_free(db);
    return 0;
}
