// Host worker pool (gva_pool.cpp): jobs from several threads at once, jobs
// posted from inside jobs, and jobs of one index; every index of every job
// must run exactly once and every job must return only after all of them.
//   pool_check <caller threads> <jobs per caller> <indices per job>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <thread>
#include <vector>

#include "../geneva_b200/csrc/gva_pool.h"

int main(int argc, char** argv) {
    const unsigned callers = argc > 1 ? (unsigned)atoi(argv[1]) : 4;
    const unsigned jobs = argc > 2 ? (unsigned)atoi(argv[2]) : 200;
    const unsigned width = argc > 3 ? (unsigned)atoi(argv[3]) : 37;
    std::atomic<int> bad{0};
    std::vector<std::thread> th;
    for (unsigned c = 0; c < callers; ++c)
        th.emplace_back([&, c]() {
            for (unsigned j = 0; j < jobs; ++j) {
                const unsigned n = (j % 5 == 0) ? 1 : width + (c + j) % 7;
                std::vector<std::atomic<int>> hits(n);
                for (auto& h : hits) h = 0;
                std::atomic<long> inner{0};
                gva::pool_run(n, [&](unsigned t) {
                    hits[t]++;
                    if (t % 3 == 0)  // a job posted from inside a job
                        gva::pool_run(4, [&](unsigned u) { inner += (long)u + 1; });
                });
                for (unsigned t = 0; t < n; ++t)
                    if (hits[t].load() != 1) bad++;
                long want = 0;
                for (unsigned t = 0; t < n; t += 3) want += 10;
                if (inner.load() != want) bad++;
            }
        });
    for (auto& t : th) t.join();
    if (bad.load()) {
        printf("FAIL %d\n", bad.load());
        return 1;
    }
    printf("ok %u threads\n", gva::pool_width());
    return 0;
}
