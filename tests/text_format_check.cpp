// Test driver (CPU only): result rows as text (format_rows, what
// partialResultsGPU.txt holds) against the plain formatting of each value with
// std::to_string, for random rows of every width 1..32 (values including 0
// and 2^32 - 1), several thread counts and row counts around the split sizes.
//
// usage: text_format_check seed [max_rows]
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

#include "../geneva_b200/csrc/gva_internal.h"

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    std::mt19937 rng(atoi(argv[1]));
    const uint64_t max_rows = argc > 2 ? strtoull(argv[2], nullptr, 10) : ~0ull;
    int cases = 0;
    for (uint32_t w = 1; w <= 32; ++w)
        for (uint64_t n : {0ull, 1ull, 7ull, 65535ull, 65537ull, 200001ull}) {
            if ((n > 70000 && w > 2) || n > max_rows) continue;
            std::vector<uint32_t> rows(n * w);
            for (auto& x : rows) {
                const uint32_t k = rng() % 4;
                x = k == 0 ? 0 : k == 1 ? 0xffffffffu : k == 2 ? rng() % 1000 : (uint32_t)rng();
            }
            std::string want;
            for (uint64_t i = 0; i < n; ++i) {
                for (uint32_t c = 0; c < w; ++c) {
                    if (c) want.push_back(' ');
                    want += std::to_string(rows[i * w + c]);
                }
                want.push_back('\n');
            }
            for (unsigned threads : {1u, 3u, 8u}) {
                std::vector<std::string> parts;
                gva::format_rows(rows.data(), n, w, threads, parts);
                std::string got;
                for (auto& p : parts) got += p;
                if (got != want) {
                    printf("width %u rows %llu threads %u: text differs\n", w, (unsigned long long)n, threads);
                    return 1;
                }
                ++cases;
            }
        }
    printf("ok %d cases\n", cases);
    return 0;
}
