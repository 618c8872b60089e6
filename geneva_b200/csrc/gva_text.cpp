// Result rows as text, the layout of the reference's partialResults files
// (src/gpumine.cpp:184-199): one row per line, its values in decimal
// separated by single spaces.
#include <algorithm>
#include <cstring>
#include <thread>

#include "gva_internal.h"

namespace gva {

namespace {

inline char* put_u32(char* p, uint32_t x) {
    char tmp[10];
    int n = 0;
    do {
        tmp[n++] = (char)('0' + x % 10);
        x /= 10;
    } while (x);
    while (n) *p++ = tmp[--n];
    return p;
}

void format_range(const uint32_t* rows, uint64_t r0, uint64_t r1, uint32_t width, std::string& out) {
    out.resize((r1 - r0) * (width * 11ull + 1));  // at most 10 digits and a separator per value
    char* p = &out[0];
    for (uint64_t i = r0; i < r1; ++i) {
        const uint32_t* row = rows + i * width;
        for (uint32_t c = 0; c < width; ++c) {
            if (c) *p++ = ' ';
            p = put_u32(p, row[c]);
        }
        *p++ = '\n';
    }
    out.resize((size_t)(p - out.data()));
}

}  // namespace

void format_rows(const uint32_t* rows, uint64_t n, uint32_t width, unsigned threads, std::vector<std::string>& parts) {
    const unsigned t = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(std::max(1u, threads), (n + 65535) / 65536));
    parts.assign(t, std::string());
    if (t == 1) {
        format_range(rows, 0, n, width, parts[0]);
        return;
    }
    std::vector<std::thread> pool;
    for (unsigned k = 0; k < t; ++k)
        pool.emplace_back([&, k]() { format_range(rows, n * k / t, n * (k + 1) / t, width, parts[k]); });
    for (auto& th : pool) th.join();
}

}  // namespace gva
