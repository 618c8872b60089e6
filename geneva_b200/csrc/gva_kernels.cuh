// Device-side building blocks shared by the per-query and the batched
// engines: kernel argument blocks, segment lookup, membership test, block
// scans.  Included by gva_engine.cu and gva_batch.cu (internal linkage).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "gva_internal.h"

namespace gva {
namespace {

constexpr int kRowsPerBlock = 256;  // rows handled by one count/write block
constexpr int kThreads = 256;
constexpr int kScanThreads = 1024;
constexpr int kMaxChecks = 8;  // fused back-edge checks per extension

// ---------------------------------------------------------------- params ----
struct ExtArgs {
    const uint32_t* in;
    uint64_t nrows;
    uint32_t* out;
    const uint32_t* off;
    const uint32_t* adj;
    uint32_t k;        // input width
    uint32_t L;        // dense labels
    uint32_t lab;      // dense candidate label
    int32_t src_col;
    int32_t bound_col;
    uint32_t bound_incl;
    uint32_t n_eq;
    uint8_t eq_cols[kMaxCols];
    // fused back edges (batched engine): a candidate c is kept only if, for
    // every check i, c lies in seg_i(row[chk_col[i]], lab) (dir 0) or
    // row[chk_col[i]] lies in seg_i(c, chk_lab[i]) (dir 1)
    uint32_t n_chk;
    uint8_t chk_col[kMaxChecks];
    uint8_t chk_dir[kMaxChecks];
    uint32_t chk_lab[kMaxChecks];
    const uint32_t* chk_off[kMaxChecks];
    const uint32_t* chk_adj[kMaxChecks];
};

struct RedArgs {
    const uint32_t* in;
    uint64_t nrows;
    uint32_t* out;
    const uint32_t* off;
    const uint32_t* adj;
    uint32_t k;
    uint32_t L;
    uint32_t n_pairs;
    uint8_t rs[16];
    uint8_t re[16];
    uint32_t rl[16];
};

__device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }

// Label segment [lo, hi) of (vertex v, dense label l) in one partition's
// segment index.  Two layouts, chosen per database; bit 31 of L (kPackedSeg)
// marks the packed one:
//   dense   off[v * L + l] .. off[v * L + l + 1], (V + 1) * L + 1 words;
//   packed  one 32-byte record per vertex (one sector): word 0 = where v's
//           list starts in adj, bytes 4 .. 3 + L = cum[1 .. L], cum[j] = v's
//           neighbours with a label below j (cum[0] = 0 is not stored); a
//           vertex with more than 255 neighbours in the partition has bit 31
//           of word 0 set and word 1 = the word index, from `off`, of its
//           L + 1 uint32 cumulative counts.  For L <= 28.
// The packed index of a 20,000-graph database with 16 labels takes half the
// bytes of the dense one and every lookup is one sector, so the index of all
// partitions stays in L2 beside the frontiers.
__device__ __forceinline__ void seg_of(const uint32_t* __restrict__ off, uint32_t L, uint32_t v, uint32_t l,
                                       uint32_t& lo, uint32_t& hi) {
    if (!(L & kPackedSeg)) {
        const uint64_t t = (uint64_t)v * L + l;
        lo = __ldg(off + t);
        hi = __ldg(off + t + 1);
        return;
    }
    // the words holding word 0, cum[l] and cum[l + 1] are loaded together
    // (independent loads of one sector): one round trip for a narrow record
    const uint32_t* rec = off + (uint64_t)v * 8;
    const uint32_t bl = 3 + l, bh = 4 + l;  // bytes of cum[l] (l > 0) and cum[l + 1]
    const uint32_t w0 = __ldg(rec);
    const uint32_t wl = __ldg(rec + (bl >> 2));
    const uint32_t wh = __ldg(rec + (bh >> 2));
    const uint32_t base = w0 & 0x7fffffffu;
    if (w0 & 0x80000000u) {  // more than 255 neighbours: a row of cumulative words
        const uint32_t* cw = off + __ldg(rec + 1);
        lo = base + __ldg(cw + l);
        hi = base + __ldg(cw + l + 1);
        return;
    }
    hi = base + ((wh >> (8 * (bh & 3))) & 0xffu);
    lo = base + (l > 0 ? (wl >> (8 * (bl & 3))) & 0xffu : 0u);
}

// first index in [lo, hi) with a[i] >= x (hi if none)
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* __restrict__ a, uint32_t lo, uint32_t hi,
                                                    uint64_t x) {
    while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if ((uint64_t)__ldg(a + mid) < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Candidate range of one row: the (source, label) segment cut below the
// restriction bound.
__device__ __forceinline__ void ext_range(const ExtArgs& p, const uint32_t* row, uint32_t& lo, uint32_t& hi) {
    seg_of(p.off, p.L, row[p.src_col], p.lab, lo, hi);
    if (p.bound_col >= 0 && lo < hi) {
        const uint64_t b = (uint64_t)row[p.bound_col] + p.bound_incl;
        hi = lower_bound_u32(p.adj, lo, hi, b);
    }
}

// Position of w in adj[lo, hi), or 0xffffffff.
__device__ __forceinline__ uint32_t find_in(const uint32_t* __restrict__ adj, uint32_t lo, uint32_t hi, uint32_t w) {
    if (lo >= hi) return 0xffffffffu;
    if (w < __ldg(adj + lo) || w > __ldg(adj + hi - 1)) return 0xffffffffu;
    const uint32_t pos = lower_bound_u32(adj, lo, hi, w);
    return (pos < hi && __ldg(adj + pos) == w) ? pos : 0xffffffffu;
}

// Candidate source of a row with fused checks: the shortest of the source
// segment and the dir-0 check segments, each cut below the restriction
// bound.  The segments stay in the state, so that membership tests of the
// candidates need no offset loads (a candidate lies below the bound, so the
// cut segments answer membership as the full ones would).
struct GenState {
    const uint32_t* gadj;
    uint32_t lo, hi;  // generator range
    int which;        // -1 = source, else the check index
    uint32_t slo, shi;                          // source segment
    uint32_t clo[kMaxChecks], chi[kMaxChecks];  // dir-0 check segments
};

__device__ __forceinline__ void ext_generator(const ExtArgs& p, const uint32_t* row, GenState& g) {
    uint32_t slo, shi;
    seg_of(p.off, p.L, row[p.src_col], p.lab, slo, shi);
    g.gadj = p.adj;
    g.which = -1;
    if (slo >= shi) {  // no candidate from the source: nothing else to look up
        g.lo = g.hi = g.slo = g.shi = slo;
        return;
    }
    // the partners' segments are looked up together (independent loads),
    // then every segment is cut below the restriction bound
    uint32_t l2[kMaxChecks], h2[kMaxChecks];
#pragma unroll
    for (int i = 0; i < kMaxChecks; ++i) {
        l2[i] = h2[i] = 0;
        if (i < (int)p.n_chk && !p.chk_dir[i]) seg_of(p.chk_off[i], p.L, row[p.chk_col[i]], p.lab, l2[i], h2[i]);
    }
    if (p.bound_col >= 0) {
        const uint64_t b = (uint64_t)row[p.bound_col] + p.bound_incl;
        shi = lower_bound_u32(p.adj, slo, shi, b);
#pragma unroll
        for (int i = 0; i < kMaxChecks; ++i)
            if (i < (int)p.n_chk && !p.chk_dir[i] && l2[i] < h2[i]) h2[i] = lower_bound_u32(p.chk_adj[i], l2[i], h2[i], b);
    }
    g.slo = slo;
    g.shi = shi;
    g.lo = slo;
    g.hi = shi;
#pragma unroll
    for (int i = 0; i < kMaxChecks; ++i) {
        if (i >= (int)p.n_chk || p.chk_dir[i]) continue;
        g.clo[i] = l2[i];
        g.chi[i] = h2[i];
        if (h2[i] - l2[i] < g.hi - g.lo) {
            g.lo = l2[i];
            g.hi = h2[i];
            g.gadj = p.chk_adj[i];
            g.which = i;
        }
    }
}

__device__ __forceinline__ bool seg_has(const uint32_t* __restrict__ off, const uint32_t* __restrict__ adj, uint32_t L,
                                        uint32_t v, uint32_t lab, uint32_t w) {
    uint32_t lo, hi;
    seg_of(off, L, v, lab, lo, hi);
    return find_in(adj, lo, hi, w) != 0xffffffffu;
}

// Whether generated candidate c survives injectivity, the source edge (when
// the generator is a check segment) and every other check.
__device__ __forceinline__ bool ext_accept(const ExtArgs& p, const uint32_t* row, uint32_t c, const GenState& g) {
    for (uint32_t j = 0; j < p.n_eq; ++j)
        if (row[p.eq_cols[j]] == c) return false;
    if (g.which >= 0 && find_in(p.adj, g.slo, g.shi, c) == 0xffffffffu) return false;
    for (uint32_t i = 0; i < p.n_chk; ++i) {
        if ((int)i == g.which) continue;
        const bool ok = p.chk_dir[i] ? seg_has(p.chk_off[i], p.chk_adj[i], p.L, c, p.chk_lab[i], row[p.chk_col[i]])
                                     : find_in(p.chk_adj[i], g.clo[i], g.chi[i], c) != 0xffffffffu;
        if (!ok) return false;
    }
    return true;
}

// Candidates of a short list [lo, hi) below bound b that equal none of the
// row's NEQ matched vertices (columns eq_cols), in one pass over the list;
// the list is ascending, so the walk stops at the bound (no search for it).
// A vertex in two columns still excludes its candidate once.
template <int NEQ>
__device__ __forceinline__ uint32_t short_list_count(const uint32_t* __restrict__ adj, uint32_t lo, uint32_t hi,
                                                     uint64_t b, const uint32_t* row, const uint8_t* eq_cols) {
    uint32_t eqv[NEQ > 0 ? NEQ : 1];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) eqv[e] = row[eq_cols[e]];
    uint32_t m = 0;
    for (uint32_t j = lo; j < hi; ++j) {
        const uint32_t c = __ldg(adj + j);
        if ((uint64_t)c >= b) break;
        bool coll = false;
#pragma unroll
        for (int e = 0; e < NEQ; ++e) coll |= c == eqv[e];
        m += coll ? 0u : 1u;
    }
    return m;
}

// Number of candidates of one row of a plain extension (no fused checks):
// the segment below the restriction bound minus the already-matched
// vertices in it.
__device__ __forceinline__ uint32_t ext_count_plain(const ExtArgs& p, const uint32_t* row) {
    uint32_t lo, hi;
    seg_of(p.off, p.L, row[p.src_col], p.lab, lo, hi);
    if (lo >= hi) return 0;
    const uint32_t n_eq = p.n_eq;
    if (hi - lo <= 8 && n_eq <= 8) {
        const uint64_t b = p.bound_col >= 0 ? (uint64_t)row[p.bound_col] + p.bound_incl : ~0ull;
        switch (n_eq) {
            case 0: return short_list_count<0>(p.adj, lo, hi, b, row, p.eq_cols);
            case 1: return short_list_count<1>(p.adj, lo, hi, b, row, p.eq_cols);
            case 2: return short_list_count<2>(p.adj, lo, hi, b, row, p.eq_cols);
            case 3: return short_list_count<3>(p.adj, lo, hi, b, row, p.eq_cols);
            case 4: return short_list_count<4>(p.adj, lo, hi, b, row, p.eq_cols);
            case 5: return short_list_count<5>(p.adj, lo, hi, b, row, p.eq_cols);
            case 6: return short_list_count<6>(p.adj, lo, hi, b, row, p.eq_cols);
            case 7: return short_list_count<7>(p.adj, lo, hi, b, row, p.eq_cols);
            default: return short_list_count<8>(p.adj, lo, hi, b, row, p.eq_cols);
        }
    }
    if (p.bound_col >= 0) {
        const uint64_t b = (uint64_t)row[p.bound_col] + p.bound_incl;
        hi = lower_bound_u32(p.adj, lo, hi, b);
        if (lo >= hi) return 0;
    }
    uint32_t n = hi - lo;
    for (uint32_t j = 0; j < p.n_eq; ++j) {
        const uint32_t w = row[p.eq_cols[j]];
        bool dup = false;  // the same vertex in two columns collides once
        for (uint32_t i = 0; i < j; ++i) dup |= (row[p.eq_cols[i]] == w);
        if (!dup && find_in(p.adj, lo, hi, w) != 0xffffffffu) --n;
    }
    return n;
}

// Number of candidates of one row, plain or with fused checks.
__device__ __forceinline__ uint32_t ext_count_row(const ExtArgs& p, const uint32_t* row) {
    if (p.n_chk) {
        GenState g;
        ext_generator(p, row, g);
        uint32_t n = 0;
        for (uint32_t j = g.lo; j < g.hi; ++j) n += ext_accept(p, row, __ldg(g.gadj + j), g) ? 1u : 0u;
        return n;
    }
    return ext_count_plain(p, row);
}

__device__ __forceinline__ bool red_keep_row(const RedArgs& p, const uint32_t* row) {
    for (uint32_t j = 0; j < p.n_pairs; ++j) {
        const uint32_t s = row[p.rs[j]];
        const uint32_t e = row[p.re[j]];
        uint32_t lo, hi;
        seg_of(p.off, p.L, s, p.rl[j], lo, hi);
        if (find_in(p.adj, lo, hi, e) == 0xffffffffu) return false;
    }
    return true;
}

// ------------------------------------------------------------ block sums ----
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void store_block_sum(uint64_t v, uint64_t* block_sums) {
    __shared__ uint64_t ws[kThreads / 32];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint64_t x = threadIdx.x < kThreads / 32 ? ws[threadIdx.x] : 0;
        x = warp_sum(x);
        if (threadIdx.x == 0) block_sums[blockIdx.x] = x;
    }
}

// Exclusive scan of 256 per-thread values in shared memory (uint64).
__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t* total) {
    __shared__ uint64_t ws[kThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint64_t w = lane < kThreads / 32 ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kThreads / 32) ws[lane] = w;
    }
    __syncthreads();
    const uint64_t before = (wid > 0 ? ws[wid - 1] : 0) + x - v;
    *total = ws[kThreads / 32 - 1];
    __syncthreads();
    return before;
}

// In-place exclusive scan of n block totals; sums[n] receives the total.
__global__ void __launch_bounds__(kScanThreads) scan_block_sums_kernel(uint64_t* __restrict__ sums, uint64_t n) {
    __shared__ uint64_t ws[kScanThreads / 32];
    __shared__ uint64_t carry_s;
    if (threadIdx.x == 0) carry_s = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint64_t base = 0; base < n; base += kScanThreads) {
        const uint64_t i = base + threadIdx.x;
        const uint64_t v = i < n ? sums[i] : 0;
        uint64_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) ws[wid] = x;
        __syncthreads();
        if (wid == 0) {
            uint64_t w = ws[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            ws[lane] = w;
        }
        __syncthreads();
        const uint64_t carry = carry_s;
        if (i < n) sums[i] = carry + (wid > 0 ? ws[wid - 1] : 0) + x - v;
        __syncthreads();
        if (threadIdx.x == 0) carry_s = carry + ws[kScanThreads / 32 - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[n] = carry_s;
}

}  // namespace
}  // namespace gva
