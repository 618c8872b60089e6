// Batched engine: many query patterns advance together.
//
// A task is (query, slice of that query's frontier, next step).  One round
// advances every active task by one step:
//   count   one launch over the 256-row blocks of all tasks (per-task step
//           parameters from a descriptor array); final steps in count mode
//           also add their rows into per-(query, graph) counters and graph
//           bitmaps here and never write rows
//   scan    exclusive scan of all block totals
//   totals  per-task output rows
//   write   persistent kernel: blocks pull 256-row items from an atomic work
//           queue (load balance across SMs however uneven the tasks are) and
//           expand / compact them into the round's output buffer
// A task whose output does not fit the memory budget is split in half (its
// input rows) and retried next round, so any frontier is processed in
// budget-sized pieces, deepest tasks first.  This replaces the reference's
// kernel-abort/host-spill protocol (src/gpumine.cpp:406-467,
// src/miningPattern.cu:3325-3343) and its one-query-per-process driver.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <map>
#include <mutex>
#include <unordered_map>
#include <numeric>
#include <string>
#include <future>
#include <tuple>
#include <thread>
#include <vector>

#include "../../include/geneva.h"
#include "gva_engine.cuh"
#include "gva_kernels.cuh"
#include "gva_pool.h"

namespace gva {

namespace {

#define GVA_CUDA_B(call)                                                                                \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return fail(GVA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));              \
    } while (0)

// WRITE: output feeds child steps; COUNT: a plan ends here; *_GRAPHS: it also
// needs per-graph accounting (slot `query`).
enum TaskMode : uint32_t { MODE_WRITE = 0, MODE_COUNT = 1, MODE_COUNT_GRAPHS = 2, MODE_WRITE_AND_GRAPHS = 3 };

// Step parameters of one trie node, uploaded once per node.  The frontier
// fields of the argument blocks (in, nrows, out) are unused here: a task's
// frontier slice comes with its TaskRef.
struct TaskDesc {
    uint32_t kind;     // STEP_EXT / STEP_REDUCE
    uint32_t mode;     // TaskMode
    uint32_t query;    // per-graph result slot
    uint32_t pad;
    union {
        ExtArgs e;
        RedArgs r;
    };
};

struct BatchCtx {
    uint64_t* graph_counts;   // [nq * G] or null
    uint32_t* graph_bits;     // [nq * words] or null
    const uint32_t* vgraph;   // vertex -> graph
    uint32_t G;
    uint32_t words;           // bitmap words per query
};

// Per-round task reference: a node's descriptor and a frontier slice.  The
// slice is cut into items of `rows_per_item` rows; task t owns the count
// pass's items [item0[t], item0[t + 1]).
struct TaskRef {
    uint32_t node;
    uint32_t pad;
    const uint32_t* in;
    uint64_t nrows;
};

constexpr int kRoundWarps = 8;          // warps per CTA of the round kernels
constexpr int kMaxItemRows = 128;       // rows of one work item (a multiple of 32)
constexpr int kTileRows = 64;           // output rows staged per warp before a coalesced flush
constexpr int kScanChunk = 4096;        // items per CTA of the item scan
constexpr int kScanChunkLog2 = 12;

// Device-side state of one round when the rounds are scheduled on the device
// (BatchSession::run_device): the count pass's tasks and items (written by
// the previous round's planning kernel, or by the host for the first round),
// the write pass's (written by this round's planning kernel) and the four
// work-queue heads (zero when the state is created).  A set `overflow` makes
// every later launch of the run find no work.
struct RunState {
    uint64_t ni, ni_light;  // count items: all, light class (the light class's items come first)
    uint64_t wi, wi_light;  // write items: all, light class
    uint32_t nt, nt_light;  // count tasks: all, light class
    uint32_t nw;            // writing tasks
    uint32_t overflow;      // frontier region, task or item capacity exceeded
    unsigned long long heads[4];  // queue heads: count light, count fused, write light, write fused
};

struct RoundArgs {
    const TaskDesc* nodes;
    const TaskRef* refs;
    const uint64_t* item0;        // [nt + 1] count-pass item prefix
    uint64_t item_base;           // first item of this launch (its task class's range)
    uint64_t n_items;             // items of this launch
    const uint32_t* wtask;        // write: task of each writing task slot (null for the count pass)
    const uint64_t* witem0;       // write: [nw + 1] item prefix over the writing tasks
    uint32_t nt;                  // tasks (count) or writing tasks (write)
    uint32_t rows_per_item;       // multiple of 32, <= kMaxItemRows
    uint32_t hub;                 // candidate lists longer than this are shared by the whole warp
    uint32_t kmax;                // widest input row of the round (shared-memory layout)
    uint64_t* items;              // count: per-item output rows; write: their exclusive scan
    const uint64_t* chunks;       // write: exclusive scan of the per-chunk sums, chunks[n_chunks] = total
    uint64_t n_count_items;       // write: items of the count pass
    uint64_t n_chunks;            // write: scan chunks of the count pass
    unsigned long long* queue;    // work-queue head (zeroed before the launch)
    uint32_t* const* task_out;    // write: output base of each task (null: not written this round)
    unsigned long long* read_words;  // optional: candidate-list words read (profiling)
    BatchCtx ctx;
    RunState* dyn;                // device-scheduled rounds: item ranges, task counts and queue heads from
                                  // here instead of the fields above (null: host-scheduled)
};

// The item range of one launch: from the arguments (host-scheduled rounds)
// or from the round's device state.
struct Span {
    uint64_t base, n;              // items [base, base + n) of this launch
    uint64_t n_count_items, n_chunks;  // write pass: items and scan chunks of the count pass
    unsigned long long* queue;
    uint32_t nt;                   // tasks (count) or writing tasks (write)
    uint32_t warps;                // resident warps of the persistent grid
};

template <bool WRITE>
__device__ __forceinline__ Span launch_span(const RoundArgs& a, bool fused) {
    Span s;
    s.warps = gridDim.x * kRoundWarps;
    if (!a.dyn) {
        s.base = a.item_base;
        s.n = a.n_items;
        s.nt = a.nt;
        s.n_count_items = a.n_count_items;
        s.n_chunks = a.n_chunks;
        s.queue = a.queue;
        return s;
    }
    const RunState& st = *a.dyn;
    const uint64_t all = WRITE ? st.wi : st.ni, light = WRITE ? st.wi_light : st.ni_light;
    s.base = fused ? light : 0;
    s.n = fused ? all - light : light;
    s.nt = WRITE ? st.nw : st.nt;
    s.n_count_items = st.ni;
    s.n_chunks = (st.ni + kScanChunk - 1) / kScanChunk;
    s.queue = a.dyn->heads + (WRITE ? 2 : 0) + (fused ? 1 : 0);
    return s;
}

// Per-(query, graph) accounting of a final-step row: lanes of a warp whose
// rows lie in the same graph (rows arrive grouped by their first vertex)
// combine their counts before one 64-bit atomic.
__device__ __forceinline__ void add_graph_count(const BatchCtx& c, uint32_t query, uint32_t first_vertex, uint32_t cnt,
                                                bool valid) {
    uint32_t g = 0xffffffffu;
    if (valid && cnt > 0) g = __ldg(c.vgraph + first_vertex);
    const bool take = g < c.G;  // vertices outside every declared graph are not counted
    const uint32_t active = __ballot_sync(0xffffffffu, take);
    if (!take) return;
    const uint32_t peers = __match_any_sync(active, g);
    const uint32_t sum = __reduce_add_sync(peers, cnt);
    if ((threadIdx.x & 31) == (uint32_t)(__ffs(peers) - 1)) {
        if (c.graph_counts) atomicAdd((unsigned long long*)(c.graph_counts + (uint64_t)query * c.G + g), (unsigned long long)sum);
        if (c.graph_bits) atomicOr(c.graph_bits + (uint64_t)query * c.words + (g >> 5), 1u << (g & 31));
    }
}

// Guided self-scheduling over a device work queue: a warp takes a chunk of
// about 1/(2 x resident warps) of the items left (at least one), so the
// queue sees few atomics while the last items still spread over every SM.
__device__ __forceinline__ bool next_chunk(const Span& a, uint64_t& begin, uint64_t& end) {
    const int lane = threadIdx.x & 31;
    unsigned long long b = 0, n = 0;
    if (lane == 0) {
        const unsigned long long head = *(volatile unsigned long long*)a.queue;
        if (head < a.n) {
            n = (a.n - head) / (2ull * a.warps);
            if (n == 0) n = 1;
            b = atomicAdd(a.queue, n);
        } else {
            b = a.n;
        }
    }
    b = __shfl_sync(0xffffffffu, b, 0);
    n = __shfl_sync(0xffffffffu, n, 0);
    begin = b;
    end = b + n < a.n ? b + n : a.n;
    return begin < a.n;
}

// last t in [0, n) with pfx[t] <= x (pfx ascending, pfx[0] <= x)
__device__ __forceinline__ uint32_t find_slot(const uint64_t* __restrict__ pfx, uint32_t n, uint64_t x) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(pfx + mid) <= x)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// One warp's copy of a node descriptor.
__device__ __forceinline__ void load_desc(TaskDesc& d, const TaskDesc* __restrict__ src) {
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    uint32_t* dw = reinterpret_cast<uint32_t*>(&d);
    for (int i = threadIdx.x & 31; i < (int)(sizeof(TaskDesc) / 4); i += 32) dw[i] = __ldg(s + i);
    __syncwarp();
}

// Rows [row0, row0 + nr) of a frontier of width k into shared memory,
// coalesced (16-byte loads when the slice is 16-byte aligned).
__device__ __forceinline__ void stage_rows(uint32_t* rows_s, const uint32_t* __restrict__ in, uint64_t row0, uint32_t nr,
                                           uint32_t k) {
    const int lane = threadIdx.x & 31;
    const uint32_t* src = in + row0 * k;
    const uint32_t nw = nr * k;
    uint32_t w0 = 0;
    if ((((uintptr_t)src | (uintptr_t)rows_s) & 15) == 0) {
        const uint32_t nv = nw >> 2;
        const uint4* s4 = reinterpret_cast<const uint4*>(src);
        uint4* d4 = reinterpret_cast<uint4*>(rows_s);
        for (uint32_t v = lane; v < nv; v += 32) d4[v] = __ldg(s4 + v);
        w0 = nv << 2;
    }
    for (uint32_t w = w0 + lane; w < nw; w += 32) rows_s[w] = __ldg(src + w);
    __syncwarp();
}

// cp.async (sm_80+ asynchronous global -> shared copies): a warp issues the
// next item's rows while it works on the current one.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Issues, without waiting, the copy of rows [row0, row0 + nr) of width k
// into rows_s (16-byte copies when the slice is 16-byte aligned); each lane
// commits one group.
__device__ __forceinline__ void stage_rows_async(uint32_t* rows_s, const uint32_t* __restrict__ in, uint64_t row0,
                                                 uint32_t nr, uint32_t k) {
    const int lane = threadIdx.x & 31;
    const uint32_t* src = in + row0 * k;
    const uint32_t nw = nr * k;
    uint32_t w0 = 0;
    if ((((uintptr_t)src | (uintptr_t)rows_s) & 15) == 0) {
        const uint32_t nv = nw >> 2;
        for (uint32_t v = lane; v < nv; v += 32) cp_async16(rows_s + 4 * v, src + 4 * v);
        w0 = nv << 2;
    }
    for (uint32_t w = w0 + lane; w < nw; w += 32) cp_async4(rows_s + w, src + w);
    cp_async_commit();
}

// Candidate test of the plain extension (no fused checks): injectivity only;
// the restriction bound is already applied to the range.
__device__ __forceinline__ bool ext_injective(const ExtArgs& p, const uint32_t* row, uint32_t c) {
    for (uint32_t j = 0; j < p.n_eq; ++j)
        if (row[p.eq_cols[j]] == c) return false;
    return true;
}

// The same test against the row's matched vertices held in registers
// (extensions with at most 8 injectivity columns; unused entries never
// equal a vertex id).
__device__ __forceinline__ void load_eqv(const ExtArgs& p, const uint32_t* row, uint32_t (&eqv)[8]) {
    const uint32_t n = p.n_eq;
#pragma unroll
    for (int e = 0; e < 8; ++e) eqv[e] = e < (int)n ? row[p.eq_cols[e]] : 0xffffffffu;
}
__device__ __forceinline__ bool injective8(const uint32_t (&eqv)[8], uint32_t c) {
    bool coll = false;
#pragma unroll
    for (int e = 0; e < 8; ++e) coll |= c == eqv[e];
    return !coll;
}

// Output staging of one warp: every accepted (row, candidate) is appended
// in ballot order to a shared tile as a pair (offset of the row among the
// warp's staged rows, candidate), and the tile is flushed 32 rows at a time:
// the lanes write the output words in order (coalesced stores), each read
// from the staged row or from the pair.  Two words per output row in shared
// memory instead of the whole row.
struct Tile {
    uint32_t* t;           // kTileRows (row offset, candidate) pairs
    const uint32_t* base;  // the staged rows the offsets point into
    uint32_t k;            // input row width
    uint32_t w;            // output row width: k + 1 (extension) or k (reduction)
    uint32_t inv;          // ceil(2^20 / w): q / w = (q * inv) >> 20 for every q < kTileRows * w
    uint32_t n;            // rows held
    uint32_t* out;         // next output row in global memory
    uint64_t room;         // rows this item may still write (its count from the count pass)
};

__device__ __forceinline__ void tile_init(Tile& tl, uint32_t* t, const uint32_t* base, uint32_t k, bool extend,
                                          uint32_t* out, uint64_t room) {
    tl.t = t;
    tl.base = base;
    tl.k = k;
    tl.w = extend ? k + 1 : k;
    tl.inv = ((1u << 20) + tl.w - 1) / tl.w;
    tl.n = 0;
    tl.out = out;
    tl.room = room;
}

__device__ __forceinline__ void tile_flush(Tile& tl, uint32_t rows) {
    const int lane = threadIdx.x & 31;
    // never past the item's counted rows, whatever the data (e.g. repeated
    // neighbours, which the count and write tests would see differently)
    const uint32_t keep = (uint32_t)umin64(rows, tl.room);
    const uint32_t kw = keep * tl.w;
    for (uint32_t q = lane; q < kw; q += 32) {
        const uint32_t r = (q * tl.inv) >> 20;
        const uint32_t col = q - r * tl.w;
        tl.out[q] = col < tl.k ? tl.base[tl.t[2 * r] + col] : tl.t[2 * r + 1];
    }
    tl.out += kw;
    tl.room -= keep;
    __syncwarp();
    const uint32_t rest = 2 * (tl.n - rows);
    for (uint32_t q = lane; q < rest; q += 32) tl.t[q] = tl.t[2 * rows + q];
    tl.n -= rows;
    __syncwarp();
}

// Appends, for every lane with `take`, its row (`row`, among the staged
// rows) extended by `c` (an extension) or alone (a reduction).
__device__ __forceinline__ void tile_append(Tile& tl, bool take, const uint32_t* row, uint32_t c) {
    const int lane = threadIdx.x & 31;
    const uint32_t m = __ballot_sync(0xffffffffu, take);
    if (take) {
        const uint32_t pos = tl.n + __popc(m & ((1u << lane) - 1u));
        tl.t[2 * pos] = (uint32_t)(row - tl.base);
        tl.t[2 * pos + 1] = c;
    }
    tl.n += __popc(m);
    __syncwarp();
    if (tl.n >= 32) tile_flush(tl, 32);
}

// ------------------------------------------------------------ one item ----
// Tasks come in two classes with their own kernels (so that each gets the
// registers, and the occupancy, its work needs):
//   light  plain extensions (no fused checks) and reductions: a lane per row;
//   fused  extensions with fused back-edge checks: a row's candidates come
//          from its generator segment (ext_generator) and every candidate is
//          tested against the other segments; each lane's generator state
//          lives in shared memory, where the whole warp can read it.
// In both, a row whose candidate list is at most `hub` long is walked by its
// lane; longer lists are shared by the warp, 32 candidates per step.  COUNT
// returns the item's accepted candidates (valid in every lane) and does the
// per-graph accounting; WRITE appends every accepted (row, candidate) to the
// tile.  Both passes visit the same candidates with the same test.
template <bool WRITE, bool FUSED>
__device__ __forceinline__ uint64_t ext_item(const TaskDesc& d, const uint32_t* rows_s, uint32_t nr, uint32_t hub,
                                             const BatchCtx& ctx, Tile* tl, GenState* gen_s,
                                             unsigned long long* read_words) {
    const ExtArgs& p = d.e;
    const int lane = threadIdx.x & 31;
    const uint32_t k = p.k;
    const bool graphs = !WRITE && (d.mode == MODE_COUNT_GRAPHS || d.mode == MODE_WRITE_AND_GRAPHS);
    uint64_t total = 0;
    uint64_t words = 0;
    for (uint32_t base = 0; base < nr; base += 32) {
        const uint32_t r = base + lane;
        const bool valid = r < nr;
        const uint32_t* row = rows_s + (valid ? r : 0) * k;
        uint32_t cnt = 0;
        if (!FUSED && !WRITE) {
            // plain extension: the segment minus the matched vertices in it
            if (valid) cnt = ext_count_plain(p, row);
        } else {
            uint32_t lo = 0, hi = 0;
            if (FUSED) {
                GenState& g = gen_s[lane];
                if (valid) {
                    ext_generator(p, row, g);
                    lo = g.lo;
                    hi = g.hi;
                }
            } else if (valid) {
                ext_range(p, row, lo, hi);
            }
            const uint32_t len = hi > lo ? hi - lo : 0;
            const bool is_hub = len > hub;
            const uint32_t mine = is_hub ? 0 : len;
            words += mine;
            const uint32_t* gadj = FUSED ? gen_s[lane].gadj : p.adj;
            const bool eq8 = p.n_eq <= 8;  // matched vertices in registers
            uint32_t eqv[8];
            if (!FUSED && eq8) load_eqv(p, row, eqv);
            // own rows: lanes step through their lists together
            const uint32_t steps = __reduce_max_sync(0xffffffffu, mine);
            for (uint32_t s = 0; s < steps; ++s) {
                bool ok = false;
                uint32_t c = 0;
                if (s < mine) {
                    c = __ldg(gadj + lo + s);
                    ok = FUSED ? ext_accept(p, row, c, gen_s[lane]) : (eq8 ? injective8(eqv, c) : ext_injective(p, row, c));
                }
                cnt += ok ? 1u : 0u;
                if (WRITE) tile_append(*tl, ok, row, c);
            }
            // hub rows: the whole warp.  Lists of 128 candidates or more are
            // read as 16-byte vectors (4 consecutive candidates per lane, 128
            // per step) from the 16-byte boundary at or below the list's
            // start: adjacency arrays start 16-byte aligned and end with 16
            // bytes of slack, so the vectors around a list's ends stay inside
            // the allocation.  Shorter ones go 32 candidates per step, one per
            // lane, which keeps every lane busy on them.
            uint32_t hubs = __ballot_sync(0xffffffffu, is_hub);
            if (FUSED) __syncwarp();  // generator states written before other lanes read them
            while (hubs) {
                const int h = __ffs(hubs) - 1;
                hubs &= hubs - 1;
                const uint32_t hlo = __shfl_sync(0xffffffffu, lo, h), hhi = __shfl_sync(0xffffffffu, hi, h);
                const uint32_t* hrow = rows_s + (base + h) * k;
                const uint32_t* hadj = FUSED ? gen_s[h].gadj : p.adj;
                if (!FUSED && eq8) load_eqv(p, hrow, eqv);
                uint32_t hc = 0;
                if (hhi - hlo >= 128) {
                    for (uint32_t j0 = hlo & ~3u; j0 < hhi; j0 += 128) {
                        const uint32_t j = j0 + 4 * lane;
                        uint4 v4 = make_uint4(0, 0, 0, 0);
                        if (j < hhi) v4 = __ldg(reinterpret_cast<const uint4*>(hadj + j));
                        const uint32_t vv[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const uint32_t c = vv[q];
                            bool ok = false;
                            if (j + q >= hlo && j + q < hhi)
                                ok = FUSED ? ext_accept(p, hrow, c, gen_s[h])
                                           : (eq8 ? injective8(eqv, c) : ext_injective(p, hrow, c));
                            hc += ok ? 1u : 0u;
                            if (WRITE) tile_append(*tl, ok, hrow, c);
                        }
                    }
                } else {
                    for (uint32_t j0 = hlo; j0 < hhi; j0 += 32) {
                        const uint32_t j = j0 + lane;
                        bool ok = false;
                        uint32_t c = 0;
                        if (j < hhi) {
                            c = __ldg(hadj + j);
                            ok = FUSED ? ext_accept(p, hrow, c, gen_s[h])
                                       : (eq8 ? injective8(eqv, c) : ext_injective(p, hrow, c));
                        }
                        hc += ok ? 1u : 0u;
                        if (WRITE) tile_append(*tl, ok, hrow, c);
                    }
                }
                hc = __reduce_add_sync(0xffffffffu, hc);
                if (lane == h) cnt += hc;
                if (lane == 0) words += hhi - hlo;
            }
            if (FUSED) __syncwarp();  // every lane done with the states before the next rows overwrite them
        }
        if (graphs) add_graph_count(ctx, d.query, row[0], cnt, valid);
        total += cnt;
    }
    if (read_words) {
        words = warp_sum(words);
        if (lane == 0 && words) atomicAdd(read_words, (unsigned long long)words);
    }
    return warp_sum(total);
}

template <bool WRITE>
__device__ __forceinline__ uint64_t red_item(const TaskDesc& d, const uint32_t* rows_s, uint32_t nr,
                                             const BatchCtx& ctx, Tile* tl) {
    const RedArgs& p = d.r;
    const int lane = threadIdx.x & 31;
    const uint32_t k = p.k;
    const bool graphs = !WRITE && (d.mode == MODE_COUNT_GRAPHS || d.mode == MODE_WRITE_AND_GRAPHS);
    uint64_t total = 0;
    for (uint32_t base = 0; base < nr; base += 32) {
        const uint32_t r = base + lane;
        const bool valid = r < nr;
        const uint32_t* row = rows_s + (valid ? r : 0) * k;
        const bool keep = valid && red_keep_row(p, row);
        if (WRITE) tile_append(*tl, keep, row, 0u);
        if (graphs) add_graph_count(ctx, d.query, row[0], keep ? 1u : 0u, valid);
        total += keep ? 1u : 0u;
    }
    return warp_sum(total);
}

// Class of a task: fused extensions apart from everything else.
__host__ __device__ __forceinline__ bool fused_class(uint32_t kind, uint32_t n_chk) {
    return kind == STEP_EXT && n_chk > 0;
}

// Shared memory of one warp: the item's rows, (write pass) the output tile
// and (fused class) the lanes' generator states; before them, one descriptor
// copy per warp.
constexpr size_t kGenBytes = 32 * sizeof(GenState);  // per warp
// The light class double-buffers the item rows (the next item's rows are
// copied in while the current item is worked on); the fused class, whose
// generator states already take shared memory, stages one item at a time.
__host__ __device__ constexpr uint32_t row_buffers(bool fused) { return fused ? 1u : 2u; }
__host__ __device__ constexpr size_t round_warp_words(uint32_t rows_per_item, uint32_t kmax, bool write, bool fused) {
    return (((size_t)row_buffers(fused) * rows_per_item * kmax + (write ? (size_t)kTileRows * 2 : 0)) + 3) &
           ~(size_t)3;
}
size_t round_smem_bytes(uint32_t rows_per_item, uint32_t kmax, bool write, bool fused) {
    return (size_t)kRoundWarps *
           (sizeof(TaskDesc) + (fused ? kGenBytes : 0) + 4 * round_warp_words(rows_per_item, kmax, write, fused));
}

struct WarpSmem {
    TaskDesc* d;
    uint32_t* rows;   // one or two buffers of rows_per_item * kmax words
    uint32_t* rows2;  // the second buffer (light class)
    uint32_t* tile;
    GenState* gen;
};
template <bool WRITE, bool FUSED>
__device__ __forceinline__ WarpSmem warp_smem(unsigned char* raw, const RoundArgs& a) {
    const int warp = threadIdx.x >> 5;
    WarpSmem w;
    w.d = reinterpret_cast<TaskDesc*>(raw) + warp;
    unsigned char* area = raw + kRoundWarps * sizeof(TaskDesc);  // 8-byte aligned: TaskDesc holds pointers
    w.gen = FUSED ? reinterpret_cast<GenState*>(area) + 32 * warp : nullptr;
    uint32_t* words = reinterpret_cast<uint32_t*>(area + (FUSED ? kRoundWarps * kGenBytes : 0));
    w.rows = words + warp * round_warp_words(a.rows_per_item, a.kmax, WRITE, FUSED);
    w.rows2 = w.rows + (size_t)(row_buffers(FUSED) - 1) * a.rows_per_item * a.kmax;
    w.tile = w.rows + (size_t)row_buffers(FUSED) * a.rows_per_item * a.kmax;
    return w;
}

// ---------------------------------------------------------- count pass ----
// Persistent: warps pull chunks of items from the work queue; each item's
// accepted rows go to items[item] (no atomics, no block barrier).  One
// instance per task class over that class's range of items.
template <bool FUSED>
__global__ void __launch_bounds__(kRoundWarps * 32, FUSED ? 5 : 6)
round_count_kernel(RoundArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const WarpSmem ws = warp_smem<false, FUSED>(smem_raw, a);
    TaskDesc& d = *ws.d;
    uint32_t t = 0xffffffffu;
    uint64_t t_lo = 0, t_hi = 0;
    const uint32_t* in = nullptr;
    uint64_t nrows = 0;
    uint64_t begin, end;
    uint32_t cur = 0;    // light class: buffer of the current item
    bool ready = false;  // light class: the current item's rows were issued with the previous item
    const Span sp = launch_span<false>(a, FUSED);
    while (next_chunk(sp, begin, end)) {
        for (uint64_t item = sp.base + begin; item < sp.base + end; ++item) {
            if (item >= t_hi || item < t_lo) {
                t = find_slot(a.item0, sp.nt + 1, item);
                t_lo = __ldg(a.item0 + t);
                t_hi = __ldg(a.item0 + t + 1);
                const TaskRef& ref = a.refs[t];
                in = ref.in;
                nrows = ref.nrows;
                __syncwarp();
                load_desc(d, a.nodes + ref.node);
            }
            const uint64_t row0 = (item - t_lo) * a.rows_per_item;
            const uint32_t nr = (uint32_t)umin64(a.rows_per_item, nrows - row0);
            const uint32_t k = d.kind == STEP_EXT ? d.e.k : d.r.k;
            uint32_t* rows = ws.rows;
            if (FUSED) {
                __syncwarp();
                stage_rows(rows, in, row0, nr, k);
            } else {
                rows = cur ? ws.rows2 : ws.rows;
                if (!ready) {
                    __syncwarp();
                    stage_rows_async(rows, in, row0, nr, k);
                }
                // the next item of the same task and chunk: its rows are copied in meanwhile
                ready = item + 1 < sp.base + end && item + 1 < t_hi;
                if (ready) {
                    const uint64_t r1 = row0 + a.rows_per_item;
                    stage_rows_async(cur ? ws.rows : ws.rows2, in, r1, (uint32_t)umin64(a.rows_per_item, nrows - r1), k);
                    cp_async_wait_one();
                } else {
                    cp_async_wait_all();
                }
                __syncwarp();
                cur ^= 1;
            }
            uint64_t c;
            if (FUSED)
                c = ext_item<false, true>(d, rows, nr, a.hub, a.ctx, nullptr, ws.gen, a.read_words);
            else if (d.kind == STEP_EXT)
                c = ext_item<false, false>(d, rows, nr, a.hub, a.ctx, nullptr, nullptr, a.read_words);
            else
                c = red_item<false>(d, rows, nr, a.ctx, nullptr);
            if (lane == 0) a.items[item] = c;
            __syncwarp();  // every lane done with these rows before the buffer is refilled
        }
    }
}

// --------------------------------------------------------- item scans ----
// Exclusive scan of per-item counts in chunks of kScanChunk (in place);
// chunks[c] receives chunk c's sum.  A block per chunk, the grid striding
// over the chunks (n from the round's device state when `dyn` is given).
__global__ void __launch_bounds__(1024) scan_items_local_kernel(uint64_t* __restrict__ v, uint64_t n,
                                                               uint64_t* __restrict__ chunks, const RunState* dyn) {
    __shared__ uint64_t ws[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (dyn) n = dyn->ni;
    for (uint64_t c = blockIdx.x; c * kScanChunk < n; c += gridDim.x) {
    const uint64_t base = c * kScanChunk + (uint64_t)threadIdx.x * 4;
    uint64_t x[4];
    uint64_t sum = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        x[i] = base + i < n ? v[base + i] : 0;
        sum += x[i];
    }
    uint64_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) ws[wid] = inc;
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
    uint64_t run = (wid > 0 ? ws[wid - 1] : 0) + inc - sum;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (base + i < n) v[base + i] = run;
        run += x[i];
    }
    if (threadIdx.x == 1023) chunks[c] = ws[31];
    __syncthreads();  // ws read by every thread before the next chunk rewrites it
    }
}

// Exclusive scan of the chunk sums (chunks[nc] = grand total), then each
// task's output rows: totals[t] = offset(item0[t + 1]) - offset(item0[t]).
__global__ void __launch_bounds__(1024) scan_items_top_kernel(uint64_t* __restrict__ chunks, uint64_t nc,
                                                             const uint64_t* __restrict__ v, uint64_t n,
                                                             const uint64_t* __restrict__ item0, uint32_t nt,
                                                             uint64_t* __restrict__ totals, const RunState* dyn) {
    __shared__ uint64_t ws[32];
    if (dyn) {
        n = dyn->ni;
        nc = (n + kScanChunk - 1) / kScanChunk;
        nt = dyn->nt;
    }
    __shared__ uint64_t carry_s;
    if (threadIdx.x == 0) carry_s = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint64_t b = 0; b < nc; b += 1024) {
        const uint64_t i = b + threadIdx.x;
        const uint64_t x = i < nc ? chunks[i] : 0;
        uint64_t inc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) ws[wid] = inc;
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
        if (i < nc) chunks[i] = carry + (wid > 0 ? ws[wid - 1] : 0) + inc - x;
        __syncthreads();
        if (threadIdx.x == 0) carry_s = carry + ws[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) chunks[nc] = carry_s;
    __syncthreads();
    const uint64_t grand = carry_s;
    auto off = [&](uint64_t i) -> uint64_t { return i >= n ? grand : v[i] + chunks[i >> kScanChunkLog2]; };
    for (uint32_t t = threadIdx.x; t < nt; t += 1024) totals[t] = off(item0[t + 1]) - off(item0[t]);
}

// ---------------------------------------------------------- write pass ----
// Persistent, over the items of the tasks that write this round (one
// instance per task class): each item's output rows go to its task's buffer
// at the item's scanned offset, in the order the count pass counted them.
// Items without output are skipped.
template <bool FUSED>
__global__ void __launch_bounds__(kRoundWarps * 32, FUSED ? 4 : 5)
round_write_kernel(RoundArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const WarpSmem ws = warp_smem<true, FUSED>(smem_raw, a);
    TaskDesc& d = *ws.d;
    uint64_t w_lo = 0, w_hi = 0;
    uint32_t t = 0;
    uint64_t t_item0 = 0, t_off0 = 0;
    uint32_t* out = nullptr;
    const uint32_t* in = nullptr;
    uint64_t nrows = 0;
    uint64_t begin, end;
    uint32_t cur = 0;    // light class: buffer of the current item
    bool ready = false;  // light class: the current item's rows were issued with the previous item
    const Span sp = launch_span<true>(a, FUSED);
    while (next_chunk(sp, begin, end)) {
        for (uint64_t wi = sp.base + begin; wi < sp.base + end; ++wi) {
            if (wi >= w_hi || wi < w_lo) {
                const uint32_t slot = find_slot(a.witem0, sp.nt + 1, wi);
                w_lo = __ldg(a.witem0 + slot);
                w_hi = __ldg(a.witem0 + slot + 1);
                t = __ldg(a.wtask + slot);
                t_item0 = __ldg(a.item0 + t);
                const TaskRef& ref = a.refs[t];
                in = ref.in;
                nrows = ref.nrows;
                out = a.task_out[t];
                __syncwarp();
                load_desc(d, a.nodes + ref.node);
                t_off0 = a.items[t_item0] + a.chunks[t_item0 >> kScanChunkLog2];
            }
            const uint64_t item = t_item0 + (wi - w_lo);
            const uint64_t off = a.items[item] + a.chunks[item >> kScanChunkLog2];
            const uint64_t off_next = item + 1 >= sp.n_count_items
                                          ? a.chunks[sp.n_chunks]
                                          : a.items[item + 1] + a.chunks[(item + 1) >> kScanChunkLog2];
            const uint64_t row0 = (wi - w_lo) * a.rows_per_item;
            const uint32_t nr = (uint32_t)umin64(a.rows_per_item, nrows - row0);
            const bool ext = d.kind == STEP_EXT;
            const uint32_t k = ext ? d.e.k : d.r.k;
            if (off_next == off) {  // nothing accepted in this item
                if (!FUSED && ready) {  // its rows were issued already: let them land before the buffer is reused
                    cp_async_wait_all();
                    __syncwarp();
                    ready = false;
                }
                continue;
            }
            uint32_t* rows = ws.rows;
            if (FUSED) {
                __syncwarp();
                stage_rows(rows, in, row0, nr, k);
            } else {
                rows = cur ? ws.rows2 : ws.rows;
                if (!ready) {
                    __syncwarp();
                    stage_rows_async(rows, in, row0, nr, k);
                }
                ready = wi + 1 < sp.base + end && wi + 1 < w_hi;
                if (ready) {
                    const uint64_t r1 = row0 + a.rows_per_item;
                    stage_rows_async(cur ? ws.rows : ws.rows2, in, r1, (uint32_t)umin64(a.rows_per_item, nrows - r1), k);
                    cp_async_wait_one();
                } else {
                    cp_async_wait_all();
                }
                __syncwarp();
                cur ^= 1;
            }
            Tile tl;
            tile_init(tl, ws.tile, rows, k, ext, out + (off - t_off0) * (ext ? k + 1 : k), off_next - off);
            if (FUSED)
                ext_item<true, true>(d, rows, nr, a.hub, a.ctx, &tl, ws.gen, nullptr);
            else if (ext)
                ext_item<true, false>(d, rows, nr, a.hub, a.ctx, &tl, nullptr, nullptr);
            else
                red_item<true>(d, rows, nr, a.ctx, &tl);
            if (tl.n) tile_flush(tl, tl.n);
            __syncwarp();  // every lane done with these rows before the buffer is refilled
        }
    }
}

// ------------------------------------------------- device-side planning ----
// Rounds scheduled on the device (BatchSession::run_device).  Every task of
// a round sits at the same trie depth (nothing is deferred or split), so a
// round's tasks are the children of the previous round's writing tasks.
// Per node: the children that can match, light class first, as a range of
// the children array, and the words of one output row.
struct NodeRun {
    uint32_t child0;
    uint16_t n_light, n_fused;
    uint32_t out_w;  // EXT: width + 1; REDUCE: width
    uint32_t pad;
};

struct PlanArgs {
    RunState* st;              // this round
    RunState* nx;              // the next round
    const TaskRef* refs;       // this round's tasks (light class first)
    const uint64_t* item0;     // [nt + 1] this round's count-pass item prefix
    const uint64_t* totals;    // [nt] output rows per task
    const NodeRun* info;
    const uint32_t* children;
    uint64_t* node_total;      // output rows per node (zeroed before the run)
    uint32_t* region;          // this round's output frontier region
    uint64_t region_words;
    uint32_t** outs;           // [nt] output base per task (null: not written)
    uint32_t* wtask;           // [nw] count-task index of each writing task
    uint64_t* witem0;          // [nw + 1] item prefix over the writing tasks
    TaskRef* next_refs;        // the next round's tasks
    uint64_t* next_item0;      // [next nt + 1]
    uint32_t refs_cap;         // capacity of next_refs
    uint64_t items_cap;        // capacity of the per-item arrays
    uint32_t rows_next;        // rows per item of the next round
    uint32_t* overflow;        // set (never cleared) when a capacity is exceeded
    uint64_t* bsum;            // [(nb + 1) * kPlanVals] per-block sums, then their exclusive scan and the totals
    uint32_t nb;               // blocks of kPlanThreads tasks covering refs_cap
};

constexpr int kPlanThreads = 512;
constexpr int kPlanVals = 8;

// Task t's contributions: 0 output words (rounded up to 16 bytes), 1 writes,
// 2 write items, 3 write items of the light class, 4 / 5 light / fused child
// tasks, 6 / 7 their items.  A task writes when it has output rows and a
// child that can match.
__device__ __forceinline__ void plan_values(const PlanArgs& p, uint32_t nt_light, uint32_t t, uint64_t v[kPlanVals],
                                            uint32_t& node, uint64_t& tot, uint64_t& per) {
    node = p.refs[t].node;
    tot = p.totals[t];
    const NodeRun nr = p.info[node];
    const bool w = tot > 0 && nr.n_light + nr.n_fused > 0;
    per = w ? (tot + p.rows_next - 1) / p.rows_next : 0;
    const uint64_t items = p.item0[t + 1] - p.item0[t];
    v[0] = w ? ((tot * nr.out_w + 3) & ~3ull) : 0;
    v[1] = w ? 1 : 0;
    v[2] = w ? items : 0;
    v[3] = w && t < nt_light ? items : 0;
    v[4] = w ? nr.n_light : 0;
    v[5] = w ? nr.n_fused : 0;
    v[6] = per * nr.n_light;
    v[7] = per * nr.n_fused;
}

// Exclusive block scan of kPlanVals values per thread; sum receives the
// block totals.
__device__ __forceinline__ void plan_scan(const uint64_t v[kPlanVals], uint64_t ex[kPlanVals], uint64_t sum[kPlanVals],
                                          uint64_t (*sh)[kPlanVals]) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    constexpr int W = kPlanThreads / 32;
    uint64_t inc[kPlanVals];
#pragma unroll
    for (int k = 0; k < kPlanVals; ++k) {
        inc[k] = v[k];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, inc[k], o);
            if (lane >= o) inc[k] += y;
        }
    }
    if (lane == 31)
        for (int k = 0; k < kPlanVals; ++k) sh[wid][k] = inc[k];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < kPlanVals; ++k) {
            uint64_t w = lane < W ? sh[lane][k] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            if (lane < W) sh[lane][k] = w;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kPlanVals; ++k) {
        ex[k] = (wid > 0 ? sh[wid - 1][k] : 0) + inc[k] - v[k];
        sum[k] = sh[W - 1][k];
    }
    __syncthreads();  // sh read by every thread before the next scan rewrites it
}

// Planning of one round in three launches over blocks of kPlanThreads
// tasks: the blocks' sums (plan_sum_kernel), their exclusive scan and the
// round's totals (plan_top_kernel, one block), then every task's places
// (plan_write_kernel): each task's output rows are recorded (node_total),
// the writing tasks' outputs placed in the round's region and listed for the
// write pass, and the next round's tasks (their children, light class first)
// listed with their item prefix.  A region, task or item capacity exceeded
// marks the run overflowed: no later launch of the run finds work, and the
// host runs the session's rounds itself.
__global__ void __launch_bounds__(kPlanThreads) plan_sum_kernel(PlanArgs p) {
    __shared__ uint64_t sh[kPlanThreads / 32][kPlanVals];
    const RunState& st = *p.st;
    const uint32_t nt = st.overflow ? 0u : st.nt;
    const uint32_t t = blockIdx.x * kPlanThreads + threadIdx.x;
    uint64_t v[kPlanVals] = {}, ex[kPlanVals], sum[kPlanVals];
    uint32_t node;
    uint64_t tot, per;
    if (t < nt) plan_values(p, st.nt_light, t, v, node, tot, per);
    plan_scan(v, ex, sum, sh);
    if (threadIdx.x < kPlanVals) p.bsum[(size_t)blockIdx.x * kPlanVals + threadIdx.x] = sum[threadIdx.x];
}

__global__ void __launch_bounds__(kPlanThreads) plan_top_kernel(PlanArgs p) {
    __shared__ uint64_t sh[kPlanThreads / 32][kPlanVals];
    RunState& st = *p.st;
    RunState& nx = *p.nx;
    uint64_t v[kPlanVals], ex[kPlanVals], sum[kPlanVals], carry[kPlanVals] = {};
    for (uint32_t base = 0; base < p.nb; base += kPlanThreads) {
        const uint32_t b = base + threadIdx.x;
#pragma unroll
        for (int k = 0; k < kPlanVals; ++k) v[k] = b < p.nb ? p.bsum[(size_t)b * kPlanVals + k] : 0;
        plan_scan(v, ex, sum, sh);
        if (b < p.nb)
#pragma unroll
            for (int k = 0; k < kPlanVals; ++k) p.bsum[(size_t)b * kPlanVals + k] = carry[k] + ex[k];
#pragma unroll
        for (int k = 0; k < kPlanVals; ++k) carry[k] += sum[k];
    }
    if (threadIdx.x == 0) {
        const uint64_t* tot = carry;
        const bool bad = st.overflow || tot[0] > p.region_words || tot[4] + tot[5] > p.refs_cap ||
                         tot[6] + tot[7] > p.items_cap;
        if (bad) {
            st.overflow = 1;
            st.nw = 0;
            st.wi = st.wi_light = 0;
            nx.overflow = 1;
            nx.nt = nx.nt_light = 0;
            nx.ni = nx.ni_light = 0;
            *p.overflow = 1;
        } else {
            st.nw = (uint32_t)tot[1];
            st.wi = tot[2];
            st.wi_light = tot[3];
            nx.nt = (uint32_t)(tot[4] + tot[5]);
            nx.nt_light = (uint32_t)tot[4];
            nx.ni = tot[6] + tot[7];
            nx.ni_light = tot[6];
            p.witem0[tot[1]] = tot[2];
            p.next_item0[tot[4] + tot[5]] = tot[6] + tot[7];
        }
#pragma unroll
        for (int k = 0; k < kPlanVals; ++k) p.bsum[(size_t)p.nb * kPlanVals + k] = tot[k];
    }
}

__global__ void __launch_bounds__(kPlanThreads) plan_write_kernel(PlanArgs p) {
    __shared__ uint64_t sh[kPlanThreads / 32][kPlanVals];
    const RunState& st = *p.st;
    if (st.overflow) return;  // uniform: set before this launch
    const uint32_t nt = st.nt;
    const uint32_t t = blockIdx.x * kPlanThreads + threadIdx.x;
    uint64_t v[kPlanVals] = {}, ex[kPlanVals], sum[kPlanVals];
    uint32_t node = 0;
    uint64_t tot = 0, per = 0;
    if (t < nt) plan_values(p, st.nt_light, t, v, node, tot, per);
    plan_scan(v, ex, sum, sh);
    if (t >= nt) return;
    const uint64_t* carry = p.bsum + (size_t)blockIdx.x * kPlanVals;
    const uint64_t light_tasks = p.bsum[(size_t)p.nb * kPlanVals + 4];
    const uint64_t light_items = p.bsum[(size_t)p.nb * kPlanVals + 6];
    p.node_total[node] = tot;
    uint32_t* out = nullptr;
    if (v[1]) {
        out = p.region + carry[0] + ex[0];
        const uint64_t slot = carry[1] + ex[1];
        p.wtask[slot] = t;
        p.witem0[slot] = carry[2] + ex[2];
        const NodeRun nr = p.info[node];
        const uint64_t j0 = carry[4] + ex[4], i0 = carry[6] + ex[6];
        for (uint32_t i = 0; i < nr.n_light; ++i) {
            p.next_refs[j0 + i] = TaskRef{__ldg(p.children + nr.child0 + i), 0u, out, tot};
            p.next_item0[j0 + i] = i0 + (uint64_t)i * per;
        }
        const uint64_t j1 = light_tasks + carry[5] + ex[5], i1 = light_items + carry[7] + ex[7];
        for (uint32_t i = 0; i < nr.n_fused; ++i) {
            p.next_refs[j1 + i] = TaskRef{__ldg(p.children + nr.child0 + nr.n_light + i), 0u, out, tot};
            p.next_item0[j1 + i] = i1 + (uint64_t)i * per;
        }
    }
    p.outs[t] = out;
}

std::atomic<uint64_t> g_batch_launches{0};

}  // namespace

uint64_t batch_kernel_launches() { return g_batch_launches.load(); }

// Pinned host buffers are expensive to create (page locking), and every
// batched run and MNI call stages through them; released buffers are kept in
// a process-wide pool and handed to the next Staging that needs one.
namespace {
std::mutex g_pin_mu;
std::vector<std::pair<char*, size_t>> g_pin_free;  // (buffer, capacity)

char* pin_take(size_t need, size_t& cap) {
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        size_t best = g_pin_free.size();
        for (size_t i = 0; i < g_pin_free.size(); ++i)
            if (g_pin_free[i].second >= need && (best == g_pin_free.size() || g_pin_free[i].second < g_pin_free[best].second))
                best = i;
        if (best < g_pin_free.size()) {
            char* p = g_pin_free[best].first;
            cap = g_pin_free[best].second;
            g_pin_free.erase(g_pin_free.begin() + best);
            return p;
        }
    }
    size_t c = (size_t)1 << 20;
    while (c < need) c <<= 1;
    char* p = nullptr;
    if (cudaMallocHost((void**)&p, c) != cudaSuccess) return nullptr;
    cap = c;
    return p;
}

void pin_give(char* p, size_t cap) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pin_free.push_back({p, cap});
}
}  // namespace

char* Staging::get(size_t need) {
    if (need > cap || !p) {
        pin_give(p, cap);
        p = pin_take(std::max(need, cap * 2), cap);
        if (!p) cap = 0;
    }
    return p;
}
Staging::~Staging() { pin_give(p, cap); }

// ---------------------------------------------------------------------------
// BatchSession: the persistent form of the batched engine.  Plans are
// submitted in waves (plans of one wave share their common step prefixes);
// every round() advances all active tasks by one step; a plan completes when
// no task on its path is left.  run_batch() is one wave run to completion;
// the serving loop submits new waves between rounds.
// Host containers of ended sessions, kept per thread for the next session:
// a batched run's trie and plan records are rebuilt on every call, and fresh
// vectors would pay a page fault per page on first touch.
namespace {
struct SessionSpare {
    std::vector<BatchSession::BNode> nodes;
    std::vector<const Step*> node_steps;
    std::vector<BatchSession::PlanRec> plans;
    std::vector<unsigned char> desc_host;
};
thread_local SessionSpare t_spare;
}  // namespace

BatchSession::BatchSession(DevDB& db_, cudaStream_t s_, uint64_t budget_, uint32_t slots_, bool graph_counts_,
                           bool profile_)
    : db(db_), s(s_), budget(budget_), nslots(slots_), want_graph_counts(graph_counts_), profile(profile_) {
    tune.rows_per_item = db.tune_rows_per_item;
    tune.hub = db.tune_hub;
    nodes.swap(t_spare.nodes);
    node_steps.swap(t_spare.node_steps);
    plans.swap(t_spare.plans);
    desc_host.swap(t_spare.desc_host);
    nodes.clear();
    node_steps.clear();
    plans.clear();
}

BatchSession::~BatchSession() {
    auto keep = [](auto& mine, auto& spare) {
        if (mine.capacity() > spare.capacity()) {
            mine.clear();
            mine.swap(spare);
        }
    };
    keep(nodes, t_spare.nodes);
    keep(node_steps, t_spare.node_steps);
    keep(plans, t_spare.plans);
    if (!waves.empty()) {  // thousands of small step vectors: freed off this thread
        auto w = std::make_shared<std::vector<std::vector<std::vector<Step>>>>(std::move(waves));
        defer([w]() mutable { w.reset(); });
    }
    if (desc_host.capacity() > t_spare.desc_host.capacity()) desc_host.swap(t_spare.desc_host);
    cudaSetDevice(db.device);
    active.clear();
    if (staged) cudaEventDestroy(staged);
    for (void* p : {(void*)d_desc, (void*)d_items, (void*)d_small, (void*)d_chunks, (void*)d_read, acc, d_nodes})
        if (p) cudaFreeAsync(p, s);
    cudaStreamSynchronize(s);
    pin_give(desc_pin, desc_pin_cap);  // the stream drained: no copy reads it any more
    if (desc_ev) cudaEventDestroy(desc_ev);
}

int BatchSession::init() {
    GVA_CUDA_B(cudaSetDevice(db.device));
    GVA_CUDA_B(cudaEventCreateWithFlags(&desc_ev, cudaEventDisableTiming));
    inited = true;
    if (budget == 0) {
        if (db.default_budget == 0) {
            size_t fr = 0, tot = 0;
            GVA_CUDA_B(cudaMemGetInfo(&fr, &tot));
            db.default_budget = (uint64_t)fr / 4 * 3;
        }
        budget = db.default_budget;
    }
    per_graph = nslots > 0;
    if (per_graph) {
        if (!db.vgraph || db.num_graphs == 0)
            return fail(GVA_ERR_ARG, "per-graph results need the database's graph ids (gva_db_set_graphs)");
        ctx_words = (db.num_graphs + 31) / 32;
        const size_t bytes = (want_graph_counts ? (size_t)nslots * db.num_graphs * 8 : 0) + (size_t)nslots * ctx_words * 4;
        acc_bytes = bytes;
        if (cudaMallocAsync(&acc, bytes, s) != cudaSuccess) return fail(GVA_ERR_NOMEM, "per-graph counters");
        GVA_CUDA_B(cudaMemsetAsync(acc, 0, bytes, s));
        for (uint32_t i = nslots; i > 0; --i) free_slots.push_back((int)i - 1);
    }
    int dev = db.device;
    static std::atomic<bool> smem_set[64];  // sessions may start on several threads (server, miner)
    if (dev < 0 || dev >= 64) return fail(GVA_ERR_ARG, "device index out of range");
    if (!smem_set[dev].load(std::memory_order_acquire)) {
        const int most = (int)std::max(round_smem_bytes(kMaxItemRows / 4, kMaxCols, true, true),
                                       round_smem_bytes(kMaxItemRows / 4, kMaxCols, true, false));  // rows per item shrink as rows widen
        GVA_CUDA_B(cudaFuncSetAttribute(round_count_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
        GVA_CUDA_B(cudaFuncSetAttribute(round_count_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
        GVA_CUDA_B(cudaFuncSetAttribute(round_write_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
        GVA_CUDA_B(cudaFuncSetAttribute(round_write_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
        smem_set[dev].store(true, std::memory_order_release);
    }
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return GVA_OK;
}

uint64_t* BatchSession::graph_counts_dev() const { return want_graph_counts ? (uint64_t*)acc : nullptr; }
uint32_t* BatchSession::graph_bits_dev() const {
    return per_graph ? (uint32_t*)((char*)acc + (want_graph_counts ? (size_t)nslots * db.num_graphs * 8 : 0)) : nullptr;
}

// Plan completion: a node closes when its parent is closed and no task is
// left at it (tasks only move down the trie, so none can arrive later);
// closing a node completes the plans that end there and tries its children.
void BatchSession::add_task(int node, const uint32_t* in, uint64_t rows, std::shared_ptr<void> owner) {
    nodes[node].at++;
    active.push_back({node, in, rows, std::move(owner)});
}

void BatchSession::try_close(int n) {
    BNode& nd = nodes[n];
    if (nd.closed || nd.at != 0 || (nd.parent >= 0 && !nodes[nd.parent].closed)) return;
    nd.closed = true;
    for (int q = nd.first_term; q >= 0; q = plans[q].next_term) {
        plans[q].done = true;
        completed.push_back(q);
    }
    for (int c = nd.first_child; c >= 0; c = nodes[c].next_sibling) try_close(c);
}

void BatchSession::finish_task(int node) {
    nodes[node].at--;
    try_close(node);
}

// Serialised step parameters (everything that decides a step's output from
// its input) into buf; returns the length.
size_t step_key_bytes(const Step& st, uint8_t* buf) {
    size_t n = 0;
    auto put = [&](const void* p, size_t k) {
        memcpy(buf + n, p, k);
        n += k;
    };
    put(&st.kind, sizeof st.kind);
    put(&st.width_in, 4);
    put(&st.part, 4);
    put(&st.label, 4);
    put(&st.always_empty, 4);
    if (st.kind == STEP_EXT) {
        put(&st.src_col, 4);
        put(&st.bound_col, 4);
        put(&st.bound_inclusive, 4);
        put(&st.n_eq, 4);
        put(st.eq_cols, st.n_eq);
        put(&st.n_chk, 4);
        put(st.chk_col, st.n_chk);
        put(st.chk_dir, st.n_chk);
        put(st.chk_part, 4 * st.n_chk);
        put(st.chk_lab, 4 * st.n_chk);
    } else if (st.kind == STEP_REDUCE) {
        put(&st.n_pairs, 4);
        put(st.rs_col, st.n_pairs);
        put(st.re_col, st.n_pairs);
        put(st.re_label, 4 * st.n_pairs);
    }
    return n;
}

// A 64-bit hash of the same fields as step_key_bytes, taken from the step
// directly (no serialisation): steps with equal key bytes hash equal.  Never 0.
uint64_t step_key_hash(const Step& st) {
    uint64_t h = 0x243f6a8885a308d3ull;
    auto mix = [&](uint64_t w) {
        h = (h ^ w) * 0x9e3779b97f4a7c15ull;
        h ^= h >> 29;
    };
    // the first n of a byte array, 8 at a time, bytes past n masked off
    auto bytes = [&](const uint8_t* a, uint32_t n) {
        for (uint32_t j = 0; j < n; j += 8) {
            uint64_t w = 0;
            memcpy(&w, a + j, n - j < 8 ? n - j : 8);
            mix(w);
        }
    };
    mix((uint64_t)st.kind | (uint64_t)st.width_in << 32);
    mix((uint64_t)st.part | (uint64_t)st.label << 32);
    mix(st.always_empty);
    if (st.kind == STEP_EXT) {
        mix((uint64_t)(uint32_t)st.src_col | (uint64_t)(uint32_t)st.bound_col << 32);
        mix((uint64_t)st.bound_inclusive | (uint64_t)st.n_eq << 32);
        bytes(st.eq_cols, st.n_eq);
        mix(st.n_chk);
        for (uint32_t i = 0; i < st.n_chk; ++i) {
            mix((uint64_t)st.chk_col[i] | (uint64_t)st.chk_dir[i] << 8);
            mix((uint64_t)st.chk_part[i] | (uint64_t)st.chk_lab[i] << 32);
        }
    } else if (st.kind == STEP_REDUCE) {
        mix(st.n_pairs);
        for (uint32_t i = 0; i < st.n_pairs; ++i)
            mix((uint64_t)st.rs_col[i] | (uint64_t)st.re_col[i] << 8 | (uint64_t)st.re_label[i] << 32);
    }
    return h | 1;
}

void BatchSession::fill_node_desc(int id, void* out) const {
    const BNode& nd = nodes[id];
    TaskDesc& d = *reinterpret_cast<TaskDesc*>(out);
    memset(&d, 0, sizeof d);
    const Step& st = *node_steps[id];
    d.kind = st.kind;
    d.mode = nd.first_child < 0 ? MODE_COUNT : MODE_WRITE;
    if (per_graph && nd.first_term >= 0) {
        d.mode = nd.first_child < 0 ? MODE_COUNT_GRAPHS : MODE_WRITE_AND_GRAPHS;
        d.query = (uint32_t)plans[nd.first_term].slot;
    }
    if (st.kind == STEP_SEED || st.always_empty || st.part == 0 || st.part > db.parts.size()) return;
    const DevPart& P = db.parts[st.part - 1];
    if (st.kind == STEP_EXT) {
        ExtArgs& a = d.e;
        a.off = P.off;
        a.adj = P.adj;
        a.k = st.width_in;
        a.L = db.kernel_L();
        a.lab = st.label;
        a.src_col = st.src_col;
        a.bound_col = st.bound_col;
        a.bound_incl = st.bound_inclusive;
        a.n_eq = st.n_eq;
        for (uint32_t i = 0; i < st.n_eq; ++i) a.eq_cols[i] = st.eq_cols[i];
        a.n_chk = st.n_chk;
        for (uint32_t i = 0; i < st.n_chk; ++i) {
            a.chk_col[i] = st.chk_col[i];
            a.chk_dir[i] = st.chk_dir[i];
            a.chk_lab[i] = st.chk_lab[i];
            if (st.chk_part[i] == 0 || st.chk_part[i] > db.parts.size()) continue;  // lowering marks such steps empty
            a.chk_off[i] = db.parts[st.chk_part[i] - 1].off;
            a.chk_adj[i] = db.parts[st.chk_part[i] - 1].adj;
        }
    } else {
        RedArgs& a = d.r;
        a.off = P.off;
        a.adj = P.adj;
        a.k = st.width_in;
        a.L = db.kernel_L();
        a.n_pairs = st.n_pairs;
        for (uint32_t i = 0; i < st.n_pairs; ++i) {
            a.rs[i] = st.rs_col[i];
            a.re[i] = st.re_col[i];
            a.rl[i] = st.re_label[i];
        }
    }
}

int BatchSession::submit(std::vector<std::vector<Step>>&& wave, const std::vector<uint64_t>& tags,
                         std::vector<int>* ids, bool presorted) {
    waves.push_back(std::move(wave));
    const std::vector<std::vector<Step>>& steps = waves.back();
    const auto t_start = std::chrono::steady_clock::now();
    struct Timer {
        std::chrono::steady_clock::time_point t0;
        double& acc;
        ~Timer() { acc += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); }
    } timer{t_start, submit_ms};
    // trie of this wave: (parent, step bytes) -> node, looked up by a 64-bit
    // hash and confirmed by comparing the bytes.  A presorted wave (plans in
    // order of their step keys, so plans that share a prefix are adjacent)
    // is matched against the previous plan only and keeps no index; a step
    // that only a non-adjacent plan shares gets a node of its own, which
    // costs sharing, not correctness.
    // open addressing over (hash, node) slots; each new node's key bytes are
    // kept in one arena so that a probe compares bytes without serialising
    // the candidate node's step again
    struct Slot {
        uint64_t h;
        int id;
        uint32_t key_at;
    };
    std::vector<Slot> index;
    std::vector<uint8_t> key_arena;
    size_t index_mask = 0;
    if (!presorted) {
        size_t total = 0;
        for (const auto& st : steps) total += st.size();
        size_t cap = 64;
        while (cap < 2 * total) cap <<= 1;
        index.assign(cap, Slot{0, -1, 0});
        index_mask = cap - 1;
        key_arena.reserve(total * 64);
    }
    const int first_node = (int)nodes.size();
    uint8_t kb[512], kb2[512];
    {  // room for the wave (a plan mostly adds a node or two past its shared
       // prefix), growing geometrically: a session may take many waves
        size_t total = 0;
        for (const auto& st : steps) total += st.size();
        const size_t guess = std::min(total, 2 * steps.size() + 64);
        auto room = [](auto& v, size_t more) {
            if (v.capacity() < v.size() + more) v.reserve(std::max(v.size() + more, 2 * v.capacity()));
        };
        room(nodes, guess);
        room(node_steps, guess);
        room(plans, steps.size());
    }
    // a new node for step `st` at `depth` under `parent` (-1: a root)
    auto new_node = [&](const Step& st, int parent, int depth) {
        const int id = (int)nodes.size();
        BNode nd;
        nd.kind = st.kind;
        nd.width_in = st.width_in;
        nd.n_eq = st.n_eq;
        nd.n_pairs = st.n_pairs;
        nd.always_empty = st.always_empty;
        nd.fused = fused_class(st.kind, st.n_chk) ? 1u : 0u;
        nd.depth = depth;
        node_steps.push_back(&st);
        nd.parent = parent;
        if (parent >= 0) {
            nd.next_sibling = nodes[parent].first_child;
            nodes.push_back(nd);
            nodes[parent].first_child = id;
        } else {
            nodes.push_back(nd);
        }
        return id;
    };
    // a presorted wave of many plans: cut into chunks at changes of the first
    // two steps and built on the host's cores (only seed nodes, which cost
    // nothing on the device, can repeat across chunks)
    const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (presorted && steps.size() >= 4096 && hw > 1) {
        const size_t np = steps.size();
        for (const auto& st : steps)
            if (st.size() < 2 || st[0].kind != STEP_SEED) return fail(GVA_ERR_ARG, "plan must start with a seed step");
        if (per_graph && free_slots.size() < np) return fail(GVA_ERR_NOMEM, "no free per-graph result slot");
        const int q0 = (int)plans.size();
        for (size_t qi = 0; qi < np; ++qi) {
            PlanRec pr;
            pr.tag = qi < tags.size() ? tags[qi] : qi;
            if (per_graph) {
                pr.slot = free_slots.back();
                free_slots.pop_back();
            }
            plans.push_back(pr);
            if (ids) ids->push_back(q0 + (int)qi);
        }
        // seed nodes first, on this thread (presorted: equal seed steps are adjacent)
        std::vector<int> root_of(np);
        {
            uint8_t ka[512], kc[512];
            int root = -1;
            for (size_t qi = 0; qi < np; ++qi) {
                const Step& s0 = steps[qi][0];
                bool same = false;
                if (qi > 0) {
                    const Step& p0 = steps[qi - 1][0];
                    same = memcmp(&s0, &p0, sizeof(Step)) == 0;
                    if (!same) {
                        const size_t n = step_key_bytes(s0, ka);
                        same = step_key_bytes(p0, kc) == n && memcmp(ka, kc, n) == 0;
                    }
                }
                if (!same) {
                    root = (int)nodes.size();
                    BNode nd;
                    nd.kind = s0.kind;
                    nd.width_in = s0.width_in;
                    nd.always_empty = s0.always_empty;
                    nd.depth = 0;
                    nodes.push_back(nd);
                    node_steps.push_back(&s0);
                }
                root_of[qi] = root;
            }
        }
        const int first_chunk_node = (int)nodes.size();
        // chunks cut where the first two steps change, so that no node below
        // a seed node is split across chunks
        const unsigned T = std::max(1u, std::min<unsigned>(hw, (unsigned)(np / 1024)));
        auto same01 = [&](size_t a, size_t b) {
            return root_of[a] == root_of[b] && memcmp(&steps[a][1], &steps[b][1], sizeof(Step)) == 0;
        };
        std::vector<size_t> cut(T + 1, np);
        cut[0] = 0;
        for (unsigned t = 1; t < T; ++t) {
            size_t c = std::max(np * t / T, cut[t - 1]);
            while (c < np && c > cut[t - 1] && same01(c - 1, c)) ++c;
            cut[t] = c;
        }
        // a chunk's nodes use local ids >= 0; a seed node is -2 - its id
        struct Local {
            std::vector<BNode> nodes;
            std::vector<const Step*> steps;
            std::vector<int> term;                       // terminal (local id) of each plan of the chunk
            std::vector<std::pair<int, int>> root_list;  // (seed node, first local child) in order seen
        };
        std::vector<Local> loc(T);
        auto build = [&](unsigned t) {
            Local& L = loc[t];
            const size_t a0 = cut[t], a1 = cut[t + 1];
            L.nodes.reserve(2 * (a1 - a0) + 16);
            L.steps.reserve(2 * (a1 - a0) + 16);
            L.term.resize(a1 - a0);
            uint8_t ka[512], kc[512];
            const std::vector<Step>* prv = nullptr;
            std::vector<int> pp, cp;
            for (size_t qi = a0; qi < a1; ++qi) {
                const std::vector<Step>& st = steps[qi];
                if (cp.size() < st.size()) cp.resize(st.size());
                int cur = -2 - root_of[qi];
                cp[0] = cur;
                for (size_t i = 1; i < st.size(); ++i) {
                    const bool up = prv && i < pp.size() && i < prv->size() && cur == pp[i - 1];
                    int id = -1;
                    if (up && memcmp(&st[i], &(*prv)[i], sizeof(Step)) == 0) {
                        id = pp[i];
                    } else if (up) {
                        const size_t n = step_key_bytes(st[i], ka);
                        if (step_key_bytes((*prv)[i], kc) == n && memcmp(ka, kc, n) == 0) id = pp[i];
                    }
                    if (id < 0) {
                        id = (int)L.nodes.size();
                        BNode nd;
                        nd.kind = st[i].kind;
                        nd.width_in = st[i].width_in;
                        nd.n_eq = st[i].n_eq;
                        nd.n_pairs = st[i].n_pairs;
                        nd.always_empty = st[i].always_empty;
                        nd.fused = fused_class(st[i].kind, st[i].n_chk) ? 1u : 0u;
                        nd.depth = (int)i;
                        nd.parent = cur;
                        if (cur >= 0) {
                            nd.next_sibling = L.nodes[cur].first_child;
                            L.nodes[cur].first_child = id;
                        } else {  // child of a seed node: chained per seed node, spliced in on merge
                            const int r = -2 - cur;
                            if (L.root_list.empty() || L.root_list.back().first != r) L.root_list.push_back({r, -1});
                            nd.next_sibling = L.root_list.back().second;
                            L.root_list.back().second = id;
                        }
                        L.nodes.push_back(nd);
                        L.steps.push_back(&st[i]);
                    }
                    cur = id;
                    cp[i] = cur;
                }
                prv = &st;
                pp.assign(cp.begin(), cp.begin() + st.size());
                const int q = q0 + (int)qi;
                L.term[qi - a0] = cur;
                plans[q].next_term = L.nodes[cur].first_term;
                L.nodes[cur].first_term = q;
            }
        };
        pool_run(T, build);
        std::vector<size_t> off(T + 1, (size_t)first_chunk_node);
        for (unsigned t = 0; t < T; ++t) off[t + 1] = off[t] + loc[t].nodes.size();
        nodes.resize(off[T]);
        node_steps.resize(off[T]);
        auto place = [&](unsigned t) {
            const int o = (int)off[t];
            Local& L = loc[t];
            for (size_t j = 0; j < L.nodes.size(); ++j) {
                BNode nd = L.nodes[j];
                nd.parent = nd.parent >= 0 ? nd.parent + o : -2 - nd.parent;
                if (nd.first_child >= 0) nd.first_child += o;
                if (nd.next_sibling >= 0) nd.next_sibling += o;
                nodes[off[t] + j] = nd;
                node_steps[off[t] + j] = L.steps[j];
            }
            for (size_t qi = cut[t]; qi < cut[t + 1]; ++qi) plans[q0 + (int)qi].terminal = L.term[qi - cut[t]] + o;
        };
        pool_run(T, place);
        // children of seed nodes: each chunk's chain joins its seed node's list
        for (unsigned t = 0; t < T; ++t)
            for (const auto& rl : loc[t].root_list) {
                if (rl.second < 0) continue;
                int last = rl.second + (int)off[t];
                while (nodes[last].next_sibling >= 0) last = nodes[last].next_sibling;
                nodes[last].next_sibling = nodes[rl.first].first_child;
                nodes[rl.first].first_child = rl.second + (int)off[t];
            }
    } else {
    const std::vector<Step>* prev = nullptr;
    std::vector<int> prev_path, path;
    for (size_t qi = 0; qi < steps.size(); ++qi) {
        const std::vector<Step>& st = steps[qi];
        if (st.size() < 2 || st[0].kind != STEP_SEED) return fail(GVA_ERR_ARG, "plan must start with a seed step");
        if (path.size() < st.size()) path.resize(st.size());
        PlanRec pr;
        pr.tag = qi < tags.size() ? tags[qi] : qi;
        if (per_graph) {
            if (free_slots.empty()) return fail(GVA_ERR_NOMEM, "no free per-graph result slot");
            pr.slot = free_slots.back();
            free_slots.pop_back();
        }
        const int q = (int)plans.size();
        plans.push_back(pr);
        if (ids) ids->push_back(q);
        int cur = -1;
        for (size_t i = 0; i < st.size(); ++i) {
            // fast path: plans usually arrive ordered by their step sequences, so
            // a step equal to the previous plan's step under the same parent is
            // that plan's node (byte-equal steps have equal keys)
            const bool under_prev = prev && i < prev_path.size() && i < prev->size() && cur == (i ? prev_path[i - 1] : -1);
            if (under_prev && memcmp(&st[i], &(*prev)[i], sizeof(Step)) == 0) {
                cur = prev_path[i];
                path[i] = cur;
                continue;
            }
            const size_t n = step_key_bytes(st[i], kb);
            if (presorted) {
                int id = -1;
                if (under_prev && step_key_bytes((*prev)[i], kb2) == n && memcmp(kb, kb2, n) == 0) id = prev_path[i];
                if (id < 0) id = new_node(st[i], cur, (int)i);
                cur = id;
                path[i] = cur;
                continue;
            }
            uint64_t h = 1469598103934665603ull ^ ((uint64_t)(int64_t)cur * 0x9e3779b97f4a7c15ull);
            for (size_t j = 0; j + 8 <= n; j += 8) {
                uint64_t w;
                memcpy(&w, kb + j, 8);
                h = (h ^ w) * 1099511628211ull;
            }
            for (size_t j = n & ~(size_t)7; j < n; ++j) h = (h ^ kb[j]) * 1099511628211ull;
            h ^= h >> 29;
            int id = -1;
            size_t at = (size_t)h & index_mask;
            for (; index[at].id >= 0; at = (at + 1) & index_mask) {
                const Slot& sl = index[at];
                if (sl.h != h || nodes[sl.id].parent != cur) continue;
                if (key_arena[sl.key_at] == n && memcmp(key_arena.data() + sl.key_at + 1, kb, n) == 0) {
                    id = sl.id;
                    break;
                }
            }
            if (id < 0) {  // `at` is the free slot that ended the probe
                id = new_node(st[i], cur, (int)i);
                index[at] = Slot{h, id, (uint32_t)key_arena.size()};
                key_arena.push_back((uint8_t)n);
                key_arena.insert(key_arena.end(), kb, kb + n);
            }
            cur = id;
            path[i] = cur;
        }
        prev = &st;
        prev_path.assign(path.begin(), path.begin() + st.size());
        plans[q].terminal = cur;
        plans[q].next_term = nodes[cur].first_term;
        nodes[cur].first_term = q;
    }
    }
    // the new nodes' descriptors, on the host's cores, into the staging that
    // the next round (or device-scheduled run) ships; only descriptors not
    // yet shipped are kept.  An initialised session stages them in pinned
    // memory (an asynchronous copy), one never initialised in host memory
    // (tries built without a device make no device call).
    {
        const size_t nn = nodes.size();
        const size_t sz = sizeof(TaskDesc);
        unsigned char* dst = nullptr;
        if (inited) {
            if (desc_pending) {  // the last shipment still reads the buffer
                GVA_CUDA_B(cudaEventSynchronize(desc_ev));
                desc_pending = false;
            }
            const size_t need = (nn - shipped) * sz;
            if (need > desc_pin_cap) {
                size_t cap = 0;
                char* p = pin_take(std::max(need, 2 * desc_pin_cap), cap);
                if (!p) return fail(GVA_ERR_NOMEM, "pinned staging allocation failed");
                if (desc_pin && first_node > (int)shipped) memcpy(p, desc_pin, (first_node - shipped) * sz);
                pin_give(desc_pin, desc_pin_cap);
                desc_pin = p;
                desc_pin_cap = cap;
            }
            dst = reinterpret_cast<unsigned char*>(desc_pin);
        } else {
            if (desc_host.size() < (nn - shipped) * sz) desc_host.resize((nn - shipped) * sz);
            dst = desc_host.data();
        }
        const size_t nnew = nn - (size_t)first_node;
        const unsigned T = nnew >= 8192 ? hw : 1u;
        auto fill = [&](unsigned t) {
            for (size_t id = (size_t)first_node + t; id < nn; id += T) fill_node_desc((int)id, dst + (id - shipped) * sz);
        };
        pool_run(T, fill);
    }
    start_seeds(first_node);
    return GVA_OK;
}

// seeds: the children of every seed node from first_node on start from its
// vertex list
void BatchSession::start_seeds(int first_node) {
    for (int id = first_node; id < (int)nodes.size(); ++id) {
        if (nodes[id].parent != -1) continue;
        const Step& sd = *node_steps[id];
        uint64_t n = 0;
        if (!sd.always_empty) n = db.seed_off[sd.label + 1] - db.seed_off[sd.label];
        if (n)
            for (int c = nodes[id].first_child; c >= 0; c = nodes[c].next_sibling)
                add_task(c, db.seed_verts + db.seed_off[sd.label], n, nullptr);
        try_close(id);
    }
}

int BatchSession::round() {
    const auto t_start = std::chrono::steady_clock::now();
    double wait_before = wait_ms;
    struct Timer {
        std::chrono::steady_clock::time_point t0;
        double& acc;
        double& wait;
        double wait0;
        ~Timer() {
            acc += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() -
                   (wait - wait0);
        }
    } timer{t_start, round_host_ms, wait_ms, wait_before};
    auto t_lap = t_start;
    auto lap = [&](int k) {
        const auto now = std::chrono::steady_clock::now();
        phase_ms[k] += std::chrono::duration<double, std::milli>(now - t_lap).count();
        t_lap = now;
    };
    GVA_CUDA_B(cudaSetDevice(db.device));
    // steps that cannot match (label or partition absent) end their task
    {
        size_t w = 0;
        std::vector<int> gone;
        for (size_t i = 0; i < active.size(); ++i) {
            if (nodes[active[i].node].always_empty)
                gone.push_back(active[i].node);
            else
                active[w++] = std::move(active[i]);
        }
        active.resize(w);
        for (int nd : gone) finish_task(nd);
    }
    if (active.empty()) return GVA_OK;
    ++rounds;
    // tasks of the light class first, then the fused class: each class's
    // items form one range, run by that class's kernels
    std::stable_partition(active.begin(), active.end(), [&](const BTask& tk) { return !nodes[tk.node].fused; });
    // the previous round's host-to-device copies read the staging area
    if (staged) {
        GVA_CUDA_B(cudaEventSynchronize(staged));
    } else {
        GVA_CUDA_B(cudaEventCreateWithFlags(&staged, cudaEventDisableTiming));
    }
    Profiler prof;
    Profiler* pf = profile ? &prof : nullptr;
    BatchCtx ctx{};
    ctx.vgraph = db.vgraph;
    ctx.G = db.num_graphs;
    ctx.words = ctx_words;
    ctx.graph_counts = graph_counts_dev();
    ctx.graph_bits = graph_bits_dev();
    const int nt = (int)active.size();
    // rows per work item: as many as fit 1024 words of rows (the widest task
    // of the round sets the shared-memory layout), a multiple of 32
    uint32_t kmax = 1;
    for (int t = 0; t < nt; ++t) kmax = std::max(kmax, nodes[active[t].node].width_in);
    uint32_t R = std::min<uint32_t>(tune.rows_per_item, std::max<uint32_t>(32, (768 / kmax) & ~31u));
    // staging: refs[nt] | item0[nt+1] | totals[nt] | outs[nt] | queue heads | wtask[nt] | witem0[nt+1]
    const size_t ref_bytes = (size_t)nt * sizeof(TaskRef);
    const size_t desc_max = 0;
    const size_t small_words = (size_t)(nt + 1) + nt + nt + 4 + nt + (nt + 1);
    char* h = staging.get(ref_bytes + desc_max + small_words * 8);
    if (!h) return fail(GVA_ERR_NOMEM, "pinned staging allocation failed");
    TaskRef* refs = (TaskRef*)h;
    uint64_t* h_item0 = (uint64_t*)(h + ref_bytes + desc_max);
    uint64_t* h_totals = h_item0 + (nt + 1);
    uint32_t** h_outs = (uint32_t**)(h_totals + nt);
    uint64_t* h_wtask = h_totals + 2 * nt + 4;  // nt 8-byte words holding uint32 task indices
    uint64_t* h_witem0 = h_wtask + nt;
    double cbytes = 0, crows = 0;
    uint64_t ni = 0, ni_light = 0;
    h_item0[0] = 0;
    for (int t = 0; t < nt; ++t) {
        const BTask& tk = active[t];
        BNode& nd = nodes[tk.node];
        if (!nd.fused) ni_light = ni + (tk.rows + R - 1) / R;
        refs[t] = TaskRef{(uint32_t)tk.node, 0u, tk.in, tk.rows};
        ni += (tk.rows + R - 1) / R;
        h_item0[t + 1] = ni;
        cbytes += (4.0 * nd.width_in + 8.0 * (nd.kind == STEP_EXT ? 1 : nd.n_pairs)) * (double)tk.rows;
        crows += (double)tk.rows;
    }
    if (ni == 0) return fail(GVA_ERR_ARG, "round without frontier rows");  // tasks always hold rows
    const uint64_t nc = (ni + kScanChunk - 1) / kScanChunk;
    auto grow = [&](void** p, size_t& cap, size_t need) -> bool {
        if (need <= cap) return true;
        if (*p) cudaFreeAsync(*p, s);
        size_t c = std::max(need, cap * 2);
        if (cudaMallocAsync(p, c, s) != cudaSuccess) {
            *p = nullptr;
            cap = 0;
            return false;
        }
        cap = c;
        return true;
    };
    {
        const int rc = ship_nodes();
        if (rc) return rc;
    }
    size_t read_cap = d_read ? 8 : 0;
    if (!grow(&d_desc, desc_cap, ref_bytes) || !grow((void**)&d_items, items_cap, std::max<uint64_t>(ni, 1) * 8) ||
        !grow((void**)&d_small, small_cap, small_words * 8) ||
        !grow((void**)&d_chunks, chunks_cap, (nc + 1) * 8) || (pf && !grow((void**)&d_read, read_cap, 8)))
        return fail(GVA_ERR_NOMEM, "batch bookkeeping allocation failed");
    uint64_t* d_item0 = d_small;
    uint64_t* d_totals = d_item0 + (nt + 1);
    uint32_t** d_outs = (uint32_t**)(d_totals + nt);
    unsigned long long* d_queue = (unsigned long long*)(d_totals + 2 * nt);  // four heads: count and write, per class
    uint64_t* d_wtask = d_totals + 2 * nt + 4;
    uint64_t* d_witem0 = d_wtask + nt;
    GVA_CUDA_B(cudaMemcpyAsync(d_desc, refs, ref_bytes, cudaMemcpyHostToDevice, s));
    GVA_CUDA_B(cudaMemcpyAsync(d_item0, h_item0, (nt + 1) * 8, cudaMemcpyHostToDevice, s));
    GVA_CUDA_B(cudaMemsetAsync(d_queue, 0, 32, s));
    if (pf) GVA_CUDA_B(cudaMemsetAsync(d_read, 0, 8, s));
    lap(0);

    RoundArgs ra{};
    ra.nodes = (const TaskDesc*)d_nodes;
    ra.refs = (const TaskRef*)d_desc;
    ra.item0 = d_item0;
    ra.n_items = ni;
    ra.nt = (uint32_t)nt;
    ra.rows_per_item = R;
    ra.hub = tune.hub;
    ra.kmax = kmax;
    ra.items = d_items;
    ra.queue = d_queue;
    ra.read_words = pf ? d_read : nullptr;
    ra.ctx = ctx;
    auto grid_for = [&](const void* fn, uint64_t items, size_t smem) -> uint32_t {
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kRoundWarps * 32, smem);
        return (uint32_t)std::min<uint64_t>((uint64_t)std::max(per_sm, 1) * (uint64_t)sms,
                                            (items + kRoundWarps - 1) / kRoundWarps);
    };
    cudaEvent_t ev = nullptr;
    if (pf) pf->begin(K_EXT_COUNT, cbytes, s, ev);
    if (ni_light > 0) {  // light class: items [0, ni_light)
        RoundArgs la = ra;
        la.item_base = 0;
        la.n_items = ni_light;
        la.queue = d_queue;
        const size_t smem = round_smem_bytes(R, kmax, false, false);
            const uint32_t g = grid_for((const void*)round_count_kernel<false>, ni_light, smem);
        round_count_kernel<false><<<g, kRoundWarps * 32, smem, s>>>(la);
        launches += 1;
        g_batch_launches += 1;
    }
    if (ni > ni_light) {  // fused class: items [ni_light, ni)
        RoundArgs fa = ra;
        fa.item_base = ni_light;
        fa.n_items = ni - ni_light;
        fa.queue = d_queue + 1;
        const size_t smem = round_smem_bytes(R, kmax, false, true);
            const uint32_t g = grid_for((const void*)round_count_kernel<true>, ni - ni_light, smem);
        round_count_kernel<true><<<g, kRoundWarps * 32, smem, s>>>(fa);
        launches += 1;
        g_batch_launches += 1;
    }
    if (pf) pf->end(ev, K_EXT_COUNT, cbytes, s, crows);
    if (pf) pf->begin(K_SCAN, 16.0 * ni, s, ev);
    scan_items_local_kernel<<<(unsigned)nc, 1024, 0, s>>>(d_items, ni, d_chunks, nullptr);
    scan_items_top_kernel<<<1, 1024, 0, s>>>(d_chunks, nc, d_items, ni, d_item0, (uint32_t)nt, d_totals, nullptr);
    if (pf) pf->end(ev, K_SCAN, 16.0 * ni, s, (double)ni);
    launches += 2;
    g_batch_launches += 2;
    GVA_CUDA_B(cudaGetLastError());
    GVA_CUDA_B(cudaMemcpyAsync(h_totals, d_totals, nt * 8, cudaMemcpyDeviceToHost, s));
    uint64_t h_read_count = 0;
    uint64_t* h_read = pf ? (uint64_t*)staging_read.get(8) : nullptr;
    if (pf && h_read) GVA_CUDA_B(cudaMemcpyAsync(h_read, d_read, 8, cudaMemcpyDeviceToHost, s));
    lap(1);
    {
        const auto w0 = std::chrono::steady_clock::now();
        cudaError_t e = cudaStreamSynchronize(s);
        wait_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
        if (e != cudaSuccess) return fail(GVA_ERR_CUDA, cudaGetErrorString(e));
        t_lap = std::chrono::steady_clock::now();
    }
    if (pf && h_read) {
        h_read_count = *h_read;
        for (auto& pe : pf->pending)
            if (pe.kind == K_EXT_COUNT) pe.bytes += 4.0 * (double)h_read_count;
    }

    // which tasks write this round: all when the outputs fit the budget,
    // else deepest first; a task larger than the budget is split
    uint64_t want = 0;
    for (int t = 0; t < nt; ++t) {
        const BNode& nd = nodes[active[t].node];
        if (nd.first_child < 0 || h_totals[t] == 0) continue;
        const BNode& st = nd;
        want += ((h_totals[t] * (st.kind == STEP_EXT ? st.width_in + 1 : st.width_in) * 4ull) + 15) & ~15ull;
    }
    std::vector<int>& order = scratch_order;
    order.clear();
    for (int t = 0; t < nt; ++t) {
        const BNode& nd = nodes[active[t].node];
        for (int q = nd.first_term; q >= 0; q = plans[q].next_term) plans[q].count += h_totals[t];
        if (nd.first_child >= 0 && h_totals[t] > 0) order.push_back(t);
    }
    if (want > budget)
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return nodes[active[a].node].depth > nodes[active[b].node].depth; });
    std::vector<BTask> next;
    std::vector<char>& chosen_flag = scratch_flag;
    chosen_flag.assign(nt, 0);
    uint64_t used = 0;
    std::vector<uint64_t>& off_words = scratch_off;
    off_words.assign(nt, 0);
    int status = GVA_OK;
    for (int t : order) {
        const BNode& st = nodes[active[t].node];
        const uint32_t w = st.kind == STEP_EXT ? st.width_in + 1 : st.width_in;
        const uint64_t bytes = h_totals[t] * w * 4ull;
        if (used + bytes <= budget) {
            off_words[t] = used / 4;
            used += (bytes + 15) & ~15ull;
            chosen_flag[t] = 1;
        } else if (bytes > budget) {
            BTask a = active[t], b = active[t];
            const uint64_t half = a.rows / 2;
            if (half == 0) {
                status = fail(GVA_ERR_NOMEM, "a single frontier row expands beyond the memory budget");
                break;
            }
            a.rows = half;
            b.in = a.in + half * st.width_in;
            b.rows = active[t].rows - half;
            nodes[a.node].at++;  // one task became two
            next.push_back(a);
            next.push_back(b);
            chosen_flag[t] = 2;
            ++splits;
        } else {
            next.push_back(active[t]);  // fits alone: waits for the next round
            chosen_flag[t] = 2;
        }
    }
    if (status) return status;
    lap(2);
    std::shared_ptr<void> buf;
    if (used > 0) {
        void* p = nullptr;
        if (cudaMallocAsync(&p, used, s) != cudaSuccess) return fail(GVA_ERR_NOMEM, "frontier allocation failed");
        cudaStream_t ss = s;
        buf = std::shared_ptr<void>(p, [ss](void* q) { cudaFreeAsync(q, ss); });
        double wbytes = 0, wrows = 0;
        uint32_t nw = 0;
        uint64_t wi = 0, wi_light = 0;
        uint32_t* h_wt = (uint32_t*)h_wtask;  // task index per writing slot (uint32)
        h_witem0[0] = 0;
        for (int t = 0; t < nt; ++t) {
            h_outs[t] = chosen_flag[t] == 1 ? (uint32_t*)p + off_words[t] : nullptr;
            if (chosen_flag[t] != 1) continue;
            h_wt[nw] = (uint32_t)t;
            wi += h_item0[t + 1] - h_item0[t];
            h_witem0[++nw] = wi;
            if (!nodes[active[t].node].fused) wi_light = wi;
            wrows += (double)active[t].rows;
            const BNode& st = nodes[active[t].node];
            const double k = st.width_in;
            wbytes += (4.0 * k + 8.0) * (double)active[t].rows +
                      (st.kind == STEP_EXT ? (4.0 + 4.0 * (k + 1)) : 4.0 * k) * (double)h_totals[t];
        }
        GVA_CUDA_B(cudaMemcpyAsync(d_outs, h_outs, nt * sizeof(uint32_t*), cudaMemcpyHostToDevice, s));
        GVA_CUDA_B(cudaMemcpyAsync(d_wtask, h_wtask, (size_t)(2 * nt + 1) * 8, cudaMemcpyHostToDevice, s));
        GVA_CUDA_B(cudaEventRecord(staged, s));  // the last read of the staging area this round
        RoundArgs wa = ra;
        wa.n_items = wi;
        wa.wtask = (const uint32_t*)d_wtask;
        wa.witem0 = d_witem0;
        wa.nt = nw;
        wa.chunks = d_chunks;
        wa.n_count_items = ni;
        wa.n_chunks = nc;
        wa.task_out = d_outs;
        wa.read_words = nullptr;
        if (pf) pf->begin(K_EXT_WRITE, wbytes, s, ev);
        if (wi_light > 0) {
            RoundArgs la = wa;
            la.item_base = 0;
            la.n_items = wi_light;
            la.queue = d_queue + 2;
            const size_t smem = round_smem_bytes(R, kmax, true, false);
            const uint32_t g = grid_for((const void*)round_write_kernel<false>, wi_light, smem);
                round_write_kernel<false><<<g, kRoundWarps * 32, smem, s>>>(la);
            launches += 1;
            g_batch_launches += 1;
        }
        if (wi > wi_light) {
            RoundArgs fa = wa;
            fa.item_base = wi_light;
            fa.n_items = wi - wi_light;
            fa.queue = d_queue + 3;
            const size_t smem = round_smem_bytes(R, kmax, true, true);
            const uint32_t g = grid_for((const void*)round_write_kernel<true>, wi - wi_light, smem);
                round_write_kernel<true><<<g, kRoundWarps * 32, smem, s>>>(fa);
            launches += 1;
            g_batch_launches += 1;
        }
        if (pf) pf->end(ev, K_EXT_WRITE, wbytes, s, wrows);
        GVA_CUDA_B(cudaGetLastError());
    } else {
        GVA_CUDA_B(cudaEventRecord(staged, s));
    }
    lap(3);
    std::vector<int> ended;
    for (int t = 0; t < nt; ++t) {
        if (chosen_flag[t] == 2) continue;  // still active (deferred or split)
        if (chosen_flag[t] == 1)
            for (int c = nodes[active[t].node].first_child; c >= 0; c = nodes[c].next_sibling) {
                nodes[c].at++;
                next.push_back({c, h_outs[t], h_totals[t], buf});
            }
        ended.push_back(active[t].node);
    }
    active.swap(next);
    for (int nd : ended) finish_task(nd);
    lap(4);
    if (pf) {
        GVA_CUDA_B(cudaStreamSynchronize(s));
        pf->resolve();
        for (int i = 0; i < K_NUM; ++i) {
            kstat[i].launches += pf->stat[i].launches;
            kstat[i].ms += pf->stat[i].ms;
            kstat[i].bytes += pf->stat[i].bytes;
            kstat[i].rows += pf->stat[i].rows;
        }
    }
    return GVA_OK;
}

int BatchSession::ship_nodes() {
    const size_t dev_need = nodes.size() * sizeof(TaskDesc);
    if (dev_need > node_cap) {  // keep the descriptors already shipped
        void* p = nullptr;
        const size_t cap = std::max(dev_need, node_cap * 2);
        if (cudaMallocAsync(&p, cap, s) != cudaSuccess) return fail(GVA_ERR_NOMEM, "node descriptor allocation failed");
        if (d_nodes && shipped > 0)
            GVA_CUDA_B(cudaMemcpyAsync(p, d_nodes, shipped * sizeof(TaskDesc), cudaMemcpyDeviceToDevice, s));
        if (d_nodes) cudaFreeAsync(d_nodes, s);
        d_nodes = p;
        node_cap = cap;
    }
    if (shipped < nodes.size()) {  // descriptors of the nodes submitted since the last shipment
        // from pinned staging: asynchronous, the next wave refills the buffer
        // after desc_ev (from host memory: complete when the call returns)
        GVA_CUDA_B(cudaMemcpyAsync((char*)d_nodes + shipped * sizeof(TaskDesc),
                                   inited ? (const void*)desc_pin : (const void*)desc_host.data(),
                                   (nodes.size() - shipped) * sizeof(TaskDesc), cudaMemcpyHostToDevice, s));
        if (inited) {
            GVA_CUDA_B(cudaEventRecord(desc_ev, s));
            desc_pending = true;
        }
        shipped = nodes.size();
    }
    return GVA_OK;
}

// Resident CTAs per SM of a round kernel at a dynamic shared memory size,
// cached per (device, kernel, size): the occupancy query is a driver call
// and a device-scheduled run makes several per round.
static uint32_t resident_ctas(int device, const void* fn, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<int, const void*, size_t>, uint32_t> known;
    const auto key = std::make_tuple(device, fn, smem);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = known.find(key);
        if (it != known.end()) return it->second;
    }
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kRoundWarps * 32, smem) != cudaSuccess) {
        cudaGetLastError();
        per_sm = 1;
    }
    const uint32_t n = (uint32_t)std::max(per_sm, 1);
    std::lock_guard<std::mutex> lk(mu);
    known[key] = n;
    return n;
}

int BatchSession::run_device() {
    if (host_rounds || profile || waves.size() != 1 || rounds != 0 || active.empty() || !db.seed_verts) return GVA_OK;
    const auto t_start = std::chrono::steady_clock::now();
    double wait_before = wait_ms;
    struct Timer {
        std::chrono::steady_clock::time_point t0;
        double& acc;
        double& wait;
        double wait0;
        ~Timer() {
            acc += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() -
                   (wait - wait0);
        }
    } timer{t_start, round_host_ms, wait_ms, wait_before};
    auto t_lap = t_start;
    auto lap = [&](int k) {  // phase_ms: schedule tables, uploads, launches, -, results
        const auto now = std::chrono::steady_clock::now();
        phase_ms[k] += std::chrono::duration<double, std::milli>(now - t_lap).count();
        t_lap = now;
    };
    const size_t nn = nodes.size();
    for (const BTask& tk : active)
        if (nodes[tk.node].depth != 1) return GVA_OK;
    int D = 0;
    for (const BNode& nd : nodes) D = std::max(D, nd.depth);
    if (D < 1) return GVA_OK;
    // per depth: widest input row, nodes, nodes of each class
    std::vector<uint32_t> kmax(D + 2, 1), at_depth(D + 2, 0), light_at(D + 2, 0), fused_at(D + 2, 0);
    for (const BNode& nd : nodes) {
        kmax[nd.depth] = std::max(kmax[nd.depth], nd.width_in);
        at_depth[nd.depth]++;
        (nd.fused ? fused_at : light_at)[nd.depth]++;
    }
    uint32_t refs_cap = 1;
    for (int d = 1; d <= D; ++d) refs_cap = std::max(refs_cap, at_depth[d]);
    std::vector<uint32_t> R(D + 2, 32);
    for (int d = 1; d <= D; ++d)
        R[d] = std::min<uint32_t>(tune.rows_per_item, std::max<uint32_t>(32, (768 / kmax[d]) & ~31u));
    // children that can match, light class first: counted per node, placed
    // by a prefix over the nodes, then listed (both passes on the host's
    // cores, by ranges of nodes)
    std::vector<NodeRun> info(nn);
    const unsigned T = nn >= 8192 ? std::min<unsigned>(pool_width(), 32) : 1u;
    std::atomic<bool> too_many{false};
    pool_run(T, [&](unsigned t) {
        for (size_t id = nn * t / T; id < nn * (t + 1) / T; ++id) {
            const BNode& nd = nodes[id];
            NodeRun r{};
            r.out_w = nd.kind == STEP_EXT ? nd.width_in + 1 : nd.width_in;
            size_t cnt[2] = {0, 0};
            for (int c = nd.first_child; c >= 0; c = nodes[c].next_sibling)
                if (!nodes[c].always_empty) cnt[nodes[c].fused ? 1 : 0]++;
            if (cnt[0] > 0xffff || cnt[1] > 0xffff) too_many = true;  // beyond the schedule's child counts
            r.n_light = (uint16_t)cnt[0];
            r.n_fused = (uint16_t)cnt[1];
            info[id] = r;
        }
    });
    if (too_many) return GVA_OK;
    uint32_t nk = 0;
    for (size_t id = 0; id < nn; ++id) {
        info[id].child0 = nk;
        nk += info[id].n_light + info[id].n_fused;
    }
    std::vector<uint32_t> kids(nk);
    pool_run(T, [&](unsigned t) {
        for (size_t id = nn * t / T; id < nn * (t + 1) / T; ++id) {
            uint32_t at[2] = {info[id].child0, info[id].child0 + info[id].n_light};
            for (int c = nodes[id].first_child; c >= 0; c = nodes[c].next_sibling)
                if (!nodes[c].always_empty) kids[at[nodes[c].fused ? 1 : 0]++] = (uint32_t)c;
        }
    });
    // the first round's tasks (depth 1, from the seed lists), light class first
    std::vector<TaskRef> r0;
    r0.reserve(active.size());
    uint32_t nt_light0 = 0;
    for (uint32_t f = 0; f < 2; ++f) {
        for (const BTask& tk : active) {
            const BNode& nd = nodes[tk.node];
            if (nd.always_empty || nd.fused != f || tk.rows == 0) continue;
            r0.push_back(TaskRef{(uint32_t)tk.node, 0u, tk.in, tk.rows});
        }
        if (f == 0) nt_light0 = (uint32_t)r0.size();
    }
    std::vector<uint64_t> i0(r0.size() + 1, 0);
    uint64_t ni_light0 = 0;
    for (size_t t = 0; t < r0.size(); ++t) {
        i0[t + 1] = i0[t] + (r0[t].nrows + R[1] - 1) / R[1];
        if (t + 1 == nt_light0) ni_light0 = i0[t + 1];
    }
    // two frontier regions (a round writes one while its tasks read the other)
    uint64_t region = db.round_region_bytes.load();
    if (region == 0) region = 2ull << 30;
    if (2 * region > budget) return GVA_OK;
    const uint64_t region_words = region / 4;
    const uint64_t items_cap = std::max<uint64_t>(i0.back(), region_words / 64 + refs_cap) + 1;
    const uint64_t chunks_cap = items_cap / kScanChunk + 2;
    // one block for the schedule's small arrays
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t o_state = 0;
    const size_t o_refs0 = o_state + al((D + 2) * sizeof(RunState));
    const size_t o_refs1 = o_refs0 + al((size_t)refs_cap * sizeof(TaskRef));
    const size_t o_item00 = o_refs1 + al((size_t)refs_cap * sizeof(TaskRef));
    const size_t o_item01 = o_item00 + al(((size_t)refs_cap + 1) * 8);
    const size_t o_totals = o_item01 + al(((size_t)refs_cap + 1) * 8);
    const size_t o_outs = o_totals + al((size_t)refs_cap * 8);
    const size_t o_wtask = o_outs + al((size_t)refs_cap * 8);
    const size_t o_witem0 = o_wtask + al((size_t)refs_cap * 4);
    const size_t o_ntot = o_witem0 + al(((size_t)refs_cap + 1) * 8);
    const size_t o_info = o_ntot + al(nn * 8);
    const size_t o_kids = o_info + al(nn * sizeof(NodeRun));
    const uint32_t nb = (refs_cap + kPlanThreads - 1) / kPlanThreads;
    const size_t o_flag = o_kids + al(std::max<size_t>(kids.size(), 1) * 4);
    const size_t o_bsum = o_flag + 256;
    const size_t o_items = o_bsum + al(((size_t)nb + 1) * kPlanVals * 8);
    const size_t o_chunks = o_items + al(items_cap * 8);
    const size_t small_bytes = o_chunks + al((chunks_cap + 1) * 8);
    {
        const int rc = ship_nodes();
        if (rc) return rc;
    }
    lap(0);
    char* blk = nullptr;
    void* reg[2] = {nullptr, nullptr};
    if (cudaMallocAsync((void**)&blk, small_bytes, s) != cudaSuccess) {  // no room: host rounds
        cudaGetLastError();
        return GVA_OK;
    }
    if (cudaMallocAsync(&reg[0], region, s) != cudaSuccess || cudaMallocAsync(&reg[1], region, s) != cudaSuccess) {
        cudaGetLastError();
        for (void* q : {(void*)blk, reg[0], reg[1]})
            if (q) cudaFreeAsync(q, s);
        return GVA_OK;
    }
    auto free_all = [&]() {
        for (void* q : {(void*)blk, reg[0], reg[1]}) cudaFreeAsync(q, s);
    };
    RunState* states = (RunState*)(blk + o_state);
    TaskRef* refs[2] = {(TaskRef*)(blk + o_refs0), (TaskRef*)(blk + o_refs1)};
    uint64_t* item0[2] = {(uint64_t*)(blk + o_item00), (uint64_t*)(blk + o_item01)};
    uint64_t* totals = (uint64_t*)(blk + o_totals);
    uint32_t** outs = (uint32_t**)(blk + o_outs);
    uint32_t* wtask = (uint32_t*)(blk + o_wtask);
    uint64_t* witem0 = (uint64_t*)(blk + o_witem0);
    uint64_t* ntot = (uint64_t*)(blk + o_ntot);
    NodeRun* d_info = (NodeRun*)(blk + o_info);
    uint32_t* d_kids = (uint32_t*)(blk + o_kids);
    uint32_t* d_flag = (uint32_t*)(blk + o_flag);
    uint64_t* items = (uint64_t*)(blk + o_items);
    uint64_t* chunks = (uint64_t*)(blk + o_chunks);
    RunState s1{};
    s1.ni = i0.back();
    s1.ni_light = ni_light0;
    s1.nt = (uint32_t)r0.size();
    s1.nt_light = nt_light0;
    // pageable sources: each copy is complete when its call returns
    GVA_CUDA_B(cudaMemsetAsync(blk + o_state, 0, (D + 2) * sizeof(RunState), s));
    GVA_CUDA_B(cudaMemsetAsync(ntot, 0, nn * 8, s));
    GVA_CUDA_B(cudaMemsetAsync(d_flag, 0, 4, s));
    GVA_CUDA_B(cudaMemcpyAsync(states + 1, &s1, sizeof s1, cudaMemcpyHostToDevice, s));
    GVA_CUDA_B(cudaMemcpyAsync(d_info, info.data(), nn * sizeof(NodeRun), cudaMemcpyHostToDevice, s));
    if (!kids.empty()) GVA_CUDA_B(cudaMemcpyAsync(d_kids, kids.data(), kids.size() * 4, cudaMemcpyHostToDevice, s));
    if (!r0.empty()) GVA_CUDA_B(cudaMemcpyAsync(refs[1], r0.data(), r0.size() * sizeof(TaskRef), cudaMemcpyHostToDevice, s));
    GVA_CUDA_B(cudaMemcpyAsync(item0[1], i0.data(), i0.size() * 8, cudaMemcpyHostToDevice, s));

    BatchCtx ctx{};
    ctx.vgraph = db.vgraph;
    ctx.G = db.num_graphs;
    ctx.words = ctx_words;
    ctx.graph_counts = graph_counts_dev();
    ctx.graph_bits = graph_bits_dev();
    auto grid = [&](const void* fn, size_t smem) -> uint32_t { return resident_ctas(db.device, fn, smem) * (uint32_t)sms; };
    lap(1);
    uint64_t nl = 0;
    for (int d = 1; d <= D; ++d) {
        const int b = d & 1;
        RoundArgs ra{};
        ra.nodes = (const TaskDesc*)d_nodes;
        ra.refs = refs[b];
        ra.item0 = item0[b];
        ra.rows_per_item = R[d];
        ra.hub = tune.hub;
        ra.kmax = kmax[d];
        ra.items = items;
        ra.ctx = ctx;
        ra.dyn = states + d;
        if (light_at[d]) {
            const size_t smem = round_smem_bytes(R[d], kmax[d], false, false);
            round_count_kernel<false><<<grid((const void*)round_count_kernel<false>, smem), kRoundWarps * 32, smem, s>>>(ra);
            ++nl;
        }
        if (fused_at[d]) {
            const size_t smem = round_smem_bytes(R[d], kmax[d], false, true);
            round_count_kernel<true><<<grid((const void*)round_count_kernel<true>, smem), kRoundWarps * 32, smem, s>>>(ra);
            ++nl;
        }
        scan_items_local_kernel<<<2 * sms, 1024, 0, s>>>(items, 0, chunks, states + d);
        scan_items_top_kernel<<<1, 1024, 0, s>>>(chunks, 0, items, 0, item0[b], 0, totals, states + d);
        PlanArgs pa{};
        pa.st = states + d;
        pa.nx = states + d + 1;
        pa.refs = refs[b];
        pa.item0 = item0[b];
        pa.totals = totals;
        pa.info = d_info;
        pa.children = d_kids;
        pa.node_total = ntot;
        pa.region = (uint32_t*)reg[b];
        pa.region_words = region_words;
        pa.outs = outs;
        pa.wtask = wtask;
        pa.witem0 = witem0;
        pa.next_refs = refs[b ^ 1];
        pa.next_item0 = item0[b ^ 1];
        pa.refs_cap = refs_cap;
        pa.items_cap = items_cap;
        pa.rows_next = R[d + 1];
        pa.overflow = d_flag;
        pa.bsum = (uint64_t*)(blk + o_bsum);
        pa.nb = nb;
        plan_sum_kernel<<<nb, kPlanThreads, 0, s>>>(pa);
        plan_top_kernel<<<1, kPlanThreads, 0, s>>>(pa);
        plan_write_kernel<<<nb, kPlanThreads, 0, s>>>(pa);
        nl += 5;
        if (d < D) {  // the deepest round's tasks have no children
            RoundArgs wa = ra;
            wa.wtask = wtask;
            wa.witem0 = witem0;
            wa.chunks = chunks;
            wa.task_out = outs;
            if (light_at[d]) {
                const size_t smem = round_smem_bytes(R[d], kmax[d], true, false);
                round_write_kernel<false><<<grid((const void*)round_write_kernel<false>, smem), kRoundWarps * 32, smem, s>>>(wa);
                ++nl;
            }
            if (fused_at[d]) {
                const size_t smem = round_smem_bytes(R[d], kmax[d], true, true);
                round_write_kernel<true><<<grid((const void*)round_write_kernel<true>, smem), kRoundWarps * 32, smem, s>>>(wa);
                ++nl;
            }
        }
    }
    launches += nl;
    lap(2);
    g_batch_launches += nl;
    {
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            free_all();
            return fail(GVA_ERR_CUDA, std::string("device-scheduled rounds: ") + cudaGetErrorString(e));
        }
    }
    char* h = staging.get(nn * 8 + 16);
    if (!h) {
        free_all();
        return fail(GVA_ERR_NOMEM, "pinned staging allocation failed");
    }
    uint64_t* h_tot = (uint64_t*)h;
    uint32_t* h_flag = (uint32_t*)(h + nn * 8);
    GVA_CUDA_B(cudaMemcpyAsync(h_tot, ntot, nn * 8, cudaMemcpyDeviceToHost, s));
    GVA_CUDA_B(cudaMemcpyAsync(h_flag, d_flag, 4, cudaMemcpyDeviceToHost, s));
    free_all();
    {
        const auto w0 = std::chrono::steady_clock::now();
        const cudaError_t e = cudaStreamSynchronize(s);
        wait_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
        if (e != cudaSuccess) return fail(GVA_ERR_CUDA, cudaGetErrorString(e));
    }
    t_lap = std::chrono::steady_clock::now();
    struct LapEnd {
        decltype(lap)& f;
        ~LapEnd() { f(4); }
    } lap_end{lap};
    if (*h_flag) {
        // a round outgrew a region: later runs get regions twice as large, and
        // this one starts over with host-scheduled rounds
        uint64_t cur = db.round_region_bytes.load();
        while (cur < 2 * region && !db.round_region_bytes.compare_exchange_weak(cur, 2 * region)) {
        }
        if (acc) GVA_CUDA_B(cudaMemsetAsync(acc, 0, acc_bytes, s));
        for (BNode& nd : nodes) {
            nd.at = 0;
            nd.closed = false;
        }
        for (PlanRec& pr : plans) {
            pr.count = 0;
            pr.done = false;
        }
        completed.clear();
        active.clear();
        start_seeds(0);
        return GVA_OK;
    }
    for (size_t q = 0; q < plans.size(); ++q) {
        PlanRec& pr = plans[q];
        pr.count = h_tot[pr.terminal];
        pr.done = true;
        completed.push_back((int)q);
    }
    for (BNode& nd : nodes) {
        nd.at = 0;
        nd.closed = true;
    }
    active.clear();
    rounds += (uint64_t)D;
    device_rounds += (uint64_t)D;
    return GVA_OK;
}

std::vector<int> BatchSession::take_completed() {
    std::vector<int> out;
    out.swap(completed);
    return out;
}

int BatchSession::read_support(int q, uint32_t* support, uint64_t* graph_counts_host) {
    // plans ending on the same node share the slot of the node's first plan
    const int slot = plans[first_peer(q)].slot;
    if (support) {
        // pinned staging: a pageable read-back would hold this thread inside
        // the driver until the stream drains
        uint32_t* bits = (uint32_t*)staging_read.get((size_t)ctx_words * 4);
        if (!bits) return fail(GVA_ERR_NOMEM, "pinned staging allocation failed");
        GVA_CUDA_B(cudaMemcpyAsync(bits, graph_bits_dev() + (size_t)slot * ctx_words, ctx_words * 4,
                                   cudaMemcpyDeviceToHost, s));
        GVA_CUDA_B(cudaStreamSynchronize(s));
        uint32_t c = 0;
        for (uint32_t i = 0; i < ctx_words; ++i) c += (uint32_t)__builtin_popcount(bits[i]);
        *support = c;
    }
    if (graph_counts_host && want_graph_counts) {
        uint64_t* h = (uint64_t*)staging_read.get((size_t)db.num_graphs * 8);
        if (!h) return fail(GVA_ERR_NOMEM, "pinned staging allocation failed");
        GVA_CUDA_B(cudaMemcpyAsync(h, graph_counts_dev() + (size_t)slot * db.num_graphs, (size_t)db.num_graphs * 8,
                                   cudaMemcpyDeviceToHost, s));
        GVA_CUDA_B(cudaStreamSynchronize(s));
        memcpy(graph_counts_host, h, (size_t)db.num_graphs * 8);
    }
    return GVA_OK;
}

void BatchSession::release(int q) {
    // a slot is recycled once every plan sharing it is released
    PlanRec& p = plans[q];
    if (p.released) return;
    p.released = true;
    if (p.slot < 0) return;
    const int t = p.terminal;
    for (int o = nodes[t].first_term; o >= 0; o = plans[o].next_term)
        if (!plans[o].released) return;
    for (int o = nodes[t].first_term; o >= 0; o = plans[o].next_term) {
        const int sl = plans[o].slot;
        if (sl < 0) continue;
        if (want_graph_counts)
            cudaMemsetAsync(graph_counts_dev() + (size_t)sl * db.num_graphs, 0, (size_t)db.num_graphs * 8, s);
        cudaMemsetAsync(graph_bits_dev() + (size_t)sl * ctx_words, 0, (size_t)ctx_words * 4, s);
        free_slots.push_back(sl);
        plans[o].slot = -1;
    }
}

__global__ void slot_popcount_kernel(const uint32_t* __restrict__ bits, uint32_t words, uint32_t nslots,
                                     uint32_t* __restrict__ out) {
    const uint32_t slot = blockIdx.x;
    if (slot >= nslots) return;
    uint32_t c = 0;
    for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) c += __popc(bits[(uint64_t)slot * words + w]);
    c = warp_sum(c);
    __shared__ uint32_t ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += ws[i];
        out[slot] = t;
    }
}

int prepare_batch(DevDB& db, std::vector<std::vector<Step>>&& steps, cudaStream_t s, uint64_t budget,
                  bool per_graph, bool graph_counts, bool profile, PreparedBatch& out, bool presorted,
                  bool host_rounds) {
    const auto t0 = std::chrono::steady_clock::now();
    GVA_CUDA_B(cudaSetDevice(db.device));
    out.nq = (int)steps.size();
    out.per_graph = per_graph;
    out.graph_counts = graph_counts;
    out.ids.clear();
    if (out.nq == 0) return GVA_OK;
    out.ses.reset(new BatchSession(db, s, budget, per_graph ? (uint32_t)out.nq : 0, graph_counts, profile));
    out.ses->host_rounds = host_rounds;
    int rc = out.ses->init();
    if (!rc) rc = out.ses->submit(std::move(steps), {}, &out.ids, presorted);
    out.prep_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

int finish_batch(DevDB& db, PreparedBatch& pb, uint64_t* counts, uint64_t* graph_counts_host, uint32_t* support_host,
                 BatchStats* stats, const volatile int* cancel, const uint32_t* order) {
    const int nq = pb.nq;
    // the result of submitted plan q goes to index at(q) of the caller's arrays
    auto at = [&](int q) -> size_t { return order ? (size_t)order[q] : (size_t)q; };
    for (int q = 0; q < nq; ++q) counts[at(q)] = 0;
    if (nq == 0) return GVA_OK;
    GVA_CUDA_B(cudaSetDevice(db.device));
    BatchSession& ses = *pb.ses;
    cudaStream_t s = ses.stream();
    if ((graph_counts_host && !pb.graph_counts) || (support_host && !pb.per_graph))
        return fail(GVA_ERR_ARG, "per-graph results were not prepared for this batch");
    static thread_local cudaEvent_t tev[64][2];
    const int dev = db.device;
    if (dev < 0 || dev >= 64) return fail(GVA_ERR_ARG, "device index out of range");
    if (!tev[dev][0]) {
        GVA_CUDA_B(cudaEventCreate(&tev[dev][0]));
        GVA_CUDA_B(cudaEventCreate(&tev[dev][1]));
    }
    const auto t_fin0 = std::chrono::steady_clock::now();
    GVA_CUDA_B(cudaEventRecord(tev[dev][0], s));
    int rc = GVA_OK;
    const auto t_loop0 = std::chrono::steady_clock::now();
    if (!(cancel && *cancel)) rc = ses.run_device();
    while (!rc && !ses.idle()) {
        if (cancel && *cancel) {
            rc = fail(GVA_ERR_CANCELLED, "cancelled");
            break;
        }
        rc = ses.round();
    }
    const double loop_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_loop0).count();
    if (stats) stats->loop_end_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_fin0).count();
    const std::vector<int>& ids = pb.ids;
    if (!rc) {
        for (int q = 0; q < nq; ++q) counts[at(q)] = ses.plan(ids[q]).count;
        if (support_host || graph_counts_host) {
            // supports counted on the device; identical plans read their first one's slot
            uint32_t* d_pop = nullptr;
            if (cudaMallocAsync((void**)&d_pop, (size_t)nq * 4, s) != cudaSuccess)
                rc = fail(GVA_ERR_NOMEM, "support counters");
            Staging pop_stage;
            uint32_t* pop = (uint32_t*)pop_stage.get((size_t)nq * 4);
            if (!rc && !pop) {
                cudaFreeAsync(d_pop, s);
                rc = fail(GVA_ERR_NOMEM, "pinned staging allocation failed");
            }
            if (!rc) {
                slot_popcount_kernel<<<nq, 256, 0, s>>>(ses.graph_bits_dev(), ses.words(), (uint32_t)nq, d_pop);
                cudaMemcpyAsync(pop, d_pop, (size_t)nq * 4, cudaMemcpyDeviceToHost, s);
                cudaFreeAsync(d_pop, s);
            }
            // per-graph counts by slot, landed in pinned staging (reused
            // across runs), then each plan's row copied to its place
            Staging gc_stage;
            const size_t G = db.num_graphs;
            uint64_t* gc = nullptr;
            if (!rc && graph_counts_host) {
                gc = (uint64_t*)gc_stage.get((size_t)nq * G * 8);
                if (!gc) rc = fail(GVA_ERR_NOMEM, "pinned staging allocation failed");
                if (!rc)
                    cudaMemcpyAsync(gc, ses.graph_counts_dev(), (size_t)nq * G * 8, cudaMemcpyDeviceToHost, s);
            }
            if (!rc)
                rc = cudaStreamSynchronize(s) == cudaSuccess ? GVA_OK : fail(GVA_ERR_CUDA, "result read-back failed");
            for (int q = 0; q < nq && !rc; ++q) {
                const int sl = ses.plan(ses.first_peer(ids[q])).slot;
                if (support_host) support_host[at(q)] = pop[sl];
                if (gc) std::copy(gc + (size_t)sl * G, gc + (size_t)(sl + 1) * G, graph_counts_host + at(q) * G);
            }
        }
    }
    if (stats) {
        stats->read_end_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_fin0).count();
        stats->submit_ms = ses.submit_ms;
        stats->round_host_ms = ses.round_host_ms;
        stats->wait_ms = ses.wait_ms;
        stats->rounds = ses.rounds;
        stats->device_rounds = ses.device_rounds;
        stats->splits = ses.splits;
        stats->launches = ses.launches;
        stats->nodes = ses.num_nodes();
        for (int i = 0; i < 5; ++i) stats->phase_ms[i] = ses.phase_ms[i];
        for (int i = 0; i < K_NUM; ++i) stats->kstat[i] = ses.kstat[i];
    }
    cudaEventRecord(tev[dev][1], s);
    pb.ses.reset();  // frees the session's device memory (stream-ordered) and syncs its stream
    cudaEventSynchronize(tev[dev][1]);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, tev[dev][0], tev[dev][1]);
    if (stats) {
        stats->gpu_ms = ms;
        const double fin_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_fin0).count();
        stats->session_ms = (pb.prep_ms - stats->submit_ms) + (fin_ms - loop_ms);
    }
    return rc;
}

// A second stream of the device for the second half of a large batched run
// (created once per device and kept), ordered after the work already on `s`.
static int second_stream(int device, cudaStream_t s, cudaStream_t& out) {
    static std::mutex mu;
    static cudaStream_t aux[64] = {};
    static cudaEvent_t ev[64] = {};
    if (device < 0 || device >= 64) return fail(GVA_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    GVA_CUDA_B(cudaSetDevice(device));
    if (!aux[device]) {
        GVA_CUDA_B(cudaStreamCreateWithFlags(&aux[device], cudaStreamNonBlocking));
        GVA_CUDA_B(cudaEventCreateWithFlags(&ev[device], cudaEventDisableTiming));
    }
    GVA_CUDA_B(cudaEventRecord(ev[device], s));
    GVA_CUDA_B(cudaStreamWaitEvent(aux[device], ev[device], 0));
    out = aux[device];
    return GVA_OK;
}

// Plans ordered by their sequences of step keys (64-bit hashes of the key
// fields), so that plans sharing a step prefix are adjacent and the trie is
// built against the previous plan only (presorted submit), with the nodes of
// the indexed build (but for seed nodes repeated across buckets, below).
// Keys hashed, bucketed and sorted on the host's cores.
static void order_by_step_keys(const std::vector<std::vector<Step>>& steps, std::vector<uint32_t>& order) {
    const size_t n = steps.size();
    size_t w = 1;
    for (const auto& v : steps) w = std::max(w, v.size());
    // 0 ends a plan's sequence; the buffer is kept per thread (a fresh one
    // of this size would be mapped and faulted in page by page every call)
    // (a local reference: the jobs below run on other threads, where the
    // thread-local name would mean their own buffer)
    static thread_local std::vector<uint64_t> key_buf;
    std::vector<uint64_t>& key = key_buf;
    key.assign(n * w, 0);
    // Plans go to buckets by their first two steps (a plan's trie path is
    // decided in its bucket: plans sharing two or more leading steps share a
    // bucket), buckets are filled by ranges of plans and sorted one job each;
    // no merge.  Equal first steps in two buckets only repeat a seed node
    // (seed nodes launch nothing; their children differ).
    const size_t T = n < 2048 ? 1 : std::min<size_t>(32, pool_width());
    const uint32_t B = (uint32_t)std::min<size_t>(256, 4 * T);
    std::vector<size_t> cut(T + 1);
    for (size_t c = 0; c <= T; ++c) cut[c] = n * c / T;
    static thread_local std::vector<uint16_t> bucket_buf;
    std::vector<uint16_t>& bucket = bucket_buf;
    bucket.resize(n);
    std::vector<uint32_t> cnt((size_t)T * B, 0);  // [chunk][bucket], then where the chunk's entries of a bucket start
    pool_run((unsigned)T, [&](unsigned c) {
        uint32_t* my = cnt.data() + (size_t)c * B;
        for (size_t i = cut[c]; i < cut[c + 1]; ++i) {
            for (size_t j = 0; j < steps[i].size(); ++j) key[i * w + j] = step_key_hash(steps[i][j]);
            uint64_t h = key[i * w] * 0x9e3779b97f4a7c15ull ^ (w > 1 ? key[i * w + 1] : 0);
            h ^= h >> 31;
            h *= 0xbf58476d1ce4e5b9ull;
            h ^= h >> 29;
            bucket[i] = (uint16_t)(h % B);
            my[bucket[i]]++;
        }
    });
    std::vector<size_t> bstart(B + 1, 0);
    {
        size_t at = 0;
        for (uint32_t b = 0; b < B; ++b) {
            bstart[b] = at;
            for (size_t c = 0; c < T; ++c) {
                const uint32_t k = cnt[c * B + b];
                cnt[c * B + b] = (uint32_t)at;
                at += k;
            }
        }
        bstart[B] = at;
    }
    order.resize(n);
    pool_run((unsigned)T, [&](unsigned c) {
        uint32_t* my = cnt.data() + (size_t)c * B;
        for (size_t i = cut[c]; i < cut[c + 1]; ++i) order[my[bucket[i]]++] = (uint32_t)i;
    });
    auto less = [&](uint32_t a, uint32_t b) {
        const uint64_t* ka = key.data() + (size_t)a * w;
        const uint64_t* kb = key.data() + (size_t)b * w;
        for (size_t j = 0; j < w; ++j)
            if (ka[j] != kb[j]) return ka[j] < kb[j];
        return a < b;
    };
    pool_run(B, [&](unsigned b) { std::sort(order.begin() + bstart[b], order.begin() + bstart[b + 1], less); });
}

int run_batch(DevDB& db, std::vector<std::vector<Step>> steps, cudaStream_t s, uint64_t budget,
              const uint32_t* vgraph, uint32_t G, uint64_t* counts, uint64_t* graph_counts_host,
              uint32_t* support_host, bool profile, BatchStats* stats, int rounds) {
    (void)vgraph;
    (void)G;
    const auto t0 = std::chrono::steady_clock::now();
    const size_t n = steps.size();
    std::vector<uint32_t> order;
    order_by_step_keys(steps, order);
    const double order_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    // a large batch runs as two contiguous halves of the sorted plans (plans
    // share prefixes within a half), each prepared and run by its own host
    // thread on its own stream: one half's host work (trie, descriptors,
    // rounds' bookkeeping) overlaps the other's kernels, and the two halves'
    // kernels fill each other's gaps on the device
    // (a profiled run keeps one stream: per-kernel event timings of two
    // overlapping streams would each include the other's kernels)
    const size_t K = n >= 12288 && !profile ? 2 : 1;
    // two halves hide each other's host round trips: host scheduling there
    // (no schedule tables or frontier regions per half; the two measure
    // alike), device scheduling for a run in one piece
    const bool host_rounds = rounds == ROUNDS_HOST || (rounds == ROUNDS_AUTO && K == 2);
    std::vector<size_t> cut(K + 1);
    for (size_t k = 0; k <= K; ++k) cut[k] = n * k / K;
    const bool per_graph = graph_counts_host || support_host;
    cudaStream_t streams[2] = {s, s};
    if (K == 2) {
        int rc0 = second_stream(db.device, s, streams[1]);
        if (rc0) return rc0;
    }
    std::vector<BatchStats> bss(K);
    std::vector<int> rcs(K, GVA_OK);
    std::vector<std::string> errs(K);
    auto run_half = [&](size_t k) {
        PreparedBatch pb;
        // this half's plans in sorted order, moved out of the caller's list
        std::vector<std::vector<Step>> part(cut[k + 1] - cut[k]);
        for (size_t j = 0; j < part.size(); ++j) part[j] = std::move(steps[order[cut[k] + j]]);
        int r = prepare_batch(db, std::move(part), streams[k], budget, per_graph, graph_counts_host != nullptr,
                              profile, pb, true, host_rounds);
        const double t_prep = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        // results straight to the caller's arrays, at each plan's index before sorting
        if (!r) r = finish_batch(db, pb, counts, graph_counts_host, support_host, &bss[k], nullptr, order.data() + cut[k]);
        bss[k].timeline_ms[1 + 4 * k] = t_prep;
        bss[k].timeline_ms[2 + 4 * k] = t_prep + bss[k].loop_end_ms;
        bss[k].timeline_ms[3 + 4 * k] = t_prep + bss[k].read_end_ms;
        bss[k].timeline_ms[4 + 4 * k] =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        rcs[k] = r;
        if (r) errs[k] = last_error_cstr();
    };
    {
        std::vector<std::thread> pool;
        for (size_t k = 1; k < K; ++k) pool.emplace_back(run_half, k);
        run_half(0);
        for (auto& th : pool) th.join();
    }
    int rc = GVA_OK;
    for (size_t k = 0; k < K && !rc; ++k)
        if (rcs[k]) rc = fail(rcs[k], errs[k]);
    BatchStats total;
    for (const BatchStats& bs : bss) {
        total.gpu_ms = std::max(total.gpu_ms, bs.gpu_ms);  // the halves overlap
        total.submit_ms += bs.submit_ms;
        total.round_host_ms += bs.round_host_ms;
        total.wait_ms += bs.wait_ms;
        total.session_ms += bs.session_ms;
        total.rounds += bs.rounds;
        total.device_rounds += bs.device_rounds;
        total.splits += bs.splits;
        total.launches += bs.launches;
        total.nodes += bs.nodes;
        for (int i = 0; i < 5; ++i) total.phase_ms[i] += bs.phase_ms[i];
        for (int i = 1; i < 9; ++i) total.timeline_ms[i] += bs.timeline_ms[i];
        for (int i = 0; i < K_NUM; ++i) {
            total.kstat[i].launches += bs.kstat[i].launches;
            total.kstat[i].ms += bs.kstat[i].ms;
            total.kstat[i].bytes += bs.kstat[i].bytes;
            total.kstat[i].rows += bs.kstat[i].rows;
        }
    }
    total.timeline_ms[0] = order_ms;
    if (stats) *stats = total;
    if (rc) return rc;
    if (stats) stats->submit_ms += order_ms;
    return GVA_OK;
}

// Candidate launch shapes: rows per work item x the list length from which a
// row's candidates are shared by its warp (1 << 30: never).  Each shape runs
// the calibration batch twice; the faster run counts.
int autotune_batch(DevDB& db, const std::vector<std::vector<Step>>& steps, cudaStream_t s, bool per_graph,
                   TuneResult& out) {
    out = TuneResult();
    if (steps.empty()) return fail(GVA_ERR_ARG, "empty calibration batch");
    const uint32_t keep_r = db.tune_rows_per_item, keep_h = db.tune_hub;
    const uint32_t rows[] = {32, 64, 128};
    const uint32_t hubs[] = {16, 32, 64, 1u << 30};
    std::vector<uint64_t> counts(steps.size()), first_counts;
    std::vector<uint32_t> sup(per_graph ? steps.size() : 0);
    double best = 1e300;
    int rc = GVA_OK;
    for (uint32_t r : rows) {
        for (uint32_t hb : hubs) {
            db.tune_rows_per_item = r;
            db.tune_hub = hb;
            double t = 1e300;
            for (int rep = 0; rep < 2 && !rc; ++rep) {
                BatchStats bs;
                rc = run_batch(db, steps, s, 0, nullptr, 0, counts.data(), nullptr, per_graph ? sup.data() : nullptr,
                               false, &bs);
                t = std::min(t, bs.gpu_ms);
            }
            if (rc) break;
            if (first_counts.empty()) {
                first_counts = counts;
            } else if (counts != first_counts) {  // every shape counts the same rows
                rc = fail(GVA_ERR_CUDA, "launch shapes disagree on the calibration counts");
                break;
            }
            out.tried.push_back({(double)r, (double)hb, t});
            if (r == 64 && hb == 32) out.default_ms = t;
            if (t < best) {
                best = t;
                out.rows_per_item = r;
                out.hub = hb;
            }
        }
        if (rc) break;
    }
    if (rc) {
        db.tune_rows_per_item = keep_r;
        db.tune_hub = keep_h;
        return rc;
    }
    out.ms = best;
    db.tune_rows_per_item = out.rows_per_item;
    db.tune_hub = out.hub;
    return GVA_OK;
}

int set_graph_ids(DevDB& db, const uint64_t* first, uint32_t num_graphs) {
    if (!first || num_graphs == 0) return fail(GVA_ERR_ARG, "graph boundaries missing");
    std::vector<uint32_t> vg(db.max_id + 1, 0xffffffffu);
    for (uint32_t g = 0; g < num_graphs; ++g) {
        if (first[g] > first[g + 1] || first[g + 1] > (uint64_t)db.max_id + 1)
            return fail(GVA_ERR_ARG, "graph boundaries must be ascending within 1..max_vertex_id+1");
        for (uint64_t v = first[g]; v < first[g + 1]; ++v) vg[v] = g;
    }
    GVA_CUDA_B(cudaSetDevice(db.device));
    if (db.vgraph) cudaFree(db.vgraph);
    db.vgraph = nullptr;
    GVA_CUDA_B(cudaMalloc(&db.vgraph, vg.size() * 4));
    GVA_CUDA_B(cudaMemcpy(db.vgraph, vg.data(), vg.size() * 4, cudaMemcpyHostToDevice));
    db.num_graphs = num_graphs;
    return GVA_OK;
}

}  // namespace gva
