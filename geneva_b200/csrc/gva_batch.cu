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
#include <vector>

#include "../../include/geneva.h"
#include "gva_engine.cuh"
#include "gva_kernels.cuh"

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

struct TaskDesc {
    uint32_t kind;     // STEP_EXT / STEP_REDUCE
    uint32_t mode;     // TaskMode
    uint32_t query;    // index into the batch
    uint32_t pad;
    uint64_t block0;   // first global block of this task
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

// Per-round task reference: the step parameters live in a per-node
// descriptor uploaded once per submitted wave; a round uploads only these.
struct TaskRef {
    uint32_t node;
    uint32_t pad;
    uint64_t block0;
    const uint32_t* in;
    uint64_t nrows;
};

// Descriptor of task t: its node's parameters patched, while they are copied,
// with the task's frontier slice (ExtArgs and RedArgs both start with `in`,
// `nrows`), so one barrier makes the copy visible.
__device__ __forceinline__ void load_task(TaskDesc& d, const TaskDesc* __restrict__ nodes,
                                          const TaskRef* __restrict__ refs, int t) {
    constexpr int kB0 = (int)(offsetof(TaskDesc, block0) / 4);
    constexpr int kIn = (int)((offsetof(TaskDesc, e) + offsetof(ExtArgs, in)) / 4);
    constexpr int kNr = (int)((offsetof(TaskDesc, e) + offsetof(ExtArgs, nrows)) / 4);
    static_assert(offsetof(ExtArgs, in) == offsetof(RedArgs, in) && offsetof(ExtArgs, nrows) == offsetof(RedArgs, nrows),
                  "extension and reduction arguments share their frontier fields");
    const TaskRef r = refs[t];
    const uint32_t* s = reinterpret_cast<const uint32_t*>(nodes + r.node);
    uint32_t* dw = reinterpret_cast<uint32_t*>(&d);
    const uint64_t in = (uint64_t)r.in;
    for (int i = threadIdx.x; i < (int)(sizeof(TaskDesc) / 4); i += blockDim.x) {
        uint32_t v;
        if (i == kB0 || i == kB0 + 1)
            v = (uint32_t)(r.block0 >> (32 * (i - kB0)));
        else if (i == kIn || i == kIn + 1)
            v = (uint32_t)(in >> (32 * (i - kIn)));
        else if (i == kNr || i == kNr + 1)
            v = (uint32_t)(r.nrows >> (32 * (i - kNr)));
        else
            v = __ldg(s + i);
        dw[i] = v;
    }
    __syncthreads();
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

__global__ void __launch_bounds__(kThreads)
batch_count_kernel(const TaskDesc* __restrict__ nodes, const TaskRef* __restrict__ refs,
                   const uint32_t* __restrict__ blk_task, uint64_t* __restrict__ block_sums, BatchCtx ctx) {
    __shared__ TaskDesc d;
    const uint64_t b = blockIdx.x;
    const int t = (int)__ldg(blk_task + b);
    load_task(d, nodes, refs, t);
    const uint64_t r = (b - d.block0) * kRowsPerBlock + threadIdx.x;
    uint32_t c = 0;
    uint32_t first = 0;
    bool valid = false;
    if (d.kind == STEP_EXT) {
        valid = r < d.e.nrows;
        if (valid) {
            const uint32_t* row = d.e.in + r * d.e.k;
            c = ext_count_row(d.e, row);
            first = row[0];
        }
    } else {
        valid = r < d.r.nrows;
        if (valid) {
            const uint32_t* row = d.r.in + r * d.r.k;
            c = red_keep_row(d.r, row) ? 1u : 0u;
            first = row[0];
        }
    }
    if (d.mode == MODE_COUNT_GRAPHS || d.mode == MODE_WRITE_AND_GRAPHS) add_graph_count(ctx, d.query, first, c, valid);
    // block total without a barrier: each warp adds its share (sums zeroed before the launch)
    const uint64_t ws = warp_sum((uint64_t)c);
    if ((threadIdx.x & 31) == 0 && ws) atomicAdd((unsigned long long*)(block_sums + b), (unsigned long long)ws);
}

__global__ void task_totals_kernel(const uint64_t* __restrict__ block0, int ntasks, const uint64_t* __restrict__ sums,
                                   uint64_t* __restrict__ totals) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ntasks) totals[t] = sums[block0[t + 1]] - sums[block0[t]];
}

// Persistent: each CTA repeatedly takes the next 256-row item.
__global__ void __launch_bounds__(kThreads)
batch_write_kernel(const TaskDesc* __restrict__ nodes, const TaskRef* __restrict__ refs,
                   const uint64_t* __restrict__ block0, const uint32_t* __restrict__ blk_task, uint64_t nblocks,
                   const uint64_t* __restrict__ sums, uint32_t* __restrict__ const* __restrict__ task_out,
                   unsigned long long* __restrict__ queue) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ TaskDesc d;
    __shared__ unsigned long long item_s;
    __shared__ uint64_t base_s;
    for (;;) {
        if (threadIdx.x == 0) item_s = atomicAdd(queue, 1ull);
        __syncthreads();
        const uint64_t b = item_s;
        if (b >= nblocks) return;
        const int t = (int)__ldg(blk_task + b);
        uint32_t* out = task_out[t];
        if (out == nullptr) {  // task deferred or counted only: nothing to write
            __syncthreads();
            continue;
        }
        if (threadIdx.x == 0) base_s = sums[b] - sums[block0[t]];  // task-local output row of this item
        load_task(d, nodes, refs, t);
        const uint64_t row0 = (b - d.block0) * kRowsPerBlock;
        const uint64_t out0 = base_s;
        if (d.kind == STEP_EXT && d.e.n_chk) {
            // fused back-edge checks: each thread walks its row's generator
            // segment twice (count, then write) and stores survivors directly
            const ExtArgs& p = d.e;
            const uint32_t k = p.k, k1 = p.k + 1;
            uint32_t* rows_s = reinterpret_cast<uint32_t*>(smem_raw);
            const uint32_t nr = (uint32_t)umin64((uint64_t)kRowsPerBlock, p.nrows - row0);
            const uint32_t* gin = p.in + row0 * k;
            for (uint32_t w = threadIdx.x; w < nr * k; w += kThreads) rows_s[w] = gin[w];
            __syncthreads();
            const uint32_t* row = rows_s + threadIdx.x * k;
            GenState g;
            g.lo = g.hi = 0;
            uint32_t cnt = 0, acc = 0;  // acc: verdicts of the first 32 candidates
            if (threadIdx.x < nr) {
                ext_generator(p, row, g);
                for (uint32_t j = g.lo; j < g.hi; ++j) {
                    const bool ok = ext_accept(p, row, __ldg(g.gadj + j), g);
                    cnt += ok ? 1u : 0u;
                    if (ok && j - g.lo < 32) acc |= 1u << (j - g.lo);
                }
            }
            uint64_t total;
            const uint64_t before = block_exclusive_scan(cnt, &total);
            if (cnt) {
                uint32_t* dst = out + (out0 + before) * k1;
                for (uint32_t j = g.lo; j < g.hi; ++j) {
                    const bool early = j - g.lo < 32;
                    if (early && !(acc >> (j - g.lo) & 1)) continue;
                    const uint32_t c = __ldg(g.gadj + j);
                    if (!early && !ext_accept(p, row, c, g)) continue;
                    for (uint32_t q = 0; q < k; ++q) dst[q] = row[q];
                    dst[k] = c;
                    dst += k1;
                }
            }
            __syncthreads();
        } else if (d.kind == STEP_EXT) {
            const ExtArgs& p = d.e;
            const uint32_t k = p.k, k1 = p.k + 1;
            uint64_t* offs_s = reinterpret_cast<uint64_t*>(smem_raw);
            uint32_t* rows_s = reinterpret_cast<uint32_t*>(offs_s + kRowsPerBlock + 1);
            uint32_t* lo_s = rows_s + kRowsPerBlock * k;
            uint32_t* ncol_s = lo_s + kRowsPerBlock;
            uint32_t* coll_s = ncol_s + kRowsPerBlock;
            uint32_t* out_s = coll_s + kRowsPerBlock * p.n_eq;
            const uint32_t nr = (uint32_t)umin64((uint64_t)kRowsPerBlock, p.nrows - row0);
            const uint32_t* gin = p.in + row0 * k;
            for (uint32_t w = threadIdx.x; w < nr * k; w += kThreads) rows_s[w] = gin[w];
            __syncthreads();
            uint64_t cnt = 0;
            if (threadIdx.x < nr) {
                const uint32_t* row = rows_s + threadIdx.x * k;
                uint32_t lo, hi;
                ext_range(p, row, lo, hi);
                uint32_t nc = 0;
                uint32_t* mine = coll_s + threadIdx.x * p.n_eq;
                if (lo < hi) {
                    for (uint32_t j = 0; j < p.n_eq; ++j) {
                        const uint32_t pos = find_in(p.adj, lo, hi, row[p.eq_cols[j]]);
                        if (pos == 0xffffffffu) continue;
                        bool dup = false;
                        for (uint32_t i = 0; i < nc; ++i) dup |= (mine[i] == pos);
                        if (dup) continue;
                        uint32_t i = nc++;
                        while (i > 0 && mine[i - 1] > pos) {
                            mine[i] = mine[i - 1];
                            --i;
                        }
                        mine[i] = pos;
                    }
                    cnt = hi - lo - nc;
                }
                lo_s[threadIdx.x] = lo;
                ncol_s[threadIdx.x] = nc;
            }
            uint64_t total;
            const uint64_t before = block_exclusive_scan(cnt, &total);
            offs_s[threadIdx.x] = before;
            if (threadIdx.x == 0) offs_s[nr] = total;
            __syncthreads();
            for (uint64_t base = 0; base < total; base += kThreads) {
                const uint64_t o = base + threadIdx.x;
                if (o < total) {
                    int a = 0, z = (int)nr - 1;
                    while (a < z) {
                        const int m = (a + z + 1) >> 1;
                        if (offs_s[m] <= o)
                            a = m;
                        else
                            z = m - 1;
                    }
                    uint32_t j = lo_s[a] + (uint32_t)(o - offs_s[a]);
                    const uint32_t* mine = coll_s + a * p.n_eq;
                    for (uint32_t c = 0; c < ncol_s[a]; ++c) j += (mine[c] <= j) ? 1u : 0u;
                    uint32_t* dst = out_s + threadIdx.x * k1;
                    const uint32_t* src = rows_s + a * k;
                    for (uint32_t c = 0; c < k; ++c) dst[c] = src[c];
                    dst[k] = __ldg(p.adj + j);
                }
                __syncthreads();
                const uint32_t n_tile = (uint32_t)umin64((uint64_t)kThreads, total - base);
                uint32_t* gout = out + (out0 + base) * k1;
                for (uint32_t w = threadIdx.x; w < n_tile * k1; w += kThreads) gout[w] = out_s[w];
                __syncthreads();
            }
        } else {
            const RedArgs& p = d.r;
            const uint32_t k = p.k;
            uint32_t* rows_s = reinterpret_cast<uint32_t*>(smem_raw);
            uint32_t* out_s = rows_s + kRowsPerBlock * k;
            const uint32_t nr = (uint32_t)umin64((uint64_t)kRowsPerBlock, p.nrows - row0);
            const uint32_t* gin = p.in + row0 * k;
            for (uint32_t w = threadIdx.x; w < nr * k; w += kThreads) rows_s[w] = gin[w];
            __syncthreads();
            bool keep = false;
            if (threadIdx.x < nr) keep = red_keep_row(p, rows_s + threadIdx.x * k);
            uint64_t total;
            const uint64_t before = block_exclusive_scan(keep ? 1 : 0, &total);
            if (keep)
                for (uint32_t c = 0; c < k; ++c) out_s[before * k + c] = rows_s[threadIdx.x * k + c];
            __syncthreads();
            uint32_t* gout = out + out0 * k;
            for (uint32_t w = threadIdx.x; w < (uint32_t)total * k; w += kThreads) gout[w] = out_s[w];
            __syncthreads();
        }
    }
}

size_t batch_smem_bytes() {
    // the larger of the extension layout at k = 31, n_eq = 32 and the reduction layout at k = 32
    const size_t ext = sizeof(uint64_t) * (kRowsPerBlock + 1) +
                       sizeof(uint32_t) * ((size_t)kRowsPerBlock * 31 + 2 * kRowsPerBlock + (size_t)kRowsPerBlock * 32 +
                                           (size_t)kRowsPerBlock * 32);
    const size_t red = sizeof(uint32_t) * 2 * (size_t)kRowsPerBlock * 32;
    return std::max(ext, red);
}

size_t batch_smem_bytes_for(uint32_t kmax, uint32_t eqmax) {
    const size_t ext = sizeof(uint64_t) * (kRowsPerBlock + 1) +
                       sizeof(uint32_t) * ((size_t)kRowsPerBlock * kmax + 2 * kRowsPerBlock +
                                           (size_t)kRowsPerBlock * eqmax + (size_t)kRowsPerBlock * (kmax + 1));
    const size_t red = sizeof(uint32_t) * 2 * (size_t)kRowsPerBlock * (kmax + 1);
    return std::max(ext, red);
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
BatchSession::BatchSession(DevDB& db_, cudaStream_t s_, uint64_t budget_, uint32_t slots_, bool graph_counts_,
                           bool profile_)
    : db(db_), s(s_), budget(budget_), nslots(slots_), want_graph_counts(graph_counts_), profile(profile_) {}

BatchSession::~BatchSession() {
    cudaSetDevice(db.device);
    active.clear();
    if (staged) cudaEventDestroy(staged);
    for (void* p : {(void*)d_desc, (void*)d_sums, (void*)d_small, (void*)d_blk, acc, d_nodes})
        if (p) cudaFreeAsync(p, s);
    cudaStreamSynchronize(s);
}

int BatchSession::init() {
    GVA_CUDA_B(cudaSetDevice(db.device));
    if (budget == 0) {
        size_t fr = 0, tot = 0;
        GVA_CUDA_B(cudaMemGetInfo(&fr, &tot));
        budget = (uint64_t)fr / 4 * 3;
    }
    per_graph = nslots > 0;
    if (per_graph) {
        if (!db.vgraph || db.num_graphs == 0)
            return fail(GVA_ERR_ARG, "per-graph results need the database's graph ids (gva_db_set_graphs)");
        ctx_words = (db.num_graphs + 31) / 32;
        const size_t bytes = (want_graph_counts ? (size_t)nslots * db.num_graphs * 8 : 0) + (size_t)nslots * ctx_words * 4;
        if (cudaMallocAsync(&acc, bytes, s) != cudaSuccess) return fail(GVA_ERR_NOMEM, "per-graph counters");
        GVA_CUDA_B(cudaMemsetAsync(acc, 0, bytes, s));
        for (uint32_t i = nslots; i > 0; --i) free_slots.push_back((int)i - 1);
    }
    int dev = db.device;
    static std::atomic<bool> smem_set[64];  // sessions may start on several threads (server, miner)
    if (dev < 0 || dev >= 64) return fail(GVA_ERR_ARG, "device index out of range");
    if (!smem_set[dev].load(std::memory_order_acquire)) {
        GVA_CUDA_B(cudaFuncSetAttribute(batch_write_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)batch_smem_bytes()));
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

void BatchSession::fill_node_desc(int id, void* out) const {
    const BNode& nd = nodes[id];
    TaskDesc& d = *reinterpret_cast<TaskDesc*>(out);
    memset(&d, 0, sizeof d);
    const Step& st = node_steps[id];
    d.kind = st.kind;
    d.mode = nd.first_child < 0 ? MODE_COUNT : MODE_WRITE;
    if (per_graph && nd.first_term >= 0) {
        d.mode = nd.first_child < 0 ? MODE_COUNT_GRAPHS : MODE_WRITE_AND_GRAPHS;
        d.query = (uint32_t)plans[nd.first_term].slot;
    }
    if (st.kind == STEP_SEED || st.always_empty || st.part == 0) return;
    const DevPart& P = db.parts[st.part - 1];
    if (st.kind == STEP_EXT) {
        ExtArgs& a = d.e;
        a.off = P.off;
        a.adj = P.adj;
        a.k = st.width_in;
        a.L = db.L;
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
            a.chk_off[i] = db.parts[st.chk_part[i] - 1].off;
            a.chk_adj[i] = db.parts[st.chk_part[i] - 1].adj;
        }
    } else {
        RedArgs& a = d.r;
        a.off = P.off;
        a.adj = P.adj;
        a.k = st.width_in;
        a.L = db.L;
        a.n_pairs = st.n_pairs;
        for (uint32_t i = 0; i < st.n_pairs; ++i) {
            a.rs[i] = st.rs_col[i];
            a.re[i] = st.re_col[i];
            a.rl[i] = st.re_label[i];
        }
    }
}

int BatchSession::submit(const std::vector<std::vector<Step>>& steps, const std::vector<uint64_t>& tags,
                         std::vector<int>* ids, bool presorted) {
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
    std::unordered_multimap<uint64_t, int> index;
    if (!presorted) index.reserve(steps.size() * 4);
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
        nd.depth = depth;
        node_steps.push_back(st);
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
            int id = -1;
            auto range = index.equal_range(h);
            for (auto it = range.first; it != range.second && id < 0; ++it) {
                const BNode& cand = nodes[it->second];
                if (cand.parent != cur) continue;
                if (step_key_bytes(node_steps[it->second], kb2) == n && memcmp(kb, kb2, n) == 0) id = it->second;
            }
            if (id < 0) {
                id = new_node(st[i], cur, (int)i);
                index.emplace(h, id);
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
    // seeds: the children of every seed node start from its vertex list
    for (int id = first_node; id < (int)nodes.size(); ++id) {
        if (nodes[id].parent != -1) continue;
        const Step& sd = node_steps[id];
        uint64_t n = 0;
        if (!sd.always_empty) n = db.seed_off[sd.label + 1] - db.seed_off[sd.label];
        if (n)
            for (int c = nodes[id].first_child; c >= 0; c = nodes[c].next_sibling)
                add_task(c, db.seed_verts + db.seed_off[sd.label], n, nullptr);
        try_close(id);
    }
    return GVA_OK;
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
    // staging: refs[nt] | new node descriptors (<= nt) | block0[nt+1] | totals[nt] | outs[nt] + queue
    const size_t ref_bytes = (size_t)nt * sizeof(TaskRef);
    const size_t desc_max = (size_t)nt * sizeof(TaskDesc);
    const size_t small_words = (size_t)(nt + 1) + nt + nt + 1;
    char* h = staging.get(ref_bytes + desc_max + small_words * 8);
    if (!h) return fail(GVA_ERR_NOMEM, "pinned staging allocation failed");
    TaskRef* refs = (TaskRef*)h;
    char* new_desc = h + ref_bytes;
    uint64_t* h_block0 = (uint64_t*)(h + ref_bytes + desc_max);
    uint64_t* h_totals = h_block0 + (nt + 1);
    uint32_t** h_outs = (uint32_t**)(h_totals + nt);
    const int dev_first = dev_count;
    uint32_t kmax = 1, eqmax = 0;
    double cbytes = 0, crows = 0;
    uint64_t nb = 0;
    h_block0[0] = 0;
    for (int t = 0; t < nt; ++t) {
        const BTask& tk = active[t];
        BNode& nd = nodes[tk.node];
        if (nd.dev < 0) {  // first task of this node: ship its parameters
            nd.dev = dev_count++;
            fill_node_desc(tk.node, new_desc + (size_t)(nd.dev - dev_first) * sizeof(TaskDesc));
        }
        const BNode& st = nd;
        refs[t] = TaskRef{(uint32_t)nd.dev, 0u, nb, tk.in, tk.rows};
        kmax = std::max(kmax, st.width_in);
        if (st.kind == STEP_EXT) eqmax = std::max(eqmax, st.n_eq);
        nb += (tk.rows + kRowsPerBlock - 1) / kRowsPerBlock;
        h_block0[t + 1] = nb;
        cbytes += (4.0 * st.width_in + 8.0 * (st.kind == STEP_EXT ? 1 : st.n_pairs)) * (double)tk.rows;
        crows += (double)tk.rows;
    }
    if (nb > 0x7fffffffull) return fail(GVA_ERR_UNSUPPORTED, "round too large for one launch");
    // block -> task, so that no block searches block0
    uint32_t* h_blk = (uint32_t*)staging_blk.get(nb * 4);
    if (!h_blk) return fail(GVA_ERR_NOMEM, "pinned staging allocation failed");
    for (int t = 0; t < nt; ++t)
        for (uint64_t b = h_block0[t]; b < h_block0[t + 1]; ++b) h_blk[b] = (uint32_t)t;
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
    const size_t dev_need = (size_t)dev_count * sizeof(TaskDesc);
    if (dev_need > node_cap) {  // keep the descriptors already shipped
        void* p = nullptr;
        const size_t cap = std::max(dev_need, node_cap * 2);
        if (cudaMallocAsync(&p, cap, s) != cudaSuccess) return fail(GVA_ERR_NOMEM, "node descriptor allocation failed");
        if (d_nodes && dev_first > 0)
            GVA_CUDA_B(cudaMemcpyAsync(p, d_nodes, (size_t)dev_first * sizeof(TaskDesc), cudaMemcpyDeviceToDevice, s));
        if (d_nodes) cudaFreeAsync(d_nodes, s);
        d_nodes = p;
        node_cap = cap;
    }
    if (!grow(&d_desc, desc_cap, ref_bytes) || !grow((void**)&d_sums, sums_cap, (nb + 1) * 8) ||
        !grow((void**)&d_small, small_cap, small_words * 8) || !grow((void**)&d_blk, blk_cap, nb * 4))
        return fail(GVA_ERR_NOMEM, "batch bookkeeping allocation failed");
    uint64_t* d_block0 = d_small;
    uint64_t* d_totals = d_block0 + (nt + 1);
    uint32_t** d_outs = (uint32_t**)(d_totals + nt);
    unsigned long long* d_queue = (unsigned long long*)(d_totals + 2 * nt);
    if (dev_count > dev_first)
        GVA_CUDA_B(cudaMemcpyAsync((char*)d_nodes + (size_t)dev_first * sizeof(TaskDesc), new_desc,
                                   (size_t)(dev_count - dev_first) * sizeof(TaskDesc), cudaMemcpyHostToDevice, s));
    GVA_CUDA_B(cudaMemcpyAsync(d_desc, refs, ref_bytes, cudaMemcpyHostToDevice, s));
    GVA_CUDA_B(cudaMemcpyAsync(d_block0, h_block0, (nt + 1) * 8, cudaMemcpyHostToDevice, s));
    GVA_CUDA_B(cudaMemcpyAsync(d_blk, h_blk, nb * 4, cudaMemcpyHostToDevice, s));

    GVA_CUDA_B(cudaMemsetAsync(d_sums, 0, (nb + 1) * 8, s));
    lap(0);
    cudaEvent_t ev = nullptr;
    if (pf) pf->begin(K_EXT_COUNT, cbytes, s, ev);
    batch_count_kernel<<<(unsigned)nb, kThreads, 0, s>>>((const TaskDesc*)d_nodes, (const TaskRef*)d_desc, d_blk,
                                                         d_sums, ctx);
    if (pf) pf->end(ev, K_EXT_COUNT, cbytes, s, crows);
    if (pf) pf->begin(K_SCAN, 16.0 * nb, s, ev);
    scan_block_sums_kernel<<<1, kScanThreads, 0, s>>>(d_sums, nb);
    if (pf) pf->end(ev, K_SCAN, 16.0 * nb, s, (double)nb);
    task_totals_kernel<<<(nt + 255) / 256, 256, 0, s>>>(d_block0, nt, d_sums, d_totals);
    launches += 3;
    g_batch_launches += 3;
    GVA_CUDA_B(cudaGetLastError());
    GVA_CUDA_B(cudaMemcpyAsync(h_totals, d_totals, nt * 8, cudaMemcpyDeviceToHost, s));
    lap(1);
    {
        const auto w0 = std::chrono::steady_clock::now();
        cudaError_t e = cudaStreamSynchronize(s);
        wait_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
        if (e != cudaSuccess) return fail(GVA_ERR_CUDA, cudaGetErrorString(e));
        t_lap = std::chrono::steady_clock::now();
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
        for (int t = 0; t < nt; ++t) {
            h_outs[t] = chosen_flag[t] == 1 ? (uint32_t*)p + off_words[t] : nullptr;
            if (chosen_flag[t] != 1) continue;
            wrows += (double)active[t].rows;
            const BNode& st = nodes[active[t].node];
            const double k = st.width_in;
            wbytes += (4.0 * k + 8.0) * (double)active[t].rows +
                      (st.kind == STEP_EXT ? (4.0 + 4.0 * (k + 1)) : 4.0 * k) * (double)h_totals[t];
        }
        GVA_CUDA_B(cudaMemcpyAsync(d_outs, h_outs, nt * sizeof(uint32_t*), cudaMemcpyHostToDevice, s));
        GVA_CUDA_B(cudaEventRecord(staged, s));  // the last read of the staging area this round
        GVA_CUDA_B(cudaMemsetAsync(d_queue, 0, 8, s));
        const size_t smem = batch_smem_bytes_for(kmax, std::max(eqmax, 1u));
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_write_kernel, kThreads, smem);
        const uint64_t grid = std::min<uint64_t>(nb, (uint64_t)std::max(per_sm, 1) * sms);
        if (pf) pf->begin(K_EXT_WRITE, wbytes, s, ev);
        batch_write_kernel<<<(unsigned)grid, kThreads, smem, s>>>((const TaskDesc*)d_nodes, (const TaskRef*)d_desc,
                                                                  d_block0, d_blk, nb, d_sums, d_outs, d_queue);
        if (pf) pf->end(ev, K_EXT_WRITE, wbytes, s, wrows);
        launches += 1;
        g_batch_launches += 1;
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

int prepare_batch(DevDB& db, const std::vector<std::vector<Step>>& steps, cudaStream_t s, uint64_t budget,
                  bool per_graph, bool graph_counts, bool profile, PreparedBatch& out, bool presorted) {
    const auto t0 = std::chrono::steady_clock::now();
    GVA_CUDA_B(cudaSetDevice(db.device));
    out.nq = (int)steps.size();
    out.per_graph = per_graph;
    out.graph_counts = graph_counts;
    out.ids.clear();
    if (out.nq == 0) return GVA_OK;
    out.ses.reset(new BatchSession(db, s, budget, per_graph ? (uint32_t)out.nq : 0, graph_counts, profile));
    int rc = out.ses->init();
    if (!rc) rc = out.ses->submit(steps, {}, &out.ids, presorted);
    out.prep_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

int finish_batch(DevDB& db, PreparedBatch& pb, uint64_t* counts, uint64_t* graph_counts_host, uint32_t* support_host,
                 BatchStats* stats, const volatile int* cancel) {
    const int nq = pb.nq;
    for (int q = 0; q < nq; ++q) counts[q] = 0;
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
    while (!rc && !ses.idle()) {
        if (cancel && *cancel) {
            rc = fail(GVA_ERR_CANCELLED, "cancelled");
            break;
        }
        rc = ses.round();
    }
    const double loop_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_loop0).count();
    const std::vector<int>& ids = pb.ids;
    if (!rc) {
        for (int q = 0; q < nq; ++q) counts[q] = ses.plan(ids[q]).count;
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
            if (!rc && graph_counts_host)
                cudaMemcpyAsync(graph_counts_host, ses.graph_counts_dev(), (size_t)nq * db.num_graphs * 8,
                                cudaMemcpyDeviceToHost, s);
            if (!rc)
                rc = cudaStreamSynchronize(s) == cudaSuccess ? GVA_OK : fail(GVA_ERR_CUDA, "result read-back failed");
            for (int q = 0; q < nq && !rc; ++q) {
                const int sl = ses.plan(ses.first_peer(ids[q])).slot, own = ses.plan(ids[q]).slot;
                if (support_host) support_host[q] = pop[sl];
                if (graph_counts_host && sl != own)
                    std::copy(graph_counts_host + (size_t)sl * db.num_graphs,
                              graph_counts_host + (size_t)(sl + 1) * db.num_graphs,
                              graph_counts_host + (size_t)own * db.num_graphs);
            }
        }
    }
    if (stats) {
        stats->submit_ms = ses.submit_ms;
        stats->round_host_ms = ses.round_host_ms;
        stats->wait_ms = ses.wait_ms;
        stats->rounds = ses.rounds;
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

int run_batch(DevDB& db, const std::vector<std::vector<Step>>& steps, cudaStream_t s, uint64_t budget,
              const uint32_t* vgraph, uint32_t G, uint64_t* counts, uint64_t* graph_counts_host,
              uint32_t* support_host, bool profile, BatchStats* stats) {
    (void)vgraph;
    (void)G;
    PreparedBatch pb;
    int rc = prepare_batch(db, steps, s, budget, graph_counts_host || support_host, graph_counts_host != nullptr,
                           profile, pb);
    if (rc) return rc;
    return finish_batch(db, pb, counts, graph_counts_host, support_host, stats);
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
