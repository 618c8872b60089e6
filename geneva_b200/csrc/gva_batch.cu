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
#include <atomic>
#include <cstring>
#include <memory>
#include <map>
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

__device__ __forceinline__ int find_task(const uint64_t* __restrict__ block0, int ntasks, uint64_t b) {
    int lo = 0, hi = ntasks - 1;  // largest t with block0[t] <= b
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(block0 + mid) <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void load_desc(TaskDesc& dst, const TaskDesc* src) {
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(TaskDesc) / 4); i += blockDim.x) d[i] = s[i];
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
batch_count_kernel(const TaskDesc* __restrict__ tasks, const uint64_t* __restrict__ block0, int ntasks,
                   uint64_t* __restrict__ block_sums, BatchCtx ctx) {
    __shared__ TaskDesc d;
    const uint64_t b = blockIdx.x;
    const int t = find_task(block0, ntasks, b);
    load_desc(d, tasks + t);
    __syncthreads();
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
    store_block_sum(c, block_sums);
}

__global__ void task_totals_kernel(const uint64_t* __restrict__ block0, int ntasks, const uint64_t* __restrict__ sums,
                                   uint64_t* __restrict__ totals) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ntasks) totals[t] = sums[block0[t + 1]] - sums[block0[t]];
}

// Persistent: each CTA repeatedly takes the next 256-row item.
__global__ void __launch_bounds__(kThreads)
batch_write_kernel(const TaskDesc* __restrict__ tasks, const uint64_t* __restrict__ block0, int ntasks, uint64_t nblocks,
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
        const int t = find_task(block0, ntasks, b);
        uint32_t* out = task_out[t];
        if (out == nullptr) {  // task deferred or counted only: nothing to write
            __syncthreads();
            continue;
        }
        load_desc(d, tasks + t);
        if (threadIdx.x == 0) base_s = sums[b] - sums[block0[t]];  // task-local output row of this item
        __syncthreads();
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
            const uint32_t* gadj = nullptr;
            uint32_t lo = 0, hi = 0, cnt = 0;
            int which = -1;
            if (threadIdx.x < nr) {
                ext_generator(p, row, gadj, lo, hi, which);
                for (uint32_t j = lo; j < hi; ++j) cnt += ext_accept(p, row, __ldg(gadj + j), which) ? 1u : 0u;
            }
            uint64_t total;
            const uint64_t before = block_exclusive_scan(cnt, &total);
            if (cnt) {
                uint32_t* dst = out + (out0 + before) * k1;
                for (uint32_t j = lo; j < hi; ++j) {
                    const uint32_t c = __ldg(gadj + j);
                    if (!ext_accept(p, row, c, which)) continue;
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

// Device buffer shared by every task whose frontier slice lives in it.
struct DevBuf {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~DevBuf() {
        if (p) cudaFreeAsync(p, s);
    }
};

// A node of the step trie: the plans of a batch that agree on their first
// steps share those steps' frontiers.
struct Node {
    Step step;
    int depth = 0;
    std::vector<int> children;
    std::vector<int> terminal;  // plans whose last step is this node
};

struct Task {
    int node;
    const uint32_t* in;          // frontier slice
    uint64_t rows;
    std::shared_ptr<DevBuf> owner;
};

// Bytes that determine a step's output from its input (everything but phase_end).
std::string step_key(const Step& st) {
    std::string k;
    auto put = [&](const void* p, size_t n) { k.append((const char*)p, n); };
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
    return k;
}

// Pinned host staging reused across rounds and calls (per thread and device).
struct Staging {
    char* p = nullptr;
    size_t cap = 0;
    char* get(size_t need) {
        if (need > cap) {
            if (p) cudaFreeHost(p);
            cap = std::max(need, cap * 2);
            if (cudaMallocHost((void**)&p, cap) != cudaSuccess) {
                p = nullptr;
                cap = 0;
            }
        }
        return p;
    }
};

}  // namespace

uint64_t batch_kernel_launches() { return g_batch_launches.load(); }

int run_batch(DevDB& db, const std::vector<std::vector<Step>>& steps, cudaStream_t s, uint64_t budget,
              const uint32_t* vgraph, uint32_t G, uint64_t* counts, uint64_t* graph_counts_host,
              uint32_t* support_host, bool profile, BatchStats* stats) {
    GVA_CUDA_B(cudaSetDevice(db.device));
    const int nq = (int)steps.size();
    for (int q = 0; q < nq; ++q) counts[q] = 0;
    if (nq == 0) return GVA_OK;
    if ((graph_counts_host || support_host) && (!vgraph || G == 0))
        return fail(GVA_ERR_ARG, "per-graph results need the database's graph ids (gva_db_set_graphs)");
    if (budget == 0) {
        size_t fr = 0, tot = 0;
        GVA_CUDA_B(cudaMemGetInfo(&fr, &tot));
        budget = (uint64_t)fr / 4 * 3;
    }
    Profiler profiler;
    Profiler* prof = profile ? &profiler : nullptr;
    static thread_local cudaEvent_t tev[64][2];
    const int dev = db.device;
    if (dev < 0 || dev >= 64) return fail(GVA_ERR_ARG, "device index out of range");
    if (!tev[dev][0]) {
        GVA_CUDA_B(cudaEventCreate(&tev[dev][0]));
        GVA_CUDA_B(cudaEventCreate(&tev[dev][1]));
    }
    cudaEvent_t ev0 = tev[dev][0], ev1 = tev[dev][1];
    GVA_CUDA_B(cudaEventRecord(ev0, s));

    // ---- step trie: plans sharing a prefix of steps share its frontiers
    std::vector<Node> nodes;
    std::map<std::string, int> roots;
    std::vector<std::map<std::string, int>> kids;
    for (int q = 0; q < nq; ++q) {
        const std::vector<Step>& st = steps[q];
        if (st.size() < 2 || st[0].kind != STEP_SEED) return fail(GVA_ERR_ARG, "plan must start with a seed step");
        int cur = -1;
        for (size_t i = 0; i < st.size(); ++i) {
            const std::string key = step_key(st[i]);
            auto& m0 = cur < 0 ? roots : kids[cur];
            auto it = m0.find(key);
            int id;
            if (it == m0.end()) {
                id = (int)nodes.size();
                nodes.push_back(Node{st[i], (int)i, {}, {}});
                kids.emplace_back();  // may reallocate: look the parent's map up again
                (cur < 0 ? roots : kids[cur])[key] = id;
                if (cur >= 0) nodes[cur].children.push_back(id);
            } else {
                id = it->second;
            }
            cur = id;
        }
        nodes[cur].terminal.push_back(q);
    }

    // per-graph accumulators: one slot per plan; plans that end on the same
    // node are filled from its first plan at the end
    BatchCtx ctx{};
    ctx.vgraph = vgraph;
    ctx.G = G;
    ctx.words = (G + 31) / 32;
    const bool per_graph = graph_counts_host || support_host;
    void* acc = nullptr;
    if (per_graph) {
        const size_t acc_bytes = (graph_counts_host ? (size_t)nq * G * 8 : 0) + (size_t)nq * ctx.words * 4;
        if (cudaMallocAsync(&acc, acc_bytes, s) != cudaSuccess) return fail(GVA_ERR_NOMEM, "per-graph counters");
        GVA_CUDA_B(cudaMemsetAsync(acc, 0, acc_bytes, s));
        char* a = (char*)acc;
        if (graph_counts_host) {
            ctx.graph_counts = (uint64_t*)a;
            a += (size_t)nq * G * 8;
        }
        ctx.graph_bits = (uint32_t*)a;
    }

    std::vector<Task> active;
    for (auto& kv : roots) {
        const Node& seed = nodes[kv.second];
        if (seed.step.always_empty) continue;
        const uint64_t n = db.seed_off[seed.step.label + 1] - db.seed_off[seed.step.label];
        if (!n) continue;
        for (int c : seed.children) active.push_back({c, db.seed_verts + db.seed_off[seed.step.label], n, nullptr});
    }

    int status = GVA_OK;
    static thread_local Staging staging[64];
    Staging& stg = staging[dev];
    TaskDesc* d_desc = nullptr;
    size_t desc_cap = 0;
    uint64_t* d_sums = nullptr;
    size_t sums_cap = 0;
    uint64_t* d_small = nullptr;  // block0[nt + 1] | totals[nt] | outs[nt] | queue
    size_t small_cap = 0;
    static bool smem_set[64] = {};
    if (!smem_set[dev]) {
        GVA_CUDA_B(cudaFuncSetAttribute(batch_write_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)batch_smem_bytes()));
        smem_set[dev] = true;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);

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

    uint64_t rounds = 0, splits = 0, launches = 0;
    std::vector<uint64_t> block0, totals;
    while (!active.empty() && status == GVA_OK) {
        // steps that cannot match (label or partition absent) end their task
        active.erase(std::remove_if(active.begin(), active.end(),
                                    [&](const Task& t) { return nodes[t.node].step.always_empty != 0; }),
                     active.end());
        if (active.empty()) break;
        ++rounds;
        const int nt = (int)active.size();
        // pinned staging: descs | block0 | totals | outs
        const size_t desc_bytes = (size_t)nt * sizeof(TaskDesc);
        const size_t small_words = (size_t)(nt + 1) + nt + nt + 1;
        char* h = stg.get(desc_bytes + small_words * 8);
        if (!h) {
            status = fail(GVA_ERR_NOMEM, "pinned staging allocation failed");
            break;
        }
        TaskDesc* descs = (TaskDesc*)h;
        uint64_t* h_block0 = (uint64_t*)(h + desc_bytes);
        uint64_t* h_totals = h_block0 + (nt + 1);
        uint32_t** h_outs = (uint32_t**)(h_totals + nt);
        block0.assign(nt + 1, 0);
        uint32_t kmax = 1, eqmax = 0;
        double cbytes = 0;
        for (int t = 0; t < nt; ++t) {
            const Task& tk = active[t];
            const Node& nd = nodes[tk.node];
            const Step& st = nd.step;
            TaskDesc& d = descs[t];
            memset(&d, 0, sizeof d);
            d.kind = st.kind;
            d.mode = MODE_WRITE;
            if (nd.children.empty()) d.mode = MODE_COUNT;
            if (per_graph && !nd.terminal.empty()) {
                d.mode = nd.children.empty() ? MODE_COUNT_GRAPHS : MODE_WRITE_AND_GRAPHS;
                d.query = (uint32_t)nd.terminal[0];
            }
            d.block0 = block0[t];
            const DevPart& P = db.parts[st.part - 1];
            if (st.kind == STEP_EXT) {
                ExtArgs& a = d.e;
                a.in = tk.in;
                a.nrows = tk.rows;
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
                eqmax = std::max(eqmax, st.n_eq);
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
                a.in = tk.in;
                a.nrows = tk.rows;
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
            kmax = std::max(kmax, st.width_in);
            block0[t + 1] = block0[t] + (tk.rows + kRowsPerBlock - 1) / kRowsPerBlock;
            cbytes += (4.0 * st.width_in + 8.0 * (st.kind == STEP_EXT ? 1 : st.n_pairs)) * (double)tk.rows;
        }
        const uint64_t nb = block0[nt];
        if (nb > 0x7fffffffull) {
            status = fail(GVA_ERR_UNSUPPORTED, "round too large for one launch");
            break;
        }
        std::copy(block0.begin(), block0.end(), h_block0);
        if (!grow((void**)&d_desc, desc_cap, desc_bytes) || !grow((void**)&d_sums, sums_cap, (nb + 1) * 8) ||
            !grow((void**)&d_small, small_cap, small_words * 8)) {
            status = fail(GVA_ERR_NOMEM, "batch bookkeeping allocation failed");
            break;
        }
        uint64_t* d_block0 = d_small;
        uint64_t* d_totals = d_block0 + (nt + 1);
        uint32_t** d_outs = (uint32_t**)(d_totals + nt);
        unsigned long long* d_queue = (unsigned long long*)(d_totals + 2 * nt);
        GVA_CUDA_B(cudaMemcpyAsync(d_desc, descs, desc_bytes, cudaMemcpyHostToDevice, s));
        GVA_CUDA_B(cudaMemcpyAsync(d_block0, h_block0, (nt + 1) * 8, cudaMemcpyHostToDevice, s));

        cudaEvent_t ev = nullptr;
        if (prof) prof->begin(K_EXT_COUNT, cbytes, s, ev);
        batch_count_kernel<<<(unsigned)nb, kThreads, 0, s>>>(d_desc, d_block0, nt, d_sums, ctx);
        if (prof) prof->end(ev, K_EXT_COUNT, cbytes, s);
        if (prof) prof->begin(K_SCAN, 16.0 * nb, s, ev);
        scan_block_sums_kernel<<<1, kScanThreads, 0, s>>>(d_sums, nb);
        if (prof) prof->end(ev, K_SCAN, 16.0 * nb, s);
        task_totals_kernel<<<(nt + 255) / 256, 256, 0, s>>>(d_block0, nt, d_sums, d_totals);
        launches += 3;
        GVA_CUDA_B(cudaGetLastError());
        GVA_CUDA_B(cudaMemcpyAsync(h_totals, d_totals, nt * 8, cudaMemcpyDeviceToHost, s));
        GVA_CUDA_B(cudaStreamSynchronize(s));
        totals.assign(h_totals, h_totals + nt);

        // choose which tasks write this round: deepest first, within the budget
        std::vector<int> order;
        std::vector<Task> next;
        for (int t = 0; t < nt; ++t) {
            const Node& nd = nodes[active[t].node];
            for (int q : nd.terminal) counts[q] += totals[t];
            if (!nd.children.empty() && totals[t] > 0) order.push_back(t);
        }
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return nodes[active[a].node].depth > nodes[active[b].node].depth; });
        uint64_t used = 0;
        std::vector<uint64_t> off_words(nt, 0);
        std::vector<int> chosen;
        for (int t : order) {
            const Step& st = nodes[active[t].node].step;
            const uint32_t w = st.kind == STEP_EXT ? st.width_in + 1 : st.width_in;
            const uint64_t bytes = totals[t] * w * 4ull;
            if (used + bytes <= budget) {
                off_words[t] = used / 4;
                used += (bytes + 15) & ~15ull;
                chosen.push_back(t);
            } else if (bytes > budget) {
                // split the task's input rows; both halves retry next round
                Task a = active[t], b = active[t];
                const uint64_t half = a.rows / 2;
                if (half == 0) {
                    status = fail(GVA_ERR_NOMEM, "a single frontier row expands beyond the memory budget");
                    break;
                }
                a.rows = half;
                b.in = a.in + half * st.width_in;
                b.rows = active[t].rows - half;
                next.push_back(a);
                next.push_back(b);
                ++splits;
            } else {
                next.push_back(active[t]);  // fits alone: waits for the next round
            }
        }
        if (status) break;
        std::shared_ptr<DevBuf> buf;
        if (used > 0) {
            buf = std::make_shared<DevBuf>();
            buf->s = s;
            if (cudaMallocAsync(&buf->p, used, s) != cudaSuccess) {
                buf->p = nullptr;
                status = fail(GVA_ERR_NOMEM, "frontier allocation failed");
                break;
            }
            double wbytes = 0;
            for (int t = 0; t < nt; ++t) h_outs[t] = nullptr;
            for (int t : chosen) {
                h_outs[t] = (uint32_t*)buf->p + off_words[t];
                const Step& st = nodes[active[t].node].step;
                const double k = st.width_in;
                wbytes += (4.0 * k + 8.0) * (double)active[t].rows +
                          (st.kind == STEP_EXT ? (4.0 + 4.0 * (k + 1)) : 4.0 * k) * (double)totals[t];
            }
            GVA_CUDA_B(cudaMemcpyAsync(d_outs, h_outs, nt * sizeof(uint32_t*), cudaMemcpyHostToDevice, s));
            GVA_CUDA_B(cudaMemsetAsync(d_queue, 0, 8, s));
            const size_t smem = batch_smem_bytes_for(kmax, std::max(eqmax, 1u));
            int per_sm = 1;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_write_kernel, kThreads, smem);
            const uint64_t grid = std::min<uint64_t>(nb, (uint64_t)std::max(per_sm, 1) * sms);
            if (prof) prof->begin(K_EXT_WRITE, wbytes, s, ev);
            batch_write_kernel<<<(unsigned)grid, kThreads, smem, s>>>(d_desc, d_block0, nt, nb, d_sums, d_outs,
                                                                      d_queue);
            if (prof) prof->end(ev, K_EXT_WRITE, wbytes, s);
            launches += 1;
            GVA_CUDA_B(cudaGetLastError());
        }
        for (int t : chosen)
            for (int c : nodes[active[t].node].children) next.push_back({c, h_outs[t], totals[t], buf});
        active.swap(next);
        if (prof) {
            GVA_CUDA_B(cudaStreamSynchronize(s));
            prof->resolve();
        }
    }
    g_batch_launches += launches;
    active.clear();  // releases frontier buffers (stream-ordered)

    if (status == GVA_OK && per_graph) {
        std::vector<uint32_t> bits((size_t)nq * ctx.words);
        GVA_CUDA_B(cudaMemcpyAsync(bits.data(), ctx.graph_bits, bits.size() * 4, cudaMemcpyDeviceToHost, s));
        if (graph_counts_host)
            GVA_CUDA_B(cudaMemcpyAsync(graph_counts_host, ctx.graph_counts, (size_t)nq * G * 8, cudaMemcpyDeviceToHost, s));
        GVA_CUDA_B(cudaStreamSynchronize(s));
        for (const Node& nd : nodes) {  // identical plans share the first one's results
            for (size_t i = 1; i < nd.terminal.size(); ++i) {
                const int q0 = nd.terminal[0], q = nd.terminal[i];
                std::copy(bits.begin() + (size_t)q0 * ctx.words, bits.begin() + (size_t)(q0 + 1) * ctx.words,
                          bits.begin() + (size_t)q * ctx.words);
                if (graph_counts_host)
                    std::copy(graph_counts_host + (size_t)q0 * G, graph_counts_host + (size_t)(q0 + 1) * G,
                              graph_counts_host + (size_t)q * G);
            }
        }
        if (support_host) {
            for (int q = 0; q < nq; ++q) {
                uint32_t c = 0;
                for (uint32_t w = 0; w < ctx.words; ++w) c += (uint32_t)__builtin_popcount(bits[(size_t)q * ctx.words + w]);
                support_host[q] = c;
            }
        }
    }
    if (acc) cudaFreeAsync(acc, s);
    for (void* p : {(void*)d_desc, (void*)d_sums, (void*)d_small})
        if (p) cudaFreeAsync(p, s);
    cudaEventRecord(ev1, s);
    cudaEventSynchronize(ev1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    if (stats) {
        stats->gpu_ms = ms;
        stats->rounds = rounds;
        stats->splits = splits;
        stats->launches = launches;
        stats->nodes = nodes.size();
        if (prof) {
            prof->resolve();
            for (int i = 0; i < K_NUM; ++i) stats->kstat[i] = prof->stat[i];
        }
    }
    return status;
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
