// CUDA engine for sm_100a: device database, phase kernels, phase executor.
//
// Frontiers are row-major uint32 tables (one column per matched query
// vertex).  Every extension or reduction runs as
//   count  (thread per row)            -> per-256-row block totals
//   scan   (one block)                 -> exclusive block offsets + total
//   write  (block per 256 rows)        -> rows staged in shared memory,
//                                         outputs balanced across the block,
//                                         flushed with coalesced stores
// so the output size is known before it is written (no device-side overflow
// protocol, unlike src/miningPattern.cu:3325-3343) and output order is
// deterministic (input-row order, candidates ascending).
//
// Label segments come from a dense (vertex, label) offset table, one load per
// lookup, replacing the warp bisection with vLabel gathers of the reference
// (FIND_LABEL_LIMIT, include/common.h:18-66).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/geneva.h"
#include "gva_engine.cuh"
#include "gva_kernels.cuh"

namespace gva {

namespace {

#define GVA_CUDA(call)                                                                                  \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return fail(GVA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));              \
    } while (0)

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// ---------------------------------------------------------------- kernels ---
__global__ void __launch_bounds__(kThreads) ext_count_kernel(ExtArgs p, uint64_t* __restrict__ block_sums) {
    const uint64_t r = (uint64_t)blockIdx.x * kRowsPerBlock + threadIdx.x;
    uint64_t c = 0;
    if (r < p.nrows) c = ext_count_row(p, p.in + r * p.k);
    store_block_sum(c, block_sums);
}

__global__ void __launch_bounds__(kThreads) red_count_kernel(RedArgs p, uint64_t* __restrict__ block_sums) {
    const uint64_t r = (uint64_t)blockIdx.x * kRowsPerBlock + threadIdx.x;
    uint64_t c = 0;
    if (r < p.nrows) c = red_keep_row(p, p.in + r * p.k) ? 1 : 0;
    store_block_sum(c, block_sums);
}

// Block b expands rows [256b, 256b + 256): every thread produces one output
// row per tile, so a block's work is balanced however the candidates are
// spread over its rows.
__global__ void __launch_bounds__(kThreads) ext_write_kernel(ExtArgs p, const uint64_t* __restrict__ block_off) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* offs_s = reinterpret_cast<uint64_t*>(smem_raw);           // 257
    uint32_t* rows_s = reinterpret_cast<uint32_t*>(offs_s + kRowsPerBlock + 1);  // 256 * k
    uint32_t* lo_s = rows_s + kRowsPerBlock * p.k;                        // 256
    uint32_t* ncol_s = lo_s + kRowsPerBlock;                              // 256
    uint32_t* coll_s = ncol_s + kRowsPerBlock;                            // 256 * n_eq
    uint32_t* out_s = coll_s + kRowsPerBlock * p.n_eq;                    // 256 * (k + 1)

    const uint64_t row0 = (uint64_t)blockIdx.x * kRowsPerBlock;
    const uint32_t nr = (uint32_t)umin64((uint64_t)kRowsPerBlock, p.nrows - row0);
    const uint32_t k = p.k, k1 = p.k + 1;

    // coalesced load of this block's rows
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
                uint32_t i = nc++;  // insertion sort, ascending
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

    const uint64_t out0 = block_off[blockIdx.x];
    for (uint64_t base = 0; base < total; base += kThreads) {
        const uint64_t o = base + threadIdx.x;
        if (o < total) {
            // largest r with offs_s[r] <= o; rows with no candidate are skipped
            int a = 0, b = (int)nr - 1;
            while (a < b) {
                const int m = (a + b + 1) >> 1;
                if (offs_s[m] <= o)
                    a = m;
                else
                    b = m - 1;
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
        uint32_t* gout = p.out + (out0 + base) * k1;
        for (uint32_t w = threadIdx.x; w < n_tile * k1; w += kThreads) gout[w] = out_s[w];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads) red_write_kernel(RedArgs p, const uint64_t* __restrict__ block_off) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* rows_s = reinterpret_cast<uint32_t*>(smem_raw);  // 256 * k (compacted in a second buffer)
    uint32_t* out_s = rows_s + kRowsPerBlock * p.k;
    const uint64_t row0 = (uint64_t)blockIdx.x * kRowsPerBlock;
    const uint32_t nr = (uint32_t)umin64((uint64_t)kRowsPerBlock, p.nrows - row0);
    const uint32_t k = p.k;
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
    uint32_t* gout = p.out + block_off[blockIdx.x] * k;
    for (uint32_t w = threadIdx.x; w < (uint32_t)total * k; w += kThreads) gout[w] = out_s[w];
}

size_t ext_smem_bytes(uint32_t k, uint32_t n_eq) {
    return sizeof(uint64_t) * (kRowsPerBlock + 1) +
           sizeof(uint32_t) * ((size_t)kRowsPerBlock * k + 2 * kRowsPerBlock + (size_t)kRowsPerBlock * n_eq +
                               (size_t)kRowsPerBlock * (k + 1));
}
size_t red_smem_bytes(uint32_t k) { return sizeof(uint32_t) * 2 * (size_t)kRowsPerBlock * k; }

std::atomic<uint64_t> g_launches{0};

int set_smem_limits() {
    static std::atomic<bool> done[64];  // callers may run on several threads
    int dev = 0;
    GVA_CUDA(cudaGetDevice(&dev));
    if (dev < 64 && done[dev].load(std::memory_order_acquire)) return GVA_OK;
    GVA_CUDA(cudaFuncSetAttribute(ext_write_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)ext_smem_bytes(kMaxCols - 1, kMaxCols)));
    GVA_CUDA(cudaFuncSetAttribute(red_write_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)red_smem_bytes(kMaxCols)));
    if (dev < 64) done[dev].store(true, std::memory_order_release);
    return GVA_OK;
}

void fill_ext(ExtArgs& a, const DevDB& db, const Step& st, const uint32_t* in, uint64_t nrows, uint32_t* out) {
    memset(&a, 0, sizeof a);
    const DevPart& P = db.parts[st.part - 1];
    a.in = in;
    a.nrows = nrows;
    a.out = out;
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
}

void fill_red(RedArgs& a, const DevDB& db, const Step& st, const uint32_t* in, uint64_t nrows, uint32_t* out) {
    memset(&a, 0, sizeof a);
    const DevPart& P = db.parts[st.part - 1];
    a.in = in;
    a.nrows = nrows;
    a.out = out;
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

// count + scan; leaves exclusive block offsets in sums[0..nb) and the total in sums[nb]
int launch_count(const DevDB& db, const Step& st, const uint32_t* in, uint64_t nrows, uint64_t* sums,
                 cudaStream_t s, Profiler* prof) {
    const uint64_t nb = (nrows + kRowsPerBlock - 1) / kRowsPerBlock;
    if (nb > 0x7fffffffull) return fail(GVA_ERR_UNSUPPORTED, "frontier too large for one launch");
    const double k = st.width_in;
    cudaEvent_t ev = nullptr;
    if (st.kind == STEP_EXT) {
        ExtArgs a;
        fill_ext(a, db, st, in, nrows, nullptr);
        const double bytes = (4.0 * k + 8.0) * (double)nrows;
        if (prof) prof->begin(K_EXT_COUNT, bytes, s, ev);
        ext_count_kernel<<<(unsigned)nb, kThreads, 0, s>>>(a, sums);
        if (prof) prof->end(ev, K_EXT_COUNT, bytes, s, (double)nrows);
    } else {
        RedArgs a;
        fill_red(a, db, st, in, nrows, nullptr);
        const double bytes = (4.0 * k + 8.0 * st.n_pairs) * (double)nrows;
        if (prof) prof->begin(K_RED_COUNT, bytes, s, ev);
        red_count_kernel<<<(unsigned)nb, kThreads, 0, s>>>(a, sums);
        if (prof) prof->end(ev, K_RED_COUNT, bytes, s, (double)nrows);
    }
    GVA_CUDA(cudaGetLastError());
    const double sbytes = 16.0 * (double)nb;
    if (prof) prof->begin(K_SCAN, sbytes, s, ev);
    scan_block_sums_kernel<<<1, kScanThreads, 0, s>>>(sums, nb);
    if (prof) prof->end(ev, K_SCAN, sbytes, s, (double)nb);
    GVA_CUDA(cudaGetLastError());
    g_launches += 2;
    return GVA_OK;
}

int launch_write(const DevDB& db, const Step& st, const uint32_t* in, uint64_t nrows, uint32_t* out,
                 const uint64_t* sums, uint64_t nout, cudaStream_t s, Profiler* prof) {
    const uint64_t nb = (nrows + kRowsPerBlock - 1) / kRowsPerBlock;
    int rc = set_smem_limits();
    if (rc) return rc;
    const double k = st.width_in;
    cudaEvent_t ev = nullptr;
    if (st.kind == STEP_EXT) {
        ExtArgs a;
        fill_ext(a, db, st, in, nrows, out);
        const double bytes = (4.0 * k + 8.0) * (double)nrows + (4.0 + 4.0 * (k + 1)) * (double)nout;
        if (prof) prof->begin(K_EXT_WRITE, bytes, s, ev);
        ext_write_kernel<<<(unsigned)nb, kThreads, ext_smem_bytes(a.k, a.n_eq), s>>>(a, sums);
        if (prof) prof->end(ev, K_EXT_WRITE, bytes, s, (double)nrows);
    } else {
        RedArgs a;
        fill_red(a, db, st, in, nrows, out);
        const double bytes = (4.0 * k + 8.0 * st.n_pairs) * (double)nrows + 4.0 * k * (double)nout;
        if (prof) prof->begin(K_RED_WRITE, bytes, s, ev);
        red_write_kernel<<<(unsigned)nb, kThreads, red_smem_bytes(a.k), s>>>(a, sums);
        if (prof) prof->end(ev, K_RED_WRITE, bytes, s, (double)nrows);
    }
    GVA_CUDA(cudaGetLastError());
    g_launches += 1;
    return GVA_OK;
}

// Per-thread, per-device host staging reused by every query: a pinned word
// for count read-backs and two timing events (creating these per call costs
// more than a small query's kernels).
struct HostStage {
    uint64_t* pinned = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

int host_stage(int device, HostStage*& out) {
    static thread_local HostStage stages[64];
    if (device < 0 || device >= 64) return fail(GVA_ERR_ARG, "device index out of range");
    HostStage& h = stages[device];
    if (!h.pinned) {
        GVA_CUDA(cudaMallocHost(&h.pinned, 64));
        GVA_CUDA(cudaEventCreate(&h.ev0));
        GVA_CUDA(cudaEventCreate(&h.ev1));
    }
    out = &h;
    return GVA_OK;
}

int ensure_pool(int device) {
    static std::atomic<bool> done[64];
    if (device < 64 && done[device].load(std::memory_order_acquire)) return GVA_OK;
    cudaMemPool_t pool;
    GVA_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = UINT64_MAX;  // keep freed frontier memory cached for the next phase / query
    GVA_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    if (device < 64) done[device].store(true, std::memory_order_release);
    return GVA_OK;
}

}  // namespace

const char* const kKernelNames[K_NUM] = {"ext_count", "ext_write", "red_count", "red_write", "scan_block_sums",
                                         "mni_search"};

uint64_t kernel_launches() { return g_launches.load() + batch_kernel_launches() + mni_kernel_launches(); }

void Profiler::begin(int kind, double bytes, cudaStream_t s, cudaEvent_t& a) {
    (void)kind;
    (void)bytes;
    cudaEventCreate(&a);
    cudaEventRecord(a, s);
}

void Profiler::end(cudaEvent_t a, int kind, double bytes, cudaStream_t s, double rows) {
    cudaEvent_t b;
    cudaEventCreate(&b);
    cudaEventRecord(b, s);
    pending.push_back({kind, a, b, bytes, rows});
}

void Profiler::resolve() {
    for (auto& p : pending) {
        float ms = 0.f;
        cudaEventSynchronize(p.b);
        cudaEventElapsedTime(&ms, p.a, p.b);
        stat[p.kind].launches += 1;
        stat[p.kind].ms += ms;
        stat[p.kind].bytes += p.bytes;
        stat[p.kind].rows += p.rows;
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    pending.clear();
}

// ------------------------------------------------------------- database ----
int upload_graph(HostGraph& g, int device, DevDB*& out) {
    out = nullptr;
    int ndev = 0;
    GVA_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(GVA_ERR_ARG, "device index out of range");
    GVA_CUDA(cudaSetDevice(device));
    // every engine (per-query, batched, MNI) allocates frontiers and round
    // buffers from the stream-ordered pool: keep freed memory cached there
    // instead of returning it to the driver at each synchronisation
    int prc = ensure_pool(device);
    if (prc) return prc;
    const uint32_t L = g.num_labels();
    // vertices grouped by dense label: the seed frontiers of init phases; the
    // same groups by total degree for rooted existence searches, which try
    // the vertices most likely to succeed first
    std::vector<uint32_t> seed_off, seed_verts, seed_deg;
    seed_groups(g, seed_off, seed_verts, seed_deg);
    // segment index per partition: packed 32-byte vertex records when the
    // label count allows (seg_of), else the dense (vertex, label) table
    bool packed = L >= 1 && L <= 28;
    for (auto& p : g.parts)
        if (!p.off.empty() && p.adj.size() >= 0x80000000ull) packed = false;
    std::vector<std::vector<uint32_t>> pidx(g.parts.size());
    if (packed) {
        const uint64_t nv = (uint64_t)g.max_id + 1;
        for (size_t i = 0; i < g.parts.size(); ++i) {
            const HostPartition& hp = g.parts[i];
            if (hp.off.empty()) continue;
            std::vector<uint32_t>& rec = pidx[i];
            rec.assign(nv * 8, 0);
            std::vector<uint32_t> wide;
            for (uint64_t v = 0; v < nv; ++v) {
                const uint32_t* o = hp.off.data() + v * L;
                const uint32_t base = o[0];
                uint32_t* r = rec.data() + v * 8;
                if (o[L] - base > 255) {
                    r[0] = base | 0x80000000u;
                    r[1] = (uint32_t)(nv * 8 + wide.size());
                    for (uint32_t j = 0; j <= L; ++j) wide.push_back(o[j] - base);
                } else {
                    r[0] = base;
                    unsigned char* b = reinterpret_cast<unsigned char*>(r);
                    for (uint32_t j = 1; j <= L; ++j) b[3 + j] = (unsigned char)(o[j] - base);
                }
            }
            if (nv * 8 + wide.size() >= 0x80000000ull) {
                packed = false;
                break;
            }
            rec.insert(rec.end(), wide.begin(), wide.end());
        }
        if (!packed) pidx.assign(g.parts.size(), {});
    }
    size_t bytes = 2 * align256(seed_verts.size() * 4 + 16);
    for (size_t i = 0; i < g.parts.size(); ++i)
        bytes += align256((packed ? pidx[i].size() : g.parts[i].off.size()) * 4) + align256(g.parts[i].adj.size() * 4 + 16);
    void* arena = nullptr;
    cudaError_t e = cudaMalloc(&arena, bytes);
    if (e != cudaSuccess) return fail(GVA_ERR_NOMEM, std::string("database allocation failed: ") + cudaGetErrorString(e));
    DevDB* db = new DevDB();
    db->device = device;
    db->max_id = g.max_id;
    db->L = L;
    db->packed = packed;
    db->labels = g.labels;
    db->seed_off = seed_off;
    db->arena = arena;
    db->arena_bytes = bytes;
    char* cur = (char*)arena;
    auto put = [&](const std::vector<uint32_t>& v) -> const uint32_t* {
        const uint32_t* at = (const uint32_t*)cur;
        if (!v.empty()) cudaMemcpy(cur, v.data(), v.size() * 4, cudaMemcpyHostToDevice);
        cur += align256(v.size() * 4 + 16);
        return at;
    };
    db->seed_verts = put(seed_verts);
    db->seed_by_degree = put(seed_deg);
    db->parts.resize(g.parts.size());
    for (size_t i = 0; i < g.parts.size(); ++i) {
        HostPartition& hp = g.parts[i];
        if (hp.off.empty()) continue;
        const uint32_t* off = (const uint32_t*)cur;
        if (packed) {
            cudaMemcpy(cur, pidx[i].data(), pidx[i].size() * 4, cudaMemcpyHostToDevice);
            cur += align256(pidx[i].size() * 4);
        } else {
            cudaMemcpy(cur, hp.off.data(), hp.off.size() * 4, cudaMemcpyHostToDevice);
            cur += align256(hp.off.size() * 4);
        }
        db->parts[i].off = off;
        db->parts[i].adj = put(hp.adj);
        db->parts[i].n_adj = hp.adj.size();
        db->n_adj += hp.adj.size();
    }
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaFree(arena);
        delete db;
        return fail(GVA_ERR_CUDA, std::string("database upload failed: ") + cudaGetErrorString(e));
    }
    // keep label tables and partition presence for planning; drop host adjacency
    db->meta.max_id = g.max_id;
    db->meta.labels = g.labels;
    db->meta.parts.resize(g.parts.size());
    for (size_t i = 0; i < g.parts.size(); ++i)
        if (!g.parts[i].off.empty()) db->meta.parts[i].off.assign(1, 0);
    out = db;
    return GVA_OK;
}

void free_devdb(DevDB* db) {
    if (!db) return;
    if (db->arena || db->vgraph) cudaSetDevice(db->device);
    if (db->arena) cudaFree(db->arena);
    if (db->vgraph) cudaFree(db->vgraph);
    delete db;
}

size_t step_scratch_bytes(uint64_t in_rows) {
    const uint64_t nb = (in_rows + kRowsPerBlock - 1) / kRowsPerBlock;
    return align256((nb + 1) * sizeof(uint64_t));
}

// ---------------------------------------------------------- one step (L4) --
int run_step(DevDB& db, const Step& st, const uint32_t* in, uint64_t in_rows, uint32_t* out, uint64_t out_cap,
             uint64_t* out_rows, void* scratch, size_t scratch_bytes, cudaStream_t s) {
    if (!out_rows) return fail(GVA_ERR_ARG, "out_rows is null");
    *out_rows = 0;
    GVA_CUDA(cudaSetDevice(db.device));
    if (st.always_empty) return GVA_OK;
    if (st.kind == STEP_SEED) {
        const uint64_t n = db.seed_off[st.label + 1] - db.seed_off[st.label];
        *out_rows = n;
        if (n > out_cap) return fail(GVA_ERR_NOMEM, "output capacity too small");
        if (n) GVA_CUDA(cudaMemcpyAsync(out, db.seed_verts + db.seed_off[st.label], n * 4, cudaMemcpyDeviceToDevice, s));
        return GVA_OK;
    }
    if (in_rows == 0) return GVA_OK;
    if (!in || !scratch) return fail(GVA_ERR_ARG, "null device buffer");
    if (scratch_bytes < step_scratch_bytes(in_rows)) return fail(GVA_ERR_ARG, "scratch too small");
    uint64_t* sums = (uint64_t*)scratch;
    int rc = launch_count(db, st, in, in_rows, sums, s, nullptr);
    if (rc) return rc;
    const uint64_t nb = (in_rows + kRowsPerBlock - 1) / kRowsPerBlock;
    uint64_t total = 0;
    GVA_CUDA(cudaMemcpyAsync(&total, sums + nb, 8, cudaMemcpyDeviceToHost, s));
    GVA_CUDA(cudaStreamSynchronize(s));
    *out_rows = total;
    if (total > out_cap) return fail(GVA_ERR_NOMEM, "output capacity too small");
    if (total == 0) return GVA_OK;
    if (!out) return fail(GVA_ERR_ARG, "null output buffer");
    return launch_write(db, st, in, in_rows, out, sums, total, s, nullptr);
}

// ------------------------------------------------------- whole query (L3) --
int run_match(DevDB& db, const Plan& plan, const std::vector<Step>& steps, cudaStream_t s, uint64_t budget,
              bool count_only, bool profile, MatchResult& res) {
    Profiler profiler;
    Profiler* prof = profile ? &profiler : nullptr;
    GVA_CUDA(cudaSetDevice(db.device));
    int rc = ensure_pool(db.device);
    if (rc) return rc;
    res = MatchResult();
    res.device = db.device;
    res.stream = s;
    res.columns = plan.columns;
    res.phase_rows.assign(plan.phases.size(), 0);
    if (budget == 0) {  // 3/4 of the memory free at the database's first run (a driver query per call is costly)
        if (db.default_budget == 0) {
            size_t fr = 0, tot = 0;
            GVA_CUDA(cudaMemGetInfo(&fr, &tot));
            db.default_budget = (uint64_t)fr / 4 * 3;
        }
        budget = db.default_budget;
    }
    HostStage* hs = nullptr;
    rc = host_stage(db.device, hs);
    if (rc) return rc;
    cudaEvent_t ev0 = hs->ev0, ev1 = hs->ev1;
    GVA_CUDA(cudaEventRecord(ev0, s));

    const uint32_t* cur = nullptr;
    uint32_t* owned = nullptr;  // frontier we must free
    uint64_t rows = 0;
    uint32_t width = 0;
    uint64_t* sums = nullptr;
    size_t sums_bytes = 0;
    uint64_t* total_h = hs->pinned;
    cudaError_t ce = cudaSuccess;
    int status = GVA_OK;
    bool counted_only = false;

    for (size_t i = 0; i < steps.size(); ++i) {
        const Step& st = steps[i];
        const bool last = (i + 1 == steps.size());
        const uint32_t out_w = st.kind == STEP_SEED ? 1 : (st.kind == STEP_EXT ? width + 1 : width);
        if (st.always_empty) {
            rows = 0;
        } else if (st.kind == STEP_SEED) {
            cur = db.seed_verts + db.seed_off[st.label];
            rows = db.seed_off[st.label + 1] - db.seed_off[st.label];
        } else if (rows > 0) {
            const size_t need = step_scratch_bytes(rows);
            if (need > sums_bytes) {
                if (sums) cudaFreeAsync(sums, s);
                ce = cudaMallocAsync((void**)&sums, need, s);
                if (ce != cudaSuccess) { status = fail(GVA_ERR_NOMEM, "scratch allocation failed"); sums = nullptr; break; }
                sums_bytes = need;
            }
            status = launch_count(db, st, cur, rows, sums, s, prof);
            if (status) break;
            const uint64_t nb = (rows + kRowsPerBlock - 1) / kRowsPerBlock;
            ce = cudaMemcpyAsync(total_h, sums + nb, 8, cudaMemcpyDeviceToHost, s);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
            if (ce != cudaSuccess) { status = fail(GVA_ERR_CUDA, cudaGetErrorString(ce)); break; }
            const uint64_t total = *total_h;
            if (last && count_only) {
                rows = total;
                counted_only = true;
            } else if (total == 0) {
                rows = 0;
            } else {
                const uint64_t bytes = total * out_w * 4ull;
                if (bytes > budget) {
                    status = fail(GVA_ERR_NOMEM, "frontier of " + std::to_string(total) + " rows exceeds the memory budget");
                    break;
                }
                uint32_t* out = nullptr;
                ce = cudaMallocAsync((void**)&out, bytes, s);
                if (ce != cudaSuccess) { status = fail(GVA_ERR_NOMEM, "frontier allocation failed"); break; }
                status = launch_write(db, st, cur, rows, out, sums, total, s, prof);
                if (status) { cudaFreeAsync(out, s); break; }
                if (owned) cudaFreeAsync(owned, s);
                owned = out;
                cur = out;
                rows = total;
            }
        }
        width = out_w;
        if (st.phase_end >= 0) res.phase_rows[st.phase_end] = rows;
        if (rows == 0) break;
    }
    if (sums) cudaFreeAsync(sums, s);
    if (status) {
        if (owned) cudaFreeAsync(owned, s);
        if (prof) prof->resolve();
        return status;
    }
    GVA_CUDA(cudaEventRecord(ev1, s));
    GVA_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    res.gpu_ms = ms;
    if (prof) {
        prof->resolve();
        for (int i = 0; i < K_NUM; ++i) res.kstat[i] = prof->stat[i];
    }
    // the final width is the number of columns of the plan
    res.width = (uint32_t)plan.columns.size();
    res.rows = rows;
    if (rows == 0 || counted_only) {
        if (owned) cudaFreeAsync(owned, s);
        res.rows_dev = nullptr;
    } else if (owned) {
        res.rows_dev = owned;
    } else {
        // the final frontier is still the seed list (cannot happen: a plan ends with an extension or reduction)
        res.rows_dev = nullptr;
    }
    GVA_CUDA(cudaStreamSynchronize(s));
    return GVA_OK;
}

void free_result(MatchResult* r) {
    if (!r) return;
    if (r->rows_dev) {
        cudaSetDevice(r->device);
        cudaFreeAsync(r->rows_dev, r->stream);
        cudaStreamSynchronize(r->stream);
    }
    delete r;
}

}  // namespace gva
