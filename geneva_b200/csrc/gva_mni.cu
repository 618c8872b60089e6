// Single-graph support: MNI (minimum image based support).
//
// For a pattern P and a data graph, the image set of a pattern vertex u is
// {f(u) : f an embedding of P} (injective, label preserving, every pattern
// edge present with its edge label; non-induced).  The MNI support of P is
// the smallest image set over u.  It is anti-monotone, so level-wise mining
// over one large graph can prune with it as the graph-count support prunes
// over a database of graphs.
//
// The reference has no support notion (it enumerates the embeddings of one
// pattern, src/gpumine.cpp:994-1061).  Enumerating embeddings to collect image
// sets is hopeless on skewed graphs (a 4-edge star around a hub of degree 10^5
// has ~10^18 embeddings), so image sets are decided by existence:
//
//   task    one automorphism orbit of one pattern (orbits share image sets),
//           rooted at a representative r; its seeds are the data vertices
//           carrying r's label
//   search  a depth-first search for one embedding with f(r) = v: per level
//           the candidates are the shortest segment among the already matched
//           neighbours, each filtered by injectivity and by binary search in
//           the other matched neighbours' segments, the first survivor taken.
//           Each lane first searches its own seed for up to 64 candidates (32
//           independent searches per warp keep many loads in flight); seeds
//           still undecided are searched by the whole warp, 32 candidates per
//           step, one seed at a time
//   stop    a task stops once its count reaches the cap (default: the minimum
//           support, which decides frequency) or the smallest exhausted orbit
//           of its pattern, so the support returned is min(MNI, cap) exactly
//
// Tasks run in rounds: each active task gets the next 2048 << round seeds,
// as work items that a persistent kernel hands to warps through an atomic
// queue (SM-level load balance however skewed the seeds' degrees are).  With
// many tasks an item is a task's whole quota, scanned by one warp in seed
// order and stopped as soon as the count reaches the cap; with few, quotas
// are cut into items of down to 128 seeds so that every warp has work.  The
// host retires capped and exhausted tasks between rounds.
// The batched form puts every task of many patterns in one round; the plain
// form runs the same rounds one pattern at a time.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/geneva.h"
#include "gva_engine.cuh"
#include "gva_kernels.cuh"

namespace gva {

namespace {

#define GVA_CUDA_M(call)                                                                                \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return fail(GVA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));              \
    } while (0)

constexpr int kMniWarps = 8;       // warps per block
constexpr uint32_t kMniItem = 128; // smallest work item (seeds); rounds with few tasks use it
constexpr uint32_t kMniFirst = 2048;  // seeds per task in the first round (doubles every round)

struct PartPtr {
    const uint32_t* off;
    const uint32_t* adj;
};

// One rooted existence search: pattern vertices in search order (level 0 =
// the orbit representative), with per level its label, the partitions of
// its edges to earlier levels, and the earlier levels sharing its label.
struct MniTask {
    uint32_t n;
    uint32_t seed_begin;  // seeds: seed_by_degree[seed_begin, seed_begin + seed_count)
    uint32_t seed_count;
    uint32_t n_rootf;
    uint16_t lab[kMniMaxVertices];
    uint8_t part[kMniMaxVertices][kMniMaxVertices];  // 1-based partition of edge (i, j), 0 = none
    uint8_t eqmask[kMniMaxVertices];                 // earlier levels with the same label
    uint8_t nbmask[kMniMaxVertices];                 // earlier levels adjacent to this one
    // the root needs >= root_mult[k] neighbours of label root_lab[k] in partition root_part[k]
    uint8_t root_part[kMniMaxVertices];
    uint8_t root_mult[kMniMaxVertices];
    uint16_t root_lab[kMniMaxVertices];
};
static_assert(sizeof(MniTask) % 4 == 0, "task copied as words");

struct MniSlot {  // one active task in one round
    uint32_t task;
    uint32_t start;  // first seed (relative to the task's seed range)
    uint32_t len;
    uint32_t cap;    // stop once counts[task] reaches this
};

enum MniProf { P_SEEDS = 0, P_ROOTS, P_OPENS, P_SCANNED, P_CHECKS, P_FOUND, P_NUM };

// item -> slot, so that no warp searches item0 for its item's slot
__global__ void mni_expand_kernel(const uint64_t* __restrict__ item0, int nslots, uint32_t* __restrict__ item_slot) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nslots; s += gridDim.x * blockDim.x)
        for (uint64_t i = item0[s]; i < item0[s + 1]; ++i) item_slot[i] = (uint32_t)s;
}

__device__ __forceinline__ bool root_ok(const MniTask& T, const PartPtr* __restrict__ parts, uint32_t L, uint32_t v) {
    for (uint32_t k = 0; k < T.n_rootf; ++k) {
        const PartPtr P = parts[T.root_part[k] - 1];
        uint32_t lo, hi;
        seg_of(P.off, L, v, T.root_lab[k], lo, hi);
        if (hi - lo < T.root_mult[k]) return false;
    }
    return true;
}

// Whether some embedding maps level 0 to `root`.  Called by all 32 lanes with
// the same root; the search state is identical in every lane.
__device__ bool mni_dfs(const MniTask& T, const PartPtr* __restrict__ parts, uint32_t L, uint32_t root, uint32_t lane,
                        unsigned long long* cnt) {
    uint32_t f[kMniMaxVertices];
    uint32_t pos[kMniMaxVertices], end[kMniMaxVertices], gsel[kMniMaxVertices];
    const uint32_t* gadj[kMniMaxVertices];
    const int n = (int)T.n;
    f[0] = root;
    if (n <= 1) return true;
    // candidates of level lv: the shortest segment among its matched neighbours
    auto open = [&](int lv) {
        uint32_t blo = 0, bhi = 0, bj = 0;
        const uint32_t* ba = nullptr;
        bool have = false;
        uint32_t m = T.nbmask[lv];
        while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            const PartPtr P = parts[T.part[lv][j] - 1];
            uint32_t lo, hi;
            seg_of(P.off, L, f[j], T.lab[lv], lo, hi);
            if (!have || hi - lo < bhi - blo) {
                blo = lo;
                bhi = hi;
                bj = (uint32_t)j;
                ba = P.adj;
                have = true;
            }
        }
        pos[lv] = blo;
        end[lv] = bhi;
        gadj[lv] = ba;
        gsel[lv] = bj;
        cnt[P_OPENS] += lane == 0 ? 1 : 0;
    };
    int i = 1;
    open(1);
    for (;;) {
        if (pos[i] >= end[i]) {
            if (--i == 0) return false;
            continue;
        }
        const uint32_t p = pos[i] + lane;
        uint32_t c = 0;
        bool ok = false;
        if (p < end[i]) {
            c = __ldg(gadj[i] + p);
            ok = true;
            cnt[P_SCANNED] += 1;
            uint32_t e = T.eqmask[i];
            while (e && ok) {
                const int j = __ffs(e) - 1;
                e &= e - 1;
                ok = c != f[j];
            }
            uint32_t m = T.nbmask[i] & ~(1u << gsel[i]);
            while (m && ok) {
                const int j = __ffs(m) - 1;
                m &= m - 1;
                const PartPtr P = parts[T.part[i][j] - 1];
                uint32_t lo, hi;
                seg_of(P.off, L, f[j], T.lab[i], lo, hi);
                ok = find_in(P.adj, lo, hi, c) != 0xffffffffu;
                cnt[P_CHECKS] += 1;
            }
        }
        const uint32_t b = __ballot_sync(0xffffffffu, ok);
        if (!b) {
            pos[i] += 32;
            continue;
        }
        const int l = __ffs(b) - 1;
        f[i] = __shfl_sync(0xffffffffu, c, l);
        pos[i] += (uint32_t)l + 1;
        if (i + 1 == n) return true;
        ++i;
        open(i);
    }
}

// One lane's own depth-first search for an embedding with level 0 at `root`,
// candidates taken one at a time: 1 = found, 0 = none exists, -1 = gave up
// after `budget` candidates (the warp-cooperative search then decides).
// Thirty-two of these run side by side in a warp, one root per lane, so
// their dependent loads overlap; most roots of frequent patterns succeed or
// fail within a few candidates.
__device__ int lane_dfs(const MniTask& T, const PartPtr* __restrict__ parts, uint32_t L, uint32_t root,
                        uint32_t budget, unsigned long long* cnt) {
    uint32_t f[kMniMaxVertices];
    uint32_t pos[kMniMaxVertices], end[kMniMaxVertices], gsel[kMniMaxVertices];
    const uint32_t* gadj[kMniMaxVertices];
    const int n = (int)T.n;
    f[0] = root;
    if (n <= 1) return 1;
    auto open = [&](int lv) {
        uint32_t blo = 0, bhi = 0, bj = 0;
        const uint32_t* ba = nullptr;
        bool have = false;
        uint32_t m = T.nbmask[lv];
        while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            const PartPtr P = parts[T.part[lv][j] - 1];
            uint32_t lo, hi;
            seg_of(P.off, L, f[j], T.lab[lv], lo, hi);
            if (!have || hi - lo < bhi - blo) {
                blo = lo;
                bhi = hi;
                bj = (uint32_t)j;
                ba = P.adj;
                have = true;
            }
        }
        pos[lv] = blo;
        end[lv] = bhi;
        gadj[lv] = ba;
        gsel[lv] = bj;
        cnt[P_OPENS] += 1;
    };
    int i = 1;
    open(1);
    uint32_t steps = 0;
    for (;;) {
        if (pos[i] >= end[i]) {
            if (--i == 0) return 0;
            continue;
        }
        if (++steps > budget) return -1;
        const uint32_t c = __ldg(gadj[i] + pos[i]);
        ++pos[i];
        cnt[P_SCANNED] += 1;
        bool ok = true;
        uint32_t e = T.eqmask[i];
        while (e && ok) {
            const int j = __ffs(e) - 1;
            e &= e - 1;
            ok = c != f[j];
        }
        uint32_t m = T.nbmask[i] & ~(1u << gsel[i]);
        while (m && ok) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            const PartPtr P = parts[T.part[i][j] - 1];
            uint32_t lo, hi;
            seg_of(P.off, L, f[j], T.lab[i], lo, hi);
            ok = find_in(P.adj, lo, hi, c) != 0xffffffffu;
            cnt[P_CHECKS] += 1;
        }
        if (!ok) continue;
        f[i] = c;
        if (i + 1 == n) return 1;
        ++i;
        open(i);
    }
}

constexpr uint32_t kLaneBudget = 64;  // candidates a lane search may take before the warp search decides

// Persistent: every warp pulls 128-seed items; per 32 seeds it checks the
// task's count against its cap, filters roots by neighbour-label degrees and
// runs one search per surviving root.
__global__ void __launch_bounds__(kMniWarps * 32, 6)
mni_search_kernel(const MniTask* __restrict__ tasks, const MniSlot* __restrict__ slots,
                  const uint64_t* __restrict__ item0, const uint32_t* __restrict__ item_slot, uint64_t nitems,
                  const uint32_t* __restrict__ seeds, uint32_t item_len,
                  const PartPtr* __restrict__ parts, uint32_t L, uint32_t* __restrict__ counts,
                  unsigned long long* __restrict__ queue, unsigned long long* __restrict__ prof) {
    __shared__ MniTask tsh[kMniWarps];
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    MniTask& T = tsh[w];
    unsigned long long cnt[P_NUM] = {0, 0, 0, 0, 0, 0};
    int cur = -1;
    for (;;) {
        unsigned long long it = 0;
        if (lane == 0) it = atomicAdd(queue, 1ull);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= nitems) break;
        const int s = (int)__ldg(item_slot + it);
        const MniSlot sl = slots[s];
        if ((int)sl.task != cur) {
            __syncwarp();
            const uint32_t* src = reinterpret_cast<const uint32_t*>(tasks + sl.task);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&T);
            for (uint32_t k = lane; k < sizeof(MniTask) / 4; k += 32) dst[k] = __ldg(src + k);
            __syncwarp();
            cur = (int)sl.task;
        }
        const uint32_t a = sl.start + (uint32_t)(it - item0[s]) * item_len;
        const uint32_t b = min(a + item_len, sl.start + sl.len);
        for (uint32_t c0 = a; c0 < b; c0 += 32) {
            // one lane reads the count so that the whole warp takes the same branch
            uint32_t seen = 0;
            if (lane == 0) seen = *(volatile const uint32_t*)(counts + sl.task);
            if (__shfl_sync(0xffffffffu, seen, 0) >= sl.cap) break;
            uint32_t v = 0;
            bool ok = false;
            if (c0 + lane < b) {
                v = __ldg(seeds + T.seed_begin + c0 + lane);
                ok = root_ok(T, parts, L, v);
                cnt[P_SEEDS] += 1;
            }
            const uint32_t roots = __ballot_sync(0xffffffffu, ok);  // all lanes vote
            if (lane == 0) cnt[P_ROOTS] += __popc(roots);
            // every lane searches its own root; roots whose search ran out of
            // budget are decided by the whole warp, one after another
            int verdict = 0;
            if (ok) verdict = lane_dfs(T, parts, L, v, kLaneBudget, cnt);
            uint32_t found = __popc(__ballot_sync(0xffffffffu, verdict == 1));
            uint32_t m = __ballot_sync(0xffffffffu, verdict < 0);
            while (m) {
                const int l = __ffs(m) - 1;
                m &= m - 1;
                const uint32_t root = __shfl_sync(0xffffffffu, v, l);
                if (mni_dfs(T, parts, L, root, lane, cnt)) ++found;
            }
            if (found && lane == 0) atomicAdd(counts + sl.task, found);
            if (lane == 0) cnt[P_FOUND] += found;
        }
    }
    if (prof) {
        for (int k = 0; k < P_NUM; ++k) {
            unsigned long long x = cnt[k];
            x = warp_sum(x);
            if (lane == 0 && x) atomicAdd(prof + k, x);
        }
    }
}

std::atomic<uint64_t> g_mni_launches{0};

// ----------------------------------------------------------- host helpers ---
// Automorphism orbits of a small pattern: orbit[v] = smallest vertex of v's orbit.
void pattern_orbits(const MniPattern& p, uint32_t* orbit) {
    const uint32_t n = p.n;
    uint32_t deg[kMniMaxVertices] = {0};
    for (uint32_t a = 0; a < n; ++a)
        for (uint32_t b = 0; b < n; ++b) deg[a] += p.el[a][b] ? 1 : 0;
    uint32_t parent[kMniMaxVertices];
    for (uint32_t v = 0; v < n; ++v) parent[v] = v;
    auto root = [&](uint32_t v) {
        while (parent[v] != v) v = parent[v] = parent[parent[v]];
        return v;
    };
    uint32_t perm[kMniMaxVertices];
    bool used[kMniMaxVertices] = {false};
    // backtracking over label- and degree-preserving maps that keep every edge label
    auto rec = [&](auto&& self, uint32_t i) -> void {
        if (i == n) {
            for (uint32_t v = 0; v < n; ++v) {
                const uint32_t a = root(v), b = root(perm[v]);
                if (a != b) parent[std::max(a, b)] = std::min(a, b);
            }
            return;
        }
        for (uint32_t c = 0; c < n; ++c) {
            if (used[c] || p.vl[c] != p.vl[i] || deg[c] != deg[i]) continue;
            bool ok = true;
            for (uint32_t j = 0; j < i && ok; ++j) ok = p.el[i][j] == p.el[c][perm[j]];
            if (!ok) continue;
            used[c] = true;
            perm[i] = c;
            self(self, i + 1);
            used[c] = false;
        }
    };
    rec(rec, 0);
    for (uint32_t v = 0; v < n; ++v) orbit[v] = root(v);
}

// Search order from `r`: repeatedly the unmatched vertex with the most
// matched neighbours, then the rarest label, then the lowest index.
void search_order(const MniPattern& p, uint32_t r, const std::vector<uint32_t>& seed_off, uint32_t* order) {
    uint32_t matched = 1u << r;
    order[0] = r;
    for (uint32_t k = 1; k < p.n; ++k) {
        uint32_t best = kNone, best_nb = 0;
        uint64_t best_freq = 0;
        for (uint32_t v = 0; v < p.n; ++v) {
            if (matched >> v & 1) continue;
            uint32_t nb = 0;
            for (uint32_t u = 0; u < p.n; ++u)
                if ((matched >> u & 1) && p.el[v][u]) ++nb;
            if (nb == 0) continue;
            const uint64_t fq = seed_off[p.vl[v] + 1] - seed_off[p.vl[v]];
            if (best == kNone || nb > best_nb || (nb == best_nb && fq < best_freq)) {
                best = v;
                best_nb = nb;
                best_freq = fq;
            }
        }
        order[k] = best;
        matched |= 1u << best;
    }
}

void build_task(const DevDB& db, const MniPattern& p, uint32_t r, MniTask& T) {
    memset(&T, 0, sizeof T);
    uint32_t order[kMniMaxVertices];
    search_order(p, r, db.seed_off, order);
    T.n = p.n;
    for (uint32_t i = 0; i < p.n; ++i) {
        T.lab[i] = (uint16_t)p.vl[order[i]];
        for (uint32_t j = 0; j < i; ++j) {
            T.part[i][j] = T.part[j][i] = p.el[order[i]][order[j]];
            if (T.part[i][j]) T.nbmask[i] |= (uint8_t)(1u << j);
            if (p.vl[order[i]] == p.vl[order[j]]) T.eqmask[i] |= (uint8_t)(1u << j);
        }
    }
    T.seed_begin = db.seed_off[p.vl[r]];
    T.seed_count = db.seed_off[p.vl[r] + 1] - db.seed_off[p.vl[r]];
    for (uint32_t w = 0; w < p.n; ++w) {
        if (!p.el[r][w]) continue;
        uint32_t k = 0;
        while (k < T.n_rootf && !(T.root_part[k] == p.el[r][w] && T.root_lab[k] == p.vl[w])) ++k;
        if (k == T.n_rootf) {
            T.root_part[k] = p.el[r][w];
            T.root_lab[k] = (uint16_t)p.vl[w];
            T.n_rootf++;
        }
        T.root_mult[k]++;
    }
}

}  // namespace

uint64_t mni_kernel_launches() { return g_mni_launches.load(); }

int mni_pattern_from_text(const DevDB& db, const std::string& text, MniPattern& p, bool& absent) {
    p = MniPattern();
    absent = false;
    std::vector<std::pair<uint32_t, uint32_t>> vs;
    std::vector<uint32_t> es;
    size_t i = 0;
    while (i < text.size()) {
        size_t j = text.find('\n', i);
        if (j == std::string::npos) j = text.size();
        const std::string line = text.substr(i, j - i);
        i = j + 1;
        char t = 0;
        unsigned a = 0, b = 0, c = 0;
        if (sscanf(line.c_str(), " %c", &t) != 1) continue;
        if (t == 'v') {
            if (sscanf(line.c_str(), " v %u %u", &a, &b) != 2) return fail(GVA_ERR_FORMAT, "bad vertex line: " + line);
            vs.push_back({a, b});
        } else if (t == 'e') {
            if (sscanf(line.c_str(), " e %u %u %u", &a, &b, &c) != 3) return fail(GVA_ERR_FORMAT, "bad edge line: " + line);
            es.insert(es.end(), {a, b, c});
        } else {
            return fail(GVA_ERR_FORMAT, "unexpected pattern line: " + line);
        }
    }
    if (vs.empty()) return fail(GVA_ERR_FORMAT, "pattern without vertices");
    if (vs.size() > (size_t)kMniMaxVertices)
        return fail(GVA_ERR_UNSUPPORTED, "MNI support handles patterns of up to 8 vertices");
    p.n = (uint32_t)vs.size();
    std::vector<bool> seen(p.n, false);
    for (auto& v : vs) {
        if (v.first >= p.n || seen[v.first]) return fail(GVA_ERR_FORMAT, "vertex ids must be 0..n-1, each once");
        seen[v.first] = true;
        const uint32_t d = db.meta.dense_label(v.second);
        if (d == kNone) absent = true;
        p.vl[v.first] = d == kNone ? 0 : d;
    }
    for (size_t k = 0; k < es.size(); k += 3) {
        const uint32_t a = es[k], b = es[k + 1], l = es[k + 2];
        if (a >= p.n || b >= p.n || a == b) return fail(GVA_ERR_FORMAT, "edge endpoints must be distinct pattern vertices");
        if (l == 0 || l > 255) return fail(GVA_ERR_FORMAT, "edge labels must be 1..255");
        if (p.el[a][b]) return fail(GVA_ERR_FORMAT, "duplicate pattern edge");
        if (l > db.parts.size() || !db.parts[l - 1].off) absent = true;
        p.el[a][b] = p.el[b][a] = (uint8_t)l;
    }
    // connected
    uint32_t seen_m = 1, frontier = 1;
    while (frontier) {
        uint32_t nxt = 0;
        for (uint32_t a = 0; a < p.n; ++a)
            if (frontier >> a & 1)
                for (uint32_t b = 0; b < p.n; ++b)
                    if (p.el[a][b]) nxt |= 1u << b;
        frontier = nxt & ~seen_m;
        seen_m |= nxt;
    }
    if (seen_m != (1u << p.n) - 1) return fail(GVA_ERR_FORMAT, "pattern is not connected");
    return GVA_OK;
}

// The host half of an MNI run: the search tasks of a batch of patterns.
struct MniPrepared {
    size_t np = 0;
    std::vector<MniTask> tasks;
    std::vector<uint32_t> task_pat;    // pattern of each task
    std::vector<uint32_t> first_task;  // np + 1 offsets
    double prep_ms = 0.0;
};

std::shared_ptr<MniPrepared> mni_prepare(const DevDB& db, const std::vector<MniPattern>& pats,
                                         const std::vector<char>& absent, unsigned host_threads) {
    const auto t0 = std::chrono::steady_clock::now();
    auto prep = std::make_shared<MniPrepared>();
    const size_t np = pats.size();
    prep->np = np;
    std::vector<MniTask>& tasks = prep->tasks;
    std::vector<uint32_t>& task_pat = prep->task_pat;
    std::vector<uint32_t>& first_task = prep->first_task;
    first_task.assign(np + 1, 0);
    // tasks: one per automorphism orbit of each pattern whose labels all
    // occur, built on all host threads over contiguous blocks of patterns
    if (np) {
        const size_t cores = host_threads ? host_threads : std::thread::hardware_concurrency();
        const unsigned nth = (unsigned)std::max<size_t>(1, std::min<size_t>({64, cores, (np + 255) / 256}));
        std::vector<std::vector<MniTask>> tl(nth);
        std::vector<uint32_t> per_pat(np, 0);
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nth; ++t)
            pool.emplace_back([&, t]() {
                const size_t q0 = np * t / nth, q1 = np * (t + 1) / nth;
                tl[t].reserve((q1 - q0) * 3);
                for (size_t q = q0; q < q1; ++q) {
                    const MniPattern& p = pats[q];
                    if ((!absent.empty() && absent[q]) || p.n == 0) continue;
                    uint32_t orbit[kMniMaxVertices];
                    pattern_orbits(p, orbit);
                    for (uint32_t v = 0; v < p.n; ++v) {
                        if (orbit[v] != v) continue;
                        tl[t].emplace_back();
                        build_task(db, p, v, tl[t].back());
                        per_pat[q]++;
                    }
                }
            });
        for (auto& th : pool) th.join();
        for (size_t q = 0; q < np; ++q) first_task[q + 1] = first_task[q] + per_pat[q];
        tasks.reserve(first_task[np]);
        for (auto& v : tl) tasks.insert(tasks.end(), v.begin(), v.end());
        task_pat.resize(tasks.size());
        for (size_t q = 0; q < np; ++q)
            for (uint32_t t = first_task[q]; t < first_task[q + 1]; ++t) task_pat[t] = (uint32_t)q;
    }
    prep->prep_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return prep;
}

int run_mni(DevDB& db, const std::vector<MniPattern>& pats, const std::vector<char>& absent, uint32_t cap, bool plain,
            bool profile, cudaStream_t s, std::vector<uint32_t>& support, MniStats& st) {
    std::shared_ptr<MniPrepared> prep = mni_prepare(db, pats, absent);
    return mni_run_prepared(db, *prep, cap, plain, profile, s, support, st);
}

int mni_run_prepared(DevDB& db, const MniPrepared& prep, uint32_t cap, bool plain, bool profile, cudaStream_t s,
                     std::vector<uint32_t>& support, MniStats& st, const volatile int* cancel, uint32_t sm_percent) {
    const auto t_host0 = std::chrono::steady_clock::now();
    st.host_ms += prep.prep_ms;
    GVA_CUDA_M(cudaSetDevice(db.device));
    const size_t np = prep.np;
    support.assign(np, 0);
    if (np == 0) return GVA_OK;
    if (cap == 0) cap = 0xffffffffu;
    const std::vector<MniTask>& tasks = prep.tasks;
    const std::vector<uint32_t>& task_pat = prep.task_pat;
    const std::vector<uint32_t>& first_task = prep.first_task;
    const size_t nt = tasks.size();
    st.tasks += nt;
    if (nt == 0) return GVA_OK;

    // device state: tasks, per-task counts, partition pointers, per-round slots
    const size_t P = db.parts.size();
    std::vector<PartPtr> hparts(P);
    for (size_t i = 0; i < P; ++i) hparts[i] = PartPtr{db.parts[i].off, db.parts[i].adj};
    const size_t bytes_tasks = nt * sizeof(MniTask), bytes_counts = nt * 4, bytes_parts = std::max<size_t>(P, 1) * sizeof(PartPtr);
    const size_t bytes_prof = P_NUM * 8;
    void* dmem = nullptr;
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t fixed = al(bytes_tasks) + al(bytes_counts) + al(bytes_parts) + al(bytes_prof) + 256;
    if (cudaMallocAsync(&dmem, fixed, s) != cudaSuccess) return fail(GVA_ERR_NOMEM, "MNI task allocation failed");
    struct Free {
        void* p;
        cudaStream_t s;
        ~Free() { cudaFreeAsync(p, s); }
    } free_fixed{dmem, s};
    char* cur = (char*)dmem;
    MniTask* d_tasks = (MniTask*)cur;
    cur += al(bytes_tasks);
    uint32_t* d_counts = (uint32_t*)cur;
    cur += al(bytes_counts);
    PartPtr* d_parts = (PartPtr*)cur;
    cur += al(bytes_parts);
    unsigned long long* d_prof = (unsigned long long*)cur;
    cur += al(bytes_prof);
    unsigned long long* d_queue = (unsigned long long*)cur;
    // every host<->device copy goes through pinned staging: a pageable copy
    // blocks its thread inside the driver until the stream drains, which
    // other threads' CUDA calls (a server's matching loop) would wait behind
    Staging tstage, cstage;
    char* ht = tstage.get(al(bytes_tasks) + P * sizeof(PartPtr));
    uint32_t* hcounts = (uint32_t*)cstage.get(bytes_counts);
    if (!ht || !hcounts) return fail(GVA_ERR_NOMEM, "pinned staging allocation failed");
    memcpy(ht, tasks.data(), bytes_tasks);
    memcpy(ht + al(bytes_tasks), hparts.data(), P * sizeof(PartPtr));
    GVA_CUDA_M(cudaMemcpyAsync(d_tasks, ht, bytes_tasks, cudaMemcpyHostToDevice, s));
    GVA_CUDA_M(cudaMemcpyAsync(d_parts, ht + al(bytes_tasks), P * sizeof(PartPtr), cudaMemcpyHostToDevice, s));
    GVA_CUDA_M(cudaMemsetAsync(d_counts, 0, bytes_counts, s));
    GVA_CUDA_M(cudaMemsetAsync(d_prof, 0, bytes_prof, s));

    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, db.device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mni_search_kernel, kMniWarps * 32, 0);
    per_sm = std::max(per_sm, 1);

    cudaEvent_t e0 = nullptr, e1 = nullptr;
    GVA_CUDA_M(cudaEventCreate(&e0));
    GVA_CUDA_M(cudaEventCreate(&e1));
    GVA_CUDA_M(cudaEventRecord(e0, s));
    Profiler prof;

    std::vector<uint32_t> processed(nt, 0), counts(nt, 0), pcap(np, cap);
    std::vector<char> done(nt, 0);
    std::vector<MniSlot> slots;
    std::vector<uint64_t> item0;
    void* dround = nullptr;
    size_t dround_cap = 0;
    Staging stage;
    int rc = GVA_OK;
    // the plain form runs each pattern's rounds alone; the batched form all at once
    const size_t groups = plain ? np : 1;
    for (size_t g = 0; g < groups && !rc; ++g) {
        const uint32_t t_lo = plain ? first_task[g] : 0, t_hi = plain ? first_task[g + 1] : (uint32_t)nt;
        std::vector<uint32_t> active;
        for (uint32_t t = t_lo; t < t_hi; ++t) {
            if (tasks[t].seed_count == 0) {  // no vertex carries the root label
                done[t] = 1;
                pcap[task_pat[t]] = 0;
            } else {
                active.push_back(t);
            }
        }
        for (uint32_t round = 0; !active.empty(); ++round) {
            if (cancel && *cancel) {
                rc = fail(GVA_ERR_CANCELLED, "cancelled");
                break;
            }
            // retire tasks already at their pattern's cap
            size_t w = 0;
            for (uint32_t t : active)
                if (counts[t] < std::min(cap, pcap[task_pat[t]])) active[w++] = t;
            active.resize(w);
            if (active.empty()) break;
            slots.clear();
            item0.assign(1, 0);
            const uint64_t quota = (uint64_t)kMniFirst << std::min(round, 20u);
            uint64_t total = 0;
            for (uint32_t t : active) {
                const uint32_t left = tasks[t].seed_count - processed[t];
                const uint32_t len = (uint32_t)std::min<uint64_t>(left, quota);
                slots.push_back(MniSlot{t, processed[t], len, std::min(cap, pcap[task_pat[t]])});
                total += len;
            }
            // items: a whole slot per warp when there are many (its count is
            // checked every 32 seeds, so a task stops right at its cap), cut
            // down to 128 seeds when few tasks must fill the GPU
            const uint64_t want_items = (uint64_t)8 * per_sm * sms * kMniWarps;
            uint64_t item_len = std::max<uint64_t>(kMniItem, (total / want_items + 31) & ~(uint64_t)31);
            item_len = std::min<uint64_t>(item_len, 1u << 30);
            for (const MniSlot& sl : slots) item0.push_back(item0.back() + (sl.len + item_len - 1) / item_len);
            const int ns = (int)slots.size();
            const uint64_t nitems = item0.back();
            // device: slots | item0 | item -> slot (filled on the device); host stages the first two
            const size_t need = al(ns * sizeof(MniSlot)) + (ns + 1) * 8;
            const size_t dneed = al(need) + nitems * 4;
            char* h = stage.get(need);
            if (!h) {
                rc = fail(GVA_ERR_NOMEM, "pinned staging allocation failed");
                break;
            }
            if (dneed > dround_cap) {
                if (dround) cudaFreeAsync(dround, s);
                dround_cap = std::max(dneed, dround_cap * 2);
                if (cudaMallocAsync(&dround, dround_cap, s) != cudaSuccess) {
                    dround = nullptr;
                    rc = fail(GVA_ERR_NOMEM, "MNI round allocation failed");
                    break;
                }
            }
            memcpy(h, slots.data(), ns * sizeof(MniSlot));
            memcpy(h + al(ns * sizeof(MniSlot)), item0.data(), (ns + 1) * 8);
            MniSlot* d_slots = (MniSlot*)dround;
            uint64_t* d_item0 = (uint64_t*)((char*)dround + al(ns * sizeof(MniSlot)));
            uint32_t* d_item_slot = (uint32_t*)((char*)dround + al(need));
            if (cudaMemcpyAsync(dround, h, need, cudaMemcpyHostToDevice, s) != cudaSuccess ||
                cudaMemsetAsync(d_queue, 0, 8, s) != cudaSuccess) {
                rc = fail(GVA_ERR_CUDA, "MNI round upload failed");
                break;
            }
            const uint64_t slots_all = (uint64_t)per_sm * sms;
            const uint64_t cta_cap = (sm_percent == 0 || sm_percent >= 100)
                                         ? slots_all
                                         : std::max<uint64_t>(1, slots_all * sm_percent / 100);
            const uint64_t grid = std::min<uint64_t>(cta_cap, (nitems + kMniWarps - 1) / kMniWarps);
            cudaEvent_t ev = nullptr;
            const double rows = (double)total;
            mni_expand_kernel<<<(unsigned)std::min<uint64_t>((ns + 255) / 256, 4096), 256, 0, s>>>(d_item0, ns,
                                                                                                  d_item_slot);
            if (profile) prof.begin(K_MNI, 0.0, s, ev);
            mni_search_kernel<<<(unsigned)std::max<uint64_t>(grid, 1), kMniWarps * 32, 0, s>>>(
                d_tasks, d_slots, d_item0, d_item_slot, nitems, db.seed_by_degree, (uint32_t)item_len, d_parts, db.kernel_L(),
                d_counts, d_queue,
                profile ? d_prof : nullptr);
            if (profile) prof.end(ev, K_MNI, 0.0, s, rows);
            st.launches += 2;
            g_mni_launches += 2;
            st.rounds++;
            cudaError_t le = cudaGetLastError();
            if (le == cudaSuccess) le = cudaMemcpyAsync(hcounts, d_counts, bytes_counts, cudaMemcpyDeviceToHost, s);
            if (le != cudaSuccess) {
                rc = fail(GVA_ERR_CUDA, std::string("MNI search launch failed: ") + cudaGetErrorString(le));
                break;
            }
            const auto w0 = std::chrono::steady_clock::now();
            const cudaError_t e = cudaStreamSynchronize(s);
            st.wait_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
            if (e != cudaSuccess) {
                rc = fail(GVA_ERR_CUDA, std::string("MNI search failed: ") + cudaGetErrorString(e));
                break;
            }
            memcpy(counts.data(), hcounts, bytes_counts);
            // exhausted tasks fix their pattern's cap; capped ones retire
            w = 0;
            for (const MniSlot& sl : slots) {
                const uint32_t t = sl.task;
                processed[t] += sl.len;
                if (counts[t] >= sl.cap) continue;
                if (processed[t] >= tasks[t].seed_count) {
                    done[t] = 1;
                    pcap[task_pat[t]] = std::min(pcap[task_pat[t]], counts[t]);
                    continue;
                }
                active[w++] = t;
            }
            active.resize(w);
        }
    }
    if (dround) cudaFreeAsync(dround, s);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    st.gpu_ms += ms;
    if (profile) {
        unsigned long long pc[P_NUM] = {0};
        GVA_CUDA_M(cudaMemcpyAsync(pc, d_prof, bytes_prof, cudaMemcpyDeviceToHost, s));
        GVA_CUDA_M(cudaStreamSynchronize(s));
        prof.resolve();
        st.seeds += pc[P_SEEDS];
        st.roots += pc[P_ROOTS];
        st.opens += pc[P_OPENS];
        st.scanned += pc[P_SCANNED];
        st.checks += pc[P_CHECKS];
        st.found += pc[P_FOUND];
        // algorithmic bytes: seed id + 8 B per root-filter segment, 8 B per
        // segment lookup (opens, checks), 4 B per scanned candidate
        double filt = 0;
        for (const MniTask& T : tasks) filt += T.n_rootf;
        filt /= (double)nt;
        const double bytes = 4.0 * pc[P_SEEDS] * (1.0 + 2.0 * filt) + 8.0 * pc[P_OPENS] * 1.0 +
                             4.0 * pc[P_SCANNED] + 8.0 * pc[P_CHECKS];
        st.kstat.launches += prof.stat[K_MNI].launches;
        st.kstat.ms += prof.stat[K_MNI].ms;
        st.kstat.bytes += bytes;
        st.kstat.rows += (double)pc[P_SEEDS];
    }
    for (size_t q = 0; q < np; ++q) {
        if (first_task[q] == first_task[q + 1]) {
            support[q] = 0;
            continue;
        }
        uint32_t m = cap;
        for (uint32_t t = first_task[q]; t < first_task[q + 1]; ++t) m = std::min(m, counts[t]);
        support[q] = m;
    }
    st.host_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_host0).count();
    return GVA_OK;
}

}  // namespace gva
