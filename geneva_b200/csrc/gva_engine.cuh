// Device-side database and the phase executor interface.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <atomic>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "gva_internal.h"

namespace gva {

struct DevPart {
    const uint32_t* off = nullptr;  // (max_id + 1) * L + 1 label-segment offsets
    const uint32_t* adj = nullptr;  // neighbour ids
    uint64_t n_adj = 0;
};

// One database resident in HBM.  A single allocation holds, 256-byte aligned:
//   seed_verts[...] | seed_by_degree[...] | per partition: off[...] adj[...]
struct DevDB {
    int device = 0;
    uint32_t max_id = 0;
    uint32_t L = 0;                       // dense vertex labels
    bool packed = false;                  // segment index layout (seg_of): packed records, else dense
    uint32_t kernel_L() const { return L | (packed ? kPackedSeg : 0u); }  // the label count kernels take
    std::vector<uint32_t> labels;         // dense -> original label
    std::vector<DevPart> parts;           // parts[p - 1] = edge label p (off == nullptr: absent)
    std::vector<uint32_t> seed_off;       // host copy of seed_off
    const uint32_t* seed_verts = nullptr; // vertices grouped by dense label, ascending id
    const uint32_t* seed_by_degree = nullptr;  // same groups (seed_off), by degree descending
    void* arena = nullptr;
    size_t arena_bytes = 0;
    uint64_t n_adj = 0;
    HostGraph meta;                       // labels/partition presence for lowering (no adjacency)
    uint32_t* vgraph = nullptr;           // optional vertex -> graph id map (graph databases)
    uint32_t num_graphs = 0;
    // launch shape of the batched engine's round kernels (autotune_batch)
    uint32_t tune_rows_per_item = 64, tune_hub = 32;
    // frontier budget of batched runs given none: 3/4 of the device memory
    // free when the first such run started (querying it costs a driver call)
    uint64_t default_budget = 0;
    // device-scheduled rounds (BatchSession::run_device): bytes of each of a
    // run's two frontier regions; doubled after a run that overflowed them
    std::atomic<uint64_t> round_region_bytes{0};
};

int upload_graph(HostGraph& g, int device, DevDB*& out);
void free_devdb(DevDB* db);

enum KernelKind { K_EXT_COUNT = 0, K_EXT_WRITE, K_RED_COUNT, K_RED_WRITE, K_SCAN, K_MNI, K_NUM };
extern const char* const kKernelNames[K_NUM];

struct KernelStat {
    uint64_t launches = 0;
    double ms = 0.0;
    double bytes = 0.0;
    double rows = 0.0;  // frontier rows read (scan: blocks)
};

// Optional per-launch CUDA-event timing.
struct Profiler {
    bool on = false;
    struct Pending { int kind; cudaEvent_t a, b; double bytes, rows; };
    std::vector<Pending> pending;
    KernelStat stat[K_NUM];
    void begin(int kind, double bytes, cudaStream_t s, cudaEvent_t& a);
    void end(cudaEvent_t a, int kind, double bytes, cudaStream_t s, double rows = 0.0);
    void resolve();  // after a stream sync
};

uint64_t kernel_launches();

struct MatchResult {
    int device = 0;
    uint64_t rows = 0;
    uint32_t width = 0;
    uint32_t* rows_dev = nullptr;         // owned (cudaMallocAsync pool), may be null
    cudaStream_t stream = nullptr;
    std::vector<uint64_t> phase_rows;
    double gpu_ms = 0.0;
    std::vector<uint32_t> columns;
    KernelStat kstat[K_NUM];
};

int run_match(DevDB& db, const Plan& plan, const std::vector<Step>& steps, cudaStream_t stream, uint64_t budget,
              bool count_only, bool profile, MatchResult& res);
void free_result(MatchResult* r);

struct BatchStats {
    double gpu_ms = 0.0;
    double submit_ms = 0.0, round_host_ms = 0.0, wait_ms = 0.0;
    double phase_ms[5] = {0, 0, 0, 0, 0};
    double session_ms = 0.0;  // session set-up, support read-back and tear-down
    uint64_t rounds = 0, splits = 0, launches = 0, nodes = 0;
    uint64_t device_rounds = 0;
    KernelStat kstat[K_NUM];
    // wall-clock marks of one run (ms from its start): plans ordered, then
    // per half (two at most) session prepared, rounds done, results read,
    // session freed
    double timeline_ms[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double loop_end_ms = 0.0;  // finish_batch: rounds done, ms after its start
    double read_end_ms = 0.0;  // finish_batch: results read, ms after its start
};

// Counts the embeddings of many plans in shared rounds.  counts[q] always;
// graph_counts [nq * G] and support [nq] when given (need db.vgraph).
// Serialised parameters of a step (everything that decides its output from
// its input); two steps are the same trie node when these bytes and their
// parents agree.  buf must hold 512 bytes.
size_t step_key_bytes(const Step& st, uint8_t* buf);
// 64-bit hash of the same fields, never 0 (a sort key: equal keys hash equal)
uint64_t step_key_hash(const Step& st);

// Round scheduling of run_batch: ROUNDS_AUTO = on the device when the run is
// one piece, on the host when it runs as two halves
enum RoundsMode { ROUNDS_AUTO = 0, ROUNDS_HOST = 1, ROUNDS_DEVICE = 2 };
int run_batch(DevDB& db, std::vector<std::vector<Step>> steps, cudaStream_t s, uint64_t budget,
              const uint32_t* vgraph, uint32_t G, uint64_t* counts, uint64_t* graph_counts_host,
              uint32_t* support_host, bool profile, BatchStats* stats, int rounds = ROUNDS_AUTO);
uint64_t batch_kernel_launches();

// Pinned host staging, grown on demand.
struct Staging {
    char* p = nullptr;
    size_t cap = 0;
    char* get(size_t need);
    ~Staging();
};

// Persistent batched engine (gva_batch.cu).  Plans are submitted in waves;
// round() advances every active task one step; completed plans are reported
// by take_completed().  Per-graph results need slots > 0 (one per live plan).
class BatchSession {
public:
    // Trie node.  The few step fields every round reads are copied here so a
    // round's passes over its tasks stay in a small array; the full step
    // lives in node_steps.
    struct BNode {
        uint32_t kind = 0, width_in = 0, n_eq = 0, n_pairs = 0;
        uint32_t always_empty = 0;
        uint32_t fused = 0;  // an extension with fused back-edge checks (its own round kernels)
        int depth = 0;
        int parent = -1;
        int first_child = -1, next_sibling = -1;  // children as a linked list
        int first_term = -1;                       // plans ending here, linked through PlanRec::next_term
        int at = 0;                                // active tasks at this node
        bool closed = false;
    };
    struct BTask {
        int node;
        const uint32_t* in;  // frontier slice
        uint64_t rows;
        std::shared_ptr<void> owner;
    };
    struct PlanRec {
        uint64_t tag = 0;
        int slot = -1;
        int terminal = -1;
        int next_term = -1;
        uint64_t count = 0;
        bool done = false;
        bool released = false;
    };

    BatchSession(DevDB& db, cudaStream_t s, uint64_t budget, uint32_t slots, bool graph_counts, bool profile);
    ~BatchSession();
    int init();
    // presorted: the plans come in order of their step keys (plans sharing a
    // prefix are adjacent); the trie is then built without a hash index
    // The session keeps the submitted steps (moved in, not copied: trie nodes
    // point at them).
    int submit(std::vector<std::vector<Step>>&& steps, const std::vector<uint64_t>& tags, std::vector<int>* ids,
               bool presorted = false);
    int submit(const std::vector<std::vector<Step>>& steps, const std::vector<uint64_t>& tags, std::vector<int>* ids,
               bool presorted = false) {
        std::vector<std::vector<Step>> copy(steps);
        return submit(std::move(copy), tags, ids, presorted);
    }
    int round();
    // Runs every round of a single-wave session on the device: each round's
    // planning kernel chooses the writing tasks, places their outputs and
    // lists the next round's tasks, so the host launches all rounds at once
    // and synchronises once.  Leaves the session idle with every plan's count
    // set; or, when the session does not qualify (several waves, profiling,
    // rounds already run, a budget below the frontier regions) or a round
    // overflowed its region, leaves the initial tasks active for round().
    int run_device();
    bool idle() const { return active.empty(); }
    std::vector<int> take_completed();
    const PlanRec& plan(int q) const { return plans[q]; }
    // the plan whose slot holds q's per-graph results: the head of the list of
    // plans ending on q's node (the node descriptor names that slot)
    int first_peer(int q) const { return nodes[plans[q].terminal].first_term; }
    int read_support(int q, uint32_t* support, uint64_t* graph_counts_host);
    void release(int q);
    size_t num_nodes() const { return nodes.size(); }
    const BNode& node(int id) const { return nodes[id]; }           // trie introspection (host only)
    const Step& node_step(int id) const { return *node_steps[id]; }
    cudaStream_t stream() const { return s; }
    size_t num_active() const { return active.size(); }
    uint32_t words() const { return ctx_words; }
    uint64_t* graph_counts_dev() const;
    uint32_t* graph_bits_dev() const;

    // Launch shape of the round kernels: rows per work item (a multiple of
    // 32, at most 128; fewer when rows are wide) and the candidate-list length
    // above which a row's candidates are shared by its whole warp.
    struct Tuning {
        uint32_t rows_per_item = 64;
        uint32_t hub = 32;
    } tune;

    uint64_t rounds = 0, splits = 0, launches = 0;
    uint64_t device_rounds = 0;  // rounds scheduled on the device (run_device)
    bool host_rounds = false;    // run_device declines: every round scheduled on the host
    double submit_ms = 0, round_host_ms = 0, wait_ms = 0;  // host time split
    // round_host_ms by part: task scan + uploads, count launches, totals and
    // budget choice, write launch, next tasks and completion
    double phase_ms[5] = {0, 0, 0, 0, 0};
    KernelStat kstat[K_NUM];

private:
    void add_task(int node, const uint32_t* in, uint64_t rows, std::shared_ptr<void> owner);
    void start_seeds(int first_node);  // tasks of the seed nodes' children, from the seed vertex lists
    int ship_nodes();                  // descriptors of nodes submitted since the last shipment
    void fill_node_desc(int id, void* out) const;
    void finish_task(int node);
    void try_close(int node);

    DevDB& db;
    cudaStream_t s;
    uint64_t budget;
    uint32_t nslots;
    bool want_graph_counts;
    bool profile;
    bool per_graph = false;
    uint32_t ctx_words = 0;
    size_t acc_bytes = 0;  // per-graph counters and bitmaps (acc)
    int sms = 148;
    void* acc = nullptr;
    std::vector<int> free_slots;
    std::vector<BNode> nodes;
    std::vector<const Step*> node_steps;  // parallel to nodes, into `waves`
    std::vector<std::vector<std::vector<Step>>> waves;  // every submitted wave's steps
    std::vector<PlanRec> plans;
    std::vector<BTask> active;
    std::vector<int> completed;
    Staging staging;
    cudaEvent_t staged = nullptr;  // marks the last copies out of `staging`
    void* d_nodes = nullptr;       // per-node step descriptors (layout private to gva_batch.cu), by node id
    size_t node_cap = 0;
    size_t shipped = 0;            // nodes whose descriptors are on the device
    std::vector<unsigned char> desc_host;  // descriptors filled at submit, shipped by the next round
                                           // (sessions never initialised: no device)
    // initialised sessions fill the descriptors into pinned memory instead,
    // so that shipping them is an asynchronous copy; desc_ev marks the last
    // copy out of it (the buffer is refilled only after that copy landed)
    bool inited = false;
    char* desc_pin = nullptr;
    size_t desc_pin_cap = 0;
    cudaEvent_t desc_ev = nullptr;
    bool desc_pending = false;
    std::vector<int> scratch_order;
    std::vector<char> scratch_flag;
    std::vector<uint64_t> scratch_off;
    void* d_desc = nullptr;  // per-round task references
    size_t desc_cap = 0;
    uint64_t* d_items = nullptr;  // per-round item counts, scanned in place
    size_t items_cap = 0;
    uint64_t* d_chunks = nullptr;  // per-round scan chunk sums
    size_t chunks_cap = 0;
    uint64_t* d_small = nullptr;
    size_t small_cap = 0;
    unsigned long long* d_read = nullptr;  // profiling: candidate-list words read
    Staging staging_read;  // pinned landing area of per-plan support read-backs
};
// run_batch in two halves, so that a caller can build the next batch's
// session (device set-up and step trie, host work) while the previous one's
// rounds run: prepare_batch may run on another thread than finish_batch.
struct PreparedBatch {
    std::unique_ptr<BatchSession> ses;
    std::vector<int> ids;
    int nq = 0;
    bool per_graph = false, graph_counts = false;
    double prep_ms = 0.0;
};
// host_rounds: finish_batch schedules every round on the host (else on the
// device when the session qualifies, BatchSession::run_device)
int prepare_batch(DevDB& db, std::vector<std::vector<Step>>&& steps, cudaStream_t s, uint64_t budget,
                  bool per_graph, bool graph_counts, bool profile, PreparedBatch& out, bool presorted = false,
                  bool host_rounds = false);
// order (optional): plan q's results go to index order[q] of the arrays
int finish_batch(DevDB& db, PreparedBatch& pb, uint64_t* counts, uint64_t* graph_counts_host, uint32_t* support_host,
                 BatchStats* stats, const volatile int* cancel = nullptr, const uint32_t* order = nullptr);
int set_graph_ids(DevDB& db, const uint64_t* first, uint32_t num_graphs);

// Times the batched count of `steps` (a calibration batch) under each
// candidate launch shape of the round kernels and stores the fastest in db.
struct TuneResult {
    uint32_t rows_per_item = 64, hub = 32;
    double ms = 0.0, default_ms = 0.0;
    std::vector<std::array<double, 3>> tried;  // rows per item, hub, ms
};
int autotune_batch(DevDB& db, const std::vector<std::vector<Step>>& steps, cudaStream_t s, bool per_graph,
                   TuneResult& out);

struct MineStats {
    uint64_t candidates = 0, frequent = 0, embeddings = 0, levels = 0, pruned = 0;
    uint64_t mni_tasks = 0, mni_rounds = 0, mni_found = 0;  // MNI mode
    double gpu_ms = 0.0, host_ms = 0.0, gen_ms = 0.0, plan_ms = 0.0, eval_ms = 0.0, merge_ms = 0.0;
    double submit_ms = 0.0, round_host_ms = 0.0, wait_ms = 0.0;
    double phase_ms[5] = {0, 0, 0, 0, 0};
    double session_ms = 0.0;
    KernelStat kstat[K_NUM];
};

// Frequent connected patterns with up to max_edges edges (support = graphs).
typedef int (*ReduceFn)(uint32_t* supports, uint64_t* embeddings, uint64_t n, void* user);
// support_mode GVA_SUPPORT_GRAPHS: graphs holding an embedding (needs graph
// ids); GVA_SUPPORT_MNI: min(MNI, mni_cap) on the whole data graph (mni_cap 0
// = min_support, which decides frequency).
int run_mine(DevDB& db, cudaStream_t s, uint64_t budget, uint32_t max_edges, uint32_t min_support,
             uint32_t batch_limit, bool profile, ReduceFn reduce, void* reduce_user, uint32_t support_mode,
             uint32_t mni_cap, std::vector<MinedPattern>& out, MineStats& st, const volatile int* cancel = nullptr,
             uint32_t sm_percent = 0, uint32_t host_threads = 0);

// mine_levels with a caller-supplied evaluator of candidate query texts
// (host only; gva_mine_host).
typedef int (*TextEvalFn)(const char* text, const uint64_t* offsets, uint64_t n, uint32_t* supports,
                          uint64_t* embeddings, void* user);
int run_mine_host(const std::vector<uint32_t>& labels, uint32_t num_edge_labels, const uint8_t* has_edge_label,
                  uint32_t max_edges, uint32_t min_support, uint32_t host_threads, TextEvalFn evaluate,
                  void* eval_user, ReduceFn reduce, void* reduce_user, std::vector<MinedPattern>& out, MineStats& st);

// ---- single-graph MNI support (gva_mni.cu) ----
constexpr int kMniMaxVertices = 8;
// A connected pattern: dense vertex labels, el[a][b] = partition (1-based
// edge label) of edge (a, b), 0 = no edge.
struct MniPattern {
    uint32_t n = 0;
    uint32_t vl[kMniMaxVertices] = {};
    uint8_t el[kMniMaxVertices][kMniMaxVertices] = {};
};
struct MniStats {
    double gpu_ms = 0.0, host_ms = 0.0, wait_ms = 0.0;
    uint64_t rounds = 0, launches = 0, tasks = 0;
    uint64_t seeds = 0, roots = 0, opens = 0, scanned = 0, checks = 0, found = 0;  // filled when profiling
    KernelStat kstat;
};
// Parses a .query-format pattern; `absent` is set when a label or edge label
// does not occur in the database (support 0).
int mni_pattern_from_text(const DevDB& db, const std::string& text, MniPattern& p, bool& absent);
// support[q] = min(MNI of pats[q], cap) (cap 0 = exact); absent[q] != 0 gives 0.
// plain: one pattern's rounds at a time instead of all patterns together.
int run_mni(DevDB& db, const std::vector<MniPattern>& pats, const std::vector<char>& absent, uint32_t cap, bool plain,
            bool profile, cudaStream_t s, std::vector<uint32_t>& support, MniStats& st);
uint64_t mni_kernel_launches();
// run_mni in two halves: the host half (orbits, search orders, task records;
// no device work, may run on another thread) and the device rounds.
struct MniPrepared;
std::shared_ptr<MniPrepared> mni_prepare(const DevDB& db, const std::vector<MniPattern>& pats,
                                         const std::vector<char>& absent, unsigned host_threads = 0);
// sm_percent: the search kernel's persistent grid fills at most this share of the SMs (0 = all)
int mni_run_prepared(DevDB& db, const MniPrepared& prep, uint32_t cap, bool plain, bool profile, cudaStream_t s,
                     std::vector<uint32_t>& support, MniStats& st, const volatile int* cancel = nullptr,
                     uint32_t sm_percent = 0);

// ---- device-side planning (gva_dplan.cu) ----
// Fixed-size query records and compact plans exchanged with the planning
// kernel (dplan on the device, one query per thread).
constexpr int kDevPlanV = 16, kDevPlanLines = 32, kDevPlanPhases = 32, kDevPlanPairs = 96, kDevPlanKeys = 64;
struct DevPlanQuery {
    uint32_t n, lines;
    uint32_t label[kDevPlanV];
    uint8_t s[kDevPlanLines], d[kDevPlanLines];
    uint32_t l[kDevPlanLines];
};
struct DevPlanOut {
    uint32_t status, vnum, nphase, npair;
    uint32_t restricts[kDevPlanV + 1];
    uint32_t ph_el[kDevPlanPhases];
    uint8_t ph_type[kDevPlanPhases], ph_at[kDevPlanPhases], ph_np[kDevPlanPhases];
    uint8_t pairs[kDevPlanPairs];
    uint32_t nrep, nstat, ncol, pad;  // repeat flags, record stats and columns (the plan text; not lowered)
    uint64_t rep_key[kDevPlanKeys];
    uint32_t rep_val[kDevPlanKeys];
    uint32_t stat_el[kDevPlanKeys], stat_vl[kDevPlanKeys];
    uint8_t columns[kDevPlanV];
};
struct DPlan;
// Plans n queries on `device` (blocking: the plans are on the host when it returns).
int plan_on_device(int device, cudaStream_t s, const DevPlanQuery* qs, uint32_t n, DevPlanOut* outs);
// The host-side DPlan of a device plan: the fields lowering reads.
void dplan_from_device(const DevPlanOut& o, DPlan& p);
uint64_t dplan_kernel_launches();

size_t step_scratch_bytes(uint64_t in_rows);
// run_step with the library's fixed device scratch array (no allocation).
int run_step_static(DevDB& db, const Step& st, const uint32_t* in, uint64_t in_rows, uint32_t* out,
                    uint64_t out_cap, uint64_t* out_rows, cudaStream_t stream);
int run_step(DevDB& db, const Step& st, const uint32_t* in, uint64_t in_rows, uint32_t* out, uint64_t out_cap,
             uint64_t* out_rows, void* scratch, size_t scratch_bytes, cudaStream_t stream);

}  // namespace gva
