// Internal types shared by the host library and the CUDA engine.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <utility>
#include <string>
#include <vector>

namespace gva {

constexpr uint32_t kNone = 0xffffffffu;
// bit of the label count handed to kernels that marks a packed segment index
// (seg_of in gva_kernels.cuh)
constexpr uint32_t kPackedSeg = 0x80000000u;
constexpr int kMaxCols = 32;

// ---------------------------------------------------------------- errors ----
void set_error(int status, const std::string& msg);  // thread-local message
int fail(int status, const std::string& msg);         // set_error + return status
const char* last_error_cstr();                        // this thread's last message

// ----------------------------------------------------------------- graph ----
// Host copy of one database: per edge label a CSR whose per-vertex lists are
// sorted by (dense vertex label, vertex id), plus a dense (vertex, label) ->
// offset table.  seg(v, l) = adj[off[v*L + l] .. off[v*L + l + 1]).
// Allocator whose default construction leaves plain values uninitialised:
// the offset tables below are written in full by their builders, so zeroing
// them first would only add a pass over memory (and its page faults on one
// thread).
template <typename T>
struct NoInitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <typename U>
    NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
    template <typename U>
    void construct(U* p) noexcept {
        ::new ((void*)p) U;
    }
    template <typename U, typename... A>
    void construct(U* p, A&&... a) {
        ::new ((void*)p) U(std::forward<A>(a)...);
    }
};

struct HostPartition {
    uint32_t edge_label = 0;                            // 1..P
    std::vector<uint32_t, NoInitAlloc<uint32_t>> off;   // (max_id + 1) * L + 1 entries, each written by the builder
    std::vector<uint32_t> adj;                          // neighbour ids
};

struct HostGraph {
    uint32_t max_id = 0;                 // vertex ids are 1..max_id
    std::vector<uint32_t> vlabel;        // original label per id (max_id + 1)
    std::vector<uint32_t> labels;        // sorted distinct original labels
    std::vector<uint32_t> dlabel;        // dense label per id (max_id + 1)
    std::vector<HostPartition> parts;    // parts[p - 1] is edge label p
    uint32_t num_labels() const { return (uint32_t)labels.size(); }
    // dense index of an original label, kNone when absent from the data
    uint32_t dense_label(uint32_t orig) const;
};

// Parses .metadata + .mygraph (src/loadDataBase.cpp:309-365 layout).
int load_mygraph(const std::string& mygraph, const std::string& metadata, HostGraph& g,
                 std::string* warnings);
// Builds from an edge list (tools/genDatabase.cpp:600-667 semantics, no renumbering).
int graph_from_edges(const uint32_t* vlabels, uint32_t max_id, const uint32_t* src, const uint32_t* dst,
                     const uint32_t* elabel, uint64_t ne, HostGraph& g);

// Init-phase frontiers: vertices grouped by dense label (seed_off[l] ..
// seed_off[l + 1] of seed_verts, ascending id) and the same groups ordered by
// total degree, largest first, ties by id (seed_by_degree).
void seed_groups(const HostGraph& g, std::vector<uint32_t>& seed_off, std::vector<uint32_t>& seed_verts,
                 std::vector<uint32_t>& seed_by_degree);

// .g -> .mygraph/.metadata/.reorder exactly as tools/genDatabase.cpp writes them.
int convert_g(const std::string& g_path, const std::string& mygraph, const std::string& metadata,
              const std::string& reorder);

// ----------------------------------------------------------------- plan -----
struct Phase {
    char type = 'E';                  // 'E' extension, 'R' reduction
    uint32_t edge_label = 0;
    std::vector<uint32_t> pairs;      // (svid, evid) pairs, flattened
};

struct Plan {
    int mode = 0;                                  // GVA_MODE_DV / GVA_MODE_SV
    uint32_t vnum = 0;
    std::vector<uint32_t> qlabel;                  // query vertex -> label
    std::vector<Phase> phases;
    std::vector<uint32_t> restricts;               // vnum + 1 entries (kNone = none)
    std::map<uint64_t, uint32_t> repeat_flag;      // (edge label << 32 | vlabel) -> flag
    std::map<uint32_t, std::vector<uint32_t>> record_stat;  // edge label -> vlabels
    std::vector<uint32_t> columns;                 // query vertex of each output column
    std::string describe() const;
};

int plan_from_text(const std::string& text, int mode, Plan& out);
// A query text's vertex labels (by id 0..n-1, first definition wins) and edge
// lines (source, target, label) in text order, read by the planner's rules;
// the vertex checks of the planner are made here, the edge checks by it.
int read_query_text(const std::string& text, std::vector<uint32_t>& labels, std::vector<uint32_t>& sdl);
// The same plan for the query "v i labels[i]" (i < n) followed by the edges
// "e sdl[3j] sdl[3j+1] sdl[3j+2]" (j < ne), without the text.
int plan_from_query(uint32_t n, const uint32_t* labels, const uint32_t* sdl, size_t ne, int mode, Plan& out);
// A plan computed by dplan (gva_dplan.h; status DPLAN_OK) as a Plan.
struct DPlan;
int plan_from_dplan(const DPlan& d, const uint32_t* labels, Plan& out);

// ---------------------------------------------------------------- steps -----
// A plan lowered to engine steps.  Every reference phase becomes one or more
// steps; the row set after the last step of a phase equals the reference's
// rows after that phase.
enum StepKind : uint32_t { STEP_SEED = 0, STEP_EXT = 1, STEP_REDUCE = 2 };

struct Step {
    StepKind kind = STEP_EXT;
    uint32_t width_in = 0;         // columns read
    uint32_t part = 0;             // edge label partition (1-based), 0 = absent
    uint32_t label = kNone;        // dense candidate label (SEED: source label)
    int32_t src_col = -1;          // EXT: column of the source vertex
    int32_t bound_col = -1;        // EXT: candidate < row[bound_col] (or <=)
    uint32_t bound_inclusive = 0;
    uint32_t n_eq = 0;             // EXT: injectivity columns
    uint8_t eq_cols[kMaxCols] = {};
    // REDUCE: pairs of (svid column, evid column, dense label of evid)
    uint32_t n_pairs = 0;
    uint8_t rs_col[16] = {}, re_col[16] = {};
    uint32_t re_label[16] = {};
    uint32_t always_empty = 0;     // reference limit reached (>16 pairs) or label absent
    int phase_end = -1;            // reference phase index completed by this step, else -1
    // EXT with fused back edges (lowered with fuse_reductions): the candidate
    // must also be adjacent to row[chk_col[i]] in partition chk_part[i];
    // dir 0 looks the candidate up in the partner's segment, dir 1 the
    // partner in the candidate's (the reference's pair orientation)
    uint32_t n_chk = 0;
    uint8_t chk_col[8] = {}, chk_dir[8] = {};
    uint32_t chk_part[8] = {}, chk_lab[8] = {};
};

// fuse_reductions: fold each reduction that only checks edges of the vertex
// just added into that extension (same final rows, fewer steps; per-phase
// counts of the folded phases are then not observable).
int lower_plan(const Plan& plan, const HostGraph& g, std::vector<Step>& steps, bool fuse_reductions = false);
// The same steps for a plan of the heap-free planner (status DPLAN_OK) over
// the query's labels, without building the host plan.
int lower_dplan(const DPlan& plan, const uint32_t* labels, const HostGraph& g, std::vector<Step>& steps,
                bool fuse_reductions = false);

// ----------------------------------------------------------------- text ----
// Rows [0, n) of `width` values as text (one line per row, decimal values
// separated by single spaces), formatted on up to `threads` threads; the
// text is the concatenation of `parts` in order.
void format_rows(const uint32_t* rows, uint64_t n, uint32_t width, unsigned threads, std::vector<std::string>& parts);

// ---------------------------------------------------------------- mining ---
struct MinedPattern {
    std::string text;  // query text, vertices in canonical order
    uint32_t edges;
    uint32_t support;
    uint64_t embeddings;
};

}  // namespace gva
