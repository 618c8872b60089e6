/*
 * geneva.h — C ABI of the B200-native Geneva subgraph-matching path.
 *
 * The reference drives its GPU path from C++ with no stable boundary: a CLI
 * (`gpumine`, `gpumineSV`), a loader returning std::map<uint, uint*>, a planner
 * filling std::vector<Phase>, and void kernel launchers that read their row
 * counts back through a device word.  This header replaces that surface with
 * plain pointers, sizes and int status codes.  Every entry point names the
 * reference interface it replaces (paths relative to the reference project).
 *
 * Conventions
 *   - Data vertex ids are 1-based uint32 (0 is never a vertex), query vertex
 *     ids are 0-based, as in the reference (src/gpumine.cpp:1-3).
 *   - A frontier ("partial embedding" table) is row-major uint32 with one
 *     column per matched query vertex, columns in match order — the order the
 *     reference prints them (src/gpumine.cpp:184-199).
 *   - Row counts are uint64 (the reference uses uint32, src/gpumine.cpp:904).
 *   - Functions return GVA_OK (0) or a positive GVA_ERR_* code; the message of
 *     the last failure on the calling thread is gva_last_error().  Nothing in
 *     the library calls exit() (the reference does, src/loadDataBase.cpp:311-319).
 *   - `stream` arguments are cudaStream_t passed as void* (NULL = the legacy
 *     default stream).  Device pointers are CUDA device addresses.
 */
#ifndef GENEVA_H
#define GENEVA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GVA_OK 0
#define GVA_ERR_IO 1          /* file missing or unreadable                 */
#define GVA_ERR_FORMAT 2      /* malformed .mygraph/.metadata/.query/.g     */
#define GVA_ERR_CUDA 3        /* a CUDA runtime call failed                  */
#define GVA_ERR_NOMEM 4       /* device or host allocation failed / budget  */
#define GVA_ERR_ARG 5         /* bad argument (null, out of range, size)    */
#define GVA_ERR_UNSUPPORTED 6 /* outside the reference's limits (see docs)  */
#define GVA_ERR_CANCELLED 7   /* the caller's cancel flag was set            */

#define GVA_MODE_DV 0 /* genMatchOrder        (src/genMatchOrder.cpp:672)       */
#define GVA_MODE_SV 1 /* genMatchOrderSingleV (src/genMatchOrderSingleV.cpp:678) */

#define GVA_MAX_QUERY_VERTICES 32 /* bitmask planner limit, src/gpumine.cpp:123-124 */
#define GVA_MAX_REDUCE_PAIRS 16   /* src/reduction.cu auxArray, src/gpumine.cpp:759-762 */

typedef struct gva_db gva_db;         /* device-resident database            */
typedef struct gva_plan gva_plan;     /* match order + restrictions          */
typedef struct gva_result gva_result; /* final frontier + per-phase counts   */

typedef struct gva_db_info {
    uint32_t max_vertex_id;   /* vLabel[0] in the reference                  */
    uint32_t num_vertex_labels;
    uint32_t num_partitions;  /* edge labels 1..num_partitions               */
    uint32_t reserved;
    uint64_t num_adjacency;   /* directed adjacency entries, all partitions  */
    uint64_t device_bytes;    /* HBM held by the database                    */
} gva_db_info;

typedef struct gva_match_opts {
    void* stream;          /* cudaStream_t; NULL = legacy default stream             */
    uint64_t budget_bytes; /* frontier memory cap (0 = 3/4 of free HBM at call time)  */
    int count_only;        /* 1: the last phase only counts (no final rows kept)      */
    int profile;           /* 1: time every kernel with CUDA events (gva_result_kernel_stats) */
} gva_match_opts;

/* Per-kernel totals of one profiled gva_match: launches, summed CUDA-event
 * milliseconds, and algorithmic bytes (the minimum traffic the kernel's
 * arithmetic needs: rows read and written, one 8-byte segment lookup per
 * row and pair, one 4-byte neighbour read per produced row). */
typedef struct gva_kernel_stat {
    char name[24];
    uint64_t launches;
    double ms;
    double bytes;
    double rows; /* frontier rows read (scan kernel: 256-row blocks) */
} gva_kernel_stat;

/* ---- status -------------------------------------------------------------- */
const char* gva_last_error(void);
const char* gva_status_string(int status);
const char* gva_version(void);
/* Kernels this library has launched in this process (all devices). */
uint64_t gva_kernel_launches(void);

/* ---- L1: database ---------------------------------------------------------
 * Replaces loadDataBase(mygraph, metadata) (src/loadDataBase.cpp:309-365,
 * include/loadDataBase.h:1) plus the per-phase partition upload of
 * src/gpumine.cpp:885-911,999-1006.  All edge-label partitions are uploaded
 * once, as label-sorted CSR with a (vertex, label) -> segment offset table, so
 * kernels never search labels.  Index vertices (tools/genDatabase.cpp:415-436)
 * are stripped.  Partitions are keyed 1..P in file order, as the reference. */
int gva_db_load(const char* mygraph_path, const char* metadata_path, int device, gva_db** out);

/* Builds the same database from an in-memory labelled edge list with the
 * semantics of tools/genDatabase.cpp:600-667 (undirected, duplicate edges
 * dropped) but without renumbering: vertex v keeps id v.  vertex_labels has
 * max_vertex_id + 1 entries (entry 0 ignored); edge labels are 1..P. */
int gva_db_from_edges(const uint32_t* vertex_labels, uint32_t max_vertex_id, const uint32_t* src,
                      const uint32_t* dst, const uint32_t* edge_labels, uint64_t num_edges, int device,
                      gva_db** out);
int gva_db_get_info(const gva_db* db, gva_db_info* out);
/* Host-only parse of .mygraph + .metadata (no device needed): fills the
 * counts of gva_db_info (device_bytes = bytes an upload would take) and
 * copies loader notes into warn (may be NULL). */
int gva_graph_probe(const char* mygraph_path, const char* metadata_path, gva_db_info* out, char* warn, size_t cap);
/* Loader notes (e.g. a header that declares more partitions than the file
 * holds, or neighbours dropped past 256 intervals); "" when none. */
const char* gva_db_warnings(const gva_db* db);
void gva_db_free(gva_db* db);

/* Converts a .g file (`v id label`, then `e src dst label` lines) into the
 * reference's database files, byte-identical to tools/genDatabase.cpp
 * (vertex renumbering :259-413, index vertices :415-436, partition layout
 * :451-580, .reorder text :826-846, .metadata :873-879).  Host-only. */
int gva_convert_g(const char* g_path, const char* mygraph_path, const char* metadata_path, const char* reorder_path);

/* ---- L2: planner ----------------------------------------------------------
 * Replaces genMatchOrder / genMatchOrderSingleV (src/genMatchOrderCPU.cpp:670-983,
 * src/genMatchOrderSingleV.cpp:678-1003): same phases, pair orientation,
 * restrictions and repeat flags for the same query text.  Host-only. */
int gva_plan_from_file(const char* query_path, int mode, gva_plan** out);
int gva_plan_from_text(const char* query_text, int mode, gva_plan** out);
/* gva_plan_batch for DV plans computed on `device` by the device planner
 * (the heap-free planner, one query per thread; queries of up to 16 vertices
 * and 32 edge lines, others planned on the host): the same plans as the host
 * planner (genMatchOrder, src/genMatchOrderCPU.cpp:670-983). */
int gva_plan_batch_device(int device, const char* const* query_texts, int n, gva_plan** out, int* status);
/* gva_plan_from_text for n queries at once on the host's cores (a batch or a
 * serving wave planned in one call): out[i] receives query i's plan (NULL on
 * failure) and status[i] (may be NULL) its status; the call returns the first
 * failure's status with its message, or GVA_OK.  Same plans as planning the
 * queries one by one. */
int gva_plan_batch(const char* const* query_texts, int n, int mode, gva_plan** out, int* status);
/* Canonical text: "vnum", "phase", "restrict", "repeat", "stat" lines.
 * Returns the needed length (excluding NUL); writes at most cap bytes. */
size_t gva_plan_describe(const gva_plan* plan, char* buf, size_t cap);
int gva_plan_num_phases(const gva_plan* plan);
int gva_plan_num_vertices(const gva_plan* plan);
/* query vertex id of each output column (match order, src/gpumine.cpp:158) */
int gva_plan_column_vertices(const gva_plan* plan, uint32_t* out, int cap);
void gva_plan_free(gva_plan* plan);

/* ---- L3: one query end to end -----------------------------------------------
 * Replaces the phase loop of gpumine / gpumineSV main (src/gpumine.cpp:932-1061):
 * init, every E and R phase, frontier growth handled by chunking against
 * budget_bytes instead of host spill.  The result stays on the device. */
int gva_match(gva_db* db, const gva_plan* plan, const gva_match_opts* opts, gva_result** out);
uint64_t gva_result_num_rows(const gva_result* res);
int gva_result_num_columns(const gva_result* res);
/* rows after each reference phase (index 0 = init) */
int gva_result_phase_rows(const gva_result* res, uint64_t* out, int cap);
/* device pointer to the row-major final rows (NULL when count_only) */
const uint32_t* gva_result_device_rows(const gva_result* res);
int gva_result_copy_rows(const gva_result* res, uint32_t* host_dst, uint64_t first_row, uint64_t num_rows);
/* partialResultsGPU.txt format (src/gpumine.cpp:184-199) */
int gva_result_write_text(const gva_result* res, const char* path);
/* GPU time of the phase loop, from CUDA events on opts->stream */
double gva_result_gpu_ms(const gva_result* res);
/* Filled when opts->profile was set; returns the number of kernel kinds. */
int gva_result_kernel_stats(const gva_result* res, gva_kernel_stat* out, int cap);
void gva_result_free(gva_result* res);

/* ---- batched form ----------------------------------------------------------
 * Many plans in shared rounds: each round advances every (plan, frontier
 * slice) task by one step with one count, scan, totals and one persistent
 * write launch fed by a device work queue; a task whose output exceeds
 * budget_bytes is split.  Replaces running the gpumine driver once per query
 * (src/gpumine.cpp:866-1072).  Results are counts: the final step of every
 * plan only counts. */
typedef struct gva_batch_opts {
    void* stream;          /* cudaStream_t; NULL = legacy default stream            */
    uint64_t budget_bytes; /* frontier memory cap (0 = 3/4 of free HBM)            */
    int profile;           /* 1: per-kernel CUDA-event timing in stats->kernels     */
    int flags;             /* GVA_BATCH_* below; 0 = none                           */
} gva_batch_opts;
/* gva_batch_count_texts: plan the queries on the device (the heap-free
 * planner, one query per thread; queries of up to 16 vertices and 32 edge
 * lines, DV mode), the others on the host */
#define GVA_BATCH_PLAN_ON_DEVICE 1
/* Round scheduling.  On the device, a planning kernel per round chooses the
 * writing tasks, places their outputs and lists the next round's tasks, so
 * the host launches every round at once and synchronises once (when the
 * budget holds two frontier regions; a round that outgrows its region makes
 * the run start over on the host).  On the host, each round's task totals
 * are read back and the host chooses the writes (splitting tasks larger than
 * the budget) and the next round's tasks.  By default a run in one piece is
 * scheduled on the device, and a run of 12,288 plans or more, which runs as
 * two halves whose round trips hide behind each other's kernels, on the
 * host (no schedule tables or frontier regions per half; the two measured
 * alike there).  The flags force one or the other; they exclude each other. */
#define GVA_BATCH_HOST_ROUNDS 2
#define GVA_BATCH_DEVICE_ROUNDS 4

typedef struct gva_batch_stats {
    double gpu_ms;
    uint64_t rounds, splits, launches;
    uint64_t trie_nodes; /* distinct step prefixes: plans sharing a prefix share its frontier */
    gva_kernel_stat kernels[5];
    /* host time (ms): lowering plans to steps, building the step trie,
     * rounds' host work (task lists, launches, budget choice), waiting for
     * the device, session set-up / read-back / tear-down */
    double lower_ms, submit_ms, round_host_ms, wait_ms, session_ms;
    /* round_host_ms by part: task list and uploads, count launches, totals
     * and budget choice, write launch, next tasks and completion */
    double round_phase_ms[5];
    /* wall-clock marks of the run (ms from the call's start of the batched
     * run): plans ordered; then for each of up to two halves (a run of
     * 12,288 plans or more runs as two, concurrently) the half's session
     * prepared, its rounds done, its results read back and its session freed
     * (0 for an absent half) */
    double timeline_ms[9];
    /* rounds scheduled on the device: the run's rounds were launched at
     * once, each round's planning kernel choosing the next round's tasks */
    uint64_t device_rounds;
} gva_batch_stats;

/* Declares the database a union of graphs: graph g owns vertex ids
 * [first[g], first[g+1]) (num_graphs + 1 entries).  Needed for per-graph
 * counts and supports. */
int gva_db_set_graphs(gva_db* db, const uint64_t* first, uint32_t num_graphs);

/* counts[nplans]: embeddings per plan.  graph_counts[nplans * num_graphs]
 * (optional): embeddings per (plan, graph).  graph_support[nplans]
 * (optional): graphs holding at least one embedding. */
int gva_batch_count(gva_db* db, const gva_plan* const* plans, int nplans, const gva_batch_opts* opts,
                    uint64_t* counts, uint64_t* graph_counts, uint32_t* graph_support, gva_batch_stats* stats);

/* gva_batch_count for query texts, in one call: every text is read and
 * planned on the host's cores (mode GVA_MODE_DV or GVA_MODE_SV; the planner
 * without heap storage where it applies, else the host planner) and the plans
 * counted in one batched run, without plan handles.  status[i] (optional)
 * receives each text's planning status; a text that fails to plan gets
 * count 0, and the call returns the first failure's status after counting
 * the others.  Replaces running gpumine once per .query file
 * (src/gpumine.cpp:866-1072). */
int gva_batch_count_texts(gva_db* db, const char* const* query_texts, int n, int mode, const gva_batch_opts* opts,
                          uint64_t* counts, uint64_t* graph_counts, uint32_t* graph_support, int* status,
                          gva_batch_stats* stats);

/* Launch shape of the batched engine's round kernels on one database: rows
 * per work item (32, 64 or 128; fewer when rows are wide) and the candidate
 * list length above which a frontier row's candidates are shared by a whole
 * warp instead of walked by one lane.  Defaults 64 / 32.  The reference's
 * launch shape is fixed (a persistent grid of GPU_SM_NUM blocks,
 * src/miningPattern.cu:3350-3377); here it is chosen per database. */
typedef struct gva_tuning {
    uint32_t rows_per_item;
    uint32_t hub;
    double ms;          /* gva_db_autotune: calibration time of the chosen shape */
    double default_ms;  /* gva_db_autotune: calibration time of the default shape */
    uint32_t tried;     /* gva_db_autotune: shapes timed */
    /* MiB of each of the two frontier regions of device-scheduled rounds
     * (0: unchanged by gva_db_set_tuning; default 2048); doubled after a run
     * whose round outgrew it */
    uint32_t round_region_mb;
} gva_tuning;
int gva_db_get_tuning(const gva_db* db, gva_tuning* out);
int gva_db_set_tuning(gva_db* db, const gva_tuning* tuning);
/* Counts a calibration batch (as gva_batch_count does, with supports when
 * the database has graph ids) under each candidate launch shape, twice each,
 * and keeps the fastest for every later batched run, mining run and session
 * on this database.  Every shape must give the same counts. */
int gva_db_autotune(gva_db* db, const gva_plan* const* plans, int nplans, void* stream, gva_tuning* out);

/* ---- serving: a persistent batch -------------------------------------------
 * The batched engine kept open: plans may be submitted at any time and join
 * the running work at the next round (continuous batching); each round
 * advances every active task one step; finished plans are polled.  Replaces
 * nothing in the reference (it serves one query per process). */
typedef struct gva_session gva_session;

/* support_slots > 0 enables per-plan supporting-graph counts (needs
 * gva_db_set_graphs); it bounds the number of plans in flight. */
int gva_session_create(gva_db* db, void* stream, uint64_t budget_bytes, uint32_t support_slots, gva_session** out);
/* tags are returned by gva_session_poll with the plan's results. */
int gva_session_submit(gva_session* s, const gva_plan* const* plans, const uint64_t* tags, int n);
/* One round; *active_tasks receives the tasks left (0 = idle). */
int gva_session_round(gva_session* s, int* active_tasks);
/* Up to cap finished plans: tag, embedding count, supporting graphs (0 when
 * support_slots == 0).  Returns how many were written. */
int gva_session_poll(gva_session* s, uint64_t* tags, uint64_t* counts, uint32_t* supports, int cap);
void gva_session_free(gva_session* s);

/* ---- mining layer (graph databases) ------------------------------------------
 * Frequent connected patterns of up to max_edges edges whose support (graphs
 * holding at least one embedding) is at least min_support.  Level-wise growth
 * with canonical dedupe and anti-monotone pruning; every level's candidates
 * are matched in one batched run.  The reference has no pattern generation
 * (it matches one given .query per process); each candidate here is matched
 * with the reference planner's plan, so its embedding count is the row count
 * gpumine would emit for that pattern. */
/* Combines one level's per-candidate supports and embedding counts across
 * processes that hold disjoint shards of the graph database (e.g. an
 * all-reduce sum); arrays are updated in place; return 0 on success. */
typedef int (*gva_reduce_fn)(uint32_t* supports, uint64_t* embeddings, uint64_t n, void* user);

#define GVA_SUPPORT_GRAPHS 0 /* graphs of the database holding an embedding (gva_db_set_graphs) */
#define GVA_SUPPORT_MNI 1    /* minimum image-based support on one data graph */

typedef struct gva_mine_opts {
    void* stream;
    uint64_t budget_bytes;
    uint32_t max_edges;
    uint32_t min_support;
    uint32_t batch_limit;  /* candidates per batched run (0 = 32768; MNI: 65536) */
    uint32_t profile;      /* 1: per-kernel CUDA-event timing (gva_mine_kernel_stats) */
    gva_reduce_fn reduce;  /* NULL on one process (GVA_SUPPORT_GRAPHS only) */
    void* reduce_user;
    uint32_t support_mode; /* GVA_SUPPORT_GRAPHS or GVA_SUPPORT_MNI */
    uint32_t mni_cap;      /* MNI: supports are min(MNI, mni_cap); 0 = min_support */
    const volatile int* cancel; /* optional: once *cancel != 0 (set by another thread), the run stops at
                                   its next batch or round boundary with GVA_ERR_CANCELLED */
    uint32_t sm_percent;   /* MNI: the search kernel fills at most this share of the SMs (0 = all),
                              leaving room for other work on the GPU (a server's matching rounds) */
    uint32_t host_threads; /* host threads for candidate generation and planning (0 = all cores) */
} gva_mine_opts;

typedef struct gva_mine_stats {
    uint64_t candidates; /* patterns whose support was decided */
    uint64_t frequent;
    uint64_t embeddings; /* embeddings enumerated over all candidates */
    uint64_t levels;
    uint64_t pruned;     /* extensions dropped by an infrequent sub-pattern (most are
                            dropped before deduplication and count once per parent
                            that generates them) */
    double gpu_ms;       /* batched matching (CUDA events) */
    double host_ms;      /* whole call, wall clock */
    double gen_ms;       /* candidate generation, dedupe and pruning (host threads) */
    double plan_ms;      /* planning and lowering of every candidate (host threads) */
    double eval_ms;      /* matching of every candidate, host bookkeeping included */
    double merge_ms;     /* merging and ordering the candidates of each level */
    double submit_ms;    /* within eval: building the step trie and descriptors */
    double round_host_ms;/* within eval: per-round host bookkeeping */
    double wait_ms;      /* within eval: host waiting for the GPU */
    uint64_t mni_tasks;  /* MNI: rooted searches set up (one per pattern orbit) */
    uint64_t mni_rounds; /* MNI: search rounds */
} gva_mine_stats;

typedef struct gva_mine_result gva_mine_result;

/* Gives the support and embedding count of n candidate patterns, passed as
 * query texts (text + offsets[i], NUL-terminated, original vertex and edge
 * labels); return 0 on success. */
typedef int (*gva_eval_fn)(const char* text, const uint64_t* offsets, uint64_t n, uint32_t* supports,
                           uint64_t* embeddings, void* user);

/* gva_mine's level loop on the host with the caller's evaluator instead of
 * the GPU matcher: the same candidates (level-wise growth over the vertex
 * labels labels[0..num_labels) (ascending, distinct) and the edge labels
 * 1..num_edge_labels with has_edge_label[el] != 0, canonical dedupe,
 * anti-monotone pruning), each level evaluated by `evaluate` and then
 * combined by `reduce` (optional, e.g. an all-reduce over processes holding
 * disjoint graph shards), patterns returned as by gva_mine (no kernel
 * statistics).  No device work: it serves evaluators elsewhere (another
 * process, a CPU checker) and the multi-process level loop's tests.  The
 * reference has no pattern generation; it has no counterpart there. */
int gva_mine_host(uint32_t num_labels, const uint32_t* labels, uint32_t num_edge_labels,
                  const uint8_t* has_edge_label, uint32_t max_edges, uint32_t min_support, uint32_t host_threads,
                  gva_eval_fn evaluate, void* eval_user, gva_reduce_fn reduce, void* reduce_user,
                  gva_mine_result** out);

int gva_mine(gva_db* db, const gva_mine_opts* opts, gva_mine_result** out);
int gva_mine_num_patterns(const gva_mine_result* res);
int gva_mine_get(const gva_mine_result* res, int index, uint32_t* edges, uint32_t* support, uint64_t* embeddings);
/* query text of pattern `index` (.query format); returns length */
size_t gva_mine_pattern_text(const gva_mine_result* res, int index, char* buf, size_t cap);
/* Every pattern in one call: texts concatenated into text_buf, each ending in
 * a NUL, pattern i's text starting at offsets[i]; edges, supports and
 * embeddings (any may be NULL) receive one entry per pattern.  Returns the
 * text bytes needed (NULs included); text_buf and offsets are written only
 * when text_cap is at least that. */
size_t gva_mine_export(const gva_mine_result* res, char* text_buf, size_t text_cap, uint64_t* offsets,
                       uint32_t* edges, uint32_t* supports, uint64_t* embeddings);
int gva_mine_get_stats(const gva_mine_result* res, gva_mine_stats* out);
/* per-kernel totals when opts->profile was set; returns the number of kinds */
int gva_mine_kernel_stats(const gva_mine_result* res, gva_kernel_stat* out, int cap);
void gva_mine_free(gva_mine_result* res);

/* ---- single-graph support: MNI ----------------------------------------------
 * The minimum image-based support of each pattern (for every pattern vertex,
 * the number of distinct data vertices some embedding maps it to; the
 * minimum over the pattern's vertices), decided by rooted existence searches
 * on the device, one per automorphism orbit and data vertex, stopped once an
 * orbit reaches the cap.  Replaces nothing in the reference (it enumerates
 * the embeddings of one pattern, src/gpumine.cpp:994-1061, and has no support
 * notion); embeddings follow its semantics (injective, vertex and edge labels
 * kept, non-induced).  Patterns are .query text (`v id label`, `e a b
 * elabel`), connected, up to 8 vertices; a label absent from the database
 * gives support 0.  plain = 1 runs one pattern at a time (the per-query
 * path); the default runs all patterns' searches in shared rounds. */
typedef struct gva_mni_opts {
    void* stream;
    uint32_t cap;  /* supports are min(MNI, cap); 0 = exact MNI */
    int plain;
    int profile;   /* 1: kernel timing and search counters in stats */
    int reserved;
} gva_mni_opts;

typedef struct gva_mni_stats {
    double gpu_ms;
    uint64_t rounds, launches, tasks;
    uint64_t seeds, roots, found; /* profile: vertices tried, roots past the degree filter, embeddings found */
    gva_kernel_stat kernel;       /* profile: mni_search launches, CUDA-event ms, algorithmic bytes */
} gva_mni_stats;

int gva_mni_support(gva_db* db, const char* const* pattern_texts, int n, const gva_mni_opts* opts, uint32_t* support,
                    gva_mni_stats* stats);

/* ---- L4: one phase step on caller-owned device buffers ----------------------
 * Replaces the kernel launchers of include/miningPattern.h:1-30
 * (initEmb_*, extEmb_1V_NoHash, extEmb_2V_*) and include/reduction.h:1-3
 * (reductionPhase).  A plan is lowered to steps (gva_plan_num_steps); a step
 * is an init seed, a one-vertex extension or a back-edge reduction.  The
 * step reads `in_rows` rows of width gva_plan_step_width_in() and writes at
 * most `out_capacity_rows` rows of width gva_plan_step_width_out().
 * Scratch: gva_step_scratch_bytes(in_rows) bytes of device memory, 256-byte
 * aligned.  *out_rows receives the produced row count; when it exceeds
 * out_capacity_rows nothing is written and GVA_ERR_NOMEM is returned (the
 * count is still valid, so the caller can grow and retry).  For a seed step
 * in_rows/in_dev are ignored. Synchronises the stream once (count read-back). */
int gva_plan_num_steps(const gva_plan* plan, const gva_db* db);
int gva_plan_step_width_in(const gva_plan* plan, const gva_db* db, int step);
int gva_plan_step_width_out(const gva_plan* plan, const gva_db* db, int step);
size_t gva_step_scratch_bytes(uint64_t in_rows);
int gva_step_run(gva_db* db, const gva_plan* plan, int step, const uint32_t* in_dev, uint64_t in_rows,
                 uint32_t* out_dev, uint64_t out_capacity_rows, uint64_t* out_rows, void* scratch_dev,
                 size_t scratch_bytes, void* stream);

/* gva_step_run for callers that cannot allocate device memory at call time
 * (a request path that must not reach cudaMalloc, or a host runtime that owns
 * all device memory); it has no counterpart in the reference.  Same
 * arguments and results as gva_step_run minus the scratch buffer: the step's
 * scratch is a fixed array in the library's device memory (512 KiB + 256
 * bytes per GPU, held until exit), so in_rows may not exceed GVA_STATIC_MAX_ROWS
 * (GVA_ERR_ARG otherwise, nothing launched).  It allocates no device memory.
 * Every call on a device shares the array: calls whose kernels overlap on the
 * GPU race, so serialise them.  The first call on a device looks up the
 * array's address (cudaGetSymbolAddress) once; make it before any stream
 * capture.  That address belongs to the device's context: after the caller
 * ends the context (cudaDeviceReset) this entry point must not be called
 * again in the same process. */
#define GVA_STATIC_MAX_ROWS 16777216u
int gva_step_run_static(gva_db* db, const gva_plan* plan, int step, const uint32_t* in_dev, uint64_t in_rows,
                        uint32_t* out_dev, uint64_t out_capacity_rows, uint64_t* out_rows, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GENEVA_H */
