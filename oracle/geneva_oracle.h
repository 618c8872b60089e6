/*
 * Test infrastructure only — the CPU oracle of the matching path.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it;
 * the product never links it.
 *
 * A plain restatement of the reference CPU matcher `cpumine`
 * (src/cpumine.cpp:54-584) and of its planner (src/genMatchOrderCPU.cpp:69-983),
 * held in memory instead of temp files, over the adjacency the reference GPU
 * driver sees (.mygraph lists without genDatabase's index vertices).  Pinned
 * against the reference itself: tests/golden holds rows/plans produced by the
 * reference binaries compiled from source (oracle/Makefile `ref`).
 */
#ifndef GENEVA_ORACLE_H
#define GENEVA_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_graph oracle_graph;

/* .mygraph + .metadata (src/loadDataBase.cpp:309-365) */
int oracle_graph_load(const char* mygraph, const char* metadata, oracle_graph** out);
/* edge list, ids kept (tools/genDatabase.cpp:600-667 without renumbering) */
int oracle_graph_from_edges(const uint32_t* vlabels, uint32_t max_id, const uint32_t* src, const uint32_t* dst,
                            const uint32_t* elabel, uint64_t ne, oracle_graph** out);
void oracle_graph_free(oracle_graph* g);

/* Canonical plan text (same lines as gva_plan_describe). Returns length. */
size_t oracle_plan(const char* query_text, char* buf, size_t cap);

/* Runs every phase.  *rows is malloc'd (free with oracle_free), row-major,
 * *width columns in match order.  phase_rows receives up to cap counts.
 * Returns 0 on success. */
int oracle_match(const oracle_graph* g, const char* query_text, uint32_t** rows, uint64_t* nrows, int* width,
                 uint64_t* phase_rows, int cap, int* nphases);
/* Counts only (no rows kept after the last phase). */
int oracle_count(const oracle_graph* g, const char* query_text, uint64_t* nrows);
/* Same, giving up (returns 2) once any frontier holds about cap_rows rows. */
int oracle_count_capped(const oracle_graph* g, const char* query_text, uint64_t cap_rows, uint64_t* nrows);
/* Embeddings per graph of a graph database: graph i owns the vertex ids
 * [first[i], first[i+1]) (first has G + 1 ascending entries); counts[i]
 * receives the final rows whose first column lies in graph i, *nrows all
 * final rows (rows outside every graph are counted only there).  The query's
 * support is the number of graphs with a nonzero count.  This is the
 * post-process that maps cpumine's rows to graph ids, done without handing
 * the rows out. */
int oracle_graph_counts(const oracle_graph* g, const char* query_text, const int64_t* first, uint32_t G,
                        uint64_t* counts, uint64_t* nrows);
void oracle_free(void* p);
const char* oracle_last_error(void);

/* MNI support on one data graph (no counterpart in the reference, which has
 * no support notion): for each automorphism orbit of the pattern, the data
 * vertices some embedding maps the orbit's representative to, decided one
 * vertex at a time by a depth-first existence search; support = the smallest
 * such set, reported as min(MNI, cap) (cap 0 = exact).  Single-threaded,
 * over its own sorted adjacency (no per-vertex maps), so it scales to the
 * large single-graph configuration for bounded samples. */
typedef struct oracle_mni_graph oracle_mni_graph;
int oracle_mni_graph_from_edges(const uint32_t* vlabels, uint32_t max_id, const uint32_t* src, const uint32_t* dst,
                                const uint32_t* elabel, uint64_t ne, oracle_mni_graph** out);
void oracle_mni_graph_free(oracle_mni_graph* g);
/* *searches receives the number of rooted searches run (may be NULL). */
int oracle_mni(const oracle_mni_graph* g, const char* pattern_text, uint32_t cap, uint32_t* support,
               uint64_t* searches);

#ifdef __cplusplus
}
#endif
#endif
