// Device-side database and the phase executor interface.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
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
//   seed_off[L + 1] | seed_verts[...] | per partition: off[...] adj[...]
struct DevDB {
    int device = 0;
    uint32_t max_id = 0;
    uint32_t L = 0;                       // dense vertex labels
    std::vector<uint32_t> labels;         // dense -> original label
    std::vector<DevPart> parts;           // parts[p - 1] = edge label p (off == nullptr: absent)
    std::vector<uint32_t> seed_off;       // host copy of seed_off
    const uint32_t* seed_verts = nullptr; // vertices grouped by dense label, ascending id
    void* arena = nullptr;
    size_t arena_bytes = 0;
    uint64_t n_adj = 0;
    HostGraph meta;                       // labels/partition presence for lowering (no adjacency)
};

int upload_graph(HostGraph& g, int device, DevDB*& out);
void free_devdb(DevDB* db);

struct MatchResult {
    int device = 0;
    uint64_t rows = 0;
    uint32_t width = 0;
    uint32_t* rows_dev = nullptr;         // owned (cudaMallocAsync pool), may be null
    cudaStream_t stream = nullptr;
    std::vector<uint64_t> phase_rows;
    double gpu_ms = 0.0;
    std::vector<uint32_t> columns;
};

int run_match(DevDB& db, const Plan& plan, const std::vector<Step>& steps, cudaStream_t stream, uint64_t budget,
              bool count_only, MatchResult& res);
void free_result(MatchResult* r);

size_t step_scratch_bytes(uint64_t in_rows);
int run_step(DevDB& db, const Step& st, const uint32_t* in, uint64_t in_rows, uint32_t* out, uint64_t out_cap,
             uint64_t* out_rows, void* scratch, size_t scratch_bytes, cudaStream_t stream);

}  // namespace gva
