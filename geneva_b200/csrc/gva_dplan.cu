// Device-side match-order planning: the heap-free planner (gva_dplan.h), one
// query per thread, for batched query admission.  The host hands over small
// fixed-size query records and reads back compact plans (phases, pairs,
// restrictions), which it lowers to engine steps as it lowers the host-side
// dplan's plans.  A query beyond the records' capacities, or one the planner
// leaves to the host planner, comes back with status DPLAN_HOST.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/geneva.h"
#include "gva_dplan.h"
#include "gva_engine.cuh"

namespace gva {

// The planner again, with device capacities: every thread's frame holds its
// arrays, so they are sized for the queries a batch admits (16 vertices, 32
// edge lines); a larger query comes back DPLAN_HOST.  The sort threshold and
// the search bounds are the host planner's, so accepted plans are the same.
namespace dev {
constexpr uint32_t kDpNone = 0xffffffffu;
constexpr int kDpV = kDevPlanV;
constexpr int kDpLines = kDevPlanLines;
constexpr int kDpPhases = kDevPlanPhases;
constexpr int kDpPairs = kDevPlanPairs;
constexpr int kDpKeys = kDevPlanKeys;
constexpr int kDpSort = gva::kDpSort;
constexpr uint64_t kDpMaxAut = gva::kDpMaxAut;
constexpr uint64_t kDpMaxSearch = gva::kDpMaxSearch;
#include "gva_dplan_body.inc"
}  // namespace dev

namespace {

__global__ void __launch_bounds__(64) dplan_kernel(const DevPlanQuery* __restrict__ qs, uint32_t n,
                                                   DevPlanOut* __restrict__ outs) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DevPlanQuery& dq = qs[i];
    DevPlanOut& o = outs[i];
    dev::DPlanQuery q;
    dev::DPlan p;
    q.n = dq.n;
    q.lines = dq.lines;
    for (uint32_t v = 0; v < dq.n; ++v) q.label[v] = dq.label[v];
    for (uint32_t e = 0; e < dq.lines; ++e) {
        q.s[e] = dq.s[e];
        q.d[e] = dq.d[e];
        q.l[e] = dq.l[e];
    }
    dev::dplan(q, p);
    o.status = DPLAN_HOST;
    if (p.status != DPLAN_OK || p.vnum > (uint32_t)kDevPlanV || p.nphase > (uint32_t)kDevPlanPhases ||
        p.npair > (uint32_t)kDevPlanPairs)
        return;
    o.vnum = p.vnum;
    o.nphase = p.nphase;
    o.npair = p.npair;
    for (uint32_t v = 0; v <= p.vnum; ++v) o.restricts[v] = p.restricts[v];
    for (uint32_t k = 0; k < p.nphase; ++k) {
        o.ph_type[k] = p.ph_type[k];
        o.ph_el[k] = p.ph_el[k];
        o.ph_at[k] = (uint8_t)p.ph_at[k];
        o.ph_np[k] = (uint8_t)p.ph_np[k];
    }
    for (uint32_t k = 0; k < p.npair; ++k) o.pairs[k] = p.pairs[k];
    o.nrep = p.nrep;
    o.nstat = p.nstat;
    o.ncol = p.ncol;
    for (uint32_t k = 0; k < p.nrep; ++k) {
        o.rep_key[k] = p.rep_key[k];
        o.rep_val[k] = p.rep_val[k];
    }
    for (uint32_t k = 0; k < p.nstat; ++k) {
        o.stat_el[k] = p.stat_el[k];
        o.stat_vl[k] = p.stat_vl[k];
    }
    for (uint32_t k = 0; k < p.ncol; ++k) o.columns[k] = p.columns[k];
    o.status = DPLAN_OK;
}

std::atomic<uint64_t> g_dplan_launches{0};

}  // namespace

uint64_t dplan_kernel_launches() { return g_dplan_launches.load(); }

int plan_on_device(int device, cudaStream_t s, const DevPlanQuery* qs, uint32_t n, DevPlanOut* outs) {
    if (n == 0) return GVA_OK;
    cudaError_t e = cudaSetDevice(device);
    void* dq = nullptr;
    void* dout = nullptr;
    if (e == cudaSuccess) e = cudaMallocAsync(&dq, (size_t)n * sizeof(DevPlanQuery), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dout, (size_t)n * sizeof(DevPlanOut), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dq, qs, (size_t)n * sizeof(DevPlanQuery), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        dplan_kernel<<<(n + 63) / 64, 64, 0, s>>>((const DevPlanQuery*)dq, n, (DevPlanOut*)dout);
        e = cudaGetLastError();
        g_dplan_launches += 1;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(outs, dout, (size_t)n * sizeof(DevPlanOut), cudaMemcpyDeviceToHost, s);
    if (dq) cudaFreeAsync(dq, s);
    if (dout) cudaFreeAsync(dout, s);
    const cudaError_t e2 = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return fail(GVA_ERR_CUDA, std::string("device planning: ") + cudaGetErrorString(e));
    return GVA_OK;
}

void dplan_from_device(const DevPlanOut& o, DPlan& p) {
    p.status = o.status;
    if (o.status != DPLAN_OK) return;
    p.vnum = o.vnum;
    p.nphase = o.nphase;
    p.npair = o.npair;
    for (uint32_t v = 0; v <= o.vnum; ++v) p.restricts[v] = o.restricts[v];
    for (uint32_t k = 0; k < o.nphase; ++k) {
        p.ph_type[k] = o.ph_type[k];
        p.ph_el[k] = o.ph_el[k];
        p.ph_at[k] = o.ph_at[k];
        p.ph_np[k] = o.ph_np[k];
    }
    for (uint32_t k = 0; k < o.npair; ++k) p.pairs[k] = o.pairs[k];
    p.nrep = o.nrep;
    p.nstat = o.nstat;
    p.ncol = o.ncol;
    for (uint32_t k = 0; k < o.nrep; ++k) {
        p.rep_key[k] = o.rep_key[k];
        p.rep_val[k] = o.rep_val[k];
    }
    for (uint32_t k = 0; k < o.nstat; ++k) {
        p.stat_el[k] = o.stat_el[k];
        p.stat_vl[k] = o.stat_vl[k];
    }
    for (uint32_t k = 0; k < o.ncol; ++k) p.columns[k] = o.columns[k];
}

}  // namespace gva
