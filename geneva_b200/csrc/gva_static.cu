// gva_step_run_static: gva_step_run without any device allocation.
//
// Some callers cannot allocate device memory when they call us: a serving
// loop whose request path must not reach cudaMalloc (it may synchronise the
// device and takes driver locks), or a host runtime that owns all device
// memory through its own pool and forbids allocations by libraries.  For
// them the one piece of scratch a step needs (the per-256-row block totals
// and their exclusive scan) lives in a fixed array in the module's device
// memory, so the caller passes only its input and output frontiers.
//
// Limits and rules:
//   * in_rows <= GVA_STATIC_MAX_ROWS (16,777,216); larger inputs are rejected
//     with GVA_ERR_ARG before anything is launched.  The array takes
//     (GVA_STATIC_MAX_ROWS / 256 + 1) * 8 bytes rounded up to 256 bytes
//     = 512 KiB + 256 bytes on every GPU that loads this library, held until
//     the process exits.
//   * Every call on a device shares that array, and it keeps whatever the
//     previous call left in it.  Nothing needs clearing: the count kernel
//     writes every block total it later scans.  Calls whose kernels overlap
//     on the GPU (two streams, two threads) race on the array; serialise them.
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (that device current), once, and caches it; make
//     that first call before any stream capture.  The cached address belongs
//     to the device's current context: a caller that ends that context
//     (cudaDeviceReset) must not call this entry point again in the same
//     process.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/geneva.h"
#include "gva_engine.cuh"

namespace gva {
namespace {

constexpr uint64_t kStaticBlocks = (uint64_t)GVA_STATIC_MAX_ROWS / 256;  // 256 rows per count block

// Block totals of one step (+1 slot for the grand total), rounded up to the
// 256-byte granule that run_step asks of every scratch buffer.  In host code
// this name is only a stand-in for the symbol, never a device address.
constexpr uint64_t kStaticScratchBytes = ((kStaticBlocks + 1) * sizeof(uint64_t) + 255) & ~(uint64_t)255;
static __device__ __align__(256) uint64_t g_step_scratch[kStaticScratchBytes / sizeof(uint64_t)];

std::mutex g_mu;
void* g_scratch_addr[64] = {};

int static_scratch(int device, void** addr) {
    if (device < 0 || device >= 64) return fail(GVA_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_step_scratch);  // caller made `device` current
        if (e != cudaSuccess || !p)
            return fail(GVA_ERR_CUDA, std::string("cudaGetSymbolAddress(step scratch): ") + cudaGetErrorString(e));
        g_scratch_addr[device] = p;
    }
    *addr = g_scratch_addr[device];
    return GVA_OK;
}

}  // namespace

int run_step_static(DevDB& db, const Step& st, const uint32_t* in, uint64_t in_rows, uint32_t* out,
                    uint64_t out_cap, uint64_t* out_rows, cudaStream_t stream) {
    if (!out_rows) return fail(GVA_ERR_ARG, "out_rows is null");
    *out_rows = 0;
    if (in_rows > (uint64_t)GVA_STATIC_MAX_ROWS)
        return fail(GVA_ERR_ARG, "gva_step_run_static: in_rows " + std::to_string(in_rows) +
                                     " exceeds GVA_STATIC_MAX_ROWS (" + std::to_string(GVA_STATIC_MAX_ROWS) + ")");
    cudaError_t e = cudaSetDevice(db.device);
    if (e != cudaSuccess) return fail(GVA_ERR_CUDA, cudaGetErrorString(e));
    void* scratch = nullptr;
    int rc = static_scratch(db.device, &scratch);
    if (rc) return rc;
    return run_step(db, st, in, in_rows, out, out_cap, out_rows, scratch, kStaticScratchBytes, stream);
}

}  // namespace gva
