// cellato_batch_run_noalloc: the batched temporal run without any device
// allocation.
//
// Who needs it.  Some callers of this library must not allocate device memory
// themselves or through it:
//   * a host application or plugin framework that owns all device memory (a
//     caching or pooled allocator reserving HBM up front) and forbids other
//     code from calling cudaMalloc;
//   * latency-critical loops, where cudaMalloc / cudaFree would add implicit
//     device synchronisation and unpredictable stalls;
//   * code running under a fixed device-memory budget that must not grow.
// cellato_batch_create allocates the batch's work lists with cudaMalloc; this
// entry point instead keeps them in a file-scope __device__ array of fixed
// size that every GPU holds from the moment the library is loaded until the
// process exits.  The caller still passes its own input and output planes.
//
// Limits: at most NOALLOC_MAX_GRIDS grids and NOALLOC_MAX_ITEMS work items
// (tiles x rounds summed over the batch) per call; larger batches are rejected
// with CELLATO_EINVAL before anything runs.
//
// Set-up: the device address of the array (and the device's SM count) is
// obtained with cudaGetSymbolAddress on the first call on each device (that
// device current) and cached for the process; a process that resets a device
// (cudaDeviceReset) must not call this entry point on it afterwards.
//
// Streams: the work list is copied from host memory the library does not pin,
// so each call waits for the work queued before it on `stream`, and a stream
// that is being captured is refused (CELLATO_EINVAL): a captured copy would
// read host memory that is gone when the graph runs.
//
// Sharing: all calls share the one array and it keeps the last call's
// contents.  Each call writes the complete work list it uses and clears the
// queue heads and tile counters the kernels count up from zero, stream-ordered
// before its kernels.  Calls whose work may overlap on the GPU -- on different
// streams, or from different host threads -- race on the array and must be
// serialised by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "batch_plan.hpp"
#include "capi_internal.hpp"
#include "cellato_b200.h"

using namespace cellato::b200;
using namespace cellato::b200::capi;

namespace {

constexpr int NOALLOC_MAX_GRIDS = CELLATO_NOALLOC_MAX_GRIDS;
constexpr int NOALLOC_MAX_ITEMS = CELLATO_NOALLOC_MAX_ITEMS;
// room for the largest plan: every rule a group
constexpr size_t NOALLOC_SCRATCH_BYTES =
    (NOALLOC_MAX_GRIDS * sizeof(batch_grid_desc) + 255) / 256 * 256 + NOALLOC_MAX_ITEMS * sizeof(batch_item) +
    (CELLATO_MAX_RULES + NOALLOC_MAX_GRIDS) * sizeof(unsigned) + 256;

// The work-list scratch: grid descriptors, work items, queue heads and counters.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_scratch_mutex;
void* g_scratch_addr[MAX_DEVICES] = {};
int g_scratch_sms[MAX_DEVICES] = {};

// Device address of g_noalloc_scratch on the current device (the host-side
// name is only a stand-in for the device symbol) and the device's SM count.
int scratch_address(void** out, int* sms) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= MAX_DEVICES) return fail(CELLATO_EINVAL, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        int n = 0;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress (no-allocation scratch)");
        e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute (SM count)");
        g_scratch_addr[dev] = p;
        g_scratch_sms[dev] = n;
    }
    *out = g_scratch_addr[dev];
    *sms = g_scratch_sms[dev];
    return CELLATO_OK;
}

}  // namespace

extern "C" int cellato_batch_run_noalloc(int layout, int word_bits, const cellato_batch_grid* grids, int n_grids,
                                         const int* k_per_rule, int n_k_per_rule, cellato_stream_t stream,
                                         int* result_in_b) {
    if (n_grids < 0 || (n_grids > 0 && (!grids || !result_in_b))) return fail(CELLATO_EINVAL, "bad grid or result array");
    if (n_grids > NOALLOC_MAX_GRIDS)
        return fail(CELLATO_EINVAL, "%d grids exceed the no-allocation limit of %d grids per call", n_grids,
                    NOALLOC_MAX_GRIDS);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &capturing);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamIsCapturing");
    if (capturing != cudaStreamCaptureStatusNone)
        return fail(CELLATO_EINVAL, "the no-allocation batch run cannot be captured into a CUDA graph");
    batch_plan plan;
    if (int rc = plan_batch(layout, word_bits, grids, n_grids, k_per_rule, n_k_per_rule, NOALLOC_MAX_ITEMS, plan))
        return rc;
    const int internal = internal_layout(layout, word_bits);

    void* scratch = nullptr;
    int sms = 0;
    if (int rc = scratch_address(&scratch, &sms)) return rc;
    // this call's layout inside the scratch: descriptors, items, then the sync words
    const batch_layout L(plan.descs.size(), plan.items.size(), plan.groups.size());
    if (L.total > NOALLOC_SCRATCH_BYTES)
        return fail(CELLATO_EINVAL, "the batch does not fit the no-allocation limit (%zu bytes)", NOALLOC_SCRATCH_BYTES);
    auto* base = static_cast<unsigned char*>(scratch);
    auto* d_descs = reinterpret_cast<batch_grid_desc*>(base);
    auto* d_items = reinterpret_cast<batch_item*>(base + L.items);
    auto* d_sync = reinterpret_cast<unsigned*>(base + L.sync);
    if (!plan.descs.empty())
        e = cudaMemcpyAsync(d_descs, plan.descs.data(), plan.descs.size() * sizeof(batch_grid_desc),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !plan.items.empty())
        e = cudaMemcpyAsync(d_items, plan.items.data(), plan.items.size() * sizeof(batch_item), cudaMemcpyHostToDevice,
                            s);
    // the queue heads and finished-tile counts start at zero
    if (e == cudaSuccess && L.sync_bytes) e = cudaMemsetAsync(d_sync, 0, L.sync_bytes, s);
    if (e != cudaSuccess) return cuda_fail(e, "writing the work list to the no-allocation scratch");
    for (const batch_group& gp : plan.groups)
        if ((e = ops_of(gp.rule)->prepare_batch(internal, gp.TH)) != cudaSuccess)
            return cuda_fail(e, "batch kernel attributes");
    if (int rc = launch_plan(plan, internal, d_descs, d_items, d_sync, sms, s)) return rc;
    for (int i = 0; i < n_grids; ++i) result_in_b[i] = plan.rounds[i] & 1;
    return CELLATO_OK;
}
