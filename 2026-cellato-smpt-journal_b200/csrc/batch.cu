// Batched execution of many independent grids (C ABI cellato_batch_*).
//
// A batch is a set of grids -- any registered rules, any sizes the layout
// accepts, each with its own step count -- that advance together.  Grids of
// one rule form a group; a group advances in rounds of k fused steps (k per
// rule), and all rounds of all its grids are ONE launch of the persistent
// temporal_batch_kernel, in which a grid's round starts as soon as its
// previous round is done (batch_plan.hpp).  The groups' launches are parallel
// branches of one CUDA graph after a single node that clears the launches'
// queue heads and per-grid counters, so one graph launch advances every grid
// of the batch.
//
// The reference has no batching: each grid is one traverser run with one
// launch per step or per k steps (include/traversers/cuda/simple.cu:67-83,
// temporal.cu:227-262).  Results are identical to those single-grid runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "batch_plan.hpp"
#include "capi_internal.hpp"
#include "cellato_b200.h"

using namespace cellato::b200;
using namespace cellato::b200::capi;

struct cellato_batch_st {
    int layout = 0, word_bits = 64, internal = 0;
    std::vector<int> rounds;  // per grid
    void* device_buf = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
    long long work_items = 0;
    int launches = 0;
    int n = 0;
};

namespace {

void release(cellato_batch_st* b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto e : b->events) cudaEventDestroy(e);
    for (auto s : b->streams) cudaStreamDestroy(s);
    if (b->device_buf) cudaFree(b->device_buf);
    delete b;
}

int fail_release(cellato_batch_st* b, int rc) {
    release(b);
    return rc;
}

}  // namespace

extern "C" {

int cellato_batch_create(int layout, int word_bits, const cellato_batch_grid* grids, int n_grids,
                         const int* k_per_rule, int n_k_per_rule, cellato_batch_t* out) {
    if (!out) return fail(CELLATO_EINVAL, "out must not be NULL");
    *out = nullptr;
    batch_plan plan;
    if (int rc = plan_batch(layout, word_bits, grids, n_grids, k_per_rule, n_k_per_rule, -1, plan)) return rc;
    auto* b = new cellato_batch_st;
    b->layout = layout;
    b->word_bits = word_bits;
    b->internal = internal_layout(layout, word_bits);
    b->n = n_grids;
    b->rounds = plan.rounds;
    b->work_items = (long long)plan.items.size();

    const batch_layout L(plan.descs.size(), plan.items.size(), plan.groups.size());
    cudaError_t e = cudaMalloc(&b->device_buf, L.total);
    if (e != cudaSuccess) return fail_release(b, cuda_fail(e, "cudaMalloc (batch work lists)"));
    auto* base = static_cast<unsigned char*>(b->device_buf);
    auto* d_descs = reinterpret_cast<batch_grid_desc*>(base);
    auto* d_items = reinterpret_cast<batch_item*>(base + L.items);
    auto* d_sync = reinterpret_cast<unsigned*>(base + L.sync);
    if (!plan.descs.empty())
        e = cudaMemcpy(d_descs, plan.descs.data(), plan.descs.size() * sizeof(batch_grid_desc), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !plan.items.empty())
        e = cudaMemcpy(d_items, plan.items.data(), plan.items.size() * sizeof(batch_item), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail_release(b, cuda_fail(e, "cudaMemcpy (batch work lists)"));

    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return fail_release(b, cuda_fail(e, "querying the device"));
    // kernel attributes, outside the capture
    for (const batch_group& gp : plan.groups)
        if ((e = ops_of(gp.rule)->prepare_batch(b->internal, gp.TH)) != cudaSuccess)
            return fail_release(b, cuda_fail(e, "batch kernel attributes"));

    // capture: clear the sync words on a root stream, fork one stream per
    // group, one persistent launch each, join back
    cudaStream_t root;
    if ((e = cudaStreamCreateWithFlags(&root, cudaStreamNonBlocking)) != cudaSuccess)
        return fail_release(b, cuda_fail(e, "cudaStreamCreate"));
    b->streams.push_back(root);
    std::vector<cudaStream_t> branch;
    std::vector<cudaEvent_t> joins;
    cudaEvent_t fork = nullptr;
    if ((e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming)) != cudaSuccess)
        return fail_release(b, cuda_fail(e, "cudaEventCreate"));
    b->events.push_back(fork);
    for (size_t g = 0; g < plan.groups.size(); ++g) {
        cudaStream_t st;
        cudaEvent_t j;
        if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess)
            return fail_release(b, cuda_fail(e, "cudaStreamCreate"));
        b->streams.push_back(st);
        branch.push_back(st);
        if ((e = cudaEventCreateWithFlags(&j, cudaEventDisableTiming)) != cudaSuccess)
            return fail_release(b, cuda_fail(e, "cudaEventCreate"));
        b->events.push_back(j);
        joins.push_back(j);
    }
    e = cudaStreamBeginCapture(root, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess && L.sync_bytes) e = cudaMemsetAsync(d_sync, 0, L.sync_bytes, root);
    if (e == cudaSuccess) e = cudaEventRecord(fork, root);
    for (size_t g = 0; g < branch.size() && e == cudaSuccess; ++g) e = cudaStreamWaitEvent(branch[g], fork, 0);
    int rc = CELLATO_OK;
    if (e == cudaSuccess)
        rc = launch_plan(plan, b->internal, d_descs, d_items, d_sync, sms, root, &b->launches, &branch);
    for (size_t g = 0; g < branch.size() && e == cudaSuccess && rc == CELLATO_OK; ++g) {
        e = cudaEventRecord(joins[g], branch[g]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(root, joins[g], 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t e_end = cudaStreamEndCapture(root, &graph);
    b->graph = graph;
    if (rc != CELLATO_OK) return fail_release(b, rc);
    if (e == cudaSuccess) e = e_end;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, graph, 0);
    if (e != cudaSuccess) return fail_release(b, cuda_fail(e, "building the batch graph"));
    *out = b;
    return CELLATO_OK;
}

int cellato_batch_launch(cellato_batch_t b, cellato_stream_t stream) {
    if (!b) return fail(CELLATO_EINVAL, "batch is NULL");
    cudaError_t e = cudaGraphLaunch(b->exec, reinterpret_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? CELLATO_OK : cuda_fail(e, "cudaGraphLaunch");
}

int cellato_batch_result_in_b(cellato_batch_t b, int grid, int* in_b) {
    if (!b || !in_b || grid < 0 || grid >= b->n) return fail(CELLATO_EINVAL, "bad batch, grid index or output");
    *in_b = b->rounds[grid] & 1;
    return CELLATO_OK;
}

int cellato_batch_info(cellato_batch_t b, int* kernel_launches, long long* work_items) {
    if (!b) return fail(CELLATO_EINVAL, "batch is NULL");
    if (kernel_launches) *kernel_launches = b->launches;
    if (work_items) *work_items = b->work_items;
    return CELLATO_OK;
}

int cellato_batch_destroy(cellato_batch_t b) {
    release(b);
    return CELLATO_OK;
}

}  // extern "C"
