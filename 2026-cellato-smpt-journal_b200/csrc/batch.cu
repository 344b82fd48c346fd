// Batched execution of many independent grids (C ABI cellato_batch_*).
//
// A batch is a set of grids -- any of the ten rules, any sizes the layout
// accepts, each with its own step count -- that advance together.  Grids of
// one rule form a group; a group advances in rounds of k fused steps (k per
// rule).  Round r of a group is ONE launch of temporal_batch_kernel over the
// work list of every tile of every grid of the group that still has steps
// left (a grid's last round runs its remaining steps).  Each group's rounds
// are a chain on its own stream; the chains are independent branches of one
// CUDA graph, so one graph launch advances every grid of the batch and the
// groups' kernels overlap on the device.
//
// The reference has no batching: each grid is one traverser run with one
// launch per step or per k steps (include/traversers/cuda/simple.cu:67-83,
// temporal.cu:227-262).  Results are identical to those single-grid runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "capi_internal.hpp"
#include "cellato_b200.h"

using namespace cellato::b200;
using namespace cellato::b200::capi;

struct cellato_batch_st {
    int layout = 0, word_bits = 64, internal = 0, R = 1;
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

struct group_plan {
    int rule = 0, k = 8, TH = 0, HY = 0;
    std::vector<int> grids;                       // indices into the batch
    std::vector<std::pair<int, int>> rounds;      // (first item, item count) per round
};

void release(cellato_batch_st* b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto e : b->events) cudaEventDestroy(e);
    for (auto s : b->streams) cudaStreamDestroy(s);
    if (b->device_buf) cudaFree(b->device_buf);
    delete b;
}

}  // namespace

extern "C" {

int cellato_batch_create(int layout, int word_bits, const cellato_batch_grid* grids, int n_grids,
                         const int* k_per_rule, cellato_batch_t* out) {
    if (!out) return fail(CELLATO_EINVAL, "out must not be NULL");
    *out = nullptr;
    if (n_grids < 0 || (n_grids > 0 && !grids)) return fail(CELLATO_EINVAL, "bad grid array");
    auto* b = new cellato_batch_st;
    b->layout = layout;
    b->word_bits = word_bits;
    b->internal = internal_layout(layout, word_bits);
    b->R = band_height(layout, word_bits);
    b->n = n_grids;
    b->rounds.assign(n_grids, 0);

    std::vector<batch_grid_desc> descs(n_grids);
    std::vector<group_plan> groups(CELLATO_RULE_COUNT);
    for (int r = 0; r < CELLATO_RULE_COUNT; ++r) {
        groups[r].rule = r;
        const int k = k_per_rule ? k_per_rule[r] : 0;
        groups[r].k = k > 0 ? std::min(k, 32) : 8;
        groups[r].TH = default_tile_rows(ops_of(r), b->R, groups[r].k, ops_of(r)->batch_words_per_lane);
        groups[r].HY = (groups[r].k + b->R - 1) / b->R * b->R;
    }
    for (int i = 0; i < n_grids; ++i) {
        const cellato_batch_grid& g = grids[i];
        const rule_ops* ops = ops_of(g.rule);
        if (!ops) {
            release(b);
            return fail(CELLATO_EINVAL, "grid %d: unknown rule id %d", i, g.rule);
        }
        if (g.steps < 0) {
            release(b);
            return fail(CELLATO_EINVAL, "grid %d: negative step count", i);
        }
        if (int rc = check_dims(layout, word_bits, g.x_cells, g.y_cells)) {
            release(b);
            return rc;
        }
        plane_set pa, pb;
        if (int rc = make_sets(ops, g.planes_a, g.planes_b, pa, pb)) {
            release(b);
            return rc;
        }
        descs[i].p[0] = pa;
        descs[i].p[1] = pb;
        descs[i].Xw = g.x_cells / 32;
        descs[i].Y = g.y_cells;
        groups[g.rule].grids.push_back(i);
        b->rounds[i] = (g.steps + groups[g.rule].k - 1) / groups[g.rule].k;
    }

    // work lists: for every group and round, every tile of every grid still running
    std::vector<batch_item> items;
    for (auto& gp : groups) {
        if (gp.grids.empty()) continue;
        const rule_ops* ops = ops_of(gp.rule);
        const int TW = 32 * ops->batch_words_per_lane;
        const int effW = TW - 2, effH = gp.TH - 2 * gp.HY;
        if (effH <= 0) {
            release(b);
            return fail(CELLATO_EINVAL, "rule %d: tile of %d rows leaves no interior for k=%d", gp.rule, gp.TH, gp.k);
        }
        int max_rounds = 0;
        for (int i : gp.grids) max_rounds = std::max(max_rounds, b->rounds[i]);
        for (int r = 0; r < max_rounds; ++r) {
            const int first = (int)items.size();
            for (int i : gp.grids) {
                if (r >= b->rounds[i]) continue;
                const int steps = std::min(gp.k, grids[i].steps - r * gp.k);
                const int tx = (descs[i].Xw + effW - 1) / effW, ty = (descs[i].Y + effH - 1) / effH;
                for (int y = 0; y < ty; ++y)
                    for (int x = 0; x < tx; ++x) items.push_back(batch_item{i, x, y, steps});
            }
            gp.rounds.emplace_back(first, (int)items.size() - first);
        }
    }
    b->work_items = (long long)items.size();

    const size_t desc_bytes = descs.size() * sizeof(batch_grid_desc);
    const size_t desc_pad = (desc_bytes + 255) / 256 * 256;
    const size_t total = desc_pad + items.size() * sizeof(batch_item) + 16;
    cudaError_t e = cudaMalloc(&b->device_buf, total);
    if (e != cudaSuccess) {
        release(b);
        return cuda_fail(e, "cudaMalloc (batch work lists)");
    }
    auto* d_descs = static_cast<batch_grid_desc*>(b->device_buf);
    auto* d_items = reinterpret_cast<batch_item*>(static_cast<char*>(b->device_buf) + desc_pad);
    if (!descs.empty()) e = cudaMemcpy(d_descs, descs.data(), desc_bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !items.empty())
        e = cudaMemcpy(d_items, items.data(), items.size() * sizeof(batch_item), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        release(b);
        return cuda_fail(e, "cudaMemcpy (batch work lists)");
    }

    // persistent CTAs: as many per SM as the tile's shared memory and the
    // kernel's registers allow
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    for (auto& gp : groups) {
        if (gp.rounds.empty()) continue;
        if ((e = ops_of(gp.rule)->prepare_batch(b->internal, gp.TH)) != cudaSuccess) {
            release(b);
            return cuda_fail(e, "batch kernel attributes");
        }
    }

    // capture: fork one stream per non-empty group from a root stream, join back
    cudaStream_t root;
    if ((e = cudaStreamCreateWithFlags(&root, cudaStreamNonBlocking)) != cudaSuccess) {
        release(b);
        return cuda_fail(e, "cudaStreamCreate");
    }
    b->streams.push_back(root);
    cudaEvent_t fork;
    cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    b->events.push_back(fork);
    e = cudaStreamBeginCapture(root, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaEventRecord(fork, root);
    std::vector<cudaEvent_t> joins;
    for (auto& gp : groups) {
        if (gp.rounds.empty() || e != cudaSuccess) continue;
        cudaStream_t s;
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        b->streams.push_back(s);
        e = cudaStreamWaitEvent(s, fork, 0);
        const int per_sm = ops_of(gp.rule)->batch_blocks_per_sm(b->internal, gp.TH);
        for (size_t r = 0; r < gp.rounds.size() && e == cudaSuccess; ++r) {
            const auto [first, count] = gp.rounds[r];
            if (count == 0) continue;
            const int ctas = std::min(count, per_sm * sms);
            e = ops_of(gp.rule)->temporal_batch(b->internal, d_descs, d_items + first, count, (int)(r & 1),
                                                (int)r * gp.k, gp.TH, gp.HY, ctas, s);
            ++b->launches;
        }
        cudaEvent_t j;
        cudaEventCreateWithFlags(&j, cudaEventDisableTiming);
        b->events.push_back(j);
        if (e == cudaSuccess) e = cudaEventRecord(j, s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(root, j, 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t e_end = cudaStreamEndCapture(root, &graph);
    if (e == cudaSuccess) e = e_end;
    b->graph = graph;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, graph, 0);
    if (e != cudaSuccess) {
        release(b);
        return cuda_fail(e, "building the batch graph");
    }
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
