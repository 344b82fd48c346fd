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
// Set-up: the device address of the array is obtained with
// cudaGetSymbolAddress on the first call on each device (that device current)
// and cached.  Make that first call before any stream capture.
//
// Sharing: all calls share the one array and it keeps the last call's
// contents.  Each call writes the complete work list it uses (nothing has to
// start at zero), stream-ordered before its kernels.  Calls whose work may
// overlap on the GPU -- on different streams, or from different host threads
// -- race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "capi_internal.hpp"
#include "cellato_b200.h"

using namespace cellato::b200;
using namespace cellato::b200::capi;

namespace {

constexpr int NOALLOC_MAX_GRIDS = CELLATO_NOALLOC_MAX_GRIDS;
constexpr int NOALLOC_MAX_ITEMS = CELLATO_NOALLOC_MAX_ITEMS;
constexpr size_t NOALLOC_DESC_BYTES = (NOALLOC_MAX_GRIDS * sizeof(batch_grid_desc) + 255) / 256 * 256;
constexpr size_t NOALLOC_SCRATCH_BYTES = NOALLOC_DESC_BYTES + NOALLOC_MAX_ITEMS * sizeof(batch_item);

// The work-list scratch: grid descriptors, then work items.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_scratch_mutex;
void* g_scratch_addr[MAX_DEVICES] = {};

// Device address of g_noalloc_scratch on the current device (the host-side
// name is only a stand-in for the device symbol).
int scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= MAX_DEVICES) return fail(CELLATO_EINVAL, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress (no-allocation scratch)");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return CELLATO_OK;
}

struct plan_group {
    int rule = 0, k = 8, TH = 0, HY = 0;
    std::vector<int> grids;
    std::vector<std::pair<int, int>> rounds;  // (first item, count)
};

}  // namespace

extern "C" int cellato_batch_run_noalloc(int layout, int word_bits, const cellato_batch_grid* grids, int n_grids,
                                         const int* k_per_rule, cellato_stream_t stream, int* result_in_b) {
    if (n_grids < 0 || (n_grids > 0 && (!grids || !result_in_b))) return fail(CELLATO_EINVAL, "bad grid or result array");
    if (n_grids > NOALLOC_MAX_GRIDS)
        return fail(CELLATO_EINVAL, "%d grids exceed the no-allocation limit of %d grids per call", n_grids,
                    NOALLOC_MAX_GRIDS);
    const int internal = internal_layout(layout, word_bits);
    const int R = band_height(layout, word_bits);

    std::vector<batch_grid_desc> descs(n_grids);
    std::vector<int> rounds(n_grids, 0);
    std::vector<plan_group> groups(CELLATO_RULE_COUNT);
    for (int r = 0; r < CELLATO_RULE_COUNT; ++r) {
        const int k = k_per_rule ? k_per_rule[r] : 0;
        groups[r].rule = r;
        groups[r].k = k > 0 ? std::min(k, 32) : 8;
        groups[r].TH = default_tile_rows(ops_of(r), R, groups[r].k, ops_of(r)->batch_words_per_lane);
        groups[r].HY = (groups[r].k + R - 1) / R * R;
    }
    for (int i = 0; i < n_grids; ++i) {
        const cellato_batch_grid& g = grids[i];
        const rule_ops* ops = ops_of(g.rule);
        if (!ops) return fail(CELLATO_EINVAL, "grid %d: unknown rule id %d", i, g.rule);
        if (g.steps < 0) return fail(CELLATO_EINVAL, "grid %d: negative step count", i);
        if (int rc = check_dims(layout, word_bits, g.x_cells, g.y_cells)) return rc;
        plane_set pa, pb;
        if (int rc = make_sets(ops, g.planes_a, g.planes_b, pa, pb)) return rc;
        descs[i].p[0] = pa;
        descs[i].p[1] = pb;
        descs[i].Xw = g.x_cells / 32;
        descs[i].Y = g.y_cells;
        groups[g.rule].grids.push_back(i);
        rounds[i] = (g.steps + groups[g.rule].k - 1) / groups[g.rule].k;
    }

    std::vector<batch_item> items;
    for (auto& gp : groups) {
        if (gp.grids.empty()) continue;
        const int effW = 32 * ops_of(gp.rule)->batch_words_per_lane - 2, effH = gp.TH - 2 * gp.HY;
        if (effH <= 0) return fail(CELLATO_EINVAL, "rule %d: tile leaves no interior for k=%d", gp.rule, gp.k);
        int max_rounds = 0;
        for (int i : gp.grids) max_rounds = std::max(max_rounds, rounds[i]);
        for (int r = 0; r < max_rounds; ++r) {
            const int first = (int)items.size();
            for (int i : gp.grids) {
                if (r >= rounds[i]) continue;
                const int steps = std::min(gp.k, grids[i].steps - r * gp.k);
                const int tx = (descs[i].Xw + effW - 1) / effW, ty = (descs[i].Y + effH - 1) / effH;
                if ((long long)items.size() + (long long)tx * ty > NOALLOC_MAX_ITEMS)
                    return fail(CELLATO_EINVAL,
                                "the batch needs more than %d work items (tiles x rounds), the no-allocation limit",
                                NOALLOC_MAX_ITEMS);
                for (int y = 0; y < ty; ++y)
                    for (int x = 0; x < tx; ++x) items.push_back(batch_item{i, x, y, steps});
            }
            gp.rounds.emplace_back(first, (int)items.size() - first);
        }
    }

    void* scratch = nullptr;
    if (int rc = scratch_address(&scratch)) return rc;
    auto* d_descs = static_cast<batch_grid_desc*>(scratch);
    auto* d_items = reinterpret_cast<batch_item*>(static_cast<unsigned char*>(scratch) + NOALLOC_DESC_BYTES);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaSuccess;
    if (n_grids > 0)
        e = cudaMemcpyAsync(d_descs, descs.data(), descs.size() * sizeof(batch_grid_desc), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !items.empty())
        e = cudaMemcpyAsync(d_items, items.data(), items.size() * sizeof(batch_item), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "copying the work list to the no-allocation scratch");

    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    for (auto& gp : groups) {
        if (gp.rounds.empty()) continue;
        const rule_ops* ops = ops_of(gp.rule);
        if ((e = ops->prepare_batch(internal, gp.TH)) != cudaSuccess) return cuda_fail(e, "batch kernel attributes");
        const int per_sm = ops->batch_blocks_per_sm(internal, gp.TH);
        for (size_t r = 0; r < gp.rounds.size(); ++r) {
            const auto [first, count] = gp.rounds[r];
            if (count == 0) continue;
            e = ops->temporal_batch(internal, d_descs, d_items + first, count, (int)(r & 1), (int)r * gp.k, gp.TH,
                                    gp.HY, std::min(count, per_sm * sms), s);
            if (e != cudaSuccess) return cuda_fail(e, "batched temporal launch");
        }
    }
    for (int i = 0; i < n_grids; ++i) result_in_b[i] = rounds[i] & 1;
    return CELLATO_OK;
}
