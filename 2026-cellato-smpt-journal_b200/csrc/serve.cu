// Simulation server (C ABI cellato_server_*): continuous batching of many
// grid-simulation requests on one device.  The policy -- admission, activation,
// the plan of each iteration -- is serve_schedule.hpp; this file owns the
// device side:
//   * a stream-ordered memory pool holding every resident request's two plane
//     buffers from admission to completion (no cudaMalloc on the request path);
//   * per iteration, one work list (grid descriptors + tile items, with each
//     item's ping-pong buffer and step parity in its flag bits) copied from a
//     pinned staging slot, then per automaton a chain of batched temporal
//     launches on its own stream, the automata forked from and joined back
//     into the server's main stream;
//   * for requests finishing in the iteration, the 4 x 4 tile checksum on the
//     device and one copy of all their sums back to pinned memory;
//   * up to max_inflight iterations queued ahead of the GPU; a slot is reused
//     only after the event of its previous iteration has completed.
// The reference has no server: its CLI runs one grid per process
// (src/main.cpp, include/experiments/experiment_manager.hpp:30-90).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <string>
#include <unordered_map>
#include <vector>

#include "capi_internal.hpp"
#include "cellato_b200.h"
#include "serve_schedule.hpp"

using namespace cellato::b200;
using namespace cellato::b200::capi;
namespace sv = cellato::b200::serve;

namespace {

constexpr size_t ALIGN = 256;
size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct req_rec {
    int rule = 0, x = 0, y = 0, steps = 0, nb = 0;
    size_t plane_bytes = 0, stride = 0;
    bool keep = false;
    bool random = true;
    unsigned long long seed = 0;
    std::vector<uint32_t> thresholds;
    std::vector<unsigned char> host;  // submitted planes, back to back, until admitted
    void* base = nullptr;             // both buffers: planes a then planes b
    plane_set p[2] = {};
    int cur = 0;
    bool completed = false;
    double submit_s = 0;
    int t0 = 0;  // number of the request's first step
};

struct slot {
    unsigned char* host = nullptr;
    size_t host_cap = 0;
    unsigned char* dev = nullptr;
    size_t dev_cap = 0;
    cudaEvent_t done = nullptr;
};

struct inflight_rec {
    int slot = 0;
    size_t sums_off = 0;
    std::vector<sv::finish_entry> finishing;
};

}  // namespace

struct cellato_server_st {
    int layout = 0, word_bits = 64, internal = 0, R = 1, dev = 0, sms = 148;
    int max_inflight = 2;
    sv::scheduler sched{sv::limits{}};
    cudaMemPool_t pool = nullptr;       // planes of requests the server drops when they finish; work lists
    cudaMemPool_t keep_pool = nullptr;  // planes of requests kept after they finish (keep)
    cudaStream_t main_stream = nullptr;
    cudaEvent_t fork = nullptr;
    // per rule id, set up when the first request of that rule is submitted
    // (rules registered after the server was created work too)
    std::vector<cudaStream_t> rs;
    std::vector<cudaEvent_t> join;
    std::vector<int> TH, HY;
    std::vector<int> per_sm;  // resident CTAs per SM of each rule's batched kernel (0: not set up)
    std::vector<slot> slots;
    int next_slot = 0;
    std::deque<inflight_rec> inflight;
    std::unordered_map<long long, req_rec> recs;
    std::deque<cellato_server_result> completed;
    long long iterations = 0, launches = 0, last_active = 0, pool_trims = 0, memory_waits = 0;
    double cell_steps = 0;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    bool broken = false;

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

int server_cuda_fail(cellato_server_st* s, cudaError_t e, const char* what) {
    s->broken = true;
    return cuda_fail(e, what);
}

void destroy_all(cellato_server_st* s) {
    if (!s) return;
    cudaStream_t m = s->main_stream;
    if (m) cudaStreamSynchronize(m);
    for (auto& [id, r] : s->recs)
        if (r.base && m) cudaFreeAsync(r.base, m);
    for (auto& sl : s->slots) {
        if (sl.dev && m) cudaFreeAsync(sl.dev, m);
        if (sl.host) cudaFreeHost(sl.host);
        if (sl.done) cudaEventDestroy(sl.done);
    }
    if (m) cudaStreamSynchronize(m);
    for (size_t r = 0; r < s->rs.size(); ++r) {
        if (s->rs[r]) cudaStreamDestroy(s->rs[r]);
        if (s->join[r]) cudaEventDestroy(s->join[r]);
    }
    if (s->fork) cudaEventDestroy(s->fork);
    if (m) cudaStreamDestroy(m);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    if (s->keep_pool) cudaMemPoolDestroy(s->keep_pool);
    delete s;
}

// Moves the oldest queued iteration's finished requests to the completed list
// once its event has completed.  Returns 1 if one was collected, 0 if none is
// queued or it is still running (non-blocking), or a negated status.
int harvest_one(cellato_server_st* s, bool block) {
    if (s->inflight.empty()) return 0;
    inflight_rec& f = s->inflight.front();
    slot& sl = s->slots[f.slot];
    const cudaError_t e = block ? cudaEventSynchronize(sl.done) : cudaEventQuery(sl.done);
    if (e == cudaErrorNotReady) return 0;
    if (e != cudaSuccess) return -server_cuda_fail(s, e, "waiting for a server iteration");
    const double t = s->now();
    const auto* sums = reinterpret_cast<const unsigned long long*>(sl.host + f.sums_off);
    for (size_t j = 0; j < f.finishing.size(); ++j) {
        const long long id = f.finishing[j].id;
        req_rec& r = s->recs[id];
        cellato_server_result res{};
        res.id = id;
        res.rule = r.rule;
        res.x_cells = r.x, res.y_cells = r.y, res.steps = r.steps;
        res.result_in_b = f.finishing[j].cur;
        std::memcpy(res.checksum, sums + 16 * j, sizeof res.checksum);
        res.submit_s = r.submit_s;
        res.done_s = t;
        s->completed.push_back(res);
        r.completed = true;
        if (!f.finishing[j].keep) s->recs.erase(id);
    }
    s->inflight.pop_front();
    return 1;
}

int harvest_ready(cellato_server_st* s) {
    for (;;) {
        const int rc = harvest_one(s, false);
        if (rc <= 0) return rc < 0 ? -rc : CELLATO_OK;
    }
}

// Waits for every queued iteration and collects its results.
int drain(cellato_server_st* s) {
    while (!s->inflight.empty()) {
        const int rc = harvest_one(s, true);
        if (rc < 0) return -rc;
    }
    return CELLATO_OK;
}

// A block of one of the server's pools, stream-ordered on the main stream.
// The pools keep freed blocks for later admissions; over a long stream of
// mixed sizes they fragment, and a pool can run out of device memory while the
// resident total is within the cap.  Then the frees already issued are
// completed, both pools' unused blocks are returned to the device, and the
// allocation is tried once more.  Kept requests, which outlive the ones around
// them, have a pool of their own so that they pin no blocks of the main one.
cudaError_t pool_alloc(cellato_server_st* s, void** p, size_t bytes, bool keep = false) {
    cudaMemPool_t pool = keep ? s->keep_pool : s->pool;
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, pool, s->main_stream);
    if (e != cudaErrorMemoryAllocation) return e;
    (void)cudaGetLastError();
    if ((e = cudaStreamSynchronize(s->main_stream)) != cudaSuccess) return e;
    if ((e = cudaMemPoolTrimTo(s->pool, 0)) != cudaSuccess) return e;
    if ((e = cudaMemPoolTrimTo(s->keep_pool, 0)) != cudaSuccess) return e;
    ++s->pool_trims;
    return cudaMallocFromPoolAsync(p, bytes, pool, s->main_stream);
}

int ensure_slot(cellato_server_st* s, slot& sl, size_t bytes) {
    if (sl.host_cap < bytes) {
        if (sl.host) cudaFreeHost(sl.host);
        sl.host = nullptr;
        sl.host_cap = 0;
        const size_t cap = round_up(bytes + bytes / 2, 1 << 16);
        const cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&sl.host), cap);
        if (e != cudaSuccess) return server_cuda_fail(s, e, "cudaMallocHost (server staging)");
        sl.host_cap = cap;
    }
    if (sl.dev_cap < bytes) {
        if (sl.dev) cudaFreeAsync(sl.dev, s->main_stream);
        sl.dev = nullptr;
        sl.dev_cap = 0;
        const size_t cap = round_up(bytes + bytes / 2, 1 << 16);
        const cudaError_t e = pool_alloc(s, reinterpret_cast<void**>(&sl.dev), cap);
        if (e != cudaSuccess) return server_cuda_fail(s, e, "cudaMallocFromPoolAsync (server work list)");
        sl.dev_cap = cap;
    }
    return CELLATO_OK;
}

// Allocates and initialises an admitted request's planes on the main stream.
// Returns NO_MEMORY, with nothing allocated, when the device has no room left.
constexpr int NO_MEMORY = -1;
int materialise(cellato_server_st* s, long long id) {
    req_rec& r = s->recs[id];
    const size_t bytes = 2 * (size_t)r.nb * r.stride;
    cudaError_t e = pool_alloc(s, &r.base, bytes, r.keep);
    if (e == cudaErrorMemoryAllocation) {
        (void)cudaGetLastError();
        r.base = nullptr;
        return NO_MEMORY;
    }
    if (e != cudaSuccess) return server_cuda_fail(s, e, "cudaMallocFromPoolAsync (request planes)");
    auto* b = static_cast<unsigned char*>(r.base);
    for (int p = 0; p < r.nb; ++p) {
        r.p[0].p[p] = reinterpret_cast<word*>(b + (size_t)p * r.stride);
        r.p[1].p[p] = reinterpret_cast<word*>(b + (size_t)(r.nb + p) * r.stride);
    }
    if (r.random) {
        if (int rc = enqueue_fill_random(s->layout, s->word_bits, r.nb, r.p[0], r.x, r.y, r.seed,
                                         r.thresholds.data(), (int)r.thresholds.size(), s->main_stream)) {
            s->broken = true;
            return rc;
        }
        ++s->launches;
    } else {
        for (int p = 0; p < r.nb; ++p) {
            e = cudaMemcpyAsync(r.p[0].p[p], r.host.data() + (size_t)p * r.plane_bytes, r.plane_bytes,
                                cudaMemcpyHostToDevice, s->main_stream);
            if (e != cudaSuccess) return server_cuda_fail(s, e, "cudaMemcpyAsync (request planes)");
        }
        // a copy from pageable memory returns once the source has been staged
        std::vector<unsigned char>().swap(r.host);
    }
    return CELLATO_OK;
}

// Tile shape, kernel attributes, stream and join event of a rule, on the
// first request of it.
int ensure_rule(cellato_server_st* s, int rule) {
    if ((int)s->per_sm.size() > rule && s->per_sm[rule] > 0) return CELLATO_OK;
    const rule_ops* ops = ops_of(rule);
    if ((int)s->per_sm.size() <= rule) {
        s->rs.resize(rule + 1, nullptr);
        s->join.resize(rule + 1, nullptr);
        s->TH.resize(rule + 1, 0);
        s->HY.resize(rule + 1, 0);
        s->per_sm.resize(rule + 1, 0);
    }
    const int k = s->sched.lim().k_of(rule);
    s->TH[rule] = default_tile_rows(ops, s->R, k, ops->batch_words_per_lane);
    s->HY[rule] = (k + s->R - 1) / s->R * s->R;
    if (s->TH[rule] - 2 * s->HY[rule] <= 0)
        return fail(CELLATO_EINVAL, "rule %d: a %d-row tile leaves no interior for k=%d", rule, s->TH[rule], k);
    cudaError_t e = ops->prepare_batch(s->internal, s->TH[rule]);
    if (e == cudaSuccess && !s->rs[rule]) e = cudaStreamCreateWithFlags(&s->rs[rule], cudaStreamNonBlocking);
    if (e == cudaSuccess && !s->join[rule]) e = cudaEventCreateWithFlags(&s->join[rule], cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(e, "setting up a rule's batched kernel");
    s->per_sm[rule] = ops->batch_blocks_per_sm(s->internal, s->TH[rule]);
    return CELLATO_OK;
}

int submit_common(cellato_server_t s, int rule, int x, int y, int steps, int t0, int keep, req_rec& r,
                  long long* id) {
    if (!s || !id) return fail(CELLATO_EINVAL, "server and id must not be NULL");
    if (s->broken) return fail(CELLATO_ECUDA, "the server stopped after a CUDA error");
    const rule_ops* ops = ops_of(rule);
    if (!ops) return fail(CELLATO_EINVAL, "unknown rule id %d", rule);
    if (steps < 0) return fail(CELLATO_EINVAL, "negative step count");
    if (int rc = check_dims(s->layout, s->word_bits, x, y)) return rc;
    if (int rc = ensure_rule(s, rule)) return rc;
    r.rule = rule, r.x = x, r.y = y, r.steps = steps, r.nb = ops->planes;
    r.keep = keep != 0;
    r.t0 = t0;
    r.plane_bytes = (size_t)x * y / 8;
    r.stride = round_up(r.plane_bytes, ALIGN);
    const int effW = 32 * ops->batch_words_per_lane - 2, effH = s->TH[rule] - 2 * s->HY[rule];
    const int tiles = ((x / 32 + effW - 1) / effW) * ((y + effH - 1) / effH);
    r.submit_s = s->now();
    *id = s->sched.submit(rule, x, y, steps, (long long)(2 * (size_t)r.nb * r.stride), tiles, r.keep, t0 & 1);
    s->recs.emplace(*id, std::move(r));
    return CELLATO_OK;
}

}  // namespace

extern "C" {

int cellato_server_create(const cellato_server_config* cfg, cellato_server_t* out) {
    if (!cfg || !out) return fail(CELLATO_EINVAL, "config and out must not be NULL");
    *out = nullptr;
    if (int rc = check_dims(cfg->layout, cfg->word_bits, 64, 64)) return rc;
    sv::limits lim;
    if (cfg->n_k_per_rule < 0 || (cfg->n_k_per_rule > 0 && !cfg->k_per_rule))
        return fail(CELLATO_EINVAL, "bad k_per_rule array");
    for (int r = 0; r < cfg->n_k_per_rule; ++r) {
        const int k = cfg->k_per_rule[r];
        if (k < 0 || k > 32) return fail(CELLATO_EINVAL, "k for rule %d must be in 1..32 (0 = 16), got %d", r, k);
        lim.k.push_back(k ? k : 16);
    }
    auto* s = new cellato_server_st;
    s->layout = cfg->layout;
    s->word_bits = cfg->word_bits;
    s->internal = internal_layout(cfg->layout, cfg->word_bits);
    s->R = band_height(cfg->layout, cfg->word_bits);
    s->max_inflight = std::min(8, std::max(1, cfg->max_inflight ? cfg->max_inflight : 2));
    cudaError_t e = cudaGetDevice(&s->dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->dev);
    size_t free_b = 0, total_b = 0;
    if (e == cudaSuccess) e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess) {
        destroy_all(s);
        return cuda_fail(e, "querying the device");
    }
    lim.cap_bytes = cfg->hbm_cap_bytes ? (long long)cfg->hbm_cap_bytes : (long long)(0.8 * (double)total_b);
    // default budget: 1024 tile words per SM per round (32 one-word-per-lane tiles), about seven waves of
    // three CTAs per SM, enough to fill the device with each automaton's launch
    lim.tile_budget = cfg->tile_budget > 0 ? cfg->tile_budget : 32LL * s->sms;
    lim.chunk_rounds = cfg->chunk_rounds > 0 ? cfg->chunk_rounds : 4;
    s->sched = sv::scheduler(lim);

    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = s->dev;
    e = cudaMemPoolCreate(&s->pool, &props);
    if (e == cudaSuccess) e = cudaMemPoolCreate(&s->keep_pool, &props);
    unsigned long long keep_all = ~0ull;  // freed blocks stay in the pools for the next admissions
    if (e == cudaSuccess) e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep_all);
    if (e == cudaSuccess) e = cudaMemPoolSetAttribute(s->keep_pool, cudaMemPoolAttrReleaseThreshold, &keep_all);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->main_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming);
    s->slots.resize(s->max_inflight);
    for (auto& sl : s->slots)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        destroy_all(s);
        return cuda_fail(e, "creating the server's pool, streams and events");
    }
    *out = s;
    return CELLATO_OK;
}

int cellato_server_submit_random(cellato_server_t s, int rule, int x, int y, int steps, unsigned long long seed,
                                 const uint32_t* thresholds, int n_thresholds, int keep, long long* id) {
    const rule_ops* ops = ops_of(rule);
    if (!ops) return fail(CELLATO_EINVAL, "unknown rule id %d", rule);
    if (n_thresholds < 0 || n_thresholds > 31 || (n_thresholds > 0 && !thresholds) ||
        n_thresholds >= (1 << ops->planes))
        return fail(CELLATO_EINVAL, "bad threshold count %d for %d planes", n_thresholds, ops->planes);
    for (int i = 1; i < n_thresholds; ++i)
        if (thresholds[i] < thresholds[i - 1]) return fail(CELLATO_EINVAL, "thresholds must be ascending");
    req_rec r;
    r.random = true;
    r.seed = seed;
    if (n_thresholds) r.thresholds.assign(thresholds, thresholds + n_thresholds);
    return submit_common(s, rule, x, y, steps, 0, keep, r, id);
}

int cellato_server_submit_resume(cellato_server_t s, int rule, int x, int y, int steps, int t0,
                                 const void* const* host_planes, int keep, long long* id) {
    if (!s) return fail(CELLATO_EINVAL, "server is NULL");
    const rule_ops* ops = ops_of(rule);
    if (!ops) return fail(CELLATO_EINVAL, "unknown rule id %d", rule);
    if (!host_planes) return fail(CELLATO_EINVAL, "host_planes must not be NULL");
    if (int rc = check_dims(s->layout, s->word_bits, x, y)) return rc;
    req_rec r;
    r.random = false;
    const size_t pb = (size_t)x * y / 8;
    r.host.resize(pb * ops->planes);
    for (int p = 0; p < ops->planes; ++p) {
        if (!host_planes[p]) return fail(CELLATO_EINVAL, "host plane %d is NULL", p);
        std::memcpy(r.host.data() + p * pb, host_planes[p], pb);
    }
    if (t0 < 0) return fail(CELLATO_EINVAL, "negative start step");
    return submit_common(s, rule, x, y, steps, t0, keep, r, id);
}

int cellato_server_submit_planes(cellato_server_t s, int rule, int x, int y, int steps,
                                 const void* const* host_planes, int keep, long long* id) {
    return cellato_server_submit_resume(s, rule, x, y, steps, 0, host_planes, keep, id);
}

int cellato_server_iterate(cellato_server_t s, int* active) {
    if (!s) return fail(CELLATO_EINVAL, "server is NULL");
    if (s->broken) return fail(CELLATO_ECUDA, "the server stopped after a CUDA error");
    if (active) *active = 0;
    if (int rc = harvest_ready(s)) return rc;
    while ((int)s->inflight.size() >= s->max_inflight) {
        const int rc = harvest_one(s, true);
        if (rc < 0) return -rc;
    }
    {
        const std::vector<long long> admitted = s->sched.admit();
        for (size_t i = 0; i < admitted.size(); ++i) {
            const int rc = materialise(s, admitted[i]);
            if (rc == NO_MEMORY) {
                // back-pressure: this request and the later ones wait, the
                // cap falls to what is resident; a request that holds the
                // device alone and still finds no room can never run
                const req_rec& r = s->recs[admitted[i]];
                if (i == 0 && s->sched.resident_bytes() == (long long)(2 * (size_t)r.nb * r.stride)) {
                    s->broken = true;
                    return fail(CELLATO_ECUDA, "request %lld does not fit in device memory alone", admitted[i]);
                }
                s->sched.unadmit(std::vector<long long>(admitted.begin() + i, admitted.end()));
                ++s->memory_waits;
                break;
            }
            if (rc) return rc;
        }
    }

    sv::iteration_plan plan = s->sched.plan();
    s->last_active = (long long)plan.active.size();
    if (plan.empty()) {
        const int rc = harvest_one(s, true);
        return rc < 0 ? -rc : CELLATO_OK;
    }

    // work list: one descriptor per active request, then per automaton the items
    // of all its rounds (ordered by round); each automaton's rounds are one
    // persistent launch in which a request's next round starts when its
    // previous one is done
    std::unordered_map<long long, int> desc_of;
    std::vector<batch_grid_desc> descs;
    descs.reserve(plan.active.size());
    for (long long id : plan.active) {
        const req_rec& r = s->recs[id];
        const rule_ops* ops = ops_of(r.rule);
        const int effW = 32 * ops->batch_words_per_lane - 2, effH = s->TH[r.rule] - 2 * s->HY[r.rule];
        desc_of[id] = (int)descs.size();
        batch_grid_desc d{};
        d.p[0] = r.p[0];
        d.p[1] = r.p[1];
        d.Xw = r.x / 32;
        d.Y = r.y;
        d.tiles = ((d.Xw + effW - 1) / effW) * ((r.y + effH - 1) / effH);
        descs.push_back(d);
    }
    struct launch_rec {
        int rule, first, count;
    };
    std::vector<batch_item> items;
    std::vector<launch_rec> launches;
    for (int rule = 0; rule < (int)plan.rounds.size(); ++rule) {
        if (plan.rounds[rule].empty()) continue;
        const rule_ops* ops = ops_of(rule);
        const int effW = 32 * ops->batch_words_per_lane - 2, effH = s->TH[rule] - 2 * s->HY[rule];
        const int first = (int)items.size();
        for (size_t q = 0; q < plan.rounds[rule].size(); ++q) {
            for (const sv::round_entry& en : plan.rounds[rule][q]) {
                const req_rec& r = s->recs[en.id];
                const int tx = (r.x / 32 + effW - 1) / effW, ty = (r.y + effH - 1) / effH;
                const int flags = en.steps | (en.src ? BATCH_FLIP_BUFFER : 0) | (en.tpar ? BATCH_FLIP_TIME : 0) |
                                  ((int)q << BATCH_ROUND_SHIFT);
                const int g = desc_of[en.id];
                for (int yy = 0; yy < ty; ++yy)
                    for (int xx = 0; xx < tx; ++xx) items.push_back(batch_item{g, xx, yy, flags});
            }
        }
        launches.push_back(launch_rec{rule, first, (int)items.size() - first});
    }
    const size_t desc_bytes = round_up(descs.size() * sizeof(batch_grid_desc), ALIGN);
    const size_t item_bytes = round_up(items.size() * sizeof(batch_item), ALIGN);
    // queue head per launch, finished-tile count per descriptor; cleared each iteration
    const size_t sync_words = launches.size() + descs.size();
    const size_t sync_bytes = round_up(sync_words * sizeof(unsigned), ALIGN);
    const size_t sums_bytes = plan.finishing.size() * 16 * sizeof(unsigned long long);
    const int si = s->next_slot;
    slot& sl = s->slots[si];
    if (int rc = ensure_slot(s, sl, desc_bytes + item_bytes + sync_bytes + sums_bytes + ALIGN)) return rc;
    std::memcpy(sl.host, descs.data(), descs.size() * sizeof(batch_grid_desc));
    std::memcpy(sl.host + desc_bytes, items.data(), items.size() * sizeof(batch_item));
    std::memset(sl.host + desc_bytes + item_bytes, 0, sync_bytes);
    cudaStream_t m = s->main_stream;
    cudaError_t e = cudaMemcpyAsync(sl.dev, sl.host, desc_bytes + item_bytes + sync_bytes, cudaMemcpyHostToDevice, m);
    if (e != cudaSuccess) return server_cuda_fail(s, e, "cudaMemcpyAsync (server work list)");
    const auto* d_descs = reinterpret_cast<const batch_grid_desc*>(sl.dev);
    const auto* d_items = reinterpret_cast<const batch_item*>(sl.dev + desc_bytes);
    auto* d_sync = reinterpret_cast<unsigned*>(sl.dev + desc_bytes + item_bytes);
    unsigned* d_done = d_sync + launches.size();

    if ((e = cudaEventRecord(s->fork, m)) != cudaSuccess) return server_cuda_fail(s, e, "cudaEventRecord");
    std::vector<char> used(s->rs.size(), 0);
    for (size_t li = 0; li < launches.size(); ++li) {
        const launch_rec& L = launches[li];
        if (L.count == 0) continue;
        cudaStream_t st = s->rs[L.rule];
        used[L.rule] = 1;
        if ((e = cudaStreamWaitEvent(st, s->fork, 0)) != cudaSuccess)
            return server_cuda_fail(s, e, "cudaStreamWaitEvent");
        e = ops_of(L.rule)->temporal_batch(s->internal, d_descs, d_items + L.first, L.count, 0, 0, s->TH[L.rule],
                                           s->HY[L.rule], d_sync + li, d_done,
                                           std::min(L.count, s->per_sm[L.rule] * s->sms), st);
        if (e != cudaSuccess) return server_cuda_fail(s, e, "batched temporal launch (server)");
        ++s->launches;
    }
    for (int rule = 0; rule < (int)used.size(); ++rule) {
        if (!used[rule]) continue;
        if ((e = cudaEventRecord(s->join[rule], s->rs[rule])) != cudaSuccess ||
            (e = cudaStreamWaitEvent(m, s->join[rule], 0)) != cudaSuccess)
            return server_cuda_fail(s, e, "joining the rule streams");
    }

    // finishing requests: checksums on the device, one copy back, free unkept planes
    inflight_rec f;
    f.slot = si;
    f.sums_off = desc_bytes + item_bytes + sync_bytes;
    f.finishing = plan.finishing;
    auto* d_sums = reinterpret_cast<unsigned long long*>(sl.dev + f.sums_off);
    for (size_t j = 0; j < plan.finishing.size(); ++j) {
        req_rec& r = s->recs[plan.finishing[j].id];
        r.cur = plan.finishing[j].cur;
        if (int rc = enqueue_checksum(ops_of(r.rule), s->layout, s->word_bits, r.p[r.cur], r.x, r.y, d_sums + 16 * j,
                                      m)) {
            s->broken = true;
            return rc;
        }
        ++s->launches;
        if (!plan.finishing[j].keep) {
            if ((e = cudaFreeAsync(r.base, m)) != cudaSuccess) return server_cuda_fail(s, e, "cudaFreeAsync");
            r.base = nullptr;
        }
    }
    if (sums_bytes &&
        (e = cudaMemcpyAsync(sl.host + f.sums_off, d_sums, sums_bytes, cudaMemcpyDeviceToHost, m)) != cudaSuccess)
        return server_cuda_fail(s, e, "cudaMemcpyAsync (checksums)");
    if ((e = cudaEventRecord(sl.done, m)) != cudaSuccess) return server_cuda_fail(s, e, "cudaEventRecord");
    s->inflight.push_back(std::move(f));
    s->next_slot = (si + 1) % (int)s->slots.size();
    ++s->iterations;
    s->cell_steps += (double)plan.cell_steps;
    if (active) *active = (int)plan.active.size();
    return CELLATO_OK;
}

int cellato_server_poll(cellato_server_t s, cellato_server_result* out, int max, int* n) {
    if (!s || !n || (max > 0 && !out)) return fail(CELLATO_EINVAL, "bad server, output or count");
    *n = 0;
    if (!s->broken)
        if (int rc = harvest_ready(s)) return rc;
    while (*n < max && !s->completed.empty()) {
        out[(*n)++] = s->completed.front();
        s->completed.pop_front();
    }
    return CELLATO_OK;
}

int cellato_server_planes(cellato_server_t s, long long id, void** planes) {
    if (!s || !planes) return fail(CELLATO_EINVAL, "server and planes must not be NULL");
    auto it = s->recs.find(id);
    if (it == s->recs.end() || !it->second.keep || !it->second.completed)
        return fail(CELLATO_EINVAL, "request %lld is not a completed request kept by the server", id);
    for (int p = 0; p < it->second.nb; ++p) planes[p] = it->second.p[it->second.cur].p[p];
    return CELLATO_OK;
}

int cellato_server_release(cellato_server_t s, long long id) {
    if (!s) return fail(CELLATO_EINVAL, "server is NULL");
    auto it = s->recs.find(id);
    if (it == s->recs.end() || !it->second.keep || !it->second.completed)
        return fail(CELLATO_EINVAL, "request %lld is not a completed request kept by the server", id);
    if (it->second.base) {
        const cudaError_t e = cudaFreeAsync(it->second.base, s->main_stream);
        if (e != cudaSuccess) return server_cuda_fail(s, e, "cudaFreeAsync");
    }
    s->sched.release(id);
    s->recs.erase(it);
    return CELLATO_OK;
}

int cellato_server_snapshot(cellato_server_t s, long long id, void* const* host_planes, int* steps_done,
                            int* next_step) {
    if (!s || !host_planes) return fail(CELLATO_EINVAL, "server and host_planes must not be NULL");
    if (s->broken) return fail(CELLATO_ECUDA, "the server stopped after a CUDA error");
    if (int rc = drain(s)) return rc;
    const sv::request* q = s->sched.find(id);
    auto it = s->recs.find(id);
    if (!q || it == s->recs.end() || q->ph == sv::phase::waiting || !it->second.base)
        return fail(CELLATO_EINVAL, "request %lld has no state on the device (unknown, not admitted or freed)", id);
    const req_rec& r = it->second;
    for (int p = 0; p < r.nb; ++p) {
        if (!host_planes[p]) return fail(CELLATO_EINVAL, "host plane %d is NULL", p);
        const cudaError_t e = cudaMemcpyAsync(host_planes[p], r.p[q->cur].p[p], r.plane_bytes,
                                              cudaMemcpyDeviceToHost, s->main_stream);
        if (e != cudaSuccess) return server_cuda_fail(s, e, "cudaMemcpyAsync (snapshot)");
    }
    const cudaError_t e = cudaStreamSynchronize(s->main_stream);
    if (e != cudaSuccess) return server_cuda_fail(s, e, "cudaStreamSynchronize (snapshot)");
    if (steps_done) *steps_done = q->done;
    if (next_step) *next_step = r.t0 + q->done;
    return CELLATO_OK;
}

int cellato_server_cancel(cellato_server_t s, long long id) {
    if (!s) return fail(CELLATO_EINVAL, "server is NULL");
    if (s->broken) return fail(CELLATO_ECUDA, "the server stopped after a CUDA error");
    if (int rc = drain(s)) return rc;
    auto it = s->recs.find(id);
    if (!s->sched.find(id) || it == s->recs.end()) return fail(CELLATO_EINVAL, "request %lld is not held", id);
    if (it->second.base) {
        const cudaError_t e = cudaFreeAsync(it->second.base, s->main_stream);
        if (e != cudaSuccess) return server_cuda_fail(s, e, "cudaFreeAsync");
    }
    s->sched.cancel(id);
    s->recs.erase(it);
    // a result not yet polled goes too
    s->completed.erase(std::remove_if(s->completed.begin(), s->completed.end(),
                                      [id](const cellato_server_result& r) { return r.id == id; }),
                       s->completed.end());
    return CELLATO_OK;
}

int cellato_server_stats_get(cellato_server_t s, cellato_server_stats* st) {
    if (!s || !st) return fail(CELLATO_EINVAL, "server and stats must not be NULL");
    st->waiting = (long long)s->sched.n_waiting();
    st->running = (long long)s->sched.n_running();
    st->active = s->last_active;
    st->completed_unpolled = (long long)s->completed.size();
    st->resident_bytes = (unsigned long long)s->sched.resident_bytes();
    st->hbm_cap_bytes = (unsigned long long)s->sched.lim().cap_bytes;
    st->iterations = s->iterations;
    st->kernel_launches = s->launches;
    st->cell_steps = s->cell_steps;
    st->pool_trims = s->pool_trims;
    st->memory_waits = s->memory_waits;
    return CELLATO_OK;
}

int cellato_server_destroy(cellato_server_t s) {
    destroy_all(s);
    return CELLATO_OK;
}

}  // extern "C"
