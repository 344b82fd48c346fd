// C ABI of the B200 bit-plane hot path (declared in include/cellato_b200.h).
// Argument checking, rule dispatch and the traverser loops; the kernels live in
// engine.cuh and are instantiated per rule in rule_<automaton>.cu.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "cellato_b200.h"
#include "capi_internal.hpp"

namespace cellato::b200 {
extern const rule_ops rule_ops_0, rule_ops_1, rule_ops_2, rule_ops_3, rule_ops_4, rule_ops_5, rule_ops_6,
    rule_ops_7, rule_ops_8, rule_ops_9;
}

using namespace cellato::b200;

namespace cellato::b200::capi {

thread_local std::string g_last_error;

int fail(int status, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return status;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(CELLATO_ECUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

// The rule table: the ten built-in rules, then registered ones in order.
// Entries are written once, before the count that publishes them, so readers
// take no lock.
namespace {
const rule_ops* g_rules[CELLATO_MAX_RULES] = {&rule_ops_0, &rule_ops_1, &rule_ops_2, &rule_ops_3, &rule_ops_4,
                                              &rule_ops_5, &rule_ops_6, &rule_ops_7, &rule_ops_8, &rule_ops_9};
std::atomic<int> g_rule_count{CELLATO_BUILTIN_RULES};
std::mutex g_register_mutex;
}  // namespace

int rule_count() { return g_rule_count.load(std::memory_order_acquire); }

const rule_ops* ops_of(int rule) {
    return (rule >= 0 && rule < rule_count()) ? g_rules[rule] : nullptr;
}

// Internal layout id and tile band height.
int internal_layout(int layout, int word_bits) {
    if (layout == CELLATO_LAYOUT_BIT_PLANES) return LAYOUT_LINEAR;
    return word_bits == 32 ? LAYOUT_TILED4 : LAYOUT_TILED8;
}

int band_height(int layout, int word_bits) {
    return layout == CELLATO_LAYOUT_BIT_PLANES ? 1 : word_bits / 8;
}

int check_dims(int layout, int word_bits, int X, int Y) {
    if (word_bits != 32 && word_bits != 64) return fail(CELLATO_EINVAL, "word_bits must be 32 or 64 (got %d)", word_bits);
    if (layout != CELLATO_LAYOUT_BIT_PLANES && layout != CELLATO_LAYOUT_TILED_BIT_PLANES)
        return fail(CELLATO_EINVAL, "unknown layout %d", layout);
    if (X <= 0 || Y <= 0) return fail(CELLATO_EINVAL_DIMS, "grid %d x %d is empty", X, Y);
    if (X % 32 != 0) return fail(CELLATO_EINVAL_DIMS, "x_size %d is not a multiple of 32", X);
    if (layout == CELLATO_LAYOUT_BIT_PLANES && X % word_bits != 0)
        return fail(CELLATO_EINVAL_DIMS, "x_size %d is not a multiple of the word size %d", X, word_bits);
    if (layout == CELLATO_LAYOUT_TILED_BIT_PLANES && Y % (word_bits / 8) != 0)
        return fail(CELLATO_EINVAL_DIMS, "y_size %d is not a multiple of the tile height %d", Y, word_bits / 8);
    if ((long long)X * Y / 32 > 0x7fffffffLL)
        return fail(CELLATO_EINVAL_DIMS, "grid %d x %d has more than 2^31 words per plane", X, Y);
    return CELLATO_OK;
}

int make_sets(const rule_ops* ops, void* const* a, void* const* b, plane_set& pa, plane_set& pb) {
    if (!a || !b) return fail(CELLATO_EINVAL, "plane arrays must not be NULL");
    std::memset(&pa, 0, sizeof pa);
    std::memset(&pb, 0, sizeof pb);
    for (int p = 0; p < ops->planes; ++p) {
        if (!a[p] || !b[p]) return fail(CELLATO_EINVAL, "plane %d pointer is NULL", p);
        if ((reinterpret_cast<uintptr_t>(a[p]) | reinterpret_cast<uintptr_t>(b[p])) & 15)
            return fail(CELLATO_EINVAL, "plane %d pointer is not 16-byte aligned", p);
        if (a[p] == b[p]) return fail(CELLATO_EINVAL, "plane %d: input and output buffers alias", p);
        pa.p[p] = static_cast<word*>(a[p]);
        pb.p[p] = static_cast<word*>(b[p]);
    }
    return CELLATO_OK;
}

int max_optin_smem() {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
    return v;
}

// Default tile height for k fused steps: `interior` rows plus the two halos
// (HY = ceil(k/R)*R rows each).  The cap is the tallest tile that lets three
// CTAs share an SM when that still leaves 96 interior rows, otherwise two.
// Taller tiles waste less on halos but leave fewer CTAs for the 148 SMs and
// fewer resident warps per SM.  Single grids use 224 interior rows for rules
// of two or more planes (with one word per lane, on B200 at 16384^2 and
// k = 16, 3-13% faster than two words per lane and 128 rows for the seven
// such rules, both layouts) and 128 for one-plane rules (224 is 2-7% slower
// there); batches, with their many small grids, use 128.
int default_tile_rows(const rule_ops* ops, int R, int k, int V, int interior) {
    const int row_bytes = ops->planes * 32 * V * 4;
    const int q = std::max(ops->temporal_warps, R);
    const int HY = (std::max(1, k) + R - 1) / R * R;
    const int three_per_sm = (75 * 1024) / row_bytes / q * q;
    const int two_per_sm = (113 * 1024) / row_bytes / q * q;
    const int cap = three_per_sm >= 2 * HY + 96 ? three_per_sm : two_per_sm;
    const int want = (2 * HY + interior + q - 1) / q * q;
    return std::min(want, std::max(cap, (2 * HY + q) / q * q));
}

}  // namespace cellato::b200::capi

using namespace cellato::b200::capi;

extern "C" {

const char* cellato_version(void) { return "cellato-b200 1.0 sm_100a"; }

const char* cellato_last_error(void) { return g_last_error.c_str(); }

int cellato_rule_from_name(const char* name) {
    if (!name) return -1;
    if (std::strcmp(name, "fire") == 0) return CELLATO_FOREST_FIRE;
    const int n = rule_count();
    for (int r = 0; r < n; ++r)
        if (std::strcmp(name, ops_of(r)->name) == 0) return r;
    return -1;
}

int cellato_rule_count(void) { return rule_count(); }

int cellato_rule_register(const cellato_rule_ops* ops, int* rule_out) {
    if (!ops || !rule_out) return fail(CELLATO_EINVAL, "ops and rule_out must not be NULL");
    *rule_out = -1;
    if (ops->abi_version != CELLATO_RULE_OPS_ABI || ops->struct_size != (int)sizeof(rule_ops))
        return fail(CELLATO_EINVAL, "rule table built for rule_ops ABI %d (size %d); this library has ABI %d (size %d)",
                    ops->abi_version, ops->struct_size, CELLATO_RULE_OPS_ABI, (int)sizeof(rule_ops));
    if (!ops->name || !ops->name[0] || ops->planes < 1 || ops->planes > MAX_PLANES || ops->states < 1 ||
        ops->states > 32 || !ops->simple || !ops->temporal || !ops->temporal_v || !ops->take_wait_timeouts ||
        !ops->prepare_batch || !ops->temporal_batch || !ops->batch_blocks_per_sm)
        return fail(CELLATO_EINVAL, "incomplete rule table");
    std::lock_guard<std::mutex> lock(g_register_mutex);
    const int n = rule_count();
    for (int r = 0; r < n; ++r) {
        if (g_rules[r] == ops) {
            *rule_out = r;
            return CELLATO_OK;
        }
        if (std::strcmp(g_rules[r]->name, ops->name) == 0 || std::strcmp(ops->name, "fire") == 0)
            return fail(CELLATO_EINVAL, "a rule named \"%s\" is already registered", ops->name);
    }
    if (n >= CELLATO_MAX_RULES) return fail(CELLATO_EINVAL, "the rule table is full (%d rules)", CELLATO_MAX_RULES);
    g_rules[n] = ops;
    g_rule_count.store(n + 1, std::memory_order_release);
    *rule_out = n;
    return CELLATO_OK;
}

const char* cellato_rule_name(int rule) {
    const rule_ops* o = ops_of(rule);
    return o ? o->name : nullptr;
}

int cellato_rule_planes(int rule) {
    const rule_ops* o = ops_of(rule);
    return o ? o->planes : -1;
}

int cellato_rule_states(int rule) {
    const rule_ops* o = ops_of(rule);
    return o ? o->states : -1;
}

size_t cellato_plane_bytes(int x_cells, int y_cells) {
    if (x_cells <= 0 || y_cells <= 0) return 0;
    return (size_t)x_cells * (size_t)y_cells / 8;
}

int cellato_check_dims(int layout, int word_bits, int x_cells, int y_cells) {
    return check_dims(layout, word_bits, x_cells, y_cells);
}

int cellato_planes_alloc(int nb, size_t bytes, void** planes_out) {
    if (nb < 1 || nb > MAX_PLANES || !planes_out) return fail(CELLATO_EINVAL, "bad plane count or output array");
    for (int p = 0; p < nb; ++p) planes_out[p] = nullptr;
    for (int p = 0; p < nb; ++p) {
        cudaError_t e = cudaMalloc(&planes_out[p], bytes ? bytes : 16);
        if (e != cudaSuccess) {
            for (int q = 0; q < p; ++q) {
                cudaFree(planes_out[q]);
                planes_out[q] = nullptr;
            }
            planes_out[p] = nullptr;
            return e == cudaErrorMemoryAllocation ? fail(CELLATO_ENOMEM, "cudaMalloc of %zu bytes failed", bytes)
                                                  : cuda_fail(e, "cudaMalloc");
        }
    }
    return CELLATO_OK;
}

int cellato_planes_free(int nb, void** planes) {
    if (nb < 1 || nb > MAX_PLANES || !planes) return fail(CELLATO_EINVAL, "bad plane count or array");
    int rc = CELLATO_OK;
    for (int p = 0; p < nb; ++p) {
        if (!planes[p]) continue;
        cudaError_t e = cudaFree(planes[p]);
        planes[p] = nullptr;
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaFree");
    }
    return rc;
}

int cellato_planes_upload(int nb, void* const* dev_planes, const void* const* host_planes, size_t bytes,
                          cellato_stream_t stream) {
    if (nb < 1 || nb > MAX_PLANES || !dev_planes || !host_planes) return fail(CELLATO_EINVAL, "bad arguments");
    for (int p = 0; p < nb; ++p) {
        if (!dev_planes[p] || !host_planes[p]) return fail(CELLATO_EINVAL, "plane %d pointer is NULL", p);
        cudaError_t e = cudaMemcpyAsync(dev_planes[p], host_planes[p], bytes, cudaMemcpyHostToDevice,
                                        reinterpret_cast<cudaStream_t>(stream));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync (upload)");
    }
    return CELLATO_OK;
}

int cellato_planes_download(int nb, void* const* host_planes, const void* const* dev_planes, size_t bytes,
                            cellato_stream_t stream) {
    if (nb < 1 || nb > MAX_PLANES || !dev_planes || !host_planes) return fail(CELLATO_EINVAL, "bad arguments");
    for (int p = 0; p < nb; ++p) {
        if (!dev_planes[p] || !host_planes[p]) return fail(CELLATO_EINVAL, "plane %d pointer is NULL", p);
        cudaError_t e = cudaMemcpyAsync(host_planes[p], dev_planes[p], bytes, cudaMemcpyDeviceToHost,
                                        reinterpret_cast<cudaStream_t>(stream));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync (download)");
    }
    return CELLATO_OK;
}

static int check_tune(const cellato_tune* t) {
    if (!t) return CELLATO_OK;
    if (t->simple_kernel < 0 || t->simple_kernel > 3)
        return fail(CELLATO_EINVAL, "tune.simple_kernel must be 0, 1, 2 or 3 (got %d)", t->simple_kernel);
    if (t->row_loop < 0 || t->row_loop > 3) return fail(CELLATO_EINVAL, "tune.row_loop must be 0 to 3 (got %d)", t->row_loop);
    if (t->words_per_lane < 0 || t->words_per_lane > 4 || t->words_per_lane == 3)
        return fail(CELLATO_EINVAL, "tune.words_per_lane must be 0, 1, 2 or 4 (got %d)", t->words_per_lane);
    if (t->tile_rows < 0) return fail(CELLATO_EINVAL, "tune.tile_rows must be >= 0 (got %d)", t->tile_rows);
    return CELLATO_OK;
}

int cellato_run_simple(int rule, int layout, int word_bits, void* const* planes_a, void* const* planes_b,
                       int x_cells, int y_cells, int t0, int steps, const cellato_tune* tune,
                       cellato_stream_t stream, int* result_in_b) {
    const rule_ops* ops = ops_of(rule);
    if (!ops) return fail(CELLATO_EINVAL, "unknown rule id %d", rule);
    if (steps < 0) return fail(CELLATO_EINVAL, "steps must be >= 0 (got %d)", steps);
    if (int rc = check_tune(tune)) return rc;
    if (int rc = check_dims(layout, word_bits, x_cells, y_cells)) return rc;
    plane_set a, b;
    if (int rc = make_sets(ops, planes_a, planes_b, a, b)) return rc;
    const int L = internal_layout(layout, word_bits);
    const int Xw = x_cells / 32;
    const int variant = tune ? tune->simple_kernel : SIMPLE_AUTO;
    const int wpl = tune ? tune->words_per_lane : 0;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    for (int i = 0; i < steps; ++i) {
        const plane_set& in = (i & 1) ? b : a;
        const plane_set& out = (i & 1) ? a : b;
        cudaError_t e = ops->simple(L, in, out, Xw, y_cells, t0 + i, variant, wpl, s);
        if (e != cudaSuccess) return cuda_fail(e, "simple step launch");
    }
    if (result_in_b) *result_in_b = steps & 1;
    return CELLATO_OK;
}

int cellato_device_wait_timeouts(unsigned* count) {
    if (!count) return fail(CELLATO_EINVAL, "count must not be NULL");
    *count = 0;
    const int n = rule_count();
    for (int r = 0; r < n; ++r) {
        unsigned c = 0;
        cudaError_t e = ops_of(r)->take_wait_timeouts(&c);
        if (e != cudaSuccess) return cuda_fail(e, "reading the device wait-timeout counter");
        *count += c;
    }
    return *count ? fail(CELLATO_ETIMEDOUT, "%u bounded device waits gave up", *count) : CELLATO_OK;
}

int cellato_temporal_max_tile_rows(int rule, int layout, int word_bits, int words_per_lane) {
    const rule_ops* ops = ops_of(rule);
    if (!ops) return -fail(CELLATO_EINVAL, "unknown rule id %d", rule);
    if (word_bits != 32 && word_bits != 64) return -fail(CELLATO_EINVAL, "word_bits must be 32 or 64");
    if (words_per_lane < 0 || words_per_lane > 2) return -fail(CELLATO_EINVAL, "words_per_lane must be 0, 1 or 2");
    const int R = band_height(layout, word_bits);
    const int row_bytes = ops->planes * 32 * ops->temporal_v(words_per_lane) * 4;
    const int q = std::max(ops->temporal_warps, R);
    return (max_optin_smem() / row_bytes) / q * q;
}

int cellato_run_temporal(int rule, int layout, int word_bits, void* const* planes_a, void* const* planes_b,
                         int x_cells, int y_cells, int t0, int steps, int k, const cellato_tune* tune,
                         cellato_stream_t stream, int* result_in_b) {
    const rule_ops* ops = ops_of(rule);
    if (!ops) return fail(CELLATO_EINVAL, "unknown rule id %d", rule);
    if (steps < 0) return fail(CELLATO_EINVAL, "steps must be >= 0 (got %d)", steps);
    if (k < 1 || k > 32) return fail(CELLATO_EINVAL, "temporal_steps must be in 1..32 (got %d)", k);
    if (int rc = check_tune(tune)) return rc;
    if (int rc = check_dims(layout, word_bits, x_cells, y_cells)) return rc;
    plane_set a, b;
    if (int rc = make_sets(ops, planes_a, planes_b, a, b)) return rc;
    const int L = internal_layout(layout, word_bits);
    const int R = band_height(layout, word_bits);
    const int q = std::max(ops->temporal_warps, R);
    const int V = ops->temporal_v(tune ? tune->words_per_lane : 0);
    const int loop = tune ? tune->row_loop : LOOP_AUTO;
    const int tile_rows = tune ? tune->tile_rows : 0;
    const int TH = tile_rows > 0 ? tile_rows : default_tile_rows(ops, R, k, V, ops->planes == 1 ? 128 : 224);
    if (TH % q != 0)
        return fail(CELLATO_EINVAL, "temporal tile rows %d must be a multiple of %d", TH, q);
    const int row_bytes = ops->planes * 32 * V * 4;
    if ((long long)TH * row_bytes > max_optin_smem())
        return fail(CELLATO_ESMEM, "Configuration exceeds maximum shared memory size. The temporal tile is too large.");
    const int Xw = x_cells / 32;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int launches = 0;
    for (int done = 0; done < steps;) {
        const int kk = std::min(k, steps - done);
        const int HY = (kk + R - 1) / R * R;
        if (TH - 2 * HY <= 0)
            return fail(CELLATO_EINVAL, "temporal tile of %d rows leaves no interior for %d steps", TH, kk);
        const plane_set& in = (launches & 1) ? b : a;
        const plane_set& out = (launches & 1) ? a : b;
        cudaError_t e = ops->temporal(L, in, out, Xw, y_cells, t0 + done, kk, TH, HY, loop, V, s);
        if (e != cudaSuccess) return cuda_fail(e, "temporal launch");
        done += kk;
        ++launches;
    }
    if (result_in_b) *result_in_b = launches & 1;
    return CELLATO_OK;
}

}  // extern "C"
