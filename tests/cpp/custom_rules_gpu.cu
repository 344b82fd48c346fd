// Test library: the custom rules of custom_rules.hpp instantiated outside the
// B200 library, through the public header-only path (b200/custom_rule.cuh).
// Only the package's public headers are used; nothing of csrc/.  The tests
// load this library, hand its tables to cellato_rule_register and run the
// rules through the C ABI.
#include "b200/custom_rule.cuh"
#include "custom_rules.hpp"

extern "C" {

// Kernel table of custom rule `which` (0 highlife, 1 star-wars, 2
// parity-shift), or NULL.
const cellato_rule_ops* custom_rule_table(int which) {
    switch (which) {
        case 0: return cellato::b200::rule_table<highlife::config>();
        case 1: return cellato::b200::rule_table<star_wars::config>();
        case 2: return cellato::b200::rule_table<parity_shift::config>();
        default: return nullptr;
    }
}

int custom_rule_count(void) { return 3; }

// A bounded device-side wait that runs out, without a device fault: one
// persistent batch launch (highlife, linear layout) whose only item is round 1
// of a 64 x 32 grid whose round 0 is not in the list, so the grid's count of
// finished tiles never reaches the one tile the item waits for.  The wait gives
// up after wait_limit polls, counts itself in this translation unit's timeout
// counter and runs the item anyway, and the launch returns.  *timeouts receives
// the count; returns a cudaError_t.
int custom_batch_wait_probe(unsigned wait_limit, unsigned* timeouts) {
    namespace cb = cellato::b200;
    using K = cb::rule_kernels<highlife::config>;
    constexpr int Xw = 2, Y = 32, HY = 1, TH = 2 * HY + Y;  // one tile covers the grid
    unsigned cleared = 0;
    cudaError_t e = K::take_wait_timeouts(&cleared);
    cb::word* planes = nullptr;
    unsigned char* misc = nullptr;  // [descriptor | item | head, done]
    if (e == cudaSuccess) e = cudaMalloc(&planes, 2 * Xw * Y * sizeof(cb::word));
    if (e == cudaSuccess) e = cudaMemset(planes, 0, 2 * Xw * Y * sizeof(cb::word));
    if (e == cudaSuccess) e = cudaMalloc(&misc, 512);
    if (e == cudaSuccess) e = cudaMemset(misc, 0, 512);
    cb::batch_grid_desc desc{};
    desc.p[0].p[0] = planes;
    desc.p[1].p[0] = planes + Xw * Y;
    desc.Xw = Xw, desc.Y = Y, desc.tiles = 1;
    const cb::batch_item item{0, 0, 0, (1 << cb::BATCH_ROUND_SHIFT) | 1};  // round 1, one step
    static_assert(sizeof(cb::batch_grid_desc) <= 256 && sizeof(cb::batch_item) <= 64, "probe layout");
    if (e == cudaSuccess) e = cudaMemcpy(misc, &desc, sizeof desc, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(misc + 256, &item, sizeof item, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        auto* sync = reinterpret_cast<unsigned*>(misc + 320);
        const size_t smem = (size_t)K::NB * TH * 32 * sizeof(cb::word);
        cb::temporal_batch_kernel<K::net, K::NB, cb::LAYOUT_LINEAR, 1, K::TEMPORAL_WARPS, true>
            <<<1, K::TEMPORAL_WARPS * 32, smem>>>(reinterpret_cast<const cb::batch_grid_desc*>(misc),
                                                  reinterpret_cast<const cb::batch_item*>(misc + 256), 1, 0, 0, TH,
                                                  HY, sync, sync + 1, wait_limit);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = K::take_wait_timeouts(timeouts);
    cudaFree(planes);
    cudaFree(misc);
    return (int)e;
}

}  // extern "C"
