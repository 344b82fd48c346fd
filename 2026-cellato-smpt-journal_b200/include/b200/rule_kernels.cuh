// Per-rule launchers: instantiate the engine kernels for one automaton config
// and expose them through a rule_ops table.  This is the B200 counterpart of
// the reference's explicit instantiations
// (src/_shared/cuda_instantiation_template.cuh:77-193): the rule stays a C++
// type and is lowered at compile time; the C ABI selects it by rule id.
//
// The ten automata of the reference are instantiated inside the library (one
// .cu file per rule, so they compile in parallel).  Any other rule written in
// the same DSL is instantiated by the caller's own translation unit, compiled
// with nvcc for sm_100a: cellato::b200::custom_rule_ops<Config>() builds its
// table there and cellato_rule_register hands it to the library, which then
// runs it under a new rule id through every entry point (b200/custom_rule.cuh).
//
// Nothing here holds mutable state: which kernel variant, row loop and tile
// width a launch uses are arguments of each call (cellato_tune in the C ABI).
#ifndef CELLATO_B200_RULE_KERNELS_CUH
#define CELLATO_B200_RULE_KERNELS_CUH

#include <cuda_runtime.h>

#include <algorithm>

#include "b200/engine.cuh"
#include "b200/tma_step.cuh"

// Version of the rule_ops layout; cellato_rule_register refuses a table built
// against another version.
#define CELLATO_RULE_OPS_ABI 4

namespace cellato::b200 {
// Single-step kernel choices (cellato_tune::simple_kernel).
enum : int { SIMPLE_AUTO = 0, SIMPLE_REGISTER = 1, SIMPLE_STREAM = 2, SIMPLE_TMA = 3 };
// Temporal row loops (cellato_tune::row_loop).
enum : int { LOOP_AUTO = 0, LOOP_ROW_BY_ROW = 1, LOOP_HOISTED = 2, LOOP_PAIRED = 3 };
}  // namespace cellato::b200

// The kernels of one rule, as function pointers into the translation unit that
// instantiated them.  Plain data, built once per rule and never modified.
struct cellato_rule_ops_st {
    int abi_version;  // CELLATO_RULE_OPS_ABI
    int struct_size;  // sizeof(cellato_rule_ops_st)
    const char* name;
    int planes;  // needed_bits
    int states;  // number_of_values
    // one time step t (its parity selects the instantiation) with single-step kernel `variant`;
    // words_per_lane: the TMA kernel's words per lane (0: its default)
    cudaError_t (*simple)(int layout, const cellato::b200::plane_set& in, const cellato::b200::plane_set& out, int Xw,
                          int Y, int t, int variant, int words_per_lane, cudaStream_t s);
    // k fused steps from t0 on a TH-row tile with an HY-row halo, row loop `loop`,
    // V words per lane (a value temporal_v returned)
    cudaError_t (*temporal)(int layout, const cellato::b200::plane_set& in, const cellato::b200::plane_set& out,
                            int Xw, int Y, int t0, int k, int TH, int HY, int loop, int V, cudaStream_t s);
    // words per lane the temporal kernel runs for a requested width (0 = the rule's default)
    int (*temporal_v)(int words_per_lane);
    int batch_words_per_lane;  // V of the batched temporal kernel
    int temporal_warps;
    // reads and clears the count of bounded waits that gave up (device-side)
    cudaError_t (*take_wait_timeouts)(unsigned* count);
    // batched temporal kernel (see temporal_batch_kernel); prepare_batch sets
    // the kernel's shared-memory limit (call outside capture)
    cudaError_t (*prepare_batch)(int layout, int TH);
    // one persistent launch over a work list of every round (queue head and
    // per-grid finished-tile counts zeroed by the caller, stream-ordered)
    cudaError_t (*temporal_batch)(int layout, const cellato::b200::batch_grid_desc* grids,
                                  const cellato::b200::batch_item* items, int n_items, int parity, int t0, int TH,
                                  int HY, unsigned* head, unsigned* done, int ctas, cudaStream_t s);
    // resident CTAs per SM of the batched kernel with a TH-row tile (after prepare_batch)
    int (*batch_blocks_per_sm)(int layout, int TH);
    // state value of each dictionary index (index_to_state), 0 past `states`
    long long state_values[32];
};

namespace cellato::b200 {

using rule_ops = ::cellato_rule_ops_st;

// Words per lane of the single-step kernel: as wide as registers allow.  A row
// of features costs about 3 words per plane plus 5 per count target per lane
// word, and three rows plus three bands of raw words are live.
template <class Net, int NB, int LAYOUT>
constexpr int simple_words_per_lane() {
    constexpr int BR = simple_band_rows<LAYOUT>();
    constexpr int feat_words = 3 * NB + 5 * Net::targets::size;
    constexpr int per_v = 3 * feat_words + 2 * BR * NB + (LAYOUT == LAYOUT_LINEAR ? 0 : BR * NB);
    return per_v * 4 <= 160 ? 4 : (per_v * 2 <= 160 ? 2 : 1);
}

template <class A>
struct rule_kernels {
    using dict = typename A::state_dictionary;
    using net = rule_net<dict, typename A::algorithm>;
    static constexpr int NB = dict::needed_bits;
    static_assert(NB <= MAX_PLANES, "too many planes");
    static constexpr int SIMPLE_WARPS = 4;
    static constexpr int TEMPORAL_V = NB <= 3 ? 2 : 1;
    // The batched kernel runs one word per lane for rules of two or more
    // planes: its tiles are 32 words wide, which wastes less on the narrow
    // grids of a batch, and its register use leaves room for three CTAs per
    // SM.  One-plane rules take two words per lane: with one word a lane has
    // too little independent work (Game of Life, maze and critters ran at
    // 0.31-0.48 of their single-grid rate in a 1024-grid batch on B200).
    static constexpr int BATCH_V = NB == 1 ? 2 : 1;
    // ... and two steps per sweep of a tile (row loop 3) for rules of up to
    // three planes; with four or five planes the second step's features cost
    // registers that leave one or two CTAs per SM (cyclic: 177 registers, one
    // CTA per SM, 12.5% warps active in a 1024-grid batch on B200)
    static constexpr bool BATCH_PAIR = NB <= 3;
    static constexpr int TEMPORAL_WARPS = 8;

    template <int LAYOUT, int V>
    static cudaError_t simple_v(const plane_set& in, const plane_set& out, int Xw, int Y, int t, cudaStream_t s) {
        constexpr int BR = simple_band_rows<LAYOUT>();
        const int nbands = (Y + BR - 1) / BR;
        const int segments = (Xw + 32 * V - 1) / (32 * V);
        const int cta_x = (segments + SIMPLE_WARPS - 1) / SIMPLE_WARPS;
        // enough warps to cover 148 SMs x 32 resident warps, at most 64 rows per CTA
        const long long want = 148LL * 32;
        const int bands = (int)std::max(1LL, std::min<long long>(std::max(1, 64 / BR), (long long)segments * nbands / want));
        const int cta_y = (nbands + bands - 1) / bands;
        const dim3 grid(cta_x, cta_y), block(SIMPLE_WARPS * 32);
        if (t & 1)
            simple_step_kernel<net, NB, LAYOUT, V, 1, SIMPLE_WARPS><<<grid, block, 0, s>>>(in, out, Xw, Y, nbands, bands);
        else
            simple_step_kernel<net, NB, LAYOUT, V, 0, SIMPLE_WARPS><<<grid, block, 0, s>>>(in, out, Xw, Y, nbands, bands);
        return cudaGetLastError();
    }

    // linear layout, 16-byte rows: the bulk-copy streaming kernel
    static constexpr int STREAM_V = NB <= 2 ? 4 : 2;
    static constexpr int STREAM_WARPS = 4;
    static cudaError_t simple_stream(const plane_set& in, const plane_set& out, int Xw, int Y, int t,
                                     cudaStream_t s) {
        constexpr int V = STREAM_V;
        const int segments = (Xw + 32 * V - 1) / (32 * V);
        const int cta_x = (segments + STREAM_WARPS - 1) / STREAM_WARPS;
        const long long want = 148LL * 32;
        const int rows = (int)std::max(16LL, std::min<long long>(512, (long long)segments * Y / want));
        const dim3 grid(cta_x, (Y + rows - 1) / rows), block(STREAM_WARPS * 32);
        const size_t smem = (size_t)STREAM_WARPS * stream_smem_per_warp<NB, V>();
        auto k0 = stream_step_kernel<net, NB, V, 0, STREAM_WARPS>;
        auto k1 = stream_step_kernel<net, NB, V, 1, STREAM_WARPS>;
        auto kern = (t & 1) ? k1 : k0;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, block, smem, s>>>(in, out, Xw, Y, rows);
        return cudaGetLastError();
    }

    // the TMA-fed single-step kernel (rows of a multiple of its strip width);
    // V words per lane: the default, or 1, 2 (rules of up to three planes) or 4
    // (one-plane rules, the 4- and 1-row layouts) when asked for
    template <int LAYOUT>
    static constexpr int TMA_V = tma_default_v<NB, LAYOUT>();
    template <int LAYOUT>
    static constexpr int TMA_VMAX = NB == 1 && LAYOUT != LAYOUT_TILED8 ? 4 : (NB <= 3 ? 2 : 1);
    template <int LAYOUT, int V>
    static bool tma_fits(int Xw, int Y) {
        using G = tma_geom<NB, LAYOUT, V>;
        return Xw % G::SW == 0 && Y / band_rows<LAYOUT>() >= G::BR;
    }
    template <int LAYOUT, int V>
    static cudaError_t simple_tma(const plane_set& in, const plane_set& out, int Xw, int Y, int t, cudaStream_t s) {
        using SM = tma_geom<NB, LAYOUT, V>;
        const int M = Y / band_rows<LAYOUT>();
        tma_maps maps;
        cudaError_t e = make_tma_maps<NB, LAYOUT, V>(in, Xw, M, maps);
        if (e != cudaSuccess) return e;
        auto kern = (t & 1) ? tma_step_kernel<net, NB, LAYOUT, V, 1> : tma_step_kernel<net, NB, LAYOUT, V, 0>;
        if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM::bytes)) !=
            cudaSuccess)
            return e;
        static int sms = 0, per_sm = 0;  // per instantiation; constant for the process's device
        if (!sms) {
            int dev = 0, n = 0, b = 0;
            if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
                (e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
                (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, SM::threads, SM::bytes)) != cudaSuccess)
                return e;
            per_sm = std::max(1, b);
            sms = n;
        }
        // one wave of resident CTAs with equal ranges (a multiple of a stage)
        const int strips = Xw / SM::SW;
        const long long target = (long long)per_sm * sms;
        int rows = (int)std::max<long long>(1, ((long long)M * strips + target - 1) / target);
        rows = (rows + SM::BR - 1) / SM::BR * SM::BR;
        const dim3 grid(strips, (M + rows - 1) / rows);
        kern<<<grid, SM::threads, SM::bytes, s>>>(maps, in, out, Xw, M, rows);
        return cudaGetLastError();
    }

    static cudaError_t take_wait_timeouts(unsigned* count) {
        unsigned zero = 0;
        cudaError_t e = cudaMemcpyFromSymbol(count, g_wait_timeouts, sizeof(unsigned));
        if (e != cudaSuccess) return e;
        return cudaMemcpyToSymbol(g_wait_timeouts, &zero, sizeof(unsigned));
    }

    template <int LAYOUT>
    static cudaError_t simple_layout(const plane_set& in, const plane_set& out, int Xw, int Y, int t, int variant,
                                     int words_per_lane, cudaStream_t s) {
        if (variant == SIMPLE_TMA) {
            const int v = words_per_lane ? words_per_lane : TMA_V<LAYOUT>;
            if (v == 1 && tma_fits<LAYOUT, 1>(Xw, Y)) return simple_tma<LAYOUT, 1>(in, out, Xw, Y, t, s);
            if constexpr (TMA_VMAX<LAYOUT> >= 2)
                if (v == 2 && tma_fits<LAYOUT, 2>(Xw, Y)) return simple_tma<LAYOUT, 2>(in, out, Xw, Y, t, s);
            if constexpr (TMA_VMAX<LAYOUT> >= 4)
                if (v == 4 && tma_fits<LAYOUT, 4>(Xw, Y)) return simple_tma<LAYOUT, 4>(in, out, Xw, Y, t, s);
        }
        if constexpr (LAYOUT == LAYOUT_LINEAR) {
            const bool stream_ok = Xw % 4 == 0;
            // default: streaming for rules with two or more planes, whose
            // register bands would otherwise cap occupancy
            const bool use_stream =
                stream_ok && (variant == SIMPLE_STREAM || (variant == SIMPLE_AUTO && NB >= 2));
            if (use_stream) return simple_stream(in, out, Xw, Y, t, s);
        }
        constexpr int VMAX = simple_words_per_lane<net, NB, LAYOUT>();
        if constexpr (VMAX >= 4)
            if (Xw % 4 == 0) return simple_v<LAYOUT, 4>(in, out, Xw, Y, t, s);
        if constexpr (VMAX >= 2)
            if (Xw % 2 == 0) return simple_v<LAYOUT, 2>(in, out, Xw, Y, t, s);
        return simple_v<LAYOUT, 1>(in, out, Xw, Y, t, s);
    }

    static cudaError_t simple(int layout, const plane_set& in, const plane_set& out, int Xw, int Y, int t,
                              int variant, int words_per_lane, cudaStream_t s) {
        switch (layout) {
            case LAYOUT_LINEAR: return simple_layout<LAYOUT_LINEAR>(in, out, Xw, Y, t, variant, words_per_lane, s);
            case LAYOUT_TILED4: return simple_layout<LAYOUT_TILED4>(in, out, Xw, Y, t, variant, words_per_lane, s);
            case LAYOUT_TILED8: return simple_layout<LAYOUT_TILED8>(in, out, Xw, Y, t, variant, words_per_lane, s);
        }
        return cudaErrorInvalidValue;
    }

    // width 0 (the default): two words per lane for one-plane rules, one for the
    // others (the narrower tile lets three CTAs of 200-256 rows share an SM;
    // with those heights, on B200 at 16384^2 and k = 16, 3-13% faster than two
    // words per lane and 128 interior rows for the rules of two to five planes)
    static int temporal_v(int words_per_lane) {
        if (TEMPORAL_V == 1 || words_per_lane == 1) return 1;
        return (words_per_lane == 2 || NB == 1) ? 2 : 1;
    }

    template <int LAYOUT, int V>
    static cudaError_t temporal_launch(const plane_set& in, const plane_set& out, int Xw, int Y, int t0, int k,
                                       int TH, int HY, int loop, cudaStream_t s) {
        auto kern = loop == LOOP_ROW_BY_ROW ? temporal_kernel<net, NB, LAYOUT, V, TEMPORAL_WARPS, false>
                    : loop == LOOP_PAIRED   ? temporal_kernel<net, NB, LAYOUT, V, TEMPORAL_WARPS, true, true>
                                            : temporal_kernel<net, NB, LAYOUT, V, TEMPORAL_WARPS, true>;
        const size_t smem = (size_t)NB * TH * 32 * V * sizeof(word);
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        const int effW = 32 * V - 2, effH = TH - 2 * HY;
        const dim3 grid((Xw + effW - 1) / effW, (Y + effH - 1) / effH), block(TEMPORAL_WARPS * 32);
        kern<<<grid, block, smem, s>>>(in, out, Xw, Y, t0, k, TH, HY);
        return cudaGetLastError();
    }

    template <int LAYOUT>
    static cudaError_t temporal_layout(const plane_set& in, const plane_set& out, int Xw, int Y, int t0, int k,
                                       int TH, int HY, int loop, int V, cudaStream_t s) {
        if constexpr (TEMPORAL_V == 2) {
            if (V == 2) return temporal_launch<LAYOUT, 2>(in, out, Xw, Y, t0, k, TH, HY, loop, s);
        }
        return temporal_launch<LAYOUT, 1>(in, out, Xw, Y, t0, k, TH, HY, loop, s);
    }

    static cudaError_t temporal(int layout, const plane_set& in, const plane_set& out, int Xw, int Y, int t0, int k,
                                int TH, int HY, int loop, int V, cudaStream_t s) {
        switch (layout) {
            case LAYOUT_LINEAR: return temporal_layout<LAYOUT_LINEAR>(in, out, Xw, Y, t0, k, TH, HY, loop, V, s);
            case LAYOUT_TILED4: return temporal_layout<LAYOUT_TILED4>(in, out, Xw, Y, t0, k, TH, HY, loop, V, s);
            case LAYOUT_TILED8: return temporal_layout<LAYOUT_TILED8>(in, out, Xw, Y, t0, k, TH, HY, loop, V, s);
        }
        return cudaErrorInvalidValue;
    }

    template <int LAYOUT>
    static auto batch_kernel() {
        return temporal_batch_kernel<net, NB, LAYOUT, BATCH_V, TEMPORAL_WARPS, BATCH_PAIR>;
    }
    static size_t tile_smem(int TH) { return (size_t)NB * TH * 32 * BATCH_V * sizeof(word); }

    static cudaError_t prepare_batch(int layout, int TH) {
        const int smem = (int)tile_smem(TH);
        switch (layout) {
            case LAYOUT_LINEAR:
                return cudaFuncSetAttribute(batch_kernel<LAYOUT_LINEAR>(), cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            case LAYOUT_TILED4:
                return cudaFuncSetAttribute(batch_kernel<LAYOUT_TILED4>(), cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            case LAYOUT_TILED8:
                return cudaFuncSetAttribute(batch_kernel<LAYOUT_TILED8>(), cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        }
        return cudaErrorInvalidValue;
    }

    static int batch_blocks_per_sm(int layout, int TH) {
        int n = 0;
        const size_t smem = tile_smem(TH);
        const int threads = TEMPORAL_WARPS * 32;
        cudaError_t e = cudaErrorInvalidValue;
        switch (layout) {
            case LAYOUT_LINEAR:
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<LAYOUT_LINEAR>(), threads, smem);
                break;
            case LAYOUT_TILED4:
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<LAYOUT_TILED4>(), threads, smem);
                break;
            case LAYOUT_TILED8:
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<LAYOUT_TILED8>(), threads, smem);
                break;
        }
        return (e == cudaSuccess && n > 0) ? n : 1;
    }

    static cudaError_t temporal_batch(int layout, const batch_grid_desc* grids, const batch_item* items, int n_items,
                                      int parity, int t0, int TH, int HY, unsigned* head, unsigned* done, int ctas,
                                      cudaStream_t s) {
        const size_t smem = tile_smem(TH);
        const dim3 block(TEMPORAL_WARPS * 32), grid(ctas);
        switch (layout) {
            case LAYOUT_LINEAR:
                batch_kernel<LAYOUT_LINEAR>()<<<grid, block, smem, s>>>(grids, items, n_items, parity, t0, TH, HY,
                                                                        head, done, BATCH_WAIT_LIMIT);
                break;
            case LAYOUT_TILED4:
                batch_kernel<LAYOUT_TILED4>()<<<grid, block, smem, s>>>(grids, items, n_items, parity, t0, TH, HY,
                                                                        head, done, BATCH_WAIT_LIMIT);
                break;
            case LAYOUT_TILED8:
                batch_kernel<LAYOUT_TILED8>()<<<grid, block, smem, s>>>(grids, items, n_items, parity, t0, TH, HY,
                                                                        head, done, BATCH_WAIT_LIMIT);
                break;
            default:
                return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }

    static rule_ops ops() {
        rule_ops o{CELLATO_RULE_OPS_ABI, (int)sizeof(rule_ops), A::name, NB, dict::number_of_values, &simple,
                   &temporal, &temporal_v, BATCH_V, TEMPORAL_WARPS, &take_wait_timeouts, &prepare_batch,
                   &temporal_batch, &batch_blocks_per_sm, {}};
        static_assert(dict::number_of_values <= 32, "state table holds 32 values");
        for (int i = 0; i < dict::number_of_values; ++i)
            o.state_values[i] = static_cast<long long>(dict::index_to_state(i));
        return o;
    }
};

// The kernel table of a rule config (members name, state_dictionary,
// algorithm, as the reference's src/<automaton>/config.hpp), instantiated in
// the calling translation unit; the table lives until the process exits.
template <class Config>
const rule_ops* custom_rule_ops() {
    static const rule_ops o = rule_kernels<Config>::ops();
    return &o;
}

}  // namespace cellato::b200

#define CELLATO_DEFINE_RULE_OPS(ID, CONFIG)                        \
    namespace cellato::b200 {                                      \
    extern const rule_ops rule_ops_##ID;                           \
    const rule_ops rule_ops_##ID = rule_kernels<CONFIG>::ops();    \
    }

#endif  // CELLATO_B200_RULE_KERNELS_CUH
