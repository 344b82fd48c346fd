// GPU packing between one-byte-per-cell grids and bit planes.
//
// Replaces the host loops of the reference grid classes: bit_planes::grid
// construction (include/memory/bit_planes_grid.hpp:234-270) and get_cell /
// to_original_representation (:97-124), and their tiled counterparts
// (include/memory/tiled_bit_planes_grid.hpp:243-288, :100-139).  Cells are
// uint8 state-dictionary indices, row-major X x Y.
//
// One warp per (band, linear word): lane i handles cell 32*gx + i of each row
// of the band.  Packing turns each plane bit into a word with one warp ballot;
// unpacking broadcasts each plane word with a shuffle and keeps the lane's bit.
// Tiled layouts reuse the engine's 4x4 byte transpose at the store / load.
#include <cuda_runtime.h>

#include <cstdint>

#include "cellato_b200.h"
#include "b200/engine.cuh"

using namespace cellato::b200;

namespace {

constexpr int PACK_WARPS = 8;

template <int LAYOUT, int NB>
__global__ void __launch_bounds__(PACK_WARPS * 32) pack_kernel(const uint8_t* __restrict__ cells, int X, int Xw,
                                                               int nbands, plane_set out) {
    constexpr int R = band_rows<LAYOUT>();
    const int lane = threadIdx.x & 31;
    const long long w = (long long)blockIdx.x * PACK_WARPS + (threadIdx.x >> 5);
    if (w >= (long long)nbands * Xw) return;  // whole warp exits together
    const int b = (int)(w / Xw), gx = (int)(w % Xw);
    word bits[R][NB];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint8_t c = cells[(size_t)(b * R + r) * X + 32 * gx + lane];
#pragma unroll
        for (int p = 0; p < NB; ++p) bits[r][p] = __ballot_sync(0xffffffffu, (c >> p) & 1);
    }
    // lane p stores plane p
    if (lane < NB) {
        word rows[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            word v = 0;
#pragma unroll
            for (int p = 0; p < NB; ++p) v = (p == lane) ? bits[r][p] : v;
            rows[r] = v;
        }
        store_word_rows<LAYOUT>(out.p[lane], Xw, b, gx, rows);
    }
}

template <int LAYOUT, int NB>
__global__ void __launch_bounds__(PACK_WARPS * 32) unpack_kernel(plane_set in, int X, int Xw, int nbands,
                                                                 uint8_t* __restrict__ cells) {
    constexpr int R = band_rows<LAYOUT>();
    const int lane = threadIdx.x & 31;
    const long long w = (long long)blockIdx.x * PACK_WARPS + (threadIdx.x >> 5);
    if (w >= (long long)nbands * Xw) return;
    const int b = (int)(w / Xw), gx = (int)(w % Xw);
    word mine[R];
#pragma unroll
    for (int r = 0; r < R; ++r) mine[r] = 0;
    if (lane < NB) load_word_rows<LAYOUT>(in.p[lane], Xw, b, gx, mine);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        uint32_t v = 0;
#pragma unroll
        for (int p = 0; p < NB; ++p) {
            const word pw = __shfl_sync(0xffffffffu, mine[r], p);
            v |= ((pw >> lane) & 1u) << p;
        }
        cells[(size_t)(b * R + r) * X + 32 * gx + lane] = (uint8_t)v;
    }
}

int check(int layout, int word_bits, int nb, int X, int Y, const void* cells, const void* const* planes,
          plane_set& ps) {
    if (nb < 1 || nb > MAX_PLANES || !cells || !planes) return CELLATO_EINVAL;
    int rc = cellato_check_dims(layout, word_bits, X, Y);
    if (rc != CELLATO_OK) return rc;
    for (int p = 0; p < MAX_PLANES; ++p) ps.p[p] = nullptr;
    for (int p = 0; p < nb; ++p) {
        if (!planes[p] || (reinterpret_cast<uintptr_t>(planes[p]) & 15)) return CELLATO_EINVAL;
        ps.p[p] = static_cast<word*>(const_cast<void*>(planes[p]));
    }
    return CELLATO_OK;
}

}  // namespace

extern "C" {

int cellato_pack_cells(int layout, int word_bits, int nb, const uint8_t* cells, int x_cells, int y_cells,
                       void* const* planes, cellato_stream_t stream) {
    plane_set ps;
    if (int rc = check(layout, word_bits, nb, x_cells, y_cells, cells, planes, ps)) return rc;
    const int Xw = x_cells / 32;
    const int R = layout == CELLATO_LAYOUT_BIT_PLANES ? 1 : word_bits / 8;
    const int nbands = y_cells / R;
    const long long warps = (long long)nbands * Xw;
    const dim3 grid((unsigned)((warps + PACK_WARPS - 1) / PACK_WARPS)), block(PACK_WARPS * 32);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    dispatch_planes(nb, [&](auto c) {
        constexpr int NB = decltype(c)::value;
        if (R == 1)
            pack_kernel<LAYOUT_LINEAR, NB><<<grid, block, 0, s>>>(cells, x_cells, Xw, nbands, ps);
        else if (R == 4)
            pack_kernel<LAYOUT_TILED4, NB><<<grid, block, 0, s>>>(cells, x_cells, Xw, nbands, ps);
        else
            pack_kernel<LAYOUT_TILED8, NB><<<grid, block, 0, s>>>(cells, x_cells, Xw, nbands, ps);
    });
    return cudaGetLastError() == cudaSuccess ? CELLATO_OK : CELLATO_ECUDA;
}

int cellato_unpack_cells(int layout, int word_bits, int nb, const void* const* planes, int x_cells, int y_cells,
                         uint8_t* cells, cellato_stream_t stream) {
    plane_set ps;
    if (int rc = check(layout, word_bits, nb, x_cells, y_cells, cells, planes, ps)) return rc;
    const int Xw = x_cells / 32;
    const int R = layout == CELLATO_LAYOUT_BIT_PLANES ? 1 : word_bits / 8;
    const int nbands = y_cells / R;
    const long long warps = (long long)nbands * Xw;
    const dim3 grid((unsigned)((warps + PACK_WARPS - 1) / PACK_WARPS)), block(PACK_WARPS * 32);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    dispatch_planes(nb, [&](auto c) {
        constexpr int NB = decltype(c)::value;
        if (R == 1)
            unpack_kernel<LAYOUT_LINEAR, NB><<<grid, block, 0, s>>>(ps, x_cells, Xw, nbands, cells);
        else if (R == 4)
            unpack_kernel<LAYOUT_TILED4, NB><<<grid, block, 0, s>>>(ps, x_cells, Xw, nbands, cells);
        else
            unpack_kernel<LAYOUT_TILED8, NB><<<grid, block, 0, s>>>(ps, x_cells, Xw, nbands, cells);
    });
    return cudaGetLastError() == cudaSuccess ? CELLATO_OK : CELLATO_ECUDA;
}

}  // extern "C"
