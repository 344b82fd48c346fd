// Conversion between the reference's bit_array layout and bit planes, on the
// device (C ABI cellato_bit_array_to_planes / cellato_planes_to_bit_array).
//
// The bit_array layout (include/memory/bit_array_grid.hpp:298-320) packs a
// cell's nb index bits next to each other: cells in row-major order,
// cpw = W / nb cells per W-bit word, cell i in word i / cpw at bit
// (i % cpw) * nb (the top W - cpw*nb bits of a word stay 0); x_size must be a
// multiple of cpw, so every row starts on a word.  The reference evaluates it
// cell by cell inside each word (include/evaluators/bit_array.hpp:73-105).
// Here a bit_array grid is converted to planes once when a run starts and back
// once when it ends, and the steps run on the bit-plane kernels: the result is
// the same automaton's, and the per-step cost is the planes'.
//
//   to planes:  one warp per (band, plane word): lane l gathers cell 32*gx + l
//               of each row of the band from its bit_array word, and one
//               ballot per plane and row forms the plane words (the packing
//               kernel's structure);
//   to array:   one thread per bit_array word: it gathers its cpw cells' bits
//               from the planes.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "capi_internal.hpp"
#include "cellato_b200.h"
#include "b200/engine.cuh"

using namespace cellato::b200;
using namespace cellato::b200::capi;

namespace {

constexpr int BA_WARPS = 8;

template <int LAYOUT, typename AW, int NB>
__global__ void __launch_bounds__(BA_WARPS * 32) bit_array_to_planes_kernel(const AW* __restrict__ arr, int X,
                                                                            int Xw, int nbands, int cpw,
                                                                            plane_set out) {
    constexpr int R = band_rows<LAYOUT>();
    const int lane = threadIdx.x & 31;
    const long long w = (long long)blockIdx.x * BA_WARPS + (threadIdx.x >> 5);
    if (w >= (long long)nbands * Xw) return;  // whole warp exits together
    const int b = (int)(w / Xw), gx = (int)(w % Xw);
    const long long row_words = X / cpw;
    const AW mask = (AW(1) << NB) - 1;
    const int x = 32 * gx + lane;
    const int wi = x / cpw, off = (x % cpw) * NB;
    word bits[R][NB];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const long long y = (long long)b * R + r;
        const int idx = (int)((arr[y * row_words + wi] >> off) & mask);
#pragma unroll
        for (int p = 0; p < NB; ++p) bits[r][p] = __ballot_sync(0xffffffffu, (idx >> p) & 1);
    }
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

// Byte of a plane holding cell (x, y), whose bit is x % 8 (all layouts are
// little-endian and LSB-first within a byte).
template <int LAYOUT>
__device__ __forceinline__ size_t cell_byte(int X, int x, int y) {
    if constexpr (LAYOUT == LAYOUT_LINEAR) {
        return ((size_t)y * X + x) >> 3;
    } else {
        constexpr int R = band_rows<LAYOUT>();  // tile rows; a tile is R bytes
        return ((size_t)(y / R) * (X / 8) + x / 8) * R + (y % R);
    }
}

template <int LAYOUT, typename AW>
__global__ void __launch_bounds__(256) planes_to_bit_array_kernel(plane_set in, int X, int Y, int nb, int cpw,
                                                                  AW* __restrict__ arr) {
    const long long row_words = X / cpw;
    const long long n = row_words * Y;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int y = (int)(i / row_words), x0 = (int)(i % row_words) * cpw;
    AW v = 0;
    for (int c = 0; c < cpw; ++c) {
        const int x = x0 + c;
        const size_t byte = cell_byte<LAYOUT>(X, x, y);
        unsigned idx = 0;
        for (int p = 0; p < nb; ++p)
            idx |= ((reinterpret_cast<const unsigned char*>(in.p[p])[byte] >> (x & 7)) & 1u) << p;
        v |= AW(idx) << (c * nb);
    }
    arr[i] = v;
}

int planes_of(int nb, void* const* planes, plane_set& ps) {
    if (!planes) return fail(CELLATO_EINVAL, "plane array must not be NULL");
    std::memset(&ps, 0, sizeof ps);
    for (int p = 0; p < nb; ++p) {
        if (!planes[p]) return fail(CELLATO_EINVAL, "plane %d pointer is NULL", p);
        if (reinterpret_cast<uintptr_t>(planes[p]) & 15)
            return fail(CELLATO_EINVAL, "plane %d pointer is not 16-byte aligned", p);
        ps.p[p] = static_cast<word*>(planes[p]);
    }
    return CELLATO_OK;
}

int check_array(int nb, int array_word_bits, int X, int Y, const void* array) {
    if (nb < 1 || nb > MAX_PLANES) return fail(CELLATO_EINVAL, "plane count %d out of range 1..%d", nb, MAX_PLANES);
    if (array_word_bits != 32 && array_word_bits != 64)
        return fail(CELLATO_EINVAL, "bit_array word size must be 32 or 64 (got %d)", array_word_bits);
    if (!array) return fail(CELLATO_EINVAL, "bit_array pointer must not be NULL");
    if (reinterpret_cast<uintptr_t>(array) & (array_word_bits / 8 - 1))
        return fail(CELLATO_EINVAL, "bit_array pointer is not aligned to its words");
    const int cpw = array_word_bits / nb;
    if (X % cpw != 0)
        return fail(CELLATO_EINVAL_DIMS,
                    "Grid x_size must be divisible by cells_per_word. x_size=%d, cells_per_word=%d (bits [%d] / "
                    "bits_per_cell [%d])",
                    X, cpw, array_word_bits, nb);
    (void)Y;
    return CELLATO_OK;
}

template <int LAYOUT, typename AW>
void launch_to_planes(const AW* arr, int X, int Y, int nb, int cpw, const plane_set& ps, cudaStream_t s) {
    constexpr int R = band_rows<LAYOUT>();
    const int Xw = X / 32, nbands = Y / R;
    const long long warps = (long long)nbands * Xw;
    const int blocks = (int)((warps + BA_WARPS - 1) / BA_WARPS);
    if (blocks > 0)
        dispatch_planes(nb, [&](auto c) {
            bit_array_to_planes_kernel<LAYOUT, AW, decltype(c)::value>
                <<<blocks, BA_WARPS * 32, 0, s>>>(arr, X, Xw, nbands, cpw, ps);
        });
}

template <int LAYOUT, typename AW>
void launch_to_array(const plane_set& ps, int X, int Y, int nb, int cpw, AW* arr, cudaStream_t s) {
    const long long n = (long long)(X / cpw) * Y;
    const int blocks = (int)((n + 255) / 256);
    if (blocks > 0) planes_to_bit_array_kernel<LAYOUT, AW><<<blocks, 256, 0, s>>>(ps, X, Y, nb, cpw, arr);
}

template <typename AW>
void to_planes(int internal, const void* array, int X, int Y, int nb, int cpw, const plane_set& ps, cudaStream_t s) {
    const AW* arr = static_cast<const AW*>(array);
    switch (internal) {
        case LAYOUT_LINEAR: return launch_to_planes<LAYOUT_LINEAR, AW>(arr, X, Y, nb, cpw, ps, s);
        case LAYOUT_TILED4: return launch_to_planes<LAYOUT_TILED4, AW>(arr, X, Y, nb, cpw, ps, s);
        case LAYOUT_TILED8: return launch_to_planes<LAYOUT_TILED8, AW>(arr, X, Y, nb, cpw, ps, s);
    }
}

template <typename AW>
void to_array(int internal, const plane_set& ps, int X, int Y, int nb, int cpw, void* array, cudaStream_t s) {
    AW* arr = static_cast<AW*>(array);
    switch (internal) {
        case LAYOUT_LINEAR: return launch_to_array<LAYOUT_LINEAR, AW>(ps, X, Y, nb, cpw, arr, s);
        case LAYOUT_TILED4: return launch_to_array<LAYOUT_TILED4, AW>(ps, X, Y, nb, cpw, arr, s);
        case LAYOUT_TILED8: return launch_to_array<LAYOUT_TILED8, AW>(ps, X, Y, nb, cpw, arr, s);
    }
}

}  // namespace

extern "C" {

size_t cellato_bit_array_bytes(int nb, int array_word_bits, int x_cells, int y_cells) {
    if (nb < 1 || nb > MAX_PLANES || (array_word_bits != 32 && array_word_bits != 64) || x_cells < 0 || y_cells < 0)
        return 0;
    const int cpw = array_word_bits / nb;
    const size_t cells = (size_t)x_cells * y_cells;
    return (cells + cpw - 1) / cpw * (array_word_bits / 8);
}

int cellato_bit_array_to_planes(int nb, int array_word_bits, const void* array, int x_cells, int y_cells, int layout,
                                int word_bits, void* const* planes, cellato_stream_t stream) {
    if (int rc = check_array(nb, array_word_bits, x_cells, y_cells, array)) return rc;
    if (int rc = check_dims(layout, word_bits, x_cells, y_cells)) return rc;
    plane_set ps;
    if (int rc = planes_of(nb, planes, ps)) return rc;
    const int internal = internal_layout(layout, word_bits);
    const int cpw = array_word_bits / nb;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (array_word_bits == 32)
        to_planes<uint32_t>(internal, array, x_cells, y_cells, nb, cpw, ps, s);
    else
        to_planes<unsigned long long>(internal, array, x_cells, y_cells, nb, cpw, ps, s);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CELLATO_OK : cuda_fail(e, "bit_array to planes launch");
}

int cellato_planes_to_bit_array(int nb, int layout, int word_bits, const void* const* planes, int x_cells,
                                int y_cells, int array_word_bits, void* array, cellato_stream_t stream) {
    if (int rc = check_array(nb, array_word_bits, x_cells, y_cells, array)) return rc;
    if (int rc = check_dims(layout, word_bits, x_cells, y_cells)) return rc;
    plane_set ps;
    if (int rc = planes_of(nb, const_cast<void* const*>(planes), ps)) return rc;
    const int internal = internal_layout(layout, word_bits);
    const int cpw = array_word_bits / nb;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (array_word_bits == 32)
        to_array<uint32_t>(internal, ps, x_cells, y_cells, nb, cpw, array, s);
    else
        to_array<unsigned long long>(internal, ps, x_cells, y_cells, nb, cpw, array, s);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CELLATO_OK : cuda_fail(e, "planes to bit_array launch");
}

}  // extern "C"
