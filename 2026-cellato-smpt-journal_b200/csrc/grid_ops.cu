// Whole-grid operations on bit planes: the 4 x 4 tile checksum, a full-grid
// diff (count of differing cells) and a seeded random initial state, all
// computed where the planes live.
//
// Checksum.  The reference reduces a grid to sixteen numbers -- the sums of
// the cells' state values over a 4 x 4 partition into tiles of ceil(X/4) x
// ceil(Y/4) cells -- on the host, after converting the planes back to one value
// per cell (include/memory/standard_grid.hpp:179-212, called from
// include/experiments/experiment_manager.hpp:89).  Here the sums come straight
// from the planes.  The state value of a cell is a function of its nb index
// bits, and every such function is a polynomial that is linear in each bit:
//     value(b) = sum over plane subsets S of a_S * prod_{p in S} b_p,
// with a_S from the Moebius transform of the value table (a_S = sum over T in S
// of (-1)^{|S|-|T|} value(T)).  The sum of values over a set of cells is then
// sum_S a_S * popcount(AND of the planes in S, masked to the set): one AND chain
// and one popcount per non-zero term and word.  For the integer-valued
// dictionaries (value = index) only the nb single-plane terms remain.
//
// Random state.  Cell (x, y) of an X-wide grid takes the dictionary index
// #{ i : thresholds[i] <= u }, u the upper 32 bits of SplitMix64 (Steele, Lea
// and Flood, OOPSLA 2014) at position seed + (y*X + x + 1) * 0x9E3779B97F4A7C15.
// Ascending thresholds t_i = floor(P(index <= i) * 2^32) give each index its
// probability to within 2^-32.  The planes are written directly; no byte grid
// exists.  This generator is this library's own (the reference seeds
// std::mt19937 in generate_random_grid, include/memory/grid_utils.hpp:36-60);
// it feeds batched and served workloads, whose results are compared with
// single-grid runs of the same planes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "capi_internal.hpp"
#include "cellato_b200.h"
#include "b200/engine.cuh"

using namespace cellato::b200;
using namespace cellato::b200::capi;

namespace {

constexpr int OPS_WARPS = 8;
constexpr int MAX_TERMS = 32;

struct checksum_terms {
    long long coef[MAX_TERMS];
    unsigned char planes[MAX_TERMS];  // bit p set: plane p is in the product (0: the constant term)
    int n;
};

struct random_thresholds {
    uint32_t t[32];
    int n;
};

// Tile-sum accumulator of one thread: per term of the value polynomial, the
// popcount total of the tile it last touched (32-bit: at most 32 cells per word
// and fewer than 2^27 words per tile and thread); the weighted sum goes to the
// CTA's shared sums when the tile changes.
template <int NT>
struct tile_acc {
    int key = -1;
    unsigned cnt[NT] = {};
    __device__ void flush(unsigned long long* sh, const checksum_terms& terms) {
        if (key >= 0) {
            long long v = 0;
#pragma unroll
            for (int i = 0; i < NT; ++i) v += terms.coef[i] * (long long)cnt[i];
            if (v) atomicAdd(&sh[key], (unsigned long long)v);
        }
#pragma unroll
        for (int i = 0; i < NT; ++i) cnt[i] = 0;
    }
    // adds the cells of one row word selected by `mask` to tile k
    template <int NB>
    __device__ void add(int k, const word (&P)[NB], word mask, const checksum_terms& terms, unsigned long long* sh) {
        if (k != key) {
            flush(sh, terms);
            key = k;
        }
#pragma unroll
        for (int i = 0; i < NT; ++i) {
            if (i >= terms.n) break;
            word m = mask;
            const unsigned sel = terms.planes[i];
#pragma unroll
            for (int p = 0; p < NB; ++p) m &= ((sel >> p) & 1u) ? P[p] : ~0u;
            cnt[i] += __popc(m);
        }
    }
};

// Each warp takes a contiguous run of (band, word) units, lane-interleaved, so
// a thread's consecutive units are 32 words apart in the same rows and its
// tile changes rarely.
template <int LAYOUT, int NB>
__global__ void __launch_bounds__(OPS_WARPS * 32) checksum_kernel(plane_set in, int X, int Y, int Xw, int nbands,
                                                                  int tw, int th, long long units_per_warp,
                                                                  checksum_terms terms,
                                                                  unsigned long long* __restrict__ out) {
    constexpr int R = band_rows<LAYOUT>();
    constexpr int NT = (1 << NB) < MAX_TERMS ? (1 << NB) : MAX_TERMS;
    __shared__ unsigned long long sh[16];
    if (threadIdx.x < 16) sh[threadIdx.x] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const long long warp = (long long)blockIdx.x * OPS_WARPS + (threadIdx.x >> 5);
    const long long units = (long long)nbands * Xw;
    const long long u0 = warp * units_per_warp;
    const long long u1 = min(units, u0 + units_per_warp);
    tile_acc<NT> acc;
    for (long long u = u0 + lane; u < u1; u += 32) {
        const int b = (int)(u / Xw), gx = (int)(u % Xw);
        word rows[NB][R];
#pragma unroll
        for (int p = 0; p < NB; ++p) load_word_rows<LAYOUT>(in.p[p], Xw, b, gx, rows[p]);
        const int x0 = 32 * gx;
        const int tx0 = x0 / tw;
        const bool whole = (tx0 + 1) * tw >= x0 + 32;  // the word lies in one tile column
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int y = b * R + r;
            if (y >= Y) break;
            const int ty = y / th;
            word P[NB];
#pragma unroll
            for (int p = 0; p < NB; ++p) P[p] = rows[p][r];
            if (whole) {
                acc.template add<NB>(ty * 4 + tx0, P, ~0u, terms, sh);
            } else {
                for (int tx = tx0; tx < 4 && tx * tw < x0 + 32; ++tx) {
                    const int lo = max(tx * tw - x0, 0), hi = min((tx + 1) * tw - x0, 32);
                    const word mask = (hi >= 32 ? ~0u : ((1u << hi) - 1u)) & ~((1u << lo) - 1u);
                    acc.template add<NB>(ty * 4 + tx, P, mask, terms, sh);
                }
            }
        }
    }
    acc.flush(sh, terms);
    __syncthreads();
    if (threadIdx.x < 16 && sh[threadIdx.x]) atomicAdd(&out[threadIdx.x], sh[threadIdx.x]);
}

__device__ __forceinline__ uint32_t splitmix_upper(unsigned long long seed, unsigned long long n) {
    unsigned long long z = seed + (n + 1ull) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (uint32_t)(z >> 32);
}

// One warp per (band, linear word), lane = cell, one ballot per plane and row
// (the layout of the packing kernel).
template <int LAYOUT, int NB>
__global__ void __launch_bounds__(OPS_WARPS * 32) fill_random_kernel(int X, int Xw, int nbands,
                                                                     unsigned long long seed, random_thresholds th,
                                                                     plane_set out) {
    constexpr int R = band_rows<LAYOUT>();
    const int lane = threadIdx.x & 31;
    const long long w = (long long)blockIdx.x * OPS_WARPS + (threadIdx.x >> 5);
    if (w >= (long long)nbands * Xw) return;  // whole warp exits together
    const int b = (int)(w / Xw), gx = (int)(w % Xw);
    word bits[R][NB];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const unsigned long long n = (unsigned long long)(b * R + r) * X + 32 * gx + lane;
        const uint32_t u = splitmix_upper(seed, n);
        int idx = 0;
        for (int i = 0; i < th.n; ++i) idx += (u >= th.t[i]) ? 1 : 0;
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

// Cells that differ between two grids of the same layout: a cell is one bit
// position in every plane, so per word the differing cells are the OR over the
// planes of a ^ b.  128-bit loads, grid-stride; one atomic per warp.
__global__ void __launch_bounds__(256) diff_kernel(plane_set a, plane_set b, int nb, long long n_words,
                                                   unsigned long long* __restrict__ out) {
    const long long n4 = n_words / 4;
    const long long stride = (long long)gridDim.x * blockDim.x;
    unsigned long long local = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
        uint4 acc = make_uint4(0, 0, 0, 0);
        for (int p = 0; p < nb; ++p) {
            const uint4 x = reinterpret_cast<const uint4*>(a.p[p])[i];
            const uint4 y = reinterpret_cast<const uint4*>(b.p[p])[i];
            acc.x |= x.x ^ y.x, acc.y |= x.y ^ y.y, acc.z |= x.z ^ y.z, acc.w |= x.w ^ y.w;
        }
        local += __popc(acc.x) + __popc(acc.y) + __popc(acc.z) + __popc(acc.w);
    }
    for (long long i = 4 * n4 + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_words; i += stride) {
        word acc = 0;
        for (int p = 0; p < nb; ++p) acc |= a.p[p][i] ^ b.p[p][i];
        local += __popc(acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(out, local);
}

// Moebius transform of the value table over the nb index bits.
int make_terms(const rule_ops* ops, checksum_terms& terms) {
    const int nb = ops->planes, n = 1 << nb;
    long long a[256];
    for (int i = 0; i < n; ++i) a[i] = i < ops->states ? ops->state_values[i] : 0;
    for (int p = 0; p < nb; ++p)
        for (int i = 0; i < n; ++i)
            if (i & (1 << p)) a[i] -= a[i ^ (1 << p)];
    std::memset(&terms, 0, sizeof terms);
    for (int i = 0; i < n; ++i) {
        if (!a[i]) continue;
        if (terms.n == MAX_TERMS) return fail(CELLATO_EUNSUPPORTED, "state table needs more than %d terms", MAX_TERMS);
        terms.coef[terms.n] = a[i];
        terms.planes[terms.n] = (unsigned char)i;
        ++terms.n;
    }
    return CELLATO_OK;
}

int planes_of(int nb, void* const* planes, plane_set& ps) {
    if (nb < 1 || nb > MAX_PLANES) return fail(CELLATO_EINVAL, "plane count %d out of range 1..%d", nb, MAX_PLANES);
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

template <int LAYOUT, int NB>
void launch_checksum(const plane_set& ps, int X, int Y, const checksum_terms& terms, unsigned long long* out,
                     cudaStream_t s) {
    constexpr int R = band_rows<LAYOUT>();
    const int Xw = X / 32, nbands = Y / R;
    const long long units = (long long)nbands * Xw;
    // about 64 warps per SM (enough loads in flight for HBM), each a
    // contiguous run of whole 32-unit groups
    const long long warps = 148LL * 64;
    long long per_warp = (units + warps - 1) / warps;
    per_warp = (per_warp + 31) / 32 * 32;
    const long long used = (units + per_warp - 1) / per_warp;
    const int blocks = (int)((used + OPS_WARPS - 1) / OPS_WARPS);
    checksum_kernel<LAYOUT, NB><<<blocks, OPS_WARPS * 32, 0, s>>>(ps, X, Y, Xw, nbands, (X + 3) / 4, (Y + 3) / 4,
                                                                   per_warp, terms, out);
}

template <int LAYOUT>
void launch_checksum_nb(int nb, const plane_set& ps, int X, int Y, const checksum_terms& terms,
                        unsigned long long* out, cudaStream_t s) {
    switch (nb) {
        case 1: return launch_checksum<LAYOUT, 1>(ps, X, Y, terms, out, s);
        case 2: return launch_checksum<LAYOUT, 2>(ps, X, Y, terms, out, s);
        case 3: return launch_checksum<LAYOUT, 3>(ps, X, Y, terms, out, s);
        case 4: return launch_checksum<LAYOUT, 4>(ps, X, Y, terms, out, s);
        case 5: return launch_checksum<LAYOUT, 5>(ps, X, Y, terms, out, s);
    }
}

}  // namespace

namespace cellato::b200::capi {

// Stream-ordered tile sums into out[16] (device); used by the C ABI and the server.
int enqueue_checksum(const rule_ops* ops, int layout, int word_bits, const plane_set& ps, int X, int Y,
                     unsigned long long* out, cudaStream_t s) {
    if (ops->planes > 5) return fail(CELLATO_EUNSUPPORTED, "checksum of more than 5 planes is not built");
    checksum_terms terms;
    if (int rc = make_terms(ops, terms)) return rc;
    cudaError_t e = cudaMemsetAsync(out, 0, 16 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync (checksum)");
    switch (internal_layout(layout, word_bits)) {
        case LAYOUT_LINEAR: launch_checksum_nb<LAYOUT_LINEAR>(ops->planes, ps, X, Y, terms, out, s); break;
        case LAYOUT_TILED4: launch_checksum_nb<LAYOUT_TILED4>(ops->planes, ps, X, Y, terms, out, s); break;
        case LAYOUT_TILED8: launch_checksum_nb<LAYOUT_TILED8>(ops->planes, ps, X, Y, terms, out, s); break;
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? CELLATO_OK : cuda_fail(e, "checksum launch");
}

int enqueue_fill_random(int layout, int word_bits, int nb, const plane_set& ps, int X, int Y, unsigned long long seed,
                        const uint32_t* thresholds, int n_thresholds, cudaStream_t s) {
    if (n_thresholds < 0 || n_thresholds > 31 || (n_thresholds > 0 && !thresholds))
        return fail(CELLATO_EINVAL, "threshold count %d out of range 0..31", n_thresholds);
    if (n_thresholds >= (1 << nb))
        return fail(CELLATO_EINVAL, "%d thresholds give indices that %d planes cannot hold", n_thresholds, nb);
    random_thresholds th{};
    th.n = n_thresholds;
    for (int i = 0; i < n_thresholds; ++i) {
        th.t[i] = thresholds[i];
        if (i && thresholds[i] < thresholds[i - 1]) return fail(CELLATO_EINVAL, "thresholds must be ascending");
    }
    const int internal = internal_layout(layout, word_bits);
    const int R = band_height(layout, word_bits);
    const int Xw = X / 32, nbands = Y / R;
    const long long warps = (long long)nbands * Xw;
    const int blocks = (int)((warps + OPS_WARPS - 1) / OPS_WARPS);
    if (blocks > 0) {
        dispatch_planes(nb, [&](auto c) {
            constexpr int NB = decltype(c)::value;
            switch (internal) {
                case LAYOUT_LINEAR:
                    fill_random_kernel<LAYOUT_LINEAR, NB><<<blocks, OPS_WARPS * 32, 0, s>>>(X, Xw, nbands, seed, th, ps);
                    break;
                case LAYOUT_TILED4:
                    fill_random_kernel<LAYOUT_TILED4, NB><<<blocks, OPS_WARPS * 32, 0, s>>>(X, Xw, nbands, seed, th, ps);
                    break;
                case LAYOUT_TILED8:
                    fill_random_kernel<LAYOUT_TILED8, NB><<<blocks, OPS_WARPS * 32, 0, s>>>(X, Xw, nbands, seed, th, ps);
                    break;
            }
        });
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CELLATO_OK : cuda_fail(e, "random fill launch");
}

}  // namespace cellato::b200::capi

extern "C" {

int cellato_checksum(int rule, int layout, int word_bits, const void* const* planes, int x_cells, int y_cells,
                     unsigned long long* sums, cellato_stream_t stream) {
    const rule_ops* ops = ops_of(rule);
    if (!ops) return fail(CELLATO_EINVAL, "unknown rule id %d", rule);
    if (!sums) return fail(CELLATO_EINVAL, "sums must not be NULL");
    if (int rc = check_dims(layout, word_bits, x_cells, y_cells)) return rc;
    plane_set ps;
    if (int rc = planes_of(ops->planes, const_cast<void* const*>(planes), ps)) return rc;
    return enqueue_checksum(ops, layout, word_bits, ps, x_cells, y_cells, sums, reinterpret_cast<cudaStream_t>(stream));
}

int cellato_fill_random(int layout, int word_bits, int nb, void* const* planes, int x_cells, int y_cells,
                        unsigned long long seed, const uint32_t* thresholds, int n_thresholds,
                        cellato_stream_t stream) {
    if (int rc = check_dims(layout, word_bits, x_cells, y_cells)) return rc;
    plane_set ps;
    if (int rc = planes_of(nb, planes, ps)) return rc;
    return enqueue_fill_random(layout, word_bits, nb, ps, x_cells, y_cells, seed, thresholds, n_thresholds,
                               reinterpret_cast<cudaStream_t>(stream));
}

int cellato_diff_cells(int nb, const void* const* planes_a, const void* const* planes_b, size_t plane_bytes,
                       unsigned long long* count, cellato_stream_t stream) {
    if (!count) return fail(CELLATO_EINVAL, "count must not be NULL");
    if (plane_bytes % 4) return fail(CELLATO_EINVAL, "plane bytes %zu are not whole 32-bit words", plane_bytes);
    plane_set pa, pb;
    if (int rc = planes_of(nb, const_cast<void* const*>(planes_a), pa)) return rc;
    if (int rc = planes_of(nb, const_cast<void* const*>(planes_b), pb)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync (diff)");
    const long long n_words = (long long)(plane_bytes / 4);
    if (n_words > 0) {
        const long long want = (n_words / 4 + 255) / 256;
        const int blocks = (int)std::max(1LL, std::min(want, 148LL * 8));
        diff_kernel<<<blocks, 256, 0, s>>>(pa, pb, nb, n_words, count);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? CELLATO_OK : cuda_fail(e, "diff launch");
}

int cellato_rule_state_value(int rule, int index, long long* value) {
    const rule_ops* ops = ops_of(rule);
    if (!ops || !value || index < 0 || index >= ops->states) return fail(CELLATO_EINVAL, "bad rule, index or output");
    *value = ops->state_values[index];
    return CELLATO_OK;
}

}  // extern "C"
