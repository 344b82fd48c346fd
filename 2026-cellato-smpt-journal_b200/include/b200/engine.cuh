// B200 kernels for the bit-plane hot path: a streaming single-step kernel
// (the "simple" traverser) and a temporally blocked shared-memory kernel (the
// "temporal" traverser), both driving one lowered rule (b200/lower.cuh).
//
// Internal representation: linear rows of 32-bit plane words (bit i of word w
// of row y = cell (32w + i, y)).  The byte formats the caller owns are adapted
// at load/store:
//   LAYOUT_LINEAR  bit_planes (reference include/memory/bit_planes_grid.hpp:255-263).
//                  32- and 64-bit words are the same bytes (little endian), so
//                  one kernel serves both word sizes.
//   LAYOUT_TILED4  tiled_bit_planes with 32-bit words: 8 x 4 cell tiles, bit
//                  y_bit*8 + x_bit (tiled_bit_planes_grid.hpp:270-282).
//   LAYOUT_TILED8  tiled_bit_planes with 64-bit words: 8 x 8 cell tiles.
// A linear word spans 4 horizontally adjacent tiles; byte r of a tile word is
// row r of the tile, so tiles <-> linear rows is a 4x4 byte transpose per group
// of four 32-bit tile rows (8 PRMTs), done in registers.
#ifndef CELLATO_B200_ENGINE_CUH
#define CELLATO_B200_ENGINE_CUH

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "b200/lower.cuh"

namespace cellato::b200 {

enum : int { LAYOUT_LINEAR = 0, LAYOUT_TILED4 = 1, LAYOUT_TILED8 = 2 };

constexpr int MAX_PLANES = 8;

// Calls f(std::integral_constant<int, nb>{}) for a runtime plane count 1..MAX_PLANES,
// so that per-plane loops in kernels run exactly nb times.
template <int NB = 1, class F>
inline void dispatch_planes(int nb, F&& f) {
    if constexpr (NB <= MAX_PLANES) {
        if (nb == NB)
            f(std::integral_constant<int, NB>{});
        else
            dispatch_planes<NB + 1>(nb, f);
    }
}

struct plane_set {
    word* p[MAX_PLANES];
};

// Rows per tile word (band height) of a layout.
template <int LAYOUT>
constexpr int band_rows() {
    return LAYOUT == LAYOUT_TILED4 ? 4 : (LAYOUT == LAYOUT_TILED8 ? 8 : 1);
}

// ------------------------------------------------------------ byte transpose
// (t0, t1, t2, t3): four 32-bit words, byte r of t_j = row r of column-block j.
// Returns row-major: r_r = (t0.b_r, t1.b_r, t2.b_r, t3.b_r).  Self-inverse.
__device__ __forceinline__ void transpose4x4(word& a, word& b, word& c, word& d) {
    const word u = __byte_perm(a, b, 0x5140);  // a0 b0 a1 b1
    const word v = __byte_perm(a, b, 0x7362);  // a2 b2 a3 b3
    const word w = __byte_perm(c, d, 0x5140);  // c0 d0 c1 d1
    const word x = __byte_perm(c, d, 0x7362);  // c2 d2 c3 d3
    a = __byte_perm(u, w, 0x5410);             // a0 b0 c0 d0
    b = __byte_perm(u, w, 0x7632);             // a1 b1 c1 d1
    c = __byte_perm(v, x, 0x5410);             // a2 b2 c2 d2
    d = __byte_perm(v, x, 0x7632);             // a3 b3 c3 d3
}

// Global loads of plane words.  Kernels whose input is not written while they
// run read through the read-only data cache (ld.global.nc); the persistent
// batched kernel, whose later rounds read what its earlier rounds wrote in the
// same launch, reads at L2 (ld.global.cg), which no stale L1 line can shadow.
enum : int { LOAD_NC = 0, LOAD_CG = 1 };

template <int LOAD, class T>
__device__ __forceinline__ T gload(const T* p) {
    if constexpr (LOAD == LOAD_CG)
        return __ldcg(p);
    else
        return __ldg(p);
}

// Load the R rows of linear word gx of band b (tile row b) of one plane.
//   linear: R == 1, word gx of row b.
//   tiled : tiles 4gx .. 4gx+3 of tile row b, transposed to R row words.
template <int LAYOUT, int LOAD = LOAD_NC>
__device__ __forceinline__ void load_word_rows(const word* __restrict__ plane, int Xw, int b, int gx,
                                               word (&rows)[band_rows<LAYOUT>()]) {
    if constexpr (LAYOUT == LAYOUT_LINEAR) {
        rows[0] = gload<LOAD>(plane + (size_t)b * Xw + gx);
    } else if constexpr (LAYOUT == LAYOUT_TILED4) {
        // 4 tiles x 4 bytes = one 16-byte vector
        const uint4 t = gload<LOAD>(reinterpret_cast<const uint4*>(plane + ((size_t)b * Xw + gx) * 4));
        word a = t.x, bb = t.y, c = t.z, d = t.w;
        transpose4x4(a, bb, c, d);
        rows[0] = a, rows[1] = bb, rows[2] = c, rows[3] = d;
    } else {
        // 4 tiles x 8 bytes: (lo, hi) per tile; lo = rows 0-3, hi = rows 4-7
        const uint4* src = reinterpret_cast<const uint4*>(plane + ((size_t)b * Xw + gx) * 8);
        const uint4 t01 = gload<LOAD>(src), t23 = gload<LOAD>(src + 1);
        word l0 = t01.x, l1 = t01.z, l2 = t23.x, l3 = t23.z;
        word h0 = t01.y, h1 = t01.w, h2 = t23.y, h3 = t23.w;
        transpose4x4(l0, l1, l2, l3);
        transpose4x4(h0, h1, h2, h3);
        rows[0] = l0, rows[1] = l1, rows[2] = l2, rows[3] = l3;
        rows[4] = h0, rows[5] = h1, rows[6] = h2, rows[7] = h3;
    }
}

template <int LAYOUT>
__device__ __forceinline__ void store_word_rows(word* __restrict__ plane, int Xw, int b, int gx,
                                                const word (&rows)[band_rows<LAYOUT>()]) {
    if constexpr (LAYOUT == LAYOUT_LINEAR) {
        plane[(size_t)b * Xw + gx] = rows[0];
    } else if constexpr (LAYOUT == LAYOUT_TILED4) {
        word a = rows[0], bb = rows[1], c = rows[2], d = rows[3];
        transpose4x4(a, bb, c, d);
        *reinterpret_cast<uint4*>(plane + ((size_t)b * Xw + gx) * 4) = make_uint4(a, bb, c, d);
    } else {
        word l0 = rows[0], l1 = rows[1], l2 = rows[2], l3 = rows[3];
        word h0 = rows[4], h1 = rows[5], h2 = rows[6], h3 = rows[7];
        transpose4x4(l0, l1, l2, l3);
        transpose4x4(h0, h1, h2, h3);
        uint4* dst = reinterpret_cast<uint4*>(plane + ((size_t)b * Xw + gx) * 8);
        dst[0] = make_uint4(l0, h0, l1, h1);
        dst[1] = make_uint4(l2, h2, l3, h3);
    }
}

// A lane's V consecutive words (gx a multiple of V, Xw a multiple of V) of the
// R rows of band b; linear rows use one 8- or 16-byte vector access.
template <int LAYOUT, int V>
__device__ __forceinline__ void load_lane(const word* __restrict__ plane, int Xw, int b, int gx,
                                          word (&rows)[band_rows<LAYOUT>()][V]) {
    if constexpr (LAYOUT == LAYOUT_LINEAR && V == 4) {
        const uint4 q = __ldg(reinterpret_cast<const uint4*>(plane + (size_t)b * Xw + gx));
        rows[0][0] = q.x, rows[0][1] = q.y, rows[0][2] = q.z, rows[0][3] = q.w;
    } else if constexpr (LAYOUT == LAYOUT_LINEAR && V == 2) {
        const uint2 q = __ldg(reinterpret_cast<const uint2*>(plane + (size_t)b * Xw + gx));
        rows[0][0] = q.x, rows[0][1] = q.y;
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) {
            word t[band_rows<LAYOUT>()];
            load_word_rows<LAYOUT>(plane, Xw, b, gx + v, t);
#pragma unroll
            for (int r = 0; r < band_rows<LAYOUT>(); ++r) rows[r][v] = t[r];
        }
    }
}

template <int LAYOUT, int V>
__device__ __forceinline__ void store_lane(word* __restrict__ plane, int Xw, int b, int gx,
                                           const word (&rows)[band_rows<LAYOUT>()][V]) {
    if constexpr (LAYOUT == LAYOUT_LINEAR && V == 4) {
        *reinterpret_cast<uint4*>(plane + (size_t)b * Xw + gx) = make_uint4(rows[0][0], rows[0][1], rows[0][2], rows[0][3]);
    } else if constexpr (LAYOUT == LAYOUT_LINEAR && V == 2) {
        *reinterpret_cast<uint2*>(plane + (size_t)b * Xw + gx) = make_uint2(rows[0][0], rows[0][1]);
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) {
            word t[band_rows<LAYOUT>()];
#pragma unroll
            for (int r = 0; r < band_rows<LAYOUT>(); ++r) t[r] = rows[r][v];
            store_word_rows<LAYOUT>(plane, Xw, b, gx + v, t);
        }
    }
}

// ------------------------------------------------------------- lane helpers
// Words to the left / right of a lane's V words, from the neighbouring lanes
// (lane 0 and lane 31 receive the wrapped value of lane 31 / lane 0, which is
// correct when the warp spans the whole row and is overridden otherwise).
__device__ __forceinline__ word from_left_lane(word v) {
    return __shfl_sync(0xffffffffu, v, (threadIdx.x + 31) & 31);
}
__device__ __forceinline__ word from_right_lane(word v) {
    return __shfl_sync(0xffffffffu, v, (threadIdx.x + 1) & 31);
}

// Features of one row of a lane's V words.  The predicates of the rule's count
// targets are computed on the lane's own words and only those one-plane
// predicates cross lanes; raw planes cross lanes only when the rule reads
// neighbours at dx != 0.  use_l / use_r: take the left / right neighbour word
// from Ledge / Redge (a lane at a segment edge that loaded it) instead of the
// neighbouring lane.
template <class Net, int NB, int V>
__device__ __forceinline__ void row_feats(const word (&C)[NB][V], const word (&Ledge)[NB], const word (&Redge)[NB],
                                          bool use_l, bool use_r, typename Net::feat (&out)[V]) {
    using preds_t = typename Net::preds_t;
    constexpr int T = Net::targets::size;
    word col[V][NB];
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
        for (int p = 0; p < NB; ++p) col[v][p] = C[p][v];
    preds_t pc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) pc[v] = Net::preds(col[v]);
    preds_t pl = pc[0], pr = pc[0];
    if constexpr (T > 0) {
#pragma unroll
        for (int t = 0; t < T; ++t) {
            pl.p[t] = from_left_lane(pc[V - 1].p[t]);
            pr.p[t] = from_right_lane(pc[0].p[t]);
        }
        if (use_l) pl = Net::preds(Ledge);
        if (use_r) pr = Net::preds(Redge);
    }
    word Lw[NB], Rw[NB];
#pragma unroll
    for (int p = 0; p < NB; ++p) {
        if constexpr (Net::need_shift) {
            Lw[p] = from_left_lane(C[p][V - 1]);
            Rw[p] = from_right_lane(C[p][0]);
            if (use_l) Lw[p] = Ledge[p];
            if (use_r) Rw[p] = Redge[p];
        } else {
            Lw[p] = Rw[p] = 0;
        }
    }
#pragma unroll
    for (int v = 0; v < V; ++v)
        out[v] = Net::make(col[v], v == 0 ? Lw : col[v == 0 ? 0 : v - 1], v == V - 1 ? Rw : col[v == V - 1 ? 0 : v + 1],
                           pc[v], v == 0 ? pl : pc[v == 0 ? 0 : v - 1], v == V - 1 ? pr : pc[v == V - 1 ? 0 : v + 1]);
}

// ======================================================= single-step kernel
// One launch = one time step.  Each warp owns a horizontal segment of 32*V
// words (lane l: words seg*32V + l*V .. +V-1) and walks down the CTA's rows in
// bands of BR rows with a rolling window of three rows' features.  The next
// band's loads are issued before the current band is computed, so a warp keeps
// BR rows x NB planes x 32V words in flight (the single-step kernel streams:
// HBM latency x bandwidth must be covered by bytes in flight).  Every input
// word is loaded once per CTA row range (+2 halo rows), every output word
// stored once.
//   linear : BR = SIMPLE_LINEAR_BAND independent rows per band
//   tiled  : BR = rows of one tile word (4 or 8)
constexpr int SIMPLE_LINEAR_BAND = 8;

template <int LAYOUT>
constexpr int simple_band_rows() {
    return LAYOUT == LAYOUT_LINEAR ? SIMPLE_LINEAR_BAND : band_rows<LAYOUT>();
}

template <class Net, int NB, int LAYOUT, int V, int TP, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) simple_step_kernel(plane_set in, plane_set out, int Xw, int Y,
                                                                 int nbands, int bands_per_cta) {
    constexpr int R = band_rows<LAYOUT>();
    constexpr int BR = simple_band_rows<LAYOUT>();
    using feat = typename Net::feat;
    const int lane = threadIdx.x & 31;
    const int seg = blockIdx.x * WARPS + (threadIdx.x >> 5);
    const int gx_raw = seg * 32 * V + lane * V;          // first word of this lane (unwrapped)
    const bool owns = gx_raw < Xw;                        // lanes past the row end only feed neighbours
    const int gx = gx_raw % Xw;
    const int gx_left = (seg * 32 * V + Xw - 1) % Xw;     // word left of the segment
    const int gx_right = (seg * 32 * V + 32 * V) % Xw;    // word right of the segment
    const bool seg_spans_row = (32 * V == Xw);            // lane 0 / 31 neighbours are lanes 31 / 0

    const int b0 = blockIdx.y * bands_per_cta;
    const int b1 = min(nbands, b0 + bands_per_cta);
    if (b0 >= b1) return;

    // Load one band: linear -> rows b*BR .. b*BR+BR-1 (wrapped), tiled -> tile row b.
    auto load_band = [&](int b, word (&raw)[BR][NB][V], word (&L)[BR][NB], word (&Rr)[BR][NB]) {
        if constexpr (LAYOUT == LAYOUT_LINEAR) {
            int y = (b * BR) % Y;
            if (y < 0) y += Y;
#pragma unroll
            for (int r = 0; r < BR; ++r) {
#pragma unroll
                for (int p = 0; p < NB; ++p) {
                    word rows[1][V];
                    load_lane<LAYOUT, V>(in.p[p], Xw, y, gx, rows);
#pragma unroll
                    for (int v = 0; v < V; ++v) raw[r][p][v] = rows[0][v];
                }
                if (!seg_spans_row && (lane == 0 || lane == 31)) {
#pragma unroll
                    for (int p = 0; p < NB; ++p) {
                        const word e = __ldg(in.p[p] + (size_t)y * Xw + (lane == 0 ? gx_left : gx_right));
                        if (lane == 0) L[r][p] = e; else Rr[r][p] = e;
                    }
                }
                if (++y == Y) y = 0;
            }
        } else {
            int bw = b % nbands;
            if (bw < 0) bw += nbands;
#pragma unroll
            for (int p = 0; p < NB; ++p) {
                word rows[R][V];
                load_lane<LAYOUT, V>(in.p[p], Xw, bw, gx, rows);
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int v = 0; v < V; ++v) raw[r][p][v] = rows[r][v];
            }
            if (!seg_spans_row && (lane == 0 || lane == 31)) {
                const int gxe = lane == 0 ? gx_left : gx_right;
#pragma unroll
                for (int p = 0; p < NB; ++p) {
                    word rows[R];
                    load_word_rows<LAYOUT>(in.p[p], Xw, bw, gxe, rows);
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        if (lane == 0) L[r][p] = rows[r]; else Rr[r][p] = rows[r];
                    }
                }
            }
        }
    };
    const bool use_l = !seg_spans_row && lane == 0;   // loaded, not shuffled
    const bool use_r = !seg_spans_row && lane == 31;
    auto feat_of = [&](const word (&raw)[BR][NB][V], const word (&L)[BR][NB], const word (&Rr)[BR][NB], int r,
                       feat (&f)[V]) {
        word C[NB][V], Lw[NB], Rw[NB];
#pragma unroll
        for (int p = 0; p < NB; ++p) {
#pragma unroll
            for (int v = 0; v < V; ++v) C[p][v] = raw[r][p][v];
            Lw[p] = L[r][p];
            Rw[p] = Rr[r][p];
        }
        row_feats<Net, NB, V>(C, Lw, Rw, use_l, use_r, f);
    };

    word cur[BR][NB][V], curL[BR][NB], curR[BR][NB];
    word nxt[BR][NB][V], nxtL[BR][NB], nxtR[BR][NB];
    feat up[V], mid[V], dn[V];

    // the row above the first band
    if constexpr (LAYOUT == LAYOUT_LINEAR) {
        int y = (b0 * BR - 1) % Y;
        if (y < 0) y += Y;
        word C[NB][V], Lw[NB], Rw[NB];
#pragma unroll
        for (int p = 0; p < NB; ++p) {
            word rows[1][V];
            load_lane<LAYOUT, V>(in.p[p], Xw, y, gx, rows);
#pragma unroll
            for (int v = 0; v < V; ++v) C[p][v] = rows[0][v];
            Lw[p] = Rw[p] = 0;
            if (use_l || use_r) {
                const word e = __ldg(in.p[p] + (size_t)y * Xw + (lane == 0 ? gx_left : gx_right));
                if (use_l) Lw[p] = e; else Rw[p] = e;
            }
        }
        row_feats<Net, NB, V>(C, Lw, Rw, use_l, use_r, up);
    } else {
        load_band(b0 - 1, nxt, nxtL, nxtR);
        feat_of(nxt, nxtL, nxtR, BR - 1, up);
    }
    load_band(b0, cur, curL, curR);
    feat_of(cur, curL, curR, 0, mid);

    for (int b = b0; b < b1; ++b) {
        load_band(b + 1, nxt, nxtL, nxtR);  // in flight while this band computes
        word res[LAYOUT == LAYOUT_LINEAR ? 1 : BR][NB][V];
#pragma unroll
        for (int r = 0; r < BR; ++r) {
            if (r + 1 < BR) {
                feat_of(cur, curL, curR, r + 1 < BR ? r + 1 : 0, dn);
            } else {
                feat_of(nxt, nxtL, nxtR, 0, dn);
            }
            const int y = b * BR + r;
            word o[NB][V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                word ov[NB];
                Net::template eval<TP>(up[v], mid[v], dn[v], y & 1, ov);
#pragma unroll
                for (int p = 0; p < NB; ++p) o[p][v] = ov[p];
            }
            if constexpr (LAYOUT == LAYOUT_LINEAR) {
                if (owns && y < Y) {
#pragma unroll
                    for (int p = 0; p < NB; ++p) {
                        word rows[1][V];
#pragma unroll
                        for (int v = 0; v < V; ++v) rows[0][v] = o[p][v];
                        store_lane<LAYOUT, V>(out.p[p], Xw, y, gx, rows);
                    }
                }
            } else {
#pragma unroll
                for (int p = 0; p < NB; ++p)
#pragma unroll
                    for (int v = 0; v < V; ++v) res[r < BR ? r : 0][p][v] = o[p][v];
            }
#pragma unroll
            for (int v = 0; v < V; ++v) {
                up[v] = mid[v];
                mid[v] = dn[v];
            }
        }
        if constexpr (LAYOUT != LAYOUT_LINEAR) {
            if (owns) {
#pragma unroll
                for (int p = 0; p < NB; ++p) {
                    word rows[R][V];
#pragma unroll
                    for (int r = 0; r < R; ++r)
#pragma unroll
                        for (int v = 0; v < V; ++v) rows[r][v] = res[r][p][v];
                    store_lane<LAYOUT, V>(out.p[p], Xw, b, gx, rows);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < BR; ++r)
#pragma unroll
            for (int p = 0; p < NB; ++p) {
#pragma unroll
                for (int v = 0; v < V; ++v) cur[r][p][v] = nxt[r][p][v];
                curL[r][p] = nxtL[r][p];
                curR[r][p] = nxtR[r][p];
            }
    }
}

// ================================================ streaming single-step kernel
// The single-step kernel for the linear layout, fed by the bulk-copy engine.
// Each warp owns a segment of 32*V words of every row (as above) and a ring of
// STAGES shared-memory stages of BR rows.  Lane 0 issues, per row and plane,
// cp.async.bulk copies of the segment and of the 16-byte blocks holding the
// words to its left and right (wrapped on the torus), completing on the stage's
// mbarrier; the warp computes from shared memory while the next stages land.
// Registers hold only the three-row feature window, so occupancy stays high and
// the bytes in flight are set by the ring, not by the register file.
//
// Shared row layout (words): [4 left-halo][32V segment][4 right-halo]; a
// segment cut short by the row end places its right halo right after its last
// word, where the first idle lane reads it.  Needs Xw % 4 == 0 (16-byte rows).
//
// Every mbarrier wait is bounded: a wait that gives up records the failure in
// g_wait_timeouts, drains the copies this warp still has in flight (again
// bounded) and returns; the host reads and clears the counter through the
// rule's status entry.
//
// g_wait_timeouts counts every bounded device-side wait of one rule's kernels
// that gave up (one counter per translation unit, i.e. per rule).
static __device__ unsigned g_wait_timeouts = 0;

constexpr int STREAM_STAGES = 3;
constexpr int STREAM_BAND = 4;
constexpr unsigned STREAM_WAIT_LIMIT = 1u << 22;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
    for (unsigned it = 0; it < STREAM_WAIT_LIMIT; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

template <int NB, int V>
constexpr int stream_row_words() {
    return 32 * V + 8;
}

template <int NB, int V>
constexpr int stream_smem_per_warp() {
    return STREAM_STAGES * STREAM_BAND * NB * stream_row_words<NB, V>() * 4 + STREAM_STAGES * 8;
}

template <class Net, int NB, int V, int TP, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) stream_step_kernel(plane_set in, plane_set out, int Xw, int Y,
                                                                 int rows_per_cta) {
    constexpr int BR = STREAM_BAND, S = STREAM_STAGES, RW = stream_row_words<NB, V>();
    using feat = typename Net::feat;
    extern __shared__ __align__(16) word smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    word* ring = smem + (size_t)warp * (S * BR * NB * RW);
    unsigned long long* bars =
        reinterpret_cast<unsigned long long*>(smem + (size_t)WARPS * S * BR * NB * RW) + warp * S;

    const int seg = blockIdx.x * WARPS + warp;
    const int gx0 = seg * 32 * V;          // first word of the segment
    if (gx0 >= Xw) return;                  // whole warp: nothing of this row range
    const int valid = min(32 * V, Xw - gx0);
    const int gx = gx0 + lane * V;
    const bool owns = gx < Xw;
    const int gl = (gx0 - 4 + Xw) % Xw;     // 16-byte block left of the segment
    const int gr = (gx0 + valid) % Xw;      // 16-byte block right of it
    const int y0 = blockIdx.y * rows_per_cta;
    const int y1 = min(Y, y0 + rows_per_cta);
    if (y0 >= y1) return;
    const int nstream = (y1 - y0) + 2;      // rows y0-1 .. y1
    const int nchunks = (nstream + BR - 1) / BR;

    auto issue = [&](int c) {  // lane 0 only
        const int s = c % S;
        const int r0 = c * BR;
        const int nr = min(BR, nstream - r0);
        const unsigned bytes = (unsigned)(nr * NB * (valid + 8) * 4);
        mbar_expect_tx(&bars[s], bytes);
        int y = (y0 - 1 + r0) % Y;
        if (y < 0) y += Y;
        for (int r = 0; r < nr; ++r) {
            for (int p = 0; p < NB; ++p) {
                word* dst = ring + ((size_t)(s * BR + r) * NB + p) * RW;
                const word* row = in.p[p] + (size_t)y * Xw;
                bulk_g2s(dst, row + gl, 16, &bars[s]);
                bulk_g2s(dst + 4, row + gx0, (unsigned)valid * 4, &bars[s]);
                bulk_g2s(dst + 4 + valid, row + gr, 16, &bars[s]);
            }
            if (++y == Y) y = 0;
        }
    };

    if (lane == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (lane == 0)
        for (int c = 0; c < min(S, nchunks); ++c) issue(c);

    feat up[V], mid[V], dn[V];
    int failed_at = -1;
    for (int c = 0; c < nchunks; ++c) {
        const int s = c % S;
        if (!mbar_wait_bounded(&bars[s], (unsigned)(c / S) & 1u)) {
            failed_at = c;
            break;
        }
#pragma unroll
        for (int r = 0; r < BR; ++r) {
            const int i = c * BR + r;  // stream row: global row y0 - 1 + i
            if (i < nstream) {
                word C[NB][V], Lw[NB], Rw[NB];
#pragma unroll
                for (int p = 0; p < NB; ++p) {
                    const word* row = ring + ((size_t)(s * BR + r) * NB + p) * RW;
                    if constexpr (V == 4) {
                        const uint4 q = *reinterpret_cast<const uint4*>(row + 4 + lane * 4);
                        C[p][0] = q.x, C[p][1] = q.y, C[p][2] = q.z, C[p][3] = q.w;
                    } else if constexpr (V == 2) {
                        const uint2 q = *reinterpret_cast<const uint2*>(row + 4 + lane * 2);
                        C[p][0] = q.x, C[p][1] = q.y;
                    } else {
                        C[p][0] = row[4 + lane];
                    }
                    Lw[p] = row[3];
                    Rw[p] = row[4 + 32 * V];
                }
                row_feats<Net, NB, V>(C, Lw, Rw, lane == 0, lane == 31, dn);
                if (i >= 2) {
                    const int y = y0 + i - 2;
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        word o[NB];
                        Net::template eval<TP>(up[v], mid[v], dn[v], y & 1, o);
#pragma unroll
                        for (int p = 0; p < NB; ++p) C[p][v] = o[p];
                    }
                    if (owns) {
#pragma unroll
                        for (int p = 0; p < NB; ++p) {
                            word rows[1][V];
#pragma unroll
                            for (int v = 0; v < V; ++v) rows[0][v] = C[p][v];
                            store_lane<LAYOUT_LINEAR, V>(out.p[p], Xw, y, gx, rows);
                        }
                    }
                }
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    up[v] = mid[v];
                    mid[v] = dn[v];
                }
            }
        }
        __syncwarp();
        if (lane == 0 && c + S < nchunks) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(c + S);
        }
    }
    if (failed_at >= 0) {
        if (lane == 0) atomicAdd(&g_wait_timeouts, 1u);
        // drain the copies this warp still has in flight (chunks failed_at ..
        // failed_at + S - 1 were issued, the one that timed out included) before
        // the CTA's shared memory is released
        for (int c = failed_at; c < min(nchunks, failed_at + S); ++c)
            mbar_wait_bounded(&bars[c % S], (unsigned)(c / S) & 1u);
    }
}

// ==================================================== temporal-blocked kernel
// One launch = k time steps on a shared-memory tile of TH rows x 32V words
// (one warp spans the tile width; lane l owns words l*V .. l*V+V-1 of every
// row).  The tile carries a 1-word (32-cell) halo left and right and HY rows
// above and below (HY >= k, a multiple of the band height), so after k steps
// its interior -- words 1 .. 32V-2, rows HY .. TH-HY-1 -- is exact.
//
// Steps update the tile in place.  At step t only rows t .. TH-1-t are
// computed (the valid region shrinks by one row per step); they are split into
// WARPS contiguous bands of equal size (within one row), so the warps stay
// balanced as the region shrinks.  Each warp sweeps its band top-down: the
// rolling window keeps the old value of the row above in registers, the row
// below is read before it is overwritten, and horizontal neighbours come from
// lane shuffles of registers, so no lane ever reads a word another lane writes
// within a step.  Only the two rows bordering a band belong to other warps:
// they are read before the first barrier of the step and every write happens
// after it.
// HOIST selects the row loop: true reads the three input rows of each 3-row
// trip before the trip's writes; false reads each row just before the row
// above it is evaluated.  Both compute the same values; which is faster
// depends on the rule's register use and the occupancy (the autotuner picks).
// LOAD: how the tile is read from global memory (LOAD_NC, or LOAD_CG when the
// input may have been written earlier in the same launch).
// PAIR: two steps per sweep (see pair_step); an odd last step runs alone.
template <class Net, int NB, int LAYOUT, int V, int WARPS, bool HOIST = true, int LOAD = LOAD_NC, bool PAIR = false>
__device__ __forceinline__ void temporal_tile(const plane_set& in, const plane_set& out, int Xw, int Y, int t0, int k,
                                              int TH, int HY, int bx, int by) {
    constexpr int R = band_rows<LAYOUT>();
    constexpr int TW = 32 * V;  // tile width in words
    using feat = typename Net::feat;
    // [TH][NB][TW]: a row's planes are adjacent, so one base address per row
    // reaches all of them through constant offsets
    extern __shared__ __align__(16) word tile[];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int effW = TW - 2;
    const int effH = TH - 2 * HY;
    const int x0 = bx * effW;  // first output word
    const int y0 = by * effH;  // first output row
    const int Yb = Y / R;

    auto at = [&](int p, int r, int s) -> word& { return tile[((size_t)r * NB + p) * TW + s]; };

    // ---- load the tile (rows wrap on the torus; words wrap per word)
    for (int band = warp; band < TH / R; band += WARPS) {
        const int gy0 = y0 - HY + band * R;                   // first global row of this band (unwrapped)
        const int bw = ((gy0 / R) % Yb + Yb) % Yb;            // gy0 is a multiple of R
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int s = lane * V + v;
            const int gx = ((x0 - 1 + s) % Xw + Xw) % Xw;
#pragma unroll
            for (int p = 0; p < NB; ++p) {
                word rows[R];
                load_word_rows<LAYOUT, LOAD>(in.p[p], Xw, bw, gx, rows);
#pragma unroll
                for (int r = 0; r < R; ++r) at(p, band * R + r, s) = rows[r];
            }
        }
    }
    __syncthreads();


    auto read_row = [&](int r, word (&C)[NB][V]) {
#pragma unroll
        for (int p = 0; p < NB; ++p) {
            if constexpr (V % 4 == 0) {
#pragma unroll
                for (int v = 0; v < V; v += 4) {
                    const uint4 q = *reinterpret_cast<const uint4*>(&at(p, r, lane * V + v));
                    C[p][v] = q.x, C[p][v + 1] = q.y, C[p][v + 2] = q.z, C[p][v + 3] = q.w;
                }
            } else if constexpr (V % 2 == 0) {
#pragma unroll
                for (int v = 0; v < V; v += 2) {
                    const uint2 q = *reinterpret_cast<const uint2*>(&at(p, r, lane * V + v));
                    C[p][v] = q.x, C[p][v + 1] = q.y;
                }
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) C[p][v] = at(p, r, lane * V + v);
            }
        }
    };
    // Lanes 0 and 31 take their outer neighbour from the opposite end of the
    // warp: those words sit in the 1-word halo, whose values do not matter.
    const word no_edge[NB] = {};
    auto feats = [&](const word (&C)[NB][V], feat (&f)[V]) { row_feats<Net, NB, V>(C, no_edge, no_edge, false, false, f); };

    auto write_row = [&](int r, const word (&o)[NB][V]) {
#pragma unroll
        for (int p = 0; p < NB; ++p) {
            if constexpr (V % 4 == 0) {
#pragma unroll
                for (int v = 0; v < V; v += 4)
                    *reinterpret_cast<uint4*>(&at(p, r, lane * V + v)) =
                        make_uint4(o[p][v], o[p][v + 1], o[p][v + 2], o[p][v + 3]);
            } else if constexpr (V % 2 == 0) {
#pragma unroll
                for (int v = 0; v < V; v += 2)
                    *reinterpret_cast<uint2*>(&at(p, r, lane * V + v)) = make_uint2(o[p][v], o[p][v + 1]);
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) at(p, r, lane * V + v) = o[p][v];
            }
        }
    };

    // One output row r: dn features from row r+1 (or the saved bottom row),
    // evaluation, in-place write.  fu/fm/fd rotate roles between calls.
    auto row_body = [&](int r, int hi, int gy, const feat (&fu)[V], const feat (&fm)[V], feat (&fd)[V],
                        const word (&botC)[NB][V], auto tp_tag) {
        constexpr int TP = decltype(tp_tag)::value;
        if (r + 1 < hi) {
            word C[NB][V];
            read_row(r + 1, C);
            feats(C, fd);
        } else {
            feats(botC, fd);
        }
        word o[NB][V];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            word ov[NB];
            Net::template eval<TP>(fu[v], fm[v], fd[v], gy & 1, ov);
#pragma unroll
            for (int p = 0; p < NB; ++p) o[p][v] = ov[p];
        }
        write_row(r, o);
    };
    // Evaluation and in-place write of row r from the three feature rows.
    auto eval_row = [&](int r, int gy, const feat (&fu)[V], const feat (&fm)[V], const feat (&fd)[V],
                        auto tp_tag) {
        constexpr int TP = decltype(tp_tag)::value;
        word o[NB][V];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            word ov[NB];
            Net::template eval<TP>(fu[v], fm[v], fd[v], gy & 1, ov);
#pragma unroll
            for (int p = 0; p < NB; ++p) o[p][v] = ov[p];
        }
        write_row(r, o);
    };

    auto step = [&](int t, auto tp_tag) {
        // the valid rows t .. TH-1-t, split evenly over the warps (the region
        // shrinks every step, so fixed bands would leave the edge warps idle)
        const int total = TH - 2 * t;
        const int base = total / WARPS, extra = total % WARPS;
        const int lo = t + warp * base + min(warp, extra);
        const int hi = lo + base + (warp < extra ? 1 : 0);
        word topC[NB][V], botC[NB][V];
        if (lo < hi) {
            read_row(lo - 1, topC);
            read_row(hi, botC);
        }
        __syncthreads();
        if (lo < hi) {
            feat fa[V], fb[V], fc[V];
            feats(topC, fa);
            {
                word C[NB][V];
                read_row(lo, C);
                feats(C, fb);
            }
            // global row of tile row lo, advanced incrementally (no division per row)
            int gy = (y0 - HY + lo) % Y;
            if (gy < 0) gy += Y;
            auto next_gy = [&](int g) { return g + 1 == Y ? 0 : g + 1; };
            int r = lo;
            // Three rows per trip; the feature buffers rotate by name, not by
            // copy.  The trip's three input rows (r+1 .. r+3) are read before
            // any of its in-place writes: they are the old values the writes replace,
            // and issuing them together keeps one shared-memory latency per
            // trip instead of one per row, with three rows of independent work.
            if constexpr (!HOIST) {
                for (; r + 3 <= hi; r += 3) {
                    row_body(r, hi, gy, fa, fb, fc, botC, tp_tag);
                    gy = next_gy(gy);
                    row_body(r + 1, hi, gy, fb, fc, fa, botC, tp_tag);
                    gy = next_gy(gy);
                    row_body(r + 2, hi, gy, fc, fa, fb, botC, tp_tag);
                    gy = next_gy(gy);
                }
            }
            // (Trips stop while r+3 is still inside the band, so all three
            // reads come from shared memory; the band's last rows go through
            // row_body below, which takes the saved row when it needs it.)
            for (; HOIST && r + 3 < hi; r += 3) {
                word C1[NB][V], C2[NB][V], C3[NB][V];
                read_row(r + 1, C1);
                read_row(r + 2, C2);
                read_row(r + 3, C3);
                feats(C1, fc);
                eval_row(r, gy, fa, fb, fc, tp_tag);
                gy = next_gy(gy);
                feats(C2, fa);
                eval_row(r + 1, gy, fb, fc, fa, tp_tag);
                gy = next_gy(gy);
                feats(C3, fb);
                eval_row(r + 2, gy, fc, fa, fb, tp_tag);
                gy = next_gy(gy);
            }
            if (r < hi) {
                row_body(r, hi, gy, fa, fb, fc, botC, tp_tag);
                gy = next_gy(gy);
                if (r + 1 < hi) {
                    row_body(r + 1, hi, gy, fb, fc, fa, botC, tp_tag);
                    gy = next_gy(gy);
                    if (r + 2 < hi) row_body(r + 2, hi, gy, fc, fa, fb, botC, tp_tag);
                }
            }
        }
        __syncthreads();
    };

    // Two steps per sweep: steps t and t+1 of a warp's band in one top-down
    // pass.  The band is cut from the rows step t+1 computes (t+1 .. TH-2-t);
    // step t's values of the band's rows and of the row on either side of it
    // are computed in registers from the old rows, two on either side of the
    // band read before the first barrier, and only step t+1's rows are written
    // back.  Per two steps a row is read from and written to shared memory
    // once instead of twice; the two step-t rows at each band edge are
    // computed by both neighbouring warps.  Rows t and TH-1-t keep their older
    // values, which no later step reads.  The values are the ones two single
    // steps give, halo words included.
    auto eval_words = [&](auto tp_tag, const feat (&fu)[V], const feat (&fm)[V], const feat (&fd)[V], int gy,
                          word (&o)[NB][V]) {
        constexpr int TP = decltype(tp_tag)::value;
#pragma unroll
        for (int v = 0; v < V; ++v) {
            word ov[NB];
            Net::template eval<TP>(fu[v], fm[v], fd[v], gy & 1, ov);
#pragma unroll
            for (int p = 0; p < NB; ++p) o[p][v] = ov[p];
        }
    };
    auto pair_step = [&](int t, auto tp_tag) {
        constexpr int TP = decltype(tp_tag)::value;
        const std::integral_constant<int, TP ^ 1> tp2{};
        const int total = TH - 2 * (t + 1);
        const int base = total / WARPS, extra = total % WARPS;
        const int lo = t + 1 + warp * base + min(warp, extra);
        const int hi = lo + base + (warp < extra ? 1 : 0);
        word A0[NB][V], A1[NB][V], B0[NB][V], B1[NB][V];  // old rows lo-2, lo-1, hi, hi+1
        if (lo < hi) {
            read_row(lo - 2, A0);
            read_row(lo - 1, A1);
            read_row(hi, B0);
            read_row(hi + 1, B1);
        }
        __syncthreads();
        if (lo < hi) {
            // E*: features of old rows; H*: features of step-t rows
            feat E0[V], E1[V], E2[V], H0[V], H1[V], H2[V];
            int gy = (y0 - HY + lo) % Y;  // global row of tile row r
            if (gy < 0) gy += Y;
            auto next_gy = [&](int g) { return g + 1 == Y ? 0 : g + 1; };
            const int gy_up = gy == 0 ? Y - 1 : gy - 1;
            {
                word o[NB][V];
                feats(A0, E0);
                feats(A1, E1);
                read_row(lo, o);
                feats(o, E2);
                eval_words(tp_tag, E0, E1, E2, gy_up, o);  // step t, row lo-1
                feats(o, H0);
                if (lo + 1 < hi) {
                    read_row(lo + 1, o);
                } else {
#pragma unroll
                    for (int p = 0; p < NB; ++p)
#pragma unroll
                        for (int v = 0; v < V; ++v) o[p][v] = B0[p][v];
                }
                feats(o, E0);
                eval_words(tp_tag, E1, E2, E0, gy, o);  // step t, row lo
                feats(o, H1);
            }
            // Output row r: old rows r, r+1 in Ea, Eb and r+2 in C; step-t
            // rows r-1, r in Ha, Hb.  Computes step t of row r+1 into Hc and
            // step t+1 of row r, written in place (old row r is no longer read).
            auto body = [&](int r, int g, const word (&C)[NB][V], const feat (&Ea)[V], const feat (&Eb)[V],
                            feat (&Ec)[V], const feat (&Ha)[V], const feat (&Hb)[V], feat (&Hc)[V]) {
                word o[NB][V];
                feats(C, Ec);
                eval_words(tp_tag, Ea, Eb, Ec, next_gy(g), o);
                feats(o, Hc);
                eval_words(tp2, Ha, Hb, Hc, g, o);
                write_row(r, o);
            };
            // old row x (lo <= x <= hi + 1): the band's own rows from shared
            // memory, the two below it from the rows saved before the barrier
            auto old_row = [&](int x, word (&C)[NB][V]) {
                if (x < hi) {
                    read_row(x, C);
                } else {
#pragma unroll
                    for (int p = 0; p < NB; ++p)
#pragma unroll
                        for (int v = 0; v < V; ++v) C[p][v] = x == hi ? B0[p][v] : B1[p][v];
                }
            };
            int r = lo;
            // feature sets rotate by name over a trip of three rows; the
            // trip's three old rows are read before any of its writes
            for (; r + 4 < hi; r += 3) {
                word C1[NB][V], C2[NB][V], C3[NB][V];
                read_row(r + 2, C1);
                read_row(r + 3, C2);
                read_row(r + 4, C3);
                body(r, gy, C1, E2, E0, E1, H0, H1, H2);
                gy = next_gy(gy);
                body(r + 1, gy, C2, E0, E1, E2, H1, H2, H0);
                gy = next_gy(gy);
                body(r + 2, gy, C3, E1, E2, E0, H2, H0, H1);
                gy = next_gy(gy);
            }
            // the band's last one to four rows
            auto tail = [&](int rr, int g, const feat (&Ea)[V], const feat (&Eb)[V], feat (&Ec)[V],
                            const feat (&Ha)[V], const feat (&Hb)[V], feat (&Hc)[V]) {
                word C[NB][V];
                old_row(rr + 2, C);
                body(rr, g, C, Ea, Eb, Ec, Ha, Hb, Hc);
            };
            if (r < hi) {
                tail(r, gy, E2, E0, E1, H0, H1, H2);
                gy = next_gy(gy);
                if (r + 1 < hi) {
                    tail(r + 1, gy, E0, E1, E2, H1, H2, H0);
                    gy = next_gy(gy);
                    if (r + 2 < hi) {
                        tail(r + 2, gy, E1, E2, E0, H2, H0, H1);
                        gy = next_gy(gy);
                        if (r + 3 < hi) tail(r + 3, gy, E2, E0, E1, H0, H1, H2);
                    }
                }
            }
        }
        __syncthreads();
    };

    int t = 1;
    if constexpr (PAIR) {
        for (; t + 1 <= k; t += 2) {
            if (((t0 + t - 1) & 1) == 0)
                pair_step(t, std::integral_constant<int, 0>{});
            else
                pair_step(t, std::integral_constant<int, 1>{});
        }
    }
    for (; t <= k; ++t) {
        if (((t0 + t - 1) & 1) == 0)
            step(t, std::integral_constant<int, 0>{});
        else
            step(t, std::integral_constant<int, 1>{});
    }

    // ---- store the interior
    for (int band = HY / R + warp; band < (TH - HY) / R; band += WARPS) {
        const int gy0 = y0 - HY + band * R;
        if (gy0 >= Y) continue;
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int s = lane * V + v;
            const int gx = x0 - 1 + s;
            if (s < 1 || s > TW - 2 || gx >= Xw) continue;
#pragma unroll
            for (int p = 0; p < NB; ++p) {
                word rows[R];
#pragma unroll
                for (int r = 0; r < R; ++r) rows[r] = at(p, band * R + r, s);
                store_word_rows<LAYOUT>(out.p[p], Xw, gy0 / R, gx, rows);
            }
        }
    }
}

template <class Net, int NB, int LAYOUT, int V, int WARPS, bool HOIST, bool PAIR = false>
__global__ void __launch_bounds__(WARPS * 32) temporal_kernel(plane_set in, plane_set out, int Xw, int Y, int t0,
                                                              int k, int TH, int HY) {
    temporal_tile<Net, NB, LAYOUT, V, WARPS, HOIST, LOAD_NC, PAIR>(in, out, Xw, Y, t0, k, TH, HY, blockIdx.x,
                                                                    blockIdx.y);
}

// ======================================================= batched temporal kernel
// Many independent grids of one rule, every round of every grid, in ONE
// persistent launch.  The work list holds an item per (grid, round, tile),
// ordered by round.  Resident CTAs claim items in list order from a device
// queue head; a grid's round r may start once all its tiles of round r - 1 are
// done, which each item checks against the grid's count of finished tiles:
//   * round r reads the buffer round r - 1 wrote (read after write), and
//   * writes the buffer round r - 1 read (write after read),
// so "every tile of round r - 1 finished" orders both.  A CTA only ever waits
// for items earlier in the list, which CTAs that are running have claimed, so
// the waits cannot deadlock whatever the number of resident CTAs.  Every wait
// is bounded; one that gives up counts in g_wait_timeouts and the item runs
// anyway, so the launch always ends.
//
// Each grid has its own planes (p[0] = a, p[1] = b), sizes and tile count.
// Items carry in their `steps` word: the step count (low 8 bits, at most the
// launch's halo HY), BATCH_FLIP_BUFFER (read p[parity ^ 1]), BATCH_FLIP_TIME
// (the first step number is t0 + 1; only the parity of a step number matters
// to the rules), and the item's round within the launch (bits 10 and up).
struct batch_grid_desc {
    plane_set p[2];
    int Xw, Y;
    int tiles;  // tiles of one round of this grid
    int pad_;
};

struct batch_item {
    int grid, tx, ty, steps;  // steps: count, flags and round (see above)
};

constexpr int BATCH_STEPS_MASK = 0xff;
constexpr int BATCH_FLIP_BUFFER = 1 << 8;
constexpr int BATCH_FLIP_TIME = 1 << 9;
constexpr int BATCH_ROUND_SHIFT = 10;
constexpr unsigned BATCH_WAIT_LIMIT = 1u << 24;  // polls with 64 ns sleeps: seconds, far above any round's time

__device__ __forceinline__ unsigned load_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// head: the launch's queue head; done[g]: finished tiles of grid g.  Both start
// at zero (the host clears them before the launch).  wait_limit: polls before
// a wait gives up (BATCH_WAIT_LIMIT in the library).  PAIR: tiles run two
// steps per sweep.
template <class Net, int NB, int LAYOUT, int V, int WARPS, bool PAIR>
__global__ void __launch_bounds__(WARPS * 32) temporal_batch_kernel(const batch_grid_desc* __restrict__ grids,
                                                                    const batch_item* __restrict__ items, int n_items,
                                                                    int parity, int t0, int TH, int HY,
                                                                    unsigned* head, unsigned* done,
                                                                    unsigned wait_limit) {
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(head, 1u);
        __syncthreads();
        const int i = s_item;
        if (i >= n_items) break;
        const batch_item it = items[i];
        const batch_grid_desc& g = grids[it.grid];
        const unsigned round = (unsigned)it.steps >> BATCH_ROUND_SHIFT;
        if (round > 0 && threadIdx.x == 0) {
            const unsigned need = round * (unsigned)g.tiles;
            unsigned polls = 0;
            while (load_acquire_gpu(done + it.grid) < need) {
                if (++polls >= wait_limit) {
                    atomicAdd(&g_wait_timeouts, 1u);
                    break;
                }
                __nanosleep(64);
            }
        }
        __syncthreads();
        const int src = parity ^ ((it.steps & BATCH_FLIP_BUFFER) ? 1 : 0);
        const int start = t0 + ((it.steps & BATCH_FLIP_TIME) ? 1 : 0);
        temporal_tile<Net, NB, LAYOUT, V, WARPS, true, LOAD_CG, PAIR>(g.p[src], g.p[src ^ 1], g.Xw, g.Y, start,
                                                                     it.steps & BATCH_STEPS_MASK, TH, HY, it.tx,
                                                                     it.ty);
        // publish the tile: every thread's stores are visible device-wide
        // before the count that releases the next round
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(done + it.grid, 1u);
        }
    }
}

}  // namespace cellato::b200

#endif  // CELLATO_B200_ENGINE_CUH
