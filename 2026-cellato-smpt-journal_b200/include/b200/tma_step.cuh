// Single-step kernel fed by the tensor memory accelerator (TMA): one time step
// per launch, the grid streamed through shared-memory tiles with halos.
//
// Work split.  A CTA owns a strip of SW linear words and a range of memory
// rows [m0, m1): a memory row is one row of the linear layout, or one tile row
// of the tiled layouts (R = 4 or 8 cell rows).  Each consumer warp owns 32 x V
// consecutive words of the strip -- V per lane (tma_default_v), so that lane
// shuffles and per-word overheads are shared by V words -- and walks the range top to bottom with a rolling
// window of three cell rows' features in registers, loading and featurising a
// group of rows at a time (a tile row's R rows, or up to four linear rows) so
// that independent work overlaps.  SW = 32 x V x consumer warps is 128 words
// for V = 1 (four warps) and 256 for V = 2 (four warps) or 4 (two warps); one
// more warp is the producer.
//
// Staging.  A ring of TMA_STAGES shared-memory stages, each BR memory rows of
// every plane:
//   * the strip itself: one cp.async.bulk.tensor box per plane and stage
//     (2-D for the linear layout, 3-D {4 tiles, words, rows} for the tiled
//     ones), completing on the stage's "full" mbarrier with expect_tx;
//   * the word to the left and to the right of the strip in each of those rows
//     (wrapped on the torus): cp.async by the producer's 32 lanes, completing
//     on the same barrier (cp.async.mbarrier.arrive.noinc);
//   * the memory row above m0 and below m1 (wrapped) with their halo words:
//     cp.async into an area of their own, on the "edge" barrier.
// Every block a consumer reads with vector loads starts on a 16-byte boundary.
// Consumers arrive on the stage's "empty" barrier once they have read it, and
// the producer refills it.  No box is ever loaded from another GPU's memory
// and none uses multicast.
//
// Shapes: Xw (linear words per row) a multiple of SW and at least BR memory
// rows.  Every global word the kernel touches is inside the planes: rows and
// words wrap by index, boxes start inside the grid, and the last box of a range
// may run past the grid's last row, where the TMA writes zeros that are never
// read.
//
// Every wait is bounded.  A consumer whose wait gives up counts it in
// g_wait_timeouts and leaves; the producer, whose copies write this CTA's
// shared memory, waits (bounded) for everything it issued before it leaves.
#ifndef CELLATO_B200_TMA_STEP_CUH
#define CELLATO_B200_TMA_STEP_CUH

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include "b200/engine.cuh"

namespace cellato::b200 {

constexpr int TMA_STAGES = 3;
constexpr unsigned TMA_WAIT_LIMIT = 1u << 22;
constexpr int TMA_STAGE_BUDGET = 8 * 1024;  // bytes of strip data per stage (all planes)

// Default words per lane of the TMA step kernel for a rule of NB planes in a
// layout: 4 for one-plane rules, 2 for two or three planes, else 1; and 1 in
// the 8-row tiled layout, whose eight rows per word already give each lane
// enough independent work.  Measured on B200 (fractions of the HBM peak): Game
// of Life on the linear layout at 32768^2, 0.65 at four words per lane against
// 0.60 at two and 0.49 at one; WireWorld 0.62 (tiled W64) and 0.79 (linear)
// at its defaults; two words per lane in the 8-row layout cost registers and
// occupancy (Greenberg-Hastings 0.52 against 0.69).  Callers may ask for
// another width per call.
template <int NB, int LAYOUT>
constexpr int tma_default_v() {
    return LAYOUT == LAYOUT_TILED8 ? 1 : (NB == 1 ? 4 : (NB <= 3 ? 2 : 1));
}

// Geometry and shared-memory layout of the kernel for (NB, LAYOUT, V).
template <int NB, int LAYOUT, int V>
struct tma_geom {
    static constexpr int WARPS = V == 4 ? 2 : 4;           // consumer warps
    static constexpr int SW = 32 * V * WARPS;              // strip width in linear words
    static constexpr int L = LAYOUT == LAYOUT_LINEAR ? 1 : (LAYOUT == LAYOUT_TILED4 ? 4 : 8);  // u32 per word
    static constexpr int G = LAYOUT == LAYOUT_LINEAR ? (V >= 4 ? 1 : 4 / V) : 1;  // memory rows per group
    static constexpr int row_bytes = NB * SW * L * 4;
    static constexpr int BR_raw = TMA_STAGE_BUDGET / row_bytes / G * G;
    static constexpr int BR = BR_raw < G ? G : (BR_raw > 32 ? 32 : BR_raw);  // memory rows per stage
    static constexpr int plane_block = BR * SW * L;        // u32 of one plane in one stage
    static constexpr int ring = TMA_STAGES * NB * plane_block;
    // halo words, rounded up to 16 bytes so the edge rows after them stay aligned
    static constexpr int halo = (TMA_STAGES * NB * BR * 2 * L + 3) / 4 * 4;
    // [strip][left halo][right halo], 16-byte multiple: the strip is read with
    // vector loads
    static constexpr int edge_row = (SW * L + 2 * L + 3) / 4 * 4;
    static constexpr int edge = NB * 2 * edge_row;
    static constexpr int words = ring + halo + edge;
    static constexpr size_t bytes = (size_t)words * 4 + (2 * TMA_STAGES + 1) * 8;
    static constexpr int threads = (WARPS + 1) * 32;
    static_assert(SW <= 256, "a TMA box holds at most 256 words per row");
};

struct tma_maps {
    CUtensorMap m[MAX_PLANES];
};

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool tma_wait(unsigned long long* bar, unsigned parity) {
    for (unsigned it = 0; it < TMA_WAIT_LIMIT; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_addr(dst)), "l"(src), "n"(BYTES)
                     : "memory");
}
__device__ __forceinline__ void cp_async_arrive_noinc(unsigned long long* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

// Copies linear word gx of memory row m of every plane (L u32 each) to dst
// (stride `stride` u32 between planes) with cp.async.
template <int NB, int L>
__device__ __forceinline__ void copy_word(const plane_set& in, int Xw, int m, int gx, unsigned* dst, int stride) {
#pragma unroll
    for (int p = 0; p < NB; ++p) {
        const word* src = in.p[p] + ((size_t)m * Xw + gx) * L;
        if constexpr (L == 1) {
            cp_async<4>(dst + p * stride, src);
        } else {
#pragma unroll
            for (int q = 0; q < L; q += 4) cp_async<16>(dst + p * stride + q, src + q);
        }
    }
}

// The R cell-row words of one linear word at s (L u32 in shared memory).
template <int LAYOUT>
__device__ __forceinline__ void rows_of(const unsigned* s, word (&r)[band_rows<LAYOUT>()]) {
    if constexpr (LAYOUT == LAYOUT_LINEAR) {
        r[0] = s[0];
    } else if constexpr (LAYOUT == LAYOUT_TILED4) {
        const uint4 t = *reinterpret_cast<const uint4*>(s);
        word a = t.x, b = t.y, c = t.z, d = t.w;
        transpose4x4(a, b, c, d);
        r[0] = a, r[1] = b, r[2] = c, r[3] = d;
    } else {
        const uint4 t01 = *reinterpret_cast<const uint4*>(s), t23 = *reinterpret_cast<const uint4*>(s + 4);
        word l0 = t01.x, l1 = t01.z, l2 = t23.x, l3 = t23.z;
        word h0 = t01.y, h1 = t01.w, h2 = t23.y, h3 = t23.w;
        transpose4x4(l0, l1, l2, l3);
        transpose4x4(h0, h1, h2, h3);
        r[0] = l0, r[1] = l1, r[2] = l2, r[3] = l3, r[4] = h0, r[5] = h1, r[6] = h2, r[7] = h3;
    }
}

// A lane's V consecutive linear words at s: R cell rows each.
template <int LAYOUT, int V>
__device__ __forceinline__ void lane_rows(const unsigned* s, word (&r)[band_rows<LAYOUT>()][V]) {
    if constexpr (LAYOUT == LAYOUT_LINEAR && V == 4) {
        const uint4 q = *reinterpret_cast<const uint4*>(s);
        r[0][0] = q.x, r[0][1] = q.y, r[0][2] = q.z, r[0][3] = q.w;
    } else if constexpr (LAYOUT == LAYOUT_LINEAR && V == 2) {
        const uint2 q = *reinterpret_cast<const uint2*>(s);
        r[0][0] = q.x, r[0][1] = q.y;
    } else {
        constexpr int L = LAYOUT == LAYOUT_LINEAR ? 1 : (LAYOUT == LAYOUT_TILED4 ? 4 : 8);
#pragma unroll
        for (int v = 0; v < V; ++v) {
            word t[band_rows<LAYOUT>()];
            rows_of<LAYOUT>(s + v * L, t);
#pragma unroll
            for (int i = 0; i < band_rows<LAYOUT>(); ++i) r[i][v] = t[i];
        }
    }
}

template <class Net, int NB, int LAYOUT, int V, int TP>
__global__ void __launch_bounds__(tma_geom<NB, LAYOUT, V>::threads)
    tma_step_kernel(const __grid_constant__ tma_maps maps, plane_set in, plane_set out, int Xw, int M,
                    int rows_per_cta) {
    using S = tma_geom<NB, LAYOUT, V>;
    constexpr int L = S::L, BR = S::BR, R = band_rows<LAYOUT>(), G = S::G, WARPS = S::WARPS, SW = S::SW;
    using feat = typename Net::feat;
    extern __shared__ __align__(1024) unsigned tma_sm[];
    unsigned* ring = tma_sm;
    unsigned* halo = tma_sm + S::ring;
    unsigned* edge = halo + S::halo;
    auto* full = reinterpret_cast<unsigned long long*>(tma_sm + S::words);
    unsigned long long* empty = full + TMA_STAGES;
    unsigned long long* edge_bar = empty + TMA_STAGES;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x0 = blockIdx.x * SW;
    const int m0 = blockIdx.y * rows_per_cta;
    const int m1 = min(M, m0 + rows_per_cta);
    const int nchunks = (m1 - m0 + BR - 1) / BR;
    if (threadIdx.x == 0) {
        for (int s = 0; s < TMA_STAGES; ++s) {
            mbar_init(&full[s], 1 + 32);     // the producer's expect_tx arrival + its 32 lanes' cp.async
            mbar_init(&empty[s], WARPS);
        }
        mbar_init(edge_bar, 32);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (m0 >= m1) return;

    if (warp == WARPS) {
        // ---------------- producer
        const int xl = (x0 + Xw - 1) % Xw, xr = (x0 + SW) % Xw;
        // the rows above and below the range, with their halo words
        for (int e = 0; e < 2; ++e) {
            const int m = e == 0 ? (m0 + M - 1) % M : m1 % M;
            unsigned* row = edge + e * S::edge_row;
            for (int j = lane; j < SW + 2; j += 32) {  // strip words, then the left and right halo
                const int gx = j < SW ? x0 + j : (j == SW ? xl : xr);
                copy_word<NB, L>(in, Xw, m, gx, row + j * L, 2 * S::edge_row);
            }
        }
        cp_async_arrive_noinc(edge_bar);
        bool ok = true;
        int issued = 0;
        for (int c = 0; c < nchunks; ++c) {
            const int s = c % TMA_STAGES;
            if (c >= TMA_STAGES && !tma_wait(&empty[s], (unsigned)(c / TMA_STAGES - 1) & 1u)) {
                ok = false;
                break;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            const int mr = m0 + c * BR;
            if (lane == 0) {
                mbar_expect_tx(&full[s], (unsigned)(NB * S::plane_block * 4));
#pragma unroll
                for (int p = 0; p < NB; ++p) {
                    unsigned* dst = ring + (s * NB + p) * S::plane_block;
                    if constexpr (LAYOUT == LAYOUT_LINEAR)
                        tma_load_2d(dst, &maps.m[p], x0, mr, &full[s]);
                    else
                        tma_load_3d(dst, &maps.m[p], 0, x0, mr, &full[s]);
                }
            }
            // halo words: lane -> (row, side); rows past the range are not needed
            for (int j = lane; j < 2 * BR; j += 32) {
                const int r = j >> 1, side = j & 1;
                if (mr + r < m1)
                    copy_word<NB, L>(in, Xw, mr + r, side ? xr : xl,
                                     halo + ((s * NB) * BR + r) * 2 * L + side * L, BR * 2 * L);
            }
            cp_async_arrive_noinc(&full[s]);
            issued = c + 1;
        }
        if (!ok && lane == 0) atomicAdd(&g_wait_timeouts, 1u);
        // every copy this warp issued lands before the CTA's shared memory is released
        asm volatile("cp.async.wait_all;" ::: "memory");
        for (int c = max(0, issued - TMA_STAGES); c < issued; ++c)
            tma_wait(&full[c % TMA_STAGES], (unsigned)(c / TMA_STAGES) & 1u);
        return;
    }

    // ---------------- consumers: lane owns linear words lw .. lw + V - 1 of the strip
    const int lw = (warp * 32 + lane) * V;
    const int gx = x0 + lw;
    const bool use_l = lane == 0, use_r = lane == 31;
    // one memory row: R cell rows of this lane's words and of the edge words
    auto load_row = [&](const unsigned* strip, int strip_stride, const unsigned* lh, const unsigned* rh,
                        int halo_stride, word (&C)[R][NB][V], word (&Lw)[R][NB], word (&Rw)[R][NB]) {
#pragma unroll
        for (int p = 0; p < NB; ++p) {
            const unsigned* sp = strip + p * strip_stride;
            word t[R][V];
            lane_rows<LAYOUT, V>(sp + lw * L, t);
#pragma unroll
            for (int i = 0; i < R; ++i)
#pragma unroll
                for (int v = 0; v < V; ++v) C[i][p][v] = t[i][v];
            word e[R];
            if (use_l) {
                rows_of<LAYOUT>(warp > 0 ? sp + (lw - 1) * L : lh + p * halo_stride, e);
#pragma unroll
                for (int i = 0; i < R; ++i) Lw[i][p] = e[i];
            }
            if (use_r) {
                rows_of<LAYOUT>(warp < WARPS - 1 ? sp + (lw + V) * L : rh + p * halo_stride, e);
#pragma unroll
                for (int i = 0; i < R; ++i) Rw[i][p] = e[i];
            }
        }
    };
    auto feats_of = [&](const word (&C)[NB][V], const word (&Lw)[NB], const word (&Rw)[NB], feat (&f)[V]) {
        row_feats<Net, NB, V>(C, Lw, Rw, use_l, use_r, f);
    };

    // Rolling window: up / mid / dn are the features of three consecutive cell
    // rows; the output row is mid's.  Output row i-1 of a memory row is made
    // while its input row i is read, so res holds a memory row's outputs with
    // compile-time row indices and is stored once its last row is made (when
    // the next memory row's first row is read).
    feat up[V], mid[V], dn[V];
    word res[R][NB][V];
    auto emit = [&](int y, int i) {  // output cell row y into res[i]
#pragma unroll
        for (int v = 0; v < V; ++v) {
            word o[NB];
            Net::template eval<TP>(up[v], mid[v], dn[v], y & 1, o);
#pragma unroll
            for (int p = 0; p < NB; ++p) res[i][p][v] = o[p];
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
            up[v] = mid[v];
            mid[v] = dn[v];
        }
    };
    auto store = [&](int m) {  // the R output rows of memory row m
#pragma unroll
        for (int p = 0; p < NB; ++p) {
            if constexpr (LAYOUT == LAYOUT_LINEAR) {
                word rr[1][V];
#pragma unroll
                for (int v = 0; v < V; ++v) rr[0][v] = res[0][p][v];
                store_lane<LAYOUT_LINEAR, V>(out.p[p], Xw, m, gx, rr);
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    word rr[R];
#pragma unroll
                    for (int q = 0; q < R; ++q) rr[q] = res[q][p][v];
                    store_word_rows<LAYOUT>(out.p[p], Xw, m, gx + v, rr);
                }
            }
        }
    };
    auto set = [&](feat (&dst)[V], const feat (&src)[V]) {
#pragma unroll
        for (int v = 0; v < V; ++v) dst[v] = src[v];
    };
    if (!tma_wait(edge_bar, 0)) {
        if (lane == 0) atomicAdd(&g_wait_timeouts, 1u);
        return;
    }
    {
        word C[R][NB][V], Lw[R][NB] = {}, Rw[R][NB] = {};
        const unsigned* row = edge;  // the row above the range: its last cell row
        load_row(row, 2 * S::edge_row, row + SW * L, row + (SW + 1) * L, 2 * S::edge_row, C, Lw, Rw);
        feats_of(C[R - 1], Lw[R - 1], Rw[R - 1], up);
    }
    for (int c = 0; c < nchunks; ++c) {
        const int s = c % TMA_STAGES;
        if (!tma_wait(&full[s], (unsigned)(c / TMA_STAGES) & 1u)) {
            if (lane == 0) atomicAdd(&g_wait_timeouts, 1u);
            return;
        }
        const int mr = m0 + c * BR;
        const unsigned* strip = ring + (s * NB) * S::plane_block;
        for (int r = 0; r < BR && mr + r < m1; r += G) {
            if constexpr (G > 1) {
                if (mr + r + G <= m1) {
                    // G linear rows at once: independent loads and features, then the window
                    word C[G][NB][V], Lw[G][NB] = {}, Rw[G][NB] = {};
#pragma unroll
                    for (int g = 0; g < G; ++g) {
                        word c1[1][NB][V], l1[1][NB] = {}, r1[1][NB] = {};
                        const unsigned* h = halo + ((s * NB) * BR + r + g) * 2 * L;
                        load_row(strip + (r + g) * SW * L, S::plane_block, h, h + L, BR * 2 * L, c1, l1, r1);
#pragma unroll
                        for (int p = 0; p < NB; ++p) {
#pragma unroll
                            for (int v = 0; v < V; ++v) C[g][p][v] = c1[0][p][v];
                            Lw[g][p] = l1[0][p];
                            Rw[g][p] = r1[0][p];
                        }
                    }
                    feat f[G][V];
#pragma unroll
                    for (int g = 0; g < G; ++g) feats_of(C[g], Lw[g], Rw[g], f[g]);
                    const int m = mr + r;
                    if (m == m0) {
                        set(mid, f[0]);
                    } else {
                        set(dn, f[0]);
                        emit(m - 1, 0);
                        store(m - 1);
                    }
#pragma unroll
                    for (int g = 1; g < G; ++g) {
                        set(dn, f[g]);
                        emit(m + g - 1, 0);
                        store(m + g - 1);
                    }
                    continue;
                }
            }
            // one memory row at a time (tiled layouts; a linear range's last rows)
            for (int q = r; q < r + G && mr + q < m1; ++q) {
                const int m = mr + q;
                word C[R][NB][V], Lw[R][NB] = {}, Rw[R][NB] = {};
                const unsigned* h = halo + ((s * NB) * BR + q) * 2 * L;
                load_row(strip + q * SW * L, S::plane_block, h, h + L, BR * 2 * L, C, Lw, Rw);
                if (m == m0) {
                    feats_of(C[0], Lw[0], Rw[0], mid);
                } else {
                    feats_of(C[0], Lw[0], Rw[0], dn);
                    emit(m * R - 1, R - 1);
                    store(m - 1);
                }
#pragma unroll
                for (int i = 1; i < R; ++i) {
                    feats_of(C[i], Lw[i], Rw[i], dn);
                    emit(m * R + i - 1, i - 1);
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
    {
        word C[R][NB][V], Lw[R][NB] = {}, Rw[R][NB] = {};
        const unsigned* row = edge + S::edge_row;  // the row below the range: its first cell row
        load_row(row, 2 * S::edge_row, row + SW * L, row + (SW + 1) * L, 2 * S::edge_row, C, Lw, Rw);
        feats_of(C[0], Lw[0], Rw[0], dn);
        emit(m1 * R - 1, R - 1);
        store(m1 - 1);
    }
}

// ---------------------------------------------------------------- host side
// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// Tensor maps of nb planes for the TMA step kernel: linear planes as 2-D
// {Xw words, M rows} of u32, tiled planes as 3-D {4 tiles, Xw linear words, M
// tile rows} of u32 (4-row tiles) or u64 (8-row tiles); boxes of one stage.
template <int NB, int LAYOUT, int V>
inline cudaError_t make_tma_maps(const plane_set& ps, int Xw, int M, tma_maps& maps) {
    auto enc = tensor_map_encoder();
    if (!enc) return cudaErrorNotSupported;
    constexpr int BR = tma_geom<NB, LAYOUT, V>::BR, SW = tma_geom<NB, LAYOUT, V>::SW;
    for (int p = 0; p < NB; ++p) {
        CUresult r;
        if constexpr (LAYOUT == LAYOUT_LINEAR) {
            const cuuint64_t dims[2] = {(cuuint64_t)Xw, (cuuint64_t)M};
            const cuuint64_t strides[1] = {(cuuint64_t)Xw * 4};
            const cuuint32_t box[2] = {SW, BR};
            const cuuint32_t es[2] = {1, 1};
            r = enc(&maps.m[p], CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, ps.p[p], dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        } else {
            constexpr bool t8 = LAYOUT == LAYOUT_TILED8;
            const cuuint64_t esz = t8 ? 8 : 4;
            const cuuint64_t dims[3] = {4, (cuuint64_t)Xw, (cuuint64_t)M};
            const cuuint64_t strides[2] = {4 * esz, (cuuint64_t)Xw * 4 * esz};
            const cuuint32_t box[3] = {4, SW, BR};
            const cuuint32_t es[3] = {1, 1, 1};
            r = enc(&maps.m[p], t8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, ps.p[p], dims,
                    strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        }
        if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    }
    return cudaSuccess;
}

}  // namespace cellato::b200

#endif  // CELLATO_B200_TMA_STEP_CUH
