// Helpers shared by the C ABI translation units (capi.cu, batch.cu, noalloc.cu,
// grid_ops.cu, serve.cu).
#ifndef CELLATO_B200_CAPI_INTERNAL_HPP
#define CELLATO_B200_CAPI_INTERNAL_HPP

#include <cuda_runtime.h>

#include <cstdint>

#include "b200/rule_kernels.cuh"

namespace cellato::b200::capi {
int fail(int status, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
const rule_ops* ops_of(int rule);
int rule_count();  // rule ids in use (built-in + registered)
int internal_layout(int layout, int word_bits);
int band_height(int layout, int word_bits);
int check_dims(int layout, int word_bits, int X, int Y);
int make_sets(const rule_ops* ops, void* const* a, void* const* b, plane_set& pa, plane_set& pb);
int default_tile_rows(const rule_ops* ops, int R, int k, int V, int interior = 128);
// grid_ops.cu: stream-ordered checksum (16 device uint64) and random fill
int enqueue_checksum(const rule_ops* ops, int layout, int word_bits, const plane_set& ps, int X, int Y,
                     unsigned long long* out, cudaStream_t s);
int enqueue_fill_random(int layout, int word_bits, int nb, const plane_set& ps, int X, int Y, unsigned long long seed,
                        const uint32_t* thresholds, int n_thresholds, cudaStream_t s);
}  // namespace cellato::b200::capi

#endif
