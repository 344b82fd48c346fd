// Measured peak of the ALU pipe for the compute roofline of the temporal
// kernels: measurement infrastructure of bench.py and profile_case.py, built
// into its own library (_build/liblop3_rate.so) by __graft_entry__.build(),
// not part of the B200 library or its C ABI.  No counterpart in the reference.
//
// The temporal kernels run k steps per launch out of shared memory, so HBM
// bounds them only at small k; above that, they are bound by the integer/logic
// (ALU) pipe that executes their LOP3 networks, funnel shifts and compares.
// This kernel measures that pipe's throughput on the device it runs on: every
// thread keeps eight words and updates them with 128 `lop3.b32` per loop trip
// (alternately XOR3 and majority, each reading two other words, so no chain
// collapses and four to eight are independent at any time), at full occupancy
// on every SM.  The rate is LOP3 lane-operations per second: threads x trips x
// 128 / CUDA-event time of the launch (the loop's own counter and branch add
// under 3% more instructions, which are not counted).
#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int RATE_THREADS = 256;
constexpr int RATE_CTAS_PER_SM = 8;     // 2048 threads: the SM's full occupancy
constexpr int RATE_OPS_PER_TRIP = 128;  // 16 rounds x 8 words

template <int IMM>
__device__ __forceinline__ uint32_t lop3_op(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t d;
    asm volatile("lop3.b32 %0, %1, %2, %3, %4;" : "=r"(d) : "r"(a), "r"(b), "r"(c), "n"(IMM));
    return d;
}

__global__ void __launch_bounds__(RATE_THREADS) lop3_rate_kernel(int trips, uint32_t seed, uint32_t* sink) {
    const uint32_t t = blockIdx.x * RATE_THREADS + threadIdx.x;
    uint32_t v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = (seed ^ t) * (2u * j + 1u) + j;
    for (int i = 0; i < trips; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (u & 1)
                    v[j] = lop3_op<0xE8>(v[j], v[(j + 1) & 7], v[(j + 3) & 7]);  // majority
                else
                    v[j] = lop3_op<0x96>(v[j], v[(j + 1) & 7], v[(j + 3) & 7]);  // xor3
            }
        }
    }
    uint32_t r = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) r ^= v[j];
    if (r == seed) sink[t] = r;  // keeps the work observable; practically never taken
}

}  // namespace

extern "C" {

// Best LOP3 lane-operations per second of three timed launches on `stream`
// (a cudaStream_t) of the current device; synchronises the stream.  Returns a
// cudaError_t (0 on success).
int lop3_rate(double* lane_ops_per_second, void* stream) {
    if (!lane_ops_per_second) return (int)cudaErrorInvalidValue;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return (int)e;
    const int ctas = sms * RATE_CTAS_PER_SM;
    const size_t threads = (size_t)ctas * RATE_THREADS;
    uint32_t* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    e = cudaMalloc(&sink, threads * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    double best = 0.0;
    const int trips = 1024;  // about 2 ms per launch on a 148-SM part at 1.9 GHz
    if (e == cudaSuccess) {
        lop3_rate_kernel<<<ctas, RATE_THREADS, 0, s>>>(trips / 8, 0x2545F491u, sink);  // warm-up
        e = cudaGetLastError();
    }
    for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
        e = cudaEventRecord(e0, s);
        if (e == cudaSuccess) {
            lop3_rate_kernel<<<ctas, RATE_THREADS, 0, s>>>(trips, 0x2545F491u + rep, sink);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess && ms > 0.f) {
            const double rate = (double)threads * trips * RATE_OPS_PER_TRIP / (ms * 1e-3);
            if (rate > best) best = rate;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (sink) cudaFree(sink);
    if (e != cudaSuccess) return (int)e;
    *lane_ops_per_second = best;
    return 0;
}

}  // extern "C"
