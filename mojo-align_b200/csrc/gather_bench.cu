// gather_bench.cu - measured random-gather roofline for the seed kernel.
//
// The seed/extend kernel's memory traffic is dominated by independent
// random reads of whole 32-byte Occ lines.  This kernel issues uniformly
// random, independent loads of `line_bytes` (32 or 64) aligned lines over a
// buffer of a chosen size, several lines in flight per thread, and reports
// the achieved bytes/s: the ceiling a perfect random-line gather reaches on
// this GPU, from HBM (buffer >> L2) or from L2 (buffer << 126 MB).
#include <cuda_runtime.h>

#include <string>

#include "ma_device.cuh"
#include "ma_internal.h"

namespace ma {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

template <int LINE>
__global__ void __launch_bounds__(256) gather_kernel(const uint4* __restrict__ buf, uint64_t line_mask,
                                                     uint32_t iters, uint64_t seed, uint32_t* __restrict__ sink) {
    constexpr int V = LINE / 16;  // uint4 per line
    constexpr int INFLIGHT = 8;
    const uint64_t tid = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    uint64_t state = mix64(seed ^ (tid * 0x9E3779B97F4A7C15ull)) | 1;
    uint32_t acc = 0;
    for (uint32_t it = 0; it < iters; it += INFLIGHT) {
        uint4 v[INFLIGHT][V];
#pragma unroll
        for (int j = 0; j < INFLIGHT; ++j) {
            state ^= state << 13;  // xorshift64
            state ^= state >> 7;
            state ^= state << 17;
            const uint4* p = buf + (state & line_mask) * V;
#pragma unroll
            for (int q = 0; q < V; ++q) v[j][q] = __ldg(p + q);
        }
#pragma unroll
        for (int j = 0; j < INFLIGHT; ++j)
#pragma unroll
            for (int q = 0; q < V; ++q) acc ^= v[j][q].x ^ v[j][q].y ^ v[j][q].z ^ v[j][q].w;
    }
    if (acc == 0x12345678u) sink[0] = acc;  // keeps the loads live
}

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

// Returns GB/s (1e9 bytes/s) of random line gathers.
double run_gather_bench(uint64_t buffer_bytes, int line_bytes, uint64_t n_loads, int sm_count, cudaStream_t st) {
    if (line_bytes != 32 && line_bytes != 64) fail(MA_ERR_ARG, "line_bytes must be 32 or 64");
    if (buffer_bytes < 1024) fail(MA_ERR_ARG, "buffer too small");
    uint64_t n_lines = 1;  // a power of two, at most buffer_bytes / line_bytes
    while (n_lines * 2 * line_bytes <= buffer_bytes) n_lines *= 2;
    void* buf = nullptr;
    uint32_t* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double gbps = 0;
    try {
        ck(cudaMalloc(&buf, n_lines * line_bytes), "cudaMalloc gather buffer");
        ck(cudaMalloc(&sink, 4), "cudaMalloc sink");
        ck(cudaMemsetAsync(buf, 0x5A, n_lines * line_bytes, st), "memset");
        ck(cudaEventCreate(&e0), "event");
        ck(cudaEventCreate(&e1), "event");
        const int block = 256;
        const uint64_t threads = static_cast<uint64_t>(sm_count) * 8 * block;  // 8 blocks per SM
        uint32_t iters = static_cast<uint32_t>((n_loads + threads - 1) / threads);
        iters = (iters + 7) & ~7u;
        const unsigned grid = static_cast<unsigned>(threads / block);
        auto launch = [&](uint64_t seed) {
            if (line_bytes == 32)
                gather_kernel<32><<<grid, block, 0, st>>>(static_cast<const uint4*>(buf), n_lines - 1, iters, seed, sink);
            else
                gather_kernel<64><<<grid, block, 0, st>>>(static_cast<const uint4*>(buf), n_lines - 1, iters, seed, sink);
        };
        launch(1);  // warm-up
        ck(cudaEventRecord(e0, st), "record");
        const int reps = 3;
        for (int r = 0; r < reps; ++r) launch(2 + r);
        ck(cudaEventRecord(e1, st), "record");
        ck(cudaEventSynchronize(e1), "gather bench");
        ck(cudaGetLastError(), "gather launch");
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        const double bytes = static_cast<double>(threads) * iters * line_bytes * reps;
        gbps = bytes / (ms * 1e-3) / 1e9;
    } catch (...) {
        cudaFree(buf);
        cudaFree(sink);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        throw;
    }
    cudaFree(buf);
    cudaFree(sink);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return gbps;
}

}  // namespace ma
