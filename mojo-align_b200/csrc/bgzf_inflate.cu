// bgzf_inflate.cu - BGZF members inflated on the device (bgzf_inflate.cuh):
// one warp per member, its lane 0 decoding with the warp's Huffman tables in
// shared memory, a grid-stride loop over the members.
#include <string>

#include "bgzf_inflate.cuh"
#include "ma_internal.h"

namespace ma {
namespace {

constexpr int THREADS = 128;
constexpr int WARPS = THREADS / 32;

__global__ void __launch_bounds__(THREADS) bgzf_inflate_kernel(bgzf_inflate::Job j) {
    __shared__ inflate::Tables tables[WARPS];
    __shared__ uint32_t crc_tab[256];
    bgzf_inflate::crc_table(crc_tab, threadIdx.x, THREADS);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t nw = static_cast<uint64_t>(gridDim.x) * WARPS;
    for (uint64_t m = static_cast<uint64_t>(blockIdx.x) * WARPS + warp; m < j.n; m += nw)
        if (lane == 0) j.status[m] = bgzf_inflate::inflate_member(j, static_cast<uint32_t>(m), tables[warp], crc_tab);
}

void check_launch(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

int bgzf_inflate_enqueue(const bgzf_inflate::Job& j, int sm_count, cudaStream_t st) {
    if (!j.n) return 0;
    const uint64_t want = (j.n + WARPS - 1) / WARPS;
    const uint64_t cap = static_cast<uint64_t>(sm_count > 0 ? sm_count : 148) * 16;
    bgzf_inflate_kernel<<<static_cast<unsigned>(want < cap ? want : cap), THREADS, 0, st>>>(j);
    check_launch(cudaGetLastError(), "bgzf_inflate_kernel");
    return 1;
}

}  // namespace ma
