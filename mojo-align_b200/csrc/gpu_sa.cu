// gpu_sa.cu - suffix array of the BWT text on the GPU, for the index
// builder (bwa index's suffix sort; not on the mapping path).
//
// Prefix doubling: round 0 sorts all suffixes by their first 21 symbols
// packed 3 bits each (0 = sentinel / past the end); round r sorts by
// (rank of the first h symbols, rank of the h symbols after them).  Ranks
// are the sorted position of a group's first member.  Sorting uses CUB's
// device radix sort on packed 64-bit keys.
#include <cuda_runtime.h>

#include <cub/cub.cuh>
#include <vector>

#include "ma_internal.h"

namespace ma {
namespace {

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

__global__ void init_keys_kernel(const uint8_t* __restrict__ t, uint64_t n, uint64_t N, uint64_t* __restrict__ key,
                                 uint32_t* __restrict__ val) {
    uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= N) return;
    uint64_t k = 0;
    for (int j = 0; j < 21; ++j) {
        uint64_t p = i + j;
        k = (k << 3) | (p < n ? static_cast<uint64_t>(t[p]) + 1 : 0);
    }
    key[i] = k;
    val[i] = static_cast<uint32_t>(i);
}

__global__ void heads_kernel(const uint64_t* __restrict__ key, uint64_t N, uint32_t* __restrict__ head,
                             uint32_t* __restrict__ flag) {
    uint64_t j = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (j >= N) return;
    bool h = j == 0 || key[j] != key[j - 1];
    head[j] = h ? static_cast<uint32_t>(j) : 0u;
    flag[j] = h ? 1u : 0u;
}

__global__ void scatter_rank_kernel(const uint32_t* __restrict__ val, const uint32_t* __restrict__ head, uint64_t N,
                                    uint32_t* __restrict__ rank) {
    uint64_t j = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (j >= N) return;
    rank[val[j]] = head[j];
}

__global__ void pair_keys_kernel(const uint32_t* __restrict__ val, const uint32_t* __restrict__ rank, uint64_t N,
                                 uint64_t h, int nb, uint64_t* __restrict__ key) {
    uint64_t j = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (j >= N) return;
    uint64_t i = val[j];
    uint64_t second = i + h < N ? rank[i + h] : 0;
    key[j] = (static_cast<uint64_t>(rank[i]) << nb) | second;
}

unsigned grid_of(uint64_t n) { return static_cast<unsigned>((n + 255) / 256); }

struct Mem {
    std::vector<void*> ptrs;
    ~Mem() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    T* alloc(size_t n) {
        void* p = nullptr;
        ck(cudaMalloc(&p, n * sizeof(T) + 16), "cudaMalloc (suffix sort)");
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
};

}  // namespace

std::vector<uint32_t> suffix_array_gpu(const uint8_t* text, uint64_t n, int device) {
    const uint64_t N = n + 1;
    if (N >= 0x7FFFFFFFull) fail(MA_ERR_UNSUPPORTED, "GPU suffix sort handles texts below 2^31 symbols");
    ck(cudaSetDevice(device), "cudaSetDevice");
    cudaStream_t st;
    ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
    std::vector<uint32_t> sa(N);
    try {
        Mem m;
        uint8_t* d_t = m.alloc<uint8_t>(n);
        uint64_t* k0 = m.alloc<uint64_t>(N);
        uint64_t* k1 = m.alloc<uint64_t>(N);
        uint32_t* v0 = m.alloc<uint32_t>(N);
        uint32_t* v1 = m.alloc<uint32_t>(N);
        uint32_t* rank = m.alloc<uint32_t>(N);
        uint32_t* head = m.alloc<uint32_t>(N);
        uint32_t* flag = m.alloc<uint32_t>(N);
        uint32_t* head2 = m.alloc<uint32_t>(N);
        unsigned long long* d_cnt = m.alloc<unsigned long long>(1);
        ck(cudaMemcpyAsync(d_t, text, n, cudaMemcpyHostToDevice, st), "H2D text");
        cub::DoubleBuffer<uint64_t> keys(k0, k1);
        cub::DoubleBuffer<uint32_t> vals(v0, v1);
        const int items = static_cast<int>(N);
        size_t tb_sort = 0, tb_scan = 0, tb_sum = 0;
        ck(cub::DeviceRadixSort::SortPairs(nullptr, tb_sort, keys, vals, items, 0, 64, st), "sort temp");
        ck(cub::DeviceScan::InclusiveScan(nullptr, tb_scan, head, head2, cub::Max(), items, st), "scan temp");
        ck(cub::DeviceReduce::Sum(nullptr, tb_sum, flag, d_cnt, items, st), "sum temp");
        size_t tb = std::max(tb_sort, std::max(tb_scan, tb_sum));
        void* temp = m.alloc<uint8_t>(tb);
        init_keys_kernel<<<grid_of(N), 256, 0, st>>>(d_t, n, N, keys.Current(), vals.Current());
        ck(cudaGetLastError(), "init_keys");
        ck(cub::DeviceRadixSort::SortPairs(temp, tb, keys, vals, items, 0, 63, st), "sort");
        int nb = 1;
        while ((1ull << nb) < N) ++nb;
        uint64_t h = 21;
        for (int round = 0; round < 40; ++round) {
            heads_kernel<<<grid_of(N), 256, 0, st>>>(keys.Current(), N, head, flag);
            ck(cub::DeviceScan::InclusiveScan(temp, tb, head, head2, cub::Max(), items, st), "scan");
            scatter_rank_kernel<<<grid_of(N), 256, 0, st>>>(vals.Current(), head2, N, rank);
            ck(cub::DeviceReduce::Sum(temp, tb, flag, d_cnt, items, st), "sum");
            unsigned long long distinct = 0;
            ck(cudaMemcpyAsync(&distinct, d_cnt, sizeof distinct, cudaMemcpyDeviceToHost, st), "D2H");
            ck(cudaStreamSynchronize(st), "suffix sort");
            if (distinct == N) break;
            if (h >= N) fail(MA_ERR_INTERNAL, "suffix sort did not converge");
            pair_keys_kernel<<<grid_of(N), 256, 0, st>>>(vals.Current(), rank, N, h, nb, keys.Current());
            ck(cudaGetLastError(), "pair_keys");
            ck(cub::DeviceRadixSort::SortPairs(temp, tb, keys, vals, items, 0, 2 * nb, st), "sort");
            h *= 2;
        }
        ck(cudaMemcpyAsync(sa.data(), vals.Current(), N * 4, cudaMemcpyDeviceToHost, st), "D2H sa");
        ck(cudaStreamSynchronize(st), "suffix sort");
    } catch (...) {
        cudaStreamDestroy(st);
        throw;
    }
    cudaStreamDestroy(st);
    return sa;
}

}  // namespace ma
