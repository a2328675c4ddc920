// radix_sort.cuh - stable LSD radix sort of (u64 key, u32 value) pairs on
// the device, 8-bit digits, for the coordinate and duplicate-key orders of
// sort_markdup.cu.
//
// A pass over digit d is three kernels:
//   rs_hist     one block per tile of TILE keys: the tile's digit counts,
//               stored digit-major (count[d][tile]);
//   rs_scan     one block per digit: exclusive prefix of count[d][*] over the
//               tiles, and the digit's total;
//   rs_scatter  one block per tile: the digit bases (exclusive scan of the
//               totals), each key's rank among the tile's keys of its digit
//               (keys in tile order: rounds of 256 consecutive keys, a warp
//               ranks its 32 with __match_any_sync and the warps' counts are
//               added in shared memory), then key and value to
//               base[d] + prefix[d][tile] + rank.
// Ranks follow the input order, so every pass is stable and the whole sort
// gives the order of a stable sort by the full key (ties by input position),
// the order of the reference's own 8-bit LSD radix.
//
// Digits whose bits are the same in every key move nothing and are skipped:
// rs_bits ORs key ^ key[0] over the input, and rs_plan (one thread) lays out
// each pass's source and destination so that the last active pass writes the
// caller's output buffers (or rs_copy copies the input there when no digit
// varies).  The plan lives in device memory: nothing waits on the host, and a
// stream capture of the sort is a plain kernel sequence.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace ma {
namespace radix {

constexpr int THREADS = 256;
constexpr int ROUNDS = 16;                 // keys per thread
constexpr int TILE = THREADS * ROUNDS;     // 4096 keys per tile
constexpr int WARPS = THREADS / 32;
constexpr int PASSES = 8;                  // 64-bit keys, 8-bit digits

struct Plan {
    const uint64_t* src_k[PASSES];
    const uint32_t* src_v[PASSES];
    uint64_t* dst_k[PASSES];
    uint32_t* dst_v[PASSES];
    int active[PASSES];
    int copy_input;  // no digit varies: the input is copied to the output
};

__global__ void rs_bits(const uint64_t* __restrict__ keys, uint64_t n, unsigned long long* __restrict__ bits) {
    const uint64_t k0 = keys[0];
    uint64_t v = 0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(THREADS) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * THREADS)
        v |= keys[i] ^ k0;
    for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicOr(bits, static_cast<unsigned long long>(v));
}

// Pass p reads the input or the previous active pass's output; the active
// passes alternate between `tmp` and `out` so that the last one writes `out`.
__global__ void rs_plan(const unsigned long long* __restrict__ bits, const uint64_t* in_k, const uint32_t* in_v,
                        uint64_t* out_k, uint32_t* out_v, uint64_t* tmp_k, uint32_t* tmp_v, Plan* plan) {
    int n_active = 0;
    for (int p = 0; p < PASSES; ++p) n_active += ((*bits >> (8 * p)) & 0xFF) != 0;
    const uint64_t* sk = in_k;
    const uint32_t* sv = in_v;
    int left = n_active;
    for (int p = 0; p < PASSES; ++p) {
        const int a = ((*bits >> (8 * p)) & 0xFF) != 0;
        plan->active[p] = a;
        plan->src_k[p] = sk;
        plan->src_v[p] = sv;
        // with `left` active passes to go (this one included), an odd count
        // writes the output, an even one the temporary
        uint64_t* dk = (left & 1) ? out_k : tmp_k;
        uint32_t* dv = (left & 1) ? out_v : tmp_v;
        plan->dst_k[p] = dk;
        plan->dst_v[p] = dv;
        if (a) {
            sk = dk;
            sv = dv;
            --left;
        }
    }
    plan->copy_input = n_active == 0;
}

__global__ void rs_copy(const Plan* __restrict__ plan, const uint64_t* __restrict__ in_k,
                        const uint32_t* __restrict__ in_v, uint64_t* __restrict__ out_k, uint32_t* __restrict__ out_v,
                        uint64_t n) {
    if (!plan->copy_input) return;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(THREADS) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * THREADS) {
        out_k[i] = in_k[i];
        out_v[i] = in_v[i];
    }
}

__global__ void __launch_bounds__(THREADS) rs_hist(const Plan* __restrict__ plan, int p, uint64_t n,
                                                  uint32_t n_tiles, uint32_t* __restrict__ count) {
    if (!plan->active[p]) return;
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t* keys = plan->src_k[p];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * TILE;
    const int sh = 8 * p;
#pragma unroll 4
    for (int j = 0; j < ROUNDS; ++j) {
        const uint64_t i = base + static_cast<uint64_t>(j) * THREADS + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> sh) & 0xFF], 1u);
    }
    __syncthreads();
    count[static_cast<uint64_t>(threadIdx.x) * n_tiles + blockIdx.x] = h[threadIdx.x];
}

// One block per digit: count[d][*] becomes its exclusive prefix over the
// tiles; total[d] the digit's count.
__global__ void __launch_bounds__(THREADS) rs_scan(const Plan* __restrict__ plan, int p, uint32_t n_tiles,
                                                  uint32_t* __restrict__ count, uint64_t* __restrict__ total) {
    if (!plan->active[p]) return;
    __shared__ uint64_t part[THREADS];
    uint32_t* c = count + static_cast<uint64_t>(blockIdx.x) * n_tiles;
    const uint32_t per = (n_tiles + THREADS - 1) / THREADS;
    const uint32_t a = threadIdx.x * per;
    const uint32_t b = a + per < n_tiles ? a + per : n_tiles;
    uint64_t s = 0;
    for (uint32_t i = a; i < b; ++i) s += c[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < THREADS; o <<= 1) {  // inclusive scan of the parts
        const uint64_t v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint64_t run = part[threadIdx.x] - s;
    for (uint32_t i = a; i < b; ++i) {
        const uint32_t v = c[i];
        c[i] = static_cast<uint32_t>(run);  // a tile prefix stays below n <= 2^32
        run += v;
    }
    if (threadIdx.x == THREADS - 1) total[blockIdx.x] = part[THREADS - 1];
}

__global__ void __launch_bounds__(THREADS) rs_scatter(const Plan* __restrict__ plan, int p, uint64_t n,
                                                     uint32_t n_tiles, const uint32_t* __restrict__ count,
                                                     const uint64_t* __restrict__ total) {
    if (!plan->active[p]) return;
    __shared__ uint64_t dbase[256];      // where digit d's keys of this tile start
    __shared__ uint32_t run[256];        // keys of digit d in the tile's earlier rounds
    __shared__ uint32_t wc[WARPS][256];  // this round's count of digit d per warp
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    // exclusive scan of the digit totals
    {
        const uint64_t v = total[t];
        dbase[t] = v;
        __syncthreads();
        for (int o = 1; o < 256; o <<= 1) {
            const uint64_t u = t >= o ? dbase[t - o] : 0;
            __syncthreads();
            dbase[t] += u;
            __syncthreads();
        }
        const uint64_t excl = dbase[t] - v + count[static_cast<uint64_t>(t) * n_tiles + blockIdx.x];
        __syncthreads();
        dbase[t] = excl;
        run[t] = 0;
        for (int k = 0; k < WARPS; ++k) wc[k][t] = 0;
        __syncthreads();
    }
    const uint64_t* sk = plan->src_k[p];
    const uint32_t* sv = plan->src_v[p];
    uint64_t* dk = plan->dst_k[p];
    uint32_t* dv = plan->dst_v[p];
    const int sh = 8 * p;
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * TILE;
    const unsigned lt = (1u << lane) - 1u;
    for (int j = 0; j < ROUNDS; ++j) {
        const uint64_t i = base + static_cast<uint64_t>(j) * THREADS + t;
        const bool valid = i < n;
        uint64_t key = 0;
        uint32_t val = 0;
        int d = 256;  // past the end: ranks among nothing
        if (valid) {
            key = sk[i];
            val = sv[i];
            d = static_cast<int>((key >> sh) & 0xFF);
        }
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
        const uint32_t in_warp = __popc(peers & lt);
        if (valid && in_warp == 0) wc[w][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            uint32_t before = run[d] + in_warp;
            for (int k = 0; k < w; ++k) before += wc[k][d];
            const uint64_t o = dbase[d] + before;
            if (o < n) {  // always true; the check keeps a wrong count from writing past the end
                dk[o] = key;
                dv[o] = val;
            }
        }
        __syncthreads();
        uint32_t add = 0;
        for (int k = 0; k < WARPS; ++k) {
            add += wc[k][t];
            wc[k][t] = 0;
        }
        run[t] += add;
        __syncthreads();
    }
}

inline uint32_t tiles_for(uint64_t n) { return static_cast<uint32_t>((n + TILE - 1) / TILE); }

// Device scratch of a sort of n pairs.
inline size_t scratch_bytes(uint64_t n) {
    auto a256 = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
    const uint64_t nt = tiles_for(n ? n : 1);
    return a256(n * 8) + a256(n * 4) + a256(256 * nt * 4) + a256(256 * 8) + a256(sizeof(Plan)) + a256(8);
}

// Sorts (in_k, in_v) into (out_k, out_v); n >= 1.  Returns the kernels
// enqueued.
inline int sort_pairs(const uint64_t* in_k, const uint32_t* in_v, uint64_t* out_k, uint32_t* out_v, uint64_t n,
                      void* scratch, int sm_count, cudaStream_t st) {
    auto a256 = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
    const uint32_t nt = tiles_for(n);
    uint8_t* s = static_cast<uint8_t*>(scratch);
    uint64_t* tmp_k = reinterpret_cast<uint64_t*>(s);
    s += a256(n * 8);
    uint32_t* tmp_v = reinterpret_cast<uint32_t*>(s);
    s += a256(n * 4);
    uint32_t* count = reinterpret_cast<uint32_t*>(s);
    s += a256(256 * static_cast<size_t>(nt) * 4);
    uint64_t* total = reinterpret_cast<uint64_t*>(s);
    s += a256(256 * 8);
    Plan* plan = reinterpret_cast<Plan*>(s);
    s += a256(sizeof(Plan));
    unsigned long long* bits = reinterpret_cast<unsigned long long*>(s);
    cudaMemsetAsync(bits, 0, 8, st);
    const unsigned grid = static_cast<unsigned>(sm_count > 0 ? sm_count * 4 : 592);
    rs_bits<<<grid, THREADS, 0, st>>>(in_k, n, bits);
    rs_plan<<<1, 1, 0, st>>>(bits, in_k, in_v, out_k, out_v, tmp_k, tmp_v, plan);
    rs_copy<<<grid, THREADS, 0, st>>>(plan, in_k, in_v, out_k, out_v, n);
    for (int p = 0; p < PASSES; ++p) {
        rs_hist<<<nt, THREADS, 0, st>>>(plan, p, n, nt, count);
        rs_scan<<<256, THREADS, 0, st>>>(plan, p, nt, count, total);
        rs_scatter<<<nt, THREADS, 0, st>>>(plan, p, n, nt, count, total);
    }
    return 3 + 3 * PASSES;
}

}  // namespace radix
}  // namespace ma
