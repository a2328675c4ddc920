// sort_markdup.cu - coordinate sort + Picard-style duplicate marking of a
// BAM tile and the gather of its records into coordinate order.
//
// Replaces gpu_sort_markdup (fq2bam-meth/src/linear_gpu_sort.mojo:24-560)
// and the record gather of _gather_perm_to_writer
// (fq2bam-meth/src/linear_gpu_fm.mojo:177-225).  The reference sorts with an
// 8-bit LSD radix of its own (eight histogram / scan / scatter rounds per
// key, each with a host round trip) and marks duplicates and gathers the
// records on the host.  Here everything stays in HBM:
//   - the three stable 64-bit key sorts (coordinate; dlo, then dhi carried
//     into that order) are LSD radix sorts of 8-bit digits carrying u32
//     record indices (radix_sort.cuh; digits that are equal in every key
//     are skipped); a stable LSD sort gives exactly the reference's order,
//     ties broken by record index;
//   - mark_dups_kernel: one thread per position of the duplicate-key order;
//     the first record of every run of equal (dhi, dlo) walks its run, picks
//     the best (highest score, then lowest pair id) and marks every record
//     of another pair (L409-466);
//   - the gather is a size pass + scan + one warp per output record that
//     copies the record and sets flag 0x400 on duplicates (_or_dup_flag,
//     L408-420).
#include <cub/device/device_scan.cuh>

#include <string>

#include "ma_internal.h"
#include "radix_sort.cuh"
#include "sort_markdup.h"

namespace ma {
namespace {

constexpr int THREADS = 256;
constexpr int GATHER_WARPS = 8;

void check_launch(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

size_t align256(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }

unsigned grid_for(uint64_t n) { return static_cast<unsigned>((n + THREADS - 1) / THREADS); }

__global__ void iota_kernel(uint32_t* idx, uint64_t n) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * THREADS + threadIdx.x;
    if (i < n) idx[i] = static_cast<uint32_t>(i);
}

// dhi carried into the dlo order (permute_u64_kernel, L130-138).
__global__ void permute_kernel(const uint64_t* src, const uint32_t* idx, uint64_t* dst, uint64_t n) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * THREADS + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}

// sdhi = dhi in duplicate-key order, merged = record indices in that order.
__global__ void mark_dups_kernel(const uint64_t* sdhi, const uint32_t* merged, const uint64_t* dlo,
                                 const uint32_t* score, const uint32_t* pair, uint32_t* is_dup, uint64_t n,
                                 unsigned long long* marked) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * THREADS + threadIdx.x;
    if (i >= n) return;
    const uint64_t h = sdhi[i];
    const uint64_t l = dlo[merged[i]];
    if (i > 0 && sdhi[i - 1] == h && dlo[merged[i - 1]] == l) return;  // not the first of its run
    uint64_t end = i + 1;
    while (end < n && sdhi[end] == h && dlo[merged[end]] == l) ++end;
    if (h == ~0ull) {  // unplaced records are never duplicates
        for (uint64_t j = i; j < end; ++j) is_dup[merged[j]] = 0;
        return;
    }
    uint32_t best_pair = pair[merged[i]], best_score = score[merged[i]];
    for (uint64_t j = i; j < end; ++j) {
        const uint32_t o = merged[j];
        const uint32_t sc = score[o], pid = pair[o];
        if (sc > best_score || (sc == best_score && pid < best_pair)) {
            best_score = sc;
            best_pair = pid;
        }
    }
    unsigned long long m = 0;
    for (uint64_t j = i; j < end; ++j) {
        const uint32_t o = merged[j];
        const uint32_t d = pair[o] != best_pair;
        is_dup[o] = d;
        m += d;
    }
    if (marked && m) atomicAdd(marked, m);
}

struct SortScratch {
    uint64_t* keys_out;
    uint64_t* key2;
    uint32_t* idx_a;
    uint32_t* idx_b;
    void* temp;
    size_t temp_bytes;
};

size_t radix_temp_bytes(uint64_t n) { return radix::scratch_bytes(n); }

SortScratch carve(void* scratch, size_t bytes, uint64_t n) {
    uint8_t* s = static_cast<uint8_t*>(scratch);
    SortScratch r;
    r.keys_out = reinterpret_cast<uint64_t*>(s);
    s += align256(n * 8);
    r.key2 = reinterpret_cast<uint64_t*>(s);
    s += align256(n * 8);
    r.idx_a = reinterpret_cast<uint32_t*>(s);
    s += align256(n * 4);
    r.idx_b = reinterpret_cast<uint32_t*>(s);
    s += align256(n * 4);
    r.temp = s;
    r.temp_bytes = bytes - (s - static_cast<uint8_t*>(scratch));
    return r;
}

int radix_sort(const SortScratch& sc, const uint64_t* keys, uint64_t* keys_out, const uint32_t* vals,
               uint32_t* vals_out, uint64_t n, cudaStream_t st) {
    if (sc.temp_bytes < radix::scratch_bytes(n)) fail(MA_ERR_INTERNAL, "radix sort scratch too small");
    const int k = radix::sort_pairs(keys, vals, keys_out, vals_out, n, sc.temp, 0, st);
    check_launch(cudaGetLastError(), "radix sort");
    return k;
}

// ---- gather -------------------------------------------------------------

// Record i of the sorted stream: its size, or 0 (and a status count) when
// its index, chunk or span is out of range.
__device__ __forceinline__ bool gather_source(const GatherDev& g, uint64_t i, const uint8_t*& src, uint32_t& len) {
    const uint32_t o = g.perm[i];
    if (o >= g.n) return false;
    const uint64_t r = g.rec[o];
    const uint64_t c = r >> 32, off = r & 0xffffffffull;
    len = g.len[o];
    if (c >= g.n_chunks || off + len > g.chunk_len[c]) return false;
    src = g.chunks[c] + off;
    return true;
}

__global__ void gather_sizes_kernel(GatherDev g, uint64_t* sizes) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * THREADS + threadIdx.x;
    unsigned bad = 0;
    if (i < g.n) {
        const uint32_t o = g.perm[i];
        uint32_t len = 0;
        if (o < g.n) len = g.len[o];
        sizes[i] = len;
        const uint8_t* src;
        uint32_t l2;
        bad = !gather_source(g, i, src, l2);
    }
    for (int k = 16; k > 0; k >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, k);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(&g.status[1], static_cast<unsigned long long>(bad));
}

__global__ void __launch_bounds__(GATHER_WARPS * 32) gather_records_kernel(GatherDev g, const uint64_t* ends) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t total = ends[g.n - 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) g.status[0] = total;
    if (total > g.cap) return;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * GATHER_WARPS + w; i < g.n;
         i += static_cast<uint64_t>(gridDim.x) * GATHER_WARPS) {
        const uint64_t start = i ? ends[i - 1] : 0;
        const uint64_t len = ends[i] - start;
        uint8_t* dst = g.out + start;
        const uint8_t* src = nullptr;
        uint32_t l2 = 0;
        const bool ok = gather_source(g, i, src, l2);
        const bool dup = ok && g.apply_dup && g.is_dup && g.is_dup[g.perm[i]] != 0;
        for (uint64_t k = lane; k < len; k += 32) {
            uint8_t v = ok ? src[k] : 0;
            if (k == 19 && dup) v |= 4;  // flag |= 0x400
            dst[k] = v;
        }
    }
}

}  // namespace

size_t sort_scratch_bytes(uint64_t n) {
    return 2 * align256(n * 8) + 2 * align256(n * 4) + align256(radix_temp_bytes(n));
}

int enqueue_sort_markdup(const SortDev& s, void* scratch, size_t scratch_bytes, cudaStream_t st) {
    const uint64_t n = s.n;
    const SortScratch sc = carve(scratch, scratch_bytes, n);
    int launches = 0;
    if (s.marked) check_launch(cudaMemsetAsync(s.marked, 0, sizeof(unsigned long long), st), "memset");
    // coordinate order (L469-525)
    iota_kernel<<<grid_for(n), THREADS, 0, st>>>(sc.idx_a, n);
    launches += 1 + radix_sort(sc, s.coord, sc.keys_out, sc.idx_a, s.perm, n, st);
    if (s.do_markdup) {
        // duplicate-key order: dlo, then dhi carried along (L311-360)
        iota_kernel<<<grid_for(n), THREADS, 0, st>>>(sc.idx_a, n);
        launches += 1 + radix_sort(sc, s.dlo, sc.keys_out, sc.idx_a, sc.idx_b, n, st);
        permute_kernel<<<grid_for(n), THREADS, 0, st>>>(s.dhi, sc.idx_b, sc.key2, n);
        uint32_t* merged = s.dup_perm ? s.dup_perm : sc.idx_a;
        launches += 1 + radix_sort(sc, sc.key2, sc.keys_out, sc.idx_b, merged, n, st);
        mark_dups_kernel<<<grid_for(n), THREADS, 0, st>>>(sc.keys_out, merged, s.dlo, s.score, s.pair, s.is_dup, n,
                                                          s.marked);
        launches += 1;
    } else {
        check_launch(cudaMemsetAsync(s.is_dup, 0, n * sizeof(uint32_t), st), "memset");
        if (s.dup_perm) {
            iota_kernel<<<grid_for(n), THREADS, 0, st>>>(s.dup_perm, n);
            ++launches;
        }
    }
    check_launch(cudaGetLastError(), "sort/markdup kernels");
    return launches;
}

size_t gather_scratch_bytes(uint64_t n) {
    size_t t = 0;
    cub::DeviceScan::InclusiveSum(nullptr, t, static_cast<const uint64_t*>(nullptr), static_cast<uint64_t*>(nullptr),
                                  static_cast<int64_t>(n));
    return 2 * align256(n * 8) + align256(t);
}

const uint64_t* gather_total_in_scratch(const void* scratch, uint64_t n) {
    return reinterpret_cast<const uint64_t*>(static_cast<const uint8_t*>(scratch) + align256(n * 8)) + (n - 1);
}

int enqueue_gather_layout(const GatherDev& g, void* scratch, size_t scratch_bytes, cudaStream_t st) {
    uint8_t* s = static_cast<uint8_t*>(scratch);
    uint64_t* sizes = reinterpret_cast<uint64_t*>(s);
    uint64_t* ends = reinterpret_cast<uint64_t*>(s + align256(g.n * 8));
    void* temp = s + 2 * align256(g.n * 8);
    size_t tb = scratch_bytes - 2 * align256(g.n * 8);
    gather_sizes_kernel<<<grid_for(g.n), THREADS, 0, st>>>(g, sizes);
    check_launch(cudaGetLastError(), "gather_sizes_kernel");
    check_launch(cub::DeviceScan::InclusiveSum(temp, tb, static_cast<const uint64_t*>(sizes), ends,
                                               static_cast<int64_t>(g.n), st),
                 "gather scan");
    return 3;
}

int enqueue_gather_records(const GatherDev& g, const void* scratch, int sm_count, cudaStream_t st) {
    const uint64_t* ends =
        reinterpret_cast<const uint64_t*>(static_cast<const uint8_t*>(scratch) + align256(g.n * 8));
    const uint64_t want = (g.n + GATHER_WARPS - 1) / GATHER_WARPS;
    const uint64_t cap = static_cast<uint64_t>(sm_count > 0 ? sm_count : 148) * 8;
    gather_records_kernel<<<static_cast<unsigned>(want < cap ? want : cap), GATHER_WARPS * 32, 0, st>>>(g, ends);
    check_launch(cudaGetLastError(), "gather_records_kernel");
    return 1;
}

}  // namespace ma
