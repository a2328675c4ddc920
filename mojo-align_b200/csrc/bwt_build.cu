// bwt_build.cu - the BWT and the sampled suffix array of a 2-bit text on
// the GPU, for the index builder (the job of `bwa index`; not on the
// mapping path).  Texts of any length up to 2^35 symbols whose working set
// fits HBM (a 3.1 Gbp genome's bwa-meth text is 12.4 G symbols).
//
// Suffixes are sorted in batches by bucket (their first 10 symbols), so
// that one batch's keys and positions fit HBM whatever the text length:
//   1. one pass counts the suffixes of every bucket; consecutive buckets are
//      grouped into batches of at most `batch` suffixes;
//   2. per batch, one pass over the text selects the batch's suffixes with
//      a 64-bit key (their first 29 symbols, past the end reading as the
//      smallest symbol, then how many of the 29 are real, 0..29), sorted by
//      a radix sort: of two suffixes whose windows read alike, the one that
//      ends sooner is smaller, as with the sentinel;
//   3. suffixes with equal keys are refined 29 symbols deeper at a time
//      (a suffix that has ended has key 0), ordered within the tie group by
//      a second, stable sort on the group; groups shrink until no two keys
//      are equal (two suffixes still tied have the same symbols and the same
//      length so far, so they part before either ends);
//   4. the batch's rows get their BWT symbol (2 bits per row) and, every
//      sa_intv rows, their SA sample.
// Then the bwa .bwt layout (128-position blocks of counts + 8 words, most
// significant symbol first, the sentinel row removed) is assembled on the
// device and copied back with the samples.  All loops are bounded: a
// refinement that outlasts the text length raises an error.
#include <cuda_runtime.h>

#include <algorithm>
#include <cub/cub.cuh>
#include <vector>

#include "ma_internal.h"

namespace ma {

namespace {

constexpr int BUCKET_SYMS = 10;  // batching buckets: 4^10
constexpr int KEY_SYMS = 29;     // symbols per sort key
constexpr uint64_t EVEN = 0x5555555555555555ull;

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

unsigned grid_of(uint64_t n, unsigned block = 256) {
    uint64_t g = (n + block - 1) / block;
    if (g > 0x7FFFFFFFull) g = 0x7FFFFFFFull;
    return static_cast<unsigned>(g ? g : 1);
}

__device__ __forceinline__ uint64_t reverse_fields(uint64_t x) {
    const uint64_t y = __brevll(x);
    return ((y >> 1) & EVEN) | ((y & EVEN) << 1);
}

// Key of the suffix at i: symbols i .. i+28 in bits 63..6 (first symbol
// most significant, 2 bits each; past the end of the text they read as 0),
// bit 5 zero, and in bits 4..0 how many of the 29 are in the text
// (min(n - i, 29)).  A position at or past the end (an ended suffix) has
// key 0.  T holds the text LSB first, 32 symbols per word, zero past n, one
// spare word.
__device__ __forceinline__ uint64_t suffix_key(const uint64_t* __restrict__ T, uint64_t n, uint64_t i) {
    if (i >= n) return 0;
    const uint64_t w = i >> 5;
    const int sh = static_cast<int>(i & 31) * 2;
    const uint64_t lo = __ldg(T + w), hi = __ldg(T + w + 1);
    const uint64_t win = sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
    const uint64_t real = n - i < KEY_SYMS ? n - i : KEY_SYMS;
    return (reverse_fields(win) & ~((1ull << 6) - 1)) | real;
}

__device__ __forceinline__ uint32_t bucket_of(uint64_t key) {
    return static_cast<uint32_t>(key >> (64 - 2 * BUCKET_SYMS));
}

__device__ __forceinline__ int text_sym(const uint64_t* __restrict__ T, uint64_t i) {
    return static_cast<int>((__ldg(T + (i >> 5)) >> (2 * (i & 31))) & 3);
}

__global__ void bucket_count_kernel(const uint64_t* __restrict__ T, uint64_t n,
                                    unsigned long long* __restrict__ counts) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n; i += stride)
        atomicAdd(counts + bucket_of(suffix_key(T, n, i)), 1ull);
}

// The suffixes of buckets [blo, bhi): key and position, appended in any
// order (one atomic per warp).  The loop is warp-uniform.
__global__ void select_kernel(const uint64_t* __restrict__ T, uint64_t n, uint32_t blo, uint32_t bhi,
                              uint64_t* __restrict__ keys, uint64_t* __restrict__ pos, uint64_t cap,
                              unsigned long long* __restrict__ cursor) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const int lane = threadIdx.x & 31;
    for (uint64_t base = blockIdx.x * static_cast<uint64_t>(blockDim.x) + (threadIdx.x & ~31u); base < n;
         base += stride) {
        const uint64_t i = base + lane;
        uint64_t key = 0;
        bool take = false;
        if (i < n) {
            key = suffix_key(T, n, i);
            const uint32_t b = bucket_of(key);
            take = b >= blo && b < bhi;
        }
        const unsigned m = __ballot_sync(0xFFFFFFFFu, take);
        if (!m) continue;
        unsigned long long at = 0;
        if (lane == 0) at = atomicAdd(cursor, static_cast<unsigned long long>(__popc(m)));
        at = __shfl_sync(0xFFFFFFFFu, at, 0);
        if (take) {
            const uint64_t slot = at + __popc(m & ((1u << lane) - 1));
            if (slot < cap) {
                keys[slot] = key;
                pos[slot] = i;
            }
        }
    }
}

// flag[j] = 1 when key[j] equals a neighbour's key (a tie to refine).
__global__ void tie_flag_kernel(const uint64_t* __restrict__ key, int64_t m, uint8_t* __restrict__ flag) {
    const int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (j >= m) return;
    const uint64_t k = key[j];
    flag[j] = (j > 0 && key[j - 1] == k) || (j + 1 < m && key[j + 1] == k);
}

// Residue set-up from the tied batch indices U[r]: positions, and the head
// of each tie group (the first r of a run of equal keys) as head ? r : 0.
__global__ void residue_init_kernel(const uint32_t* __restrict__ U, int64_t u, const uint64_t* __restrict__ key,
                                    const uint64_t* __restrict__ pos, uint64_t* __restrict__ rpos,
                                    uint32_t* __restrict__ head) {
    const int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (r >= u) return;
    rpos[r] = pos[U[r]];
    head[r] = (r == 0 || key[U[r]] != key[U[r - 1]]) ? static_cast<uint32_t>(r) : 0u;
}

__global__ void refine_key_kernel(const uint64_t* __restrict__ T, uint64_t n, const uint64_t* __restrict__ rpos,
                                  int64_t u, uint64_t depth, uint64_t* __restrict__ rkey, uint32_t* __restrict__ idx) {
    const int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (r >= u) return;
    rkey[r] = suffix_key(T, n, rpos[r] + depth);
    idx[r] = static_cast<uint32_t>(r);
}

__global__ void gather_u32_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ idx, int64_t u,
                                  uint32_t* __restrict__ dst) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t < u) dst[t] = src[idx[t]];
}

// After the (group, key) order idx: the positions go back into the batch at
// the tied slots U (a group's slots, in order), with their refinement keys.
__global__ void refine_apply_kernel(const uint64_t* __restrict__ T, uint64_t n, const uint32_t* __restrict__ idx,
                                    int64_t u, uint64_t depth, const uint32_t* __restrict__ U,
                                    const uint64_t* __restrict__ rpos, uint64_t* __restrict__ pos,
                                    uint64_t* __restrict__ rpos2, uint64_t* __restrict__ rkey2) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t >= u) return;
    const uint64_t p = rpos[idx[t]];
    pos[U[t]] = p;
    rpos2[t] = p;
    rkey2[t] = suffix_key(T, n, p + depth);
}

// The ties that remain: equal group and equal refinement key.
__global__ void refine_ties_kernel(const uint32_t* __restrict__ g, const uint64_t* __restrict__ k, int64_t u,
                                   uint8_t* __restrict__ flag) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t >= u) return;
    flag[t] = (t > 0 && g[t - 1] == g[t] && k[t - 1] == k[t]) || (t + 1 < u && g[t + 1] == g[t] && k[t + 1] == k[t]);
}

// The next residue: the tied elements sel[r] (ascending), their slots and
// positions, and the head of each new group as head ? r : 0.
__global__ void residue_next_kernel(const uint32_t* __restrict__ sel, int64_t u2, const uint32_t* __restrict__ U,
                                    const uint64_t* __restrict__ rpos2, const uint64_t* __restrict__ rkey2,
                                    const uint32_t* __restrict__ g, uint32_t* __restrict__ U2,
                                    uint64_t* __restrict__ rpos, uint32_t* __restrict__ head) {
    const int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (r >= u2) return;
    const uint32_t t = sel[r];
    U2[r] = U[t];
    rpos[r] = rpos2[t];
    bool h = r == 0;
    if (!h) {
        const uint32_t tp = sel[r - 1];
        h = g[tp] != g[t] || rkey2[tp] != rkey2[t];
    }
    head[r] = h ? static_cast<uint32_t>(r) : 0u;
}

// Rows row0 + j of a sorted batch: BWT symbol (2 bits per row, least
// significant first within a u32; the sentinel row is marked in *primary)
// and every intv-th row's SA sample.
__global__ void emit_kernel(const uint64_t* __restrict__ T, const uint64_t* __restrict__ pos, int64_t m,
                            uint64_t row0, uint64_t intv, uint32_t* __restrict__ rowsym,
                            uint64_t* __restrict__ samples, unsigned long long* __restrict__ primary) {
    const int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (j >= m) return;
    const uint64_t row = row0 + static_cast<uint64_t>(j);
    const uint64_t p = pos[j];
    if (p == 0) *primary = row;
    else atomicOr(rowsym + (row >> 4), static_cast<uint32_t>(text_sym(T, p - 1)) << (2 * (row & 15)));
    if (row % intv == 0) samples[row / intv - 1] = p;
}

struct Cnt4 {
    unsigned long long c[4];
};
struct Cnt4Sum {
    __host__ __device__ Cnt4 operator()(const Cnt4& a, const Cnt4& b) const {
        Cnt4 r;
        for (int i = 0; i < 4; ++i) r.c[i] = a.c[i] + b.c[i];
        return r;
    }
};

// bwa block b: stored positions [128b, 128b+128) (row = k + (k >= primary))
// as 8 words, most significant symbol first, and the block's symbol counts.
__global__ void bwa_words_kernel(const uint32_t* __restrict__ rowsym, uint64_t n, uint64_t primary,
                                 uint64_t n_blocks, uint32_t* __restrict__ bwt, Cnt4* __restrict__ cnt) {
    const uint64_t b = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (b >= n_blocks) return;
    Cnt4 c{{0, 0, 0, 0}};
    for (int w = 0; w < 8; ++w) {
        const uint64_t k0 = b * 128 + 16 * w;
        if (k0 >= n) break;
        uint32_t word = 0;
        for (int i = 0; i < 16; ++i) {
            const uint64_t k = k0 + i;
            if (k >= n) break;
            const uint64_t row = k + (k >= primary ? 1 : 0);
            const uint32_t s = (rowsym[row >> 4] >> (2 * (row & 15))) & 3;
            word |= s << (2 * (15 - i));
            c.c[s]++;
        }
        bwt[b * 16 + 8 + w] = word;
    }
    cnt[b] = c;
}

__global__ void bwa_counts_kernel(const Cnt4* __restrict__ before, uint64_t n_blocks, uint32_t* __restrict__ bwt) {
    const uint64_t b = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (b >= n_blocks) return;
    const Cnt4 c = before[b];
    for (int s = 0; s < 4; ++s) {
        bwt[b * 16 + 2 * s] = static_cast<uint32_t>(c.c[s]);
        bwt[b * 16 + 2 * s + 1] = static_cast<uint32_t>(c.c[s] >> 32);
    }
}

struct DevMem {
    std::vector<void*> ptrs;
    ~DevMem() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    T* alloc(uint64_t n) {
        void* p = nullptr;
        ck(cudaMalloc(&p, n * sizeof(T) + 16), "cudaMalloc (BWT construction)");
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    void release(void* p) {
        for (auto& q : ptrs)
            if (q == p) {
                cudaFree(q);
                q = nullptr;
            }
    }
};

}  // namespace

BwtBuild bwt_build_gpu(const std::vector<uint64_t>& text_words, uint64_t n, int sa_intv, uint64_t batch_limit,
                       int device) {
    if (n == 0) fail(MA_ERR_ARG, "empty text");
    if (n > (1ull << 35) - 2) fail(MA_ERR_UNSUPPORTED, "the GPU BWT construction handles texts below 2^35 symbols");
    if (text_words.size() < n / 32 + 2) fail(MA_ERR_INTERNAL, "text words short of the text length");
    ck(cudaSetDevice(device), "cudaSetDevice");
    cudaStream_t st;
    ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
    BwtBuild out;
    try {
        DevMem m;
        const uint64_t n_words = text_words.size();
        uint64_t* T = m.alloc<uint64_t>(n_words);
        ck(cudaMemcpyAsync(T, text_words.data(), n_words * 8, cudaMemcpyHostToDevice, st), "H2D text");
        const uint64_t rows = n + 1;
        const uint64_t intv = static_cast<uint64_t>(sa_intv);
        const uint64_t n_sa = (n + intv) / intv;
        uint32_t* rowsym = m.alloc<uint32_t>((rows + 15) / 16);
        uint64_t* samples = m.alloc<uint64_t>(n_sa);
        unsigned long long* d_small = m.alloc<unsigned long long>(4);  // [0] primary, [1] cursor, [2] count
        ck(cudaMemsetAsync(rowsym, 0, ((rows + 15) / 16) * 4, st), "memset");
        ck(cudaMemsetAsync(d_small, 0, 32, st), "memset");
        // row 0 is the sentinel suffix: SA[0] = n, BWT symbol T[n-1]
        {
            std::vector<uint32_t> first(1, 0);
            const uint64_t last = (text_words[(n - 1) >> 5] >> (2 * ((n - 1) & 31))) & 3;
            first[0] = static_cast<uint32_t>(last);
            ck(cudaMemcpyAsync(rowsym, first.data(), 4, cudaMemcpyHostToDevice, st), "H2D row 0");
            ck(cudaStreamSynchronize(st), "row 0");
        }

        // 1. bucket sizes
        const uint64_t n_buckets = 1ull << (2 * BUCKET_SYMS);
        unsigned long long* d_counts = m.alloc<unsigned long long>(n_buckets);
        ck(cudaMemsetAsync(d_counts, 0, n_buckets * 8, st), "memset");
        bucket_count_kernel<<<148 * 16, 256, 0, st>>>(T, n, d_counts);
        ck(cudaGetLastError(), "bucket_count");
        std::vector<unsigned long long> counts(n_buckets);
        ck(cudaMemcpyAsync(counts.data(), d_counts, n_buckets * 8, cudaMemcpyDeviceToHost, st), "D2H counts");
        ck(cudaStreamSynchronize(st), "bucket counts");
        m.release(d_counts);

        // batch size: what fits next to the text, the rows and the samples
        // (keys and positions double-buffered: 32 B; tie residue up to
        // 60 B; radix-sort temporaries), at most 2^30 suffixes
        size_t f = 0, tot = 0;
        ck(cudaMemGetInfo(&f, &tot), "cudaMemGetInfo");
        uint64_t cap = static_cast<uint64_t>(static_cast<double>(f) * 0.85) / 112;
        cap = std::min<uint64_t>(cap, 1ull << 30);
        if (batch_limit) cap = std::min<uint64_t>(cap, batch_limit);
        uint64_t biggest = 0;
        for (auto c : counts) biggest = std::max<uint64_t>(biggest, c);
        if (biggest > cap)
            fail(MA_ERR_NOMEM, "a suffix bucket of " + std::to_string(biggest) + " suffixes exceeds the batch of " +
                                   std::to_string(cap));
        cap = std::max<uint64_t>(cap, 1);
        const uint64_t M = std::min<uint64_t>(cap, n);  // largest batch allocated
        uint64_t* k0 = m.alloc<uint64_t>(M);
        uint64_t* k1 = m.alloc<uint64_t>(M);
        uint64_t* p0 = m.alloc<uint64_t>(M);
        uint64_t* p1 = m.alloc<uint64_t>(M);
        uint8_t* flag = m.alloc<uint8_t>(M);
        uint32_t* U = m.alloc<uint32_t>(M);
        uint32_t* U2 = m.alloc<uint32_t>(M);
        uint32_t* sel = m.alloc<uint32_t>(M);
        uint32_t* head = m.alloc<uint32_t>(M);
        uint32_t* grp = m.alloc<uint32_t>(M);
        uint32_t* ga = m.alloc<uint32_t>(M);
        uint32_t* gb = m.alloc<uint32_t>(M);
        uint32_t* ia = m.alloc<uint32_t>(M);
        uint32_t* ib = m.alloc<uint32_t>(M);
        uint64_t* rpos = m.alloc<uint64_t>(M);
        uint64_t* ka = m.alloc<uint64_t>(M);
        uint64_t* kb = m.alloc<uint64_t>(M);
        uint64_t* rpos2 = m.alloc<uint64_t>(M);
        uint64_t* rkey2 = m.alloc<uint64_t>(M);
        const int Mi = static_cast<int>(M);
        size_t tb = 0, t1 = 0;
        {
            cub::DoubleBuffer<uint64_t> kk(k0, k1), pp(p0, p1);
            ck(cub::DeviceRadixSort::SortPairs(nullptr, t1, kk, pp, Mi, 0, 64, st), "temp");
            tb = std::max(tb, t1);
            cub::DoubleBuffer<uint64_t> rk(ka, kb);
            cub::DoubleBuffer<uint32_t> ix(ia, ib);
            ck(cub::DeviceRadixSort::SortPairs(nullptr, t1, rk, ix, Mi, 0, 64, st), "temp");
            tb = std::max(tb, t1);
            cub::DoubleBuffer<uint32_t> gg(ga, gb);
            ck(cub::DeviceRadixSort::SortPairs(nullptr, t1, gg, ix, Mi, 0, 32, st), "temp");
            tb = std::max(tb, t1);
            ck(cub::DeviceSelect::Flagged(nullptr, t1, cub::CountingInputIterator<uint32_t>(0), flag, U, d_small + 2,
                                          Mi, st), "temp");
            tb = std::max(tb, t1);
            ck(cub::DeviceScan::InclusiveScan(nullptr, t1, head, grp, cub::Max(), Mi, st), "temp");
            tb = std::max(tb, t1);
        }
        void* temp = m.alloc<uint8_t>(tb);

        // 2-4. batches of consecutive buckets
        uint64_t row0 = 1, done_suffixes = 0;
        uint32_t b = 0;
        while (b < n_buckets) {
            uint32_t e = b;
            uint64_t cnt = 0;
            while (e < n_buckets && cnt + counts[e] <= cap) cnt += counts[e++];
            if (cnt == 0) {
                b = e;
                continue;
            }
            const int mi = static_cast<int>(cnt);
            ck(cudaMemsetAsync(d_small + 1, 0, 8, st), "memset");
            select_kernel<<<148 * 8, 256, 0, st>>>(T, n, b, e, k0, p0, cnt, d_small + 1);
            ck(cudaGetLastError(), "select");
            cub::DoubleBuffer<uint64_t> kk(k0, k1), pp(p0, p1);
            ck(cub::DeviceRadixSort::SortPairs(temp, tb, kk, pp, mi, 0, 64, st), "sort");
            uint64_t* key = kk.Current();
            uint64_t* pos = pp.Current();
            // refinement of ties, 29 symbols deeper per round
            tie_flag_kernel<<<grid_of(cnt), 256, 0, st>>>(key, mi, flag);
            ck(cub::DeviceSelect::Flagged(temp, tb, cub::CountingInputIterator<uint32_t>(0), flag, U, d_small + 2,
                                          mi, st), "select ties");
            unsigned long long u = 0;
            ck(cudaMemcpyAsync(&u, d_small + 2, 8, cudaMemcpyDeviceToHost, st), "D2H");
            ck(cudaStreamSynchronize(st), "ties");
            if (u) {
                residue_init_kernel<<<grid_of(u), 256, 0, st>>>(U, static_cast<int64_t>(u), key, pos, rpos, head);
                ck(cub::DeviceScan::InclusiveScan(temp, tb, head, grp, cub::Max(), static_cast<int>(u), st), "scan");
            }
            uint64_t depth = KEY_SYMS;
            while (u) {
                if (depth > n + KEY_SYMS) fail(MA_ERR_INTERNAL, "suffix refinement did not converge");
                const int ui = static_cast<int>(u);
                const int64_t ul = static_cast<int64_t>(u);
                int gbits = 1;
                while (gbits < 32 && (1ull << gbits) < u) ++gbits;
                // order by refinement key, then (stable) by group
                refine_key_kernel<<<grid_of(u), 256, 0, st>>>(T, n, rpos, ul, depth, ka, ia);
                cub::DoubleBuffer<uint64_t> rk(ka, kb);
                cub::DoubleBuffer<uint32_t> ix(ia, ib);
                ck(cub::DeviceRadixSort::SortPairs(temp, tb, rk, ix, ui, 0, 64, st), "sort refinement keys");
                gather_u32_kernel<<<grid_of(u), 256, 0, st>>>(grp, ix.Current(), ul, ga);
                cub::DoubleBuffer<uint32_t> gg(ga, gb);
                ck(cub::DeviceRadixSort::SortPairs(temp, tb, gg, ix, ui, 0, gbits, st), "sort groups");
                const uint32_t* g = gg.Current();
                refine_apply_kernel<<<grid_of(u), 256, 0, st>>>(T, n, ix.Current(), ul, depth, U, rpos, pos, rpos2,
                                                                rkey2);
                refine_ties_kernel<<<grid_of(u), 256, 0, st>>>(g, rkey2, ul, flag);
                ck(cub::DeviceSelect::Flagged(temp, tb, cub::CountingInputIterator<uint32_t>(0), flag, sel,
                                              d_small + 2, ui, st), "select ties");
                unsigned long long u2 = 0;
                ck(cudaMemcpyAsync(&u2, d_small + 2, 8, cudaMemcpyDeviceToHost, st), "D2H");
                ck(cudaStreamSynchronize(st), "refinement");
                if (u2) {
                    residue_next_kernel<<<grid_of(u2), 256, 0, st>>>(sel, static_cast<int64_t>(u2), U, rpos2, rkey2,
                                                                     g, U2, rpos, head);
                    ck(cub::DeviceScan::InclusiveScan(temp, tb, head, grp, cub::Max(), static_cast<int>(u2), st),
                       "scan");
                    std::swap(U, U2);
                }
                u = u2;
                depth += KEY_SYMS;
            }
            emit_kernel<<<grid_of(cnt), 256, 0, st>>>(T, pos, mi, row0, intv, rowsym, samples, d_small);
            ck(cudaGetLastError(), "emit");
            row0 += cnt;
            done_suffixes += cnt;
            b = e;
        }
        if (done_suffixes != n) fail(MA_ERR_INTERNAL, "BWT construction sorted a wrong number of suffixes");
        unsigned long long primary = 0;
        ck(cudaMemcpyAsync(&primary, d_small, 8, cudaMemcpyDeviceToHost, st), "D2H primary");
        ck(cudaStreamSynchronize(st), "suffix batches");
        if (primary == 0 || primary > n) fail(MA_ERR_INTERNAL, "no primary row");
        for (void* q : {static_cast<void*>(k0), static_cast<void*>(k1), static_cast<void*>(p0),
                        static_cast<void*>(p1), static_cast<void*>(flag), static_cast<void*>(U),
                        static_cast<void*>(U2), static_cast<void*>(sel), static_cast<void*>(head),
                        static_cast<void*>(grp), static_cast<void*>(ga), static_cast<void*>(gb),
                        static_cast<void*>(ia), static_cast<void*>(ib), static_cast<void*>(rpos),
                        static_cast<void*>(ka), static_cast<void*>(kb), static_cast<void*>(rpos2),
                        static_cast<void*>(rkey2), temp})
            m.release(q);

        // bwa .bwt words: blocks of 4 u64 counts + 8 words per 128 stored
        // positions, then one block of 4 u64 totals
        const uint64_t n_blocks = (n + 127) / 128;
        const uint64_t n_occ = n_blocks + 1;
        const uint64_t n_bwt = (n + 15) / 16 + 8 * n_occ;
        uint32_t* bwt = m.alloc<uint32_t>(n_bwt);
        Cnt4* cnt = m.alloc<Cnt4>(n_blocks + 1);
        Cnt4* before = m.alloc<Cnt4>(n_blocks + 1);
        ck(cudaMemsetAsync(bwt, 0, n_bwt * 4, st), "memset");
        bwa_words_kernel<<<grid_of(n_blocks), 256, 0, st>>>(rowsym, n, primary, n_blocks, bwt, cnt);
        ck(cudaMemsetAsync(cnt + n_blocks, 0, sizeof(Cnt4), st), "memset");
        size_t ts = 0;
        const Cnt4 zero{{0, 0, 0, 0}};
        const int nb1 = static_cast<int>(n_blocks + 1);
        ck(cub::DeviceScan::ExclusiveScan(nullptr, ts, cnt, before, Cnt4Sum(), zero, nb1, st), "scan temp");
        void* stemp = m.alloc<uint8_t>(ts);
        ck(cub::DeviceScan::ExclusiveScan(stemp, ts, cnt, before, Cnt4Sum(), zero, nb1, st), "scan");
        bwa_counts_kernel<<<grid_of(n_blocks), 256, 0, st>>>(before, n_blocks, bwt);
        ck(cudaGetLastError(), "bwa layout");
        Cnt4 totals;
        ck(cudaMemcpyAsync(&totals, before + n_blocks, sizeof totals, cudaMemcpyDeviceToHost, st), "D2H totals");
        out.bwt.resize(n_bwt);
        ck(cudaMemcpyAsync(out.bwt.data(), bwt, n_bwt * 4, cudaMemcpyDeviceToHost, st), "D2H bwt");
        out.samples.resize(n_sa - 1);
        if (n_sa > 1)
            ck(cudaMemcpyAsync(out.samples.data(), samples, (n_sa - 1) * 8, cudaMemcpyDeviceToHost, st), "D2H sa");
        ck(cudaStreamSynchronize(st), "BWT download");
        // closing totals block, where the host layout puts it
        uint64_t at = (n / 128) * 16;
        if (n % 128 != 0) at = (n / 128) * 16 + 8 + ((n % 128) + 15) / 16;
        for (int c = 0; c < 4; ++c) {
            out.bwt[at + 2 * c] = static_cast<uint32_t>(totals.c[c]);
            out.bwt[at + 2 * c + 1] = static_cast<uint32_t>(totals.c[c] >> 32);
        }
        out.primary = primary;
    } catch (...) {
        cudaStreamDestroy(st);
        throw;
    }
    cudaStreamDestroy(st);
    return out;
}

}  // namespace ma
