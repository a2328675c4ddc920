// device_index.cu - builds the HBM-resident index from bwa 0.7 files.
//
// The reference uploads the bwa words as they are and walks the sampled SA
// on every lookup (linear_gpu_fm.mojo:2034-2069, 1390-1508).  Here the
// upload is followed by one-time device passes that re-lay the index for
// random 32-byte gathers:
//   relayout_occ      bwa 64-B blocks of 128 positions -> 32-B lines of 64,
//                     counts relative to the line's superblock
//   relayout_pac      MSB-first pac bytes -> LSB-first u64 words, padded
//   reconstruct_sa    sampled SA -> full SA, one LF chain per sampled row
//   build_kmer        k-mer -> backward-search interval table
//   kmer3_*           3-letter k-mer tables from passes over the full SA
//   lcp / summary     capped LCPs of adjacent SA rows -> per-position
//                     shortest-unique lengths and k-mer counts
// The passes over all SA rows run in chunks of rows (with the few rows of
// overlap each pass needs), so that their staging stays a few GB whatever
// the text length.  Every kernel's loops are bounded; a chain that runs
// past its bound (only possible on an inconsistent index) raises a device
// error flag instead of spinning.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

#include "ma_device.cuh"
#include "ma_internal.h"

namespace ma {

namespace {

__device__ __forceinline__ uint32_t rev2(uint32_t v) {
    // reverse the order of the 16 2-bit symbols of a word
    v = __brev(v);
    return ((v >> 1) & 0x55555555u) | ((v & 0x55555555u) << 1);
}

__device__ __forceinline__ uint32_t count_sym32(uint32_t w_lsb, int c, int nbases) {
    // occurrences of c among the first nbases symbols (LSB first) of w
    uint32_t pat = static_cast<uint32_t>(c) * 0x55555555u;
    uint32_t t = w_lsb ^ pat;
    uint32_t m = ~(t | (t >> 1)) & 0x55555555u;
    if (nbases < 16) m &= (1u << (2 * nbases)) - 1;
    return __popc(m);
}

__global__ void relayout_occ_kernel(const uint32_t* __restrict__ bwa, uint64_t seq_len, uint64_t n_lines,
                                    const unsigned long long* __restrict__ super, int super_shift,
                                    OccLine* __restrict__ out) {
    uint64_t L = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (L >= n_lines) return;
    uint64_t blk = L >> 1;
    int half = static_cast<int>(L & 1);
    const uint32_t* b = bwa + blk * 16;
    uint64_t cnt[4];
    for (int c = 0; c < 4; ++c) cnt[c] = static_cast<uint64_t>(b[2 * c]) | (static_cast<uint64_t>(b[2 * c + 1]) << 32);
    if (half) {
        for (int i = 0; i < 4; ++i) {
            uint32_t w = rev2(b[8 + i]);
            for (int c = 0; c < 4; ++c) cnt[c] += count_sym32(w, c, 16);
        }
    }
    OccLine o;
    const unsigned long long* sb = super + (((L * 64) >> super_shift) << 2);
    for (int c = 0; c < 4; ++c) o.cnt[c] = static_cast<uint32_t>(cnt[c] - sb[c]);
    for (int i = 0; i < 4; ++i) {
        uint64_t p0 = L * 64 + 16 * i;  // first position held by word i
        uint32_t w = 0;
        if (p0 < seq_len) {
            w = rev2(b[8 + 4 * half + i]);
            uint64_t valid = seq_len - p0;
            if (valid < 16) w &= (1u << (2 * valid)) - 1;
        }
        o.w[i] = w;
    }
    out[L] = o;
}

__global__ void relayout_pac_kernel(const uint8_t* __restrict__ pac, uint64_t l_pac, uint64_t n_words,
                                    uint64_t* __restrict__ out) {
    uint64_t w = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (w >= n_words) return;  // n_words covers the text plus padding on both sides
    int64_t tw = static_cast<int64_t>(w) - PAC_PAD;  // text word index
    uint64_t v = 0;
    if (tw >= 0) {
        for (int i = 0; i < 32; ++i) {
            uint64_t p = static_cast<uint64_t>(tw) * 32 + i;
            if (p >= l_pac) break;
            uint64_t sym = (pac[p >> 2] >> ((~p & 3) << 1)) & 3;
            v |= sym << (2 * i);
        }
    }
    out[w] = v;
}

// Full-SA stores of either layout (index preparation only).  A 40-bit value
// is written byte by byte, so rows sharing a 16-byte chunk never race.
__device__ __forceinline__ void sa_put(const DevIndex& ix, uint32_t* sa, uint8_t* sa40, uint64_t row, uint64_t v) {
    if (!ix.sa_wide) {
        sa[row] = static_cast<uint32_t>(v);
        return;
    }
    const uint64_t ch = row / 3;
    uint8_t* p = sa40 + ch * 16 + (row - ch * 3) * 5;
    for (int i = 0; i < 5; ++i) p[i] = static_cast<uint8_t>(v >> (8 * i));
}

// One chain per sampled row i (i % intv == 0, i <= seq_len): SA[i] is known
// (row 0 is the sentinel suffix, SA[0] = seq_len).  LF steps from i visit
// the rows of text positions SA[i]-1, SA[i]-2, ... until a sampled row or
// text position 0; every row visited gets its SA value.
__global__ void reconstruct_sa_kernel(DevIndex ix, const uint64_t* __restrict__ samples, uint64_t n_chains,
                                      uint64_t intv, uint32_t* __restrict__ sa, uint8_t* __restrict__ sa40,
                                      uint64_t max_steps, int* __restrict__ err) {
    uint64_t ci = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (ci >= n_chains) return;
    uint64_t r = ci * intv;
    uint64_t s = ci == 0 ? ix.seq_len : samples[ci - 1];
    if (s > ix.seq_len) {
        atomicExch(err, 1);
        return;
    }
    sa_put(ix, sa, sa40, r, s);
    for (uint64_t step = 0; step < max_steps; ++step) {
        if (s == 0) return;
        if (r == ix.primary) {  // position 0 reached through a bad sample
            atomicExch(err, 2);
            return;
        }
        uint64_t x = r - (r > ix.primary ? 1 : 0);
        int c = bwt_sym(ix.occ, x);
        r = ix.L2[c] + occ_row(ix, r, c);
        s -= 1;
        if (r > ix.seq_len) {
            atomicExch(err, 3);
            return;
        }
        if (r % intv == 0) return;
        sa_put(ix, sa, sa40, r, s);
    }
    atomicExch(err, 4);  // chain longer than any consistent index allows
}

__global__ void count_unset_kernel(DevIndex ix, uint64_t n, unsigned long long* cnt) {
    uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t unset = ix.sa_wide ? SA40_UNSET : 0xFFFFFFFFull;
    unsigned long long local = 0;
    for (; i < n; i += stride) local += sa_at(ix, i) == unset;
    if (local) atomicAdd(cnt, local);
}

// Packed k-mer table entry of the interval [k, l] (count l - k + 1 >= 1).
__device__ __forceinline__ uint64_t kmer_entry(uint64_t k, uint64_t count) {
    return count > KMER_MAX_COUNT ? KMER_UNTABLED : (k | (count << KMER_K_BITS));
}

__global__ void build_kmer_kernel(DevIndex ix, int K, uint64_t n_kmers, uint64_t* __restrict__ out) {
    uint64_t idx = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (idx >= n_kmers) return;
    uint64_t k = 0, l = ix.seq_len;
    for (int t = 0; t < K; ++t) {
        int c = static_cast<int>((idx >> (2 * t)) & 3);  // last base of W first
        uint64_t ok = k != 0 ? occ_row(ix, k - 1, c) : 0;
        uint64_t ol = occ_row(ix, l, c);
        k = ix.L2[c] + ok + 1;
        l = ix.L2[c] + ol;
        if (k > l) {
            out[idx] = 0;  // count 0: W does not occur
            return;
        }
    }
    out[idx] = kmer_entry(k, l - k + 1);
}

// A/T window outcome table: one thread per window W of K bases over A/T
// (index bit i set where base i of W is T).  The backward search over W
// from its last base with seed length sl and no max_occ stop, as
// search_start / search_next in seed_core.cuh run it: the first length
// >= sl with one row ends it with that seed; an empty interval ends it
// with the last interval of <= 16 rows at a length >= sl, if any; else it
// continues past W from the rows of all of W.
__global__ void build_atw_kernel(DevIndex ix, int K, int sl, uint64_t n, uint4* __restrict__ out) {
    const uint64_t idx = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (idx >= n) return;
    uint64_t k = 0, l = ix.seq_len, c_sl = 0;
    uint64_t kept_k = 0, kept_n = 0;
    int kept_o = -1;
    uint64_t lo = 0, hi = 0;  // kind 0 unless set below
    bool done = false;
    for (int t = 0; t < K && !done; ++t) {
        const int c = (idx >> (K - 1 - t)) & 1 ? 3 : 0;  // base K-1-t of W
        const uint64_t ok = k != 0 ? occ_row(ix, k - 1, c) : 0;
        const uint64_t ol = occ_row(ix, l, c);
        k = ix.L2[c] + ok + 1;
        l = ix.L2[c] + ol;
        const int mlen = t + 1;
        if (k > l) {
            if (kept_o >= 0) {
                lo = kept_k | static_cast<uint64_t>(kept_o) << 35 | 1ull << 40;
                hi = kept_n;
            }
            done = true;
            break;
        }
        const uint64_t rows = l - k + 1;
        if (mlen == sl) c_sl = rows < ATW_COUNT_CAP ? rows : ATW_COUNT_CAP;
        if (mlen >= sl) {
            if (rows == 1) {
                lo = k | static_cast<uint64_t>(mlen - 1) << 35 | 1ull << 40;
                hi = 1;
                done = true;
                break;
            }
            if (rows <= 16) {
                kept_k = k;
                kept_n = rows;
                kept_o = mlen - 1;
            }
        }
    }
    if (!done) {  // continues from the rows of W (>= 2 of them)
        lo = k | 2ull << 40;
        hi = l - k + 1;
    }
    hi |= c_sl << 35;
    out[idx] = make_uint4(static_cast<uint32_t>(lo), static_cast<uint32_t>(lo >> 32), static_cast<uint32_t>(hi),
                          static_cast<uint32_t>(hi >> 32));
}

// 2-bit codes of text T[p, p+K) (T = the pac followed by its reverse
// complement), first base most significant; ~0 when p + K > seq_len.
__device__ uint64_t text_kmer(const DevIndex& ix, uint64_t p, int K) {
    if (p + K > ix.seq_len) return ~0ull;
    const uint64_t L = ix.l_pac;
    const uint64_t mask = (1ull << (2 * K)) - 1;
    uint64_t v = 0;
    if (p + K <= L) {
        const uint64_t w = ref_window(ix.pacw, static_cast<int64_t>(p));  // base p at bits 0-1
        for (int i = 0; i < K; ++i) v = (v << 2) | ((w >> (2 * i)) & 3);
    } else if (p >= L) {
        // T[p+i] = 3 - pac[2L-1-p-i]: the forward window [q0, q0+K) read
        // backwards and complemented, which is the LSB-first window itself
        const uint64_t q0 = 2 * L - p - K;
        v = (ref_window(ix.pacw, static_cast<int64_t>(q0)) & mask) ^ mask;
    } else {
        for (int i = 0; i < K; ++i) {
            const uint64_t q = p + i;
            const uint64_t f = q < L ? q : 2 * L - 1 - q;
            const uint64_t c = (ix.pacw[(f >> 5) + PAC_PAD] >> (2 * (f & 31))) & 3;
            v = (v << 2) | (q < L ? c : 3 - c);
        }
    }
    return v;
}

// K-mer codes of SA rows [row0, row0 + n) into codes[0, n).
__global__ void kmer3_rows_kernel(DevIndex ix, int K, uint64_t row0, uint64_t n, uint64_t* __restrict__ codes) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    codes[i] = text_kmer(ix, sa_at(ix, row0 + i), K);
}

__global__ void fill_u64_kernel(uint64_t* __restrict__ t, uint64_t n, uint64_t v) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) t[i] = v;
}

// Base-3 index of a 3-letter k-mer code and the tables it belongs to.
__device__ __forceinline__ uint32_t kmer3_index(uint64_t c, int K, bool& agt, bool& act) {
    const uint64_t lo = c & kEven, hi = (c >> 1) & kEven;
    agt = (lo & ~hi) == 0;  // no C
    act = (hi & ~lo) == 0;  // no G
    uint32_t idx = 0;
    for (int j = K - 1; j >= 0; --j) idx = idx * 3 + static_cast<uint32_t>(__popcll((c >> (2 * j)) & 3));
    return idx;
}

// Rows with the same k-mer are contiguous in SA order; the first and last
// row of each run are the interval (k, l) of that k-mer.  One chunk of rows
// [a, b): codes[j] is the code of row a - 1 + j (one row of overlap on each
// side, ~0 outside [0, n_rows)).  pass 0 records the first row of every
// run starting in the chunk; pass 1 turns the entry of every run ending in
// the chunk into its packed interval (its first row was recorded by pass 0
// of this chunk or of an earlier one).
__global__ void kmer3_bounds_kernel(const uint64_t* __restrict__ codes, uint64_t a, uint64_t n, int K, int pass,
                                    uint64_t* __restrict__ t_agt, uint64_t* __restrict__ t_act) {
    const uint64_t j = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (j >= n) return;
    const uint64_t c = codes[j + 1];
    if (c == ~0ull) return;
    bool agt, act;
    if (pass == 0) {
        if (codes[j] == c) return;
        const uint32_t idx = kmer3_index(c, K, agt, act);
        if (agt) t_agt[idx] = a + j;
        if (act) t_act[idx] = a + j;
    } else {
        if (codes[j + 2] == c) return;
        const uint32_t idx = kmer3_index(c, K, agt, act);
        const uint64_t row = a + j;
        if (agt) t_agt[idx] = kmer_entry(t_agt[idx], row - t_agt[idx] + 1);
        if (act) t_act[idx] = kmer_entry(t_act[idx], row - t_act[idx] + 1);
    }
}

// 32 symbols of T from position p (T[p] in bits 0-1); symbols past the end
// of T read as 0 (callers bound comparisons by the suffix lengths).
__device__ uint64_t text_window32(const DevIndex& ix, uint64_t p) {
    const uint64_t L = ix.l_pac;
    if (p + 32 <= L) return ref_window(ix.pacw, static_cast<int64_t>(p));
    if (p >= L && p + 32 <= 2 * L) {
        // T[p+i] = 3 - pac[2L-1-p-i]: the forward window [2L-p-32, 2L-p)
        // complemented, with its 32 symbols in reverse order
        uint64_t w = ~ref_window(ix.pacw, static_cast<int64_t>(2 * L - p - 32));
        w = __brevll(w);
        return ((w >> 1) & kEven) | ((w & kEven) << 1);
    }
    uint64_t v = 0;
    for (int i = 0; i < 32; ++i) {
        const uint64_t q = p + i;
        if (q >= 2 * L) break;
        const uint64_t f = q < L ? q : 2 * L - 1 - q;
        const uint64_t c = (ix.pacw[(f >> 5) + PAC_PAD] >> (2 * (f & 31))) & 3;
        v |= (q < L ? c : 3 - c) << (2 * i);
    }
    return v;
}

constexpr int LCP_CAP = 255;

// lcp[j] = min(common prefix of the suffixes of rows i-1 and i, 255) for
// rows i = row0 + j, j < n (row 0: 0).
__global__ void lcp_kernel(DevIndex ix, uint64_t row0, uint64_t n, uint8_t* __restrict__ lcp) {
    const uint64_t j = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (j >= n) return;
    const uint64_t i = row0 + j;
    if (i == 0) {
        lcp[j] = 0;
        return;
    }
    const uint64_t len = ix.seq_len;
    const uint64_t a = sa_at(ix, i - 1), b = sa_at(ix, i);
    uint64_t maxl = len - (a > b ? a : b);  // the shorter suffix
    if (maxl > LCP_CAP) maxl = LCP_CAP;
    uint64_t l = 0;
    while (l < maxl) {
        const uint64_t x = text_window32(ix, a + l) ^ text_window32(ix, b + l);
        const uint64_t d = (x | (x >> 1)) & kEven;
        if (d) {
            l += static_cast<uint64_t>(__ffsll(static_cast<long long>(d)) - 1) / 2;
            break;
        }
        l += 32;
    }
    lcp[j] = static_cast<uint8_t>(l < maxl ? l : maxl);
}

// Row i holds the suffix starting at y = SA[i]; its shortest unique prefix
// is 1 + max(lcp[i], lcp[i+1]) and its K-mer occurs as often as the run of
// adjacent rows with lcp >= K around i.  Stored at x = 2L-1-y.  Rows
// [a, b) of one chunk; lcp[j] holds the LCP of row l0 + j for rows
// [l0, l1), which covers [a - 255, b + 256) within [0, n_rows).
__global__ void summary_kernel(DevIndex ix, uint64_t n_rows, int K, uint64_t a, uint64_t b,
                               const uint8_t* __restrict__ lcp, uint64_t l0, uint64_t l1,
                               uint16_t* __restrict__ summary) {
    const uint64_t i = a + blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i == 0 || i >= b) return;  // row 0 is the sentinel suffix
    const uint64_t n = ix.seq_len;
    const uint64_t y = sa_at(ix, i);
    const uint8_t* L = lcp - l0;  // L[r] = LCP of row r, r in [l0, l1)
    const int l1v = L[i], l2v = i + 1 < n_rows ? L[i + 1] : 0;
    const uint64_t m = 1 + static_cast<uint64_t>(l1v > l2v ? l1v : l2v);
    const uint32_t mul = (m < LCP_CAP && y + m <= n) ? static_cast<uint32_t>(m) : 255u;
    uint32_t occ = 255;
    if (y + K <= n) {
        occ = 1;
        for (uint64_t j = i; j >= 1 && j > l0 && L[j] >= K && occ < 255; --j) ++occ;
        for (uint64_t j = i + 1; j < n_rows && j < l1 && L[j] >= K && occ < 255; ++j) ++occ;
    }
    summary[n - 1 - y] = static_cast<uint16_t>(mul | (occ << 8));
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

unsigned grid_for(uint64_t n, unsigned block) {
    uint64_t g = (n + block - 1) / block;
    return static_cast<unsigned>(g ? g : 1);
}

}  // namespace

uint64_t pow3(int k) {
    uint64_t v = 1;
    for (int i = 0; i < k; ++i) v *= 3;
    return v;
}

namespace {

bool wide_rows(const BwaIndexHost& h, const LayoutOptions& lo) {
    return lo.wide_rows || h.seq_len + 1 >= 0xFFFFFFFFull;
}

uint64_t n_super(const BwaIndexHost& h, const LayoutOptions& lo) {
    return ((h.seq_len ? h.seq_len - 1 : 0) >> lo.occ_super_shift) + 1;
}

uint64_t sa_bytes(const BwaIndexHost& h, const LayoutOptions& lo) {
    const uint64_t rows = h.seq_len + 1;
    return wide_rows(h, lo) ? ((rows + 2) / 3) * 16 : rows * 4;
}

// Rows per preparation pass over the SA.
uint64_t chunk_rows(const BwaIndexHost& h, const LayoutOptions& lo) {
    const uint64_t rows = h.seq_len + 1;
    uint64_t c = lo.prep_chunk_rows ? lo.prep_chunk_rows : (1ull << 30);
    if (c < 512) c = 512;
    return c < rows ? c : rows;
}

constexpr uint64_t LCP_HALO = 256;  // rows of LCP a summary row may look at on each side

}  // namespace

uint64_t device_index_bytes(const BwaIndexHost& h, const LayoutOptions& lo) {
    uint64_t n_lines = (h.seq_len + 63) / 64;
    uint64_t b = n_lines * sizeof(OccLine) + n_super(h, lo) * 32;
    b += sa_bytes(h, lo);
    b += ((h.l_pac + 31) / 32 + 2 * PAC_PAD) * 8;
    if (lo.kmer_k > 0) b += (1ull << (2 * lo.kmer_k)) * 8;
    if (lo.kmer3_k > 0) b += 2 * pow3(lo.kmer3_k) * 8 + h.seq_len * 2;
    if (lo.at_k > 0) b += (1ull << lo.at_k) * 16;
    b += h.contigs.size() * 12;
    return b;
}

// Temporary device memory of the preparation passes: the uploaded bwa
// files, then (after they are freed) one chunk of k-mer codes or LCPs.
uint64_t device_index_staging_bytes(const BwaIndexHost& h, const LayoutOptions& lo) {
    uint64_t b = h.bwt.size() * 4 + h.pac.size() + 8 + (h.sa.size() + 1) * 8;
    if (lo.kmer3_k > 0) b = std::max<uint64_t>(b, (chunk_rows(h, lo) + 2) * 8);
    return b;
}

// Builds the resident index on the current device; returns its DevIndex and
// fills `bufs`.  Temporary upload buffers are freed before returning.
DevIndex build_device_index(const BwaIndexHost& h, const LayoutOptions& lo, cudaStream_t st,
                            DeviceIndexBuffers& bufs, uint64_t* reject_below) {
    if (h.seq_len > MAX_SEQ_LEN)
        fail(MA_ERR_UNSUPPORTED, "resident layout holds texts of at most 2^35 - 2 symbols");
    if (lo.kmer_k < 0 || lo.kmer_k > 14) fail(MA_ERR_ARG, "kmer_k must be in 0..14");
    if (lo.kmer3_k < 0 || lo.kmer3_k > 20) fail(MA_ERR_ARG, "kmer3_k must be in 0..20");
    if (lo.occ_super_shift < 7 || lo.occ_super_shift > 31) fail(MA_ERR_ARG, "occ superblock shift must be in 7..31");
    if (lo.at_k < 0 || lo.at_k > ATW_MAX_K || (lo.at_k > 0 && (lo.at_seed_len < 1 || lo.at_seed_len > lo.at_k)))
        fail(MA_ERR_ARG, "at_k must be 0 or in at_seed_len..30, at_seed_len >= 1");
    const int kmer_k = lo.kmer_k, kmer3_k = lo.kmer3_k;
    const uint64_t n_lines = (h.seq_len + 63) / 64;
    const uint64_t n_pacw = (h.l_pac + 31) / 32 + 2 * PAC_PAD;
    const uint64_t n_rows = h.seq_len + 1;
    const bool wide = wide_rows(h, lo);
    DevIndex ix{};
    ix.seq_len = h.seq_len;
    ix.l_pac = h.l_pac;
    ix.primary = h.primary;
    for (int c = 0; c < 5; ++c) ix.L2[c] = h.L2[c];
    ix.n_contigs = static_cast<int64_t>(h.contigs.size());
    ix.kmer_k = kmer_k;
    ix.kmer3_k = 0;  // set once the tables are built
    ix.occ_super_shift = lo.occ_super_shift;
    ix.sa_wide = wide ? 1 : 0;

    // symbols before each superblock, from the bwa block counts (a
    // superblock starts on a 128-position block boundary)
    const uint64_t ns = n_super(h, lo);
    std::vector<unsigned long long> super(ns * 4, 0);
    for (uint64_t sb = 0; sb < ns; ++sb) {
        const uint64_t blk = (sb << lo.occ_super_shift) >> 7;
        for (int c = 0; c < 4; ++c) {
            const uint64_t w = blk * 16 + 2 * static_cast<uint64_t>(c);
            if (w + 1 >= h.bwt.size()) fail(MA_ERR_FORMAT, "FmIndex .bwt shorter than seq_len implies");
            super[sb * 4 + c] = static_cast<uint64_t>(h.bwt[w]) | (static_cast<uint64_t>(h.bwt[w + 1]) << 32);
        }
    }

    uint32_t* d_bwa = nullptr;
    uint8_t* d_pac = nullptr;
    uint64_t* d_samples = nullptr;
    int* d_err = nullptr;
    unsigned long long* d_cnt = nullptr;
    uint64_t* d_codes = nullptr;
    auto free_uploads = [&]() {
        cudaFree(d_bwa);
        cudaFree(d_pac);
        cudaFree(d_samples);
        d_bwa = nullptr;
        d_pac = nullptr;
        d_samples = nullptr;
    };
    auto cleanup = [&]() {
        free_uploads();
        cudaFree(d_err);
        cudaFree(d_cnt);
        cudaFree(d_codes);
    };
    try {
        check(cudaMalloc(&bufs.occ, n_lines * sizeof(OccLine)), "cudaMalloc occ");
        check(cudaMalloc(&bufs.occ_super, ns * 32), "cudaMalloc occ superblocks");
        if (wide) check(cudaMalloc(&bufs.sa40, sa_bytes(h, lo)), "cudaMalloc sa");
        else check(cudaMalloc(&bufs.sa, sa_bytes(h, lo)), "cudaMalloc sa");
        check(cudaMalloc(&bufs.pacw, n_pacw * 8), "cudaMalloc pac");
        check(cudaMalloc(&bufs.coff, (h.contigs.size() + 1) * 8), "cudaMalloc contig_off");
        check(cudaMalloc(&bufs.clen, (h.contigs.size() + 1) * 4), "cudaMalloc contig_len");
        if (kmer_k > 0) check(cudaMalloc(&bufs.kmer, (1ull << (2 * kmer_k)) * 8), "cudaMalloc kmer");
        check(cudaMalloc(&d_bwa, h.bwt.size() * 4), "cudaMalloc bwt staging");
        check(cudaMalloc(&d_pac, h.pac.size() + 8), "cudaMalloc pac staging");
        check(cudaMalloc(&d_samples, (h.sa.size() + 1) * 8), "cudaMalloc sa staging");
        check(cudaMalloc(&d_err, sizeof(int)), "cudaMalloc err");
        check(cudaMalloc(&d_cnt, sizeof(unsigned long long)), "cudaMalloc cnt");
        check(cudaMemsetAsync(d_err, 0, sizeof(int), st), "memset");
        check(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), st), "memset");
        check(cudaMemcpyAsync(bufs.occ_super, super.data(), ns * 32, cudaMemcpyHostToDevice, st), "H2D superblocks");
        check(cudaMemcpyAsync(d_bwa, h.bwt.data(), h.bwt.size() * 4, cudaMemcpyHostToDevice, st), "H2D bwt");
        check(cudaMemsetAsync(d_pac, 0, h.pac.size() + 8, st), "memset");
        check(cudaMemcpyAsync(d_pac, h.pac.data(), h.pac.size(), cudaMemcpyHostToDevice, st), "H2D pac");
        if (!h.sa.empty())
            check(cudaMemcpyAsync(d_samples, h.sa.data(), h.sa.size() * 8, cudaMemcpyHostToDevice, st), "H2D sa");
        std::vector<uint64_t> coff(h.contigs.size());
        std::vector<uint32_t> clen(h.contigs.size());
        for (size_t i = 0; i < h.contigs.size(); ++i) {
            coff[i] = h.contigs[i].offset;
            clen[i] = h.contigs[i].len;
        }
        if (!coff.empty()) {
            check(cudaMemcpyAsync(bufs.coff, coff.data(), coff.size() * 8, cudaMemcpyHostToDevice, st), "H2D coff");
            check(cudaMemcpyAsync(bufs.clen, clen.data(), clen.size() * 4, cudaMemcpyHostToDevice, st), "H2D clen");
        }
        relayout_occ_kernel<<<grid_for(n_lines, 256), 256, 0, st>>>(d_bwa, h.seq_len, n_lines, bufs.occ_super,
                                                                     lo.occ_super_shift, bufs.occ);
        relayout_pac_kernel<<<grid_for(n_pacw, 256), 256, 0, st>>>(d_pac, h.l_pac, n_pacw, bufs.pacw);
        check(cudaGetLastError(), "relayout launch");
        ix.occ = bufs.occ;
        ix.occ_super = bufs.occ_super;
        ix.pacw = bufs.pacw;
        ix.coff = bufs.coff;
        ix.clen = bufs.clen;
        ix.sa = bufs.sa;
        ix.sa40 = bufs.sa40;
        // full SA from the samples
        check(cudaMemsetAsync(wide ? static_cast<void*>(bufs.sa40) : static_cast<void*>(bufs.sa), 0xFF,
                              sa_bytes(h, lo), st), "memset sa");
        const uint64_t intv = static_cast<uint64_t>(h.sa_intv);
        const uint64_t n_chains = h.seq_len / intv + 1;  // rows 0, intv, ..., <= seq_len
        if (h.sa.size() + 1 < n_chains) fail(MA_ERR_FORMAT, "FmIndex .sa holds fewer samples than seq_len implies");
        reconstruct_sa_kernel<<<grid_for(n_chains, 128), 128, 0, st>>>(
            ix, d_samples, n_chains, intv, bufs.sa, reinterpret_cast<uint8_t*>(bufs.sa40), 1ull << 20, d_err);
        check(cudaGetLastError(), "reconstruct_sa launch");
        count_unset_kernel<<<1184, 256, 0, st>>>(ix, n_rows, d_cnt);
        int herr = 0;
        unsigned long long hcnt = 0;
        check(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H err");
        check(cudaMemcpyAsync(&hcnt, d_cnt, sizeof(hcnt), cudaMemcpyDeviceToHost, st), "D2H cnt");
        check(cudaStreamSynchronize(st), "index preparation");
        if (herr) fail(MA_ERR_FORMAT, "FmIndex BWT and SA samples are inconsistent (code " + std::to_string(herr) + ")");
        if (hcnt) fail(MA_ERR_FORMAT, "FmIndex SA reconstruction left " + std::to_string(hcnt) + " rows unset");
        free_uploads();
        // rejection bound of the reference's sampled walk: the smallest text
        // position whose BWT row is sampled (rows >= intv; row 0 is the
        // sentinel suffix and is never reached by a walk)
        uint64_t p0 = h.seq_len;
        for (uint64_t v : h.sa) p0 = v < p0 ? v : p0;
        ix.sa_reject_below = p0;
        *reject_below = p0;
        if (kmer_k > 0) {
            const uint64_t nk = 1ull << (2 * kmer_k);
            build_kmer_kernel<<<grid_for(nk, 256), 256, 0, st>>>(ix, kmer_k, nk, bufs.kmer);
            check(cudaGetLastError(), "build_kmer launch");
            ix.kmer = bufs.kmer;
        }
        if (lo.at_k > 0) {
            const uint64_t na = 1ull << lo.at_k;
            check(cudaMalloc(&bufs.atw, na * 16), "cudaMalloc A/T window table");
            build_atw_kernel<<<grid_for(na, 256), 256, 0, st>>>(ix, lo.at_k, lo.at_seed_len, na, bufs.atw);
            check(cudaGetLastError(), "build_atw launch");
            ix.atw = bufs.atw;
            ix.at_k = lo.at_k;
            ix.at_seed_len = lo.at_seed_len;
        }
        if (kmer3_k > 0) {
            const uint64_t n3 = pow3(kmer3_k);
            const uint64_t C = chunk_rows(h, lo);
            check(cudaMalloc(&bufs.kmer3[0], n3 * 8), "cudaMalloc kmer3");
            check(cudaMalloc(&bufs.kmer3[1], n3 * 8), "cudaMalloc kmer3");
            check(cudaMalloc(&bufs.summary, h.seq_len * 2), "cudaMalloc summary");
            check(cudaMalloc(&d_codes, (C + 2) * 8), "cudaMalloc kmer3 staging");
            fill_u64_kernel<<<4096, 256, 0, st>>>(bufs.kmer3[0], n3, 0);
            fill_u64_kernel<<<4096, 256, 0, st>>>(bufs.kmer3[1], n3, 0);
            // tables: codes of rows [a - 1, b + 1) per chunk
            for (uint64_t a = 0; a < n_rows; a += C) {
                const uint64_t b = std::min(n_rows, a + C);
                const uint64_t r0 = a ? a - 1 : 0, r1 = std::min(n_rows, b + 1);
                if (!a) fill_u64_kernel<<<1, 32, 0, st>>>(d_codes, 1, ~0ull);
                if (r1 == b) fill_u64_kernel<<<1, 32, 0, st>>>(d_codes + (b - a + 1), 1, ~0ull);
                kmer3_rows_kernel<<<grid_for(r1 - r0, 256), 256, 0, st>>>(ix, kmer3_k, r0, r1 - r0,
                                                                          d_codes + (a ? 0 : 1));
                for (int pass = 0; pass < 2; ++pass)
                    kmer3_bounds_kernel<<<grid_for(b - a, 256), 256, 0, st>>>(d_codes, a, b - a, kmer3_k, pass,
                                                                              bufs.kmer3[0], bufs.kmer3[1]);
                check(cudaGetLastError(), "kmer3 launch");
            }
            // summary: LCPs of rows [a - 256, b + 256) per chunk (the codes
            // buffer, 8 B per row, holds them as bytes)
            uint8_t* d_lcp = reinterpret_cast<uint8_t*>(d_codes);
            for (uint64_t a = 0; a < n_rows; a += C) {
                const uint64_t b = std::min(n_rows, a + C);
                const uint64_t l0 = a > LCP_HALO ? a - LCP_HALO : 0, l1 = std::min(n_rows, b + LCP_HALO);
                lcp_kernel<<<grid_for(l1 - l0, 256), 256, 0, st>>>(ix, l0, l1 - l0, d_lcp);
                summary_kernel<<<grid_for(b - a, 256), 256, 0, st>>>(ix, n_rows, kmer3_k, a, b, d_lcp, l0, l1,
                                                                     bufs.summary);
                check(cudaGetLastError(), "summary launch");
            }
            check(cudaStreamSynchronize(st), "kmer3 tables");
            cudaFree(d_codes);
            d_codes = nullptr;
            ix.kmer3[0] = bufs.kmer3[0];
            ix.kmer3[1] = bufs.kmer3[1];
            ix.summary = bufs.summary;
            ix.kmer3_k = kmer3_k;
        }
        check(cudaStreamSynchronize(st), "index preparation");
    } catch (...) {
        cleanup();
        throw;
    }
    cleanup();
    bufs.bytes = device_index_bytes(h, lo);
    return ix;
}

void free_device_index(DeviceIndexBuffers& b) {
    cudaFree(b.occ);
    cudaFree(b.occ_super);
    cudaFree(b.sa);
    cudaFree(b.sa40);
    cudaFree(b.pacw);
    cudaFree(b.kmer);
    cudaFree(b.kmer3[0]);
    cudaFree(b.kmer3[1]);
    cudaFree(b.summary);
    cudaFree(b.atw);
    cudaFree(b.coff);
    cudaFree(b.clen);
    b = DeviceIndexBuffers{};
}

}  // namespace ma
