// ma_device.cuh - HBM layout of the resident index and the device helpers
// shared by the index-preparation and mapping kernels (sm_100a).
//
// Layout (all resident in HBM, built once per index by device_index.cu).
// Rows and text positions are 64-bit throughout (texts up to 2^35 symbols):
//   occ   one 32-byte line per 64 BWT positions of the stored BWT string
//         (the sentinel removed, as in bwa): u32 cnt[4] = symbols c in
//         positions [S, 64*line) where S is the start of the line's
//         superblock of 2^occ_super_shift positions, then 4 u32 words of
//         2-bit symbols, 16 per word, least significant first.  An Occ query
//         is one 32-B sector plus the superblock's count (a table of
//         4 u64 per superblock, a few entries, cached).
//   sa    the full suffix array: u32 per row when every row and position
//         fits 32 bits, else 40-bit values packed three to a 16-byte chunk
//         (bytes 5*slot .. 5*slot+4 of chunk row/3), one 16-B load either way.
//   pacw  the forward text, 32 bases per u64 word, least significant first,
//         with PAC_PAD zero words before text position 0 and after the end,
//         so that a 32-base window starting anywhere in [-512, l_pac + 480)
//         is two aligned loads and a funnel shift.
//   kmer  for every k-mer W (first base most significant, 2 bits per base)
//         the backward-search interval (k, l) after the k steps that consume
//         W, packed in a u64 as k | (l - k + 1) << 35 (count 0: W does not
//         occur; KMER_UNTABLED: count too large to pack, search from scratch).
//   kmer3 the same intervals for k-mers over the alphabets of converted
//         reads, indexed in base 3: table 0 holds the words without C
//         (A, G, T -> digits 0, 1, 2; C->T reads), table 1 the words
//         without G (A, C, T -> 0, 1, 2; G->A reads).
//   summary  per position x of T (pac + reverse complement), for the
//         substrings of T that end at x: bits 0-7 the smallest length m with
//         T[x-m+1, x] occurring once in T (255: none up to 254), bits 8-15 the
//         occurrences of the kmer3_k-mer ending at x (capped at 255).  T is
//         its own reverse complement, so these are the shortest unique prefix
//         and the k-mer count of the suffix starting at 2*l_pac-1-x.
//   atw   for every read window W of at_k bases over A and T alone (bit i
//         of the index set where base i of W, first base at bit 0, is T),
//         the outcome of the backward search from W's last base over W
//         with seed length at_seed_len and no max_occ stop, 16 bytes:
//         lo = k (bits 0-34) | o (35-39) | kind (40-41),
//         hi = n (bits 0-34) | c (35-63), where kind 0: the search ends with
//         no seed; kind 1: it ends with the seed of rows [k, k+n) whose
//         pattern is the last o+1 bases of W; kind 2: it continues past W
//         from the n >= 2 rows [k, k+n) of all of W; c = the rows at
//         length at_seed_len (0 when empty before it, capped at 2^29 - 1),
//         which decides the max_occ stop at run time.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/mojoalign_b200.h"

namespace ma {

constexpr int PAC_PAD = 16;           // u64 words of zero padding each side
constexpr int MAX_READ_LEN = 1024;    // linear_gpu_fm.mojo:2192,2447
constexpr int MAX_WORDS = MAX_READ_LEN / 32;

struct __align__(32) OccLine {
    uint32_t cnt[4];
    uint32_t w[4];
};

// Largest text (seq_len) the resident layout holds: positions and k-mer
// table rows fit 35 bits.
constexpr uint64_t MAX_SEQ_LEN = (1ull << 35) - 2;
constexpr int KMER_K_BITS = 35;
constexpr uint64_t KMER_K_MASK = (1ull << KMER_K_BITS) - 1;
constexpr uint64_t KMER_MAX_COUNT = (1ull << (64 - KMER_K_BITS)) - 2;
constexpr uint64_t KMER_UNTABLED = ~0ull;
constexpr uint64_t SA40_UNSET = (1ull << 40) - 1;
constexpr int OCC_SUPER_SHIFT = 31;  // default superblock: 2^31 positions
constexpr int ATW_MAX_K = 30;                            // longest A/T window of the outcome table
constexpr uint64_t ATW_COUNT_CAP = (1ull << 29) - 1;     // rows at the seed length, saturated

struct DevIndex {
    const OccLine* occ;
    const unsigned long long* occ_super;  // [n_super][4] symbols before each superblock
    int32_t occ_super_shift;
    int32_t sa_wide;                      // 0: u32 rows in sa; 1: 40-bit rows in sa40
    const uint32_t* sa;
    const uint4* sa40;
    const uint64_t* pacw;
    const uint64_t* kmer;
    const uint64_t* kmer3[2];
    const uint16_t* summary;  // per text end position x: see "summary" above
    const uint64_t* coff;
    const uint32_t* clen;
    int64_t n_contigs;
    uint64_t seq_len, l_pac, primary;
    uint64_t L2[5];
    uint64_t sa_reject_below;  // sa_pos below this is rejected (see seed kernel)
    int32_t kmer_k;
    int32_t kmer3_k;
    const uint4* atw;         // A/T window outcome table (see "atw" above), or null
    int32_t at_k;             // window length of atw (0: no table)
    int32_t at_seed_len;      // seed length the outcomes hold for
};

// Mapping parameters after the reference's clamps are applied per read.
struct DevParams {
    int32_t seed_len, seed_stride, max_occ, max_diff, max_soft, max_adj, rescue_win;
};

// Packed read batch: per read r, 4 arrays of `words` u64 at
// base + r * 4 * words: forward codes, reverse-complement codes, N mask of
// the forward codes, N mask of the reverse complement.  Codes are 2 bits
// per base, base j of a word at bits 2*(j%32); an N mask has bit 2*(j%32)
// set where base j is not A/C/G/T.
struct DevReads {
    const uint64_t* packed;
    const uint32_t* lens;
    int32_t words;
    int64_t n_seq;
};

// One request's piece of a merged batch (pack_parts_kernel).
struct PackPart {
    uint64_t src;      // byte offset of the piece's first row in the staged bases
    int64_t row0;      // index of that row among all staged rows of the batch
    uint32_t c;        // pairs (or single reads) in the piece
    uint32_t max_len;  // row stride of the piece's staged rows
    int32_t bs_r1, bs_r2;
    uint32_t dst;      // batch pair offset of the piece's first pair
    uint32_t pad;
};

struct DevOut {
    int32_t* rid;
    uint32_t* pos;
    uint32_t* mapq;
    int32_t* flag;
    uint32_t* sl;
    uint32_t* sr;
    uint32_t* nm;
    uint64_t* uk;  // debug outputs, may be null
    uint64_t* ul;
    int32_t* us;
    int32_t* e;
    int32_t* score;
};

constexpr uint64_t kEven = 0x5555555555555555ull;

__device__ __forceinline__ uint64_t ldg64(const uint64_t* p) { return __ldg(p); }

// Count of symbol c in stored-BWT positions [0 .. x] (x < seq_len).
__device__ __forceinline__ uint64_t occ_at(const DevIndex& ix, uint64_t x, int c) {
    const uint4* p = reinterpret_cast<const uint4*>(ix.occ + (x >> 6));
    uint4 cnt = __ldg(p);
    uint4 bw = __ldg(p + 1);
    uint32_t base = c == 0 ? cnt.x : c == 1 ? cnt.y : c == 2 ? cnt.z : cnt.w;
    const uint64_t sb = __ldg(ix.occ_super + ((x >> ix.occ_super_shift) << 2) + c);
    uint64_t lo = static_cast<uint64_t>(bw.x) | (static_cast<uint64_t>(bw.y) << 32);
    uint64_t hi = static_cast<uint64_t>(bw.z) | (static_cast<uint64_t>(bw.w) << 32);
    uint64_t pat = static_cast<uint64_t>(c) * kEven;
    uint64_t tl = lo ^ pat, th = hi ^ pat;
    uint64_t ml = ~(tl | (tl >> 1)) & kEven;
    uint64_t mh = ~(th | (th >> 1)) & kEven;
    uint32_t w = static_cast<uint32_t>(x & 63);
    uint64_t keep_lo = w >= 31 ? ~0ull : ((1ull << (2 * w + 2)) - 1);
    uint64_t keep_hi = w < 32 ? 0ull : (w >= 63 ? ~0ull : ((1ull << (2 * (w - 32) + 2)) - 1));
    return sb + static_cast<uint64_t>(base) + __popcll(ml & keep_lo) + __popcll(mh & keep_hi);
}

// Occ(k, c) of the reference: count of c in BWT rows [0..k] (k a row index
// in [0, seq_len]), with the sentinel row `primary` removed
// (linear_gpu_fm.mojo:1261-1345).
__device__ __forceinline__ uint64_t occ_row(const DevIndex& ix, uint64_t k, int c) {
    if (k == ix.seq_len) return ix.L2[c + 1] - ix.L2[c];
    uint64_t x = k - (k >= ix.primary ? 1 : 0);
    return occ_at(ix, x, c);
}

// Text position of SA row `row` (one 16-byte load in either layout).
__device__ __forceinline__ uint64_t sa_at(const DevIndex& ix, uint64_t row) {
    if (!ix.sa_wide) return __ldg(ix.sa + row);
    const uint64_t ch = row / 3;
    const uint32_t slot = static_cast<uint32_t>(row - ch * 3);
    const uint4 v = __ldg(ix.sa40 + ch);
    const uint64_t lo = static_cast<uint64_t>(v.x) | (static_cast<uint64_t>(v.y) << 32);
    const uint64_t hi = static_cast<uint64_t>(v.z) | (static_cast<uint64_t>(v.w) << 32);
    const uint64_t r = slot == 0 ? lo : (slot == 1 ? (lo >> 40) | (hi << 24) : hi >> 16);
    return r & SA40_UNSET;
}

// Interval (k, l) of a packed k-mer table entry; false when the entry is
// KMER_UNTABLED (the caller searches without the table).  An empty
// interval comes back as k = 1 > l = 0.
__device__ __forceinline__ bool kmer_interval(uint64_t e, uint64_t& k, uint64_t& l) {
    if (e == KMER_UNTABLED) return false;
    const uint64_t cnt = e >> KMER_K_BITS;
    if (cnt == 0) {
        k = 1;
        l = 0;
    } else {
        k = e & KMER_K_MASK;
        l = k + cnt - 1;
    }
    return true;
}

// Symbol of the stored BWT at position x.
__device__ __forceinline__ int bwt_sym(const OccLine* __restrict__ occ, uint64_t x) {
    uint32_t w = __ldg(&occ[x >> 6].w[(x >> 4) & 3]);
    return static_cast<int>((w >> (2 * (x & 15))) & 3);
}

// 32 text bases starting at forward text position p, p in [-512, l_pac+480).
__device__ __forceinline__ uint64_t ref_window(const uint64_t* __restrict__ pacw, int64_t p) {
    int64_t q = p + 32 * PAC_PAD;
    uint64_t wi = static_cast<uint64_t>(q) >> 5;
    int sh = static_cast<int>(q & 31) * 2;
    uint64_t lo = ldg64(pacw + wi), hi = ldg64(pacw + wi + 1);
    return sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
}

// Even-bit mask for read positions [a, b) inside the word starting at 32*w.
__device__ __forceinline__ uint64_t range_mask(int w, int a, int b) {
    int lo = a - 32 * w, hi = b - 32 * w;
    if (lo < 0) lo = 0;
    if (hi > 32) hi = 32;
    if (hi <= lo) return 0;
    uint64_t m_hi = hi >= 32 ? ~0ull : ((1ull << (2 * hi)) - 1);
    uint64_t m_lo = (1ull << (2 * lo)) - 1;
    return m_hi & ~m_lo & kEven;
}

// Device buffers of one resident index (owned by an ma_index).
struct DeviceIndexBuffers {
    OccLine* occ = nullptr;
    unsigned long long* occ_super = nullptr;
    uint32_t* sa = nullptr;
    uint4* sa40 = nullptr;
    uint64_t* pacw = nullptr;
    uint64_t* kmer = nullptr;
    uint64_t* kmer3[2] = {nullptr, nullptr};
    uint16_t* summary = nullptr;
    uint4* atw = nullptr;
    uint64_t* coff = nullptr;
    uint32_t* clen = nullptr;
    uint64_t bytes = 0;
};

// Layout choices of the resident index (all result-neutral).
struct LayoutOptions {
    int kmer_k = 12;
    int kmer3_k = 0;
    bool wide_rows = false;         // 40-bit SA rows even when u32 would do
    int occ_super_shift = OCC_SUPER_SHIFT;
    uint64_t prep_chunk_rows = 0;   // rows per preparation pass (0 = automatic)
    int at_k = 0;                   // A/T window outcome table: window length (0 = none)
    int at_seed_len = 0;            // and the seed length its outcomes hold for
};

struct BwaIndexHost;
uint64_t pow3(int k);
uint64_t device_index_bytes(const BwaIndexHost& h, const LayoutOptions& lo);
uint64_t device_index_staging_bytes(const BwaIndexHost& h, const LayoutOptions& lo);
DevIndex build_device_index(const BwaIndexHost& h, const LayoutOptions& lo, cudaStream_t st,
                            DeviceIndexBuffers& bufs, uint64_t* reject_below);
void free_device_index(DeviceIndexBuffers& b);

}  // namespace ma
