// bgzf.cu - BGZF members compressed on the device.
//
// Replaces the BGZF layer of the reference's BAM writer
// (fq2bam-meth/python/bam_emit.py: _bgzf_block L77-98, _BgzfWriter
// L101-186): the uncompressed stream is cut every 65280 bytes, each piece
// becomes one gzip member with the BC extra field holding its size, the
// deflate data, the CRC-32 and the length, and the 28-byte EOF member ends
// the file.  The reference runs zlib (level 1) on a host thread pool; here
// one CTA compresses one piece at a time with everything in shared memory:
//
//   * CRC-32: every thread folds 64 bytes with a byte table; the segment
//     remainders are combined by multiplying with x^(8k) mod P (GF(2)), and
//     the standard pre/post inversion is applied at the end.
//   * LZ77: positions are hashed on 3 bytes in phases of 1024; each
//     position links to the previous position with the same hash (from
//     earlier phases through a head table, inside its warp through
//     __match_any_sync) in a 32 KB ring of 16-bit links, and follows up to
//     `chain` links for its longest match (deflate's 32 KB window, 258
//     bytes at most).  Each 32-byte sub-block (one warp's positions of a
//     phase) is parsed greedily from its own start right after it is matched,
//     the warp walking it together with shuffles; matches are cut at the
//     sub-block's end, so the parse needs no cross-warp order.
//   * Huffman: dynamic codes (literal/length, distance, code-length
//     alphabets) built per piece: symbols ranked by (count, symbol) over a
//     warp, Huffman merge with two queues, lengths limited to 15 (7) bits by
//     moving codes down one level at a time until the Kraft sum fits,
//     canonical codes (RFC 1951 3.2.2).
//   * Bits: every thread counts the bits of its sub-blocks' tokens; a block
//     scan gives its offset and the thread ORs its codes into a shared-memory
//     word buffer.
//     A piece whose dynamic coding is not smaller than storing it is stored.
//
// Level 0 writes stored blocks exactly as zlib does for one compress +
// finish call: one final stored block up to 32767 bytes, a non-final one
// followed by an empty final one above that.
#include <cub/block/block_scan.cuh>
#include <cub/device/device_scan.cuh>

#include <string>

#include "bgzf.h"
#include "ma_internal.h"

namespace ma {
namespace {

constexpr int THREADS = 512;                   // two CTAs per SM
constexpr int SUB = 32;                        // bytes per parse sub-block
constexpr int NSUB = (BGZF_BLOCK + SUB - 1) / SUB;  // 2040
constexpr int SUBS_PER_THREAD = (NSUB + THREADS - 1) / THREADS;  // 4
static_assert(SUB == 32, "a parse sub-block is one warp's positions");
constexpr int WBITS = 13;
constexpr uint32_t WSIZE = 1u << WBITS;        // match window (deflate allows up to 32 KB)
constexpr uint32_t WMASK = WSIZE - 1;
constexpr int HBITS = 12;
constexpr int HSIZE = 1 << HBITS;
constexpr uint16_t NONE = 0xffff;              // no previous position
constexpr int CRC_SEG = 128;
constexpr uint32_t CRC_POLY = 0xedb88320u;     // CRC-32, reflected
constexpr int NLL = 286, NDIST = 30, NCL = 19;

void check_launch(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

size_t align256(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }

// ---- CRC-32 arithmetic in the reflected representation (bit 31 = x^0) ----

__device__ __forceinline__ uint32_t gf2_mul(uint32_t a, uint32_t b) {
    uint32_t r = 0;
    for (int i = 0; i < 32; ++i) {
        if (a & (0x80000000u >> i)) r ^= b;
        b = (b & 1u) ? (b >> 1) ^ CRC_POLY : b >> 1;
    }
    return r;
}

// x^k mod P
__device__ uint32_t gf2_xpow(uint64_t k) {
    uint32_t r = 0x80000000u, b = 0x40000000u;
    while (k) {
        if (k & 1) r = gf2_mul(r, b);
        b = gf2_mul(b, b);
        k >>= 1;
    }
    return r;
}

// ---- deflate symbol tables (RFC 1951 3.2.5) ----

__device__ __forceinline__ void length_code(uint32_t len, uint32_t& sym, uint32_t& ebits, uint32_t& eval) {
    if (len <= 10) {
        sym = 257 + len - 3;
        ebits = 0;
        eval = 0;
    } else if (len == 258) {
        sym = 285;
        ebits = 0;
        eval = 0;
    } else {
        const uint32_t v = len - 3;
        const uint32_t e = 31 - __clz(v) - 2;
        sym = 257 + 4 * e + (v >> e);
        ebits = e;
        eval = v & ((1u << e) - 1);
    }
}

__device__ __forceinline__ void dist_code(uint32_t dist, uint32_t& sym, uint32_t& ebits, uint32_t& eval) {
    const uint32_t v = dist - 1;
    if (v < 4) {
        sym = v;
        ebits = 0;
        eval = 0;
    } else {
        const uint32_t e = 31 - __clz(v) - 1;
        sym = 2 * e + (v >> e);
        ebits = e;
        eval = v & ((1u << e) - 1);
    }
}

// Order in which the code-length code lengths are sent.
__constant__ uint8_t CL_ORDER[NCL] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

// Scratch of the Huffman builder (one warp).
struct HuffScratch {
    uint32_t a[NLL];         // sorted weights -> in-place tree -> depths
    uint16_t sorted[NLL];    // symbols by ascending (count, symbol)
    uint32_t bl_count[16 + 8];
    uint32_t next_code[16];
};

constexpr int RANK_SLOTS = (NLL + 31) / 32;  // symbols per lane in the rank pass

__device__ __forceinline__ uint32_t A_len(uint32_t depth, int maxbits) {
    return depth > static_cast<uint32_t>(maxbits) ? maxbits : depth;
}

// Code lengths <= maxbits for counts freq[0, n) (at least two nonzero).
// Called by a whole warp.  The symbols are ranked by (count, symbol) with
// every lane holding its symbols in registers while the counts stream past;
// the optimal lengths come from the in-place algorithm of Moffat and
// Katajainen (1995) on the sorted counts (lane 0): the counts array becomes
// the tree (parent indices), then internal depths, then leaf depths; lengths
// above maxbits are pulled up and the Kraft sum restored by splitting
// shorter codes, and the lengths are dealt out again with the heaviest
// symbols taking the shortest.
__device__ void huff_lengths(const uint32_t* freq, int n, int maxbits, uint8_t* len, HuffScratch& hs, int lane) {
    uint32_t f[RANK_SLOTS], r[RANK_SLOTS];
    int used = 0;
#pragma unroll
    for (int k = 0; k < RANK_SLOTS; ++k) {
        const int i = lane + 32 * k;
        f[k] = i < n ? freq[i] : 0;
        r[k] = 0;
        used += __popc(__ballot_sync(0xffffffffu, f[k] != 0));
        if (i < n) len[i] = 0;
    }
    for (int j = 0; j < n; ++j) {
        const uint32_t g = freq[j];
        if (!g) continue;
#pragma unroll
        for (int k = 0; k < RANK_SLOTS; ++k) r[k] += g < f[k] || (g == f[k] && j < lane + 32 * k);
    }
#pragma unroll
    for (int k = 0; k < RANK_SLOTS; ++k)
        if (f[k]) hs.sorted[r[k]] = static_cast<uint16_t>(lane + 32 * k);
    if (lane < 16 + 8) hs.bl_count[lane] = 0;
    __syncwarp();
    const int m = used;
    for (int k = lane; k < m; k += 32) hs.a[k] = freq[hs.sorted[k]];
    __syncwarp();
    if (lane == 0) {
        uint32_t* A = hs.a;
        // tree: A[t] = weight of internal node t; a consumed node's slot
        // takes its parent's index
        A[0] += A[1];
        int root = 0, leaf = 2;
        for (int next = 1; next < m - 1; ++next) {
            if (leaf >= m || A[root] < A[leaf]) {
                A[next] = A[root];
                A[root++] = next;
            } else {
                A[next] = A[leaf++];
            }
            if (leaf >= m || (root < next && A[root] < A[leaf])) {
                A[next] += A[root];
                A[root++] = next;
            } else {
                A[next] += A[leaf++];
            }
        }
        // internal depths
        A[m - 2] = 0;
        for (int t = m - 3; t >= 0; --t) A[t] = A[A[t]] + 1;
        // leaf depths, heaviest leaf (index m - 1) first
        int avail = 1, nused = 0, depth = 0, rt = m - 2, nx = m - 1;
        while (avail > 0) {
            while (rt >= 0 && static_cast<int>(A[rt]) == depth) {
                ++nused;
                --rt;
            }
            while (avail > nused) {
                A[nx--] = depth;
                --avail;
            }
            avail = 2 * nused;
            ++depth;
            nused = 0;
        }
    }
    __syncwarp();
    for (int k = lane; k < m; k += 32) atomicAdd(&hs.bl_count[A_len(hs.a[k], maxbits)], 1u);
    __syncwarp();
    if (lane == 0) {
        uint32_t kraft = 0;
        for (int b = 1; b <= maxbits; ++b) kraft += hs.bl_count[b] << (maxbits - b);
        while (kraft > (1u << maxbits)) {
            --hs.bl_count[maxbits];
            for (int b = maxbits - 1; b > 0; --b) {
                if (hs.bl_count[b]) {
                    --hs.bl_count[b];
                    hs.bl_count[b + 1] += 2;
                    break;
                }
            }
            --kraft;
        }
    }
    __syncwarp();
    // the rank-th heaviest symbol takes the rank-th shortest length
    for (int k = lane; k < m; k += 32) {
        const uint32_t rank = m - 1 - k;
        uint32_t cum = 0;
        int b = 1;
        for (; b < maxbits; ++b) {
            cum += hs.bl_count[b];
            if (rank < cum) break;
        }
        len[hs.sorted[k]] = static_cast<uint8_t>(b);
    }
    __syncwarp();
}

// Canonical codes, bit-reversed for LSB-first output (RFC 1951 3.2.2):
// symbol i of length l gets next_code[l] plus the number of earlier
// symbols of length l, counted 32 symbols at a time with __match_any_sync.
__device__ void huff_codes(const uint8_t* len, int n, uint16_t* code, HuffScratch& hs, int lane) {
    if (lane < 16) hs.bl_count[lane] = 0;
    __syncwarp();
    for (int i = lane; i < n; i += 32)
        if (len[i]) atomicAdd(&hs.bl_count[len[i]], 1u);
    __syncwarp();
    if (lane == 0) {
        uint32_t c = 0;
        for (int b = 1; b < 16; ++b) {
            c = (c + (b > 1 ? hs.bl_count[b - 1] : 0)) << 1;
            hs.next_code[b] = c;
        }
    }
    __syncwarp();
    for (int base = 0; base < n; base += 32) {
        const int i = base + lane;
        const uint32_t l = i < n ? len[i] : 0;
        const uint32_t peers = __match_any_sync(0xffffffffu, l);
        const uint32_t c = (l ? hs.next_code[l] : 0) + __popc(peers & ((1u << lane) - 1));
        if (i < n) code[i] = l ? static_cast<uint16_t>(__brev(c) >> (32 - l)) : 0;
        __syncwarp();
        if (l && lane == 31 - __clz(peers)) hs.next_code[l] += __popc(peers);
        __syncwarp();
    }
}

// Everything one CTA keeps for its two pieces in flight (the one being
// matched and the one being coded); under half of an SM's shared memory, so
// two CTAs run per SM.
struct Smem {
    union {
        uint8_t data[BGZF_BLOCK + 64];
        uint32_t out[(BGZF_BLOCK + 64) / 4];  // deflate bits, once the tokens hold the data
    } u;
    uint16_t prev[WSIZE];  // LZ77 links, a ring over the window
    uint32_t head[HSIZE];  // per hash: last position + 1 of earlier phases
    uint32_t crc_seg[THREADS];
    uint32_t crc_tab[256];
    uint32_t freq_ll[2][NLL + 2], freq_d[2][NDIST + 2], freq_cl[NCL + 1];  // [piece & 1]
    uint16_t code_ll[NLL + 2], code_d[NDIST + 2], code_cl[NCL + 1];
    uint8_t len_ll[NLL + 2], len_d[NDIST + 2], len_cl[NCL + 1];
    uint8_t sub_cnt[2][NSUB];
    uint8_t lens_all[NLL + NDIST];
    uint16_t rle[NLL + NDIST];  // code-length symbol | extra value << 5
    uint32_t hdr[112];          // header bits
    HuffScratch hs;
    uint32_t hdr_bits, n_rle, crc[2], x_seg, x_lane, lane_len[32], lane_crc[32];
    uint32_t nl_nd[2];
    typename cub::BlockScan<uint32_t, THREADS>::TempStorage scan;
};
// two CTAs per SM: 228 KB of shared memory, 1 KB of it reserved per CTA
static_assert(2 * (sizeof(Smem) + 1024) <= 228 * 1024, "two CTAs per SM");

// Four bytes of the piece starting at byte i (two aligned shared loads).
__device__ __forceinline__ uint32_t load4(const uint32_t* w, uint32_t i) {
    return __funnelshift_r(w[i >> 2], w[(i >> 2) + 1], 8 * (i & 3));
}

// Length of the common prefix of the piece at q and at p, at most lim
// (reads may run into the 64 padding bytes; the result is clamped).
__device__ __forceinline__ uint32_t match_len(const uint32_t* w, uint32_t q, uint32_t p, uint32_t lim) {
    uint32_t L = 0;
    while (L < lim) {
        const uint32_t x = load4(w, q + L) ^ load4(w, p + L);
        if (x) {
            L += (__ffs(x) - 1) >> 3;
            break;
        }
        L += 4;
    }
    return L < lim ? L : lim;
}

__device__ __forceinline__ uint32_t hash3(const uint8_t* d) {
    const uint32_t v = (static_cast<uint32_t>(d[0]) << 16) | (static_cast<uint32_t>(d[1]) << 8) | d[2];
    return (v * 2654435761u) >> (32 - HBITS);
}

// Bit writer over a word buffer: bits go LSB first; words are ORed so
// neighbouring writers may share a word.
struct BitOut {
    uint32_t* words;
    uint64_t acc;
    uint32_t nacc, w;
    __device__ BitOut(uint32_t* buf, uint32_t bitpos) : words(buf), acc(0), nacc(bitpos & 31), w(bitpos >> 5) {}
    __device__ __forceinline__ void put(uint32_t v, uint32_t nbits) {
        acc |= static_cast<uint64_t>(v) << nacc;
        nacc += nbits;
        if (nacc >= 32) {
            atomicOr(&words[w++], static_cast<uint32_t>(acc));
            acc >>= 32;
            nacc -= 32;
        }
    }
    __device__ __forceinline__ void flush() {
        if (nacc) atomicOr(&words[w], static_cast<uint32_t>(acc));
    }
};

// Sequential writer into the (zeroed) header words (one thread).
__device__ __forceinline__ void hdr_put(uint32_t* hdr, uint32_t& pos, uint32_t v, uint32_t nbits) {
    const uint64_t x = static_cast<uint64_t>(v) << (pos & 31);
    hdr[pos >> 5] |= static_cast<uint32_t>(x);
    if ((pos & 31) + nbits > 32) hdr[(pos >> 5) + 1] |= static_cast<uint32_t>(x >> 32);
    pos += nbits;
}

// One atomic per distinct symbol of the warp's active lanes.
__device__ __forceinline__ void warp_count(uint32_t* freq, uint32_t sym, bool on) {
    const uint32_t act = __ballot_sync(0xffffffffu, on);
    if (!on) return;
    const uint32_t same = __match_any_sync(act, sym);
    if ((threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(&freq[sym], static_cast<uint32_t>(__popc(same)));
}

__device__ __forceinline__ void token_bits(const Smem& S, uint32_t tokv, uint32_t& bits) {
    if ((tokv >> 16) == 0) {
        bits += S.len_ll[tokv];
    } else {
        uint32_t sym, eb, ev, dsym, deb, dev;
        length_code(tokv >> 16, sym, eb, ev);
        dist_code(tokv & 0xffff, dsym, deb, dev);
        bits += S.len_ll[sym] + eb + S.len_d[dsym] + deb;
    }
}

// CRC-32 of the piece from the segment remainders (one warp): each lane
// folds its run of segments, lane 0 folds the lanes, and the
// standard initial and final inversion contribute F x^(8n) + F.
__device__ void crc_combine(Smem& S, uint32_t n, int lane, int buf) {
    const uint32_t x64 = S.x_seg, x2048 = S.x_lane;
    uint32_t c = 0, len = 0;
    constexpr int PER_LANE = THREADS / 32;
    for (int k = 0; k < PER_LANE; ++k) {
        const uint32_t s0 = (lane * PER_LANE + k) * CRC_SEG;
        if (s0 >= n) break;
        const uint32_t sl = s0 + CRC_SEG <= n ? CRC_SEG : n - s0;
        c = gf2_mul(c, sl == CRC_SEG ? x64 : gf2_xpow(8ull * sl)) ^ S.crc_seg[lane * PER_LANE + k];
        len += sl;
    }
    S.lane_crc[lane] = c;
    S.lane_len[lane] = len;
    __syncwarp();
    if (lane == 0) {
        uint32_t r = 0;
        for (int l = 0; l < 32; ++l) {
            const uint32_t ll = S.lane_len[l];
            if (ll) r = gf2_mul(r, ll == (THREADS / 32) * CRC_SEG ? x2048 : gf2_xpow(8ull * ll)) ^ S.lane_crc[l];
        }
        S.crc[buf] = r ^ gf2_mul(0xffffffffu, gf2_xpow(8ull * n)) ^ 0xffffffffu;
    }
}

// The member's 18-byte header (BC extra field with BSIZE = member - 1) and
// 8-byte trailer, _bgzf_block L77-98.
__device__ void write_frame(uint8_t* slot, uint32_t payload, uint32_t crc, uint32_t n, int t) {
    const uint32_t bsize = 25 + payload;
    if (t < 18) {
        const uint8_t h[18] = {31, 139, 8, 4, 0, 0, 0, 0, 0, 255, 6, 0, 66, 67, 2, 0,
                               static_cast<uint8_t>(bsize & 255), static_cast<uint8_t>(bsize >> 8)};
        slot[t] = h[t];
    } else if (t < 26) {
        const int k = t - 18;
        const uint32_t v = k < 4 ? crc : n;
        slot[18 + payload + k] = static_cast<uint8_t>(v >> (8 * (k & 3)));
    }
}

// ---- the stages of one piece ----

// Piece bytes into shared memory (64 zero bytes after them), its CRC
// segment remainders, and a cleared head table and symbol counts.
__device__ void load_piece(Smem& S, const uint8_t* src, uint32_t n, int buf, int t) {
    if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
        const uint4* s4 = reinterpret_cast<const uint4*>(src);
        uint4* d4 = reinterpret_cast<uint4*>(S.u.data);
        for (uint32_t i = t; i < n / 16; i += THREADS) d4[i] = s4[i];
        for (uint32_t i = (n & ~15u) + t; i < n + 64; i += THREADS) S.u.data[i] = i < n ? src[i] : 0;
    } else {
        for (uint32_t i = t; i < n + 64; i += THREADS) S.u.data[i] = i < n ? src[i] : 0;
    }
    for (int i = t; i < HSIZE; i += THREADS) S.head[i] = 0;
    for (int i = t; i < NLL + 2; i += THREADS) S.freq_ll[buf][i] = 0;
    if (t < NDIST + 2) S.freq_d[buf][t] = 0;
    __syncthreads();
    const uint32_t s0 = t * CRC_SEG, s1 = s0 + CRC_SEG < n ? s0 + CRC_SEG : n;
    uint32_t c = 0;
    for (uint32_t i = s0; i < s1; ++i) c = (c >> 8) ^ S.crc_tab[(c ^ S.u.data[i]) & 255u];
    S.crc_seg[t] = c;
}

constexpr int MATCH_WARPS = THREADS / 32 - 1;  // warp 0 builds codes meanwhile
constexpr uint32_t PHASE = MATCH_WARPS * 32;   // positions per matching phase

// Barrier of the matching warps only (warps 1..15); warp 0 never takes it.
__device__ __forceinline__ void match_barrier() { asm volatile("bar.sync 1, %0;" ::"n"(PHASE) : "memory"); }

// LZ77 + greedy parse of the piece in shared memory by warps 1..15:
// phases of PHASE positions (one thread each); tokens to `tok`, symbol
// counts to freq[buf], token counts per 32-byte sub-block to sub_cnt[buf].
__device__ void match_piece(Smem& S, uint32_t n, int chain, uint32_t* tok, int buf, int wt, int lane, int mw) {
    const uint32_t n_phase = (n + PHASE - 1) / PHASE;
    for (uint32_t k = 0; k < n_phase; ++k) {
        const uint32_t p = k * PHASE + wt;
        const bool valid = p + 3 <= n;
        const uint32_t h = valid ? hash3(S.u.data + p) : 0;
        const uint32_t same = __match_any_sync(0xffffffffu, valid ? h : (0x80000000u | wt));
        const uint32_t lower = same & ((1u << lane) - 1);
        uint32_t prev_p = NONE;
        if (valid) {
            if (lower) {
                prev_p = p - (lane - (31 - __clz(lower)));
            } else {
                const uint32_t hv = S.head[h];
                prev_p = hv ? hv - 1 : NONE;
            }
        }
        if (p < n) S.prev[p & WMASK] = static_cast<uint16_t>(prev_p);
        match_barrier();
        uint32_t bm = 0;
        if (valid) {
            const uint32_t sub_end = (p & ~static_cast<uint32_t>(SUB - 1)) + SUB;
            const uint32_t lim = (sub_end < n ? sub_end : n) - p;
            if (lim >= 3) {
                uint32_t q = prev_p, best_len = 2, best_d = 0;
                for (int c = 0; c < chain && q != NONE && q < p && p - q <= WSIZE; ++c) {
                    // a candidate can only win if it also matches the byte
                    // just past the current best
                    const bool may = best_len >= lim || S.u.data[q + best_len] == S.u.data[p + best_len];
                    const uint32_t L = may ? match_len(S.u.out, q, p, lim) : 0;
                    if (L > best_len) {
                        best_len = L;
                        best_d = p - q;
                        if (L == lim) break;
                    }
                    const uint32_t nq = S.prev[q & WMASK];
                    if (nq == NONE || nq >= q) break;
                    q = nq;
                }
                if (best_len >= 3) bm = (best_len << 16) | best_d;
            }
        }
        if (valid) atomicMax(&S.head[h], p + 1);
        // greedy parse of this warp's 32-byte sub-block, which its lanes just
        // matched: the walk position is warp-uniform, the lane at that
        // position hands over its match by shuffle; token i ends up in lane i
        const uint32_t s0 = k * PHASE + 32 * mw;
        if (s0 < n) {
            const uint32_t e = n - s0 < SUB ? n - s0 : SUB;
            const uint32_t lit = p < n ? S.u.data[p] : 0;
            uint32_t q = 0, cnt = 0, mine = 0;
            while (q < e) {
                const uint32_t m = __shfl_sync(0xffffffffu, bm, q);
                const uint32_t tv = m ? m : __shfl_sync(0xffffffffu, lit, q);
                if (lane == cnt) mine = tv;
                ++cnt;
                q += m ? (m >> 16) : 1;
            }
            const bool on = lane < cnt;
            const bool is_match = on && (mine >> 16) != 0;
            uint32_t sym = mine, eb, ev, dsym = 0;
            if (is_match) {
                length_code(mine >> 16, sym, eb, ev);
                dist_code(mine & 0xffff, dsym, eb, ev);
            }
            warp_count(S.freq_ll[buf], sym, on);
            warp_count(S.freq_d[buf], dsym, is_match);
            if (on) tok[s0 + lane] = mine;
            if (lane == 0) S.sub_cnt[buf][s0 / SUB] = static_cast<uint8_t>(cnt);
        }
        match_barrier();
    }
}

// Dynamic Huffman codes of a matched piece from freq[buf], and the block
// header bits (warp 0).
__device__ void build_codes(Smem& S, int buf, int lane) {
    uint32_t* freq_ll = S.freq_ll[buf];
    uint32_t* freq_d = S.freq_d[buf];
    for (int i = lane; i < 112; i += 32) S.hdr[i] = 0;
    if (lane < NCL + 1) S.freq_cl[lane] = 0;
    if (lane == 0) {
        freq_ll[256] += 1;  // end of block
        // at least two codes in each alphabet
        int used = 0;
        for (int i = 0; i < NLL; ++i) used += freq_ll[i] != 0;
        if (used < 2) freq_ll[freq_ll[0] ? 1 : 0] = 1;
        used = 0;
        for (int i = 0; i < NDIST; ++i) used += freq_d[i] != 0;
        for (int i = 0; used < 2; ++i)
            if (!freq_d[i]) {
                freq_d[i] = 1;
                ++used;
            }
    }
    __syncwarp();
    huff_lengths(freq_ll, NLL, 15, S.len_ll, S.hs, lane);
    huff_lengths(freq_d, NDIST, 15, S.len_d, S.hs, lane);
    huff_codes(S.len_ll, NLL, S.code_ll, S.hs, lane);
    huff_codes(S.len_d, NDIST, S.code_d, S.hs, lane);
    if (lane == 0) {
        int nl = NLL, nd = NDIST;
        while (nl > 257 && !S.len_ll[nl - 1]) --nl;
        while (nd > 1 && !S.len_d[nd - 1]) --nd;
        for (int i = 0; i < nl; ++i) S.lens_all[i] = S.len_ll[i];
        for (int i = 0; i < nd; ++i) S.lens_all[nl + i] = S.len_d[i];
        // run-length code the lengths: 16 = repeat the previous length
        // 3..6 times, 17 / 18 = 3..10 / 11..138 zeros
        const int tot = nl + nd;
        uint32_t nr = 0;
        for (int i = 0; i < tot;) {
            const uint32_t v = S.lens_all[i];
            int run = 1;
            while (i + run < tot && S.lens_all[i + run] == v) ++run;
            i += run;
            if (v == 0) {
                while (run >= 11) {
                    const int k = run < 138 ? run : 138;
                    S.rle[nr++] = static_cast<uint16_t>(18 | (k - 11) << 5);
                    run -= k;
                }
                if (run >= 3) {
                    S.rle[nr++] = static_cast<uint16_t>(17 | (run - 3) << 5);
                    run = 0;
                }
                while (run-- > 0) S.rle[nr++] = 0;
            } else {
                S.rle[nr++] = static_cast<uint16_t>(v);
                --run;
                while (run >= 3) {
                    const int k = run < 6 ? run : 6;
                    S.rle[nr++] = static_cast<uint16_t>(16 | (k - 3) << 5);
                    run -= k;
                }
                while (run-- > 0) S.rle[nr++] = static_cast<uint16_t>(v);
            }
        }
        S.n_rle = nr;
        for (uint32_t i = 0; i < nr; ++i) ++S.freq_cl[S.rle[i] & 31];
        int used = 0;
        for (int i = 0; i < NCL; ++i) used += S.freq_cl[i] != 0;
        for (int i = 0; used < 2; ++i)
            if (!S.freq_cl[i]) {
                S.freq_cl[i] = 1;
                ++used;
            }
        S.nl_nd[0] = nl;
        S.nl_nd[1] = nd;
    }
    __syncwarp();
    huff_lengths(S.freq_cl, NCL, 7, S.len_cl, S.hs, lane);
    huff_codes(S.len_cl, NCL, S.code_cl, S.hs, lane);
    if (lane == 0) {
        const uint32_t nl = S.nl_nd[0], nd = S.nl_nd[1];
        int hclen = NCL;
        while (hclen > 4 && !S.len_cl[CL_ORDER[hclen - 1]]) --hclen;
        uint32_t pos = 0;
        hdr_put(S.hdr, pos, 1, 1);  // BFINAL
        hdr_put(S.hdr, pos, 2, 2);  // BTYPE = dynamic
        hdr_put(S.hdr, pos, nl - 257, 5);
        hdr_put(S.hdr, pos, nd - 1, 5);
        hdr_put(S.hdr, pos, hclen - 4, 4);
        for (int i = 0; i < hclen; ++i) hdr_put(S.hdr, pos, S.len_cl[CL_ORDER[i]], 3);
        for (uint32_t i = 0; i < S.n_rle; ++i) {
            const uint32_t r = S.rle[i], sym = r & 31, ex = r >> 5;
            hdr_put(S.hdr, pos, S.code_cl[sym], S.len_cl[sym]);
            if (sym == 16) hdr_put(S.hdr, pos, ex, 2);
            else if (sym == 17) hdr_put(S.hdr, pos, ex, 3);
            else if (sym == 18) hdr_put(S.hdr, pos, ex, 7);
        }
        S.hdr_bits = pos;
    }
    __syncwarp();
}

// Stored deflate blocks of a piece with zlib's framing for one compress +
// finish call, read from `src`.
__device__ void write_stored(uint8_t* slot, const uint8_t* src, uint32_t n, uint32_t crc, uint32_t* size, int t) {
    const uint32_t two = n > 32767;
    const uint32_t payload = n + (two ? 10 : 5);
    uint8_t* pl = slot + 18;
    for (uint32_t i = t; i < n; i += THREADS) pl[5 + i] = src[i];
    if (t == 0) {
        pl[0] = two ? 0 : 1;
        pl[1] = n & 255;
        pl[2] = n >> 8;
        pl[3] = ~n & 255;
        pl[4] = (~n >> 8) & 255;
        if (two) {
            const uint8_t e[5] = {1, 0, 0, 255, 255};
            for (int k = 0; k < 5; ++k) pl[5 + n + k] = e[k];
        }
        *size = 26 + payload;
    }
    write_frame(slot, payload, crc, n, t);
}

// Bits of a coded piece (all threads): per-thread bit counts of its
// sub-blocks, a block scan, the codes ORed into the shared word buffer
// (which reuses the piece bytes), the member to its slot; stored instead
// when that is not larger.  `src` is the piece in global memory.
__device__ void emit_piece(Smem& S, const uint32_t* tok, const uint8_t* src, uint32_t n, int buf, uint8_t* slot,
                           uint32_t* size, int t) {
    const uint32_t n_sub = (n + SUB - 1) / SUB;
    const uint8_t* sub_cnt = S.sub_cnt[buf];
    uint32_t bits = 0;
    const uint32_t s_first = SUBS_PER_THREAD * t, s_last = s_first + SUBS_PER_THREAD;
    for (uint32_t s = s_first; s < s_last && s < n_sub; ++s) {
        const uint4* tv = reinterpret_cast<const uint4*>(tok + s * SUB);
        const uint32_t c = sub_cnt[s];
        for (uint32_t i = 0; i < c; i += 4) {
            const uint4 v = tv[i >> 2];
            token_bits(S, v.x, bits);
            if (i + 1 < c) token_bits(S, v.y, bits);
            if (i + 2 < c) token_bits(S, v.z, bits);
            if (i + 3 < c) token_bits(S, v.w, bits);
        }
    }
    uint32_t off, sum;
    cub::BlockScan<uint32_t, THREADS>(S.scan).ExclusiveSum(bits, off, sum);
    const uint32_t total = S.hdr_bits + sum + S.len_ll[256];
    const uint32_t dyn_bytes = (total + 7) / 8;
    const uint32_t stored_bytes = n + (n > 32767 ? 10 : 5);
    if (dyn_bytes >= stored_bytes) {
        write_stored(slot, src, n, S.crc[buf], size, t);
        return;
    }
    for (int i = t; i < static_cast<int>((BGZF_BLOCK + 64) / 4); i += THREADS) S.u.out[i] = 0;
    __syncthreads();
    for (uint32_t i = t; i < (S.hdr_bits + 31) / 32; i += THREADS) atomicOr(&S.u.out[i], S.hdr[i]);
    BitOut bo(S.u.out, S.hdr_bits + off);
    for (uint32_t s = s_first; s < s_last && s < n_sub; ++s) {
        const uint4* tv4 = reinterpret_cast<const uint4*>(tok + s * SUB);
        const uint32_t c = sub_cnt[s];
        for (uint32_t i = 0; i < c; i += 4) {
            const uint4 v = tv4[i >> 2];
            const uint32_t four[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (i + k >= c) break;
                const uint32_t tv = four[k];
                if ((tv >> 16) == 0) {
                    bo.put(S.code_ll[tv], S.len_ll[tv]);
                } else {
                    uint32_t sym, eb, ev;
                    length_code(tv >> 16, sym, eb, ev);
                    bo.put(S.code_ll[sym], S.len_ll[sym]);
                    if (eb) bo.put(ev, eb);
                    dist_code(tv & 0xffff, sym, eb, ev);
                    bo.put(S.code_d[sym], S.len_d[sym]);
                    if (eb) bo.put(ev, eb);
                }
            }
        }
    }
    bo.flush();
    if (t == 0) {
        BitOut eob(S.u.out, S.hdr_bits + sum);
        eob.put(S.code_ll[256], S.len_ll[256]);
        eob.flush();
    }
    __syncthreads();
    const uint8_t* ob = reinterpret_cast<const uint8_t*>(S.u.out);
    for (uint32_t i = t; i < dyn_bytes; i += THREADS) slot[18 + i] = ob[i];
    write_frame(slot, dyn_bytes, S.crc[buf], n, t);
    if (t == 0) *size = 26 + dyn_bytes;
}

// One CTA walks its pieces b = blockIdx.x + j gridDim.x.  At levels 1..9 it
// runs a two-stage pipeline: while warps 1..15 match piece j, warp 0 builds
// the codes of piece j-1 (and folds piece j's CRC); then all warps emit
// piece j-1.  Tokens and symbol counts are double-buffered by piece parity.
__global__ void __launch_bounds__(THREADS, 2)
    bgzf_kernel(const uint8_t* in, uint64_t n_total, uint32_t n_blocks, int level, int chain, uint8_t* slots,
                uint32_t* sizes, uint32_t* tok_all) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>(smem_raw);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int i = t; i < 256; i += THREADS) {
        uint32_t c = i;
        for (int k = 0; k < 8; ++k) c = (c & 1u) ? (c >> 1) ^ CRC_POLY : c >> 1;
        S.crc_tab[i] = c;
    }
    if (t == 0) {
        S.x_seg = gf2_xpow(8ull * CRC_SEG);
        S.x_lane = gf2_xpow(8ull * (THREADS / 32) * CRC_SEG);
    }
    auto piece_len = [&](uint32_t b) {
        const uint64_t base = static_cast<uint64_t>(b) * BGZF_BLOCK;
        return static_cast<uint32_t>(n_total - base < BGZF_BLOCK ? n_total - base : BGZF_BLOCK);
    };
    if (level == 0) {
        for (uint32_t b = blockIdx.x; b < n_blocks; b += gridDim.x) {
            const uint32_t n = piece_len(b);
            const uint8_t* src = in + static_cast<uint64_t>(b) * BGZF_BLOCK;
            __syncthreads();
            load_piece(S, src, n, 0, t);
            __syncthreads();
            if (warp == 0) crc_combine(S, n, lane, 0);
            __syncthreads();
            write_stored(slots + static_cast<size_t>(b) * 65536, src, n, S.crc[0], sizes + b, t);
        }
        return;
    }
    const uint32_t count = blockIdx.x < n_blocks ? (n_blocks - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    uint32_t* tok2 = tok_all + static_cast<size_t>(blockIdx.x) * 2 * BGZF_BLOCK;
    for (uint32_t j = 0; j <= count; ++j) {
        const bool cur = j < count, prv = j > 0;
        const uint32_t b = blockIdx.x + j * gridDim.x, bp = b - gridDim.x;
        const int buf = j & 1, pbuf = buf ^ 1;
        __syncthreads();  // the previous emission is done with shared memory
        const uint32_t n = cur ? piece_len(b) : 0;
        if (cur) load_piece(S, in + static_cast<uint64_t>(b) * BGZF_BLOCK, n, buf, t);
        __syncthreads();
        if (warp == 0) {
            if (cur) crc_combine(S, n, lane, buf);
            if (prv) build_codes(S, pbuf, lane);
        } else if (cur) {
            match_piece(S, n, chain, tok2 + buf * BGZF_BLOCK, buf, t - 32, lane, warp - 1);
        }
        __syncthreads();
        if (prv)
            emit_piece(S, tok2 + pbuf * BGZF_BLOCK, in + static_cast<uint64_t>(bp) * BGZF_BLOCK, piece_len(bp), pbuf,
                       slots + static_cast<size_t>(bp) * 65536, sizes + bp, t);
    }
}

// Members from their slots to their final offsets; the last CTA appends the
// EOF member.
__global__ void bgzf_pack_kernel(const uint8_t* slots, const uint32_t* sizes, const uint64_t* ends, uint32_t n_blocks,
                                 uint8_t* out, int append_eof) {
    for (uint32_t b = blockIdx.x; b < n_blocks; b += gridDim.x) {
        const uint64_t end = ends[b], len = sizes[b], start = end - len;
        const uint8_t* src = slots + static_cast<size_t>(b) * 65536;
        for (uint64_t i = threadIdx.x; i < len; i += blockDim.x) out[start + i] = src[i];
    }
    if (append_eof && blockIdx.x == 0) {
        const uint64_t end = n_blocks ? ends[n_blocks - 1] : 0;
        const uint8_t eof[BGZF_EOF_BYTES] = {31, 139, 8, 4, 0, 0, 0, 0, 0, 255, 6, 0, 66, 67,
                                             2,  0,   27, 0, 3, 0, 0, 0, 0, 0, 0,   0, 0, 0};
        if (threadIdx.x < BGZF_EOF_BYTES) out[end + threadIdx.x] = eof[threadIdx.x];
    }
}

int chain_for(int level) {
    static const int c[10] = {0, 4, 6, 8, 12, 16, 24, 32, 64, 128};
    return c[level < 0 ? 0 : (level > 9 ? 9 : level)];
}

}  // namespace

uint64_t bgzf_bound(uint64_t n_bytes) {
    const uint64_t nb = (n_bytes + BGZF_BLOCK - 1) / BGZF_BLOCK;
    return nb * (BGZF_MEMBER_MAX) + BGZF_EOF_BYTES;
}

namespace {
// CTAs of the compression kernel: two per SM.
uint64_t bgzf_grid(uint64_t nb, int sm_count) {
    const uint64_t g = 2ull * static_cast<uint64_t>(sm_count > 0 ? sm_count : 148);
    return nb < g ? nb : g;
}
}  // namespace

size_t bgzf_scratch_bytes(uint64_t n_bytes, int sm_count) {
    const uint64_t nb = (n_bytes + BGZF_BLOCK - 1) / BGZF_BLOCK;
    size_t t = 0;
    cub::DeviceScan::InclusiveSum(nullptr, t, static_cast<const uint32_t*>(nullptr), static_cast<uint64_t*>(nullptr),
                                  static_cast<int64_t>(nb ? nb : 1));
    const size_t grid = bgzf_grid(nb ? nb : 1, sm_count);
    // tokens (two pieces) per CTA, member slots, sizes, ends, scan temp
    return align256(grid * 2 * BGZF_BLOCK * 4) + align256(nb * 65536) + align256(nb * 4) + align256(nb * 8) +
           align256(t) + 256;
}

uint64_t bgzf_compress(const uint8_t* in, uint64_t n, int level, uint8_t* out, uint64_t out_cap, int append_eof,
                       void* scratch, size_t scratch_bytes, int sm_count, cudaStream_t st, uint64_t* need,
                       int* launches, float* kernel_ms) {
    const uint64_t nb = (n + BGZF_BLOCK - 1) / BGZF_BLOCK;
    const uint64_t gmax = bgzf_grid(nb ? nb : 1, sm_count);
    const int grid = static_cast<int>(nb < gmax ? nb : gmax);
    uint8_t* s = static_cast<uint8_t*>(scratch);
    uint32_t* tok = reinterpret_cast<uint32_t*>(s);
    s += align256(gmax * 2 * BGZF_BLOCK * 4);
    uint8_t* slots = s;
    s += align256(nb * 65536);
    uint32_t* sizes = reinterpret_cast<uint32_t*>(s);
    s += align256(nb * 4);
    uint64_t* ends = reinterpret_cast<uint64_t*>(s);
    s += align256(nb * 8);
    void* temp = s;
    size_t tb = scratch_bytes - (s - static_cast<uint8_t*>(scratch));
    *launches = 0;
    if (kernel_ms) *kernel_ms = 0;
    uint64_t total = 0;
    if (nb) {
        const size_t smem = sizeof(Smem);
        check_launch(cudaFuncSetAttribute(bgzf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(smem)),
                     "bgzf smem");
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (kernel_ms) {
            check_launch(cudaEventCreate(&e0), "event");
            check_launch(cudaEventCreate(&e1), "event");
            check_launch(cudaEventRecord(e0, st), "event");
        }
        bgzf_kernel<<<grid, THREADS, smem, st>>>(in, n, static_cast<uint32_t>(nb), level, chain_for(level), slots,
                                                 sizes, tok);
        check_launch(cudaGetLastError(), "bgzf_kernel");
        if (kernel_ms) check_launch(cudaEventRecord(e1, st), "event");
        check_launch(cub::DeviceScan::InclusiveSum(temp, tb, static_cast<const uint32_t*>(sizes), ends,
                                                   static_cast<int64_t>(nb), st),
                     "bgzf scan");
        check_launch(cudaMemcpyAsync(&total, ends + nb - 1, 8, cudaMemcpyDeviceToHost, st), "D2H bgzf size");
        check_launch(cudaStreamSynchronize(st), "bgzf");
        if (kernel_ms) {
            cudaEventElapsedTime(kernel_ms, e0, e1);
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
        }
        *launches = 3;
    }
    const uint64_t all = total + (append_eof ? BGZF_EOF_BYTES : 0);
    *need = all;
    if (all > out_cap) return 0;
    const unsigned pg = static_cast<unsigned>(nb ? (nb < 4096 ? nb : 4096) : 1);
    bgzf_pack_kernel<<<pg, 256, 0, st>>>(slots, sizes, ends, static_cast<uint32_t>(nb), out, append_eof);
    check_launch(cudaGetLastError(), "bgzf_pack_kernel");
    ++*launches;
    check_launch(cudaStreamSynchronize(st), "bgzf pack");
    return all;
}

}  // namespace ma
