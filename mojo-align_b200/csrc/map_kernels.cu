// map_kernels.cu - the mapping kernels of the linear bisulfite FM path.
//
//   pack_reads_kernel     _cvt + pack_bases_kernel
//                         (linear_fastq.mojo:37-46, linear_gpu_fm.mojo:1136-1154),
//                         fused into a 2-bit packing of both strands
//   seed_extend_kernel    fm_seed_extend_kernel (linear_gpu_fm.mojo:1156-1837)
//   mate_rescue_kernel    fm_mate_rescue_kernel (linear_gpu_fm.mojo:1839-2011)
//
// The exactness argument and the device functions shared with the
// wavefront kernels are in seed_core.cuh.
// Loop bounds: every loop runs over a read (<= 1024 bases), an SA interval
// (<= 16 rows, or 1), 2*adj_cap+1 <= 25 shifts, or a rescue window
// (<= 2049 positions); nothing waits on another thread.
#include <cuda_runtime.h>

#include "ma_device.cuh"
#include "seed_core.cuh"

namespace ma {

namespace {

// Word w of packed read row `row` (len bases, conversion `mode`): forward
// codes, reverse-complement codes and the two non-ACGT masks, each at
// `words` stride from `out`.
__device__ __forceinline__ void pack_word(const uint8_t* __restrict__ row, int len, int mode, int w, int words,
                                          uint64_t* __restrict__ out) {
    uint64_t f = 0, fn = 0, rw = 0, rn = 0;
    for (int i = 0; i < 32; ++i) {
        const int j = 32 * w + i;
        if (j >= len) break;
        const int c = code_of(cvt_base(row[j], mode));
        if (c > 3) fn |= 1ull << (2 * i);
        else f |= static_cast<uint64_t>(c) << (2 * i);
        const int c2 = code_of(cvt_base(row[len - 1 - j], mode));
        if (c2 > 3) rn |= 1ull << (2 * i);
        else rw |= static_cast<uint64_t>(3 - c2) << (2 * i);
    }
    out[w] = f;
    out[words + w] = rw;
    out[2 * words + w] = fn;
    out[3 * words + w] = rn;
}

// Source row r (stride max_len) lands at batch row dst1 + r for the first
// n1 rows and dst2 + (r - n1) after them; lens are read at the batch row.  A
// plain batch uses dst1 = 0, dst2 = n1.
__global__ void __launch_bounds__(256) pack_reads_kernel(const uint8_t* __restrict__ bases,
                                                         const uint32_t* __restrict__ lens, int64_t n_seq,
                                                         int64_t n1, int max_len, int words, int bs_r1,
                                                         int bs_r2, int64_t dst1, int64_t dst2,
                                                         uint64_t* __restrict__ packed, int* __restrict__ err) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t r = t / words;
    const int w = static_cast<int>(t - r * words);
    if (r >= n_seq) return;
    const int64_t d = r < n1 ? dst1 + r : dst2 + (r - n1);
    int len = static_cast<int>(lens[d]);
    if (len > max_len) {
        atomicExch(err, 1);
        len = max_len;
    }
    pack_word(bases + r * static_cast<int64_t>(max_len), len, r < n1 ? bs_r1 : bs_r2, w, words,
              packed + d * 4 * static_cast<int64_t>(words));
}

// Four bases at base[x .. x+3] (reversed: base[x+3] first) from 4-byte
// aligned loads; base must be 4-byte aligned.
__device__ __forceinline__ uint32_t load4(const uint8_t* base, int x, bool reversed) {
    const uint32_t* a = reinterpret_cast<const uint32_t*>(base + (x & ~3));
    const uint32_t o = static_cast<uint32_t>(x & 3) * 0x1111u;
    return __byte_perm(a[0], a[1], (reversed ? 0x0123u : 0x3210u) + o);
}

// 2-bit codes (bits 0,2,4,6) and N flags (bits 0,2,4,6) of four ASCII bases
// after conversion `mode` (linear_fastq.mojo:37-46): A/a 0, C/c 1, G/g 2,
// T/t 3 (C -> T under C2T, G -> A under G2A), anything else N (code 0).
// Bits 1-2 of the ASCII letters give the codes, ((b >> 1) ^ (b >> 2)) & 3;
// a byte is a base exactly when its upper-case form equals the letter of
// its code (a byte permute of "ACGT" by the codes).
__device__ __forceinline__ void codes4(uint32_t v, int mode, uint32_t& codes, uint32_t& nflags) {
    const uint32_t u = v & 0xDFDFDFDFu;
    uint32_t c = ((v >> 1) ^ (v >> 2)) & 0x03030303u;
    const uint32_t sel = (c & 0x3u) | ((c >> 4) & 0x30u) | ((c >> 8) & 0x300u) | ((c >> 12) & 0x3000u);
    const uint32_t x = u ^ __byte_perm(0x54474341u, 0u, sel);
    const uint32_t nz = (((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x) & 0x80808080u;  // high bit: byte not a base
    if (mode == MA_BS_C2T) c |= (c & ~(c >> 1) & 0x01010101u) << 1;
    if (mode == MA_BS_G2A) c &= ~(((c >> 1) & ~c & 0x01010101u) << 1);
    const uint32_t nb = nz >> 7;
    c &= ~(nb * 3u);
    codes = (c & 0x3u) | ((c >> 6) & 0xCu) | ((c >> 12) & 0x30u) | ((c >> 18) & 0xC0u);
    nflags = (nb & 0x1u) | ((nb >> 6) & 0x4u) | ((nb >> 12) & 0x10u) | ((nb >> 18) & 0x40u);
}

// Order of the 32 two-bit fields of a word reversed.
__device__ __forceinline__ uint64_t reverse_fields(uint64_t x) {
    const uint64_t y = __brevll(x);
    return ((y >> 1) & kEven) | ((y & kEven) << 1);
}

// One packed read from a staged row (`row` = its offset in the 4-byte
// aligned `base`): forward words from the bytes 4 bases at a time, then the
// reverse-complement words from the forward ones (fields reversed, shifted
// by 32 * ceil(len / 32) - len bases, complemented).  Reads may touch up to
// 7 bytes after the row's last base.
__device__ __forceinline__ void pack_row_staged(const uint8_t* base, int row, int len, int mode, int words,
                                                uint64_t* __restrict__ out) {
    const int wr = (len + 31) >> 5;     // words holding bases
    const int sh = 2 * (32 * wr - len);  // bits the reversed stream is shifted by
    uint64_t r_prev = 0, rn_prev = 0;    // reversed word j - 1
    for (int k = wr - 1; k >= 0; --k) {  // j = wr - 1 - k ascending
        uint64_t f = 0, fn = 0;
        for (int g = 0; g < 8; ++g) {
            if (32 * k + 4 * g >= len) break;
            uint32_t c, n;
            codes4(load4(base, row + 32 * k + 4 * g, false), mode, c, n);
            f |= static_cast<uint64_t>(c) << (8 * g);
            fn |= static_cast<uint64_t>(n) << (8 * g);
        }
        const int nv = len - 32 * k;
        const uint64_t keep = nv >= 32 ? ~0ull : ((1ull << (2 * nv)) - 1);
        f &= keep;
        fn &= keep;
        out[k] = f;
        out[2 * words + k] = fn;
        const uint64_t r = reverse_fields(f), rn = reverse_fields(fn);
        const int j = wr - 1 - k;
        if (j > 0) {
            // reverse-complement word j - 1 from reversed words j - 1 and j
            const uint64_t sr = sh ? ((r_prev >> sh) | (r << (64 - sh))) : r_prev;
            const uint64_t sn = sh ? ((rn_prev >> sh) | (rn << (64 - sh))) : rn_prev;
            out[words + j - 1] = (sr ^ ~0ull) & ~(sn * 3ull);
            out[3 * words + j - 1] = sn;
        }
        r_prev = r;
        rn_prev = rn;
    }
    if (wr > 0) {
        const int nv = len - 32 * (wr - 1);
        const uint64_t keep = nv >= 32 ? ~0ull : ((1ull << (2 * nv)) - 1);
        const uint64_t sr = r_prev >> sh, sn = rn_prev >> sh;
        out[words + wr - 1] = (sr ^ ~0ull) & ~(sn * 3ull) & keep;
        out[3 * words + wr - 1] = sn & keep;
    }
    for (int w = wr; w < words; ++w) {
        out[w] = 0;
        out[words + w] = 0;
        out[2 * words + w] = 0;
        out[3 * words + w] = 0;
    }
}

// Staged form of pack_reads_kernel: a block copies the bytes of its rows
// (one contiguous range of the row-major input) into shared memory with
// 16-byte loads, then packs one row per thread from there.
// rows_per_block * max_len must fit PACK_STAGE bytes.
constexpr int PACK_THREADS = 256;
constexpr int PACK_STAGE = 40960;
constexpr int PACK_SLACK = 16;  // before and after the staged bytes

__global__ void __launch_bounds__(PACK_THREADS) pack_rows_kernel(const uint8_t* __restrict__ bases,
                                                                const uint32_t* __restrict__ lens, int64_t n_seq,
                                                                int64_t n1, int max_len, int words,
                                                                int rows_per_block, int bs_r1, int bs_r2,
                                                                int64_t dst1, int64_t dst2,
                                                                uint64_t* __restrict__ packed,
                                                                int* __restrict__ err) {
    __shared__ __align__(16) uint8_t s_rows[PACK_SLACK + PACK_STAGE + 16 + PACK_SLACK];
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * rows_per_block;
    if (r0 >= n_seq) return;
    const int nr = static_cast<int>(n_seq - r0 < rows_per_block ? n_seq - r0 : rows_per_block);
    const uint8_t* g = bases + r0 * static_cast<int64_t>(max_len);
    const int bytes = nr * max_len;
    // s_rows[PACK_SLACK + off + j] = g[j]; off lines up the 16-byte
    // boundaries of g with those of s_rows
    const int off = static_cast<int>(reinterpret_cast<uintptr_t>(g) & 15);
    const int head = off ? (16 - off < bytes ? 16 - off : bytes) : 0;
    const int n16 = (bytes - head) >> 4;
    uint8_t* st = s_rows + PACK_SLACK + off;
    for (int j = threadIdx.x; j < head; j += blockDim.x) st[j] = g[j];
    const uint4* g16 = reinterpret_cast<const uint4*>(g + head);
    uint4* s16 = reinterpret_cast<uint4*>(st + head);
    for (int k = threadIdx.x; k < n16; k += blockDim.x) s16[k] = __ldg(g16 + k);
    for (int j = head + 16 * n16 + threadIdx.x; j < bytes; j += blockDim.x) st[j] = g[j];
    __syncthreads();
    for (int lr = threadIdx.x; lr < nr; lr += blockDim.x) {
        const int64_t r = r0 + lr;
        const int64_t d = r < n1 ? dst1 + r : dst2 + (r - n1);
        int len = static_cast<int>(lens[d]);
        if (len > max_len) {
            atomicExch(err, 1);
            len = max_len;
        }
        pack_row_staged(s_rows, PACK_SLACK + off + lr * max_len, len, r < n1 ? bs_r1 : bs_r2, words,
                        packed + d * 4 * static_cast<int64_t>(words));
    }
}

// A batch merged from several requests.  Part j holds c pairs (or single
// reads) staged at byte `src` of `bases`: its c first mates, then its c
// second mates, rows of stride max_len.  Its pair i lands at batch row
// dst + i and, when paired, n1_batch + dst + i.  Source rows of all parts
// are numbered consecutively from 0 (part j's first row is row0).
__global__ void __launch_bounds__(256) pack_parts_kernel(const uint8_t* __restrict__ bases,
                                                         const uint32_t* __restrict__ lens,
                                                         const PackPart* __restrict__ parts, int n_parts,
                                                         int64_t n_rows, int64_t n1_batch, int words,
                                                         uint64_t* __restrict__ packed, int* __restrict__ err) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t r = t / words;
    const int w = static_cast<int>(t - r * words);
    if (r >= n_rows) return;
    int lo = 0, hi = n_parts - 1;  // last part with row0 <= r
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (parts[mid].row0 <= r) lo = mid;
        else hi = mid - 1;
    }
    const PackPart pp = parts[lo];
    const int64_t local = r - pp.row0;
    const bool second = local >= pp.c;
    const int64_t i = second ? local - pp.c : local;
    const int64_t d = second ? n1_batch + pp.dst + i : pp.dst + i;
    int len = static_cast<int>(lens[d]);
    if (len > static_cast<int>(pp.max_len)) {
        atomicExch(err, 1);
        len = static_cast<int>(pp.max_len);
    }
    pack_word(bases + pp.src + local * static_cast<int64_t>(pp.max_len), len, second ? pp.bs_r2 : pp.bs_r1, w,
              words, packed + d * 4 * static_cast<int64_t>(words));
}

// Stage 1: one thread per read, right endpoints [0, ep_limit).  A read
// whose best hit is not nm == 0 and that has endpoints left is handed to
// stage 2 with its running best and the loci it evaluated.  With
// ep_limit >= every read's endpoint count this is the whole algorithm.
template <bool S, int MINB>
__global__ void __launch_bounds__(128, MINB) seed_stage1_kernel(DevIndex ix, DevReads R, DevParams P, DevOut out,
                                                          int ep_limit, int max_rows, Handoff h,
                                                          unsigned long long* __restrict__ tally_out) {
    const int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (r >= R.n_seq) return;
    Tally t{};
    const ReadView rd = read_view(R, r);
    const int qlen = rd.qlen;
    Best best;
    best.key = ~0ull;
    best.crid = -1;
    best.us = -1;
    best.e = -1;
    best.uk = best.ul = 0;
    constexpr int MEMO = 16;
    int64_t memo_b0[MEMO];
    int memo_n = 0;
    const int n_end = endpoint_count(P, qlen);
    const int n_run = n_end < ep_limit ? n_end : ep_limit;
    int resume = n_run;  // first endpoint stage 2 searches
    if (n_run > 0) {
        const Clamps cl = clamps_for(P, qlen);
        for (int ei = 0; ei < n_run; ++ei) {
            const int e = P.seed_len - 1 + ei * P.seed_stride;
            const Seed sd = search_endpoint<S>(ix, rd, e, P, t);
            if (!sd.found) continue;
            if (h.pending && sd.l - sd.k >= static_cast<uint64_t>(max_rows)) {
                // many SA rows: stage 2 spreads them over a warp
                resume = ei;
                break;
            }
            for (uint64_t hi = sd.k; hi <= sd.l; ++hi) {
                const uint64_t sa_pos = sa_at(ix, hi);
                if constexpr (S) t.sa_loads++;
                int64_t b0;
                int is_rev;
                if (!locus_of_row(ix, sa_pos, sd.s, e, qlen, b0, is_rev)) continue;
                // shortcut 1: a locus already evaluated cannot win again
                const int64_t tag = b0 * 2 + is_rev;
                bool seen = false;
                const int mn = memo_n < MEMO ? memo_n : MEMO;
                for (int i = 0; i < mn; ++i) seen |= memo_b0[i] == tag;
                if (seen) continue;
                memo_b0[memo_n % MEMO] = tag;
                ++memo_n;
                const uint32_t ord_row = (static_cast<uint32_t>(ei) * 16 + static_cast<uint32_t>(hi - sd.k)) * ADJ_SPAN;
                eval_locus<S>(ix, rd, b0, is_rev, cl.adj_cap, cl.budget, cl.clip_cap, ord_row, best, sd.k, sd.l,
                              sd.s, e, t);
                if ((best.key >> ORD_SHIFT) == 0) goto done;  // nm == 0 returns (L1708-1728)
            }
        }
    }
done:
    write_hit(out, r, best, qlen);
    {
        bool pend = h.pending && (best.key >> ORD_SHIFT) != 0 && n_end > resume;
        const int bnm = static_cast<int>(best.key >> ORD_SHIFT);
        if (pend && bnm <= 2 && full_compare_key(best.key)) {
            const int64_t bstart = static_cast<int64_t>(__ldg(ix.coff + best.crid)) + best.pos - best.sl;
            if (better_hit_impossible<S>(ix, rd, bstart, (best.flag & 16) ? 1 : 0, clamps_for(P, qlen).clip_cap, bnm,
                                         t))
                pend = false;
        }
        if (pend) {
            h.key[r] = best.key;
            h.resume[r] = static_cast<uint16_t>(resume);
            const int mn = memo_n < MEMO1 ? memo_n : MEMO1;
            for (int i = 0; i < mn; ++i) h.memo[r * MEMO1 + i] = static_cast<uint64_t>(memo_b0[i]);
            h.memo_n[r] = static_cast<uint8_t>(mn);
        }
        const unsigned m = __activemask();
        const unsigned b = __ballot_sync(m, pend);
        if (b) {
            const int lane = threadIdx.x & 31;
            const int leader = __ffs(b) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(h.counters, static_cast<uint32_t>(__popc(b)));
            base = __shfl_sync(m, base, leader);
            if (pend) h.pending[base + __popc(b & ((1u << lane) - 1))] = static_cast<uint32_t>(r);
        }
    }
    flush_tally<S>(t, tally_out);
}

// A locus staged for the warp's shift evaluations.
struct Locus {
    int64_t b0;
    uint64_t uk, ul;
    uint32_t ord_row;
    int32_t us, e, rev;
    ContigHint hint;
};

constexpr int S2_WARPS = 8;   // warps per block of the stage-2 kernel
constexpr int MEMO2 = 64;     // loci remembered per read in stage 2


// Stage 2: one warp per pending read, persistent over the pending list.
// Lanes search 32 right endpoints at a time; the candidate rows of those
// endpoints, in the reference's order (endpoint, then row), are resolved
// 32 at a time, de-duplicated (within the group by __match_any_sync,
// against earlier groups and stage 1 through the memo), and every (locus,
// shift) pair is evaluated by one lane.  The warp minimum of the (nm,
// ordinal) keys is folded into the read's running best.  The read stops
// after the group of endpoints in which an nm == 0 hit appears.
template <bool S, int MINB>
__global__ void __launch_bounds__(S2_WARPS * 32, MINB) seed_stage2_kernel(DevIndex ix, DevReads R, DevParams P,
                                                                    DevOut out, Handoff h, int first_wave,
                                                                    unsigned long long* __restrict__ tally_out) {
    __shared__ uint64_t s_words_all[S2_WARPS][4 * MAX_WORDS];
    __shared__ uint64_t s_memo_all[S2_WARPS][MEMO2];
    __shared__ Locus s_loci_all[S2_WARPS][32];
    constexpr unsigned FULL = 0xFFFFFFFFu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint64_t* s_words = s_words_all[warp];
    uint64_t* s_memo = s_memo_all[warp];
    Locus* s_loci = s_loci_all[warp];
    Tally t{};
    const uint32_t n_pending = *reinterpret_cast<volatile uint32_t*>(h.counters);
    for (;;) {
        uint32_t qi = 0;
        if (lane == 0) qi = atomicAdd(h.counters + 1, 1u);
        qi = __shfl_sync(FULL, qi, 0);
        if (qi >= n_pending) break;
        const int64_t r = h.pending[qi];
        if constexpr (S) t.s2_reads += lane == 0;
        const int words = R.words;
        const uint64_t* g = R.packed + r * 4 * static_cast<int64_t>(words);
        for (int i = lane; i < 4 * words; i += 32) s_words[i] = g[i];
        const int qlen = static_cast<int>(R.lens[r]);
        int n_memo = h.memo_n[r];
        for (int i = lane; i < n_memo; i += 32) s_memo[i] = h.memo[r * MEMO1 + i];
        __syncwarp();
        ReadView rd;
        rd.fwd = s_words;
        rd.rc = s_words + words;
        rd.nf = s_words + 2 * words;
        rd.nr = s_words + 3 * words;
        rd.qlen = qlen;
        const Clamps cl = clamps_for(P, qlen);
        const int n_end = endpoint_count(P, qlen);
        uint64_t best_key = h.key[r];
        uint64_t tested_key = best_key;  // stage 1 ran the early-stop test on its best
        Best win;  // valid when improved
        win.crid = -1;
        bool improved = false;
        int64_t best_tag = -1;  // locus of the best hit found in this stage (b0*2+strand)
        const bool can_predict = ix.summary && ix.kmer3_k > 0 && ix.kmer3_k <= P.seed_len;
        int width = first_wave;
        for (int j0 = h.resume[r]; j0 < n_end; j0 += width, width = 32) {
            if constexpr (S) t.s2_groups += lane == 0;
            const int j = j0 + lane;
            const int e = P.seed_len - 1 + j * P.seed_stride;
            Seed sd{0, 0, -1, false};
            if (lane < width && j < n_end) {
                const bool dup = can_predict && predicted_duplicate<S>(ix, rd, e, P, best_tag, s_memo,
                                                                       n_memo < 4 ? n_memo : 4, t);
                if constexpr (S) t.skipped += dup;
                if (!dup) sd = search_endpoint<S>(ix, rd, e, P, t);
            }
            const int nrows = sd.found ? static_cast<int>(sd.l - sd.k + 1) : 0;
            int incl = nrows;
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += v;
            }
            const int total = __shfl_sync(FULL, incl, 31);
            for (int c0 = 0; c0 < total; c0 += 32) {
                const int idx = c0 + lane;
                int owner = 0;  // lanes whose rows end at or before idx
                for (int step = 16; step >= 1; step >>= 1) {
                    const int v = __shfl_sync(FULL, incl, owner + step - 1);
                    if (v <= idx) owner += step;
                }
                const int own = owner < 32 ? owner : 31;
                const uint64_t o_k = __shfl_sync(FULL, sd.k, own);
                const uint64_t o_l = __shfl_sync(FULL, sd.l, own);
                const int o_s = __shfl_sync(FULL, sd.s, own);
                const int o_first = __shfl_sync(FULL, incl - nrows, own);
                const bool valid = idx < total;
                const int o_e = P.seed_len - 1 + (j0 + own) * P.seed_stride;
                const uint64_t hi = o_k + static_cast<uint64_t>(idx - o_first);
                uint64_t tag = 0x8000000000000000ull | static_cast<uint64_t>(lane);
                int64_t b0 = 0;
                int rev = 0;
                bool ok = false;
                if (valid) {
                    const uint64_t sa_pos = sa_at(ix, hi);
                    if constexpr (S) t.sa_loads++;
                    ok = locus_of_row(ix, sa_pos, o_s, o_e, qlen, b0, rev);
                    if (ok) tag = static_cast<uint64_t>(b0 * 2 + rev);
                }
                const unsigned peers = __match_any_sync(FULL, tag);
                bool keep = ok && (__ffs(peers) - 1) == lane;
                if (keep)
                    for (int m = 0; m < n_memo; ++m)
                        if (s_memo[m] == tag) {
                            keep = false;
                            break;
                        }
                const unsigned kb = __ballot_sync(FULL, keep);
                const int rank = __popc(kb & ((1u << lane) - 1));
                if (keep) {
                    if (n_memo + rank < MEMO2) s_memo[n_memo + rank] = tag;
                    Locus L;
                    L.b0 = b0;
                    L.uk = o_k;
                    L.ul = o_l;
                    L.ord_row = (static_cast<uint32_t>(j0 + own) * 16 + static_cast<uint32_t>(hi - o_k)) * ADJ_SPAN;
                    L.us = o_s;
                    L.e = o_e;
                    L.rev = rev;
                    L.hint = contig_hint(ix, b0);
                    s_loci[rank] = L;
                    if constexpr (S) tally_locus(t, b0, cl.adj_cap, qlen);
                }
                n_memo += __popc(kb);
                if (n_memo > MEMO2) n_memo = MEMO2;
                __syncwarp();
                const int U = __popc(kb);
                Best lb;
                lb.key = ~0ull;
                lb.crid = -1;
                int64_t lb_tag = -1;
                const uint64_t bn = best_key >> ORD_SHIFT;
                const int prune = bn < (1u << 20) ? static_cast<int>(bn) : (1 << 20);
                // lane u filters the shifts of locus u; the shifts left are
                // spread over the lanes
                uint32_t live = 0;
                if (lane < U) {
                    const Locus& L = s_loci[lane];
                    live = live_shifts<S>(ix, rd, L.b0, L.rev, cl.adj_cap, cl.budget, cl.clip_cap, prune, t);
                }
                const int n_live = __popc(live);
                int live_incl = n_live;
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(FULL, live_incl, o);
                    if (lane >= o) live_incl += v;
                }
                const int live_total = __shfl_sync(FULL, live_incl, 31);
                for (int c = 0; c < live_total; c += 32) {
                    const int idx = c + lane;
                    int owner = 0;  // first lane whose inclusive count exceeds idx
                    for (int step = 16; step >= 1; step >>= 1) {
                        const int v = __shfl_sync(FULL, live_incl, owner + step - 1);
                        if (v <= idx) owner += step;
                    }
                    const int own = owner < 32 ? owner : 31;
                    const uint32_t o_live = __shfl_sync(FULL, live, own);
                    const int o_first = __shfl_sync(FULL, live_incl - n_live, own);
                    if (idx < live_total) {
                        const int bit = static_cast<int>(__fns(o_live, 0, idx - o_first + 1));
                        const Locus L = s_loci[own];
                        const uint64_t before = lb.key;
                        eval_adj<S>(ix, rd, L.b0, L.rev, bit - cl.adj_cap, cl.budget, cl.clip_cap, L.ord_row, lb,
                                    L.uk, L.ul, L.us, L.e, prune, L.hint, t);
                        if (lb.key != before) lb_tag = L.b0 * 2 + L.rev;
                    }
                }
                const uint64_t wmin = warp_min64(lb.key);
                if (wmin < best_key) {
                    const int wl = __ffs(__ballot_sync(FULL, lb.key == wmin)) - 1;
                    best_key = wmin;
                    win.key = wmin;
                    win.crid = __shfl_sync(FULL, lb.crid, wl);
                    win.pos = __shfl_sync(FULL, lb.pos, wl);
                    win.sl = __shfl_sync(FULL, lb.sl, wl);
                    win.sr = __shfl_sync(FULL, lb.sr, wl);
                    win.mapq = __shfl_sync(FULL, lb.mapq, wl);
                    win.flag = __shfl_sync(FULL, lb.flag, wl);
                    win.uk = __shfl_sync(FULL, lb.uk, wl);
                    win.ul = __shfl_sync(FULL, lb.ul, wl);
                    win.us = __shfl_sync(FULL, lb.us, wl);
                    win.e = __shfl_sync(FULL, lb.e, wl);
                    best_tag = __shfl_sync(FULL, lb_tag, wl);
                    improved = true;
                }
                __syncwarp();
            }
            if ((best_key >> ORD_SHIFT) == 0) break;
            if ((best_key >> ORD_SHIFT) <= 2 && best_key != tested_key && full_compare_key(best_key)) {
                tested_key = best_key;
                // every lane runs the same test on the same data
                const int32_t crid = improved ? win.crid : out.rid[r];
                const int64_t pos = improved ? win.pos : out.pos[r];
                const int sl = improved ? win.sl : static_cast<int>(out.sl[r]);
                const int rev = ((improved ? win.flag : out.flag[r]) & 16) ? 1 : 0;
                const int64_t bstart = static_cast<int64_t>(__ldg(ix.coff + crid)) + pos - sl;
                if (better_hit_impossible<S>(ix, rd, bstart, rev, cl.clip_cap, static_cast<int>(best_key >> ORD_SHIFT), t))
                    break;
            }
        }
        if (improved && lane == 0) write_hit(out, r, win, qlen);
        __syncwarp();
    }
    flush_tally<S>(t, tally_out);
}

// One warp per pair.  Keys are 32-bit: nm (<= budget+5 <= 517) << 13 |
// ordinal, ordinal = pass << 12 | offset in the window (<= 2048).
__global__ void __launch_bounds__(256) mate_rescue_kernel(DevIndex ix, DevReads R, DevParams P, DevOut out,
                                                          int64_t n_pairs) {
    const int64_t pi = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (pi >= n_pairs) return;  // whole warp
    const int64_t i1 = pi, i2 = pi + n_pairs;
    const bool m1 = out.rid[i1] >= 0, m2 = out.rid[i2] >= 0;
    if (m1 == m2) return;
    const int64_t src = m2 ? i2 : i1, dst = m2 ? i1 : i2;
    const int64_t crid = out.rid[src];
    if (crid < 0 || crid >= ix.n_contigs) return;
    const ReadView rd = read_view(R, dst);
    const int qlen = rd.qlen;
    if (qlen < 24) return;
    const int64_t coff = static_cast<int64_t>(ix.coff[crid]);
    const int64_t clen = static_cast<int64_t>(ix.clen[crid]);
    const int64_t mate_pos = static_cast<int64_t>(out.pos[src]);
    int64_t win = P.rescue_win;
    if (win < 32) win = 32;
    if (win > 1024) win = 1024;
    int64_t lo = mate_pos - win;
    if (lo < 0) lo = 0;
    int64_t hi = mate_pos + win;
    if (hi > clen - 24) hi = clen - 24;
    if (hi <= lo) return;
    int budget = P.max_diff;
    if (budget < 2) budget = 2;
    if (budget > qlen / 2) budget = qlen / 2;
    const bool mate_rev = (out.flag[src] & 16) != 0;
    const int span = static_cast<int>(hi - lo + 1);
    Tally tz{};
    uint32_t scan_key = 0xFFFFFFFFu, best_key = 0xFFFFFFFFu;
    for (int pass = 0; pass < 2; ++pass) {
        const int is_rev = pass == 0 ? (mate_rev ? 0 : 1) : (mate_rev ? 1 : 0);
        const uint64_t* q = is_rev ? rd.rc : rd.fwd;
        const uint64_t* qn = is_rev ? rd.nr : rd.nf;
        for (int i = lane; i < span; i += 32) {
            const int64_t bstart = coff + lo + i;
            if (bstart < 0 || static_cast<uint64_t>(bstart + qlen) > ix.l_pac) continue;
            const int nm = count_mm<false>(ix.pacw, q, qn, bstart, 0, qlen, budget + 5, tz);
            const uint32_t key = (static_cast<uint32_t>(nm) << 13) | (static_cast<uint32_t>(pass) << 12) |
                                 static_cast<uint32_t>(i);
            scan_key = key < scan_key ? key : scan_key;
            if (nm <= budget) best_key = key < best_key ? key : best_key;
        }
    }
    scan_key = __reduce_min_sync(0xFFFFFFFFu, scan_key);
    best_key = __reduce_min_sync(0xFFFFFFFFu, best_key);
    int best_nm = 9999;
    int64_t best_pos = 0;
    int best_flag = 0;
    auto rev_of = [&](uint32_t pass) -> int { return pass == 0 ? (mate_rev ? 0 : 1) : (mate_rev ? 1 : 0); };
    if (best_key != 0xFFFFFFFFu) {
        best_nm = static_cast<int>(best_key >> 13);
        best_pos = lo + (best_key & 4095);
        best_flag = rev_of((best_key >> 12) & 1) * 16;
    }
    if (best_nm > budget && scan_key != 0xFFFFFFFFu) {
        // deletion probe at the minimum-nm scan locus (L1957-1998)
        const int64_t scan_local = lo + (scan_key & 4095);
        const int scan_rev = rev_of((scan_key >> 12) & 1);
        const int64_t bstart = coff + scan_local;
        if (bstart >= 0 && static_cast<uint64_t>(bstart + qlen + 1) <= ix.l_pac) {
            const uint64_t* q = scan_rev ? rd.rc : rd.fwd;
            const uint64_t* qn = scan_rev ? rd.nr : rd.nf;
            uint32_t dkey = 0xFFFFFFFFu;
            if (lane == 0) {
                deletion_scan<false>(ix.pacw, q, qn, bstart, qlen, budget, tz, [&](int g, int nmd) {
                    if (nmd > budget) return;
                    const uint32_t k2 = (static_cast<uint32_t>(nmd) << 13) | static_cast<uint32_t>(g / 4);
                    dkey = k2 < dkey ? k2 : dkey;
                });
            }
            dkey = __shfl_sync(0xFFFFFFFFu, dkey, 0);
            if (dkey != 0xFFFFFFFFu) {
                best_nm = static_cast<int>(dkey >> 13);
                best_pos = scan_local;
                best_flag = scan_rev * 16;
            }
        }
    }
    if (best_nm <= budget && lane == 0) {  // L1999-2011
        out.rid[dst] = static_cast<int32_t>(crid);
        out.pos[dst] = static_cast<uint32_t>(best_pos);
        out.mapq[dst] = best_nm == 0 ? 60u : (best_nm <= 2 ? 40u : 20u);
        out.flag[dst] = best_flag;
        out.sl[dst] = 0;
        out.sr[dst] = 0;
        out.nm[dst] = static_cast<uint32_t>(best_nm);
        if (out.score) out.score[dst] = qlen - 5 * best_nm;
    }
}

unsigned grid_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    return static_cast<unsigned>(g > 0 ? g : 1);
}

}  // namespace

// Host launchers (stream-ordered).  Returns the number of kernels launched.
int launch_pack(const uint8_t* d_bases, const uint32_t* d_lens, int64_t n_seq, int64_t n1, int max_len, int words,
                int bs_r1, int bs_r2, uint64_t* d_packed, int* d_err, cudaStream_t st) {
    int rows = PACK_STAGE / max_len;
    if (rows > PACK_THREADS) rows = PACK_THREADS;
    if (rows >= 1) {
        pack_rows_kernel<<<grid_for(n_seq, rows), PACK_THREADS, 0, st>>>(d_bases, d_lens, n_seq, n1, max_len, words,
                                                                        rows, bs_r1, bs_r2, 0, n1, d_packed, d_err);
    } else {  // rows longer than the stage
        const int64_t n = n_seq * words;
        pack_reads_kernel<<<grid_for(n, 256), 256, 0, st>>>(d_bases, d_lens, n_seq, n1, max_len, words, bs_r1,
                                                            bs_r2, 0, n1, d_packed, d_err);
    }
    return 1;
}

// Packs the parts of a merged batch (see pack_parts_kernel); d_lens is the
// batch's length array, already at the batch rows.
int launch_pack_parts(const uint8_t* d_bases, const uint32_t* d_lens, const PackPart* d_parts, int n_parts,
                      int64_t n_rows, int64_t n1_batch, int words, uint64_t* d_packed, int* d_err, cudaStream_t st) {
    const int64_t n = n_rows * words;
    pack_parts_kernel<<<grid_for(n, 256), 256, 0, st>>>(d_bases, d_lens, d_parts, n_parts, n_rows, n1_batch, words,
                                                        d_packed, d_err);
    return 1;
}

// Register budgets of the seed kernels (result-neutral): level 0 leaves the
// compiler free (about 120 registers), level 1 asks for 3 stage-2 / 6
// stage-1 blocks per SM (80 registers), level 2 for 4 / 8 (64 registers,
// with spills to L1).
template <bool S, int L>
struct SeedKernels {
    static constexpr int B1 = L == 0 ? 1 : (L == 1 ? 6 : 8);
    static constexpr int B2 = L == 0 ? 1 : (L == 1 ? 3 : 4);
    static void stage1(dim3 g, cudaStream_t st, const DevIndex& ix, const DevReads& R, const DevParams& P,
                       const DevOut& out, int ep, int max_rows, const Handoff& h, unsigned long long* tally) {
        seed_stage1_kernel<S, B1><<<g, 128, 0, st>>>(ix, R, P, out, ep, max_rows, h, tally);
    }
    static void stage2(dim3 g, cudaStream_t st, const DevIndex& ix, const DevReads& R, const DevParams& P,
                       const DevOut& out, int first_wave, int, const Handoff& h, unsigned long long* tally) {
        seed_stage2_kernel<S, B2><<<g, S2_WARPS * 32, 0, st>>>(ix, R, P, out, h, first_wave, tally);
    }
    static int stage2_occupancy() {  // computed once (calls may be inside a stream capture later)
        static const int v = [] {
            int nb = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, seed_stage2_kernel<S, B2>, S2_WARPS * 32, 0);
            return nb > 0 ? nb : 1;
        }();
        return v;
    }
};

template <bool S>
void launch_levels(int level, bool second, dim3 g, cudaStream_t st, const DevIndex& ix, const DevReads& R,
                   const DevParams& P, const DevOut& out, int ep, int max_rows, const Handoff& h,
                   unsigned long long* tally) {
    if (level == 1) {
        second ? SeedKernels<S, 1>::stage2(g, st, ix, R, P, out, ep, max_rows, h, tally)
               : SeedKernels<S, 1>::stage1(g, st, ix, R, P, out, ep, max_rows, h, tally);
    } else if (level == 2) {
        second ? SeedKernels<S, 2>::stage2(g, st, ix, R, P, out, ep, max_rows, h, tally)
               : SeedKernels<S, 2>::stage1(g, st, ix, R, P, out, ep, max_rows, h, tally);
    } else {
        second ? SeedKernels<S, 0>::stage2(g, st, ix, R, P, out, ep, max_rows, h, tally)
               : SeedKernels<S, 0>::stage1(g, st, ix, R, P, out, ep, max_rows, h, tally);
    }
}

int launch_seed_extend(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out,
                       unsigned long long* d_tally, int level, cudaStream_t st) {
    Handoff none{};
    const dim3 g(grid_for(R.n_seq, 128));
    if (d_tally)
        SeedKernels<true, 0>::stage1(g, st, ix, R, P, out, 1 << 30, 16, none, d_tally);
    else
        launch_levels<false>(level, false, g, st, ix, R, P, out, 1 << 30, 16, none, nullptr);
    return 1;
}

// Two-stage form: stage 1 over every read for the first `stage1_endpoints`
// right endpoints, then the persistent stage-2 warps over the reads left.
// `scratch` must hold two_stage_scratch_bytes(n_seq) bytes.
size_t two_stage_scratch_bytes(int64_t n_seq) {
    const size_t n = static_cast<size_t>(n_seq);
    return 256 + n * 8 + n * 8 * MEMO1 + ((n + 255) / 256) * 256 + ((2 * n + 255) / 256) * 256 + n * 4 + 256;
}

int launch_seed_two_stage(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out,
                          int stage1_endpoints, int stage1_max_rows, int stage2_blocks, int level,
                          int first_wave, void* scratch, unsigned long long* d_tally, cudaEvent_t mid,
                          cudaStream_t st) {
    const size_t n = static_cast<size_t>(R.n_seq);
    char* p = static_cast<char*>(scratch);
    Handoff h;
    h.counters = reinterpret_cast<uint32_t*>(p);
    p += 256;
    h.key = reinterpret_cast<uint64_t*>(p);
    p += n * 8;
    h.memo = reinterpret_cast<uint64_t*>(p);
    p += n * 8 * MEMO1;
    h.memo_n = reinterpret_cast<uint8_t*>(p);
    p += ((n + 255) / 256) * 256;
    h.resume = reinterpret_cast<uint16_t*>(p);
    p += ((2 * n + 255) / 256) * 256;
    h.pending = reinterpret_cast<uint32_t*>(p);
    cudaMemsetAsync(h.counters, 0, 256, st);
    const dim3 g1(grid_for(R.n_seq, 128)), g2(stage2_blocks);
    if (d_tally) {
        SeedKernels<true, 0>::stage1(g1, st, ix, R, P, out, stage1_endpoints, stage1_max_rows, h, d_tally);
        if (mid) cudaEventRecord(mid, st);
        SeedKernels<true, 0>::stage2(g2, st, ix, R, P, out, first_wave, stage1_max_rows, h, d_tally);
    } else {
        launch_levels<false>(level, false, g1, st, ix, R, P, out, stage1_endpoints, stage1_max_rows, h, nullptr);
        if (mid) cudaEventRecord(mid, st);
        launch_levels<false>(level, true, g2, st, ix, R, P, out, first_wave, stage1_max_rows, h, nullptr);
    }
    return 2;
}

// Stage 2 over reads another form left unfinished: best keys, memos,
// resume endpoints and the pending list in the stage-2 hand-off layout;
// counters[0] holds the pending count, counters[1] the work cursor (0).
int launch_stage2_pending(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out,
                          uint64_t* key, uint64_t* memo, uint8_t* memo_n, uint16_t* resume, uint32_t* pending,
                          uint32_t* counters, int blocks, int level, int first_wave, unsigned long long* tally,
                          cudaStream_t st) {
    Handoff h;
    h.key = key;
    h.memo = memo;
    h.memo_n = memo_n;
    h.resume = resume;
    h.pending = pending;
    h.counters = counters;
    const dim3 g(blocks > 0 ? blocks : 1);
    if (tally)
        SeedKernels<true, 0>::stage2(g, st, ix, R, P, out, first_wave, 0, h, tally);
    else
        launch_levels<false>(level, true, g, st, ix, R, P, out, first_wave, 0, h, nullptr);
    return 1;
}

int stage2_blocks_per_sm(int level, bool counting) {
    if (counting) return SeedKernels<true, 0>::stage2_occupancy();
    if (level == 1) return SeedKernels<false, 1>::stage2_occupancy();
    if (level == 2) return SeedKernels<false, 2>::stage2_occupancy();
    return SeedKernels<false, 0>::stage2_occupancy();
}

int launch_rescue(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out, int64_t n_pairs,
                  cudaStream_t st) {
    mate_rescue_kernel<<<grid_for(n_pairs * 32, 256), 256, 0, st>>>(ix, R, P, out, n_pairs);
    return 1;
}

// Loads (under lazy module loading) the kernels that the no-allocation
// entry point launches: pack, the two seed stages at register level
// `level`, and rescue.  Querying a kernel's attributes loads it.
void load_noalloc_kernels(int level) {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, pack_rows_kernel);
    cudaFuncGetAttributes(&a, pack_reads_kernel);
    cudaFuncGetAttributes(&a, mate_rescue_kernel);
    if (level == 1) {
        cudaFuncGetAttributes(&a, seed_stage1_kernel<false, SeedKernels<false, 1>::B1>);
        cudaFuncGetAttributes(&a, seed_stage2_kernel<false, SeedKernels<false, 1>::B2>);
    } else if (level == 2) {
        cudaFuncGetAttributes(&a, seed_stage1_kernel<false, SeedKernels<false, 2>::B1>);
        cudaFuncGetAttributes(&a, seed_stage2_kernel<false, SeedKernels<false, 2>::B2>);
    } else {
        cudaFuncGetAttributes(&a, seed_stage1_kernel<false, SeedKernels<false, 0>::B1>);
        cudaFuncGetAttributes(&a, seed_stage2_kernel<false, SeedKernels<false, 0>::B2>);
    }
}

}  // namespace ma
