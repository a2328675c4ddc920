// seed_core.cuh - device functions of the seed-and-extend kernels, shared
// by the two-stage kernels (map_kernels.cu) and the wavefront kernels
// (wavefront.cu).  Reference: fm_seed_extend_kernel,
// fq2bam-meth/src/linear_gpu_fm.mojo:1156-1837.
//
// Exactness argument used by the seed/extend kernels.  The reference walks
// candidates in a fixed order (right endpoint e ascending, SA row ascending,
// adj ascending, the full compare before the deletion probe at each g) and
// keeps a candidate only when its mismatch count is strictly below the best
// so far; it returns at the first nm == 0.  The hit it reports is therefore
// the minimum of the key (nm, ordinal) over all accepted candidates, where
// the ordinal is the candidate's position in that order.  The kernels
// compute the same minimum with shortcuts that cannot change it:
//   1. A locus (b0, strand) evaluated before is not evaluated again: its
//      adj loop would produce the same (nm) values at larger ordinals.
//   2. The SA row is resolved with one load from the full suffix array
//      instead of the LF walk to a sampled row.  The walk's only effect
//      besides the position is its rejection when it reaches the text's
//      first row unsampled (L1396-1398); that happens exactly for positions
//      below the smallest sampled position, `sa_reject_below`.
//   3. The first k steps of a backward search read the k-mer table: for
//      k <= seed_len nothing is recorded before step k, so the interval
//      after step k (or the emptiness that stops the search) is all the
//      reference keeps from those steps.
// Loop bounds: every loop runs over a read (<= 1024 bases), an SA interval
// (<= 16 rows, or 1), 2*adj_cap+1 <= 25 shifts; nothing waits on another
// thread.
#pragma once

#include <cuda_runtime.h>

#include "ma_device.cuh"

namespace ma {
namespace {


__device__ __forceinline__ uint8_t cvt_base(uint8_t c, int mode) {
    if (mode == MA_BS_C2T) return (c == 67 || c == 99) ? 84 : c;
    if (mode == MA_BS_G2A) return (c == 71 || c == 103) ? 65 : c;
    return c;
}

__device__ __forceinline__ int code_of(uint8_t b) {
    switch (b) {
        case 65: case 97: return 0;
        case 67: case 99: return 1;
        case 71: case 103: return 2;
        case 84: case 116: return 3;
        default: return 4;
    }
}

struct ReadView {
    const uint64_t* fwd;
    const uint64_t* rc;
    const uint64_t* nf;
    const uint64_t* nr;
    int qlen;
};

__device__ __forceinline__ ReadView read_view(const DevReads& R, int64_t r) {
    const uint64_t* b = R.packed + r * 4 * static_cast<int64_t>(R.words);
    ReadView v;
    v.fwd = b;
    v.rc = b + R.words;
    v.nf = b + 2 * R.words;
    v.nr = b + 3 * R.words;
    v.qlen = static_cast<int>(__ldg(R.lens + r));
    return v;
}

// Read words may live in global or shared memory (generic loads).
__device__ __forceinline__ int code_at(const ReadView& v, int s) {
    int w = s >> 5, sh = 2 * (s & 31);
    if ((v.nf[w] >> sh) & 1) return 4;
    return static_cast<int>((v.fwd[w] >> sh) & 3);
}

// 2*n bits (n <= 32 bases) of packed read words starting at base s, base s
// in the lowest two bits.  Reads only words that hold bases of the window.
__device__ __forceinline__ uint64_t window_bits(const uint64_t* words, int s, int n) {
    const int w = s >> 5, off = s & 31;
    uint64_t v = words[w] >> (2 * off);
    if (off && off + n > 32) v |= words[w + 1] << (64 - 2 * off);
    return n >= 32 ? v : (v & ((1ull << (2 * n)) - 1));
}

// Bits 0, 2, 4, ... of x gathered into bits 0, 1, 2, ...
__device__ __forceinline__ uint32_t compact_even(uint64_t x) {
    x &= kEven;
    x = (x | (x >> 1)) & 0x3333333333333333ull;
    x = (x | (x >> 2)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x >> 4)) & 0x00FF00FF00FF00FFull;
    x = (x | (x >> 8)) & 0x0000FFFF0000FFFFull;
    x = (x | (x >> 16)) & 0x00000000FFFFFFFFull;
    return static_cast<uint32_t>(x);
}

// Per-thread traffic tally of the counting kernel variant (S = true).  The
// timed kernel is the S = false instantiation, where every tally compiles
// away.
struct Tally {
    uint32_t occ_lines, kmer_loads, sa_loads, pac_sectors, steps, endpoints, loci, read_words, skipped;
    uint32_t s2_reads, s2_groups, shifts;  // stage-2 reads, stage-2 endpoint groups, shift evaluations
};
constexpr int TALLY_N = 12;

// Mismatch bits (even positions) of read word w against the text at
// bstart + 32*w; N bases always mismatch.
template <bool S>
__device__ __forceinline__ uint64_t mm_word(const uint64_t* __restrict__ pacw, const uint64_t* q,
                                            const uint64_t* qn, int64_t bstart, int w, Tally& t) {
    if constexpr (S) t.read_words += 2;
    uint64_t x = q[w] ^ ref_window(pacw, bstart + 32 * w);
    return ((x | (x >> 1)) & kEven) | qn[w];
}

// Even-bit mask for read positions [a, b) inside the 16-base half word
// starting at 16*h (h within [a >> 4, (b - 1) >> 4]).
__device__ __forceinline__ uint32_t range_mask16(int h, int a, int b) {
    int lo = a - 16 * h, hi = b - 16 * h;
    if (lo < 0) lo = 0;
    const uint32_t m_hi = hi >= 16 ? ~0u : ((1u << (2 * hi)) - 1);
    return m_hi & ~((1u << (2 * lo)) - 1) & 0x55555555u;
}

// min(mismatches over read positions [a, b), cap): the reference's counting
// loops stop as soon as the count exceeds their budget.  Works on 16-base
// halves of the packed words (32-bit operations: one funnel shift aligns
// the text), stopping as soon as the count reaches the cap.
template <bool S>
__device__ __forceinline__ int count_mm(const uint64_t* __restrict__ pacw, const uint64_t* q, const uint64_t* qn,
                                        int64_t bstart, int a, int b, int cap, Tally& t) {
    if (a >= b) return 0;
    const uint32_t* p32 = reinterpret_cast<const uint32_t*>(pacw);
    const uint32_t* q32 = reinterpret_cast<const uint32_t*>(q);
    const uint32_t* n32 = reinterpret_cast<const uint32_t*>(qn);
    const int h0 = a >> 4, h1 = (b - 1) >> 4;
    int n = 0;
    for (int h = h0; h <= h1; ++h) {
        if constexpr (S) t.read_words += 1;
        const int64_t pos = bstart + 16 * h + 32 * PAC_PAD;
        const uint64_t wi = static_cast<uint64_t>(pos) >> 4;
        const uint32_t tx = __funnelshift_r(__ldg(p32 + wi), __ldg(p32 + wi + 1), static_cast<uint32_t>(pos & 15) * 2);
        const uint32_t x = q32[h] ^ tx;
        uint32_t m = ((x | (x >> 1)) & 0x55555555u) | n32[h];
        if (h == h0 || h == h1) m &= range_mask16(h, a, b);
        n += __popc(m);
        if (n >= cap) return cap;
    }
    return n;
}

// First / last read position in [a, b) whose base matches the text.
template <bool S>
__device__ __forceinline__ int first_match(const uint64_t* __restrict__ pacw, const uint64_t* q,
                                           const uint64_t* qn, int64_t bstart, int a, int b, Tally& t) {
    if (a >= b) return -1;
    for (int w = a >> 5; w <= (b - 1) >> 5; ++w) {
        uint64_t m = ~mm_word<S>(pacw, q, qn, bstart, w, t) & range_mask(w, a, b);
        if (m) return 32 * w + (__ffsll(static_cast<long long>(m)) - 1) / 2;
    }
    return -1;
}

template <bool S>
__device__ __forceinline__ int last_match(const uint64_t* __restrict__ pacw, const uint64_t* q,
                                          const uint64_t* qn, int64_t bstart, int a, int b, Tally& t) {
    if (a >= b) return -1;
    for (int w = (b - 1) >> 5; w >= (a >> 5); --w) {
        uint64_t m = ~mm_word<S>(pacw, q, qn, bstart, w, t) & range_mask(w, a, b);
        if (m) return 32 * w + (63 - __clzll(static_cast<long long>(m))) / 2;
    }
    return -1;
}

// Running best of the seed kernel: key = nm << 27 | ordinal.
struct Best {
    uint64_t key;
    int32_t crid;
    uint32_t pos;
    int32_t sl, sr;
    uint32_t mapq;
    int32_t flag;
    uint64_t uk, ul;
    int32_t us, e;
};

constexpr int ORD_SHIFT = 27;
constexpr int MEMO1 = 8;  // loci handed from stage 1 to stage 2 per read

// State of reads that stage 1 hands to stage 2 (scratch, sized n_seq).
struct Handoff {
    uint64_t* key;       // running best key
    uint64_t* memo;      // [n_seq][MEMO1] loci already evaluated (b0*2+strand)
    uint8_t* memo_n;     // entries used in memo
    uint16_t* resume;    // first right endpoint stage 2 searches
    uint32_t* pending;   // read ids handed over
    uint32_t* counters;  // [0] pending count, [1] stage-2 work cursor
};
constexpr uint32_t KIND_SPAN = 260;  // full compare + up to 257 deletion offsets
constexpr uint32_t ADJ_SPAN = 25;    // 2*12+1 shifts

__device__ __forceinline__ int64_t contig_of(const DevIndex& ix, int64_t probe) {
    int64_t lo = 0, hi = ix.n_contigs;
    while (lo < hi) {  // binary search as in linear_gpu_fm.mojo:1536-1549
        int64_t mid = (lo + hi) / 2;
        int64_t off = static_cast<int64_t>(__ldg(ix.coff + mid));
        int64_t ln = static_cast<int64_t>(__ldg(ix.clen + mid));
        if (probe < off) hi = mid;
        else if (probe >= off + ln) lo = mid + 1;
        else return mid;
    }
    return -1;
}

// 1-bp deletion probe on the coarse g grid (linear_gpu_fm.mojo:1729-1825):
// nm_d(g) = min(1 + mismatches(read[0,g) vs text at bstart) +
//           mismatches(read[g,qlen) vs text at bstart+1), budget+1).
// Text positions below 0 read as "not a base" (a mismatch).
template <bool S, typename Visit>
__device__ __forceinline__ void deletion_scan(const uint64_t* __restrict__ pacw, const uint64_t* q,
                                              const uint64_t* qn, int64_t bstart, int qlen, int budget,
                                              Tally& t, Visit visit) {
    const int nw = (qlen + 31) >> 5;
    int R = 0;
    for (int w = 0; w < nw; ++w) {
        uint64_t m1 = mm_word<S>(pacw, q, qn, bstart + 1, w, t);
        if (bstart + 1 < 0) m1 |= range_mask(w, 0, static_cast<int>(-(bstart + 1)));
        R += __popcll(m1 & range_mask(w, 0, qlen));
    }
    int L = 0;
    int cw = -1;
    uint64_t m0 = 0, m1 = 0;
    for (int g = 0; g <= qlen; g += 4) {
        int nmd = 1 + L + R;
        if (nmd > budget + 1) nmd = budget + 1;
        visit(g, nmd);
        if (g < qlen) {
            int w = g >> 5;
            if (w != cw) {
                cw = w;
                m0 = mm_word<S>(pacw, q, qn, bstart, w, t);
                m1 = mm_word<S>(pacw, q, qn, bstart + 1, w, t);
                if (bstart < 0) m0 |= range_mask(w, 0, static_cast<int>(-bstart));
                if (bstart + 1 < 0) m1 |= range_mask(w, 0, static_cast<int>(-(bstart + 1)));
                uint64_t in = range_mask(w, 0, qlen);
                m0 &= in;
                m1 &= in;
            }
            uint64_t four = 0xFFull << (2 * (g & 31));
            L += __popcll(m0 & four);
            R -= __popcll(m1 & four);
        }
    }
}

// One shift adj of one locus (b0, strand): the body of the reference's adj
// loop, linear_gpu_fm.mojo:1528-1826.  Folds the candidate (full compare,
// or the deletion probe's offsets) into `best` by its (nm, ordinal) key.
// Tally of one evaluated locus: the distinct 32-B pac sectors its shifts
// read, the text [b0 - adj_cap, b0 + adj_cap + qlen] at 4 bases a byte.
__device__ __forceinline__ void tally_locus(Tally& t, int64_t b0, int adj_cap, int qlen) {
    t.loci++;
    int64_t lo = b0 - adj_cap;
    if (lo < 0) lo = 0;
    const int64_t hi = b0 + adj_cap + qlen;
    if (hi >= lo) t.pac_sectors += static_cast<uint32_t>(((hi >> 2) >> 5) - ((lo >> 2) >> 5) + 1);
}

// Contig of a locus, looked up once for all of its shifts.
struct ContigHint {
    int64_t crid, coff, clen;
};

__device__ __forceinline__ ContigHint contig_hint(const DevIndex& ix, int64_t b0) {
    int64_t probe = b0 < 0 ? 0 : b0;
    if (probe >= static_cast<int64_t>(ix.l_pac)) probe = static_cast<int64_t>(ix.l_pac) - 1;
    ContigHint h{contig_of(ix, probe), 0, 0};
    if (h.crid >= 0) {
        h.coff = static_cast<int64_t>(__ldg(ix.coff + h.crid));
        h.clen = static_cast<int64_t>(__ldg(ix.clen + h.crid));
    }
    return h;
}

__device__ __forceinline__ void set_best(Best& best, uint64_t key, int64_t crid, int64_t pos, int sl, int sr,
                                         uint32_t mapq, int flag, uint64_t uk, uint64_t ul, int us, int e) {
    best.key = key;
    best.crid = static_cast<int32_t>(crid);
    best.pos = static_cast<uint32_t>(pos);
    best.sl = sl;
    best.sr = sr;
    best.mapq = mapq;
    best.flag = flag;
    best.uk = uk;
    best.ul = ul;
    best.us = us;
    best.e = e;
}

// The deletion probe of a failed forward shift (L1729-1825), kept out of
// line: it is rare on the hot path.  Every read position mismatches under
// shift 0 or under shift +1 for every g unless it matches under one of
// them, so nm_d(g) >= 1 + popc(M0 & M1) for all g; when that bound already
// exceeds the budget or cannot beat the best so far, no offset is tried.
template <bool S>
__device__ __noinline__ void deletion_candidates(const uint64_t* __restrict__ pacw, const uint64_t* q,
                                                 const uint64_t* qn, int64_t bstart, int qlen, int budget,
                                                 int prune_nm, uint32_t ord, int64_t crid, int64_t local,
                                                 Best& best, uint64_t uk, uint64_t ul, int us, int e, Tally& t) {
    const int nw = (qlen + 31) >> 5;
    const int stop = prune_nm < budget + 1 ? prune_nm : budget + 1;  // 1 + bound >= stop: nothing to gain
    int both = 0;
    for (int w = 0; w < nw; ++w) {
        uint64_t m0 = mm_word<S>(pacw, q, qn, bstart, w, t);
        uint64_t m1 = mm_word<S>(pacw, q, qn, bstart + 1, w, t);
        if (bstart < 0) m0 |= range_mask(w, 0, static_cast<int>(-bstart));
        if (bstart + 1 < 0) m1 |= range_mask(w, 0, static_cast<int>(-(bstart + 1)));
        both += __popcll(m0 & m1 & range_mask(w, 0, qlen));
        if (1 + both >= stop) return;
    }
    deletion_scan<S>(pacw, q, qn, bstart, qlen, budget, t, [&](int g, int nmd) {
        if (nmd > budget) return;
        const uint64_t key = (static_cast<uint64_t>(nmd) << ORD_SHIFT) | (ord + 1 + g / 4);
        if (key < best.key) set_best(best, key, crid, local, 0, 0, 20u, 0, uk, ul, us, e);
    });
}

// Soft-clip retry of L1591-1694: sl grows to the first matching in-contig
// base below clip_cap, sr likewise from the right; then the recount.
template <bool S>
__device__ __noinline__ int soft_clip_recount(const uint64_t* __restrict__ pacw, const uint64_t* q,
                                              const uint64_t* qn, int64_t bstart, int qlen, int64_t local,
                                              int64_t clen, int sl0, int sr0, int clip_cap, int budget, int* sl_out,
                                              int* sr_out, Tally& t) {
    int64_t lim = clen - local;
    if (lim > clip_cap) lim = clip_cap;
    const int j = first_match<S>(pacw, q, qn, bstart, sl0, static_cast<int>(lim), t);
    const int sl = j >= 0 ? j : clip_cap;
    const int64_t jlo = sl > qlen - 1 - clip_cap ? sl : qlen - 1 - clip_cap;
    int64_t jhi = qlen - 1 - sr0;
    if (jhi > clen - local - 1) jhi = clen - local - 1;
    const int j2 = last_match<S>(pacw, q, qn, bstart, static_cast<int>(jlo + 1), static_cast<int>(jhi + 1), t);
    int sr;
    if (j2 >= 0) {
        sr = qlen - 1 - j2;
    } else {
        const int64_t sstar = sr0 > qlen - 1 - sl ? sr0 : qlen - 1 - sl;
        sr = static_cast<int>(sstar < clip_cap ? sstar : clip_cap);
    }
    *sl_out = sl;
    *sr_out = sr;
    return count_mm<S>(pacw, q, qn, bstart, sl, qlen - sr, budget + 1, t);
}

// One shift adj of one locus (b0, strand): the body of the reference's adj
// loop, linear_gpu_fm.mojo:1528-1826.  Folds the candidate (full compare,
// or the deletion probe's offsets) into `best` by its (nm, ordinal) key.
// prune_nm: a candidate of this call can only matter when its nm is below
// prune_nm (every candidate of the call comes after the current best in the
// reference's order); 1 << 20 disables pruning.  `hint` is the contig of
// b0; a shift that stays inside it needs no contig search.
template <bool S>
__device__ void eval_adj(const DevIndex& ix, const ReadView& rd, int64_t b0, int is_rev, int adj, int budget,
                         int clip_cap, uint32_t ord_row, Best& best, uint64_t uk, uint64_t ul, int us, int e,
                         int prune_nm, const ContigHint& hint, Tally& t) {
    if constexpr (S) t.shifts++;
    const int qlen = rd.qlen;
    const uint64_t* q = is_rev ? rd.rc : rd.fwd;
    const uint64_t* qn = is_rev ? rd.nr : rd.nf;
    const int64_t bstart = b0 + adj;
    int64_t crid = hint.crid, coff = hint.coff, clen = hint.clen;
    if (crid < 0 || bstart < coff || bstart >= coff + clen) {
        // the contig holding the clamped probe (binary search, L1536-1549)
        int64_t probe = bstart < 0 ? 0 : bstart;
        if (probe >= static_cast<int64_t>(ix.l_pac)) probe = static_cast<int64_t>(ix.l_pac) - 1;
        crid = contig_of(ix, probe);
        if (crid < 0) return;
        coff = static_cast<int64_t>(__ldg(ix.coff + crid));
        clen = static_cast<int64_t>(__ldg(ix.clen + crid));
    }
    const int64_t local = bstart - coff;
    const int64_t sl0 = local < 0 ? -local : 0;
    const int64_t sr0 = local + qlen > clen ? local + qlen - clen : 0;
    if (!(sl0 + sr0 < qlen && sl0 <= clip_cap && sr0 <= clip_cap)) return;
    const uint32_t ord = (ord_row + static_cast<uint32_t>(adj + 12)) * KIND_SPAN;
    const bool del_probe = adj == 0 && is_rev == 0;
    const bool del_room = del_probe && prune_nm > 1 && bstart + qlen + 1 <= coff + clen;
    // Exact pruning.  sl0, sr0 and every soft clip are at most clip_cap, so
    // the full compare and any clipped recount both span read positions
    // [clip_cap, qlen - clip_cap); their mismatches bound nm from below.
    if (!del_probe) {
        // a shift without deletion probe only matters with a core below
        // both the budget and the best so far: count no further
        const int cap = prune_nm < budget + 1 ? prune_nm : budget + 1;
        if (count_mm<S>(ix.pacw, q, qn, bstart, clip_cap, qlen - clip_cap, cap, t) >= cap) return;
    }
    const int core = del_probe ? count_mm<S>(ix.pacw, q, qn, bstart, clip_cap, qlen - clip_cap, budget + 1, t) : 0;
    if (core > budget) {
        // neither compare is accepted: only the deletion probe remains
        if (del_room)
            deletion_candidates<S>(ix.pacw, q, qn, bstart, qlen, budget, prune_nm, ord, crid, local, best, uk, ul,
                                   us, e, t);
        return;
    }
    // whether the compare is accepted decides the deletion probe, so only
    // shifts without one can stop here
    if (core >= prune_nm && !del_probe) return;
    int nm = count_mm<S>(ix.pacw, q, qn, bstart, static_cast<int>(sl0), static_cast<int>(qlen - sr0), budget + 1, t);
    int sl = static_cast<int>(sl0), sr = static_cast<int>(sr0);
    if (nm > budget && clip_cap > 0)
        nm = soft_clip_recount<S>(ix.pacw, q, qn, bstart, qlen, local, clen, sl, sr, clip_cap, budget, &sl, &sr, t);
    const int alen = qlen - sl - sr;
    if (nm <= budget && alen >= 24) {
        const uint64_t key = (static_cast<uint64_t>(nm) << ORD_SHIFT) | ord;
        if (key < best.key)
            set_best(best, key, crid, local + sl, sl, sr, nm == 0 ? 60u : 20u, is_rev * 16, uk, ul, us, e);
    } else if (del_room) {
        deletion_candidates<S>(ix.pacw, q, qn, bstart, qlen, budget, prune_nm, ord, crid, local, best, uk, ul, us,
                               e, t);
    }
}

// Shifts of one locus that can fold a candidate into a best of nm prune_nm
// (bit adj + adj_cap set), from the first three 16-base halves of the core
// [clip_cap, qlen - clip_cap) alone.  A shift's full and clipped compares
// have at least as many mismatches as any part of the core, so a shift
// whose partial core count reaches min(prune_nm, budget + 1) has no
// acceptable compare; the deletion probe of shift 0 (forward) has
// nm_d >= 1 + popc(M0 & M1) (shift 0 and +1 mismatch bits, any part of the
// read), so it is dropped only when that bound reaches the same cap too.
// The per-shift count leaves out the read's N bases (an N mismatches every
// text base, so leaving it out only lowers the count: the filter stays a
// lower bound and keeps every shift that can win).  Loci of a read shorter
// than the core halves keep every shift.
template <bool S>
__device__ uint32_t live_shifts(const DevIndex& ix, const ReadView& rd, int64_t b0, int is_rev, int adj_cap,
                                int budget, int clip_cap, int prune_nm, Tally& t) {
    const int qlen = rd.qlen;
    const int A = 2 * adj_cap + 1;
    const uint32_t all = A >= 32 ? ~0u : ((1u << A) - 1);
    const int c0 = clip_cap, c1 = qlen - clip_cap;
    if (c1 - c0 < 16) return all;
    const int cap = prune_nm < budget + 1 ? prune_nm : budget + 1;
    const uint64_t* q = is_rev ? rd.rc : rd.fwd;
    const uint64_t* qn = is_rev ? rd.nr : rd.nf;
    const int h0 = c0 >> 4;
    const int hl = (c1 - 1) >> 4;  // last half holding core bases
    const int nh = hl - h0 + 1 < 3 ? hl - h0 + 1 : 3;
    // loci whose filter window leaves the text are left to eval_adj
    if (b0 - adj_cap + 16 * h0 < 0 || b0 + adj_cap + 1 + 16 * (h0 + nh) > static_cast<int64_t>(ix.l_pac)) return all;
    // the text of every shift's halves lies in six 16-base words from wlo:
    // shift i starts s0 + i bases into them
    const uint32_t* p32 = reinterpret_cast<const uint32_t*>(ix.pacw);
    const int64_t p0 = b0 - adj_cap + 16 * h0 + 32 * PAC_PAD;
    const uint64_t wlo = static_cast<uint64_t>(p0) >> 4;
    const int s0 = static_cast<int>(p0 & 15);
    const uint32_t w0 = __ldg(p32 + wlo), w1 = __ldg(p32 + wlo + 1), w2 = __ldg(p32 + wlo + 2);
    const uint32_t w3 = __ldg(p32 + wlo + 3), w4 = __ldg(p32 + wlo + 4), w5 = __ldg(p32 + wlo + 5);
    const uint32_t* q32 = reinterpret_cast<const uint32_t*>(q);
    const uint32_t* n32 = reinterpret_cast<const uint32_t*>(qn);
    const uint32_t qa = q32[h0], ma = range_mask16(h0, c0, c1);
    const uint32_t qb = nh > 1 ? q32[h0 + 1] : 0u, mb = nh > 1 ? range_mask16(h0 + 1, c0, c1) : 0u;
    const uint32_t qc = nh > 2 ? q32[h0 + 2] : 0u, mc = nh > 2 ? range_mask16(h0 + 2, c0, c1) : 0u;
    if constexpr (S) t.read_words += 6;
    // The text words realigned so that shift i starts i bases into them:
    // the offset of a shift's words and its funnel-shift amount are then the
    // same for every lane (no divergence between loci whose windows start at
    // different bases).  Mismatch bits of half b go to the odd bit
    // positions (the halves' masks hold even bits), so halves a and b share
    // one popcount.
    const uint32_t sa = static_cast<uint32_t>(s0) * 2;
    const uint32_t W0 = __funnelshift_r(w0, w1, sa), W1 = __funnelshift_r(w1, w2, sa);
    const uint32_t W2 = __funnelshift_r(w2, w3, sa), W3 = __funnelshift_r(w3, w4, sa);
    const uint32_t W4 = __funnelshift_r(w4, w5, sa);
    const uint32_t mb_odd = mb << 1;
    uint32_t live = 0;
#pragma unroll
    for (int k = 0; k < 2; ++k) {  // A <= 25: shifts 0..15 and 16..A-1
        const uint32_t a = k == 0 ? W0 : W1, b = k == 0 ? W1 : W2;
        const uint32_t c = k == 0 ? W2 : W3, d = k == 0 ? W3 : W4;
        const int hi = A < 16 * k + 16 ? A : 16 * k + 16;
        for (int i = 16 * k; i < hi; ++i) {
            const uint32_t sh = static_cast<uint32_t>(i - 16 * k) * 2;
            const uint32_t ta = qa ^ __funnelshift_r(a, b, sh);
            const uint32_t tb = qb ^ __funnelshift_r(b, c, sh);
            const uint32_t tc = qc ^ __funnelshift_r(c, d, sh);
            const uint32_t xab = ((ta | (ta >> 1)) & ma) | ((tb | (tb << 1)) & mb_odd);
            const uint32_t xc = (tc | (tc >> 1)) & mc;
            if (__popc(xab) + __popc(xc) < cap) live |= 1u << i;
        }
    }
    if (!is_rev && !((live >> adj_cap) & 1u)) {
        // the deletion probe's bound from the exact mismatch bits (N bases
        // included) of shifts 0 and +1
        const uint32_t na = n32[h0], nb = nh > 1 ? n32[h0 + 1] : 0u, nc = nh > 2 ? n32[h0 + 2] : 0u;
        auto halves = [&](int i, uint32_t& xa, uint32_t& xb, uint32_t& xc) {
            const bool hi16 = i >= 16;
            const uint32_t sh = static_cast<uint32_t>(i & 15) * 2;
            const uint32_t a = hi16 ? W1 : W0, b = hi16 ? W2 : W1, c = hi16 ? W3 : W2, d = hi16 ? W4 : W3;
            const uint32_t ta = qa ^ __funnelshift_r(a, b, sh), tb = qb ^ __funnelshift_r(b, c, sh);
            const uint32_t tc = qc ^ __funnelshift_r(c, d, sh);
            xa = (((ta | (ta >> 1)) & 0x55555555u) | na) & ma;
            xb = (((tb | (tb >> 1)) & 0x55555555u) | nb) & mb;
            xc = (((tc | (tc >> 1)) & 0x55555555u) | nc) & mc;
        };
        uint32_t z0a, z0b, z0c, z1a, z1b, z1c;
        halves(adj_cap, z0a, z0b, z0c);
        halves(adj_cap + 1, z1a, z1b, z1c);
        if (1 + __popc(z0a & z1a) + __popc(z0b & z1b) + __popc(z0c & z1c) < cap) live |= 1u << adj_cap;
    }
    return live;
}

// Every shift of one locus, in adj order (L1526-1827); shifts that cannot
// yield a candidate against the best at the locus' start are skipped.
template <bool S>
__device__ void eval_locus(const DevIndex& ix, const ReadView& rd, int64_t b0, int is_rev, int adj_cap,
                           int budget, int clip_cap, uint32_t ord_row, Best& best, uint64_t uk, uint64_t ul,
                           int us, int e, Tally& t) {
    if constexpr (S) tally_locus(t, b0, adj_cap, rd.qlen);
    const ContigHint hint = contig_hint(ix, b0);
    const uint64_t b_start = best.key >> ORD_SHIFT;
    uint32_t live = live_shifts<S>(ix, rd, b0, is_rev, adj_cap, budget, clip_cap,
                                   b_start < (1u << 20) ? static_cast<int>(b_start) : (1 << 20), t);
    while (live) {
        const int adj = __ffs(live) - 1 - adj_cap;
        live &= live - 1;
        const uint64_t bn = best.key >> ORD_SHIFT;
        eval_adj<S>(ix, rd, b0, is_rev, adj, budget, clip_cap, ord_row, best, uk, ul, us, e,
                    bn < (1u << 20) ? static_cast<int>(bn) : (1 << 20), hint, t);
    }
}

// Exact early stop for a best hit with nm == b, b = 1 or 2, from a full or
// clipped compare aligning the read at text position bstart (strand rev).
// Every later candidate comes after the best in the reference's order, so
// only one with nm < b could replace it.  Soft and contig-edge clips are at
// most clip_cap each, so a full or clipped candidate has at most nm
// mismatches over the read's core [clip_cap, qlen - clip_cap); a deletion
// candidate has nm = 1 + its mismatches over the whole read.  The best
// hit's k core mismatches (k <= b, N bases included) split the core into
// k + 1 segments matching the text at bstart exactly; "unique" below means
// a segment's text occurs once in the dual-strand text (its length reaches
// the shortest unique length ending at its last base, from the summary).
// A candidate at another text position (either strand) that matches a
// segment exactly holds it a second time, so that segment is not unique.
// A candidate at bstart on the same strand is the same compare (nm = b).
//   b = 1: a better candidate has nm == 0, a full or clipped compare with
//          every segment exact: one unique segment rules it out.
//   b = 2, k = 2: a full or clipped candidate with <= 1 core mismatch has
//          at least two exact segments; a deletion candidate (nm_d = 1) has
//          no mismatch, so each segment lies exact in its left part (text
//          at bs) or right part (bs + 1) unless it spans the split, and at
//          most one part coincides with the best hit's alignment: then the
//          best hit's mismatches lie in the other part and so do at least
//          two segments.  Either way at most one non-unique segment rules
//          it out.
//   b = 2, k = 1 (one mismatch outside the core): a full or clipped
//          candidate with <= 1 core mismatch matches one of the two
//          segments exactly; for a deletion candidate, if a part coincides
//          with the best hit's alignment both mismatches lie in the other
//          part and so does the segment beyond the core mismatch, otherwise
//          a segment that does not span the split lies shifted.  Two unique
//          segments rule out both.
// N bases mismatch every candidate: b of them in the core rule out both
// kinds (full: nm >= b; deletion: nm_d >= 1 + b).
template <bool S>
__device__ bool better_hit_impossible(const DevIndex& ix, const ReadView& rd, int64_t bstart, int rev, int clip_cap,
                                      int b, Tally& t) {
    const int qlen = rd.qlen;
    const int c0 = clip_cap, c1 = qlen - clip_cap;
    if (!ix.summary || b < 1 || b > 2 || c1 <= c0 || bstart + c0 < 0 ||
        bstart + c1 > static_cast<int64_t>(ix.l_pac))
        return false;
    const uint64_t* q = rev ? rd.rc : rd.fwd;
    const uint64_t* qn = rev ? rd.nr : rd.nf;
    int p[2] = {-1, -1};
    int k = 0, n_n = 0;
    for (int w = c0 >> 5; w <= (c1 - 1) >> 5; ++w) {
        const uint64_t rm = range_mask(w, c0, c1);
        n_n += __popcll(qn[w] & rm);
        uint64_t m = mm_word<S>(ix.pacw, q, qn, bstart, w, t) & rm;
        while (m) {
            if (k == 2) return false;  // more core mismatches than this test handles
            p[k++] = 32 * w + (__ffsll(static_cast<long long>(m)) - 1) / 2;
            m &= m - 1;
        }
    }
    if (n_n >= b) return true;
    if (k > b || (b == 2 && k < 1)) return false;
    // segments [c0, p0), (p0, p1), (p1, c1) of the k mismatches
    int non_unique = 0;
    for (int i = 0; i <= k; ++i) {
        const int u = i == 0 ? c0 : p[i - 1] + 1, v = i == k ? c1 : p[i];
        bool uniq = false;
        if (v > u) {
            const int mul = __ldg(ix.summary + bstart + v - 1) & 0xFF;
            uniq = mul != 255 && mul <= v - u;
        }
        non_unique += !uniq;
    }
    if (b == 1) return non_unique <= k;
    return k == 2 ? non_unique <= 1 : non_unique == 0;
}

// Whether a best key is a full or clipped compare (not a deletion offset).
__device__ __forceinline__ bool full_compare_key(uint64_t key) {
    return (static_cast<uint32_t>(key & ((1ull << ORD_SHIFT) - 1)) % KIND_SPAN) == 0;
}

struct Seed {
    uint64_t k, l;
    int s;
    bool found;
};

// Unique-SMEM left extension from right endpoint e (L1235-1385), as a
// start (the table steps) and single backward steps, so that a caller can
// interleave the steps of many endpoints.  SeedSearch is the state between
// steps.
struct SeedSearch {
    uint64_t k, l, last_k;
    int s;
    int last;  // the last interval of <= 16 rows at mlen >= seed_len: its start | (rows - 1) << 16; -1 = none
};

__device__ __forceinline__ void search_keep(SeedSearch& q, uint64_t k, uint64_t l, int s) {
    q.last_k = k;
    q.last = s | static_cast<int>(l - k) << 16;
}

// The seed a search that stops here returns: the last kept interval, if any.
__device__ __forceinline__ Seed search_result(const SeedSearch& q) {
    return q.last >= 0 ? Seed{q.last_k, q.last_k + static_cast<uint64_t>(q.last >> 16), q.last & 0xFFFF, true}
                       : Seed{0, 0, -1, false};
}

// Starts the search at endpoint e.  Returns true when backward steps follow
// (from q.s); false when the search is over, its seed (if any) in `out`.
template <bool S>
__device__ __forceinline__ bool search_start(const DevIndex& ix, const ReadView& rd, int e, const DevParams& P,
                                             SeedSearch& q, Seed& out, Tally& t) {
    if constexpr (S) t.endpoints++;
    q.k = 0;
    q.l = ix.seq_len;
    q.last_k = 0;
    q.s = e;
    q.last = -1;
    out = Seed{0, 0, -1, false};
    bool have = false;  // a table gave the interval after the first K steps
    int K = 0;
    // A/T window outcome table: the whole search over the last at_k bases
    // in one lookup when they are all A or T.  Counts never grow as the
    // pattern extends, so the max_occ stop can only come at seed_len: with
    // c rows there (c > max_occ) the search stops with no seed, unless
    // c <= 16 made that interval the kept one (then the steps below run).
    const int AK = ix.at_k;
    if (AK > 0 && P.seed_len == ix.at_seed_len && e >= AK - 1) {
        const int s0 = e - AK + 1;
        const uint64_t win = window_bits(rd.fwd, s0, AK);
        const uint64_t lo = win & kEven, hi = (win >> 1) & kEven;
        if (lo == hi && window_bits(rd.nf, s0, AK) == 0) {
            const uint4 v = __ldg(ix.atw + compact_even(lo));
            if constexpr (S) t.kmer_loads++;
            const uint64_t elo = static_cast<uint64_t>(v.x) | static_cast<uint64_t>(v.y) << 32;
            const uint64_t ehi = static_cast<uint64_t>(v.z) | static_cast<uint64_t>(v.w) << 32;
            const uint64_t c_sl = ehi >> 35;
            const uint64_t rk = elo & KMER_K_MASK, rn = ehi & KMER_K_MASK;
            const int kind = static_cast<int>(elo >> 40) & 3;
            if (c_sl > static_cast<uint64_t>(P.max_occ)) {
                if (c_sl > 16) return false;  // stopped at seed_len, nothing kept
            } else if (kind == 0) {
                return false;
            } else if (kind == 1) {
                out = Seed{rk, rk + rn - 1, e - static_cast<int>((elo >> 35) & 31), true};
                return false;
            } else {
                q.k = rk;
                q.l = rk + rn - 1;
                if (rn <= 16) search_keep(q, q.k, q.l, s0);
                q.s = s0 - 1;
                if (q.s < 0) {
                    out = search_result(q);
                    return false;
                }
                return true;
            }
        }
    }
    // Steps before mlen reaches seed_len record nothing, so with K <= seed_len
    // a window holding a non-ACGT base, or an empty interval, ends the search
    // with no seed, and otherwise the interval after K steps is all that is
    // kept from them.
    const int K3 = ix.kmer3_k;
    if (K3 > 0 && K3 <= P.seed_len) {
        const int s0 = e - K3 + 1;
        if (window_bits(rd.nf, s0, K3) != 0) return false;
        const uint64_t win = window_bits(rd.fwd, s0, K3);
        const uint64_t lo = win & kEven, hi = (win >> 1) & kEven;
        const bool has_c = (lo & ~hi) != 0, has_g = (hi & ~lo) != 0;
        if (!(has_c && has_g)) {
            uint32_t idx = 0;
            for (int i = 0; i < K3; ++i) idx = idx * 3 + static_cast<uint32_t>(__popcll((win >> (2 * i)) & 3));
            const uint64_t kl = __ldg(ix.kmer3[has_c ? 1 : 0] + idx);
            if constexpr (S) t.kmer_loads++;
            if (kmer_interval(kl, q.k, q.l)) {
                have = true;
                K = K3;
            }
        }
    }
    if (!have && ix.kmer_k > 0 && ix.kmer_k <= P.seed_len) {
        const int s0 = e - ix.kmer_k + 1;
        if (window_bits(rd.nf, s0, ix.kmer_k) != 0) return false;
        const uint64_t win = window_bits(rd.fwd, s0, ix.kmer_k);
        uint32_t idx = 0;
        for (int i = 0; i < ix.kmer_k; ++i) idx = (idx << 2) | static_cast<uint32_t>((win >> (2 * i)) & 3);
        const uint64_t kl = __ldg(ix.kmer + idx);
        if constexpr (S) t.kmer_loads++;
        if (kmer_interval(kl, q.k, q.l)) {  // an untabled entry leaves (k, l) = (0, seq_len)
            have = true;
            K = ix.kmer_k;
        }
    }
    if (have) {
        const int s0 = e - K + 1;
        if (q.k > q.l) return false;
        if (K >= P.seed_len) {
            const int64_t occ_n = static_cast<int64_t>(q.l - q.k + 1);
            if (occ_n == 1) {
                out = Seed{q.k, q.l, s0, true};
                return false;
            }
            if (occ_n >= 1 && occ_n <= 16) search_keep(q, q.k, q.l, s0);
            if (occ_n > P.max_occ) {
                out = search_result(q);
                return false;
            }
        }
        q.s = s0 - 1;
    }
    if (q.s < 0) {
        out = search_result(q);
        return false;
    }
    return true;
}

// One backward step (base q.s).  Returns true when more steps follow; false
// when the search is over, its seed (if any) in `out`.
template <bool S>
__device__ __forceinline__ bool search_next(const DevIndex& ix, const ReadView& rd, int e, const DevParams& P,
                                            SeedSearch& q, Seed& out, Tally& t) {
    const int cc = code_at(rd, q.s);
    if (cc > 3) {
        out = search_result(q);
        return false;
    }
    uint64_t ok = 0;
    if constexpr (S) {
        t.steps++;
        const int64_t lk = q.k != 0 ? static_cast<int64_t>((q.k - 1 - (q.k - 1 >= ix.primary)) >> 6) : -1;
        const int64_t ll = q.l != ix.seq_len ? static_cast<int64_t>((q.l - (q.l >= ix.primary)) >> 6) : -2;
        t.occ_lines += (lk >= 0) + (ll >= 0 && ll != lk);
    }
    if (q.k != 0) ok = occ_row(ix, q.k - 1, cc);
    const uint64_t ol = occ_row(ix, q.l, cc);
    const uint64_t Lc = ix.L2[cc];
    q.k = Lc + ok + 1;
    q.l = Lc + ol;
    if (q.k > q.l) {
        out = search_result(q);
        return false;
    }
    const int64_t occ_n = static_cast<int64_t>(q.l - q.k + 1);
    if (e - q.s + 1 >= P.seed_len) {
        if (occ_n == 1) {
            out = Seed{q.k, q.l, q.s, true};
            return false;
        }
        if (occ_n <= 16) search_keep(q, q.k, q.l, q.s);
        if (occ_n > P.max_occ) {
            out = search_result(q);
            return false;
        }
    }
    if (--q.s < 0) {
        out = search_result(q);
        return false;
    }
    return true;
}

// The whole search of endpoint e.
template <bool S>
__device__ __forceinline__ Seed search_endpoint(const DevIndex& ix, const ReadView& rd, int e, const DevParams& P,
                                                Tally& t) {
    SeedSearch q;
    Seed out;
    if (search_start<S>(ix, rd, e, P, q, out, t))
        while (search_next<S>(ix, rd, e, P, q, out, t)) {
        }
    return out;
}

// Per-read clamps of linear_gpu_fm.mojo:1204-1216.
struct Clamps {
    int budget, clip_cap, adj_cap;
};

__device__ __forceinline__ Clamps clamps_for(const DevParams& P, int qlen) {
    Clamps c;
    c.budget = P.max_diff;
    if (c.budget < 2) c.budget = 2;
    if (c.budget > qlen / 2) c.budget = qlen / 2;
    c.clip_cap = P.max_soft;
    if (c.clip_cap > qlen / 4) c.clip_cap = qlen / 4;
    c.adj_cap = P.max_adj;
    if (c.adj_cap < 0) c.adj_cap = 0;
    if (c.adj_cap > 12) c.adj_cap = 12;
    return c;
}

// Number of right endpoints e = seed_len-1 + j*stride below qlen.
__device__ __forceinline__ int endpoint_count(const DevParams& P, int qlen) {
    return qlen >= P.seed_len ? (qlen - P.seed_len) / P.seed_stride + 1 : 0;
}

// SA row -> candidate locus (b0, strand) of L1503-1524; false = rejected.
__device__ __forceinline__ bool locus_of_row(const DevIndex& ix, uint64_t sa_pos, int us, int e, int qlen,
                                             int64_t& b0, int& is_rev) {
    if (sa_pos < ix.sa_reject_below) return false;  // the sampled walk would hit the first row
    const int64_t plen = e - us + 1;
    if (sa_pos < ix.l_pac) {
        b0 = static_cast<int64_t>(sa_pos) - us;
        is_rev = 0;
        return true;
    }
    if (sa_pos + static_cast<uint64_t>(plen) - 1 >= 2 * ix.l_pac) return false;
    const int64_t fp_end = 2 * static_cast<int64_t>(ix.l_pac) - 1 - static_cast<int64_t>(sa_pos);
    const int64_t fp_start = fp_end - (plen - 1);
    b0 = fp_start - (qlen - 1 - e);
    is_rev = 1;
    return true;
}

__device__ __forceinline__ void write_hit(const DevOut& out, int64_t r, const Best& b, int qlen) {
    if (b.crid >= 0) {
        const int nm = static_cast<int>(b.key >> ORD_SHIFT);
        out.rid[r] = b.crid;
        out.pos[r] = b.pos;
        out.mapq[r] = b.mapq;
        out.flag[r] = b.flag;
        out.sl[r] = static_cast<uint32_t>(b.sl);
        out.sr[r] = static_cast<uint32_t>(b.sr);
        out.nm[r] = static_cast<uint32_t>(nm);
        if (out.score) out.score[r] = qlen - b.sl - b.sr - 5 * nm;
    } else {  // defaults of L1194-1200
        out.rid[r] = -1;
        out.pos[r] = 0;
        out.mapq[r] = 0;
        out.flag[r] = 4;
        out.sl[r] = 0;
        out.sr[r] = 0;
        out.nm[r] = 0;
        if (out.score) out.score[r] = 0;
    }
    if (out.us) {
        out.uk[r] = b.uk;
        out.ul[r] = b.ul;
        out.us[r] = b.us;
        out.e[r] = b.e;
    }
}

template <bool S>
__device__ __forceinline__ void flush_tally(const Tally& t, unsigned long long* tally_out) {
    if constexpr (S) {
        const uint32_t v[TALLY_N] = {t.occ_lines, t.kmer_loads, t.sa_loads, t.pac_sectors, t.steps,
                                     t.endpoints, t.loci, t.read_words, t.skipped, t.s2_reads, t.s2_groups,
                                     t.shifts};
        for (int i = 0; i < TALLY_N; ++i)
            if (v[i]) atomicAdd(tally_out + i, static_cast<unsigned long long>(v[i]));
    }
}

__device__ __forceinline__ uint64_t warp_min64(uint64_t v) {
    for (int o = 16; o > 0; o >>= 1) {
        const uint64_t w = __shfl_xor_sync(0xFFFFFFFFu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

// Duplicate prediction.  Let the read's bases ending at right endpoint e
// match the text exactly at an evaluated locus (b0, strand), over the
// length mlen = max(seed_len, m), m the shortest unique length of the text
// substring ending there (summary).  Then the reference's backward search
// from e only ever follows that text (no empty interval, no non-ACGT base),
// occ never exceeds its value at mlen = seed_len (<= max_occ, from the
// summary's k-mer count, or 1 when m <= seed_len), and it stops at mlen with
// a single SA row whose text position resolves to b0: the locus again, which
// cannot win.  Such endpoints are skipped without touching the index.
template <bool S>
__device__ __forceinline__ bool predicted_duplicate(const DevIndex& ix, const ReadView& rd, int e,
                                                    const DevParams& P, int64_t first_tag, const uint64_t* memo,
                                                    int n_check, Tally& t) {
    const int qlen = rd.qlen;
    const int64_t L = static_cast<int64_t>(ix.l_pac);
    // the best hit's locus first (valid tags are >= -2^40; -1 marks none),
    // then the first memo entries
    for (int m = first_tag == -1 ? 0 : -1; m < n_check; ++m) {
        if (m >= 0 && static_cast<int64_t>(memo[m]) == first_tag) continue;
        const int64_t tag = m < 0 ? first_tag : static_cast<int64_t>(memo[m]);
        const int64_t b0 = tag >> 1;
        const int rev = static_cast<int>(tag & 1);
        // text position (in T) of the window's right end
        const int64_t x = rev ? 2 * L - 1 - (b0 + qlen - 1 - e) : b0 + e;
        if (rev ? (b0 + qlen - 1 - e < 0 || b0 + qlen - 1 - e >= L) : (x < 0 || x >= L)) continue;
        const uint32_t sm = __ldg(ix.summary + x);
        const int mul = static_cast<int>(sm & 0xFF), occ = static_cast<int>(sm >> 8);
        if (mul == 255) continue;
        const int mlen = mul > P.seed_len ? mul : P.seed_len;
        if (mlen > e + 1) continue;
        if (mul > P.seed_len && (occ == 255 || occ > P.max_occ)) continue;
        const int sA = e - mlen + 1;
        int mm;
        if (!rev) {
            if (b0 + sA < 0) continue;
            mm = count_mm<S>(ix.pacw, rd.fwd, rd.nf, b0, sA, e + 1, 1, t);
        } else {
            const int a = qlen - 1 - e, bb = qlen - sA;  // reverse-complement read positions
            if (b0 + bb - 1 >= L) continue;
            mm = count_mm<S>(ix.pacw, rd.rc, rd.nr, b0, a, bb, 1, t);
        }
        if (mm == 0) return true;
    }
    return false;
}

}  // namespace
}  // namespace ma
