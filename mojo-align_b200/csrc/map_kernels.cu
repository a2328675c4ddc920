// map_kernels.cu - the mapping kernels of the linear bisulfite FM path.
//
//   pack_reads_kernel     _cvt + pack_bases_kernel
//                         (linear_fastq.mojo:37-46, linear_gpu_fm.mojo:1136-1154),
//                         fused into a 2-bit packing of both strands
//   seed_extend_kernel    fm_seed_extend_kernel (linear_gpu_fm.mojo:1156-1837)
//   mate_rescue_kernel    fm_mate_rescue_kernel (linear_gpu_fm.mojo:1839-2011)
//
// Exactness argument used by the seed/extend kernel.  The reference walks
// candidates in a fixed order (right endpoint e ascending, SA row ascending,
// adj ascending, the full compare before the deletion probe at each g) and
// keeps a candidate only when its mismatch count is strictly below the best
// so far; it returns at the first nm == 0.  The hit it reports is therefore
// the minimum of the key (nm, ordinal) over all accepted candidates, where
// the ordinal is the candidate's position in that order.  This kernel
// computes the same minimum with three shortcuts that cannot change it:
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
// (<= 16 rows, or 1), 2*adj_cap+1 <= 25 shifts, or a rescue window
// (<= 2049 positions); nothing waits on another thread.
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

// min(mismatches over read positions [a, b), cap): the reference's counting
// loops stop as soon as the count exceeds their budget.
template <bool S>
__device__ __forceinline__ int count_mm(const uint64_t* __restrict__ pacw, const uint64_t* q, const uint64_t* qn,
                                        int64_t bstart, int a, int b, int cap, Tally& t) {
    if (a >= b) return 0;
    int n = 0;
    for (int w = a >> 5; w <= (b - 1) >> 5; ++w) {
        n += __popcll(mm_word<S>(pacw, q, qn, bstart, w, t) & range_mask(w, a, b));
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

// Every shift of one locus, in adj order (L1526-1827).
template <bool S>
__device__ void eval_locus(const DevIndex& ix, const ReadView& rd, int64_t b0, int is_rev, int adj_cap,
                           int budget, int clip_cap, uint32_t ord_row, Best& best, uint64_t uk, uint64_t ul,
                           int us, int e, Tally& t) {
    if constexpr (S) tally_locus(t, b0, adj_cap, rd.qlen);
    const ContigHint hint = contig_hint(ix, b0);
    for (int adj = -adj_cap; adj <= adj_cap; ++adj) {
        const uint64_t bn = best.key >> ORD_SHIFT;
        eval_adj<S>(ix, rd, b0, is_rev, adj, budget, clip_cap, ord_row, best, uk, ul, us, e,
                    bn < (1u << 20) ? static_cast<int>(bn) : (1 << 20), hint, t);
    }
}

// Exact early stop for a best hit with nm == 1.  Every later candidate
// comes after the best in the reference's order, so only an nm == 0
// candidate could replace it; deletion-probe candidates have nm >= 1, so it
// would be a full or clipped compare with no mismatch over the read's core
// [clip_cap, qlen - clip_cap) (soft and contig-edge clips are at most
// clip_cap each).  The best hit, a full or clipped compare aligning the read
// at text position bstart, has at most one mismatch p in the core, which
// splits the core into at most two segments matching the text at bstart
// exactly.  An nm == 0 candidate at any other text position (either strand)
// would hold each segment a second time, so if one segment's text is unique
// in the dual-strand text (its length reaches the shortest unique length of
// the text ending at its last base, from the summary), no nm == 0 candidate
// exists.  A candidate at bstart itself on the same strand is the same
// compare and has nm == 1.  An N in the core mismatches every candidate, so
// then no nm == 0 candidate exists either.
template <bool S>
__device__ bool exact_hit_impossible(const DevIndex& ix, const ReadView& rd, int64_t bstart, int rev, int clip_cap,
                                     Tally& t) {
    const int qlen = rd.qlen;
    const int c0 = clip_cap, c1 = qlen - clip_cap;
    if (!ix.summary || c1 <= c0 || bstart + c0 < 0 || bstart + c1 > static_cast<int64_t>(ix.l_pac)) return false;
    const uint64_t* q = rev ? rd.rc : rd.fwd;
    const uint64_t* qn = rev ? rd.nr : rd.nf;
    int p = -1;
    for (int w = c0 >> 5; w <= (c1 - 1) >> 5; ++w) {
        const uint64_t rm = range_mask(w, c0, c1);
        if (qn[w] & rm) return true;
        uint64_t m = mm_word<S>(ix.pacw, q, qn, bstart, w, t) & rm;
        while (m) {
            if (p >= 0) return false;
            p = 32 * w + (__ffsll(static_cast<long long>(m)) - 1) / 2;
            m &= m - 1;
        }
    }
    const int u0 = c0, v0 = p < 0 ? c1 : p, u1 = p + 1, v1 = c1;
    for (int k = 0; k < (p < 0 ? 1 : 2); ++k) {
        const int u = k ? u1 : u0, v = k ? v1 : v0;
        if (v <= u) continue;
        const int mul = __ldg(ix.summary + bstart + v - 1) & 0xFF;
        if (mul != 255 && mul <= v - u) return true;
    }
    return false;
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

// Unique-SMEM left extension from right endpoint e (L1235-1385).
template <bool S>
__device__ __forceinline__ Seed search_endpoint(const DevIndex& ix, const ReadView& rd, int e, const DevParams& P,
                                                Tally& t) {
    if constexpr (S) t.endpoints++;
    uint64_t k = 0, l = ix.seq_len, last_k = 0, last_l = 0;
    int s = e, last_s = -1;
    Seed res{0, 0, -1, false};
    bool stop = false;
    bool have = false;  // a table gave the interval after the first K steps
    int K = 0;
    // Steps before mlen reaches seed_len record nothing, so with K <= seed_len
    // a window holding a non-ACGT base, or an empty interval, ends the search
    // with no seed, and otherwise the interval after K steps is all that is
    // kept from them.
    const int K3 = ix.kmer3_k;
    if (K3 > 0 && K3 <= P.seed_len) {
        const int s0 = e - K3 + 1;
        if (window_bits(rd.nf, s0, K3) != 0) return res;
        const uint64_t win = window_bits(rd.fwd, s0, K3);
        const uint64_t lo = win & kEven, hi = (win >> 1) & kEven;
        const bool has_c = (lo & ~hi) != 0, has_g = (hi & ~lo) != 0;
        if (!(has_c && has_g)) {
            uint32_t idx = 0;
            for (int i = 0; i < K3; ++i) idx = idx * 3 + static_cast<uint32_t>(__popcll((win >> (2 * i)) & 3));
            const uint2 kl = __ldg(ix.kmer3[has_c ? 1 : 0] + idx);
            if constexpr (S) t.kmer_loads++;
            k = kl.x;
            l = kl.y;
            have = true;
            K = K3;
        }
    }
    if (!have && ix.kmer_k > 0 && ix.kmer_k <= P.seed_len) {
        K = ix.kmer_k;
        const int s0 = e - K + 1;
        if (window_bits(rd.nf, s0, K) != 0) return res;
        const uint64_t win = window_bits(rd.fwd, s0, K);
        uint32_t idx = 0;
        for (int i = 0; i < K; ++i) idx = (idx << 2) | static_cast<uint32_t>((win >> (2 * i)) & 3);
        const uint2 kl = __ldg(ix.kmer + idx);
        if constexpr (S) t.kmer_loads++;
        k = kl.x;
        l = kl.y;
        have = true;
    }
    if (have) {
        const int s0 = e - K + 1;
        if (k > l) return res;
        if (K >= P.seed_len) {
            const int64_t occ_n = static_cast<int64_t>(l - k + 1);
            if (occ_n == 1) return Seed{k, l, s0, true};
            if (occ_n >= 1 && occ_n <= 16) {
                last_k = k;
                last_l = l;
                last_s = s0;
            }
            if (occ_n > P.max_occ) stop = true;
        }
        s = s0 - 1;
    }
    if (!stop) {
        while (s >= 0) {
            const int cc = code_at(rd, s);
            if (cc > 3) break;
            uint64_t ok = 0;
            if constexpr (S) {
                t.steps++;
                const int64_t lk = k != 0 ? static_cast<int64_t>((k - 1 - (k - 1 >= ix.primary)) >> 6) : -1;
                const int64_t ll = l != ix.seq_len ? static_cast<int64_t>((l - (l >= ix.primary)) >> 6) : -2;
                t.occ_lines += (lk >= 0) + (ll >= 0 && ll != lk);
            }
            if (k != 0) ok = occ_row(ix, k - 1, cc);
            const uint64_t ol = occ_row(ix, l, cc);
            const uint64_t Lc = ix.L2[cc];
            k = Lc + ok + 1;
            l = Lc + ol;
            if (k > l) break;
            const int64_t occ_n = static_cast<int64_t>(l - k + 1);
            const int mlen = e - s + 1;
            if (mlen >= P.seed_len) {
                if (occ_n == 1) return Seed{k, l, s, true};
                if (occ_n <= 16) {
                    last_k = k;
                    last_l = l;
                    last_s = s;
                }
                if (occ_n > P.max_occ) break;
            }
            --s;
        }
    }
    if (last_s >= 0) return Seed{last_k, last_l, last_s, true};
    return res;
}

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
                const uint64_t sa_pos = __ldg(ix.sa + hi);
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
        if (pend && (best.key >> ORD_SHIFT) == 1 && full_compare_key(best.key)) {
            const int64_t bstart = static_cast<int64_t>(__ldg(ix.coff + best.crid)) + best.pos - best.sl;
            if (exact_hit_impossible<S>(ix, rd, bstart, (best.flag & 16) ? 1 : 0, clamps_for(P, qlen).clip_cap, t))
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

__device__ __forceinline__ uint64_t warp_min64(uint64_t v) {
    for (int o = 16; o > 0; o >>= 1) {
        const uint64_t w = __shfl_xor_sync(0xFFFFFFFFu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

// Stage 2: one warp per pending read, persistent over the pending list.
// Lanes search 32 right endpoints at a time; the candidate rows of those
// endpoints, in the reference's order (endpoint, then row), are resolved
// 32 at a time, de-duplicated (within the group by __match_any_sync,
// against earlier groups and stage 1 through the memo), and every (locus,
// shift) pair is evaluated by one lane.  The warp minimum of the (nm,
// ordinal) keys is folded into the read's running best.  The read stops
// after the group of endpoints in which an nm == 0 hit appears.
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
        const int A = 2 * cl.adj_cap + 1;
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
                    const uint64_t sa_pos = __ldg(ix.sa + hi);
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
                for (int it = lane; it < U * A; it += 32) {
                    const int u = it / A, a = it - u * A;
                    const Locus L = s_loci[u];
                    const uint64_t before = lb.key;
                    eval_adj<S>(ix, rd, L.b0, L.rev, a - cl.adj_cap, cl.budget, cl.clip_cap, L.ord_row, lb, L.uk,
                                L.ul, L.us, L.e, prune, L.hint, t);
                    if (lb.key != before) lb_tag = L.b0 * 2 + L.rev;
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
            if ((best_key >> ORD_SHIFT) == 1 && best_key != tested_key && full_compare_key(best_key)) {
                tested_key = best_key;
                // every lane runs the same test on the same data
                const int32_t crid = improved ? win.crid : out.rid[r];
                const int64_t pos = improved ? win.pos : out.pos[r];
                const int sl = improved ? win.sl : static_cast<int>(out.sl[r]);
                const int rev = ((improved ? win.flag : out.flag[r]) & 16) ? 1 : 0;
                const int64_t bstart = static_cast<int64_t>(__ldg(ix.coff + crid)) + pos - sl;
                if (exact_hit_impossible<S>(ix, rd, bstart, rev, cl.clip_cap, t)) break;
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
    const int64_t n = n_seq * words;
    pack_reads_kernel<<<grid_for(n, 256), 256, 0, st>>>(d_bases, d_lens, n_seq, n1, max_len, words, bs_r1, bs_r2,
                                                        0, n1, d_packed, d_err);
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
    static int stage2_occupancy() {
        int nb = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, seed_stage2_kernel<S, B2>, S2_WARPS * 32, 0);
        return nb > 0 ? nb : 1;
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

}  // namespace ma
