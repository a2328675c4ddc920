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

__device__ __forceinline__ int code_at(const ReadView& v, int s) {
    int w = s >> 5, sh = 2 * (s & 31);
    if ((__ldg(v.nf + w) >> sh) & 1) return 4;
    return static_cast<int>((__ldg(v.fwd + w) >> sh) & 3);
}

// Per-thread traffic tally of the counting kernel variant (S = true).  The
// timed kernel is the S = false instantiation, where every tally compiles
// away.
struct Tally {
    uint32_t occ_lines, kmer_loads, sa_loads, pac_sectors, steps, endpoints, loci, read_words;
};

// Mismatch bits (even positions) of read word w against the text at
// bstart + 32*w; N bases always mismatch.
template <bool S>
__device__ __forceinline__ uint64_t mm_word(const uint64_t* __restrict__ pacw, const uint64_t* q,
                                            const uint64_t* qn, int64_t bstart, int w, Tally& t) {
    if constexpr (S) {
        // the window reads 16 bytes at word (bstart + 32w + 32*PAC_PAD) >> 5
        const uint64_t wi = static_cast<uint64_t>(bstart + 32 * w + 32 * PAC_PAD) >> 5;
        t.pac_sectors += ((wi * 8) >> 5) == ((wi * 8 + 15) >> 5) ? 1 : 2;
        t.read_words += 2;
    }
    uint64_t x = __ldg(q + w) ^ ref_window(pacw, bstart + 32 * w);
    return ((x | (x >> 1)) & kEven) | __ldg(qn + w);
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

// Evaluates every shift adj of one locus (b0, strand): the body of the
// reference's adj loop, L1526-1826.
template <bool S>
__device__ void eval_locus(const DevIndex& ix, const ReadView& rd, int64_t b0, int is_rev, int adj_cap,
                           int budget, int clip_cap, uint32_t ord_row, Best& best, uint64_t uk, uint64_t ul,
                           int us, int e, Tally& t) {
    if constexpr (S) t.loci++;
    const int qlen = rd.qlen;
    const uint64_t* q = is_rev ? rd.rc : rd.fwd;
    const uint64_t* qn = is_rev ? rd.nr : rd.nf;
    for (int adj = -adj_cap; adj <= adj_cap; ++adj) {
        const int64_t bstart = b0 + adj;
        int64_t probe = bstart < 0 ? 0 : bstart;
        if (probe >= static_cast<int64_t>(ix.l_pac)) probe = static_cast<int64_t>(ix.l_pac) - 1;
        const int64_t crid = contig_of(ix, probe);
        if (crid < 0) continue;
        const int64_t coff = static_cast<int64_t>(__ldg(ix.coff + crid));
        const int64_t clen = static_cast<int64_t>(__ldg(ix.clen + crid));
        const int64_t local = bstart - coff;
        const int64_t sl0 = local < 0 ? -local : 0;
        const int64_t sr0 = local + qlen > clen ? local + qlen - clen : 0;
        if (!(sl0 + sr0 < qlen && sl0 <= clip_cap && sr0 <= clip_cap)) continue;
        const uint32_t ord = (ord_row + static_cast<uint32_t>(adj + 12)) * KIND_SPAN;
        int nm = count_mm<S>(ix.pacw, q, qn, bstart, static_cast<int>(sl0), static_cast<int>(qlen - sr0), budget + 1, t);
        int sl = static_cast<int>(sl0), sr = static_cast<int>(sr0);
        if (nm > budget && clip_cap > 0) {
            // soft-clip retry, L1591-1694: grow sl to the first matching
            // in-contig base below clip_cap, sr likewise from the right
            int64_t lim = clen - local;
            if (lim > clip_cap) lim = clip_cap;
            int j = first_match<S>(ix.pacw, q, qn, bstart, sl, static_cast<int>(lim), t);
            sl = j >= 0 ? j : clip_cap;
            int64_t jlo = sl > qlen - 1 - clip_cap ? sl : qlen - 1 - clip_cap;
            int64_t jhi = qlen - 1 - sr0;
            if (jhi > clen - local - 1) jhi = clen - local - 1;
            int j2 = last_match<S>(ix.pacw, q, qn, bstart, static_cast<int>(jlo + 1), static_cast<int>(jhi + 1), t);
            if (j2 >= 0) {
                sr = qlen - 1 - j2;
            } else {
                int64_t sstar = sr0 > qlen - 1 - sl ? sr0 : qlen - 1 - sl;
                sr = static_cast<int>(sstar < clip_cap ? sstar : clip_cap);
            }
            nm = count_mm<S>(ix.pacw, q, qn, bstart, sl, qlen - sr, budget + 1, t);
        }
        const int alen = qlen - sl - sr;
        if (nm <= budget && alen >= 24) {
            const uint64_t key = (static_cast<uint64_t>(nm) << ORD_SHIFT) | ord;
            if (key < best.key) {
                best.key = key;
                best.crid = static_cast<int32_t>(crid);
                best.pos = static_cast<uint32_t>(local + sl);
                best.sl = sl;
                best.sr = sr;
                best.mapq = nm == 0 ? 60u : 20u;
                best.flag = is_rev * 16;
                best.uk = uk;
                best.ul = ul;
                best.us = us;
                best.e = e;
            }
        } else if (adj == 0 && is_rev == 0) {
            if (bstart + qlen + 1 <= coff + clen) {
                deletion_scan<S>(ix.pacw, q, qn, bstart, qlen, budget, t, [&](int g, int nmd) {
                    if (nmd > budget) return;
                    const uint64_t key = (static_cast<uint64_t>(nmd) << ORD_SHIFT) | (ord + 1 + g / 4);
                    if (key < best.key) {
                        best.key = key;
                        best.crid = static_cast<int32_t>(crid);
                        best.pos = static_cast<uint32_t>(local);
                        best.sl = 0;
                        best.sr = 0;
                        best.mapq = 20u;
                        best.flag = 0;
                        best.uk = uk;
                        best.ul = ul;
                        best.us = us;
                        best.e = e;
                    }
                });
            }
        }
    }
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
    const int K = ix.kmer_k;
    bool stop = false;
    if (K > 0 && K <= P.seed_len) {
        const int s0 = e - K + 1;
        uint32_t idx = 0;
        for (int t = s0; t <= e; ++t) {
            int c = code_at(rd, t);
            if (c > 3) return res;  // a non-ACGT before mlen reaches seed_len
            idx = (idx << 2) | static_cast<uint32_t>(c);
        }
        const uint2 kl = __ldg(ix.kmer + idx);
        if constexpr (S) t.kmer_loads++;
        k = kl.x;
        l = kl.y;
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

__global__ void __launch_bounds__(256) pack_reads_kernel(const uint8_t* __restrict__ bases,
                                                         const uint32_t* __restrict__ lens, int64_t n_seq,
                                                         int64_t n1, int max_len, int words, int bs_r1,
                                                         int bs_r2, uint64_t* __restrict__ packed,
                                                         int* __restrict__ err) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t r = t / words;
    const int w = static_cast<int>(t - r * words);
    if (r >= n_seq) return;
    int len = static_cast<int>(lens[r]);
    if (len > max_len) {
        atomicExch(err, 1);
        len = max_len;
    }
    const int mode = r < n1 ? bs_r1 : bs_r2;
    const uint8_t* row = bases + r * static_cast<int64_t>(max_len);
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
    uint64_t* out = packed + r * 4 * static_cast<int64_t>(words);
    out[w] = f;
    out[words + w] = rw;
    out[2 * words + w] = fn;
    out[3 * words + w] = rn;
}

template <bool S>
__global__ void __launch_bounds__(256) seed_extend_kernel(DevIndex ix, DevReads R, DevParams P, DevOut out,
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
    if (qlen >= P.seed_len) {
        // clamps of L1204-1216
        int budget = P.max_diff;
        if (budget < 2) budget = 2;
        if (budget > qlen / 2) budget = qlen / 2;
        int clip_cap = P.max_soft;
        if (clip_cap > qlen / 4) clip_cap = qlen / 4;
        int adj_cap = P.max_adj;
        if (adj_cap < 0) adj_cap = 0;
        if (adj_cap > 12) adj_cap = 12;
        constexpr int MEMO = 16;
        int64_t memo_b0[MEMO];
        int memo_n = 0;
        const int64_t l_pac = static_cast<int64_t>(ix.l_pac);
        int ei = 0;
        for (int e = P.seed_len - 1; e < qlen; e += P.seed_stride, ++ei) {
            const Seed sd = search_endpoint<S>(ix, rd, e, P, t);
            if (!sd.found) continue;
            const int us = sd.s;
            const int64_t plen = e - us + 1;
            for (uint64_t hi = sd.k; hi <= sd.l; ++hi) {
                const uint64_t sa_pos = __ldg(ix.sa + hi);
                if constexpr (S) t.sa_loads++;
                if (sa_pos < ix.sa_reject_below) continue;
                int64_t b0;
                int is_rev;
                if (sa_pos < ix.l_pac) {  // L1509-1524
                    b0 = static_cast<int64_t>(sa_pos) - us;
                    is_rev = 0;
                } else {
                    if (sa_pos + static_cast<uint64_t>(plen) - 1 >= 2 * ix.l_pac) continue;
                    const int64_t fp_end = 2 * l_pac - 1 - static_cast<int64_t>(sa_pos);
                    const int64_t fp_start = fp_end - (plen - 1);
                    b0 = fp_start - (qlen - 1 - e);
                    is_rev = 1;
                }
                // shortcut 1: a locus already evaluated cannot win again
                const int64_t tag = b0 * 2 + is_rev;
                bool seen = false;
                const int mn = memo_n < MEMO ? memo_n : MEMO;
                for (int i = 0; i < mn; ++i) seen |= memo_b0[i] == tag;
                if (seen) continue;
                memo_b0[memo_n % MEMO] = tag;
                ++memo_n;
                const uint32_t ord_row = (static_cast<uint32_t>(ei) * 16 + static_cast<uint32_t>(hi - sd.k)) * ADJ_SPAN;
                eval_locus<S>(ix, rd, b0, is_rev, adj_cap, budget, clip_cap, ord_row, best, sd.k, sd.l, us, e, t);
                if ((best.key >> ORD_SHIFT) == 0) goto done;  // nm == 0 returns (L1708-1728)
            }
        }
    }
done:
    if (best.crid >= 0) {
        const int nm = static_cast<int>(best.key >> ORD_SHIFT);
        out.rid[r] = best.crid;
        out.pos[r] = best.pos;
        out.mapq[r] = best.mapq;
        out.flag[r] = best.flag;
        out.sl[r] = static_cast<uint32_t>(best.sl);
        out.sr[r] = static_cast<uint32_t>(best.sr);
        out.nm[r] = static_cast<uint32_t>(nm);
        if (out.score) out.score[r] = qlen - best.sl - best.sr - 5 * nm;
    } else {
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
        out.uk[r] = best.uk;
        out.ul[r] = best.ul;
        out.us[r] = best.us;
        out.e[r] = best.e;
    }
    if constexpr (S) {
        const uint32_t v[8] = {t.occ_lines, t.kmer_loads, t.sa_loads, t.pac_sectors, t.steps, t.endpoints, t.loci,
                               t.read_words};
        for (int i = 0; i < 8; ++i)
            if (v[i]) atomicAdd(tally_out + i, static_cast<unsigned long long>(v[i]));
    }
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
                                                        d_packed, d_err);
    return 1;
}

int launch_seed_extend(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out,
                       unsigned long long* d_tally, cudaStream_t st) {
    if (d_tally)
        seed_extend_kernel<true><<<grid_for(R.n_seq, 128), 128, 0, st>>>(ix, R, P, out, d_tally);
    else
        seed_extend_kernel<false><<<grid_for(R.n_seq, 128), 128, 0, st>>>(ix, R, P, out, nullptr);
    return 1;
}

int launch_rescue(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out, int64_t n_pairs,
                  cudaStream_t st) {
    mate_rescue_kernel<<<grid_for(n_pairs * 32, 256), 256, 0, st>>>(ix, R, P, out, n_pairs);
    return 1;
}

}  // namespace ma
