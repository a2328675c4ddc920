// sam_emit.cu - SAM text lines of one mapped batch on the device.
//
// Replaces the per-record host loop of map_fastq_fm_gpu's SAM path
// (fq2bam-meth/src/linear_gpu_fm.mojo:2787-2836), which builds a LinearHit
// per read with _hit_from_fm (L987-1025), pairs mates with pair_hits
// (fq2bam-meth/src/linear_extend.mojo:263-294), formats each line with
// hit_to_sam_line (L297-320) + the RG tag (_sam_with_rg_fm, L80-81) and
// writes it.  Here the lines of a whole batch are built in HBM in three
// passes:
//   1. sam_layout_kernel (one thread per pair): both hits and the pair
//      fields, each line's byte length and a compact record of its fields,
//      names' bytes >= 0x80 counted (each becomes U+FFFD), SEQ / QUAL
//      checked for strict UTF-8, mapped records and error bits;
//   2. a device scan of the lengths (line end offsets);
//   3. sam_write_kernel (one warp per line): the line assembled in a
//      shared-memory stage at its destination's 16-byte phase (lanes copy the name, the
//      contig names, SEQ reverse-complemented on flag 16, QUAL and the RG
//      tag from aligned word loads; lane 0 writes the integer fields), then
//      stored with 16-byte stores; lines longer than the stage are built in
//      place.
#include <cub/device/device_scan.cuh>

#include <string>

#include "ma_internal.h"
#include "sam_emit.h"

namespace ma {
namespace {

constexpr int THREADS = 256;
constexpr int WARPS = THREADS / 32;
constexpr unsigned FULL = 0xffffffffu;
constexpr uint32_t STAGE = 2048;  // bytes of a warp's line stage in shared memory
constexpr int SPAN_UNROLL = 2;    // words a lane loads per round of a span copy

enum : unsigned { E_OVER = 1, E_UTF8 = 2, E_RID = 4, E_SPAN = 8 };
enum : uint8_t { K_NAME = 0, K_STAR = 1, K_EQ = 2 };

void check_launch(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

size_t align256(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }

// One record's SAM fields before and after pairing (LinearHit,
// linear_extend.mojo:11-48).
struct Hit {
    int64_t flag, pos1, mapq, pnext, tlen, sl, m, sr;
    uint64_t contig_off, rnext_off;
    uint32_t contig_len, rnext_len;
    uint32_t canon;
    uint8_t contig_kind, rnext_kind;
    bool mapped;  // placed by _hit_from_fm (CIGAR and strand apply)
    bool star;    // RNAME "*": unplaced, or a canonical name "*"
};

// _hit_from_fm: unplaced when rid < 0 or no base is left between the clips.
__device__ Hit hit_of(const SamDev& d, uint64_t r, unsigned& err) {
    Hit h{};
    h.rnext_kind = K_STAR;
    h.rnext_len = 1;
    const int32_t rid = d.rid[r];
    const int64_t m = static_cast<int64_t>(d.seq_len[r]) - d.sl[r] - d.sr[r];
    bool ok = rid >= 0 && m >= 1;
    if (rid >= 0 && static_cast<uint32_t>(rid) >= d.n_contigs) {
        err |= E_RID;
        ok = false;
    }
    uint64_t co = 0;
    uint32_t cl = 0;
    if (ok) {
        co = d.cname_off[rid];
        cl = d.cname_len[rid];
        if (co > d.names_bytes || cl > d.names_bytes - co) {
            err |= E_SPAN;
            ok = false;
        }
    }
    if (!ok) {
        h.star = true;
        h.flag = 4;
        h.contig_kind = K_STAR;
        h.contig_len = 1;
        return h;
    }
    h.mapped = true;
    h.flag = d.flag[r];
    h.pos1 = static_cast<int64_t>(d.pos[r]) + 1;
    h.mapq = d.mapq[r];
    h.sl = d.sl[r];
    h.sr = d.sr[r];
    h.m = m;
    h.contig_kind = K_NAME;
    h.contig_off = co;
    h.contig_len = cl;
    h.canon = d.canon[rid];
    h.star = cl == 1 && d.names[co] == '*';
    return h;
}

// pair_hits (linear_extend.mojo:263-294); len2 = len(SEQ of R2).
__device__ void pair_up(Hit& a, Hit& b, uint32_t len2) {
    a.flag |= 1 | 64;
    b.flag |= 1 | 128;
    if (!a.star && !b.star && a.canon == b.canon) {
        a.flag |= 2;
        b.flag |= 2;
        a.rnext_kind = b.rnext_kind = K_EQ;
        a.pnext = b.pos1;
        b.pnext = a.pos1;
        int64_t t = b.pos1 - a.pos1;
        if (t < 0) t = -t;
        t += len2;
        a.tlen = t;
        b.tlen = -t;
        return;
    }
    if (a.star) b.flag |= 8;
    if (b.star) a.flag |= 8;
    if (!a.star) {
        b.rnext_kind = K_NAME;
        b.rnext_off = a.contig_off;
        b.rnext_len = a.contig_len;
        b.pnext = a.pos1;
    }
    if (!b.star) {
        a.rnext_kind = K_NAME;
        a.rnext_off = b.contig_off;
        a.rnext_len = b.contig_len;
        a.pnext = b.pos1;
    }
}

// Decimal digits of u: comparisons against powers of ten below 2^32, a
// division loop above.
__device__ __forceinline__ uint32_t ndig(uint64_t u) {
    if (u >> 32) {
        uint32_t k = 10;
        u /= 10000000000ull;
        while (u) {
            u /= 10;
            ++k;
        }
        return k;
    }
    const uint32_t v = static_cast<uint32_t>(u);
    return 1 + (v >= 10u) + (v >= 100u) + (v >= 1000u) + (v >= 10000u) + (v >= 100000u) + (v >= 1000000u) +
           (v >= 10000000u) + (v >= 100000000u) + (v >= 1000000000u);
}

__device__ __forceinline__ uint64_t mag(int64_t v) {
    return v < 0 ? uint64_t(0) - static_cast<uint64_t>(v) : static_cast<uint64_t>(v);
}

__device__ __forceinline__ uint32_t sdig(int64_t v) { return (v < 0) + ndig(mag(v)); }

__device__ __forceinline__ uint32_t cigar_len(const Hit& h) {
    if (!h.mapped) return 1;
    return (h.sl > 0 ? sdig(h.sl) + 1 : 0) + sdig(h.m) + 1 + (h.sr > 0 ? sdig(h.sr) + 1 : 0);
}

// Bytes from the line's start to SEQ: the name (width name_w) and the
// tab-separated fields FLAG .. TLEN.
__device__ __forceinline__ uint64_t head_len(const Hit& h, uint64_t name_w) {
    return name_w + 1 + sdig(h.flag) + 1 + h.contig_len + 1 + sdig(h.pos1) + 1 + sdig(h.mapq) + 1 + cigar_len(h) +
           1 + h.rnext_len + 1 + sdig(h.pnext) + 1 + sdig(h.tlen) + 1;
}

// Strict UTF-8 (RFC 3629): no overlong forms, surrogates or code points
// above U+10FFFF.
__device__ bool utf8_ok(const uint8_t* p, uint64_t n) {
    uint64_t i = 0;
    while (i < n) {
        const uint8_t c = p[i];
        if (c < 0x80) {
            ++i;
            continue;
        }
        int k;
        uint8_t lo = 0x80, hi = 0xbf;
        if (c >= 0xc2 && c <= 0xdf) {
            k = 1;
        } else if (c >= 0xe0 && c <= 0xef) {
            k = 2;
            if (c == 0xe0) lo = 0xa0;
            if (c == 0xed) hi = 0x9f;
        } else if (c >= 0xf0 && c <= 0xf4) {
            k = 3;
            if (c == 0xf0) lo = 0x90;
            if (c == 0xf4) hi = 0x8f;
        } else {
            return false;
        }
        if (n - i - 1 < static_cast<uint64_t>(k)) return false;
        if (p[i + 1] < lo || p[i + 1] > hi) return false;
        for (int j = 2; j <= k; ++j)
            if (p[i + j] < 0x80 || p[i + j] > 0xbf) return false;
        i += k + 1;
    }
    return true;
}

__device__ __forceinline__ bool span_ok(uint64_t off, uint32_t len, uint64_t n) { return off <= n && len <= n - off; }

__device__ __forceinline__ bool spans_ok(const SamDev& d, uint64_t r) {
    return span_ok(d.name_off[r], d.name_len[r], d.arena_bytes) && span_ok(d.seq_off[r], d.seq_len[r], d.arena_bytes) &&
           span_ok(d.qual_off[r], d.qual_len[r], d.arena_bytes);
}

// What the write pass needs of a line, resolved once by the layout pass.
struct LineRec {
    int64_t flag, pos1, pnext, tlen;
    uint64_t contig_off, rnext_off;
    uint32_t mapq, sl, sr, m;
    uint32_t contig_len, rnext_len;
    uint8_t contig_kind, rnext_kind, mapped, widen;
    uint32_t pad;
};
static_assert(sizeof(LineRec) == 80, "line record layout");

// Bytes >= 0x80 in p[0, n), from the aligned 16-byte blocks that cover the
// span (their bytes outside the span lie in the same block as one inside).
__device__ __forceinline__ uint32_t count_high(const uint8_t* p, uint32_t n) {
    if (!n) return 0;
    const uintptr_t a = reinterpret_cast<uintptr_t>(p), e = a + n;
    uint32_t c = 0;
    for (uintptr_t q = a & ~uintptr_t(15); q < e; q += 16) {
        const uint4 v = *reinterpret_cast<const uint4*>(q);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uint32_t m = w[k] & 0x80808080u;
            if (m) {
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const uintptr_t x = q + 4 * k + b;
                    if (x < a || x >= e) m &= ~(0x80u << (8 * b));
                }
                c += __popc(m);
            }
        }
    }
    return c;
}

// One thread per pair (one per read single-end): both hits, the pairing,
// each line's length and record; the SEQ / QUAL UTF-8 check; mapped records
// and error bits gathered per block.
__global__ void __launch_bounds__(THREADS) sam_layout_kernel(SamDev d, uint64_t n_units, uint32_t* line_len,
                                                             LineRec* recs) {
    __shared__ unsigned long long blk_mapped;
    __shared__ unsigned blk_err;
    if (threadIdx.x == 0) {
        blk_mapped = 0;
        blk_err = 0;
    }
    __syncthreads();
    unsigned err = 0;
    uint32_t mapped = 0;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * THREADS;
    for (uint64_t u = static_cast<uint64_t>(blockIdx.x) * THREADS + threadIdx.x; u < n_units; u += stride) {
        Hit hs[2];
        hs[0] = hit_of(d, u, err);
        const int k = d.paired ? 2 : 1;
        if (d.paired) {
            hs[1] = hit_of(d, u + d.n1, err);
            pair_up(hs[0], hs[1], d.seq_len[u + d.n1]);
        }
        for (int m = 0; m < k; ++m) {
            const Hit& h = hs[m];
            const uint64_t r = u + static_cast<uint64_t>(m) * d.n1;
            const uint64_t L = d.paired ? 2 * u + m : u;
            if (!spans_ok(d, r)) {
                err |= E_SPAN;
                line_len[L] = 0;
                continue;
            }
            const uint8_t* sq = d.arena + d.seq_off[r];
            const uint8_t* ql = d.arena + d.qual_off[r];
            const uint32_t n_nm = d.name_len[r], n_sq = d.seq_len[r], n_ql = d.qual_len[r];
            const uint32_t high = count_high(d.arena + d.name_off[r], n_nm);
            if ((count_high(sq, n_sq) || count_high(ql, n_ql)) && !(utf8_ok(sq, n_sq) && utf8_ok(ql, n_ql)))
                err |= E_UTF8;
            const uint64_t len = head_len(h, n_nm + 2ull * high) + n_sq + 1 + n_ql + 6 + d.rg_n + 1;
            if (len > 0xffffffffull) err |= E_OVER;
            line_len[L] = static_cast<uint32_t>(len);
            mapped += !h.star;
            LineRec rc;
            rc.flag = h.flag;
            rc.pos1 = h.pos1;
            rc.pnext = h.pnext;
            rc.tlen = h.tlen;
            rc.contig_off = h.contig_off;
            rc.rnext_off = h.rnext_off;
            rc.mapq = static_cast<uint32_t>(h.mapq);
            rc.sl = static_cast<uint32_t>(h.sl);
            rc.sr = static_cast<uint32_t>(h.sr);
            rc.m = static_cast<uint32_t>(h.mapped ? h.m : 0);
            rc.contig_len = h.contig_len;
            rc.rnext_len = h.rnext_len;
            rc.contig_kind = h.contig_kind;
            rc.rnext_kind = h.rnext_kind;
            rc.mapped = h.mapped;
            rc.widen = high != 0;
            rc.pad = 0;
            recs[L] = rc;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        err |= __shfl_xor_sync(FULL, err, o);
        mapped += __shfl_xor_sync(FULL, mapped, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (mapped) atomicAdd(&blk_mapped, static_cast<unsigned long long>(mapped));
        if (err) atomicOr(&blk_err, err);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (blk_mapped) atomicAdd(&d.status[1], blk_mapped);
        if (blk_err) atomicOr(&d.status[2], static_cast<unsigned long long>(blk_err));
    }
}

// The aligned 4-byte words covering a span, up to 32 * SPAN_UNROLL of them
// (256 bytes) loaded at once: one round of loads for a span that fits.
struct SpanWords {
    uint32_t v[SPAN_UNROLL];
    uint32_t lead, nw;
};

__device__ __forceinline__ bool span_fits(const uint8_t* src, uint32_t n) {
    return ((reinterpret_cast<uintptr_t>(src) & 3) + n + 3) / 4 <= 32u * SPAN_UNROLL;
}

__device__ __forceinline__ void span_load(SpanWords& s, const uint8_t* src, uint32_t n, int lane) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(src);
    const uint32_t* w0 = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
    s.lead = static_cast<uint32_t>(a & 3);
    s.nw = n ? (s.lead + n + 3) >> 2 : 0;
#pragma unroll
    for (int t = 0; t < SPAN_UNROLL; ++t) {
        const uint32_t i = 32 * t + lane;
        s.v[t] = i < s.nw ? w0[i] : 0u;
    }
}

template <typename F>
__device__ __forceinline__ void span_scatter(const SpanWords& s, uint32_t n, int lane, F&& f) {
#pragma unroll
    for (int t = 0; t < SPAN_UNROLL; ++t) {
        const uint32_t i = 32 * t + lane;
        if (i < s.nw) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t j = 4 * i + k - s.lead;  // wraps below the span's start
                if (j < n) f(j, static_cast<uint8_t>(s.v[t] >> (8 * k)));
            }
        }
    }
}

// Calls f(j, byte) for every byte j of src[0, n), any length, 32 *
// SPAN_UNROLL words per round.
template <typename F>
__device__ __forceinline__ void for_span_bytes(const uint8_t* src, uint32_t n, int lane, F&& f) {
    for (uint32_t b = 0; b < n;) {
        const uint8_t* p = src + b;
        const uint32_t lead = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(p) & 3);
        const uint32_t take = min(n - b, 32u * SPAN_UNROLL * 4 - lead);
        SpanWords s;
        span_load(s, p, take, lane);
        span_scatter(s, take, lane, [&](uint32_t j, uint8_t c) { f(b + j, c); });
        b += take;
    }
}

// The decimal text of v at o (k = sdig(v) bytes); 32-bit divisions while
// the value fits.
__device__ __forceinline__ void put_int(uint8_t* o, int64_t v, uint32_t k) {
    uint64_t u = mag(v);
    uint32_t j = k;
    while (u >> 32) {
        o[--j] = static_cast<uint8_t>('0' + u % 10);
        u /= 10;
    }
    uint32_t x = static_cast<uint32_t>(u);
    do {
        o[--j] = static_cast<uint8_t>('0' + x % 10);
        x /= 10;
    } while (x);
    if (v < 0) o[0] = '-';
}

// Lanes copy a contig field: a name span, "*" or "=".
__device__ __forceinline__ void put_field(uint8_t* o, const SamDev& d, uint8_t kind, uint64_t off, uint32_t len,
                                          int lane) {
    if (kind == K_NAME) {
        for (uint32_t j = lane; j < len; j += 32) o[j] = d.names[off + j];
    } else if (lane == 0) {
        o[0] = kind == K_EQ ? '=' : '*';
    }
}

__device__ __forceinline__ uint8_t complement(uint8_t c) {
    return c == 'A' ? 'T' : c == 'T' ? 'A' : c == 'C' ? 'G' : c == 'G' ? 'C' : 'N';
}

// One line at o (shared-memory stage or the output itself) by the warp.
// The name, SEQ and QUAL words are loaded before the integer fields are
// formatted, so the loads overlap that work.
__device__ void build_line(uint8_t* o, const SamDev& d, const LineRec& h, const uint8_t* nm, uint32_t n_nm,
                           const uint8_t* sq, uint32_t n_sq, const uint8_t* ql, uint32_t n_ql, int lane) {
    const bool pre = !h.widen && span_fits(nm, n_nm) && span_fits(sq, n_sq) && span_fits(ql, n_ql);
    SpanWords wn, ws, wq;
    if (pre) {
        span_load(wn, nm, n_nm, lane);
        span_load(ws, sq, n_sq, lane);
        span_load(wq, ql, n_ql, lane);
    }
    uint64_t w = n_nm;
    if (h.widen) {  // each byte >= 0x80 of the name becomes U+FFFD
        w = 0;
        for (uint32_t b = 0; b < n_nm; b += 32) {
            const uint32_t i = b + lane;
            const uint8_t c = i < n_nm ? nm[i] : 0;
            const uint32_t wd = i < n_nm ? (c >= 0x80 ? 3u : 1u) : 0u;
            uint32_t incl = wd;
            for (int s = 1; s < 32; s <<= 1) {
                const uint32_t v = __shfl_up_sync(FULL, incl, s);
                if (lane >= s) incl += v;
            }
            const uint32_t ex = incl - wd;
            if (wd == 1) {
                o[w + ex] = c;
            } else if (wd == 3) {
                o[w + ex] = 0xef;
                o[w + ex + 1] = 0xbf;
                o[w + ex + 2] = 0xbd;
            }
            w += __shfl_sync(FULL, incl, 31);
        }
    }
    // FLAG, RNAME, POS, MAPQ, CIGAR, RNEXT, PNEXT, TLEN: every lane knows the
    // layout
    const uint32_t d_flag = sdig(h.flag), d_pos = sdig(h.pos1), d_mapq = ndig(h.mapq);
    const uint32_t d_sl = h.sl > 0 ? ndig(h.sl) + 1 : 0, d_m = h.mapped ? ndig(h.m) : 0;
    const uint32_t d_sr = h.sr > 0 ? ndig(h.sr) + 1 : 0, d_pn = sdig(h.pnext), d_tl = sdig(h.tlen);
    const uint32_t cig = h.mapped ? d_sl + d_m + 1 + d_sr : 1;
    const uint64_t w_contig = w + 2 + d_flag;
    const uint64_t p_tab3 = w_contig + h.contig_len, p_pos = p_tab3 + 1, p_mapq = p_pos + d_pos + 1;
    const uint64_t p_cig = p_mapq + d_mapq + 1;
    const uint64_t w_rnext = p_cig + cig + 1;
    const uint64_t p_tab7 = w_rnext + h.rnext_len, p_pnext = p_tab7 + 1, p_tlen = p_pnext + d_pn + 1;
    const uint64_t w_seq = p_tlen + d_tl + 1;
    // each of lanes 0-7 picks one number, lanes 3-5 and 8-16 one separator;
    // the picks are selects, the writes one code path for all lanes
    int64_t v = 0;
    uint64_t vp = 0, cp = 0;
    uint32_t vn = 0;
    uint8_t ch = '\t';
    bool vb = lane < 8, cb = lane >= 8 && lane <= 16;
    if (lane == 0) {
        v = h.flag, vp = w + 1, vn = d_flag;
    } else if (lane == 1) {
        v = h.pos1, vp = p_pos, vn = d_pos;
    } else if (lane == 2) {
        v = h.mapq, vp = p_mapq, vn = d_mapq;
    } else if (lane == 3) {
        vb = cb = h.mapped && h.sl > 0;
        v = h.sl, vp = p_cig, vn = d_sl - 1, cp = p_cig + d_sl - 1, ch = 'S';
    } else if (lane == 4) {
        vb = h.mapped;
        cb = true;
        v = h.m, vp = p_cig + d_sl, vn = d_m;
        cp = h.mapped ? p_cig + d_sl + d_m : p_cig;
        ch = h.mapped ? 'M' : '*';
    } else if (lane == 5) {
        vb = cb = h.mapped && h.sr > 0;
        v = h.sr, vp = p_cig + d_sl + d_m + 1, vn = d_sr - 1, cp = p_cig + d_sl + d_m + d_sr, ch = 'S';
    } else if (lane == 6) {
        v = h.pnext, vp = p_pnext, vn = d_pn;
    } else if (lane == 7) {
        v = h.tlen, vp = p_tlen, vn = d_tl;
    } else {  // the nine tabs
        cp = lane == 8    ? w
             : lane == 9  ? w_contig - 1
             : lane == 10 ? p_tab3
             : lane == 11 ? p_mapq - 1
             : lane == 12 ? p_cig - 1
             : lane == 13 ? w_rnext - 1
             : lane == 14 ? p_tab7
             : lane == 15 ? p_tlen - 1
                          : w_seq - 1;
    }
    if (vb) put_int(o + vp, v, vn);
    if (cb) o[cp] = ch;
    put_field(o + w_contig, d, h.contig_kind, h.contig_off, h.contig_len, lane);
    put_field(o + w_rnext, d, h.rnext_kind, h.rnext_off, h.rnext_len, lane);
    uint8_t* os = o + w_seq;
    uint8_t* oq = os + n_sq + 1;
    const bool rc = h.mapped && (h.flag & 16);
    auto seq_f = [&](uint32_t j, uint8_t c) { os[j] = c; };
    auto seq_r = [&](uint32_t j, uint8_t c) { os[n_sq - 1 - j] = complement(c); };
    auto qual_f = [&](uint32_t j, uint8_t c) { oq[j] = c; };
    if (pre) {
        span_scatter(wn, n_nm, lane, [&](uint32_t j, uint8_t c) { o[j] = c; });
        if (rc) span_scatter(ws, n_sq, lane, seq_r);
        else span_scatter(ws, n_sq, lane, seq_f);
        span_scatter(wq, n_ql, lane, qual_f);
    } else {
        if (!h.widen) for_span_bytes(nm, n_nm, lane, [&](uint32_t j, uint8_t c) { o[j] = c; });
        if (rc) for_span_bytes(sq, n_sq, lane, seq_r);
        else for_span_bytes(sq, n_sq, lane, seq_f);
        for_span_bytes(ql, n_ql, lane, qual_f);
    }
    // SEQ <tab> QUAL, then "\tRG:Z:" + id + "\n"
    if (lane == 0) os[n_sq] = '\t';
    uint8_t* ot = oq + n_ql;
    const uint32_t n_tail = 7 + d.rg_n;
    for (uint32_t j = lane; j < n_tail; j += 32) {
        uint8_t c;
        if (j < 6) c = "\tRG:Z:"[j];
        else if (j < 6 + d.rg_n) c = d.rg[j - 6];
        else c = '\n';
        ot[j] = c;
    }
}

// One warp per line: the line in the warp's shared-memory stage at its
// destination's 16-byte phase, then 16-byte stores (byte stores at the
// ragged ends); lines longer than the stage are built in place.
__global__ void __launch_bounds__(THREADS) sam_write_kernel(SamDev d, uint64_t n_lines, const uint64_t* ends,
                                                            const LineRec* recs) {
    __shared__ __align__(16) uint8_t stage[WARPS][STAGE];
    const uint64_t total = ends[n_lines - 1];
    const bool over = total > d.cap;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        d.status[0] = total;
        if (over) atomicOr(&d.status[2], static_cast<unsigned long long>(E_OVER));
    }
    // error bits of the layout pass (the overflow bit above only repeats
    // `over`)
    if (over || *static_cast<volatile unsigned long long*>(&d.status[2]) != 0) return;
    const int lane = threadIdx.x & 31;
    uint8_t* sb = stage[threadIdx.x >> 5];
    const uint64_t w0 = (static_cast<uint64_t>(blockIdx.x) * THREADS + threadIdx.x) >> 5;
    const uint64_t nw = static_cast<uint64_t>(gridDim.x) * WARPS;
    for (uint64_t L = w0; L < n_lines; L += nw) {
        const LineRec h = recs[L];
        const uint64_t r = d.paired ? (L >> 1) + (L & 1) * d.n1 : L;
        const uint64_t start = L ? ends[L - 1] : 0, len = ends[L] - start;
        const uint8_t* nm = d.arena + d.name_off[r];
        const uint8_t* sq = d.arena + d.seq_off[r];
        const uint8_t* ql = d.arena + d.qual_off[r];
        const uint32_t n_nm = d.name_len[r], n_sq = d.seq_len[r], n_ql = d.qual_len[r];
        const uintptr_t gs = reinterpret_cast<uintptr_t>(d.sam) + start, ge = gs + len;
        const uint32_t ph = static_cast<uint32_t>(gs & 15);
        if (ph + len > STAGE) {
            build_line(d.sam + start, d, h, nm, n_nm, sq, n_sq, ql, n_ql, lane);
            continue;
        }
        build_line(sb + ph, d, h, nm, n_nm, sq, n_sq, ql, n_ql, lane);
        __syncwarp();
        const uintptr_t a0 = gs - ph;  // sb[0] stands for this aligned address
        for (uintptr_t c = a0 + 16 * lane; c < ge; c += 512) {
            const uint32_t so = static_cast<uint32_t>(c - a0);
            if (c >= gs && c + 16 <= ge) {
                *reinterpret_cast<uint4*>(c) = *reinterpret_cast<const uint4*>(sb + so);
            } else {
                for (int k = 0; k < 16; ++k) {
                    const uintptr_t x = c + k;
                    if (x >= gs && x < ge) *reinterpret_cast<uint8_t*>(x) = sb[so + k];
                }
            }
        }
        __syncwarp();
    }
}

}  // namespace

size_t sam_scratch_bytes(uint64_t n_lines) {
    size_t t = 0;
    cub::DeviceScan::InclusiveSum(nullptr, t, static_cast<const uint32_t*>(nullptr), static_cast<uint64_t*>(nullptr),
                                  static_cast<int64_t>(n_lines ? n_lines : 1));
    return align256(n_lines * 4) + align256(n_lines * 8) + align256(n_lines * sizeof(LineRec)) + align256(t);
}

int enqueue_sam(const SamDev& d, void* scratch, size_t scratch_bytes, int sm_count, cudaStream_t st) {
    const uint64_t n_lines = static_cast<uint64_t>(d.n1) * (d.paired ? 2 : 1);
    if (!n_lines) return 0;
    uint8_t* s = static_cast<uint8_t*>(scratch);
    uint32_t* line_len = reinterpret_cast<uint32_t*>(s);
    s += align256(n_lines * 4);
    uint64_t* ends = reinterpret_cast<uint64_t*>(s);
    s += align256(n_lines * 8);
    LineRec* recs = reinterpret_cast<LineRec*>(s);
    s += align256(n_lines * sizeof(LineRec));
    void* temp = s;
    size_t tb = scratch_bytes - static_cast<size_t>(s - static_cast<uint8_t*>(scratch));
    const uint64_t sms = static_cast<uint64_t>(sm_count > 0 ? sm_count : 148);
    const uint64_t n_units = d.n1;  // pairs, or reads single-end
    const uint64_t g1w = (n_units + THREADS - 1) / THREADS, g1c = sms * 8;
    sam_layout_kernel<<<static_cast<unsigned>(g1w < g1c ? g1w : g1c), THREADS, 0, st>>>(d, n_units, line_len, recs);
    check_launch(cudaGetLastError(), "sam_layout_kernel");
    check_launch(cub::DeviceScan::InclusiveSum(temp, tb, static_cast<const uint32_t*>(line_len), ends,
                                               static_cast<int64_t>(n_lines), st),
                 "sam scan");
    const uint64_t g2w = (n_lines + WARPS - 1) / WARPS, g2c = sms * 16;
    sam_write_kernel<<<static_cast<unsigned>(g2w < g2c ? g2w : g2c), THREADS, 0, st>>>(d, n_lines, ends, recs);
    check_launch(cudaGetLastError(), "sam_write_kernel");
    return 4;
}

}  // namespace ma
