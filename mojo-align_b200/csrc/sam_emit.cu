// sam_emit.cu - SAM text lines of one mapped batch on the device.
//
// Replaces the per-record host loop of map_fastq_fm_gpu's SAM path
// (fq2bam-meth/src/linear_gpu_fm.mojo:2787-2836), which builds a LinearHit
// per read with _hit_from_fm (L987-1025), pairs mates with pair_hits
// (fq2bam-meth/src/linear_extend.mojo:263-294), formats each line with
// hit_to_sam_line (L297-320) + the RG tag (_sam_with_rg_fm, L80-81) and
// writes it.  Here the lines of a whole batch are built in HBM in three
// passes over one warp per line:
//   1. sam_layout_kernel: each line's byte length (the hit and its mate are
//      both resolved, so pair fields are known), names' bytes >= 0x80
//      counted (each becomes U+FFFD), SEQ / QUAL checked for strict UTF-8,
//      mapped records and error bits gathered per block;
//   2. a device scan of the lengths (line end offsets);
//   3. sam_write_kernel: the line assembled in a per-warp shared-memory
//      stage at its destination's 16-byte phase (lanes copy the name, the
//      contig names, SEQ reverse-complemented on flag 16, QUAL and the RG
//      tag from aligned word loads; lane 0 writes the integer fields), then
//      stored with 16-byte stores; lines longer than the stage and names
//      that widen are built in place.
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
constexpr int SPAN_UNROLL = 4;    // words a lane loads per round of a span copy

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

// The hit of line L after pairing, and its read index.
__device__ Hit line_hit(const SamDev& d, uint64_t L, uint64_t& r, unsigned& err) {
    if (!d.paired) {
        r = L;
        return hit_of(d, L, err);
    }
    const uint64_t p = L >> 1;
    Hit a = hit_of(d, p, err);
    Hit b = hit_of(d, p + d.n1, err);
    pair_up(a, b, d.seq_len[p + d.n1]);
    r = p + (L & 1) * d.n1;
    return (L & 1) ? b : a;
}

__device__ __forceinline__ uint32_t ndig(uint64_t u) {
    uint32_t k = 1;
    while (u >= 10) {
        u /= 10;
        ++k;
    }
    return k;
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

__device__ __forceinline__ uint32_t warp_sum(uint32_t v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// Calls f(j, byte) for every byte j of src[0, n): the lanes split the
// aligned 4-byte words that cover the span, 512 bytes per round with the
// round's loads issued together.  (A word is read whole; its bytes outside
// the span lie in the same aligned word as a byte inside it.)
template <typename F>
__device__ __forceinline__ void for_span_bytes(const uint8_t* src, uint32_t n, int lane, F&& f) {
    if (!n) return;
    const uintptr_t a = reinterpret_cast<uintptr_t>(src);
    const uint32_t* w0 = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
    const uint32_t lead = static_cast<uint32_t>(a & 3);
    const uint32_t nw = (lead + n + 3) >> 2;
    for (uint32_t base = 0; base < nw; base += 32 * SPAN_UNROLL) {
        uint32_t v[SPAN_UNROLL];
#pragma unroll
        for (int t = 0; t < SPAN_UNROLL; ++t) {
            const uint32_t i = base + 32 * t + lane;
            v[t] = i < nw ? w0[i] : 0u;
        }
#pragma unroll
        for (int t = 0; t < SPAN_UNROLL; ++t) {
            const uint32_t i = base + 32 * t + lane;
            if (i < nw) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int64_t j = static_cast<int64_t>(4 * i + k) - lead;
                    if (j >= 0 && j < n) f(static_cast<uint32_t>(j), static_cast<uint8_t>(v[t] >> (8 * k)));
                }
            }
        }
    }
}

__global__ void __launch_bounds__(THREADS) sam_layout_kernel(SamDev d, uint64_t n_lines, uint32_t* line_len) {
    __shared__ unsigned long long blk_mapped;
    __shared__ unsigned blk_err;
    if (threadIdx.x == 0) {
        blk_mapped = 0;
        blk_err = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint64_t w0 = (static_cast<uint64_t>(blockIdx.x) * THREADS + threadIdx.x) >> 5;
    const uint64_t nw = static_cast<uint64_t>(gridDim.x) * WARPS;
    unsigned err = 0;
    uint32_t mapped = 0;
    for (uint64_t L = w0; L < n_lines; L += nw) {
        uint64_t r;
        const Hit h = line_hit(d, L, r, err);
        if (!spans_ok(d, r)) {
            err |= E_SPAN;
            if (lane == 0) line_len[L] = 0;
            continue;
        }
        const uint8_t* nm = d.arena + d.name_off[r];
        const uint8_t* sq = d.arena + d.seq_off[r];
        const uint8_t* ql = d.arena + d.qual_off[r];
        const uint32_t n_nm = d.name_len[r], n_sq = d.seq_len[r], n_ql = d.qual_len[r];
        uint32_t high = 0, any = 0;
        for_span_bytes(nm, n_nm, lane, [&](uint32_t, uint8_t c) { high += c >> 7; });
        for_span_bytes(sq, n_sq, lane, [&](uint32_t, uint8_t c) { any |= c >> 7; });
        for_span_bytes(ql, n_ql, lane, [&](uint32_t, uint8_t c) { any |= c >> 7; });
        high = warp_sum(high);
        if (__any_sync(FULL, any)) {  // rare: validate on one lane
            bool ok = true;
            if (lane == 0) ok = utf8_ok(sq, n_sq) && utf8_ok(ql, n_ql);
            if (!__shfl_sync(FULL, ok, 0)) err |= E_UTF8;
        }
        const uint64_t len = head_len(h, n_nm + 2ull * high) + n_sq + 1 + n_ql + 6 + d.rg_n + 1;
        if (len > 0xffffffffull) err |= E_OVER;
        if (lane == 0) {
            line_len[L] = static_cast<uint32_t>(len);
            mapped += !h.star;
        }
    }
    for (int o = 16; o > 0; o >>= 1) err |= __shfl_xor_sync(FULL, err, o);
    if (lane == 0) {
        if (mapped) atomicAdd(&blk_mapped, static_cast<unsigned long long>(mapped));
        if (err) atomicOr(&blk_err, err);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (blk_mapped) atomicAdd(&d.status[1], blk_mapped);
        if (blk_err) atomicOr(&d.status[2], static_cast<unsigned long long>(blk_err));
    }
}

__device__ __forceinline__ uint32_t put_int(uint8_t* o, int64_t v) {
    const uint32_t k = sdig(v);
    uint64_t u = mag(v);
    uint32_t j = k;
    do {
        o[--j] = static_cast<uint8_t>('0' + u % 10);
        u /= 10;
    } while (u);
    if (v < 0) o[0] = '-';
    return k;
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

// One line at o (shared-memory stage or the output itself) by the warp.
// widen: the name holds bytes >= 0x80, each written as U+FFFD.
__device__ void build_line(uint8_t* o, const SamDev& d, const Hit& h, uint64_t r, bool widen, int lane) {
    const uint8_t* nm = d.arena + d.name_off[r];
    const uint32_t n_nm = d.name_len[r];
    uint64_t w = 0;
    if (!widen) {
        for_span_bytes(nm, n_nm, lane, [&](uint32_t j, uint8_t c) { o[j] = c; });
        w = n_nm;
    } else {
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
    // FLAG, RNAME, POS, MAPQ, CIGAR, RNEXT, PNEXT, TLEN
    const uint64_t w_contig = w + 2 + sdig(h.flag);
    const uint64_t w_rnext = w_contig + h.contig_len + 4 + sdig(h.pos1) + sdig(h.mapq) + cigar_len(h);
    const uint64_t w_seq = w_rnext + h.rnext_len + 3 + sdig(h.pnext) + sdig(h.tlen);
    if (lane == 0) {
        uint64_t k = w;
        o[k++] = '\t';
        k += put_int(o + k, h.flag);
        o[k] = '\t';
        k = w_contig + h.contig_len;
        o[k++] = '\t';
        k += put_int(o + k, h.pos1);
        o[k++] = '\t';
        k += put_int(o + k, h.mapq);
        o[k++] = '\t';
        if (!h.mapped) {
            o[k++] = '*';
        } else {
            if (h.sl > 0) {
                k += put_int(o + k, h.sl);
                o[k++] = 'S';
            }
            k += put_int(o + k, h.m);
            o[k++] = 'M';
            if (h.sr > 0) {
                k += put_int(o + k, h.sr);
                o[k++] = 'S';
            }
        }
        o[k] = '\t';
        k = w_rnext + h.rnext_len;
        o[k++] = '\t';
        k += put_int(o + k, h.pnext);
        o[k++] = '\t';
        k += put_int(o + k, h.tlen);
        o[k] = '\t';
    }
    put_field(o + w_contig, d, h.contig_kind, h.contig_off, h.contig_len, lane);
    put_field(o + w_rnext, d, h.rnext_kind, h.rnext_off, h.rnext_len, lane);
    // SEQ (reverse complement on flag 16: A<->T, C<->G, anything else N)
    const uint8_t* sq = d.arena + d.seq_off[r];
    const uint32_t n_sq = d.seq_len[r];
    uint8_t* os = o + w_seq;
    if (h.mapped && (h.flag & 16)) {
        for_span_bytes(sq, n_sq, lane, [&](uint32_t j, uint8_t c) {
            os[n_sq - 1 - j] = c == 'A' ? 'T' : c == 'T' ? 'A' : c == 'C' ? 'G' : c == 'G' ? 'C' : 'N';
        });
    } else {
        for_span_bytes(sq, n_sq, lane, [&](uint32_t j, uint8_t c) { os[j] = c; });
    }
    // QUAL, then "\tRG:Z:" + id + "\n"
    const uint8_t* ql = d.arena + d.qual_off[r];
    const uint32_t n_ql = d.qual_len[r];
    uint8_t* oq = os + n_sq + 1;
    if (lane == 0) os[n_sq] = '\t';
    for_span_bytes(ql, n_ql, lane, [&](uint32_t j, uint8_t c) { oq[j] = c; });
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

__global__ void __launch_bounds__(THREADS) sam_write_kernel(SamDev d, uint64_t n_lines, const uint64_t* ends) {
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
        uint64_t r;
        unsigned err = 0;
        const Hit h = line_hit(d, L, r, err);
        const uint64_t start = L ? ends[L - 1] : 0, len = ends[L] - start;
        // the name's width follows from the line's length: wider than the
        // name when it holds bytes >= 0x80
        const uint64_t rest = head_len(h, 0) + d.seq_len[r] + 1 + d.qual_len[r] + 7 + d.rg_n;
        const bool widen = len - rest != d.name_len[r];
        const uintptr_t gs = reinterpret_cast<uintptr_t>(d.sam) + start, ge = gs + len;
        const uint32_t ph = static_cast<uint32_t>(gs & 15);
        if (widen || ph + len > STAGE) {  // long lines and widened names: straight to the output
            build_line(d.sam + start, d, h, r, widen, lane);
            continue;
        }
        build_line(sb + ph, d, h, r, false, lane);
        __syncwarp();
        // the stage out in 16-byte stores (sb[0] is the aligned address
        // gs - ph), byte stores at the ragged ends
        const uintptr_t a0 = gs - ph;
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
    return align256(n_lines * 4) + align256(n_lines * 8) + align256(t);
}

int enqueue_sam(const SamDev& d, void* scratch, size_t scratch_bytes, int sm_count, cudaStream_t st) {
    const uint64_t n_lines = static_cast<uint64_t>(d.n1) * (d.paired ? 2 : 1);
    if (!n_lines) return 0;
    uint8_t* s = static_cast<uint8_t*>(scratch);
    uint32_t* line_len = reinterpret_cast<uint32_t*>(s);
    uint64_t* ends = reinterpret_cast<uint64_t*>(s + align256(n_lines * 4));
    void* temp = s + align256(n_lines * 4) + align256(n_lines * 8);
    size_t tb = scratch_bytes - align256(n_lines * 4) - align256(n_lines * 8);
    const uint64_t want = (n_lines + WARPS - 1) / WARPS;
    const uint64_t cap_blocks = static_cast<uint64_t>(sm_count > 0 ? sm_count : 148) * 16;
    const unsigned g = static_cast<unsigned>(want < cap_blocks ? want : cap_blocks);
    sam_layout_kernel<<<g, THREADS, 0, st>>>(d, n_lines, line_len);
    check_launch(cudaGetLastError(), "sam_layout_kernel");
    check_launch(cub::DeviceScan::InclusiveSum(temp, tb, static_cast<const uint32_t*>(line_len), ends,
                                               static_cast<int64_t>(n_lines), st),
                 "sam scan");
    sam_write_kernel<<<g, THREADS, 0, st>>>(d, n_lines, ends);
    check_launch(cudaGetLastError(), "sam_write_kernel");
    return 4;
}

}  // namespace ma
