// bam_pack.cu - BAM records of one mapped batch, packed on the device.
//
// Replaces the host loop _emit_bam_from_batch / _pack_bam_aln
// (fq2bam-meth/src/linear_gpu_fm.mojo:497-666, 669-984).  The reference
// packs records one after another into a host buffer; here the layout is
// split from the bytes so every record is written in parallel at the same
// offset the serial loop would give it:
//   1. bam_layout_kernel   one thread per read (single-end) or pair: flags,
//                          mate fields and the record sizes, plus every
//                          sort/markdup metadata entry except `rec`.
//   2. an inclusive scan of the record sizes (CUB) -> end offsets.
//   3. bam_records_kernel  one warp per read or pair: the warp assembles
//                          the records in a shared-memory stage placed at
//                          the destination's 16-byte phase, then stores the
//                          aligned middle with 16-byte stores and the two
//                          ragged ends with byte stores.  Records too long
//                          for the stage are assembled in place in HBM.
// All byte-order, clamping and truncation rules are the reference's; every
// integer is formed in 64-bit arithmetic and truncated where the reference
// stores 32 bits.
#include <cub/device/device_scan.cuh>

#include <string>

#include "bam_pack.h"
#include "ma_internal.h"

namespace ma {
namespace {

constexpr int LAYOUT_THREADS = 256;
constexpr int REC_WARPS = 8;
constexpr int REC_STAGE = 4096;  // bytes of shared memory per warp

// Per-record fields after the mate logic of _emit_bam_from_batch.
struct BamRec {
    int64_t flag, tid, pos, mapq, sl, sr, nm, qlen, ntid, npos, tlen;
    uint64_t name_off, orig_off, qual_off;
    uint32_t name_len, qual_len;
    bool has_qual;  // qualities exist and their length equals qlen
    bool bad;       // an arena span lies outside the arena
};

// One read's own fields; `mate_bit` is 64 for R1 and 128 for R2
// (L756-768, L838-848).
__device__ __forceinline__ void load_read(const BamDev& b, uint64_t r, int64_t mate_bit, BamRec& o) {
    const int64_t rid = b.rid[r];
    o.pos = b.pos[r];
    o.mapq = b.mapq[r];
    o.flag = static_cast<int64_t>(b.flag[r]) | 1 | mate_bit;
    o.sl = b.sl[r];
    o.sr = b.sr[r];
    o.nm = b.nm[r];
    o.tid = -1;
    if (rid >= 0 && rid < b.n_tid) o.tid = b.rid_to_tid[rid];
    else o.flag |= 4;
    o.qlen = b.orig_len[r];
    o.name_off = b.name_off[r];
    o.name_len = b.name_len[r];
    o.orig_off = b.orig_off[r];
    o.ntid = o.npos = -1;
    o.tlen = 0;
    o.bad = o.name_off + o.name_len > b.arena_bytes || o.orig_off + static_cast<uint64_t>(o.qlen) > b.arena_bytes;
    o.has_qual = false;
    o.qual_off = 0;
    o.qual_len = 0;
    if (b.qual_off) {
        o.qual_off = b.qual_off[r];
        o.qual_len = b.qual_len[r];
        o.has_qual = static_cast<int64_t>(o.qual_len) == o.qlen;
        if (o.has_qual && o.qual_off + o.qual_len > b.arena_bytes) o.bad = true;
    }
    if (o.bad) o.has_qual = false;
}

// Mate flags, mate fields and TLEN of a pair (L849-874).
__device__ __forceinline__ void pair_up(BamRec& a, BamRec& c) {
    if (a.tid < 0) c.flag |= 8;
    if (c.tid < 0) a.flag |= 8;
    if (a.tid >= 0 && c.tid >= 0 && a.tid == c.tid) {
        a.flag |= 2;
        c.flag |= 2;
        a.ntid = a.tid;
        c.ntid = c.tid;
        a.npos = c.pos;
        c.npos = a.pos;
        int64_t tl = c.pos - a.pos;
        if (tl < 0) tl = -tl;
        tl += c.qlen;
        a.tlen = a.pos <= c.pos ? tl : -tl;
        c.tlen = -a.tlen;
    } else {
        if (a.tid >= 0) {
            c.ntid = a.tid;
            c.npos = a.pos;
        }
        if (c.tid >= 0) {
            a.ntid = c.tid;
            a.npos = c.pos;
        }
    }
}

// Loads unit u (a read, or pair u) into r[0] (and r[1]).
__device__ __forceinline__ void load_unit(const BamDev& b, uint64_t u, BamRec* r) {
    load_read(b, u, 64, r[0]);
    if (b.paired) {
        load_read(b, static_cast<uint64_t>(b.n1) + u, 128, r[1]);
        pair_up(r[0], r[1]);
    }
}

// Clip clamping of _pack_bam_aln (L521-530) and _unclipped5 (L371-386).
__device__ __forceinline__ void clamp_clips(const BamRec& r, int64_t& sl, int64_t& sr, int64_t& mid) {
    sl = r.sl < 0 ? 0 : r.sl;
    sr = r.sr < 0 ? 0 : r.sr;
    if (sl + sr >= r.qlen) sl = sr = 0;
    mid = r.qlen - sl - sr;
}

__device__ __forceinline__ bool placed(const BamRec& r) { return r.tid >= 0 && (r.flag & 4) == 0; }

__device__ __forceinline__ int64_t n_cigar_of(const BamRec& r) {
    int64_t sl, sr, mid;
    clamp_clips(r, sl, sr, mid);
    return placed(r) ? (sl > 0) + (mid > 0) + (sr > 0) : 0;
}

// Bytes of the record including its block_size word (L545-546).
__device__ __forceinline__ uint64_t record_bytes(const BamRec& r, uint32_t rg_n) {
    const int64_t block = 32 + (static_cast<int64_t>(r.name_len) + 1) + 4 * n_cigar_of(r) + (r.qlen + 1) / 2 +
                          r.qlen + (3 + static_cast<int64_t>(rg_n) + 1 + 4);
    return static_cast<uint64_t>(4 + block);
}

__device__ __forceinline__ int64_t unclipped5(const BamRec& r) {
    if ((r.flag & 4) != 0 || r.qlen <= 0) return 0;
    int64_t sl, sr, mid;
    clamp_clips(r, sl, sr, mid);
    return (r.flag & 16) ? r.pos + mid + sl - 1 : r.pos - sl;
}

__device__ __forceinline__ uint64_t coord_key(int64_t tid, int64_t pos, uint64_t orig) {
    if (tid < 0) return (0xffffffffull << 32) | (orig & 0xffffffffull);
    return (static_cast<uint64_t>(tid) << 32) | static_cast<uint64_t>(pos < 0 ? 0 : pos);
}

__device__ __forceinline__ uint64_t pack_end(const BamRec& r) {
    const uint64_t t = r.tid >= 0 ? static_cast<uint64_t>(r.tid + 1) : 0;
    int64_t u = unclipped5(r) + 1073741824;
    if (u < 0) u = 0;
    return (t << 48) | (static_cast<uint64_t>((r.flag >> 4) & 1) << 47) |
           (static_cast<uint64_t>(u) & 140737488355327ull);
}

__device__ __forceinline__ int64_t clamp255(int64_t v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }

// Metadata and sizes, one thread per unit (L799-822, L928-982).
__global__ void __launch_bounds__(LAYOUT_THREADS) bam_layout_kernel(BamDev b, uint64_t* rec_bytes) {
    const uint64_t n_units = b.n1;
    const uint64_t u = static_cast<uint64_t>(blockIdx.x) * LAYOUT_THREADS + threadIdx.x;
    unsigned mapped = 0;
    unsigned bad = 0;
    if (u < n_units) {
        BamRec r[2];
        load_unit(b, u, r);
        if (!b.paired) {
            const uint64_t t = b.n_reads + u, m = t - b.meta_origin;
            b.coord[m] = coord_key(r[0].tid, r[0].pos, t);
            if (r[0].tid >= 0) {
                b.dhi[m] = pack_end(r[0]);
                b.dlo[m] = 0;
            } else {
                b.dhi[m] = ~0ull;
                b.dlo[m] = t;
            }
            const uint64_t n = record_bytes(r[0], b.rg_n);
            rec_bytes[u] = n;
            b.len[m] = static_cast<uint32_t>(n);
            b.score[m] = static_cast<uint32_t>((r[0].mapq << 8) | (255 - clamp255(r[0].nm)));
            b.pair[m] = static_cast<uint32_t>(b.n_total + t);
            mapped = r[0].tid >= 0;
            bad = r[0].bad;
        } else {
            const uint64_t i1 = b.n_reads + 2 * u, i2 = i1 + 1;
            const uint32_t pid = static_cast<uint32_t>((b.n_total + i1) / 2);
            const uint32_t pscore =
                static_cast<uint32_t>(((r[0].mapq + r[1].mapq) << 8) | (255 - clamp255(r[0].nm + r[1].nm)));
            uint64_t dhi = ~0ull, dlo = i1;
            if (r[0].tid >= 0 || r[1].tid >= 0) {
                const uint64_t e1 = pack_end(r[0]), e2 = pack_end(r[1]);
                if (r[0].tid < 0) {
                    dhi = e2;
                    dlo = 0;
                } else if (r[1].tid < 0) {
                    dhi = e1;
                    dlo = 0;
                } else {
                    dhi = e1 <= e2 ? e1 : e2;
                    dlo = e1 <= e2 ? e2 : e1;
                }
            }
            const uint64_t n1b = record_bytes(r[0], b.rg_n), n2b = record_bytes(r[1], b.rg_n);
            rec_bytes[2 * u] = n1b;
            rec_bytes[2 * u + 1] = n2b;
            const uint64_t m1 = i1 - b.meta_origin, m2 = m1 + 1;
            b.coord[m1] = coord_key(r[0].tid, r[0].pos, i1);
            b.coord[m2] = coord_key(r[1].tid, r[1].pos, i2);
            b.dhi[m1] = b.dhi[m2] = dhi;
            b.dlo[m1] = b.dlo[m2] = dlo;
            b.len[m1] = static_cast<uint32_t>(n1b);
            b.len[m2] = static_cast<uint32_t>(n2b);
            b.score[m1] = b.score[m2] = pscore;
            b.pair[m1] = b.pair[m2] = pid;
            mapped = (r[0].tid >= 0) + (r[1].tid >= 0);
            bad = r[0].bad + r[1].bad;
        }
    }
    // one atomic per warp for each counter
    for (int o = 16; o > 0; o >>= 1) {
        mapped += __shfl_xor_sync(0xffffffffu, mapped, o);
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (mapped) atomicAdd(&b.status[1], static_cast<unsigned long long>(mapped));
        if (bad) atomicAdd(&b.status[2], static_cast<unsigned long long>(bad));
    }
}

// _nt16 (L455-464): A/C/G/T in either case -> 1/2/4/8, anything else 15.
// b | 32 folds exactly the two cases of each letter onto the lower one.
__device__ __forceinline__ uint32_t nt16(uint32_t b) {
    const uint32_t c = b | 32;
    return c == 97 ? 1 : c == 99 ? 2 : c == 103 ? 4 : c == 116 ? 8 : 15;
}
// _nt16_comp (L467-476) on codes 1/2/4/8/15: reversing the four bits swaps
// A<->T and C<->G and keeps 15.
__device__ __forceinline__ uint32_t nt16_comp(uint32_t x) { return __brev(x) >> 28; }

__device__ __forceinline__ int64_t reg2bin(int64_t beg, int64_t end) {
    if (end <= beg) end = beg + 1;
    --end;
    if ((beg >> 14) == (end >> 14)) return 4681 + (beg >> 14);
    if ((beg >> 17) == (end >> 17)) return 585 + (beg >> 17);
    if ((beg >> 20) == (end >> 20)) return 73 + (beg >> 20);
    if ((beg >> 23) == (end >> 23)) return 9 + (beg >> 23);
    if ((beg >> 26) == (end >> 26)) return 1 + (beg >> 26);
    return 0;
}

// Word k of the nine little-endian header words of _pack_bam_aln
// (L551-572): block_size, refID, pos, bin_mq_nl, flag_nc, l_seq,
// next_refID, next_pos, tlen.
__device__ __forceinline__ uint32_t header_word(int k, uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3,
                                                uint32_t w4, uint32_t w5, uint32_t w6, uint32_t w7, uint32_t w8) {
    uint32_t v = w8;
    v = k == 7 ? w7 : v;
    v = k == 6 ? w6 : v;
    v = k == 5 ? w5 : v;
    v = k == 4 ? w4 : v;
    v = k == 3 ? w3 : v;
    v = k == 2 ? w2 : v;
    v = k == 1 ? w1 : v;
    return k == 0 ? w0 : v;
}

// The warp writes one record at dst (shared or global), _pack_bam_aln
// L520-666.  Returns the record's byte count.
__device__ __forceinline__ uint64_t write_record(uint8_t* dst, const BamDev& b, const BamRec& r, int lane) {
    const bool rev = (r.flag & 16) != 0;
    int64_t sl, sr, mid;
    clamp_clips(r, sl, sr, mid);
    if (rev) {
        const int64_t t = sl;
        sl = sr;
        sr = t;
    }
    const bool pl = placed(r);
    const int n_cigar = pl ? (sl > 0) + (mid > 0) + (sr > 0) : 0;
    const int64_t l_qname = static_cast<int64_t>(r.name_len) + 1;
    const int64_t qlen = r.qlen;
    const int64_t nb = (qlen + 1) / 2;
    const int64_t n_tags = 3 + static_cast<int64_t>(b.rg_n) + 1 + 4;
    const int64_t block = 32 + l_qname + 4 * n_cigar + nb + qlen + n_tags;
    const int64_t mq = clamp255(r.mapq);
    if (lane < 9) {
        const int64_t bin = pl ? reg2bin(r.pos, r.pos + mid) : 4680;
        const uint32_t v = header_word(
            lane, static_cast<uint32_t>(block), static_cast<uint32_t>(pl ? r.tid : -1),
            static_cast<uint32_t>(pl ? r.pos : -1), static_cast<uint32_t>((bin << 16) | (mq << 8) | l_qname),
            static_cast<uint32_t>((r.flag << 16) | n_cigar), static_cast<uint32_t>(qlen),
            static_cast<uint32_t>(r.ntid < 0 ? -1 : r.ntid), static_cast<uint32_t>(r.ntid < 0 ? -1 : r.npos),
            static_cast<uint32_t>(r.tlen));
        uint8_t* h = dst + 4 * lane;
        h[0] = v & 255;
        h[1] = (v >> 8) & 255;
        h[2] = (v >> 16) & 255;
        h[3] = v >> 24;
    }

    const uint8_t* name = b.arena + r.name_off;
    uint8_t* p = dst + 36;
    for (int64_t i = lane; i < l_qname; i += 32) p[i] = (i < r.name_len && !r.bad) ? name[i] : 0;
    p += l_qname;

    if (lane < n_cigar) {
        // the lane-th present op of S(sl) M(mid) S(sr)
        int k = lane;
        uint32_t op;
        if (sl > 0 && k-- == 0) op = static_cast<uint32_t>((sl << 4) | 4);
        else if (mid > 0 && k-- == 0) op = static_cast<uint32_t>(mid << 4);
        else op = static_cast<uint32_t>((sr << 4) | 4);
        uint8_t* c = p + 4 * lane;
        c[0] = op & 255;
        c[1] = (op >> 8) & 255;
        c[2] = (op >> 16) & 255;
        c[3] = op >> 24;
    }
    p += 4 * n_cigar;

    // SEQ: byte k holds bases 2k and 2k+1 of the stored strand; on the
    // reverse strand base i is the complement of original base qlen-1-i,
    // so the odd tail reads original base 0 (L617-639).
    const uint8_t* seq = b.arena + r.orig_off;
    for (int64_t k = lane; k < nb; k += 32) {
        uint32_t v = 0;
        if (!r.bad) {
            const int64_t i0 = 2 * k;
            const bool two = i0 + 1 < qlen;
            uint32_t a, c = 0;
            if (rev) {
                a = nt16_comp(nt16(seq[qlen - 1 - i0]));
                if (two) c = nt16_comp(nt16(seq[qlen - 2 - i0]));
            } else {
                a = nt16(seq[i0]);
                if (two) c = nt16(seq[i0 + 1]);
            }
            v = (a << 4) | c;
        }
        p[k] = static_cast<uint8_t>(v);
    }
    p += nb;

    // QUAL: phred+33 minus 33, 255 below '!', all 255 without qualities of
    // the read's length; reversed on the reverse strand (L640-654).
    const uint8_t* qual = b.arena + r.qual_off;
    for (int64_t k = lane; k < qlen; k += 32) {
        uint32_t v = 255;
        if (r.has_qual) {
            const uint32_t q = qual[rev ? qlen - 1 - k : k];
            v = q >= 33 ? q - 33 : 255;
        }
        p[k] = static_cast<uint8_t>(v);
    }
    p += qlen;

    // RG:Z:<rg> and NM:C:<nm> (L655-665)
    const int64_t rg_n = b.rg_n;
    for (int64_t i = lane; i < n_tags; i += 32) {
        uint32_t v;
        if (i < 3) v = i == 0 ? 82 : (i == 1 ? 71 : 90);
        else if (i < 3 + rg_n) v = b.rg[i - 3];
        else if (i == 3 + rg_n) v = 0;
        else if (i < 3 + rg_n + 4) v = (i == 4 + rg_n) ? 78 : (i == 5 + rg_n ? 77 : 67);
        else v = static_cast<uint32_t>(clamp255(r.nm));
        p[i] = static_cast<uint8_t>(v);
    }
    return static_cast<uint64_t>(4 + block);
}

// Copies `span` staged bytes (the stage holds them from offset g & 15,
// g = the destination address) to the destination: 16-byte stores for the
// aligned middle, byte stores for the ragged ends.
__device__ __forceinline__ void flush_stage(uint8_t* gdst, const uint8_t* stage, uint64_t span, int lane) {
    const uintptr_t g0 = reinterpret_cast<uintptr_t>(gdst);
    const uint32_t s0 = static_cast<uint32_t>(g0 & 15);
    const uintptr_t a = (g0 + 15) & ~static_cast<uintptr_t>(15);
    const uintptr_t e = (g0 + span) & ~static_cast<uintptr_t>(15);
    uint64_t head = span, tail_from = span;
    if (e > a) {
        head = a - g0;
        tail_from = e - g0;
        const uint64_t n16 = (e - a) / 16;
        const uint4* src = reinterpret_cast<const uint4*>(stage + s0 + head);
        uint4* dst = reinterpret_cast<uint4*>(a);
        for (uint64_t c = lane; c < n16; c += 32) dst[c] = src[c];
    }
    for (uint64_t i = lane; i < head; i += 32) gdst[i] = stage[s0 + i];
    for (uint64_t i = tail_from + lane; i < span; i += 32) gdst[i] = stage[s0 + i];
}

__global__ void __launch_bounds__(REC_WARPS * 32) bam_records_kernel(BamDev b, const uint64_t* rec_end) {
    __shared__ __align__(16) uint8_t stage[REC_WARPS][REC_STAGE];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t n_units = b.n1;
    const uint64_t n_rec = b.paired ? 2 * n_units : n_units;
    const uint64_t total = rec_end[n_rec - 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) b.status[0] = total;
    if (total > b.cap) return;
    const uint64_t chunk_hi = static_cast<uint64_t>(b.chunk) << 32;
    for (uint64_t u = static_cast<uint64_t>(blockIdx.x) * REC_WARPS + w; u < n_units;
         u += static_cast<uint64_t>(gridDim.x) * REC_WARPS) {
        BamRec r[2];
        load_unit(b, u, r);
        const uint64_t j0 = b.paired ? 2 * u : u;
        const uint64_t start = j0 ? rec_end[j0 - 1] : 0;
        const uint64_t end = rec_end[b.paired ? j0 + 1 : j0];
        uint8_t* gdst = b.bam + start;
        const uint32_t s0 = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(gdst) & 15);
        const uint64_t span = end - start;
        const bool staged = s0 + span <= REC_STAGE;
        uint8_t* dst = staged ? stage[w] + s0 : gdst;
        const uint64_t n0 = write_record(dst, b, r[0], lane);
        if (b.paired) write_record(dst + n0, b, r[1], lane);
        if (lane == 0) {
            const uint64_t m = b.n_reads + j0 - b.meta_origin;
            b.rec[m] = chunk_hi | start;
            if (b.paired) b.rec[m + 1] = chunk_hi | (start + n0);
        }
        if (staged) {
            __syncwarp();
            flush_stage(gdst, stage[w], span, lane);
            __syncwarp();
        }
    }
}

void check_launch(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

size_t align256(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }

size_t scan_temp_bytes(uint64_t n_rec) {
    size_t t = 0;
    cub::DeviceScan::InclusiveSum(nullptr, t, static_cast<const uint64_t*>(nullptr),
                                  static_cast<uint64_t*>(nullptr), static_cast<int64_t>(n_rec));
    return t;
}

}  // namespace

size_t bam_scratch_bytes(uint64_t n_rec) {
    return 2 * align256(n_rec * sizeof(uint64_t)) + align256(scan_temp_bytes(n_rec));
}

const uint64_t* bam_total_in_scratch(const void* scratch, uint64_t n_rec) {
    const uint8_t* s = static_cast<const uint8_t*>(scratch);
    return reinterpret_cast<const uint64_t*>(s + align256(n_rec * sizeof(uint64_t))) + (n_rec - 1);
}

int enqueue_bam_layout(const BamDev& b, void* scratch, size_t scratch_bytes, cudaStream_t st) {
    const uint64_t n_rec = b.paired ? 2ull * b.n1 : b.n1;
    uint8_t* s = static_cast<uint8_t*>(scratch);
    uint64_t* sizes = reinterpret_cast<uint64_t*>(s);
    uint64_t* ends = reinterpret_cast<uint64_t*>(s + align256(n_rec * sizeof(uint64_t)));
    void* temp = s + 2 * align256(n_rec * sizeof(uint64_t));
    size_t temp_bytes = scratch_bytes - 2 * align256(n_rec * sizeof(uint64_t));
    const unsigned grid = static_cast<unsigned>((b.n1 + LAYOUT_THREADS - 1) / LAYOUT_THREADS);
    bam_layout_kernel<<<grid, LAYOUT_THREADS, 0, st>>>(b, sizes);
    check_launch(cudaGetLastError(), "bam_layout_kernel");
    check_launch(cub::DeviceScan::InclusiveSum(temp, temp_bytes, static_cast<const uint64_t*>(sizes), ends,
                                               static_cast<int64_t>(n_rec), st),
                 "bam record scan");
    return 3;  // the layout kernel and the scan's two
}

int enqueue_bam_records(const BamDev& b, const void* scratch, int sm_count, cudaStream_t st) {
    const uint64_t n_rec = b.paired ? 2ull * b.n1 : b.n1;
    const uint64_t* ends =
        reinterpret_cast<const uint64_t*>(static_cast<const uint8_t*>(scratch) + align256(n_rec * sizeof(uint64_t)));
    const uint64_t want = (b.n1 + REC_WARPS - 1) / REC_WARPS;
    const uint64_t cap = static_cast<uint64_t>(sm_count > 0 ? sm_count : 148) * 6;
    const unsigned grid = static_cast<unsigned>(want < cap ? want : cap);
    bam_records_kernel<<<grid, REC_WARPS * 32, 0, st>>>(b, ends);
    check_launch(cudaGetLastError(), "bam_records_kernel");
    return 1;
}

}  // namespace ma
