// fastq_parse.cu - FASTQ record split on the device.
//
// Replaces the host record split of the FM path's two FASTQ readers and
// the row packing fq_pack_bases (fq2bam-meth/src/linear_fastq.mojo:454-492):
//   rules 0, the BAM path's reader (linear_fastq.mojo: _pipe_line L233-280,
//     _qname_span L308-325, _store_rec L365-417, fq_read_batch L437-451):
//     one trailing '\r' dropped per line, a record cut short is an error;
//   rules 1, the SAM path's reader (fq2bam-meth/python/fastq_batch.py:
//     _qname L18-28, FastqPairReader._one / read_batch L250-317): every
//     trailing '\r' dropped, four lines per record whatever they hold, and
//     at the end of the stream a record cut short reads its missing lines
//     as empty.  The reference walks the decompressed
// bytes one record at a time on one host thread and copies name, original
// bases, converted bases and qualities into an arena; here the uncompressed
// bytes are copied to HBM once and become the arena themselves:
//   1. nl_count_kernel / scan / nl_write_kernel: positions of every '\n'
//      (one thread per 64-byte segment, 16-byte loads where a whole aligned
//      chunk lies in the buffer);
//   2. fq_lines_kernel (one thread): lines, complete records, the bytes
//      consumed and the truncation error, exactly as the reference's line
//      reader sees the stream;
//   3. fq_records_kernel: one thread per record, name span (leading '@'
//      dropped, cut at ' ' or '/'), SEQ and QUAL spans without their
//      trailing '\r' (one, or all), the longest SEQ;
//   4. fq_rows_kernel: one warp per read builds the padded row the mapper
//      takes ('N' fill).  The C->T / G->A conversion is applied by the
//      mapper's pack kernel, so the rows hold the original bases.
#include <cub/device/device_scan.cuh>

#include <string>

#include "fastq_parse.h"
#include "ma_internal.h"

namespace ma {
namespace {

constexpr int THREADS = 256;
constexpr int SEG = 64;  // bytes per thread in the newline passes

void check_launch(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

size_t align256(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }

__device__ __forceinline__ uint32_t nl_in_word(uint32_t w) {
    // '\n' bytes of w become zero bytes of x; the exact zero-byte test sets
    // 0x80 in exactly those byte lanes
    const uint32_t x = w ^ 0x0a0a0a0au;
    return __popc(~(((x & 0x7f7f7f7fu) + 0x7f7f7f7fu) | x | 0x7f7f7f7fu));
}

// Calls f(i) for every '\n' at byte i of segment s, in order.
template <typename F>
__device__ __forceinline__ void for_each_newline(const uint8_t* buf, uint64_t n, uint64_t s, F&& f) {
    const uint64_t b = s * SEG, e = b + SEG < n ? b + SEG : n;
    const uintptr_t base = reinterpret_cast<uintptr_t>(buf);
    uint64_t i = b;
    while (i < e) {
        if (((base + i) & 15) == 0 && i + 16 <= e) {
            const uint4 v = *reinterpret_cast<const uint4*>(buf + i);
            const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (nl_in_word(w[k])) {
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if (((w[k] >> (8 * j)) & 255u) == 10u) f(i + 4 * k + j);
                }
            }
            i += 16;
        } else {
            if (buf[i] == 10) f(i);
            ++i;
        }
    }
}

__global__ void nl_count_kernel(const uint8_t* buf, uint64_t n, uint64_t n_seg, uint32_t* counts) {
    const uint64_t s = static_cast<uint64_t>(blockIdx.x) * THREADS + threadIdx.x;
    if (s >= n_seg) return;
    uint32_t c = 0;
    for_each_newline(buf, n, s, [&](uint64_t) { ++c; });
    counts[s] = c;
}

__global__ void nl_write_kernel(const uint8_t* buf, uint64_t n, uint64_t n_seg, const uint32_t* seg_base,
                                uint32_t* nl) {
    const uint64_t s = static_cast<uint64_t>(blockIdx.x) * THREADS + threadIdx.x;
    if (s >= n_seg) return;
    uint32_t k = seg_base[s];
    for_each_newline(buf, n, s, [&](uint64_t i) { nl[k++] = static_cast<uint32_t>(i); });
}

// st[0] lines, [1] records, [2] bytes consumed, [3] error (0, or 1/2/3 for a
// record missing its SEQ / + / QUAL line), [4] newlines, [5] max SEQ length
__global__ void fq_lines_kernel(const uint8_t* buf, uint64_t n, int at_eof, uint64_t max_records, int rules,
                                const uint32_t* nl, const uint32_t* seg_base, const uint32_t* counts, uint64_t n_seg,
                                unsigned long long* st) {
    const uint64_t n_nl = n_seg ? static_cast<uint64_t>(seg_base[n_seg - 1]) + counts[n_seg - 1] : 0;
    const uint64_t rest = n_nl ? static_cast<uint64_t>(nl[n_nl - 1]) + 1 : 0;
    uint64_t lines = n_nl;
    if (at_eof && rest < n) {
        if (rules == 1) {
            ++lines;  // readline() returns any non-empty rest
        } else {      // the rest counts when not empty after the '\r' strip
            uint64_t e = n;
            if (buf[e - 1] == 13) --e;
            if (e > rest) ++lines;
        }
    }
    // rules 1 at the end of the stream: a header line starts a record, its
    // missing lines read as empty
    const uint64_t whole = (rules == 1 && at_eof) ? (lines + 3) / 4 : lines / 4;
    const uint64_t recs = whole < max_records ? whole : max_records;
    st[0] = lines;
    st[1] = recs;
    // the reference reads one record past the complete ones only while it
    // still wants records
    st[3] = (rules == 0 && at_eof && max_records > whole && (lines & 3)) ? (lines & 3) : 0;
    uint64_t consumed = 0;
    if (recs) {
        const uint64_t last = 4 * recs - 1;  // index of the last QUAL line
        consumed = last < n_nl ? static_cast<uint64_t>(nl[last]) + 1 : n;
    }
    st[2] = consumed;
    st[4] = n_nl;
    st[5] = 0;
}

__global__ void fq_records_kernel(const uint8_t* buf, uint64_t n, uint64_t base, int rules, const uint32_t* nl,
                                  uint64_t n_nl, const unsigned long long* st, FastqRecordsDev out,
                                  unsigned long long* max_len) {
    const uint64_t r = static_cast<uint64_t>(blockIdx.x) * THREADS + threadIdx.x;
    uint32_t seq_len = 0;
    if (r < st[1]) {
        const uint64_t lines = st[0];
        uint64_t s[4], e[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint64_t li = 4 * r + k;
            if (li >= lines) {  // past the end of the stream (rules 1): empty
                s[k] = e[k] = n;
                continue;
            }
            s[k] = li ? static_cast<uint64_t>(nl[li - 1]) + 1 : 0;
            e[k] = li < n_nl ? nl[li] : n;
            if (rules == 1) {
                while (e[k] > s[k] && buf[e[k] - 1] == 13) --e[k];
            } else if (e[k] > s[k] && buf[e[k] - 1] == 13) {
                --e[k];
            }
        }
        uint64_t ns = s[0], ne = e[0];
        if (ne > ns && buf[ns] == 64) ++ns;
        for (uint64_t i = ns; i < ne; ++i) {
            const uint8_t c = buf[i];
            if (c == 32 || c == 47) {
                ne = i;
                break;
            }
        }
        out.name_off[r] = base + ns;
        out.name_len[r] = static_cast<uint32_t>(ne > ns ? ne - ns : 0);
        seq_len = static_cast<uint32_t>(e[1] - s[1]);
        out.seq_off[r] = base + s[1];
        out.seq_len[r] = seq_len;
        out.qual_off[r] = base + s[3];
        out.qual_len[r] = static_cast<uint32_t>(e[3] - s[3]);
    }
    for (int o = 16; o > 0; o >>= 1) seq_len = max(seq_len, __shfl_xor_sync(0xffffffffu, seq_len, o));
    if ((threadIdx.x & 31) == 0 && seq_len) atomicMax(max_len, static_cast<unsigned long long>(seq_len));
}

__global__ void fq_rows_kernel(const uint8_t* arena, const uint64_t* seq_off, const uint32_t* seq_len, uint64_t n_seq,
                               uint32_t max_len, uint8_t* rows, uint32_t* lens) {
    const int lane = threadIdx.x & 31;
    const uint64_t r = (static_cast<uint64_t>(blockIdx.x) * THREADS + threadIdx.x) >> 5;
    if (r >= n_seq) return;
    const uint32_t len = seq_len[r];
    const uint8_t* src = arena + seq_off[r];
    uint8_t* dst = rows + r * max_len;
    for (uint32_t j = lane; j < max_len; j += 32) dst[j] = j < len ? src[j] : 78;
    if (lane == 0 && lens) lens[r] = len;
}

}  // namespace

size_t fastq_scratch_bytes(uint64_t n_bytes) {
    const uint64_t n_seg = (n_bytes + SEG - 1) / SEG;
    size_t t = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, t, static_cast<const uint32_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                  static_cast<int64_t>(n_seg ? n_seg : 1));
    // counts, segment bases, status, scan temp
    return 2 * align256(n_seg * 4) + 256 + align256(t);
}

int fastq_parse_enqueue(const uint8_t* buf, uint64_t n, int at_eof, uint64_t max_records, uint64_t base, int rules,
                        const FastqRecordsDev& out, void* scratch, size_t scratch_bytes,
                        void* (*newline_buffer)(void* user, size_t bytes), void* user, cudaStream_t st,
                        unsigned long long* h_status) {
    const uint64_t n_seg = (n + SEG - 1) / SEG;
    uint8_t* s = static_cast<uint8_t*>(scratch);
    uint32_t* counts = reinterpret_cast<uint32_t*>(s);
    uint32_t* seg_base = reinterpret_cast<uint32_t*>(s + align256(n_seg * 4));
    unsigned long long* status = reinterpret_cast<unsigned long long*>(s + 2 * align256(n_seg * 4));
    void* temp = s + 2 * align256(n_seg * 4) + 256;
    size_t tb = scratch_bytes - (2 * align256(n_seg * 4) + 256);
    int launches = 0;
    uint32_t* nl = nullptr;
    if (n_seg) {
        const unsigned g = static_cast<unsigned>((n_seg + THREADS - 1) / THREADS);
        nl_count_kernel<<<g, THREADS, 0, st>>>(buf, n, n_seg, counts);
        check_launch(cudaGetLastError(), "nl_count_kernel");
        check_launch(cub::DeviceScan::ExclusiveSum(temp, tb, static_cast<const uint32_t*>(counts), seg_base,
                                                   static_cast<int64_t>(n_seg), st),
                     "newline scan");
        launches += 3;
        uint32_t last[2];
        check_launch(cudaMemcpyAsync(&last[0], seg_base + n_seg - 1, 4, cudaMemcpyDeviceToHost, st), "D2H");
        check_launch(cudaMemcpyAsync(&last[1], counts + n_seg - 1, 4, cudaMemcpyDeviceToHost, st), "D2H");
        check_launch(cudaStreamSynchronize(st), "newline count");
        const uint64_t n_nl = static_cast<uint64_t>(last[0]) + last[1];
        nl = static_cast<uint32_t*>(newline_buffer(user, (n_nl ? n_nl : 1) * 4));
        nl_write_kernel<<<g, THREADS, 0, st>>>(buf, n, n_seg, seg_base, nl);
        check_launch(cudaGetLastError(), "nl_write_kernel");
        ++launches;
    }
    fq_lines_kernel<<<1, 1, 0, st>>>(buf, n, at_eof, max_records, rules, nl, seg_base, counts, n_seg, status);
    check_launch(cudaGetLastError(), "fq_lines_kernel");
    ++launches;
    unsigned long long head[6];
    check_launch(cudaMemcpyAsync(head, status, sizeof(head), cudaMemcpyDeviceToHost, st), "D2H parse status");
    check_launch(cudaStreamSynchronize(st), "fastq lines");
    const uint64_t recs = head[1];
    if (recs) {
        const unsigned g = static_cast<unsigned>((recs + THREADS - 1) / THREADS);
        fq_records_kernel<<<g, THREADS, 0, st>>>(buf, n, base, rules, nl, head[4], status, out, status + 5);
        check_launch(cudaGetLastError(), "fq_records_kernel");
        ++launches;
        check_launch(cudaMemcpyAsync(head + 5, status + 5, 8, cudaMemcpyDeviceToHost, st), "D2H max_len");
        check_launch(cudaStreamSynchronize(st), "fastq records");
    }
    for (int i = 0; i < 6; ++i) h_status[i] = head[i];
    return launches;
}

int fastq_rows_enqueue(const uint8_t* arena, const uint64_t* seq_off, const uint32_t* seq_len, uint64_t n_seq,
                       uint32_t max_len, uint8_t* rows, uint32_t* lens, cudaStream_t st) {
    if (!n_seq) return 0;
    const unsigned g = static_cast<unsigned>((n_seq * 32 + THREADS - 1) / THREADS);
    fq_rows_kernel<<<g, THREADS, 0, st>>>(arena, seq_off, seq_len, n_seq, max_len, rows, lens);
    check_launch(cudaGetLastError(), "fq_rows_kernel");
    return 1;
}

}  // namespace ma
