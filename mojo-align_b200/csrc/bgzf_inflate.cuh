// bgzf_inflate.cuh - inflating the members of a BGZF file on the device, one
// warp per member (bgzf_inflate.cu: lane 0 decodes tokens, the warp writes
// their bytes and folds the CRC-32).  The per-member step below is the host
// form: the same token decoder (inflate.cuh) with the sequential writer, so
// the host tests run the decoder the kernel runs.
#pragma once

#include <cstdint>

#include "inflate.cuh"

namespace ma {
namespace bgzf_inflate {

// Per-member status codes: 0 ok, 1..7 the inflate::Status of the deflate
// data, then:
enum : uint32_t {
    S_SIZE = 8,   // inflated size differs from the member's ISIZE
    S_CRC = 9,    // CRC-32 of the inflated bytes differs from the member's
    S_SPAN = 10,  // the member's compressed or inflated span lies outside its buffer
};

// Members of one compressed buffer: the deflate payload of member m is
// in[src_off[m], src_off[m] + src_len[m]); its ISIZE bytes go to
// out[dst_off[m], ...); crc[m] is its stored CRC-32.
struct Job {
    const uint8_t* in;
    uint64_t in_bytes;
    const uint64_t* src_off;
    const uint32_t* src_len;
    const uint64_t* dst_off;
    const uint32_t* isize;
    const uint32_t* crc;
    uint32_t n;
    uint8_t* out;
    uint64_t out_bytes;
    uint32_t* status;  // [n]
};

// CRC-32 (reflected polynomial 0xEDB88320) table, 256 entries.
MA_HD inline void crc_table(uint32_t* tab, int first, int step) {
    for (int i = first; i < 256; i += step) {
        uint32_t c = static_cast<uint32_t>(i);
        for (int k = 0; k < 8; ++k) c = (c & 1u) ? (c >> 1) ^ 0xEDB88320u : c >> 1;
        tab[i] = c;
    }
}

// Inflates member m and checks its size and CRC-32; returns its status.
MA_HD inline uint32_t inflate_member(const Job& j, uint32_t m, inflate::Tables& t, const uint32_t* crc_tab) {
    const uint64_t so = j.src_off[m], sl = j.src_len[m], dof = j.dst_off[m], isz = j.isize[m];
    if (so > j.in_bytes || sl > j.in_bytes - so || dof > j.out_bytes || isz > j.out_bytes - dof) return S_SPAN;
    uint32_t got = 0;
    const int rc = inflate::inflate_raw(j.in + so, static_cast<uint32_t>(sl), j.out + dof, static_cast<uint32_t>(isz),
                                        &got, t);
    if (rc != inflate::OK) return static_cast<uint32_t>(rc);
    if (got != isz) return S_SIZE;
    uint32_t c = 0xffffffffu;
    const uint8_t* p = j.out + dof;
    for (uint32_t i = 0; i < got; ++i) c = (c >> 8) ^ crc_tab[(c ^ p[i]) & 255u];
    return (c ^ 0xffffffffu) == j.crc[m] ? 0u : S_CRC;
}

}  // namespace bgzf_inflate

#ifdef __CUDACC__
// Enqueues the inflate kernel for every member of j on `st` (bgzf_inflate.cu);
// returns the number of launches.
int bgzf_inflate_enqueue(const bgzf_inflate::Job& j, int sm_count, cudaStream_t st);
#endif

}  // namespace ma
