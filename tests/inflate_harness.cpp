// Test harness (test infrastructure only): the device inflate decoder of
// mojo-align_b200/csrc/inflate.cuh compiled as host code, for checking it
// against zlib on the CPU.
#include <cstdint>

#include "inflate.cuh"

extern "C" int harness_inflate(const uint8_t* in, uint32_t n, uint8_t* out, uint32_t cap, uint32_t* out_len) {
    ma::inflate::Tables t;
    return ma::inflate::inflate_raw(in, n, out, cap, out_len, t);
}

#include "bgzf_inflate.cuh"

// The per-member step of the device kernel (bgzf_inflate_kernel), run on the
// host over every member.
extern "C" void harness_inflate_members(const uint8_t* in, uint64_t in_bytes, const uint64_t* src_off,
                                        const uint32_t* src_len, const uint64_t* dst_off, const uint32_t* isize,
                                        const uint32_t* crc, uint32_t n, uint8_t* out, uint64_t out_bytes,
                                        uint32_t* status) {
    ma::bgzf_inflate::Job j{in, in_bytes, src_off, src_len, dst_off, isize, crc, n, out, out_bytes, status};
    uint32_t tab[256];
    ma::bgzf_inflate::crc_table(tab, 0, 1);
    ma::inflate::Tables t;
    for (uint32_t m = 0; m < n; ++m) status[m] = ma::bgzf_inflate::inflate_member(j, m, t, tab);
}
