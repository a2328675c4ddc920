// Test harness (test infrastructure only): the device inflate decoder of
// mojo-align_b200/csrc/inflate.cuh compiled as host code, for checking it
// against zlib on the CPU.
#include <cstdint>

#include "inflate.cuh"

extern "C" int harness_inflate(const uint8_t* in, uint32_t n, uint8_t* out, uint32_t cap, uint32_t* out_len) {
    ma::inflate::Tables t;
    return ma::inflate::inflate_raw(in, n, out, cap, out_len, t);
}
