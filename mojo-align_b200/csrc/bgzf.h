// bgzf.h - BGZF compression on the device (bgzf.cu), shared with the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace ma {

// Uncompressed bytes per BGZF member (_MAX_UNCOMPRESSED, bam_emit.py:24).
constexpr uint32_t BGZF_BLOCK = 65280;
// Largest member: 18-byte header, a stored deflate stream (two stored
// blocks: 10 bytes of framing) and the 8-byte trailer.
constexpr uint32_t BGZF_MEMBER_MAX = 18 + 10 + BGZF_BLOCK + 8;
constexpr uint32_t BGZF_EOF_BYTES = 28;

size_t bgzf_scratch_bytes(uint64_t n_bytes, int sm_count);
// Upper bound of the compressed size of n bytes (plus the EOF member).
uint64_t bgzf_bound(uint64_t n_bytes);

// Compresses in[0, n) into BGZF members written back to back at out, then
// the EOF member when append_eof.  level 0: stored deflate blocks with the
// framing zlib gives for one compress + finish call; 1..9: LZ77 + dynamic
// Huffman, the hash-chain depth growing with the level.  Synchronous on
// st; returns the bytes written (0 when they would exceed out_cap, with
// *need set).  *launches receives the number of kernels launched.
uint64_t bgzf_compress(const uint8_t* in, uint64_t n, int level, uint8_t* out, uint64_t out_cap, int append_eof,
                       void* scratch, size_t scratch_bytes, int sm_count, cudaStream_t st, uint64_t* need,
                       int* launches, float* kernel_ms);

}  // namespace ma
