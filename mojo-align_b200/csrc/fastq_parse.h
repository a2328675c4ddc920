// fastq_parse.h - FASTQ record split and row packing on the device
// (fastq_parse.cu), shared with the C ABI in capi.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace ma {

// Device arrays of one entry per record.
struct FastqRecordsDev {
    uint64_t* name_off;
    uint32_t* name_len;
    uint64_t* seq_off;
    uint32_t* seq_len;
    uint64_t* qual_off;
    uint32_t* qual_len;
};

size_t fastq_scratch_bytes(uint64_t n_bytes);

// Splits buf[0, n) into records (synchronous on st) under `rules`: 0 the
// BAM path's reader (linear_fastq.mojo), 1 the SAM path's (fastq_batch.py).  newline_buffer(user,
// bytes) supplies the device array of newline positions once their count is
// known.  h_status: [0] lines, [1] records, [2] bytes consumed, [3] error (0,
// or 1/2/3: a record missing its SEQ / + / QUAL line), [4] newlines, [5] the
// longest SEQ.  Returns the number of kernels launched.
int fastq_parse_enqueue(const uint8_t* buf, uint64_t n, int at_eof, uint64_t max_records, uint64_t base, int rules,
                        const FastqRecordsDev& out, void* scratch, size_t scratch_bytes,
                        void* (*newline_buffer)(void* user, size_t bytes), void* user, cudaStream_t st,
                        unsigned long long* h_status);

// Padded rows [n_seq][max_len] of the SEQ spans ('N' fill) and their lengths.
int fastq_rows_enqueue(const uint8_t* arena, const uint64_t* seq_off, const uint32_t* seq_len, uint64_t n_seq,
                       uint32_t max_len, uint8_t* rows, uint32_t* lens, cudaStream_t st);

}  // namespace ma
