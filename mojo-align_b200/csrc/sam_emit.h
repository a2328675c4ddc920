// sam_emit.h - device-side SAM text of one mapped batch (sam_emit.cu),
// shared with the C ABI in capi.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace ma {

// Every pointer is a device pointer.  Inputs follow the SAM loop of
// map_fastq_fm_gpu (fq2bam-meth/src/linear_gpu_fm.mojo:2787-2836): the
// mapping outputs [n_seq] (R1 rows then R2 rows), the arena spans of every
// record (name, original bases, qualities), the canonical contig table and
// the RG id.
struct SamDev {
    const int32_t* rid;
    const uint32_t* pos;
    const uint32_t* mapq;
    const int32_t* flag;
    const uint32_t* sl;
    const uint32_t* sr;
    const uint8_t* arena;
    uint64_t arena_bytes;
    const uint64_t* name_off;
    const uint32_t* name_len;
    const uint64_t* seq_off;
    const uint32_t* seq_len;
    const uint64_t* qual_off;
    const uint32_t* qual_len;
    const uint8_t* names;  // canonical contig names
    uint64_t names_bytes;
    const uint64_t* cname_off;  // [n_contigs]
    const uint32_t* cname_len;
    const uint32_t* canon;
    uint32_t n_contigs;
    const uint8_t* rg;
    uint32_t rg_n;
    uint32_t n1;
    int paired;
    uint8_t* sam;
    uint64_t cap;
    // [0] text bytes of the batch, [1] mapped records, [2] error bits:
    // 1 text larger than cap, 2 SEQ/QUAL not valid UTF-8, 4 rid outside the
    // contig table, 8 an arena or contig-name span out of range.  Text is
    // written only when [2] == 0.
    unsigned long long* status;
};

// Device scratch for a batch of n_lines lines.
size_t sam_scratch_bytes(uint64_t n_lines);

// Enqueues the layout pass, the scan and the write pass on `st` (status
// must be zeroed before).  Returns the number of kernels launched.
int enqueue_sam(const SamDev& d, void* scratch, size_t scratch_bytes, int sm_count, cudaStream_t st);

}  // namespace ma
