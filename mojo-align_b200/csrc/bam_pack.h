// bam_pack.h - device-side BAM record packing of one mapped batch
// (bam_pack.cu), shared with the C ABI in capi.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace ma {

// Every pointer is a device pointer.  Inputs follow _emit_bam_from_batch
// (fq2bam-meth/src/linear_gpu_fm.mojo:669-984): the seven mapping outputs
// [n_seq] (R1 rows then R2 rows), the FASTQ arena spans of every record,
// the rid -> tid table and the RG id.  Metadata arrays are the tile's,
// written at [n_reads, n_reads + n_seq) - meta_origin.
struct BamDev {
    const int32_t* rid;
    const uint32_t* pos;
    const uint32_t* mapq;
    const int32_t* flag;
    const uint32_t* sl;
    const uint32_t* sr;
    const uint32_t* nm;
    const uint8_t* arena;
    uint64_t arena_bytes;
    const uint64_t* name_off;
    const uint64_t* orig_off;
    const uint64_t* qual_off;  // nullptr: no qualities
    const uint32_t* name_len;
    const uint32_t* orig_len;
    const uint32_t* qual_len;
    const int32_t* rid_to_tid;
    int32_t n_tid;
    const uint8_t* rg;
    uint32_t rg_n;
    uint32_t n1;
    int paired;
    uint64_t n_reads, n_total;
    uint64_t meta_origin;  // tile index of element 0 of the metadata arrays
    uint32_t chunk;
    uint8_t* bam;
    uint64_t cap;
    uint64_t *coord, *dhi, *dlo, *rec;
    uint32_t *len, *score, *pair;
    // [0] total record bytes of the batch, [1] mapped records, [2] records
    // whose arena spans fall outside the arena (written with zero bytes in
    // their place).  Records are written only when [0] <= cap.
    unsigned long long* status;
};

// Device scratch for a batch of n_rec records.
size_t bam_scratch_bytes(uint64_t n_rec);

// Enqueues the metadata pass and the scan on `st`; record i's end offset
// lands in the scratch, the batch total in status[0] after the pack pass.
// Returns the number of kernels launched.
int enqueue_bam_layout(const BamDev& b, void* scratch, size_t scratch_bytes, cudaStream_t st);
// Enqueues the record pass (after enqueue_bam_layout on the same scratch).
int enqueue_bam_records(const BamDev& b, const void* scratch, int sm_count, cudaStream_t st);
// Device address of the batch total inside the scratch.
const uint64_t* bam_total_in_scratch(const void* scratch, uint64_t n_rec);

}  // namespace ma
