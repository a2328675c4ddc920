// sort_markdup.h - coordinate sort, duplicate marking and the sorted record
// gather of a BAM tile on the device (sort_markdup.cu), shared with the
// C ABI in capi.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace ma {

// Device pointers; arrays of n entries in tile (record) order.
struct SortDev {
    uint64_t n;
    const uint64_t* coord;
    const uint64_t* dhi;
    const uint64_t* dlo;
    const uint32_t* score;
    const uint32_t* pair;
    uint32_t* is_dup;    // out, record order
    uint32_t* perm;      // out, coordinate order
    uint32_t* dup_perm;  // out (may be null), duplicate-key order
    int do_markdup;
    unsigned long long* marked;  // out (may be null): records marked
};

size_t sort_scratch_bytes(uint64_t n);
// Returns the number of kernels launched (CUB's included).
int enqueue_sort_markdup(const SortDev& s, void* scratch, size_t scratch_bytes, cudaStream_t st);

// The records of a tile in perm order, flag 0x400 set on duplicates.
struct GatherDev {
    uint64_t n;
    const uint32_t* perm;
    const uint64_t* rec;  // chunk << 32 | byte offset
    const uint32_t* len;
    const uint32_t* is_dup;  // may be null when !apply_dup
    int apply_dup;
    const uint8_t* const* chunks;  // device array of chunk base pointers
    const uint64_t* chunk_len;     // device array of chunk sizes
    uint32_t n_chunks;
    uint8_t* out;
    uint64_t cap;
    // [0] bytes of the sorted stream, [1] records whose index, chunk or span
    // is out of range (written as zero bytes).  Records are written only
    // when [0] <= cap.
    unsigned long long* status;
};

size_t gather_scratch_bytes(uint64_t n);
int enqueue_gather_layout(const GatherDev& g, void* scratch, size_t scratch_bytes, cudaStream_t st);
int enqueue_gather_records(const GatherDev& g, const void* scratch, int sm_count, cudaStream_t st);
const uint64_t* gather_total_in_scratch(const void* scratch, uint64_t n);

}  // namespace ma
