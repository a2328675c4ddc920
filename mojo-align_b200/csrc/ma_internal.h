// ma_internal.h - host-side types shared by the C++ and CUDA sources of
// libmojoalign_b200.  Nothing here crosses the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mojoalign_b200.h"

namespace ma {

// Error carrying an MA_ERR_* code; converted to a status at the C ABI.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }

// One .ann record (bwa bntann1_t): name, annotation, offset and length.
struct Contig {
    std::string name;
    std::string anno;
    uint64_t offset = 0;
    uint32_t len = 0;
    int32_t n_ambs = 0;
};

// A run of ambiguous bases replaced in the pac (bwa bntamb1_t).
struct Hole {
    uint64_t offset = 0;
    uint32_t len = 0;
    char amb = 'N';
};

// A bwa 0.7 FM-index as the reference reads it
// (fq2bam-meth/src/linear_fm_index.mojo:88-175).
struct BwaIndexHost {
    uint64_t primary = 0, seq_len = 0, l_pac = 0;
    uint64_t L2[5] = {0, 0, 0, 0, 0};
    int64_t sa_intv = 32, n_sa = 0;
    std::vector<uint32_t> bwt;  // interleaved words after the 40-byte header
    std::vector<uint64_t> sa;   // sa[1..n_sa-1]: element i = SA[(i+1)*sa_intv]
    std::vector<uint8_t> pac;   // forward text, 4 bases per byte, MSB first
    std::vector<Contig> contigs;
};

// Reads prefix.{bwt,sa,pac,ann} with FmIndex.load's checks.
BwaIndexHost load_bwa_index(const std::string& prefix);

// FASTA records (name = first word of the header, anno = the rest).
struct FastaRecord {
    std::string name;
    std::string anno;
    std::string seq;
};
std::vector<FastaRecord> read_fasta(const std::string& path);

// Suffix array of text[0..n) over {0,1,2,3} with a virtual smallest
// sentinel at n: returns SA[0..n] (SA[0] == n).  n must be < 2^32 - 1.
std::vector<uint32_t> suffix_array_cpu(const uint8_t* text, uint64_t n);

// BWT of a text in the bwa .bwt word layout (after the 40-byte header),
// its primary row and SA samples SA[i * sa_intv], i = 1 .. n_sa - 1.
struct BwtBuild {
    uint64_t primary = 0;
    std::vector<uint32_t> bwt;
    std::vector<uint64_t> samples;
};
// Built on GPU `device` from the text packed 32 symbols per word, least
// significant first, zero past n, with at least two words after the last
// symbol's word.  batch_limit caps the suffixes sorted at once (0 = what
// fits the device).
BwtBuild bwt_build_gpu(const std::vector<uint64_t>& text_words, uint64_t n, int sa_intv, uint64_t batch_limit,
                       int device);

// Events around the kernels of each wavefront round (profiling): e[3k]
// before round k's search, e[3k+1] before its eval, e[3k+2] before its
// finalize, e[3R] after the last round (rounds past MAX_ROUNDS untimed),
// and around the stage-2 launch after the rounds.
struct WaveTimer {
    static constexpr int MAX_ROUNDS = 64;
    cudaEvent_t e[3 * MAX_ROUNDS + 1] = {};
    cudaEvent_t s2[2] = {};  // around the stage-2 warps of the reads left over
    int recorded = 0;  // rounds timed in the last call
    bool complete = true;
};

void build_index(const std::string& fasta, const std::string& out_prefix, bool bwameth_c2t,
                 int sa_intv, int device, uint64_t batch_limit = 0);

}  // namespace ma
