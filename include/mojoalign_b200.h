/*
 * mojoalign_b200.h - C ABI of the B200 linear bisulfite seed-and-extend path.
 *
 * This library replaces the FM engine of the mojo-align linear mapper
 * (align.linear.mojo, the bwa-meth method class).  Every entry point below
 * names the reference interface it stands in for.  Reference paths are
 * relative to the mojo-align source tree.
 *
 * Conventions
 *   - Every call returns MA_OK (0) or a negative MA_ERR_* code.  No C++
 *     exception crosses this boundary.  ma_last_error() returns the message
 *     of the last failing call made on a context (thread-local for calls
 *     that take no context).
 *   - One ma_ctx per host thread.  The caller owns every host buffer; the
 *     library owns device buffers it allocates.
 *   - Host pointers are plain pageable or pinned memory.  "_device" entry
 *     points take device pointers and a cudaStream_t passed as void*.
 *   - The CUDA kernels are the only compute path: with no usable sm_100
 *     device every mapping call fails with MA_ERR_CUDA.
 */
#ifndef MOJOALIGN_B200_H
#define MOJOALIGN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define MA_OK 0
#define MA_ERR_ARG -1         /* invalid argument / size                    */
#define MA_ERR_IO -2          /* file missing or unreadable                 */
#define MA_ERR_FORMAT -3      /* malformed bwa index / FASTA / FASTQ        */
#define MA_ERR_CUDA -4        /* CUDA runtime failure or no device          */
#define MA_ERR_NOMEM -5       /* HBM admission budget exceeded / OOM        */
#define MA_ERR_UNSUPPORTED -6 /* input outside what this build handles      */
#define MA_ERR_TIMEOUT -7     /* a bounded device wait ran out              */
#define MA_ERR_INTERNAL -8    /* device-side consistency check failed       */

/* bisulfite conversion modes, fq2bam-meth/src/linear_fastq.mojo:29-34 */
#define MA_BS_NONE 0
#define MA_BS_C2T 1
#define MA_BS_G2A 2

typedef struct ma_ctx ma_ctx;
typedef struct ma_index ma_index;

/*
 * Mapping parameters.  Field names and defaults follow the env knobs read at
 * fq2bam-meth/src/linear_gpu_fm.mojo:2074-2082 (METHYLGRAPHER_FM_*).
 */
typedef struct ma_params {
    int32_t seed_len;    /* METHYLGRAPHER_FM_SEED_LEN     default 18   */
    int32_t seed_stride; /* METHYLGRAPHER_FM_SEED_STRIDE  default 2    */
    int32_t max_occ;     /* METHYLGRAPHER_FM_MAX_OCC      default 4096 */
    int32_t max_diff;    /* METHYLGRAPHER_FM_MAX_DIFF     default 12   */
    int32_t max_soft;    /* METHYLGRAPHER_FM_MAX_SOFT     default 20   */
    int32_t max_adj;     /* METHYLGRAPHER_FM_ADJ          default 8    */
    int32_t rescue_win;  /* METHYLGRAPHER_FM_RESCUE_WIN   default 512  */
} ma_params;

/* Fills the reference defaults (linear_gpu_fm.mojo:2074-2082). */
void ma_params_default(ma_params* p);

/*
 * Per-read outputs, structure of arrays, each [n_seq] (R1 rows then R2 rows).
 * Same fields and meaning as the seven output buffers of
 * fm_seed_extend_kernel (linear_gpu_fm.mojo:1183-1189): rid is the index of
 * the f<name>/r<name> contig of the .ann (-1 unmapped), pos is 0-based and
 * contig-local, flag is 4 (unmapped) or 16*is_rev, sl/sr soft clips.
 */
typedef struct ma_hits {
    int32_t* rid;
    uint32_t* pos;
    uint32_t* mapq;
    int32_t* flag;
    uint32_t* sl;
    uint32_t* sr;
    uint32_t* nm;
} ma_hits;

/*
 * Optional side outputs (not emitted by the reference kernel, which keeps
 * them in locals at linear_gpu_fm.mojo:1238-1240,1369-1385).  For the
 * candidate that won the best-hit selection: the SA interval [uk, ul], its
 * left read offset us and its right endpoint e; us = e = -1 when the seed
 * kernel chose no hit.  score = (qlen - sl - sr) - 5*nm for a mapped read
 * (match +1 / mismatch -4 over the aligned part), 0 for an unmapped one.
 * Any pointer may be NULL.
 */
typedef struct ma_debug {
    uint64_t* uk;
    uint64_t* ul;
    int32_t* us;
    int32_t* e;
    int32_t* score;
} ma_debug;

typedef struct ma_index_info {
    uint64_t seq_len;      /* BWT length 2*l_pac (linear_fm_index.mojo:126) */
    uint64_t l_pac;        /* forward pac length (.ann line 1)               */
    uint64_t primary;      /* BWT row of the whole text                      */
    uint64_t L2[5];        /* cumulative symbol counts                       */
    int64_t sa_intv;       /* SA sampling interval of the .sa file           */
    int64_t n_sa;          /* (seq_len + sa_intv) / sa_intv                  */
    int64_t n_contigs;     /* .ann records (f<name> and r<name>)             */
    uint64_t sa_reject_below; /* text positions below this are rejected by
                                 the reference's sampled-SA walk (it reaches
                                 the first text row unsampled) */
    int32_t kmer_k;        /* k of the resident k-mer interval table         */
    int32_t kmer3_k;       /* k of the converted-alphabet k-mer tables       */
    uint64_t device_bytes; /* HBM held by this index                         */
} ma_index_info;

/*
 * Resident-index options (all result-neutral).
 *   kmer_k    k-mer interval table over A/C/G/T, 4^k entries of 8 bytes
 *             (0 = none, 1..14; default 12).
 *   kmer3_k   interval tables over the converted-read alphabets A/G/T
 *             (C->T reads) and A/C/T (G->A reads), 2 * 3^k entries of 8
 *             bytes (0 = none, 1..20; default 0).  k = seed_len replaces
 *             the first seed_len backward-search steps with one lookup.
 *   hbm_budget_bytes  admission budget (0 = all free HBM).
 *   wide_rows 1: store SA rows as 40-bit values even when the text is
 *             short enough for 32-bit rows (automatic from 2^32 - 1 rows).
 *   occ_super_shift   log2 of the Occ superblock (7..31; 0 = 31): Occ
 *             lines count symbols from the start of their superblock.
 *   prep_chunk_rows   SA rows per preparation pass of the k-mer tables and
 *             the seed summary (0 = 2^30; at least 512).
 *   at_k, at_seed_len   A/T window outcome table: for every read window of
 *             at_k bases that holds only A and T (2^at_k windows, 16 bytes
 *             each; 0 = none, else at_seed_len..30), the whole outcome of
 *             the backward search over it for seed length at_seed_len (the
 *             seed it returns, none, or the interval it continues from).
 *             Reads from the strand the conversion does not match are
 *             nearly all A/T after conversion, and their searches step back
 *             several bases past the k-mer tables; a search whose last
 *             at_k bases are A/T starts from this one lookup instead.  Used
 *             only by calls whose seed_len equals at_seed_len.
 * A table is used by a mapping call only when its k <= seed_len.  Texts of
 * up to 2^35 - 2 symbols (seq_len) are supported.
 */
typedef struct ma_index_options {
    int32_t kmer_k;
    int32_t kmer3_k;
    uint64_t hbm_budget_bytes;
    int32_t wide_rows;
    int32_t occ_super_shift;
    uint64_t prep_chunk_rows;
    int32_t at_k;
    int32_t at_seed_len;
} ma_index_options;
void ma_index_options_default(ma_index_options* o);

/* ---- context ------------------------------------------------------- */

/* Opens a CUDA context on device `device_ordinal` (select_device,
 * gpu-common/src/gpu_device.mojo:19-64; DeviceContext(api),
 * linear_gpu_fm.mojo:2014).  Fails with MA_ERR_CUDA without an sm_100 GPU. */
int ma_ctx_create(int device_ordinal, ma_ctx** out);
void ma_ctx_destroy(ma_ctx* ctx);
const char* ma_last_error(const ma_ctx* ctx);
/* Free / total HBM of the context's device (replaces the nvidia-smi probe
 * hbm_info, gpu-common/python/gpu_mem.py:28-57). */
int ma_hbm_info(ma_ctx* ctx, uint64_t* free_bytes, uint64_t* total_bytes);

/* ---- index --------------------------------------------------------- */

/*
 * Builds a bwa-0.7-format FM-index (.bwt/.sa/.pac/.ann/.amb) of `fasta`.
 * bwameth_c2t != 0 first writes the bwa-meth dual-strand text (r<name> =
 * G->A, f<name> = C->T) as `out_prefix` itself (fq2bam_meth.py:91-93) and
 * indexes that, replacing `bwameth.py index` + `bwa index`
 * (fq2bam-meth/scripts/ensure_bwameth_index.sh:23-50).  sa_intv is the SA
 * sampling interval written to .sa (bwa default 32).  device_ordinal >= 0
 * builds the BWT on that GPU (texts up to 2^35 - 2 symbols, e.g. the
 * 12.4 G-symbol text of a 3.1 Gbp genome); -1 sorts on the host (texts
 * below 2^32 symbols).
 */
int ma_index_build(const char* fasta, const char* out_prefix, int bwameth_c2t,
                   int sa_intv, int device_ordinal);

/*
 * ma_index_build with the GPU construction's batch size: at most
 * batch_suffixes suffixes are sorted at once (0 = what fits the device);
 * the files do not depend on it.  No counterpart in the reference.
 */
int ma_index_build_batched(const char* fasta, const char* out_prefix,
                           int bwameth_c2t, int sa_intv, int device_ordinal,
                           uint64_t batch_suffixes);

/*
 * Loads prefix.{bwt,sa,pac,ann} with the header checks of
 * FmIndex.load (fq2bam-meth/src/linear_fm_index.mojo:88-175) and makes the
 * index resident in HBM (upload at linear_gpu_fm.mojo:2034-2069) in this
 * library's own layout.  The HBM preflight (_require_hbm,
 * linear_gpu_locate.mojo:211-214; gpu_mem.require_index_capacity) becomes a
 * cudaMemGetInfo check of the resident bytes plus staging against
 * opt->hbm_budget_bytes, failing with MA_ERR_NOMEM.  opt may be NULL.
 */
int ma_index_open(ma_ctx* ctx, const char* prefix, const ma_index_options* opt,
                  ma_index** out);
void ma_index_close(ma_index* idx);
/* Host-only preflight of prefix.{bwt,sa,pac,ann}: the checks of
 * FmIndex.load (linear_fm_index.mojo:88-175) without a GPU; device_bytes
 * reports the HBM ma_index_open would need (resident + staging) with these
 * k-mer tables and no A/T window outcome table (that table adds
 * 2^at_k * 16 bytes). */
int ma_index_probe(const char* prefix, int kmer_k, int kmer3_k, ma_index_info* out);
int ma_index_get_info(const ma_index* idx, ma_index_info* out);
/* Contig record i of the .ann (FmIndex.contig_name/offset/length,
 * linear_fm_index.mojo:337-347).  *name stays valid until ma_index_close. */
int ma_index_contig(const ma_index* idx, int64_t i, const char** name,
                    uint64_t* offset, uint64_t* length);

/* ---- mapping ------------------------------------------------------- */

/*
 * One batch through the plain single-launch form, synchronous.  Replaces
 * _fm_fire_batch (linear_gpu_fm.mojo:2279-2417): H2D of bases and lengths,
 * then on-device conversion + 2-bit pack (pack_bases_kernel L1136-1154 and
 * _cvt, linear_fastq.mojo:37-46), the seed/extend kernel
 * (fm_seed_extend_kernel L1156-1837), the mate rescue kernel when paired
 * (fm_mate_rescue_kernel L1839-2011), D2H of the outputs.
 *
 *   bases   ASCII, row-major [n_seq][max_len]; R1 rows 0..n1-1, then R2
 *           rows n1..2*n1-1 when paired (fq_pack_bases layout,
 *           linear_fastq.mojo:454-492).  Bytes past a read's length are
 *           ignored.
 *   lens    [n_seq] read lengths, each <= max_len <= 1024.
 *   bs_r1 / bs_r2   MA_BS_* conversion applied on the device to R1 / R2.
 *   out     host arrays [n_seq]; dbg may be NULL.
 */
int ma_map_batch(ma_ctx* ctx, const ma_index* idx, const uint8_t* bases,
                 const uint32_t* lens, uint32_t n1, int paired,
                 uint32_t max_len, int bs_r1, int bs_r2, const ma_params* p,
                 ma_hits* out, ma_debug* dbg);

/*
 * Same computation on device-resident buffers, asynchronous on `stream`
 * (a cudaStream_t, NULL = the context's stream).  Scratch comes from the
 * context's pool, sized on first use for (n_seq, max_len).
 */
int ma_map_batch_device(ma_ctx* ctx, const ma_index* idx,
                        const uint8_t* d_bases, const uint32_t* d_lens,
                        uint32_t n1, int paired, uint32_t max_len, int bs_r1,
                        int bs_r2, const ma_params* p, ma_hits* d_out,
                        ma_debug* d_dbg, void* stream);

/*
 * Same computation as ma_map_batch_device, with no device allocation.  No
 * counterpart in the reference (its batch step allocates through its
 * DeviceContext).  For callers that must not let the library call
 * cudaMalloc: a framework whose caching allocator already holds the free
 * HBM, or a latency-bound serving loop sharing the GPU with other streams,
 * where cudaMalloc's implicit device synchronisation would stall them.
 * Inputs and outputs stay the caller's device buffers; scratch comes from
 * one fixed file-scope device array of about 11 MiB.  Limits: at most 32768
 * reads per call (16384 pairs) of at most 256 bases; larger calls fail with
 * MA_ERR_ARG.  Set-up: the first call on a device looks up the array's
 * device address and loads the kernels it runs; under CUDA's default lazy
 * module loading that is also when the array itself is placed on the
 * device (with CUDA_MODULE_LOADING=EAGER, when the library loads), so the
 * set-up can take device memory, as can a kernel's first launch (the driver
 * sizes its local memory then).  A call with n1 = 0 does the set-up and
 * launches every kernel of a call over zero reads: make it before a caching
 * allocator reserves the free HBM, and before any stream capture.  The array then stays on the device until
 * the process exits.  Calls share the array: calls whose kernels overlap on
 * the GPU race.  Synchronous: the call waits for `stream` (a cudaStream_t,
 * NULL = the legacy default stream) to read the device error word back.
 * The caller's current device is restored on return.  Errors are reported
 * by ma_last_error(NULL).
 */
int ma_map_batch_device_noalloc(const ma_index* idx, const uint8_t* d_bases,
                                const uint32_t* d_lens, uint32_t n1,
                                int paired, uint32_t max_len, int bs_r1,
                                int bs_r2, const ma_params* p, ma_hits* d_out,
                                ma_debug* d_dbg, void* stream);

/* Number of kernel launches the last mapping call on ctx issued. */
int ma_last_launch_count(const ma_ctx* ctx);

/*
 * Result-neutral execution choices (every setting gives identical outputs).
 *   seed_kernel           0: one thread per read over all right endpoints
 *                         (the reference's launch shape, L2336-2382);
 *                         1: two stages: one thread per read over
 *                         the first stage1_endpoints endpoints, then one
 *                         warp per remaining read in a persistent kernel
 *                         fed by a work queue;
 *                         2: wavefront: rounds of batch-wide passes (one
 *                         thread per read and endpoint, then one per
 *                         candidate locus and shift), stage1_endpoints
 *                         endpoints in the first round and wave_endpoints in
 *                         each later one; reads left over go to the stage-2
 *                         warps (default);
 *                         3: the wavefront with lane refill in its search
 *                         pass: each lane steps its own endpoint and takes
 *                         a new one when its search ends, so lanes do not
 *                         wait for the longest search of their warp, and
 *                         staged shifts in its eval pass: the live shifts
 *                         of a warp's loci are gathered in shared memory
 *                         and evaluated 32 at a time, every lane busy;
 *                         4: the wavefront with the search pass of 2 and
 *                         the staged eval pass of 3.
 *   stage1_endpoints      endpoints stage 1 (or the first round) covers
 *                         (default 1).
 *   stage2_blocks_per_sm  persistent blocks per SM for stage 2 (0 = the
 *                         occupancy maximum).
 *   reg_level             register budget of the seed kernels: 0 = the
 *                         compiler's choice, 1 = 80 registers, 2 = 64
 *                         registers (stage kernels); for the wavefront's
 *                         search / eval kernels 0 = the compiler's choice,
 *                         1 = 5 / 4 blocks of 256 threads per SM, 2 = 6 / 5,
 *                         and for the lane-refill search 1 = 4, 2 = 5
 *                         (default 2).
 *   stage1_max_rows       stage 1 hands a read to stage 2 as soon as one of
 *                         its seeds has more SA rows than this (1..16,
 *                         default 1; 16 = never).
 *   stage2_first_wave     right endpoints stage 2 searches in its first
 *                         group for a read (1..32, default 1); later groups
 *                         take 32.
 *   wave_endpoints        right endpoints per read in each wavefront round
 *                         after the first (1..256, default 8).
 *   wave_loci_per_read    wavefront locus list capacity per read of the
 *                         batch (1..64, default 4; at least 1024 entries);
 *                         reads whose loci do not fit a round are finished
 *                         by the stage-2 warps.
 *   wave_max_rounds       wavefront rounds before the reads still active
 *                         go to the stage-2 warps (0 = as many as the
 *                         longest read needs, default).
 *   wave_growth           1: each wavefront round after the second covers
 *                         twice the endpoints of the one before (fewer,
 *                         fuller rounds for the reads that stay active
 *                         longest; default); 0: every later round covers
 *                         wave_endpoints.
 */
typedef struct ma_tuning {
    int32_t seed_kernel;
    int32_t stage1_endpoints;
    int32_t stage2_blocks_per_sm;
    int32_t reg_level;
    int32_t stage1_max_rows;
    int32_t stage2_first_wave;
    int32_t wave_endpoints;
    int32_t wave_loci_per_read;
    int32_t wave_max_rounds;
    int32_t wave_growth;
} ma_tuning;
int ma_ctx_set_tuning(ma_ctx* ctx, const ma_tuning* t);
int ma_ctx_get_tuning(const ma_ctx* ctx, ma_tuning* t);

/*
 * enable != 0: ma_map_batch_device replays a CUDA graph of its launch
 * sequence while its arguments (buffers, sizes, parameters, stream, tuning)
 * repeat: the first call with new arguments runs as usual, the second
 * captures the sequence into a graph and launches it, later ones launch the
 * graph (one host launch per call).  Result-neutral; off while profiling.
 * No counterpart in the reference.
 */
int ma_ctx_set_graphs(ma_ctx* ctx, int enable);

/*
 * Chunking of ma_map_batch's copy / compute pipeline (result-neutral; no
 * reference counterpart: _fm_fire_batch runs fixed 16384-pair batches two
 * deep, linear_gpu_fm.mojo:2438-3094).  Chunk k+1 is copied in and chunk k-1
 * copied out while chunk k computes.  Host arrays that are not page-locked
 * (lengths, outputs) are staged through page-locked buffers of the context,
 * so that their copies do not hold the calling thread; page-locked reads
 * (bases) let their copies overlap the kernels as well.
 *   first_chunk_pairs  pairs of the first chunk (0 = max(65536, n1 / 64))
 *   growth_percent     each chunk is this much larger than the one before
 *                      (default 50)
 *   max_chunk_pairs    chunk size cap (0 = min(2000000, max(131072, n1 / 16)))
 *   compute_streams    1: chunks compute in turn on the context's stream;
 *                      2 or 3 (default): consecutive chunks compute on that
 *                      many streams with their own work buffers, so one
 *                      chunk's last kernels overlap the next one's first.
 */
typedef struct ma_pipeline {
    uint32_t first_chunk_pairs;
    uint32_t growth_percent;
    uint32_t max_chunk_pairs;
    uint32_t compute_streams;
} ma_pipeline;
int ma_ctx_set_pipeline(ma_ctx* ctx, const ma_pipeline* p);
int ma_ctx_get_pipeline(const ma_ctx* ctx, ma_pipeline* p);

/* ---- served form: a request loop over a resident index ----------------
 *
 * No counterpart in the reference, whose map_fastq_fm_gpu maps one FASTQ
 * stream in fixed 16384-pair batches (linear_gpu_fm.mojo:2074, 2438-3094).
 * A server keeps one resident index and maps requests (read batches of any
 * size, from any number of samples) submitted from any host thread:
 *   - admission: the server reserves hbm_budget_bytes of device memory
 *     once and carves every launch group's buffers out of it; a group is
 *     issued only when its buffers fit in what is free, so the work in
 *     flight never exceeds the budget;
 *   - continuous batching: one launch group takes the pending work of
 *     several requests (in arrival order, up to max_group_pairs pairs;
 *     requests with the same `paired` and parameters merge; lengths and
 *     bisulfite modes may differ) and a large request is split over
 *     several groups, so requests that arrive while others are on the GPU
 *     join the next group as memory frees;
 *   - overlap: up to max_inflight groups are in flight on their own
 *     streams, so one group's copies and kernels overlap another's.
 * Every read's outputs are those ma_map_batch gives for it alone.  The
 * caller's host buffers (reads and ma_hits arrays) must stay valid and
 * unmodified until the request completes.  Requests complete in any
 * order; latency is measured from submit to completion on the host clock.
 */
typedef struct ma_server ma_server;

/* MA_SERVE_SCHEDULER_TEST: no device work at all; each launch group's
 * "mapping" is a host function of the packed reads (rid = read length,
 * pos = FNV-1a hash of the converted read, nm = the mate's hash, mapq =
 * seed_len, flag = 128 for second mates, sl/sr = 0).  It is not an
 * aligner: it exercises admission, grouping and result scatter without a
 * GPU. */
#define MA_SERVE_SCHEDULER_TEST 1

typedef struct ma_serve_options {
    uint64_t hbm_budget_bytes; /* 0 = min(free HBM / 4, 16 GiB)             */
    uint32_t max_group_pairs;  /* pairs (or SE reads) per launch group,
                                  default 262144                            */
    uint32_t max_inflight;     /* launch groups in flight, default 3        */
    uint32_t flags;            /* MA_SERVE_* bits                           */
} ma_serve_options;

typedef struct ma_serve_stats {
    uint64_t requests_submitted, requests_completed, requests_failed;
    uint64_t reads_completed;   /* each mate counts as one read             */
    uint64_t groups_issued, parts_issued; /* parts: request pieces in groups */
    uint64_t max_requests_in_group;
    uint64_t max_groups_in_flight;
    uint64_t budget_bytes, peak_bytes; /* reserved budget, peak in use     */
    uint64_t admission_waits;   /* times a group waited for memory         */
} ma_serve_stats;

void ma_serve_options_default(ma_serve_options* o);
/* ctx supplies the device and the kernel tuning (copied); idx must stay open
 * until the server is destroyed.  With MA_SERVE_SCHEDULER_TEST, ctx and idx
 * may be NULL. */
int ma_serve_create(ma_ctx* ctx, const ma_index* idx,
                    const ma_serve_options* opt, ma_server** out);
/* Queues a request (the ma_map_batch arguments, host buffers) and returns
 * at once with its id.  Fails with MA_ERR_ARG on bad arguments and
 * MA_ERR_NOMEM when one pair of the request cannot fit the budget. */
int ma_serve_submit(ma_server* s, const uint8_t* bases, const uint32_t* lens,
                    uint32_t n1, int paired, uint32_t max_len, int bs_r1,
                    int bs_r2, const ma_params* p, const ma_hits* out,
                    uint64_t* request_id);
/* *done = 1 once the request has completed; returns its status then. */
int ma_serve_poll(ma_server* s, uint64_t request_id, int* done);
/* Waits for one request (timeout_ms < 0: no limit); MA_ERR_TIMEOUT when
 * the time runs out first, else the request's status. */
int ma_serve_wait(ma_server* s, uint64_t request_id, int timeout_ms);
/* Waits until every submitted request has completed. */
int ma_serve_drain(ma_server* s, int timeout_ms);
int ma_serve_get_stats(ma_server* s, ma_serve_stats* out);
/* Completed requests in completion order: ids, reads and latency (ms).
 * Copies min(cap, count) entries; *count gets the total. */
int ma_serve_latencies(ma_server* s, uint64_t* ids, uint64_t* reads,
                       double* ms, uint64_t cap, uint64_t* count);
/* Message of the last failure on the server (or of a failed request). */
const char* ma_serve_last_error(const ma_server* s);
/* Drains, stops the worker threads and frees the reserved memory. */
void ma_serve_destroy(ma_server* s);

/* ---- FASTQ records on the device ------------------------------------ */

/* Per-record spans of a parsed FASTQ buffer, arrays of max_records entries:
 * the read name (qname span), the bases and the qualities, as byte offsets
 * (plus `base`) into the buffer.  These are the name / orig / qual columns
 * of ma_fastq_arena with the buffer as the arena. */
typedef struct ma_fastq_records {
    uint64_t* name_off;
    uint32_t* name_len;
    uint64_t* seq_off;
    uint32_t* seq_len;
    uint64_t* qual_off;
    uint32_t* qual_len;
} ma_fastq_records;

/*
 * Splits uncompressed FASTQ bytes into records.  Replaces the record split of
 * fq_read_batch (fq2bam-meth/src/linear_fastq.mojo:437-451) with _store_rec
 * (L365-417), _pipe_line (L233-280: lines end at '\n', one trailing '\r'
 * dropped; at the end of the stream an unterminated rest is a line when it is
 * not empty after that strip) and _qname_span (L308-325: leading '@' dropped,
 * name cut at the first ' ' or '/').  Takes at most max_records records.
 * at_eof == 0: the buffer continues in a later one, so only records whose
 * four lines all end in '\n' are taken.  out3 (host) receives the records
 * taken, the bytes they span (where the next buffer must start) and the
 * longest SEQ.  n_bytes < 2^32.  A record cut short at the end of the stream
 * fails with MA_ERR_FORMAT and the reference's message ("truncated FASTQ
 * (missing SEQ)" / "(missing +)" / "(missing QUAL)").  Host buffers.
 */
int ma_fastq_parse(ma_ctx* ctx, const uint8_t* buf, uint64_t n_bytes, int at_eof,
                   uint32_t max_records, uint64_t base, const ma_fastq_records* out,
                   uint64_t* out3);

/* Same on a device buffer with device outputs; returns when the counts are
 * known (the split needs two small device-to-host reads). */
int ma_fastq_parse_device(ma_ctx* ctx, const uint8_t* d_buf, uint64_t n_bytes, int at_eof,
                          uint32_t max_records, uint64_t base, const ma_fastq_records* d_out,
                          uint64_t* out3, void* stream);

/* Which reader's rules a FASTQ split follows: the BAM path's
 * (fq_read_batch above) or the SAM path's, fastq_batch.FastqPairReader
 * (fq2bam-meth/python/fastq_batch.py:230-317 with _qname L18-28): every
 * trailing '\r' dropped from a line, four lines per record whatever they
 * hold, a non-empty unterminated rest is a line, and at the end of the stream
 * a record cut short reads its missing lines as empty (no error). */
#define MA_FASTQ_RULES_STREAM 0
#define MA_FASTQ_RULES_PAIR_READER 1

/* ma_fastq_parse / ma_fastq_parse_device under `rules` (those two are
 * MA_FASTQ_RULES_STREAM). */
int ma_fastq_parse_rules(ma_ctx* ctx, const uint8_t* buf, uint64_t n_bytes, int at_eof,
                         uint32_t max_records, uint64_t base, int rules,
                         const ma_fastq_records* out, uint64_t* out3);
int ma_fastq_parse_rules_device(ma_ctx* ctx, const uint8_t* d_buf, uint64_t n_bytes, int at_eof,
                                uint32_t max_records, uint64_t base, int rules,
                                const ma_fastq_records* d_out, uint64_t* out3, void* stream);

/* The mapper's input rows from parsed records: [n_seq][max_len] bytes, each
 * SEQ span followed by 'N' up to max_len, and the lengths (fq_pack_bases,
 * linear_fastq.mojo:454-492; the bases stay unconverted: the mapping call's
 * bisulfite modes convert them).  d_lens may be NULL.  Asynchronous. */
int ma_fastq_rows_device(ma_ctx* ctx, const uint8_t* d_arena, const uint64_t* d_seq_off,
                         const uint32_t* d_seq_len, uint32_t n_seq, uint32_t max_len,
                         uint8_t* d_rows, uint32_t* d_lens, void* stream);

/* ---- BAM records of a mapped batch ---------------------------------- */

/*
 * The FASTQ arena of a batch (FastqArena, fq2bam-meth/src/linear_fastq.mojo:
 * 75-95, as fq_export_ptrs L518-544 hands it to the BAM packer): one byte
 * array and, per record [n_seq] (R1 rows then R2 rows), the byte offset and
 * length of the read name (the qname span), of the original (unconverted)
 * bases and of the qualities.  qual_off == NULL: no qualities.
 */
typedef struct ma_fastq_arena {
    const uint8_t* data;
    uint64_t data_bytes;
    const uint64_t* name_off;
    const uint32_t* name_len;
    const uint64_t* orig_off;
    const uint32_t* orig_len;
    const uint64_t* qual_off;
    const uint32_t* qual_len;
} ma_fastq_arena;

/*
 * Sort / duplicate-marking metadata of a tile (h_coord .. h_pair,
 * linear_gpu_fm.mojo:2133-2139), arrays of meta_cap entries indexed by the
 * record's position in the tile.
 *   coord  _coord_key (L389-395): tid << 32 | pos, unplaced records
 *          0xffffffff << 32 | tile index
 *   dhi, dlo  duplicate key: _pack_end (L398-405) of the 5' ends, pair-wise
 *          ordered; unplaced: ~0 and the tile index
 *   rec    chunk << 32 | byte offset of the record in its chunk
 *   len    record bytes including the block_size word
 *   score  mapq << 8 | (255 - clamp(NM)), summed over a pair
 *   pair   pair id, unique across tiles
 */
typedef struct ma_bam_meta {
    uint64_t* coord;
    uint64_t* dhi;
    uint64_t* dlo;
    uint64_t* rec;
    uint32_t* len;
    uint32_t* score;
    uint32_t* pair;
} ma_bam_meta;

/* Tile state carried from batch to batch: the n_reads / n_mapped / n_total /
 * tile_chunks / meta_cap arguments of _emit_bam_from_batch. */
typedef struct ma_bam_tile {
    uint64_t n_reads;  /* records already in the tile (in/out)            */
    uint64_t n_mapped; /* mapped records so far (in/out)                  */
    uint64_t n_total;  /* records of tiles flushed before this one        */
    uint64_t meta_cap; /* entries of the metadata arrays                  */
    uint32_t chunk;    /* index of this batch's BAM chunk in the tile     */
} ma_bam_tile;

/*
 * Packs the BAM records of one mapped batch.  Replaces _emit_bam_from_batch
 * (linear_gpu_fm.mojo:669-984) and _pack_bam_aln (L497-666): single-end
 * records get flags 1|64, pairs 1|64 and 1|128 with the mate fields, proper
 * pair flag and TLEN; SEQ is the original bases (reverse-complemented on the
 * reverse strand), QUAL phred-33 (0xff without qualities of the read's
 * length), tags RG:Z:<rg> and NM:C.  Records are written to `bam` in R1,R2
 * order exactly as the reference's serial loop writes them; metadata goes to
 * entries [n_reads, n_reads + n_seq) and the tile's n_reads / n_mapped
 * advance.  Host buffers, synchronous.
 *   hits        the batch's mapping outputs (host arrays [n_seq])
 *   rid_to_tid  [n_tid] contig index -> SAM tid (_rid_to_tid_table L423-435)
 *   rg, rg_n    read-group id bytes
 * Errors (nothing is written, the tile is unchanged):
 *   MA_ERR_ARG  "FM sort cap exceeded" (n_reads + n_seq > meta_cap),
 *               "BAM batch buffer overflow" (records exceed bam_cap), or an
 *               arena span outside the arena.
 */
int ma_emit_bam_batch(ma_ctx* ctx, const ma_hits* hits, uint32_t n1, int paired,
                      const ma_fastq_arena* arena, const int32_t* rid_to_tid, int32_t n_tid,
                      const uint8_t* rg, uint32_t rg_n, uint8_t* bam, uint64_t bam_cap,
                      uint64_t* bam_bytes, const ma_bam_meta* meta, ma_bam_tile* tile);

/*
 * Same on device buffers, asynchronous on `stream` (NULL = the context's
 * stream); the metadata arrays are the tile's, on the device.  d_status
 * (device, 3 x u64) receives the batch's record bytes, its mapped records
 * and the number of records whose arena spans fall outside data_bytes
 * (written with zero bytes in their place; a caller treats the batch as
 * failed).  Records and `rec` are written only when d_status[0] <= bam_cap.
 * The tile is read, not advanced: the caller adds n_seq and d_status[1].
 */
int ma_emit_bam_batch_device(ma_ctx* ctx, const ma_hits* d_hits, uint32_t n1, int paired,
                             const ma_fastq_arena* d_arena, const int32_t* d_rid_to_tid, int32_t n_tid,
                             const uint8_t* d_rg, uint32_t rg_n, uint8_t* d_bam, uint64_t bam_cap,
                             const ma_bam_meta* d_meta, const ma_bam_tile* tile, uint64_t* d_status,
                             void* stream);

/* ---- coordinate sort, duplicate marking, sorted record gather -------- */

/*
 * Sorts a tile of n records (n < 2^32) by coordinate and marks duplicates.
 * Replaces gpu_sort_markdup (fq2bam-meth/src/linear_gpu_sort.mojo:24-560),
 * whose results do not depend on its tile size (METHYLGRAPHER_FM_SORT_TILE):
 *   perm      record indices in coordinate order: stable by coord, ties in
 *             record order (L469-525)
 *   is_dup    1 for a duplicate, in record order.  Records are grouped by
 *             equal (dhi, dlo); in each group except the unplaced one
 *             (dhi == ~0) the pair with the highest score, then the lowest
 *             pair id, is kept and every record of another pair is marked
 *             (L409-466).  All 0 when do_markdup == 0.
 *   dup_perm  (optional) record indices in (dhi, dlo, index) order; the
 *             identity when do_markdup == 0
 *   n_marked  (optional) number of records marked
 * Inputs are the ma_bam_meta arrays of the tile.  Host buffers, synchronous.
 */
int ma_sort_markdup(ma_ctx* ctx, uint64_t n, const uint64_t* coord, const uint64_t* dhi,
                    const uint64_t* dlo, const uint32_t* score, const uint32_t* pair,
                    uint32_t* is_dup, uint32_t* perm, int do_markdup, uint32_t* dup_perm,
                    uint64_t* n_marked);

/* Same on device buffers, asynchronous on `stream` (NULL = the context's
 * stream); d_marked (device u64, optional) receives the marked count. */
int ma_sort_markdup_device(ma_ctx* ctx, uint64_t n, const uint64_t* d_coord,
                           const uint64_t* d_dhi, const uint64_t* d_dlo, const uint32_t* d_score,
                           const uint32_t* d_pair, uint32_t* d_is_dup, uint32_t* d_perm,
                           int do_markdup, uint32_t* d_dup_perm, uint64_t* d_marked, void* stream);

/*
 * The tile's records in perm order as one uncompressed BAM record stream,
 * flag 0x400 set on records with is_dup != 0 when apply_dup.  Replaces the
 * record gather of _gather_perm_to_writer (linear_gpu_fm.mojo:177-225; the
 * flag edit is _or_dup_flag, L408-420).  rec[i] = chunk << 32 | offset
 * locates record i in chunks[chunk] (chunk_len bytes each); len[i] is its
 * size.  Host buffers, synchronous.  MA_ERR_ARG when the stream exceeds
 * out_cap or a record lies outside its chunk.
 */
int ma_gather_sorted_bam(ma_ctx* ctx, uint64_t n, const uint32_t* perm, const uint64_t* rec,
                         const uint32_t* len, const uint32_t* is_dup, int apply_dup,
                         const uint8_t* const* chunks, const uint64_t* chunk_len, uint32_t n_chunks,
                         uint8_t* out, uint64_t out_cap, uint64_t* out_bytes);

/* Same on device buffers (d_chunks: a device array of device chunk
 * pointers), asynchronous.  d_status (device, 2 x u64) receives the stream's
 * size and the number of records whose index, chunk or span is out of range
 * (written as zero bytes).  Records are written only when d_status[0] <=
 * out_cap. */
int ma_gather_sorted_bam_device(ma_ctx* ctx, uint64_t n, const uint32_t* d_perm,
                                const uint64_t* d_rec, const uint32_t* d_len,
                                const uint32_t* d_is_dup, int apply_dup,
                                const uint8_t* const* d_chunks, const uint64_t* d_chunk_len,
                                uint32_t n_chunks, uint8_t* d_out, uint64_t out_cap,
                                uint64_t* d_status, void* stream);

/* ---- SAM records of a mapped batch ---------------------------------- */

/* Per rid, the canonical contig name the SAM text carries (_canonical_contig,
 * fq2bam-meth/src/linear_gpu_locate.mojo:156-162: bwa-meth's leading f / r
 * dropped) as a span of `names`, and a canonical id that is equal for two
 * rids exactly when their canonical names are equal. */
typedef struct ma_sam_contigs {
    const uint8_t* names;
    uint64_t names_bytes;
    const uint64_t* name_off;
    const uint32_t* name_len;
    const uint32_t* canon;
    uint32_t n;
} ma_sam_contigs;

/*
 * The SAM text lines of one mapped batch: for each read (single-end) or pair
 * (R1 line, then R2 line), in batch order.  Replaces the SAM loop of
 * map_fastq_fm_gpu (fq2bam-meth/src/linear_gpu_fm.mojo:2787-2836) with
 * _hit_from_fm (L987-1025), pair_hits and hit_to_sam_line
 * (fq2bam-meth/src/linear_extend.mojo:263-320) and the RG tag of
 * _sam_with_rg_fm (L80-81):
 *   - unmapped (rid < 0, or no base left between the clips): FLAG 4, RNAME
 *     "*", POS 0, MAPQ 0, CIGAR "*"; otherwise the hit's flag, RNAME the
 *     canonical name, POS pos + 1, CIGAR [slS]mM[srS];
 *   - SEQ the original bases (arena orig span), reverse-complemented on
 *     flag 16 (byte-wise, any byte but A/C/G/T becomes N); QUAL the record's
 *     qualities as they are (an empty span gives an empty field);
 *   - pairs: flags 1|64 / 1|128; both placed on the same canonical contig:
 *     flag 2, RNEXT "=", PNEXT the mate's POS, TLEN |POS2 - POS1| + len(SEQ2)
 *     (negated on R2); otherwise flag 8 on the mate of an unplaced record and
 *     RNEXT / PNEXT of a placed mate (a canonical name "*" counts as
 *     unplaced);
 *   - names: each byte >= 0x80 is written as U+FFFD (EF BF BD), the ASCII
 *     decode with replacement of the reference's reader; SEQ and QUAL must be
 *     valid UTF-8 (the reference decodes them strictly).
 * Hits and arena columns hold R1 rows then R2 rows; the arena's qual_off
 * must be set.  mapped receives the records whose RNAME is not "*".  Host
 * buffers, synchronous.  Errors: MA_ERR_ARG "SAM batch buffer overflow"
 * (sam_cap too small; sam_bytes still receives the size), "FASTQ SEQ/QUAL is
 * not valid UTF-8", "hit rid outside the contig table", or an arena span
 * outside the arena.
 */
int ma_emit_sam_batch(ma_ctx* ctx, const ma_hits* hits, uint32_t n1, int paired,
                      const ma_fastq_arena* arena, const ma_sam_contigs* contigs,
                      const uint8_t* rg, uint32_t rg_n, uint8_t* sam, uint64_t sam_cap,
                      uint64_t* sam_bytes, uint64_t* mapped);

/* Same on device buffers (hits, arena columns, contig table, rg, output),
 * asynchronous on `stream`.  d_status (device, 3 x u64): [0] the batch's
 * text size, [1] mapped records, [2] error bits (1 text larger than sam_cap,
 * 2 SEQ/QUAL not valid UTF-8, 4 rid outside the contig table, 8 an arena span
 * outside the arena).  Text is written only when [2] == 0. */
int ma_emit_sam_batch_device(ma_ctx* ctx, const ma_hits* d_hits, uint32_t n1, int paired,
                             const ma_fastq_arena* d_arena, const ma_sam_contigs* d_contigs,
                             const uint8_t* d_rg, uint32_t rg_n, uint8_t* d_sam, uint64_t sam_cap,
                             uint64_t* d_status, void* stream);

/* ---- BGZF ------------------------------------------------------------ */

/*
 * Compresses an uncompressed BAM stream (header + records) into BGZF.
 * Replaces the BGZF layer of the reference's BAM writer
 * (fq2bam-meth/python/bam_emit.py: _BgzfWriter L101-186, _bgzf_block
 * L77-98): the stream is cut every 65280 bytes; each piece becomes a gzip
 * member (FEXTRA "BC" subfield with BSIZE, raw deflate, CRC-32, ISIZE) and,
 * with append_eof, the 28-byte EOF member closes the file.  level 0 stores
 * the pieces with the framing zlib produces for one compress + finish call,
 * so the file is byte-identical to the reference's at that level; levels
 * 1..9 use this library's LZ77 + dynamic-Huffman coder (the deflate data
 * differ from zlib's, the members decompress to the same bytes, and the
 * framing, block boundaries, CRCs and sizes are the reference's).  Host
 * buffers, synchronous; out_bytes receives the file size.  MA_ERR_ARG when
 * out_cap is smaller (ma_bgzf_bound gives a safe size).
 */
int ma_bgzf_compress(ma_ctx* ctx, const uint8_t* in, uint64_t n, int level, int append_eof,
                     uint8_t* out, uint64_t out_cap, uint64_t* out_bytes);

/* Same on device buffers; returns when the size is known (synchronous on
 * `stream`, NULL = the context's stream). */
int ma_bgzf_compress_device(ma_ctx* ctx, const uint8_t* d_in, uint64_t n, int level,
                            int append_eof, uint8_t* d_out, uint64_t out_cap,
                            uint64_t* out_bytes, void* stream);

/* An output size large enough for n input bytes (EOF member included). */
uint64_t ma_bgzf_bound(uint64_t n);

/*
 * Inflates the members of a BGZF file (compressed FASTQ as bgzip writes it)
 * on the device, one member per warp: the deflate payload of member m is
 * in[src_off[m], + src_len[m]) and its isize[m] bytes go to
 * out[dst_off[m], ...); each member's size and CRC-32 (crc[m]) are checked.
 * The member table comes from the gzip headers (BSIZE of the "BC" extra
 * field), parsed on the host.  Replaces the decompression of the
 * reference's FASTQ readers (`pigz -dc` / the gzip module,
 * fq2bam-meth/python/fastq_batch.py:31-46, linear_fastq.mojo _looks_gz
 * L49-51) for BGZF inputs.  status[m]: 0, 1..7 invalid deflate data (ends
 * early, block type, stored lengths, code lengths, code, distance, more data
 * than ISIZE), 8 size or 9 CRC-32 mismatch, 10 a span outside its buffer.
 * Host buffers, synchronous; MA_ERR_FORMAT names the first failing member.
 */
int ma_bgzf_inflate(ma_ctx* ctx, const uint8_t* in, uint64_t in_bytes, const uint64_t* src_off,
                    const uint32_t* src_len, const uint64_t* dst_off, const uint32_t* isize,
                    const uint32_t* crc, uint32_t n_members, uint8_t* out, uint64_t out_bytes,
                    uint32_t* status);

/* Same on device buffers, asynchronous on `stream`; d_status receives the
 * per-member codes. */
int ma_bgzf_inflate_device(ma_ctx* ctx, const uint8_t* d_in, uint64_t in_bytes,
                           const uint64_t* d_src_off, const uint32_t* d_src_len,
                           const uint64_t* d_dst_off, const uint32_t* d_isize,
                           const uint32_t* d_crc, uint32_t n_members, uint8_t* d_out,
                           uint64_t out_bytes, uint32_t* d_status, void* stream);

/* ---- measurement (no reference counterpart; the reference only prints
 * perf_counter stage timers, linear_gpu_fm.mojo:2270-2273,3317-3340) ---- */

/* flags bit 0: time each kernel of a mapping call with CUDA events on its
 * stream; bit 1: run the counting instantiation of the seed kernel, which
 * tallies its index and text accesses (slower; for traffic accounting). */
int ma_ctx_set_profiling(ma_ctx* ctx, int flags);
/* Device time (ms) in the last call of: pack, seed/extend (both stages),
 * rescue, and stage 1 alone (equal to seed/extend for seed_kernel 0). */
int ma_ctx_kernel_ms(const ma_ctx* ctx, float* out4);
/* Profiling (flag 1), wavefront form: the last call's wf_search, wf_eval and
 * wf_finalize kernel times summed over its rounds (ms), the rounds timed
 * (negative when the call had more than 64 rounds: only the first 64 are in
 * the sums), and the time of the stage-2 warps that finish the reads the
 * rounds left over (ms). */
int ma_ctx_wave_ms(const ma_ctx* ctx, float* out5);
/* The part of ma_ctx_traffic's tallies that the wavefront form's stage-2
 * warps made (counting flag 2; zeros for the other forms). */
int ma_ctx_traffic_stage2(const ma_ctx* ctx, uint64_t* out12);
/* Tallies of the last counting call: 32-B Occ lines, k-mer entries, SA
 * entries, distinct 32-B pac sectors per evaluated locus, backward steps,
 * endpoints searched, loci evaluated, read words read, endpoints skipped as
 * predicted duplicates, reads handled by stage 2, stage-2 endpoint groups,
 * shift evaluations. */
int ma_ctx_traffic(const ma_ctx* ctx, uint64_t* out12);
/* Random aligned `line_bytes` (32 or 64) gathers over a buffer of
 * buffer_bytes: achieved GB/s (the random-gather roofline). */
int ma_bench_gather(ma_ctx* ctx, uint64_t buffer_bytes, int line_bytes, uint64_t n_loads, double* gbps);

/* ---- synthetic workloads (bench and tests; no reference counterpart) -- */

/*
 * Writes a FASTA of total_len bases split into n_contigs contigs, from a
 * first-order base model with GC fraction gc and CpG frequency cpg.
 */
int ma_synth_reference(const char* fasta_out, uint64_t total_len,
                       int n_contigs, double gc, double cpg, uint64_t seed);

/* Repeat content of a synthetic reference (ma_synth_reference_model). */
typedef struct ma_repeat_model {
    double repeat_frac;   /* share of bases in copies of family elements    */
    double tandem_frac;   /* share of bases in low-complexity tandem runs    */
    uint32_t families;    /* element families per length class               */
    uint32_t short_len;   /* element length of the short class (e.g. 300)    */
    uint32_t long_len;    /* element length of the long class (e.g. 6000);
                             long copies are 5' fragments, 1/8..1 of it      */
    double long_share;    /* share of copied bases from the long class       */
    double div_min, div_max; /* per-copy divergence, uniform in this range:
                             substitutions at that rate, 1-bp insertions and
                             deletions at a twentieth of it each             */
    uint32_t unit_min, unit_max; /* tandem unit length range (bases)         */
    uint32_t run_min, run_max;   /* tandem run length range (bases), 2% of
                             the run's bases substituted                     */
} ma_repeat_model;

/*
 * The base model of ma_synth_reference, generated contig by contig on host
 * threads (the output depends on the seed only), with copies of repeat
 * family elements (either orientation) and tandem runs interleaved with the
 * background when rm is not NULL.
 */
int ma_synth_reference_model(const char* fasta_out, uint64_t total_len,
                             int n_contigs, double gc, double cpg,
                             uint64_t seed, const ma_repeat_model* rm);

typedef struct ma_read_model {
    uint32_t len_fixed;     /* >0: every read this long                       */
    double len_lognorm_median; /* used when len_fixed == 0                    */
    double len_lognorm_sigma;
    uint32_t len_min, len_max;
    double frag_mean, frag_sd; /* paired fragments                            */
    double conv_non_cpg;    /* P(non-CpG C converted)                         */
    double cpg_retain;      /* P(CpG C retained)                              */
    double sub_rate;        /* uniform substitution error rate                */
    double random_frac;     /* fraction of fully random reads                 */
    double non_directional; /* fraction of CTOT/CTOB reads                    */
} ma_read_model;

/*
 * Simulates bisulfite reads from `fasta` into padded row-major ASCII
 * buffers (the ma_map_batch layout).  bases must hold n_seq*max_len bytes,
 * lens n_seq entries, where n_seq = n1 * (paired ? 2 : 1).  truth_pos /
 * truth_rev (optional, [n_seq]) receive the forward text coordinate and
 * strand each read was drawn from (UINT64_MAX for random reads).
 */
int ma_synth_reads(const char* fasta, const ma_read_model* m, uint32_t n1,
                   int paired, uint32_t max_len, uint64_t seed,
                   uint8_t* bases, uint32_t* lens, uint64_t* truth_pos,
                   uint8_t* truth_rev);

#ifdef __cplusplus
}
#endif
#endif /* MOJOALIGN_B200_H */
