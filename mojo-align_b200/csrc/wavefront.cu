// wavefront.cu - seed_kernels 2, 3 and 4: the seed/extend search as rounds of
// data-parallel passes over the whole batch (fm_seed_extend_kernel,
// fq2bam-meth/src/linear_gpu_fm.mojo:1156-1837, with the candidate order
// and exactness argument of seed_core.cuh).
//
// Round k covers right endpoints [resume, resume + width) of every read
// still active (width w0 in round 0, w after it):
//   search   one thread per (read, endpoint): duplicate prediction, backward
//            search, SA rows -> candidate loci appended to a batch-wide
//            locus list (one atomic per warp);
//   eval     one thread per (locus, shift): the shift's candidates (full
//            compare, soft-clip retry, deletion probe) and an atomicMin of
//            the best key per read, packed with the locus' list index;
//   finalize one thread per active read: the new best (its fields are
//            recomputed from the winning locus and shift), the nm == 0 stop,
//            the exact nm == 1 early stop, the next round's active list.
// Every candidate of a round comes after the best of the rounds before it
// in the reference's order, so pruning against that best and taking the
// minimum key over the round gives the reference's hit.  A read whose loci
// do not fit the list is left out of its round (its memo and best roll
// back) and finished by the stage-2 warp kernel from that round's first
// endpoint, as are reads still active after the last round.
#include <cuda_runtime.h>

#include "ma_device.cuh"
#include "ma_internal.h"
#include "seed_core.cuh"

namespace ma {

int launch_stage2_pending(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out,
                          uint64_t* key, uint64_t* memo, uint8_t* memo_n, uint16_t* resume, uint32_t* pending,
                          uint32_t* counters, int blocks, int level, int first_wave, unsigned long long* tally,
                          cudaStream_t st);

namespace {

// counters[]
constexpr int C_ACTIVE = 0;    // reads active in the current round
constexpr int C_NEXT = 1;      // reads appended to the next round's list
constexpr int C_LOCI = 4;      // loci appended in the current round: a u64 in counters[4..5]
constexpr int C_ROUNDS = 3;    // read-rounds processed (tally)
constexpr int C_HANDOFF = 8;   // [8] reads for stage 2, [9] its work cursor
constexpr int N_COUNTERS = 16;

// Round keys: nm << (27 + ib) | ordinal << ib | locus index, ib bits of
// index: what the largest nm of the call leaves of the 64 bits, at most 31.
constexpr uint64_t MAX_LOCI = (1ull << 31) - 1;  // list capacity limit (indices fit 31 bits)

constexpr uint32_t DEAD_LOCUS = 0xFFFFFFFFu;  // WLocus.read of a slot without a locus
constexpr int PREDICT_MEMO = 4;  // memo loci a duplicate prediction checks besides the best

// One candidate locus of a round (32 bytes: two per 64-B line).
struct WLocus {
    int64_t b0;
    uint64_t uk;         // first SA row of the seed's interval
    uint32_t read, ord_row;
    int32_t crid_rev;    // contig * 2 + strand (contig -1: -2 | strand)
    uint16_t us;         // seed start
    uint16_t e_dl;       // right endpoint (bits 0-10) | (ul - uk) << 11
    __device__ int crid() const { return crid_rev >> 1; }
    __device__ int rev() const { return crid_rev & 1; }
    __device__ int e() const { return e_dl & 0x7FF; }
    __device__ uint64_t ul() const { return uk + (e_dl >> 11); }
};
static_assert(sizeof(WLocus) == 32, "WLocus is 32 bytes");

struct Wave {
    uint32_t* counters;
    uint64_t* best_key;   // nm << 27 | ordinal of the best so far, ~0 = none
    uint64_t* round_key;  // this round's minimum, packed with the locus index
    uint64_t* memo;       // [n][MEMO1] loci evaluated (b0 * 2 + strand)
    uint8_t* memo_n;      // memo entries valid at the start of the round
    uint32_t* memo_next;  // memo entries claimed during the round
    uint16_t* resume;     // first right endpoint of the read's next round
    uint8_t* overflow;    // the read's loci did not fit the list this round
    int64_t* best_tag;    // locus of the best hit, -1 = none
    uint32_t* active[2];  // ping-pong lists of active reads
    uint32_t* pending;    // reads handed to stage 2
    WLocus* loci;
    uint64_t locus_cap;
    int idx_bits;  // locus-index bits of the round keys
};

size_t align256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

// The round's locus count (64-bit: the rows a round asks for can exceed 2^32).
__device__ __forceinline__ unsigned long long* loci_count(const Wave& w) {
    return reinterpret_cast<unsigned long long*>(w.counters + C_LOCI);
}

// Carves the scratch; returns the bytes used (layout only when p != null).
size_t wave_layout(char* p, int64_t n_seq, uint64_t locus_cap, Wave* w) {
    const size_t n = static_cast<size_t>(n_seq);
    size_t o = 0;
    auto take = [&](size_t bytes) {
        char* q = p ? p + o : nullptr;
        o += align256(bytes);
        return q;
    };
    Wave v{};
    v.counters = reinterpret_cast<uint32_t*>(take(N_COUNTERS * 4));
    v.best_key = reinterpret_cast<uint64_t*>(take(n * 8));
    v.round_key = reinterpret_cast<uint64_t*>(take(n * 8));
    v.memo = reinterpret_cast<uint64_t*>(take(n * 8 * MEMO1));
    v.memo_n = reinterpret_cast<uint8_t*>(take(n));
    v.memo_next = reinterpret_cast<uint32_t*>(take(n * 4));
    v.resume = reinterpret_cast<uint16_t*>(take(n * 2));
    v.overflow = reinterpret_cast<uint8_t*>(take(n));
    v.best_tag = reinterpret_cast<int64_t*>(take(n * 8));
    v.active[0] = reinterpret_cast<uint32_t*>(take(n * 4));
    v.active[1] = reinterpret_cast<uint32_t*>(take(n * 4));
    v.pending = reinterpret_cast<uint32_t*>(take(n * 4));
    v.loci = reinterpret_cast<WLocus*>(take(locus_cap * sizeof(WLocus)));
    v.locus_cap = locus_cap;
    if (w) *w = v;
    return o;
}

uint64_t locus_capacity(int64_t n_seq, int per_read) {
    uint64_t c = static_cast<uint64_t>(per_read) * static_cast<uint64_t>(n_seq);
    if (c < 1024) c = 1024;
    return c < MAX_LOCI ? c : MAX_LOCI;
}

__global__ void __launch_bounds__(256) wf_init_kernel(Wave w, DevOut out, const uint32_t* __restrict__ lens,
                                                      int64_t n_seq) {
    const int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (r == 0) {
        for (int i = 0; i < N_COUNTERS; ++i) w.counters[i] = 0;
        w.counters[C_ACTIVE] = static_cast<uint32_t>(n_seq);
    }
    if (r >= n_seq) return;
    w.best_key[r] = ~0ull;
    w.round_key[r] = ~0ull;
    w.memo_n[r] = 0;
    w.memo_next[r] = 0;
    w.resume[r] = 0;
    w.overflow[r] = 0;
    w.best_tag[r] = -1;
    w.active[0][r] = static_cast<uint32_t>(r);
    Best none;
    none.key = ~0ull;
    none.crid = -1;
    none.uk = none.ul = 0;
    none.us = none.e = -1;
    write_hit(out, r, none, static_cast<int>(lens[r]));
}

// Moves the next round's active count into place (one thread).
__global__ void wf_round_begin_kernel(Wave w) {
    w.counters[C_ACTIVE] = w.counters[C_NEXT];
    w.counters[C_NEXT] = 0;
    *loci_count(w) = 0;
}

// Whether an SA row of a found seed gives a locus not evaluated before.
__device__ __forceinline__ bool fresh_locus(const DevIndex& ix, const Wave& w, int64_t r, int n_memo, uint64_t sa_pos,
                                            int us, int e, int qlen, int64_t& b0, int& rev) {
    if (!locus_of_row(ix, sa_pos, us, e, qlen, b0, rev)) return false;
    const uint64_t tag = static_cast<uint64_t>(b0 * 2 + rev);
    for (int m = 0; m < n_memo; ++m)
        if (w.memo[r * MEMO1 + m] == tag) return false;
    return true;
}

// Search: one thread per (active read, endpoint of the round).  The loop
// is warp-uniform (whole warps step together) for the warp-wide append.
template <bool S, int MINB>
__global__ void __launch_bounds__(256, MINB) wf_search_kernel(DevIndex ix, DevReads R, DevParams P, Wave w,
                                                        const uint32_t* __restrict__ act, int width,
                                                        unsigned long long* __restrict__ tally_out) {
    Tally t{};
    const uint64_t n_items = static_cast<uint64_t>(w.counters[C_ACTIVE]) * static_cast<uint64_t>(width);
    const int lane = threadIdx.x & 31;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const bool can_predict = ix.summary && ix.kmer3_k > 0 && ix.kmer3_k <= P.seed_len;
    for (uint64_t base = (blockIdx.x * static_cast<uint64_t>(blockDim.x)) + (threadIdx.x & ~31u); base < n_items;
         base += stride) {
        const uint64_t item = base + lane;
        Seed sd{0, 0, -1, false};
        int64_t r = 0;
        int ei = 0, e = 0, qlen = 0, n_memo = 0;
        ReadView rd{};
        if (item < n_items) {
            const uint64_t a = item < (1ull << 32) ? static_cast<uint32_t>(item) / static_cast<uint32_t>(width)
                                                   : item / static_cast<uint64_t>(width);
            const int j = static_cast<int>(item - a * static_cast<uint64_t>(width));
            r = act[a];
            rd = read_view(R, r);
            qlen = rd.qlen;
            ei = static_cast<int>(w.resume[r]) + j;
            if (ei < endpoint_count(P, qlen)) {
                e = P.seed_len - 1 + ei * P.seed_stride;
                n_memo = w.memo_n[r];
                // a read with no hit yet gains little from predicting its
                // rejected loci again: only reads with a best try the memo
                const int64_t best_tag = w.best_tag[r];
                const bool dup = can_predict && best_tag != -1 &&
                                 predicted_duplicate<S>(ix, rd, e, P, best_tag, w.memo + r * MEMO1,
                                                        n_memo < PREDICT_MEMO ? n_memo : PREDICT_MEMO, t);
                if constexpr (S) t.skipped += dup;
                if (!dup) sd = search_endpoint<S>(ix, rd, e, P, t);
            }
        }
        // every SA row takes a list slot (one atomic per warp); rows that
        // give no new locus leave their slot dead
        const uint32_t n_rows = sd.found ? static_cast<uint32_t>(sd.l - sd.k + 1) : 0u;
        uint32_t incl = n_rows;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += v;
        }
        const uint32_t warp_total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        unsigned long long wbase = 0;
        if (lane == 31 && warp_total) wbase = atomicAdd(loci_count(w), static_cast<unsigned long long>(warp_total));
        wbase = __shfl_sync(0xFFFFFFFFu, wbase, 31);
        // the warp's rows, 32 at a time, one per lane (seeds have 1..16 rows)
        for (uint32_t c0 = 0; c0 < warp_total; c0 += 32) {
            const uint32_t idx = c0 + lane;
            int owner = 0;  // first lane whose inclusive row count exceeds idx
            for (int step = 16; step >= 1; step >>= 1) {
                const uint32_t v = __shfl_sync(0xFFFFFFFFu, incl, owner + step - 1);
                if (v <= idx) owner += step;
            }
            const int own = owner < 32 ? owner : 31;
            const uint64_t o_k = __shfl_sync(0xFFFFFFFFu, sd.k, own);
            const uint64_t o_l = __shfl_sync(0xFFFFFFFFu, sd.l, own);
            const int o_s = __shfl_sync(0xFFFFFFFFu, sd.s, own);
            const int o_e = __shfl_sync(0xFFFFFFFFu, e, own);
            const int o_ei = __shfl_sync(0xFFFFFFFFu, ei, own);
            const int o_qlen = __shfl_sync(0xFFFFFFFFu, qlen, own);
            const int o_memo = __shfl_sync(0xFFFFFFFFu, n_memo, own);
            const int64_t o_r = __shfl_sync(0xFFFFFFFFu, r, own);
            const uint32_t o_first = __shfl_sync(0xFFFFFFFFu, incl - n_rows, own);
            if (idx >= warp_total) continue;
            const uint64_t hi = o_k + (idx - o_first);
            const uint64_t slot = static_cast<uint64_t>(wbase) + idx;
            if (slot >= w.locus_cap) {
                w.overflow[o_r] = 1;
                continue;
            }
            const uint64_t sa_pos = sa_at(ix, hi);
            if constexpr (S) t.sa_loads++;
            WLocus L;
            int64_t b0;
            int rev;
            if (!fresh_locus(ix, w, o_r, o_memo, sa_pos, o_s, o_e, o_qlen, b0, rev)) {
                L.read = DEAD_LOCUS;
                w.loci[slot] = L;
                continue;
            }
            L.b0 = b0;
            L.uk = o_k;
            L.read = static_cast<uint32_t>(o_r);
            L.ord_row = (static_cast<uint32_t>(o_ei) * 16 + static_cast<uint32_t>(hi - o_k)) * ADJ_SPAN;
            L.us = static_cast<uint16_t>(o_s);
            L.e_dl = static_cast<uint16_t>(o_e | ((o_l - o_k) << 11));
            L.crid_rev = static_cast<int32_t>(contig_hint(ix, b0).crid) * 2 + rev;
            w.loci[slot] = L;
            if constexpr (S) tally_locus(t, b0, clamps_for(P, o_qlen).adj_cap, o_qlen);
            const uint32_t m = atomicAdd(&w.memo_next[o_r], 1u);
            if (m < static_cast<uint32_t>(MEMO1)) w.memo[o_r * MEMO1 + m] = static_cast<uint64_t>(b0 * 2 + rev);
        }
    }
    flush_tally<S>(t, tally_out);
}

// Search with lane refill (seed_kernel 3): the same items as
// wf_search_kernel, but each lane steps its own endpoint's search and takes
// a new item when its search ends.  Search lengths differ by two orders of
// magnitude (a table hit ends at once; a seed in a repeat steps back to the
// read's start), so a warp that waits for its longest lane runs most steps
// with few lanes busy.  Here the warp alternates two passes:
//   refill  when at least REFILL_MIN lanes are idle (or all are), the idle
//           lanes take the next items of the warp's chunk sequence and run
//           the duplicate prediction and the table steps;
//   step    the busy lanes take one backward step each.
// Seeds found are staged in shared memory and appended to the locus list at
// least 32 rows at a time (one atomic per flush, one lane per row), as in
// wf_search_kernel.  Which lane or pass finds a seed does not change the
// round's result: the eval keys carry the candidate order.
constexpr int REFILL_MIN = 16;    // idle lanes that trigger a refill pass
constexpr int REFILL_STAGE = 64;  // staged seeds per warp (flushed above 32)
constexpr int SEARCH_WARPS = 8;   // 256 threads

struct StagedSeed {  // 24 bytes
    uint64_t k;
    uint32_t read, rows_end;  // rows_end: staged rows up to and including this seed
    uint16_t s, e, ei, qlen;
};

// Words of read r for the backward steps (qlen is not needed there).
__device__ __forceinline__ ReadView step_view(const DevReads& R, uint32_t r) {
    const uint64_t* b = R.packed + static_cast<uint64_t>(r) * 4 * static_cast<uint64_t>(R.words);
    ReadView v;
    v.fwd = b;
    v.rc = nullptr;
    v.nf = b + 2 * R.words;
    v.nr = nullptr;
    v.qlen = 0;
    return v;
}

template <bool S, int MINB>
__global__ void __launch_bounds__(256, MINB) wf_search_refill_kernel(DevIndex ix, DevReads R, DevParams P, Wave w,
                                                               const uint32_t* __restrict__ act, int width,
                                                               unsigned long long* __restrict__ tally_out) {
    __shared__ StagedSeed s_stage[SEARCH_WARPS][REFILL_STAGE];
    constexpr unsigned FULL = 0xFFFFFFFFu;
    Tally t{};
    const uint64_t n_items = static_cast<uint64_t>(w.counters[C_ACTIVE]) * static_cast<uint64_t>(width);
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1;
    const uint64_t n_warps = static_cast<uint64_t>(gridDim.x) * SEARCH_WARPS;
    const bool can_predict = ix.summary && ix.kmer3_k > 0 && ix.kmer3_k <= P.seed_len;
    StagedSeed* stage = s_stage[threadIdx.x >> 5];
    // the warp's items: chunks of 32 items, warp g takes chunks g, g + n_warps, ...
    uint64_t chunk = static_cast<uint64_t>(blockIdx.x) * SEARCH_WARPS + (threadIdx.x >> 5);
    uint32_t off = 0;          // items of the chunk handed out
    int n_staged = 0;          // warp-uniform
    uint32_t staged_rows = 0;  // warp-uniform
    // the lane's search
    bool busy = false;
    SeedSearch q;
    uint32_t r = 0;
    int e_ei = 0;  // right endpoint | endpoint index << 16
    for (;;) {
        const unsigned idle = __ballot_sync(FULL, !busy);
        const uint64_t cur = chunk * 32 + off;
        const bool more = off < 32 && cur < n_items;
        if (!more && idle == FULL && n_staged == 0) break;
        bool fin = false;  // this lane's search ended in this pass
        Seed sd{0, 0, -1, false};
        if (more && (__popc(idle) >= REFILL_MIN || idle == FULL)) {
            const uint64_t left = min(static_cast<uint64_t>(32 - off), n_items - cur);
            const unsigned take = min(static_cast<uint64_t>(__popc(idle)), left);
            const unsigned rank = __popc(idle & lt_mask);
            if (!busy && rank < take) {
                const uint64_t item = cur + rank;
                const uint64_t a = item < (1ull << 32) ? static_cast<uint32_t>(item) / static_cast<uint32_t>(width)
                                                       : item / static_cast<uint64_t>(width);
                const int j = static_cast<int>(item - a * static_cast<uint64_t>(width));
                r = act[a];
                const ReadView rd = read_view(R, r);
                const int ei = static_cast<int>(w.resume[r]) + j;
                fin = true;
                if (ei < endpoint_count(P, rd.qlen)) {
                    const int e = P.seed_len - 1 + ei * P.seed_stride;
                    e_ei = e | ei << 16;
                    const int n_memo = w.memo_n[r];
                    const int64_t best_tag = w.best_tag[r];
                    const bool dup = can_predict && best_tag != -1 &&
                                     predicted_duplicate<S>(ix, rd, e, P, best_tag, w.memo + r * MEMO1,
                                                            n_memo < PREDICT_MEMO ? n_memo : PREDICT_MEMO, t);
                    if constexpr (S) t.skipped += dup;
                    if (!dup) {
                        busy = search_start<S>(ix, rd, e, P, q, sd, t);
                        fin = !busy;
                    }
                }
            }
            off += take;
            if (off >= 32 || chunk * 32 + off >= n_items) {  // the warp's next chunk
                chunk += n_warps;
                off = 0;
            }
        } else if (busy) {
            busy = search_next<S>(ix, step_view(R, r), e_ei & 0xFFFF, P, q, sd, t);
            fin = !busy;
        }
        // stage the seeds found in this pass (at most 32: n_staged <= 32 here)
        const bool found = fin && sd.found;
        const unsigned fb = __ballot_sync(FULL, found);
        if (fb) {
            const uint32_t n_rows = found ? static_cast<uint32_t>(sd.l - sd.k + 1) : 0u;
            uint32_t incl = n_rows;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += v;
            }
            if (found) {
                StagedSeed g;
                g.k = sd.k;
                g.read = r;
                g.rows_end = staged_rows + incl;
                g.s = static_cast<uint16_t>(sd.s);
                g.e = static_cast<uint16_t>(e_ei & 0xFFFF);
                g.ei = static_cast<uint16_t>(e_ei >> 16);
                g.qlen = static_cast<uint16_t>(__ldg(R.lens + r));
                stage[n_staged + __popc(fb & lt_mask)] = g;
            }
            n_staged += __popc(fb);
            staged_rows += __shfl_sync(FULL, incl, 31);
        }
        if (n_staged == 0) continue;
        if (staged_rows < 32 && n_staged <= REFILL_STAGE - 32) {
            // keep staging unless the warp's items are all searched
            const bool out_of_items = off >= 32 || chunk * 32 + off >= n_items;
            if (!out_of_items || __ballot_sync(FULL, busy)) continue;
        }
        // flush: one list slot per staged row, 32 rows at a time
        __syncwarp();
        unsigned long long wbase = 0;
        if (lane == 0) wbase = atomicAdd(loci_count(w), static_cast<unsigned long long>(staged_rows));
        wbase = __shfl_sync(FULL, wbase, 0);
        for (uint32_t idx = lane; idx < staged_rows; idx += 32) {
            int lo = 0, hi = n_staged - 1;  // first staged seed whose rows_end exceeds idx
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (stage[mid].rows_end > idx) hi = mid;
                else lo = mid + 1;
            }
            const StagedSeed g = stage[lo];
            const uint32_t first = lo ? stage[lo - 1].rows_end : 0u;
            const uint64_t row = g.k + (idx - first);
            const int64_t o_r = g.read;
            const uint64_t slot = static_cast<uint64_t>(wbase) + idx;
            if (slot >= w.locus_cap) {
                w.overflow[o_r] = 1;
                continue;
            }
            const uint64_t sa_pos = sa_at(ix, row);
            if constexpr (S) t.sa_loads++;
            WLocus L;
            int64_t b0;
            int rev;
            if (!fresh_locus(ix, w, o_r, w.memo_n[o_r], sa_pos, g.s, g.e, g.qlen, b0, rev)) {
                L.read = DEAD_LOCUS;
                w.loci[slot] = L;
                continue;
            }
            L.b0 = b0;
            L.uk = g.k;
            L.read = g.read;
            L.ord_row = (static_cast<uint32_t>(g.ei) * 16 + (idx - first)) * ADJ_SPAN;
            L.us = g.s;
            L.e_dl = static_cast<uint16_t>(g.e | ((g.rows_end - first - 1) << 11));
            L.crid_rev = static_cast<int32_t>(contig_hint(ix, b0).crid) * 2 + rev;
            w.loci[slot] = L;
            if constexpr (S) tally_locus(t, b0, clamps_for(P, g.qlen).adj_cap, g.qlen);
            const uint32_t m = atomicAdd(&w.memo_next[o_r], 1u);
            if (m < static_cast<uint32_t>(MEMO1)) w.memo[o_r * MEMO1 + m] = static_cast<uint64_t>(b0 * 2 + rev);
        }
        __syncwarp();
        n_staged = 0;
        staged_rows = 0;
    }
    flush_tally<S>(t, tally_out);
}

// Eval: one thread per locus filters its shifts (live_shifts); the shifts
// left in the warp are spread over its lanes.  Candidates are pruned
// against the read's best from earlier rounds; the round's minimum key per
// read is an atomicMin of (nm, ordinal, locus index) packed in 64 bits.  The
// loop over loci is warp-uniform for the redistribution.
constexpr int EVAL_THREADS = 256;

// One shift (adj) of the locus at list index li: its candidates, pruned
// against the read's best from earlier rounds, and the atomicMin of the
// round key.
template <bool S>
__device__ __forceinline__ void eval_shift(const DevIndex& ix, const DevReads& R, const DevParams& P, const Wave& w,
                                           const WLocus& L, uint32_t li, int adj, Tally& t) {
    const int64_t r = L.read;
    const ReadView rd = read_view(R, r);
    const Clamps cl = clamps_for(P, rd.qlen);
    const uint64_t bn = w.best_key[r] >> ORD_SHIFT;
    const int prune = bn < (1u << 20) ? static_cast<int>(bn) : (1 << 20);
    const int crid = L.crid();
    ContigHint hint{crid, 0, 0};
    if (crid >= 0) {
        hint.coff = static_cast<int64_t>(__ldg(ix.coff + crid));
        hint.clen = static_cast<int64_t>(__ldg(ix.clen + crid));
    }
    Best lb;
    lb.key = ~0ull;
    lb.crid = -1;
    eval_adj<S>(ix, rd, L.b0, L.rev(), adj, cl.budget, cl.clip_cap, L.ord_row, lb, L.uk, L.ul(), L.us, L.e(), prune,
                hint, t);
    if (lb.key != ~0ull) {
        const uint64_t nm = lb.key >> ORD_SHIFT;
        const uint64_t ord = lb.key & ((1ull << ORD_SHIFT) - 1);
        atomicMin(reinterpret_cast<unsigned long long*>(w.round_key + r),
                  static_cast<unsigned long long>((nm << (ORD_SHIFT + w.idx_bits)) | (ord << w.idx_bits) | li));
    }
}

template <bool S, int MINB>
__global__ void __launch_bounds__(EVAL_THREADS, MINB) wf_eval_kernel(DevIndex ix, DevReads R, DevParams P, Wave w,
                                                               unsigned long long* __restrict__ tally_out) {
    __shared__ WLocus s_loci[EVAL_THREADS];
    constexpr unsigned FULL = 0xFFFFFFFFu;
    Tally t{};
    uint64_t n_loci = *loci_count(w);
    if (n_loci > w.locus_cap) n_loci = w.locus_cap;
    const int adj_cap = clamps_for(P, 1 << 20).adj_cap;  // read-independent
    const int lane = threadIdx.x & 31;
    WLocus* wl = s_loci + (threadIdx.x & ~31u);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n_loci; base += stride) {
        const uint32_t li = base + lane;
        uint32_t live = 0;
        if (li < n_loci) {
            const WLocus L = w.loci[li];
            wl[lane] = L;
            const int64_t r = L.read;
            if (L.read != DEAD_LOCUS && !w.overflow[r]) {
                const ReadView rd = read_view(R, r);
                const Clamps cl = clamps_for(P, rd.qlen);
                const uint64_t bn = w.best_key[r] >> ORD_SHIFT;
                const int prune = bn < (1u << 20) ? static_cast<int>(bn) : (1 << 20);
                live = live_shifts<S>(ix, rd, L.b0, L.rev(), adj_cap, cl.budget, cl.clip_cap, prune, t);
            }
        }
        __syncwarp();
        const int n_live = __popc(live);
        int incl = n_live;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(FULL, incl, 31);
        for (int c = 0; c < total; c += 32) {
            const int idx = c + lane;
            int owner = 0;  // first lane whose inclusive count exceeds idx
            for (int step = 16; step >= 1; step >>= 1) {
                const int v = __shfl_sync(FULL, incl, owner + step - 1);
                if (v <= idx) owner += step;
            }
            const int own = owner < 32 ? owner : 31;
            const uint32_t o_live = __shfl_sync(FULL, live, own);
            const int o_first = __shfl_sync(FULL, incl - n_live, own);
            if (idx < total) {
                const int adj = static_cast<int>(__fns(o_live, 0, idx - o_first + 1)) - adj_cap;
                eval_shift<S>(ix, R, P, w, wl[own], base + own, adj, t);
            }
        }
        __syncwarp();
    }
    flush_tally<S>(t, tally_out);
}

// Eval with staged shifts (seed_kernels 3 and 4): the filter pass as in
// wf_eval_kernel, but the live shifts (a fraction of a shift per locus at
// genome scale) are staged per warp in shared memory and evaluated 32 at a
// time, so the full compares run with every lane busy.
constexpr int SHIFT_STAGE = 64;  // staged shifts per warp: locus index << 5 | shift

template <bool S, int MINB>
__global__ void __launch_bounds__(EVAL_THREADS, MINB) wf_eval_staged_kernel(DevIndex ix, DevReads R, DevParams P,
                                                                      Wave w,
                                                                      unsigned long long* __restrict__ tally_out) {
    __shared__ uint64_t s_shift[EVAL_THREADS / 32][SHIFT_STAGE];
    constexpr unsigned FULL = 0xFFFFFFFFu;
    Tally t{};
    uint64_t n_loci = *loci_count(w);
    if (n_loci > w.locus_cap) n_loci = w.locus_cap;
    const int adj_cap = clamps_for(P, 1 << 20).adj_cap;  // read-independent
    const int lane = threadIdx.x & 31;
    uint64_t* stage = s_shift[threadIdx.x >> 5];
    int staged = 0;  // warp-uniform
    const uint32_t stride = gridDim.x * blockDim.x;
    // one more pass after the warp's last loci empties the stage
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u);; base += stride) {
        const bool have = base < n_loci;
        const uint32_t li = base + lane;
        uint32_t rem = 0;  // the lane's live shifts not yet staged
        if (have && li < n_loci) {
            const WLocus L = w.loci[li];
            const int64_t r = L.read;
            if (L.read != DEAD_LOCUS && !w.overflow[r]) {
                const ReadView rd = read_view(R, r);
                const Clamps cl = clamps_for(P, rd.qlen);
                const uint64_t bn = w.best_key[r] >> ORD_SHIFT;
                const int prune = bn < (1u << 20) ? static_cast<int>(bn) : (1 << 20);
                rem = live_shifts<S>(ix, rd, L.b0, L.rev(), adj_cap, cl.budget, cl.clip_cap, prune, t);
            }
        }
        for (;;) {
            // stage as many live shifts as fit (lanes in order)
            if (__ballot_sync(FULL, rem != 0)) {
                const int n = __popc(rem);
                int incl = n;
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += v;
                }
                int at = staged + incl - n;
                while (rem && at < SHIFT_STAGE) {
                    stage[at++] = static_cast<uint64_t>(li) << 5 | static_cast<uint32_t>(__ffs(rem) - 1);
                    rem &= rem - 1;
                }
                const int total = staged + __shfl_sync(FULL, incl, 31);
                staged = total < SHIFT_STAGE ? total : SHIFT_STAGE;
            }
            const bool pending = __ballot_sync(FULL, rem != 0) != 0;
            if (staged < 32 && (have || staged == 0)) break;
            // evaluate the first 32 (or the last few) staged shifts, one per lane
            const int n = staged < 32 ? staged : 32;
            __syncwarp();
            if (lane < n) {
                const uint64_t v = stage[lane];
                const uint32_t sli = static_cast<uint32_t>(v >> 5);
                eval_shift<S>(ix, R, P, w, w.loci[sli], sli, static_cast<int>(v & 31) - adj_cap, t);
            }
            __syncwarp();
            const uint64_t v = lane < staged - n ? stage[n + lane] : 0;
            __syncwarp();
            if (lane < staged - n) stage[lane] = v;
            staged -= n;
            __syncwarp();
            if (!pending && staged < 32 && have) break;
        }
        if (!have) break;
    }
    flush_tally<S>(t, tally_out);
}

// Finalize: one thread per active read (warp-uniform loop for the list
// appends).  last_round: reads with endpoints left go to stage 2.
template <bool S>
__global__ void __launch_bounds__(256) wf_finalize_kernel(DevIndex ix, DevReads R, DevParams P, DevOut out, Wave w,
                                                          const uint32_t* __restrict__ act,
                                                          uint32_t* __restrict__ next, int width, int last_round,
                                                          int* __restrict__ err,
                                                          unsigned long long* __restrict__ tally_out) {
    Tally t{};
    const uint32_t n_act = w.counters[C_ACTIVE];
    const int lane = threadIdx.x & 31;
    const uint32_t stride = gridDim.x * blockDim.x;
    if constexpr (S) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&w.counters[C_ROUNDS], n_act);
    }
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n_act; base += stride) {
        const uint32_t a = base + lane;
        bool to_next = false, to_stage2 = false;
        int64_t r = 0;
        if (a < n_act) {
            r = act[a];
            const ReadView rd = read_view(R, r);
            const int qlen = rd.qlen;
            const Clamps cl = clamps_for(P, qlen);
            const int n_end = endpoint_count(P, qlen);
            if (w.overflow[r]) {
                // left out of this round: roll back and let stage 2 redo it
                w.overflow[r] = 0;
                w.memo_next[r] = w.memo_n[r];
                to_stage2 = true;
            } else {
                const uint32_t mn = w.memo_next[r];
                w.memo_n[r] = static_cast<uint8_t>(mn < static_cast<uint32_t>(MEMO1) ? mn : MEMO1);
                const uint64_t rk = w.round_key[r];
                const uint64_t old = w.best_key[r];
                bool stop = false;
                const uint64_t rkey = rk >> w.idx_bits;  // nm << ORD_SHIFT | ordinal, the best-key format
                if (rk != ~0ull && rkey < old) {
                    // the new best: recompute its fields from the winning locus and shift
                    const WLocus L = w.loci[rk & ((1ull << w.idx_bits) - 1)];
                    const uint32_t ord = static_cast<uint32_t>(rkey & ((1ull << ORD_SHIFT) - 1));
                    const int adj = static_cast<int>(ord / KIND_SPAN) - static_cast<int>(L.ord_row) - 12;
                    const uint64_t bn = old >> ORD_SHIFT;
                    const int prune = bn < (1u << 20) ? static_cast<int>(bn) : (1 << 20);
                    const int crid = L.crid();
                    ContigHint hint{crid, 0, 0};
                    if (crid >= 0) {
                        hint.coff = static_cast<int64_t>(__ldg(ix.coff + crid));
                        hint.clen = static_cast<int64_t>(__ldg(ix.clen + crid));
                    }
                    Best lb;
                    lb.key = ~0ull;
                    lb.crid = -1;
                    eval_adj<S>(ix, rd, L.b0, L.rev(), adj, cl.budget, cl.clip_cap, L.ord_row, lb, L.uk, L.ul(),
                                L.us, L.e(), prune, hint, t);
                    if (lb.key != rkey) {
                        atomicExch(err, 3);  // the recomputed candidate must be the round's minimum
                    } else {
                        write_hit(out, r, lb, qlen);
                        w.best_key[r] = lb.key;
                        w.best_tag[r] = L.b0 * 2 + L.rev();
                        const uint64_t nm = lb.key >> ORD_SHIFT;
                        if (nm == 0) {
                            stop = true;
                        } else if (nm <= 2 && full_compare_key(lb.key)) {
                            const int64_t bstart = static_cast<int64_t>(__ldg(ix.coff + lb.crid)) + lb.pos - lb.sl;
                            stop = better_hit_impossible<S>(ix, rd, bstart, (lb.flag & 16) ? 1 : 0, cl.clip_cap,
                                                            static_cast<int>(nm), t);
                        }
                    }
                }
                w.round_key[r] = ~0ull;
                const int nxt = static_cast<int>(w.resume[r]) + width;
                if (!stop && nxt < n_end) {
                    w.resume[r] = static_cast<uint16_t>(nxt);
                    if (last_round) to_stage2 = true;
                    else to_next = true;
                }
            }
        }
        const unsigned bn = __ballot_sync(0xFFFFFFFFu, to_next);
        if (bn) {
            uint32_t b = 0;
            if (lane == 0) b = atomicAdd(&w.counters[C_NEXT], static_cast<uint32_t>(__popc(bn)));
            b = __shfl_sync(0xFFFFFFFFu, b, 0);
            if (to_next) next[b + __popc(bn & ((1u << lane) - 1))] = static_cast<uint32_t>(r);
        }
        const unsigned bs = __ballot_sync(0xFFFFFFFFu, to_stage2);
        if (bs) {
            uint32_t b = 0;
            if (lane == 0) b = atomicAdd(&w.counters[C_HANDOFF], static_cast<uint32_t>(__popc(bs)));
            b = __shfl_sync(0xFFFFFFFFu, b, 0);
            if (to_stage2) w.pending[b + __popc(bs & ((1u << lane) - 1))] = static_cast<uint32_t>(r);
        }
    }
    flush_tally<S>(t, tally_out);
}

int endpoint_count_host(const DevParams& P, int qlen) {
    return qlen >= P.seed_len ? (qlen - P.seed_len) / P.seed_stride + 1 : 0;
}

template <typename K>
int grid_blocks(K kernel, int sm_count) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, 256, 0);
    if (nb < 1) nb = 1;
    return nb * sm_count;
}

// Register budget of the search / eval kernels (result-neutral): blocks of
// 256 threads asked per SM (1 = the compiler's choice).
template <bool S, int MS, int ME, int MR>
int launch_rounds(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out, const Wave& w,
                  int max_len, int w0, int wn, int max_rounds, int growth, bool refill, bool staged, int sm_count,
                  int* d_err,
                  unsigned long long* tally, WaveTimer* timer, cudaStream_t st) {
    const int n_end_max = endpoint_count_host(P, max_len);
    // round widths: w0, then wn (doubling from the third round with growth)
    int widths[1100];
    int rounds = 0, covered = 0;
    for (int width = w0; covered < n_end_max || rounds == 0; ++rounds) {
        widths[rounds] = width;
        covered += width;
        if (rounds == 0) width = wn;
        else if (growth && width < 4096) width *= 2;
    }
    if (max_rounds > 0 && rounds > max_rounds) rounds = max_rounds;
    static const int g_search = grid_blocks(wf_search_kernel<S, MS>, sm_count);
    static const int g_refill = grid_blocks(wf_search_refill_kernel<S, MR>, sm_count);
    static const int g_eval = grid_blocks(wf_eval_kernel<S, ME>, sm_count);  // EVAL_THREADS = 256
    static const int g_eval_staged = grid_blocks(wf_eval_staged_kernel<S, ME>, sm_count);
    static const int g_fin = grid_blocks(wf_finalize_kernel<S>, sm_count);
    const unsigned init_blocks = static_cast<unsigned>((R.n_seq + 255) / 256);
    wf_init_kernel<<<init_blocks ? init_blocks : 1, 256, 0, st>>>(w, out, R.lens, R.n_seq);
    int launches = 1;
    for (int k = 0; k < rounds; ++k) {
        const int width = widths[k];
        const uint32_t* act = w.active[k & 1];
        uint32_t* nxt = w.active[(k + 1) & 1];
        if (k > 0) {
            wf_round_begin_kernel<<<1, 1, 0, st>>>(w);
            ++launches;
        }
        const bool timed = timer && k < WaveTimer::MAX_ROUNDS;
        if (timed) cudaEventRecord(timer->e[3 * k], st);
        if (refill) wf_search_refill_kernel<S, MR><<<g_refill, 256, 0, st>>>(ix, R, P, w, act, width, tally);
        else wf_search_kernel<S, MS><<<g_search, 256, 0, st>>>(ix, R, P, w, act, width, tally);
        if (timed) cudaEventRecord(timer->e[3 * k + 1], st);
        if (staged) wf_eval_staged_kernel<S, ME><<<g_eval_staged, 256, 0, st>>>(ix, R, P, w, tally);
        else wf_eval_kernel<S, ME><<<g_eval, 256, 0, st>>>(ix, R, P, w, tally);
        if (timed) cudaEventRecord(timer->e[3 * k + 2], st);
        wf_finalize_kernel<S><<<g_fin, 256, 0, st>>>(ix, R, P, out, w, act, nxt, width, k == rounds - 1, d_err,
                                                     tally);
        launches += 3;
    }
    if (timer) {
        const int timed = rounds < WaveTimer::MAX_ROUNDS ? rounds : WaveTimer::MAX_ROUNDS;
        cudaEventRecord(timer->e[3 * timed], st);
        timer->recorded = timed;
        timer->complete = rounds <= WaveTimer::MAX_ROUNDS;
    }
    return launches;
}

}  // namespace

size_t wavefront_scratch_bytes(int64_t n_seq, int loci_per_read) {
    return wave_layout(nullptr, n_seq, locus_capacity(n_seq, loci_per_read), nullptr);
}

// The wavefront form; `scratch` holds wavefront_scratch_bytes(n_seq,
// t.wave_loci_per_read) bytes, d_err is the batch's error word.  Returns
// the number of kernel launches.
int launch_seed_wavefront(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out, int max_len,
                          const ma_tuning& t, int stage2_blocks, void* scratch, int sm_count, int* d_err,
                          unsigned long long* d_tally, WaveTimer* timer, cudaStream_t st) {
    Wave w;
    wave_layout(static_cast<char*>(scratch), R.n_seq, locus_capacity(R.n_seq, t.wave_loci_per_read), &w);
    // an accepted candidate has nm <= its read's budget <= max(2, max_diff)
    // (and <= 512): the round keys give the rest to the locus index
    const int max_nm = P.max_diff < 2 ? 2 : (P.max_diff > 512 ? 512 : P.max_diff);
    int nm_bits = 1;
    while ((1 << nm_bits) <= max_nm) ++nm_bits;
    w.idx_bits = 64 - ORD_SHIFT - nm_bits < 31 ? 64 - ORD_SHIFT - nm_bits : 31;
    if (w.locus_cap > (1ull << w.idx_bits) - 1) w.locus_cap = (1ull << w.idx_bits) - 1;
    const int w0 = t.stage1_endpoints > 0 ? t.stage1_endpoints : 1;
    const int wn = t.wave_endpoints > 0 ? t.wave_endpoints : 1;
    int launches = 0;
    const int mr = t.wave_max_rounds, gr = t.wave_growth;
    const bool refill = t.seed_kernel == 3;                         // lane-refill search
    const bool staged = t.seed_kernel == 3 || t.seed_kernel == 4;  // staged-shift eval
    if (d_tally)
        launches = launch_rounds<true, 1, 1, 1>(ix, R, P, out, w, max_len, w0, wn, mr, gr, refill, staged, sm_count, d_err, d_tally, timer, st);
    else if (t.reg_level == 1)
        launches = launch_rounds<false, 5, 4, 4>(ix, R, P, out, w, max_len, w0, wn, mr, gr, refill, staged, sm_count, d_err, nullptr, timer, st);
    else if (t.reg_level == 2)
        launches = launch_rounds<false, 6, 5, 5>(ix, R, P, out, w, max_len, w0, wn, mr, gr, refill, staged, sm_count, d_err, nullptr, timer, st);
    else
        launches = launch_rounds<false, 1, 1, 1>(ix, R, P, out, w, max_len, w0, wn, mr, gr, refill, staged, sm_count, d_err, nullptr, timer, st);
    // reads that overflowed the locus list or outlived the rounds (their
    // tallies in the second half of the tally array, their time between
    // the timer's stage-2 events)
    if (timer) cudaEventRecord(timer->s2[0], st);
    launches += launch_stage2_pending(ix, R, P, out, w.best_key, w.memo, w.memo_n, w.resume, w.pending,
                                      w.counters + C_HANDOFF, stage2_blocks, t.reg_level, 32,
                                      d_tally ? d_tally + TALLY_N : nullptr, st);
    if (timer) cudaEventRecord(timer->s2[1], st);
    return launches;
}

}  // namespace ma
