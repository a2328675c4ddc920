// capi.cu - the C ABI of libmojoalign_b200 (declared in
// include/mojoalign_b200.h).  Every entry point catches ma::Error and
// returns its code; the message is kept on the context (or thread-locally
// for calls without one).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "bam_pack.h"
#include "bgzf_inflate.cuh"
#include "bgzf.h"
#include "fastq_parse.h"
#include "sam_emit.h"
#include "sort_markdup.h"
#include "ma_device.cuh"
#include "ma_internal.h"

namespace ma {
int launch_pack(const uint8_t* d_bases, const uint32_t* d_lens, int64_t n_seq, int64_t n1, int max_len, int words,
                int bs_r1, int bs_r2, uint64_t* d_packed, int* d_err, cudaStream_t st);
int launch_seed_extend(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out,
                       unsigned long long* d_tally, int level, cudaStream_t st);
double run_gather_bench(uint64_t buffer_bytes, int line_bytes, uint64_t n_loads, int sm_count, cudaStream_t st);
size_t two_stage_scratch_bytes(int64_t n_seq);
size_t wavefront_scratch_bytes(int64_t n_seq, int loci_per_read);
int launch_seed_wavefront(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out, int max_len,
                          const ma_tuning& t, int stage2_blocks, void* scratch, int sm_count, int* d_err,
                          unsigned long long* d_tally, WaveTimer* timer, cudaStream_t st);
int launch_seed_two_stage(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out,
                          int stage1_endpoints, int stage1_max_rows, int stage2_blocks, int level,
                          int first_wave, void* scratch, unsigned long long* d_tally, cudaEvent_t mid,
                          cudaStream_t st);
int stage2_blocks_per_sm(int level, bool counting);
int launch_rescue(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out, int64_t n_pairs,
                  cudaStream_t st);
}  // namespace ma

extern "C" int ma_synth_reference_impl(const char*, uint64_t, int, double, double, uint64_t, char*, size_t);
extern "C" int ma_synth_reference_model_impl(const char*, uint64_t, int, double, double, uint64_t,
                                             const ma_repeat_model*, char*, size_t);
extern "C" int ma_synth_reads_impl(const char*, const ma_read_model*, uint32_t, int, uint32_t, uint64_t, uint8_t*,
                                   uint32_t*, uint64_t*, uint8_t*, char*, size_t);

using namespace ma;

namespace {

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// A grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    void ensure(size_t n) {
        if (n <= cap) return;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        ck(cudaMalloc(&p, n ? n : 1), "cudaMalloc scratch");
        cap = n;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

// A grow-only page-locked host buffer (staging of host arrays that are
// not page-locked, so that their copies can run asynchronously).
struct HostBuf {
    void* p = nullptr;
    size_t cap = 0;
    void ensure(size_t n) {
        if (n <= cap) return;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        ck(cudaHostAlloc(&p, n ? n : 1, cudaHostAllocDefault), "cudaHostAlloc staging");
        cap = n;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

// Whether a host pointer is ordinary pageable memory (a copy from or to it
// is synchronous for the calling thread).
bool pageable(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

}  // namespace

struct ma_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int last_launches = 0;
    int profiling = 0;           // bit 0: per-kernel events, bit 1: traffic tally
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // pack | stage 1 | stage 2 | rescue
    float kernel_ms[4] = {0, 0, 0, 0};  // pack, seed (both stages), rescue, stage 1 alone
    WaveTimer wave_timer;              // per-round events of the wavefront form
    float wave_ms[5] = {0, 0, 0, 0, 0};  // search, eval, finalize (summed over rounds), rounds timed, stage 2
    uint64_t traffic[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    uint64_t traffic_stage2[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // the part of the wavefront's stage 2
    bool rescue_ran = false;
    DevBuf tally;
    // two-slot pipeline of ma_map_batch: H2D of chunk k+1 on copy_stream
    // and D2H of chunk k-1 on d2h_stream while chunk k computes on `stream`
    cudaStream_t copy_stream = nullptr, d2h_stream = nullptr;
    static constexpr int NSLOT = 3;  // chunks whose host copies are in flight
    cudaEvent_t h2d_done[NSLOT] = {}, slot_free[NSLOT] = {}, comp_done[NSLOT] = {};
    struct Slot {
        DevBuf bases, lens, out[12];
        HostBuf h_lens, h_out[12];  // staging of pageable caller arrays
    } slot[NSLOT];
    struct Lane {  // a second compute stream with its own work buffers
        DevBuf packed, seed_scratch;
        cudaStream_t stream = nullptr;
    } lane[3];
    cudaEvent_t err_reset = nullptr;
    ma_pipeline pipeline{0, 50, 0, 3};
    ma_tuning tuning{2, 1, 0, 2, 1, 1, 8, 4, 0, 1};
    int sm_count = 0;
    DevBuf seed_scratch;
    DevBuf bases, lens, packed, err_flag;
    DevBuf o_rid, o_pos, o_mapq, o_flag, o_sl, o_sr, o_nm;
    DevBuf d_uk, d_ul, d_us, d_e, d_score;
    // BAM packing: inputs of the host-buffer form, records, metadata,
    // layout scratch and status
    DevBuf bam_in, bam_arena, bam_out, bam_meta, bam_scratch, bam_status;
    // sort / markdup / gather of a tile
    DevBuf sort_in, sort_out, sort_scratch, gather_in, gather_chunks, gather_out, gather_scratch;
    // FASTQ split
    DevBuf fq_in, fq_out, fq_scratch, fq_newlines;
    // BGZF
    DevBuf bgzf_in, bgzf_out, bgzf_scratch;
    // SAM text of a batch
    DevBuf sam_in, sam_arena, sam_out, sam_scratch, sam_status;
    // BGZF inflate (host form)
    DevBuf inf_in, inf_cols, inf_out;
    // CUDA graphs of the device mapping call (ma_ctx_set_graphs): the launch
    // sequences of the last few argument sets, each captured when its
    // arguments come a second time and replayed while they repeat
    struct GraphEntry {
        unsigned char key[512] = {};
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        int launches = 0;
        uint64_t used = 0;
    };
    static constexpr size_t MAX_GRAPHS = 8;
    bool graphs = false;
    std::vector<GraphEntry> graph_cache;
    uint64_t graph_clock = 0;
};

struct ma_index {
    ma_ctx* ctx = nullptr;
    DevIndex dix{};
    DeviceIndexBuffers bufs;
    ma_index_info info{};
    std::vector<Contig> contigs;
};

namespace ma {
// Device view and device ordinal of a resident index, for entry points
// defined in other translation units.
const DevIndex* index_device_view(const ma_index* idx, int* device) {
    if (!idx || !idx->ctx) return nullptr;
    if (device) *device = idx->ctx->device;
    return &idx->dix;
}

// Device ordinal, SM count and kernel tuning of a context.
void ctx_launch_config(const ma_ctx* ctx, int* device, int* sm_count, ma_tuning* tuning) {
    *device = ctx->device;
    *sm_count = ctx->sm_count;
    *tuning = ctx->tuning;
}
}  // namespace ma

namespace {
thread_local std::string t_err;
}  // namespace

namespace ma {
// Message returned by ma_last_error(NULL) on this thread.
void set_thread_error(const std::string& msg) { t_err = msg; }
}  // namespace ma

namespace {

template <typename F>
int guarded(ma_ctx* ctx, F&& f) {
    try {
        f();
        if (ctx) ctx->err.clear();
        return MA_OK;
    } catch (const Error& e) {
        if (ctx) ctx->err = e.what();
        t_err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        if (ctx) ctx->err = "host out of memory";
        t_err = "host out of memory";
        return MA_ERR_NOMEM;
    } catch (const std::exception& e) {
        if (ctx) ctx->err = e.what();
        t_err = e.what();
        return MA_ERR_INTERNAL;
    }
}

void use_device(ma_ctx* ctx) { ck(cudaSetDevice(ctx->device), "cudaSetDevice"); }

void validate_params(const ma_params* p) {
    if (!p) fail(MA_ERR_ARG, "params must not be NULL");
    if (p->seed_len < 1 || p->seed_len > MAX_READ_LEN) fail(MA_ERR_ARG, "seed_len must be in 1..1024");
    if (p->seed_stride < 1) fail(MA_ERR_ARG, "seed_stride must be >= 1");
    if (p->max_occ < 1) fail(MA_ERR_ARG, "max_occ must be >= 1");
}

DevParams to_dev(const ma_params* p) {
    DevParams d;
    d.seed_len = p->seed_len;
    d.seed_stride = p->seed_stride;
    d.max_occ = p->max_occ;
    d.max_diff = p->max_diff;
    d.max_soft = p->max_soft;
    d.max_adj = p->max_adj;
    d.rescue_win = p->rescue_win;
    return d;
}

// Enqueues pack -> seed/extend -> rescue for device-resident inputs, with
// `packed` and `seed_scratch` as work buffers (the context's own by
// default).
void enqueue_map(ma_ctx* ctx, const ma_index* idx, const uint8_t* d_bases, const uint32_t* d_lens, uint32_t n1,
                 int paired, uint32_t max_len, int bs_r1, int bs_r2, const ma_params* p, const DevOut& out,
                 cudaStream_t st, bool reset_err = true, DevBuf* packed = nullptr, DevBuf* seed_scratch = nullptr) {
    if (!packed) packed = &ctx->packed;
    if (!seed_scratch) seed_scratch = &ctx->seed_scratch;
    const int64_t n_seq = paired ? 2 * static_cast<int64_t>(n1) : n1;
    const int words = static_cast<int>((max_len + 31) / 32);
    packed->ensure(static_cast<size_t>(n_seq) * 4 * words * 8);
    ctx->err_flag.ensure(sizeof(int));
    if (reset_err) ck(cudaMemsetAsync(ctx->err_flag.p, 0, sizeof(int), st), "memset");
    int launches = 0;
    const bool timed = ctx->profiling & 1;
    unsigned long long* d_tally = nullptr;
    if (ctx->profiling & 2) {
        ctx->tally.ensure(24 * sizeof(unsigned long long));  // wavefront rounds, then stage 2
        d_tally = ctx->tally.as<unsigned long long>();
        ck(cudaMemsetAsync(d_tally, 0, 24 * sizeof(unsigned long long), st), "memset");
    }
    if (timed) ck(cudaEventRecord(ctx->ev[0], st), "event");
    launches += launch_pack(d_bases, d_lens, n_seq, n1, static_cast<int>(max_len), words, bs_r1, bs_r2,
                            packed->as<uint64_t>(), ctx->err_flag.as<int>(), st);
    if (timed) ck(cudaEventRecord(ctx->ev[1], st), "event");
    DevReads R{packed->as<uint64_t>(), d_lens, words, n_seq};
    DevParams P = to_dev(p);
    const int level = ctx->tuning.reg_level;
    if (ctx->tuning.seed_kernel == 0) {
        launches += launch_seed_extend(idx->dix, R, P, out, d_tally, level, st);
    } else if (ctx->tuning.seed_kernel >= 2) {
        seed_scratch->ensure(wavefront_scratch_bytes(n_seq, ctx->tuning.wave_loci_per_read));
        const int bps = ctx->tuning.stage2_blocks_per_sm > 0 ? ctx->tuning.stage2_blocks_per_sm
                                                             : stage2_blocks_per_sm(level, d_tally != nullptr);
        launches += launch_seed_wavefront(idx->dix, R, P, out, static_cast<int>(max_len), ctx->tuning,
                                          bps * ctx->sm_count, seed_scratch->p, ctx->sm_count,
                                          ctx->err_flag.as<int>(), d_tally, timed ? &ctx->wave_timer : nullptr, st);
    } else {
        seed_scratch->ensure(two_stage_scratch_bytes(n_seq));
        const int bps = ctx->tuning.stage2_blocks_per_sm > 0 ? ctx->tuning.stage2_blocks_per_sm
                                                             : stage2_blocks_per_sm(level, d_tally != nullptr);
        launches += launch_seed_two_stage(idx->dix, R, P, out, ctx->tuning.stage1_endpoints,
                                          ctx->tuning.stage1_max_rows, bps * ctx->sm_count, level,
                                          ctx->tuning.stage2_first_wave, seed_scratch->p, d_tally,
                                          timed ? ctx->ev[4] : nullptr, st);
    }
    if (timed) ck(cudaEventRecord(ctx->ev[2], st), "event");
    ctx->rescue_ran = paired && p->rescue_win > 0;
    if (ctx->rescue_ran) launches += launch_rescue(idx->dix, R, P, out, n1, st);
    if (timed) ck(cudaEventRecord(ctx->ev[3], st), "event");
    ck(cudaGetLastError(), "kernel launch");
    ctx->last_launches = launches;
}

void drop_graphs(ma_ctx* ctx) {
    for (auto& g : ctx->graph_cache) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    ctx->graph_cache.clear();
}

// enqueue_map through CUDA graphs.  Everything the launch sequence depends
// on is in the key: the arguments, the stream, the tuning and the work
// buffers (grow-only, so their addresses change only when they grow).  The
// first call with a key runs uncaptured (it may allocate); the second
// captures the sequence and launches the graph; later ones launch it.  The
// least recently used of MAX_GRAPHS keys is dropped for a new one.
void enqueue_map_graph(ma_ctx* ctx, const ma_index* idx, const uint8_t* d_bases, const uint32_t* d_lens,
                       uint32_t n1, int paired, uint32_t max_len, int bs_r1, int bs_r2, const ma_params* p,
                       const DevOut& out, cudaStream_t st) {
    struct Key {
        const void* ptrs[20];
        int64_t vals[24];
    } key;
    static_assert(sizeof(Key) <= sizeof(ma_ctx::GraphEntry::key), "graph key");
    auto make_key = [&]() {
        std::memset(&key, 0, sizeof key);
        const void* ptrs[20] = {idx, d_bases, d_lens, out.rid, out.pos, out.mapq, out.flag, out.sl, out.sr, out.nm,
                                out.uk, out.ul, out.us, out.e, out.score, st, ctx->packed.p, ctx->seed_scratch.p,
                                ctx->err_flag.p, nullptr};
        std::memcpy(key.ptrs, ptrs, sizeof ptrs);
        const int64_t vals[24] = {n1, paired, max_len, bs_r1, bs_r2, p->seed_len, p->seed_stride, p->max_occ,
                                  p->max_diff, p->max_soft, p->max_adj, p->rescue_win, ctx->tuning.seed_kernel,
                                  ctx->tuning.stage1_endpoints, ctx->tuning.stage2_blocks_per_sm,
                                  ctx->tuning.reg_level, ctx->tuning.stage1_max_rows, ctx->tuning.stage2_first_wave,
                                  ctx->tuning.wave_endpoints, ctx->tuning.wave_loci_per_read,
                                  ctx->tuning.wave_max_rounds, ctx->tuning.wave_growth, 0, 0};
        std::memcpy(key.vals, vals, sizeof vals);
    };
    make_key();
    ma_ctx::GraphEntry* e = nullptr;
    for (auto& g : ctx->graph_cache)
        if (std::memcmp(g.key, &key, sizeof key) == 0) e = &g;
    if (e && e->exec) {
        e->used = ++ctx->graph_clock;
        ck(cudaGraphLaunch(e->exec, st), "cudaGraphLaunch");
        ctx->last_launches = e->launches;
        return;
    }
    if (!e) {
        enqueue_map(ctx, idx, d_bases, d_lens, n1, paired, max_len, bs_r1, bs_r2, p, out, st);
        make_key();  // the work buffers are sized now
        if (ctx->graph_cache.size() >= ma_ctx::MAX_GRAPHS) {
            auto old = std::min_element(ctx->graph_cache.begin(), ctx->graph_cache.end(),
                                        [](const ma_ctx::GraphEntry& a, const ma_ctx::GraphEntry& b) {
                                            return a.used < b.used;
                                        });
            if (old->exec) cudaGraphExecDestroy(old->exec);
            if (old->graph) cudaGraphDestroy(old->graph);
            ctx->graph_cache.erase(old);
        }
        ma_ctx::GraphEntry ne;
        std::memcpy(ne.key, &key, sizeof key);
        ne.used = ++ctx->graph_clock;
        ctx->graph_cache.push_back(ne);
        return;
    }
    ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    try {
        enqueue_map(ctx, idx, d_bases, d_lens, n1, paired, max_len, bs_r1, bs_r2, p, out, st);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    ck(cudaStreamEndCapture(st, &e->graph), "cudaStreamEndCapture");
    ck(cudaGraphInstantiate(&e->exec, e->graph, 0), "cudaGraphInstantiate");
    e->launches = ctx->last_launches;
    e->used = ++ctx->graph_clock;
    ck(cudaGraphLaunch(e->exec, st), "cudaGraphLaunch");
}

void check_err_flag(ma_ctx* ctx, cudaStream_t st) {
    int h = 0;
    ck(cudaMemcpyAsync(&h, ctx->err_flag.p, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H err");
    ck(cudaStreamSynchronize(st), "mapping kernels");
    if (h == 1) fail(MA_ERR_ARG, "a read length exceeds max_len");
    if (h) fail(MA_ERR_INTERNAL, "device error flag " + std::to_string(h));
    if (ctx->profiling & 1) {
        for (int i = 0; i < 3; ++i) ck(cudaEventElapsedTime(&ctx->kernel_ms[i], ctx->ev[i], ctx->ev[i + 1]), "elapsed");
        if (!ctx->rescue_ran) ctx->kernel_ms[2] = 0;
        ctx->kernel_ms[3] = ctx->kernel_ms[1];
        if (ctx->tuning.seed_kernel == 1) ck(cudaEventElapsedTime(&ctx->kernel_ms[3], ctx->ev[1], ctx->ev[4]), "elapsed");
        for (float& v : ctx->wave_ms) v = 0;
        if (ctx->tuning.seed_kernel >= 2) {
            const WaveTimer& w = ctx->wave_timer;
            for (int k = 0; k < w.recorded; ++k) {
                float a = 0, b = 0, c = 0;
                ck(cudaEventElapsedTime(&a, w.e[3 * k], w.e[3 * k + 1]), "elapsed");
                ck(cudaEventElapsedTime(&b, w.e[3 * k + 1], w.e[3 * k + 2]), "elapsed");
                ck(cudaEventElapsedTime(&c, w.e[3 * k + 2], w.e[3 * k + 3]), "elapsed");
                ctx->wave_ms[0] += a;
                ctx->wave_ms[1] += b;
                ctx->wave_ms[2] += c;
            }
            ctx->wave_ms[3] = w.complete ? static_cast<float>(w.recorded) : -static_cast<float>(w.recorded);
            ck(cudaEventElapsedTime(&ctx->wave_ms[4], w.s2[0], w.s2[1]), "elapsed");
        }
    }
    if (ctx->profiling & 2) {
        unsigned long long t[24];
        ck(cudaMemcpy(t, ctx->tally.p, sizeof t, cudaMemcpyDeviceToHost), "D2H tally");
        for (int i = 0; i < 12; ++i) {
            ctx->traffic[i] = t[i] + t[12 + i];
            ctx->traffic_stage2[i] = t[12 + i];
        }
    }
}

}  // namespace

extern "C" {

void ma_params_default(ma_params* p) {
    if (!p) return;
    p->seed_len = 18;
    p->seed_stride = 2;
    p->max_occ = 4096;
    p->max_diff = 12;
    p->max_soft = 20;
    p->max_adj = 8;
    p->rescue_win = 512;
}

const char* ma_last_error(const ma_ctx* ctx) { return ctx ? ctx->err.c_str() : t_err.c_str(); }

int ma_ctx_create(int device_ordinal, ma_ctx** out) {
    if (!out) return MA_ERR_ARG;
    *out = nullptr;
    ma_ctx* ctx = new ma_ctx();
    int rc = guarded(nullptr, [&] {
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess || n == 0) fail(MA_ERR_CUDA, "no CUDA device available");
        if (device_ordinal < 0 || device_ordinal >= n) fail(MA_ERR_ARG, "device ordinal out of range");
        cudaDeviceProp prop;
        ck(cudaGetDeviceProperties(&prop, device_ordinal), "cudaGetDeviceProperties");
        if (prop.major != 10)
            fail(MA_ERR_CUDA, "this library is built for sm_100a (B200); device reports sm_" +
                                  std::to_string(prop.major) + std::to_string(prop.minor));
        ctx->device = device_ordinal;
        ck(cudaSetDevice(device_ordinal), "cudaSetDevice");
        ck(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ctx->sm_count = prop.multiProcessorCount;
    });
    if (rc != MA_OK) {
        delete ctx;
        return rc;
    }
    *out = ctx;
    return MA_OK;
}

void ma_ctx_destroy(ma_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    drop_graphs(ctx);
    for (cudaEvent_t& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : ctx->wave_timer.e)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : ctx->wave_timer.s2)
        if (e) cudaEventDestroy(e);
    ctx->tally.release();
    ctx->seed_scratch.release();
    for (auto& sl : ctx->slot) {
        sl.bases.release();
        sl.lens.release();
        for (DevBuf& b : sl.out) b.release();
        sl.h_lens.release();
        for (HostBuf& b : sl.h_out) b.release();
    }
    for (auto& ln : ctx->lane) {
        ln.packed.release();
        ln.seed_scratch.release();
        if (ln.stream) cudaStreamDestroy(ln.stream);
    }
    if (ctx->err_reset) cudaEventDestroy(ctx->err_reset);
    for (int i = 0; i < ma_ctx::NSLOT; ++i) {
        if (ctx->h2d_done[i]) cudaEventDestroy(ctx->h2d_done[i]);
        if (ctx->slot_free[i]) cudaEventDestroy(ctx->slot_free[i]);
        if (ctx->comp_done[i]) cudaEventDestroy(ctx->comp_done[i]);
    }
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->d2h_stream) cudaStreamDestroy(ctx->d2h_stream);
    for (DevBuf* b : {&ctx->bases, &ctx->lens, &ctx->packed, &ctx->err_flag, &ctx->o_rid, &ctx->o_pos, &ctx->o_mapq,
                      &ctx->o_flag, &ctx->o_sl, &ctx->o_sr, &ctx->o_nm, &ctx->d_uk, &ctx->d_ul, &ctx->d_us,
                      &ctx->d_e, &ctx->d_score, &ctx->bam_in, &ctx->bam_arena, &ctx->bam_out, &ctx->bam_meta,
                      &ctx->bam_scratch, &ctx->bam_status, &ctx->sort_in, &ctx->sort_out, &ctx->sort_scratch,
                      &ctx->gather_in, &ctx->gather_chunks, &ctx->gather_out, &ctx->gather_scratch, &ctx->fq_in,
                      &ctx->fq_out, &ctx->fq_scratch, &ctx->fq_newlines, &ctx->bgzf_in, &ctx->bgzf_out,
                      &ctx->bgzf_scratch})
        b->release();
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int ma_hbm_info(ma_ctx* ctx, uint64_t* free_bytes, uint64_t* total_bytes) {
    if (!ctx || !free_bytes || !total_bytes) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        use_device(ctx);
        size_t f = 0, t = 0;
        ck(cudaMemGetInfo(&f, &t), "cudaMemGetInfo");
        *free_bytes = f;
        *total_bytes = t;
    });
}

int ma_index_build(const char* fasta, const char* out_prefix, int bwameth_c2t, int sa_intv, int device_ordinal) {
    if (!fasta || !out_prefix) {
        t_err = "null path";
        return MA_ERR_ARG;
    }
    return guarded(nullptr, [&] { build_index(fasta, out_prefix, bwameth_c2t != 0, sa_intv, device_ordinal); });
}

int ma_index_build_batched(const char* fasta, const char* out_prefix, int bwameth_c2t, int sa_intv,
                           int device_ordinal, uint64_t batch_suffixes) {
    if (!fasta || !out_prefix) {
        t_err = "null path";
        return MA_ERR_ARG;
    }
    return guarded(nullptr, [&] {
        build_index(fasta, out_prefix, bwameth_c2t != 0, sa_intv, device_ordinal, batch_suffixes);
    });
}

void ma_index_options_default(ma_index_options* o) {
    if (!o) return;
    o->kmer_k = 12;
    o->kmer3_k = 0;
    o->hbm_budget_bytes = 0;
    o->wide_rows = 0;
    o->occ_super_shift = 0;
    o->prep_chunk_rows = 0;
    o->at_k = 0;
    o->at_seed_len = 0;
}

namespace {
LayoutOptions layout_of(const ma_index_options& o) {
    LayoutOptions lo;
    lo.kmer_k = o.kmer_k;
    lo.kmer3_k = o.kmer3_k;
    lo.wide_rows = o.wide_rows != 0;
    lo.occ_super_shift = o.occ_super_shift ? o.occ_super_shift : OCC_SUPER_SHIFT;
    lo.prep_chunk_rows = o.prep_chunk_rows;
    lo.at_k = o.at_k;
    lo.at_seed_len = o.at_seed_len;
    return lo;
}
}  // namespace

int ma_index_probe(const char* prefix, int kmer_k, int kmer3_k, ma_index_info* out) {
    if (!prefix || !out) {
        t_err = "null argument";
        return MA_ERR_ARG;
    }
    return guarded(nullptr, [&] {
        if (kmer_k < 0 || kmer_k > 14 || kmer3_k < 0 || kmer3_k > 20) fail(MA_ERR_ARG, "bad k-mer table sizes");
        BwaIndexHost h = load_bwa_index(prefix);
        ma_index_info I{};
        I.seq_len = h.seq_len;
        I.l_pac = h.l_pac;
        I.primary = h.primary;
        for (int c = 0; c < 5; ++c) I.L2[c] = h.L2[c];
        I.sa_intv = h.sa_intv;
        I.n_sa = h.n_sa;
        I.n_contigs = static_cast<int64_t>(h.contigs.size());
        uint64_t p0 = h.seq_len;
        for (uint64_t v : h.sa) p0 = v < p0 ? v : p0;
        I.sa_reject_below = p0;
        I.kmer_k = kmer_k;
        I.kmer3_k = kmer3_k;
        LayoutOptions lo;
        lo.kmer_k = kmer_k;
        lo.kmer3_k = kmer3_k;
        I.device_bytes = device_index_bytes(h, lo) + device_index_staging_bytes(h, lo);
        *out = I;
    });
}

int ma_index_open(ma_ctx* ctx, const char* prefix, const ma_index_options* opt, ma_index** out) {
    if (!ctx || !prefix || !out) return MA_ERR_ARG;
    *out = nullptr;
    ma_index_options o;
    ma_index_options_default(&o);
    if (opt) o = *opt;
    ma_index* idx = new ma_index();
    int rc = guarded(ctx, [&] {
        use_device(ctx);
        BwaIndexHost h = load_bwa_index(prefix);
        const LayoutOptions lo = layout_of(o);
        const uint64_t need = device_index_bytes(h, lo);
        size_t f = 0, t = 0;
        ck(cudaMemGetInfo(&f, &t), "cudaMemGetInfo");
        // fail-closed admission like gpu_mem.require_index_capacity: the
        // resident index plus the preparation passes' staging must fit
        const uint64_t staging = device_index_staging_bytes(h, lo);
        const uint64_t budget = o.hbm_budget_bytes ? std::min<uint64_t>(o.hbm_budget_bytes, f) : f;
        if (need + staging > budget)
            fail(MA_ERR_NOMEM, "index needs " + std::to_string((need + staging) >> 20) + " MiB of HBM, budget " +
                                   std::to_string(budget >> 20) + " MiB");
        uint64_t p0 = 0;
        idx->dix = build_device_index(h, lo, ctx->stream, idx->bufs, &p0);
        idx->ctx = ctx;
        idx->contigs = h.contigs;
        ma_index_info& I = idx->info;
        I.seq_len = h.seq_len;
        I.l_pac = h.l_pac;
        I.primary = h.primary;
        for (int c = 0; c < 5; ++c) I.L2[c] = h.L2[c];
        I.sa_intv = h.sa_intv;
        I.n_sa = h.n_sa;
        I.n_contigs = static_cast<int64_t>(h.contigs.size());
        I.sa_reject_below = p0;
        I.kmer_k = o.kmer_k;
        I.kmer3_k = o.kmer3_k;
        I.device_bytes = idx->bufs.bytes;
    });
    if (rc != MA_OK) {
        free_device_index(idx->bufs);
        delete idx;
        return rc;
    }
    *out = idx;
    return MA_OK;
}

void ma_index_close(ma_index* idx) {
    if (!idx) return;
    if (idx->ctx) cudaSetDevice(idx->ctx->device);
    free_device_index(idx->bufs);
    delete idx;
}

int ma_index_get_info(const ma_index* idx, ma_index_info* out) {
    if (!idx || !out) return MA_ERR_ARG;
    *out = idx->info;
    return MA_OK;
}

int ma_index_contig(const ma_index* idx, int64_t i, const char** name, uint64_t* offset, uint64_t* length) {
    if (!idx || i < 0 || i >= static_cast<int64_t>(idx->contigs.size())) return MA_ERR_ARG;
    if (name) *name = idx->contigs[static_cast<size_t>(i)].name.c_str();
    if (offset) *offset = idx->contigs[static_cast<size_t>(i)].offset;
    if (length) *length = idx->contigs[static_cast<size_t>(i)].len;
    return MA_OK;
}

int ma_map_batch(ma_ctx* ctx, const ma_index* idx, const uint8_t* bases, const uint32_t* lens, uint32_t n1,
                 int paired, uint32_t max_len, int bs_r1, int bs_r2, const ma_params* p, ma_hits* out,
                 ma_debug* dbg) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        if (!idx || !out || (n1 && (!bases || !lens))) fail(MA_ERR_ARG, "null argument");
        if (idx->ctx != ctx) fail(MA_ERR_ARG, "index belongs to another context");
        validate_params(p);
        if (max_len < 1 || max_len > MAX_READ_LEN) fail(MA_ERR_ARG, "max_len must be in 1..1024");
        if (bs_r1 < 0 || bs_r1 > 2 || bs_r2 < 0 || bs_r2 > 2) fail(MA_ERR_ARG, "bad bisulfite mode");
        ctx->last_launches = 0;
        if (n1 == 0) return;
        const int64_t n_seq = paired ? 2 * static_cast<int64_t>(n1) : n1;
        for (int64_t i = 0; i < n_seq; ++i)
            if (lens[i] > max_len) fail(MA_ERR_ARG, "read " + std::to_string(i) + " longer than max_len");
        if (!out->rid || !out->pos || !out->mapq || !out->flag || !out->sl || !out->sr || !out->nm)
            fail(MA_ERR_ARG, "null output array");
        use_device(ctx);
        cudaStream_t st = ctx->stream;
        if (!ctx->copy_stream) {
            ck(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
            ck(cudaStreamCreateWithFlags(&ctx->d2h_stream, cudaStreamNonBlocking), "cudaStreamCreate");
            for (int i = 0; i < ma_ctx::NSLOT; ++i) {
                ck(cudaEventCreateWithFlags(&ctx->h2d_done[i], cudaEventDisableTiming), "cudaEventCreate");
                ck(cudaEventCreateWithFlags(&ctx->slot_free[i], cudaEventDisableTiming), "cudaEventCreate");
                ck(cudaEventCreateWithFlags(&ctx->comp_done[i], cudaEventDisableTiming), "cudaEventCreate");
            }
            for (auto& ln : ctx->lane)
                ck(cudaStreamCreateWithFlags(&ln.stream, cudaStreamNonBlocking), "cudaStreamCreate");
            ck(cudaEventCreateWithFlags(&ctx->err_reset, cudaEventDisableTiming), "cudaEventCreate");
        }
        const bool want_dbg = dbg && (dbg->uk || dbg->ul || dbg->us || dbg->e || dbg->score);
        // Pipeline over chunks of pairs (pairs never split: rescue reads both
        // mates).  Chunk k's R1 rows and R2 rows are copied into one slot as
        // a batch of its own while chunk k-1 computes, and chunk k-1's results
        // go back into the caller's arrays (at the pairs' positions) while
        // chunk k computes: three slots, three or four streams (ma_pipeline).
        // Chunks grow from a small first one (the pipeline fills quickly,
        // while large later chunks keep the kernels' per-call overhead
        // small).  Caller arrays that are not page-locked (lengths,
        // outputs) go through page-locked staging buffers of the slot: a
        // copy from or to pageable memory would hold the calling thread
        // until the chunk's kernels end and serialise the pipeline.  A
        // slot's staged outputs are copied out when the slot is reused and
        // after the last chunk.
        const ma_pipeline& pl = ctx->pipeline;
        const uint32_t first = std::min<uint32_t>(
            n1, pl.first_chunk_pairs ? pl.first_chunk_pairs : std::max<uint32_t>(65536u, n1 / 64));
        const uint32_t cap = std::max<uint32_t>(
            first, pl.max_chunk_pairs ? pl.max_chunk_pairs
                                      : std::min<uint32_t>(2000000u, std::max<uint32_t>(131072u, n1 / 16)));
        const int lanes = static_cast<int>(pl.compute_streams);
        const bool two = lanes > 1;
        const int mates = paired ? 2 : 1;
        void* host_out[12] = {out->rid, out->pos, out->mapq, out->flag, out->sl, out->sr, out->nm,
                              want_dbg ? dbg->uk : nullptr, want_dbg ? dbg->ul : nullptr,
                              want_dbg ? dbg->us : nullptr, want_dbg ? dbg->e : nullptr,
                              want_dbg ? dbg->score : nullptr};
        const size_t width[12] = {4, 4, 4, 4, 4, 4, 4, 8, 8, 4, 4, 4};
        const bool stage_lens = pageable(lens);
        bool stage_out[12];
        bool any_stage = stage_lens;
        for (int f = 0; f < 12; ++f) {
            stage_out[f] = host_out[f] && pageable(host_out[f]);
            any_stage = any_stage || stage_out[f];
        }
        int k = 0;
        float acc_ms[4] = {0, 0, 0, 0};
        // every slot sized for the largest chunk before any copy starts
        // (growing a buffer later would free memory still in use)
        for (auto& sl : ctx->slot) {
            const int64_t cs = static_cast<int64_t>(std::min(cap, n1)) * mates;
            sl.bases.ensure(static_cast<size_t>(cs) * max_len);
            sl.lens.ensure(cs * 4);
            for (int f = 0; f < 12; ++f) sl.out[f].ensure(cs * width[f]);
            if (stage_lens) sl.h_lens.ensure(cs * 4);
            for (int f = 0; f < 12; ++f)
                if (stage_out[f]) sl.h_out[f].ensure(cs * width[f]);
        }
        // the chunk (first pair, pairs) whose staged outputs slot i holds
        uint32_t pend_a[ma_ctx::NSLOT], pend_c[ma_ctx::NSLOT];
        bool pend[ma_ctx::NSLOT] = {};
        auto drain = [&](int si) {  // the slot's previous chunk done: staged outputs out
            if (!pend[si]) return;
            ck(cudaEventSynchronize(ctx->slot_free[si]), "cudaEventSynchronize");
            pend[si] = false;
            const ma_ctx::Slot& sl = ctx->slot[si];
            for (int f = 0; f < 12; ++f) {
                if (!stage_out[f]) continue;
                for (int m = 0; m < mates; ++m) {
                    const size_t row0 = static_cast<size_t>(m) * n1 + pend_a[si];
                    std::memcpy(static_cast<char*>(host_out[f]) + row0 * width[f],
                                sl.h_out[f].as<char>() + static_cast<size_t>(m) * pend_c[si] * width[f],
                                pend_c[si] * width[f]);
                }
            }
        };
        // one error word for the call, cleared before any chunk computes
        ctx->err_flag.ensure(sizeof(int));
        ck(cudaMemsetAsync(ctx->err_flag.p, 0, sizeof(int), st), "memset");
        if (two) {
            ck(cudaEventRecord(ctx->err_reset, st), "cudaEventRecord");
            for (auto& ln : ctx->lane) ck(cudaStreamWaitEvent(ln.stream, ctx->err_reset, 0), "cudaStreamWaitEvent");
        }
        uint32_t chunk = first;
        auto grow = [&](uint32_t x) {
            const uint64_t g = static_cast<uint64_t>(x) + static_cast<uint64_t>(x) * pl.growth_percent / 100;
            return static_cast<uint32_t>(std::min<uint64_t>(cap, std::max<uint64_t>(g, 1)));
        };
        for (uint32_t a = 0, c = 0; a < n1; a += c, ++k, chunk = grow(chunk)) {
            c = std::min(chunk, n1 - a);
            const int si = k % ma_ctx::NSLOT;
            ma_ctx::Slot& sl = ctx->slot[si];
            ma_ctx::Lane& ln = ctx->lane[k % (lanes > 1 ? lanes : 1)];
            cudaStream_t cst = two ? ln.stream : st;
            // copy: wait until the slot's previous chunk has been read back
            // (on the host too when its staging buffers are reused)
            drain(si);
            ck(cudaStreamWaitEvent(ctx->copy_stream, ctx->slot_free[si], 0), "cudaStreamWaitEvent");
            for (int m = 0; m < mates; ++m) {
                const size_t row0 = static_cast<size_t>(m) * n1 + a;
                ck(cudaMemcpyAsync(sl.bases.as<uint8_t>() + static_cast<size_t>(m) * c * max_len,
                                   bases + row0 * max_len, static_cast<size_t>(c) * max_len, cudaMemcpyHostToDevice,
                                   ctx->copy_stream), "H2D bases");
                const uint32_t* lsrc = lens + row0;
                if (stage_lens) {
                    uint32_t* h = sl.h_lens.as<uint32_t>() + static_cast<size_t>(m) * c;
                    std::memcpy(h, lsrc, c * 4);
                    lsrc = h;
                }
                ck(cudaMemcpyAsync(sl.lens.as<uint32_t>() + static_cast<size_t>(m) * c, lsrc, c * 4,
                                   cudaMemcpyHostToDevice, ctx->copy_stream), "H2D lens");
            }
            ck(cudaEventRecord(ctx->h2d_done[si], ctx->copy_stream), "cudaEventRecord");
            // compute the chunk, then read it back on the compute stream
            ck(cudaStreamWaitEvent(cst, ctx->h2d_done[si], 0), "cudaStreamWaitEvent");
            DevOut o{sl.out[0].as<int32_t>(), sl.out[1].as<uint32_t>(), sl.out[2].as<uint32_t>(),
                     sl.out[3].as<int32_t>(), sl.out[4].as<uint32_t>(), sl.out[5].as<uint32_t>(),
                     sl.out[6].as<uint32_t>(), nullptr, nullptr, nullptr, nullptr, nullptr};
            if (want_dbg) {
                o.uk = sl.out[7].as<uint64_t>();
                o.ul = sl.out[8].as<uint64_t>();
                o.us = sl.out[9].as<int32_t>();
                o.e = sl.out[10].as<int32_t>();
                o.score = sl.out[11].as<int32_t>();
            }
            enqueue_map(ctx, idx, sl.bases.as<uint8_t>(), sl.lens.as<uint32_t>(), c, paired, max_len, bs_r1, bs_r2,
                        p, o, cst, false, two ? &ln.packed : nullptr, two ? &ln.seed_scratch : nullptr);
            if (ctx->profiling & 1) {
                // profiling runs give up the overlap to time every chunk
                ck(cudaStreamSynchronize(cst), "chunk");
                float ms[4] = {0, 0, 0, 0};
                for (int i = 0; i < 3; ++i) ck(cudaEventElapsedTime(&ms[i], ctx->ev[i], ctx->ev[i + 1]), "elapsed");
                if (!ctx->rescue_ran) ms[2] = 0;
                ms[3] = ms[1];
                if (ctx->tuning.seed_kernel == 1) ck(cudaEventElapsedTime(&ms[3], ctx->ev[1], ctx->ev[4]), "elapsed");
                for (int i = 0; i < 4; ++i) acc_ms[i] += ms[i];
            }
            ck(cudaEventRecord(ctx->comp_done[si], cst), "cudaEventRecord");
            ck(cudaStreamWaitEvent(ctx->d2h_stream, ctx->comp_done[si], 0), "cudaStreamWaitEvent");
            for (int f = 0; f < 12; ++f) {
                if (!host_out[f]) continue;
                if (stage_out[f]) {  // one copy of the chunk into the staging buffer
                    ck(cudaMemcpyAsync(sl.h_out[f].p, sl.out[f].p, static_cast<size_t>(mates) * c * width[f],
                                       cudaMemcpyDeviceToHost, ctx->d2h_stream), "D2H");
                    continue;
                }
                for (int m = 0; m < mates; ++m) {
                    const size_t row0 = static_cast<size_t>(m) * n1 + a;
                    ck(cudaMemcpyAsync(static_cast<char*>(host_out[f]) + row0 * width[f],
                                       sl.out[f].as<char>() + static_cast<size_t>(m) * c * width[f], c * width[f],
                                       cudaMemcpyDeviceToHost, ctx->d2h_stream), "D2H");
                }
            }
            ck(cudaEventRecord(ctx->slot_free[si], ctx->d2h_stream), "cudaEventRecord");
            pend[si] = any_stage;
            pend_a[si] = a;
            pend_c[si] = c;
        }
        // the error word after the last copies back
        ck(cudaStreamWaitEvent(st, ctx->slot_free[(k - 1) % ma_ctx::NSLOT], 0), "cudaStreamWaitEvent");
        check_err_flag(ctx, st);
        for (int i = 0; i < ma_ctx::NSLOT; ++i) drain(i);
        if (ctx->profiling & 1)
            for (int i = 0; i < 4; ++i) ctx->kernel_ms[i] = acc_ms[i];
    });
}

int ma_map_batch_device(ma_ctx* ctx, const ma_index* idx, const uint8_t* d_bases, const uint32_t* d_lens,
                        uint32_t n1, int paired, uint32_t max_len, int bs_r1, int bs_r2, const ma_params* p,
                        ma_hits* d_out, ma_debug* d_dbg, void* stream) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        if (!idx || !d_out || (n1 && (!d_bases || !d_lens))) fail(MA_ERR_ARG, "null argument");
        if (idx->ctx != ctx) fail(MA_ERR_ARG, "index belongs to another context");
        validate_params(p);
        if (max_len < 1 || max_len > MAX_READ_LEN) fail(MA_ERR_ARG, "max_len must be in 1..1024");
        if (bs_r1 < 0 || bs_r1 > 2 || bs_r2 < 0 || bs_r2 > 2) fail(MA_ERR_ARG, "bad bisulfite mode");
        ctx->last_launches = 0;
        if (n1 == 0) return;
        use_device(ctx);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
        DevOut o{d_out->rid, d_out->pos, d_out->mapq, d_out->flag, d_out->sl, d_out->sr, d_out->nm,
                 nullptr, nullptr, nullptr, nullptr, nullptr};
        if (d_dbg) {
            if (!d_dbg->uk || !d_dbg->ul || !d_dbg->us || !d_dbg->e || !d_dbg->score)
                fail(MA_ERR_ARG, "device debug outputs must be all set or NULL");
            o.uk = d_dbg->uk;
            o.ul = d_dbg->ul;
            o.us = d_dbg->us;
            o.e = d_dbg->e;
            o.score = d_dbg->score;
        }
        if (ctx->graphs && ctx->profiling == 0) enqueue_map_graph(ctx, idx, d_bases, d_lens, n1, paired, max_len,
                                                                 bs_r1, bs_r2, p, o, st);
        else enqueue_map(ctx, idx, d_bases, d_lens, n1, paired, max_len, bs_r1, bs_r2, p, o, st);
        check_err_flag(ctx, st);
    });
}

int ma_ctx_set_graphs(ma_ctx* ctx, int enable) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        use_device(ctx);
        drop_graphs(ctx);
        ctx->graphs = enable != 0;
    });
}

namespace {

// Checks shared by both BAM entry points; returns the record count.
uint64_t bam_records_checked(const ma_hits* hits, uint32_t n1, int paired, const ma_fastq_arena* arena,
                             const int32_t* rid_to_tid, int32_t n_tid, const uint8_t* rg, uint32_t rg_n,
                             const void* bam, uint64_t bam_cap, const ma_bam_meta* meta, const ma_bam_tile* tile) {
    if (!hits || !arena || !meta || !tile) fail(MA_ERR_ARG, "null argument");
    const uint64_t n_rec = paired ? 2ull * n1 : n1;
    if (n_rec == 0) return 0;
    if (!hits->rid || !hits->pos || !hits->mapq || !hits->flag || !hits->sl || !hits->sr || !hits->nm)
        fail(MA_ERR_ARG, "null mapping output");
    if (!arena->name_off || !arena->name_len || !arena->orig_off || !arena->orig_len ||
        (arena->qual_off && !arena->qual_len) || (arena->data_bytes && !arena->data))
        fail(MA_ERR_ARG, "null arena array");
    if (!meta->coord || !meta->dhi || !meta->dlo || !meta->rec || !meta->len || !meta->score || !meta->pair)
        fail(MA_ERR_ARG, "null metadata array");
    if (n_tid < 0 || (n_tid && !rid_to_tid) || (rg_n && !rg) || (bam_cap && !bam))
        fail(MA_ERR_ARG, "null argument");
    // _emit_bam_from_batch raises when a record would land at or past
    // meta_cap (L772-775, L875-878)
    if (tile->n_reads + n_rec > tile->meta_cap) fail(MA_ERR_ARG, "FM sort cap exceeded");
    return n_rec;
}

ma::BamDev bam_view(const ma_hits& h, uint32_t n1, int paired, const ma_fastq_arena& a, const int32_t* rid_to_tid,
                    int32_t n_tid, const uint8_t* rg, uint32_t rg_n, uint8_t* bam, uint64_t cap, const ma_bam_meta& m,
                    const ma_bam_tile& t, uint64_t meta_origin, unsigned long long* status) {
    ma::BamDev b{};
    b.rid = h.rid;
    b.pos = h.pos;
    b.mapq = h.mapq;
    b.flag = h.flag;
    b.sl = h.sl;
    b.sr = h.sr;
    b.nm = h.nm;
    b.arena = a.data;
    b.arena_bytes = a.data_bytes;
    b.name_off = a.name_off;
    b.orig_off = a.orig_off;
    b.qual_off = a.qual_off;
    b.name_len = a.name_len;
    b.orig_len = a.orig_len;
    b.qual_len = a.qual_len;
    b.rid_to_tid = rid_to_tid;
    b.n_tid = n_tid;
    b.rg = rg;
    b.rg_n = rg_n;
    b.n1 = n1;
    b.paired = paired ? 1 : 0;
    b.n_reads = t.n_reads;
    b.n_total = t.n_total;
    b.meta_origin = meta_origin;
    b.chunk = t.chunk;
    b.bam = bam;
    b.cap = cap;
    b.coord = m.coord;
    b.dhi = m.dhi;
    b.dlo = m.dlo;
    b.rec = m.rec;
    b.len = m.len;
    b.score = m.score;
    b.pair = m.pair;
    b.status = status;
    return b;
}

}  // namespace

int ma_emit_bam_batch(ma_ctx* ctx, const ma_hits* hits, uint32_t n1, int paired, const ma_fastq_arena* arena,
                      const int32_t* rid_to_tid, int32_t n_tid, const uint8_t* rg, uint32_t rg_n, uint8_t* bam,
                      uint64_t bam_cap, uint64_t* bam_bytes, const ma_bam_meta* meta, ma_bam_tile* tile) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        if (!bam_bytes) fail(MA_ERR_ARG, "null argument");
        *bam_bytes = 0;
        ctx->last_launches = 0;
        const uint64_t n_rec =
            bam_records_checked(hits, n1, paired, arena, rid_to_tid, n_tid, rg, rg_n, bam, bam_cap, meta, tile);
        if (n_rec == 0) return;
        const bool quals = arena->qual_off != nullptr;
        for (uint64_t i = 0; i < n_rec; ++i) {
            const bool bad = arena->name_off[i] + arena->name_len[i] > arena->data_bytes ||
                             arena->orig_off[i] + arena->orig_len[i] > arena->data_bytes ||
                             (quals && arena->qual_off[i] + arena->qual_len[i] > arena->data_bytes);
            if (bad) fail(MA_ERR_ARG, "arena span of record " + std::to_string(i) + " lies outside the arena");
        }
        use_device(ctx);
        cudaStream_t st = ctx->stream;
        // inputs: 7 hit arrays, 3 offset and 3 length arrays, the tid table
        // and the RG id, packed into one buffer at 256-byte boundaries
        auto al = [](uint64_t n) { return (n + 255) & ~uint64_t(255); };
        const uint64_t hb = al(n_rec * 4), ob = al(n_rec * 8);
        const uint64_t in_bytes = 7 * hb + 3 * ob + (quals ? 3 : 2) * hb + al(uint64_t(n_tid) * 4) + al(rg_n);
        ctx->bam_in.ensure(in_bytes);
        ctx->bam_arena.ensure(arena->data_bytes);
        uint8_t* d = ctx->bam_in.as<uint8_t>();
        auto put = [&](const void* src, uint64_t bytes, uint64_t slot) -> void* {
            void* dst = d;
            if (bytes) ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st), "H2D bam input");
            d += slot;
            return dst;
        };
        ma_hits dh;
        dh.rid = static_cast<int32_t*>(put(hits->rid, n_rec * 4, hb));
        dh.pos = static_cast<uint32_t*>(put(hits->pos, n_rec * 4, hb));
        dh.mapq = static_cast<uint32_t*>(put(hits->mapq, n_rec * 4, hb));
        dh.flag = static_cast<int32_t*>(put(hits->flag, n_rec * 4, hb));
        dh.sl = static_cast<uint32_t*>(put(hits->sl, n_rec * 4, hb));
        dh.sr = static_cast<uint32_t*>(put(hits->sr, n_rec * 4, hb));
        dh.nm = static_cast<uint32_t*>(put(hits->nm, n_rec * 4, hb));
        ma_fastq_arena da{};
        da.data = ctx->bam_arena.as<uint8_t>();
        da.data_bytes = arena->data_bytes;
        if (arena->data_bytes)
            ck(cudaMemcpyAsync(ctx->bam_arena.p, arena->data, arena->data_bytes, cudaMemcpyHostToDevice, st),
               "H2D arena");
        da.name_off = static_cast<const uint64_t*>(put(arena->name_off, n_rec * 8, ob));
        da.orig_off = static_cast<const uint64_t*>(put(arena->orig_off, n_rec * 8, ob));
        da.name_len = static_cast<const uint32_t*>(put(arena->name_len, n_rec * 4, hb));
        da.orig_len = static_cast<const uint32_t*>(put(arena->orig_len, n_rec * 4, hb));
        if (quals) {
            da.qual_off = static_cast<const uint64_t*>(put(arena->qual_off, n_rec * 8, ob));
            da.qual_len = static_cast<const uint32_t*>(put(arena->qual_len, n_rec * 4, hb));
        }
        const int32_t* d_tids = static_cast<const int32_t*>(put(rid_to_tid, uint64_t(n_tid) * 4, al(uint64_t(n_tid) * 4)));
        const uint8_t* d_rg = static_cast<const uint8_t*>(put(rg, rg_n, al(rg_n)));
        // batch-local metadata, copied into the tile arrays at n_reads
        const uint64_t mb8 = al(n_rec * 8), mb4 = al(n_rec * 4);
        ctx->bam_meta.ensure(4 * mb8 + 3 * mb4);
        uint8_t* m = ctx->bam_meta.as<uint8_t>();
        ma_bam_meta dm{reinterpret_cast<uint64_t*>(m), reinterpret_cast<uint64_t*>(m + mb8),
                       reinterpret_cast<uint64_t*>(m + 2 * mb8), reinterpret_cast<uint64_t*>(m + 3 * mb8),
                       reinterpret_cast<uint32_t*>(m + 4 * mb8), reinterpret_cast<uint32_t*>(m + 4 * mb8 + mb4),
                       reinterpret_cast<uint32_t*>(m + 4 * mb8 + 2 * mb4)};
        ctx->bam_status.ensure(4 * sizeof(unsigned long long));
        unsigned long long* d_status = ctx->bam_status.as<unsigned long long>();
        ck(cudaMemsetAsync(d_status, 0, 3 * sizeof(unsigned long long), st), "memset");
        const size_t scratch = bam_scratch_bytes(n_rec);
        ctx->bam_scratch.ensure(scratch);
        ma::BamDev b = bam_view(dh, n1, paired, da, d_tids, n_tid, d_rg, rg_n, nullptr, 0, dm, *tile, tile->n_reads,
                                d_status);
        int launches = enqueue_bam_layout(b, ctx->bam_scratch.p, scratch, st);
        uint64_t total = 0;
        ck(cudaMemcpyAsync(&total, bam_total_in_scratch(ctx->bam_scratch.p, n_rec), 8, cudaMemcpyDeviceToHost, st),
           "D2H bam size");
        ck(cudaStreamSynchronize(st), "bam layout");
        if (total > bam_cap) fail(MA_ERR_ARG, "BAM batch buffer overflow");
        ctx->bam_out.ensure(total);
        b.bam = ctx->bam_out.as<uint8_t>();
        b.cap = total;
        launches += enqueue_bam_records(b, ctx->bam_scratch.p, ctx->sm_count, st);
        unsigned long long status[3] = {0, 0, 0};
        ck(cudaMemcpyAsync(status, d_status, sizeof(status), cudaMemcpyDeviceToHost, st), "D2H bam status");
        ck(cudaMemcpyAsync(bam, b.bam, total, cudaMemcpyDeviceToHost, st), "D2H bam records");
        const uint64_t t0 = tile->n_reads;
        ck(cudaMemcpyAsync(meta->coord + t0, dm.coord, n_rec * 8, cudaMemcpyDeviceToHost, st), "D2H meta");
        ck(cudaMemcpyAsync(meta->dhi + t0, dm.dhi, n_rec * 8, cudaMemcpyDeviceToHost, st), "D2H meta");
        ck(cudaMemcpyAsync(meta->dlo + t0, dm.dlo, n_rec * 8, cudaMemcpyDeviceToHost, st), "D2H meta");
        ck(cudaMemcpyAsync(meta->rec + t0, dm.rec, n_rec * 8, cudaMemcpyDeviceToHost, st), "D2H meta");
        ck(cudaMemcpyAsync(meta->len + t0, dm.len, n_rec * 4, cudaMemcpyDeviceToHost, st), "D2H meta");
        ck(cudaMemcpyAsync(meta->score + t0, dm.score, n_rec * 4, cudaMemcpyDeviceToHost, st), "D2H meta");
        ck(cudaMemcpyAsync(meta->pair + t0, dm.pair, n_rec * 4, cudaMemcpyDeviceToHost, st), "D2H meta");
        ck(cudaStreamSynchronize(st), "bam records");
        if (status[0] != total || status[2] != 0) fail(MA_ERR_INTERNAL, "BAM record pass disagrees with its layout");
        ctx->last_launches = launches;
        *bam_bytes = total;
        tile->n_reads += n_rec;
        tile->n_mapped += status[1];
    });
}

int ma_emit_bam_batch_device(ma_ctx* ctx, const ma_hits* d_hits, uint32_t n1, int paired,
                             const ma_fastq_arena* d_arena, const int32_t* d_rid_to_tid, int32_t n_tid,
                             const uint8_t* d_rg, uint32_t rg_n, uint8_t* d_bam, uint64_t bam_cap,
                             const ma_bam_meta* d_meta, const ma_bam_tile* tile, uint64_t* d_status, void* stream) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        if (!d_status) fail(MA_ERR_ARG, "null argument");
        const uint64_t n_rec = bam_records_checked(d_hits, n1, paired, d_arena, d_rid_to_tid, n_tid, d_rg, rg_n,
                                                   d_bam, bam_cap, d_meta, tile);
        use_device(ctx);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
        unsigned long long* status = reinterpret_cast<unsigned long long*>(d_status);
        ck(cudaMemsetAsync(status, 0, 3 * sizeof(unsigned long long), st), "memset");
        if (n_rec == 0) return;
        const size_t scratch = bam_scratch_bytes(n_rec);
        ctx->bam_scratch.ensure(scratch);
        ma::BamDev b = bam_view(*d_hits, n1, paired, *d_arena, d_rid_to_tid, n_tid, d_rg, rg_n, d_bam, bam_cap,
                                *d_meta, *tile, 0, status);
        int launches = enqueue_bam_layout(b, ctx->bam_scratch.p, scratch, st);
        launches += enqueue_bam_records(b, ctx->bam_scratch.p, ctx->sm_count, st);
        ck(cudaGetLastError(), "bam kernels");
        ctx->last_launches = launches;
    });
}

namespace {
void check_tile_size(uint64_t n) {
    if (n >= (uint64_t(1) << 32)) fail(MA_ERR_ARG, "a tile holds fewer than 2^32 records");
}
}  // namespace

int ma_sort_markdup(ma_ctx* ctx, uint64_t n, const uint64_t* coord, const uint64_t* dhi, const uint64_t* dlo,
                    const uint32_t* score, const uint32_t* pair, uint32_t* is_dup, uint32_t* perm, int do_markdup,
                    uint32_t* dup_perm, uint64_t* n_marked) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        if (n_marked) *n_marked = 0;
        if (n == 0) return;
        check_tile_size(n);
        if (!coord || !is_dup || !perm || (do_markdup && (!dhi || !dlo || !score || !pair)))
            fail(MA_ERR_ARG, "null argument");
        use_device(ctx);
        cudaStream_t st = ctx->stream;
        const uint64_t b8 = (n * 8 + 255) & ~uint64_t(255), b4 = (n * 4 + 255) & ~uint64_t(255);
        ctx->sort_in.ensure(3 * b8 + 2 * b4);
        ctx->sort_out.ensure(3 * b4 + 256);
        uint8_t* in = ctx->sort_in.as<uint8_t>();
        uint8_t* out = ctx->sort_out.as<uint8_t>();
        SortDev s{};
        s.n = n;
        s.coord = reinterpret_cast<const uint64_t*>(in);
        s.dhi = reinterpret_cast<const uint64_t*>(in + b8);
        s.dlo = reinterpret_cast<const uint64_t*>(in + 2 * b8);
        s.score = reinterpret_cast<const uint32_t*>(in + 3 * b8);
        s.pair = reinterpret_cast<const uint32_t*>(in + 3 * b8 + b4);
        s.is_dup = reinterpret_cast<uint32_t*>(out);
        s.perm = reinterpret_cast<uint32_t*>(out + b4);
        s.dup_perm = dup_perm ? reinterpret_cast<uint32_t*>(out + 2 * b4) : nullptr;
        s.do_markdup = do_markdup ? 1 : 0;
        s.marked = reinterpret_cast<unsigned long long*>(out + 3 * b4);
        ck(cudaMemcpyAsync(in, coord, n * 8, cudaMemcpyHostToDevice, st), "H2D sort keys");
        if (do_markdup) {
            ck(cudaMemcpyAsync(in + b8, dhi, n * 8, cudaMemcpyHostToDevice, st), "H2D sort keys");
            ck(cudaMemcpyAsync(in + 2 * b8, dlo, n * 8, cudaMemcpyHostToDevice, st), "H2D sort keys");
            ck(cudaMemcpyAsync(in + 3 * b8, score, n * 4, cudaMemcpyHostToDevice, st), "H2D sort keys");
            ck(cudaMemcpyAsync(in + 3 * b8 + b4, pair, n * 4, cudaMemcpyHostToDevice, st), "H2D sort keys");
        }
        const size_t scratch = sort_scratch_bytes(n);
        ctx->sort_scratch.ensure(scratch);
        const int launches = enqueue_sort_markdup(s, ctx->sort_scratch.p, scratch, st);
        unsigned long long marked = 0;
        ck(cudaMemcpyAsync(is_dup, s.is_dup, n * 4, cudaMemcpyDeviceToHost, st), "D2H is_dup");
        ck(cudaMemcpyAsync(perm, s.perm, n * 4, cudaMemcpyDeviceToHost, st), "D2H perm");
        if (dup_perm) ck(cudaMemcpyAsync(dup_perm, s.dup_perm, n * 4, cudaMemcpyDeviceToHost, st), "D2H dup_perm");
        ck(cudaMemcpyAsync(&marked, s.marked, 8, cudaMemcpyDeviceToHost, st), "D2H marked");
        ck(cudaStreamSynchronize(st), "sort/markdup");
        if (n_marked) *n_marked = marked;
        ctx->last_launches = launches;
    });
}

int ma_sort_markdup_device(ma_ctx* ctx, uint64_t n, const uint64_t* d_coord, const uint64_t* d_dhi,
                           const uint64_t* d_dlo, const uint32_t* d_score, const uint32_t* d_pair, uint32_t* d_is_dup,
                           uint32_t* d_perm, int do_markdup, uint32_t* d_dup_perm, uint64_t* d_marked, void* stream) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        use_device(ctx);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
        if (d_marked) ck(cudaMemsetAsync(d_marked, 0, 8, st), "memset");
        if (n == 0) return;
        check_tile_size(n);
        if (!d_coord || !d_is_dup || !d_perm || (do_markdup && (!d_dhi || !d_dlo || !d_score || !d_pair)))
            fail(MA_ERR_ARG, "null argument");
        SortDev s{n, d_coord, d_dhi, d_dlo, d_score, d_pair, d_is_dup, d_perm, d_dup_perm, do_markdup ? 1 : 0,
                  reinterpret_cast<unsigned long long*>(d_marked)};
        const size_t scratch = sort_scratch_bytes(n);
        ctx->sort_scratch.ensure(scratch);
        ctx->last_launches = enqueue_sort_markdup(s, ctx->sort_scratch.p, scratch, st);
    });
}

int ma_gather_sorted_bam(ma_ctx* ctx, uint64_t n, const uint32_t* perm, const uint64_t* rec, const uint32_t* len,
                         const uint32_t* is_dup, int apply_dup, const uint8_t* const* chunks,
                         const uint64_t* chunk_len, uint32_t n_chunks, uint8_t* out, uint64_t out_cap,
                         uint64_t* out_bytes) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        if (!out_bytes) fail(MA_ERR_ARG, "null argument");
        *out_bytes = 0;
        if (n == 0) return;
        check_tile_size(n);
        if (!perm || !rec || !len || (apply_dup && !is_dup) || (n_chunks && (!chunks || !chunk_len)) ||
            (out_cap && !out))
            fail(MA_ERR_ARG, "null argument");
        use_device(ctx);
        cudaStream_t st = ctx->stream;
        // the chunks back to back in one device buffer
        std::vector<uint64_t> base(n_chunks + 1, 0);
        for (uint32_t c = 0; c < n_chunks; ++c) base[c + 1] = base[c] + ((chunk_len[c] + 15) & ~uint64_t(15));
        ctx->gather_chunks.ensure(base[n_chunks] + (n_chunks + 1) * 16);
        uint8_t* dch = ctx->gather_chunks.as<uint8_t>();
        std::vector<const uint8_t*> ptrs(n_chunks);
        for (uint32_t c = 0; c < n_chunks; ++c) {
            if (chunk_len[c] && !chunks[c]) fail(MA_ERR_ARG, "null chunk");
            if (chunk_len[c])
                ck(cudaMemcpyAsync(dch + base[c], chunks[c], chunk_len[c], cudaMemcpyHostToDevice, st), "H2D chunk");
            ptrs[c] = dch + base[c];
        }
        const uint64_t b8 = (n * 8 + 255) & ~uint64_t(255), b4 = (n * 4 + 255) & ~uint64_t(255);
        const uint64_t tb = ((n_chunks + 1) * 8 + 255) & ~uint64_t(255);
        ctx->gather_in.ensure(b8 + 3 * b4 + 2 * tb + 256);
        uint8_t* in = ctx->gather_in.as<uint8_t>();
        GatherDev g{};
        g.n = n;
        g.rec = reinterpret_cast<const uint64_t*>(in);
        g.perm = reinterpret_cast<const uint32_t*>(in + b8);
        g.len = reinterpret_cast<const uint32_t*>(in + b8 + b4);
        g.is_dup = apply_dup ? reinterpret_cast<const uint32_t*>(in + b8 + 2 * b4) : nullptr;
        g.apply_dup = apply_dup ? 1 : 0;
        g.chunks = reinterpret_cast<const uint8_t* const*>(in + b8 + 3 * b4);
        g.chunk_len = reinterpret_cast<const uint64_t*>(in + b8 + 3 * b4 + tb);
        g.n_chunks = n_chunks;
        g.status = reinterpret_cast<unsigned long long*>(in + b8 + 3 * b4 + 2 * tb);
        ck(cudaMemcpyAsync(in, rec, n * 8, cudaMemcpyHostToDevice, st), "H2D rec");
        ck(cudaMemcpyAsync(in + b8, perm, n * 4, cudaMemcpyHostToDevice, st), "H2D perm");
        ck(cudaMemcpyAsync(in + b8 + b4, len, n * 4, cudaMemcpyHostToDevice, st), "H2D len");
        if (apply_dup) ck(cudaMemcpyAsync(in + b8 + 2 * b4, is_dup, n * 4, cudaMemcpyHostToDevice, st), "H2D is_dup");
        if (n_chunks) {
            ck(cudaMemcpyAsync(in + b8 + 3 * b4, ptrs.data(), n_chunks * 8, cudaMemcpyHostToDevice, st), "H2D chunks");
            ck(cudaMemcpyAsync(in + b8 + 3 * b4 + tb, chunk_len, n_chunks * 8, cudaMemcpyHostToDevice, st),
               "H2D chunk sizes");
        }
        ck(cudaMemsetAsync(g.status, 0, 16, st), "memset");
        const size_t scratch = gather_scratch_bytes(n);
        ctx->gather_scratch.ensure(scratch);
        int launches = enqueue_gather_layout(g, ctx->gather_scratch.p, scratch, st);
        uint64_t total = 0;
        unsigned long long status[2] = {0, 0};
        ck(cudaMemcpyAsync(&total, gather_total_in_scratch(ctx->gather_scratch.p, n), 8, cudaMemcpyDeviceToHost, st),
           "D2H size");
        ck(cudaMemcpyAsync(status, g.status, 16, cudaMemcpyDeviceToHost, st), "D2H status");
        ck(cudaStreamSynchronize(st), "gather layout");
        if (status[1]) fail(MA_ERR_ARG, std::to_string(status[1]) + " records lie outside their chunks");
        if (total > out_cap) fail(MA_ERR_ARG, "BAM record stream larger than the output buffer");
        ctx->gather_out.ensure(total);
        g.out = ctx->gather_out.as<uint8_t>();
        g.cap = total;
        launches += enqueue_gather_records(g, ctx->gather_scratch.p, ctx->sm_count, st);
        ck(cudaMemcpyAsync(out, g.out, total, cudaMemcpyDeviceToHost, st), "D2H records");
        ck(cudaStreamSynchronize(st), "gather records");
        ctx->last_launches = launches;
        *out_bytes = total;
    });
}

int ma_gather_sorted_bam_device(ma_ctx* ctx, uint64_t n, const uint32_t* d_perm, const uint64_t* d_rec,
                                const uint32_t* d_len, const uint32_t* d_is_dup, int apply_dup,
                                const uint8_t* const* d_chunks, const uint64_t* d_chunk_len, uint32_t n_chunks,
                                uint8_t* d_out, uint64_t out_cap, uint64_t* d_status, void* stream) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        if (!d_status) fail(MA_ERR_ARG, "null argument");
        use_device(ctx);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
        ck(cudaMemsetAsync(d_status, 0, 16, st), "memset");
        if (n == 0) return;
        check_tile_size(n);
        if (!d_perm || !d_rec || !d_len || (apply_dup && !d_is_dup) || (n_chunks && (!d_chunks || !d_chunk_len)) ||
            (out_cap && !d_out))
            fail(MA_ERR_ARG, "null argument");
        GatherDev g{};
        g.n = n;
        g.perm = d_perm;
        g.rec = d_rec;
        g.len = d_len;
        g.is_dup = apply_dup ? d_is_dup : nullptr;
        g.apply_dup = apply_dup ? 1 : 0;
        g.chunks = d_chunks;
        g.chunk_len = d_chunk_len;
        g.n_chunks = n_chunks;
        g.out = d_out;
        g.cap = out_cap;
        g.status = reinterpret_cast<unsigned long long*>(d_status);
        const size_t scratch = gather_scratch_bytes(n);
        ctx->gather_scratch.ensure(scratch);
        int launches = enqueue_gather_layout(g, ctx->gather_scratch.p, scratch, st);
        launches += enqueue_gather_records(g, ctx->gather_scratch.p, ctx->sm_count, st);
        ctx->last_launches = launches;
    });
}

namespace {
void* fq_newline_buffer(void* user, size_t bytes) {
    DevBuf* b = static_cast<DevBuf*>(user);
    b->ensure(bytes);
    return b->p;
}

const char* fastq_error(unsigned long long code) {
    return code == 1 ? "truncated FASTQ (missing SEQ)"
                     : code == 2 ? "truncated FASTQ (missing +)" : "truncated FASTQ (missing QUAL)";
}

// Parses on the device; outputs in d_out.  Returns the status of
// fastq_parse_enqueue.
void parse_on_device(ma_ctx* ctx, const uint8_t* d_buf, uint64_t n, int at_eof, uint32_t max_records, uint64_t base,
                     int rules, const ma_fastq_records& d_out, cudaStream_t st, unsigned long long* status) {
    if (n >= (uint64_t(1) << 32)) fail(MA_ERR_ARG, "a FASTQ buffer holds fewer than 2^32 bytes");
    if (rules != MA_FASTQ_RULES_STREAM && rules != MA_FASTQ_RULES_PAIR_READER) fail(MA_ERR_ARG, "unknown FASTQ rules");
    const size_t scratch = fastq_scratch_bytes(n);
    ctx->fq_scratch.ensure(scratch);
    FastqRecordsDev o{d_out.name_off, d_out.name_len, d_out.seq_off, d_out.seq_len, d_out.qual_off, d_out.qual_len};
    ctx->last_launches = fastq_parse_enqueue(d_buf, n, at_eof, max_records, base, rules, o, ctx->fq_scratch.p, scratch,
                                             fq_newline_buffer, &ctx->fq_newlines, st, status);
    if (status[3]) fail(MA_ERR_FORMAT, fastq_error(status[3]));
}

void check_records(const ma_fastq_records* o) {
    if (!o || !o->name_off || !o->name_len || !o->seq_off || !o->seq_len || !o->qual_off || !o->qual_len)
        fail(MA_ERR_ARG, "null record array");
}
}  // namespace

int ma_fastq_parse_rules(ma_ctx* ctx, const uint8_t* buf, uint64_t n_bytes, int at_eof, uint32_t max_records,
                         uint64_t base, int rules, const ma_fastq_records* out, uint64_t* out3) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        if (!out3 || (n_bytes && !buf)) fail(MA_ERR_ARG, "null argument");
        check_records(out);
        out3[0] = out3[1] = out3[2] = 0;
        use_device(ctx);
        cudaStream_t st = ctx->stream;
        ctx->fq_in.ensure(n_bytes + 16);
        if (n_bytes) ck(cudaMemcpyAsync(ctx->fq_in.p, buf, n_bytes, cudaMemcpyHostToDevice, st), "H2D FASTQ");
        const uint64_t m = max_records;
        const uint64_t b8 = (m * 8 + 255) & ~uint64_t(255), b4 = (m * 4 + 255) & ~uint64_t(255);
        ctx->fq_out.ensure(3 * (b8 + b4) + 256);
        uint8_t* o = ctx->fq_out.as<uint8_t>();
        ma_fastq_records d{reinterpret_cast<uint64_t*>(o), reinterpret_cast<uint32_t*>(o + b8),
                           reinterpret_cast<uint64_t*>(o + b8 + b4), reinterpret_cast<uint32_t*>(o + 2 * b8 + b4),
                           reinterpret_cast<uint64_t*>(o + 2 * b8 + 2 * b4),
                           reinterpret_cast<uint32_t*>(o + 3 * b8 + 2 * b4)};
        unsigned long long status[6] = {0, 0, 0, 0, 0, 0};
        parse_on_device(ctx, ctx->fq_in.as<uint8_t>(), n_bytes, at_eof, max_records, base, rules, d, st, status);
        const uint64_t r = status[1];
        if (r) {
            ck(cudaMemcpyAsync(out->name_off, d.name_off, r * 8, cudaMemcpyDeviceToHost, st), "D2H records");
            ck(cudaMemcpyAsync(out->name_len, d.name_len, r * 4, cudaMemcpyDeviceToHost, st), "D2H records");
            ck(cudaMemcpyAsync(out->seq_off, d.seq_off, r * 8, cudaMemcpyDeviceToHost, st), "D2H records");
            ck(cudaMemcpyAsync(out->seq_len, d.seq_len, r * 4, cudaMemcpyDeviceToHost, st), "D2H records");
            ck(cudaMemcpyAsync(out->qual_off, d.qual_off, r * 8, cudaMemcpyDeviceToHost, st), "D2H records");
            ck(cudaMemcpyAsync(out->qual_len, d.qual_len, r * 4, cudaMemcpyDeviceToHost, st), "D2H records");
            ck(cudaStreamSynchronize(st), "D2H records");
        }
        out3[0] = r;
        out3[1] = status[2];
        out3[2] = status[5];
    });
}

int ma_fastq_parse_rules_device(ma_ctx* ctx, const uint8_t* d_buf, uint64_t n_bytes, int at_eof,
                                uint32_t max_records, uint64_t base, int rules, const ma_fastq_records* d_out,
                                uint64_t* out3, void* stream) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        if (!out3 || (n_bytes && !d_buf)) fail(MA_ERR_ARG, "null argument");
        check_records(d_out);
        out3[0] = out3[1] = out3[2] = 0;
        use_device(ctx);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
        unsigned long long status[6] = {0, 0, 0, 0, 0, 0};
        parse_on_device(ctx, d_buf, n_bytes, at_eof, max_records, base, rules, *d_out, st, status);
        out3[0] = status[1];
        out3[1] = status[2];
        out3[2] = status[5];
    });
}

int ma_fastq_parse(ma_ctx* ctx, const uint8_t* buf, uint64_t n_bytes, int at_eof, uint32_t max_records, uint64_t base,
                   const ma_fastq_records* out, uint64_t* out3) {
    return ma_fastq_parse_rules(ctx, buf, n_bytes, at_eof, max_records, base, MA_FASTQ_RULES_STREAM, out, out3);
}

int ma_fastq_parse_device(ma_ctx* ctx, const uint8_t* d_buf, uint64_t n_bytes, int at_eof, uint32_t max_records,
                          uint64_t base, const ma_fastq_records* d_out, uint64_t* out3, void* stream) {
    return ma_fastq_parse_rules_device(ctx, d_buf, n_bytes, at_eof, max_records, base, MA_FASTQ_RULES_STREAM, d_out,
                                       out3, stream);
}

int ma_fastq_rows_device(ma_ctx* ctx, const uint8_t* d_arena, const uint64_t* d_seq_off, const uint32_t* d_seq_len,
                         uint32_t n_seq, uint32_t max_len, uint8_t* d_rows, uint32_t* d_lens, void* stream) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        if (n_seq == 0) return;
        if (!d_arena || !d_seq_off || !d_seq_len || !d_rows) fail(MA_ERR_ARG, "null argument");
        use_device(ctx);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
        ctx->last_launches = fastq_rows_enqueue(d_arena, d_seq_off, d_seq_len, n_seq, max_len, d_rows, d_lens, st);
    });
}

namespace {
uint64_t sam_lines_checked(const ma_hits* h, uint32_t n1, int paired, const ma_fastq_arena* a,
                           const ma_sam_contigs* c, const uint8_t* rg, uint32_t rg_n, const uint8_t* out,
                           uint64_t cap) {
    const uint64_t n_seq = static_cast<uint64_t>(n1) * (paired ? 2 : 1);
    if (!h || !a || !c) fail(MA_ERR_ARG, "null argument");
    if (n_seq == 0) return 0;
    if (!h->rid || !h->pos || !h->mapq || !h->flag || !h->sl || !h->sr) fail(MA_ERR_ARG, "null hit array");
    if (!a->name_off || !a->name_len || !a->orig_off || !a->orig_len || !a->qual_off || !a->qual_len ||
        (a->data_bytes && !a->data))
        fail(MA_ERR_ARG, "null arena array (SAM needs qualities)");
    if (c->n && (!c->name_off || !c->name_len || !c->canon || (c->names_bytes && !c->names)))
        fail(MA_ERR_ARG, "null contig table array");
    if ((rg_n && !rg) || (cap && !out)) fail(MA_ERR_ARG, "null argument");
    return n_seq;
}

SamDev sam_view(const ma_hits& h, uint32_t n1, int paired, const ma_fastq_arena& a, const ma_sam_contigs& c,
                const uint8_t* rg, uint32_t rg_n, uint8_t* out, uint64_t cap, unsigned long long* status) {
    SamDev d{};
    d.rid = h.rid;
    d.pos = h.pos;
    d.mapq = h.mapq;
    d.flag = h.flag;
    d.sl = h.sl;
    d.sr = h.sr;
    d.arena = a.data;
    d.arena_bytes = a.data_bytes;
    d.name_off = a.name_off;
    d.name_len = a.name_len;
    d.seq_off = a.orig_off;
    d.seq_len = a.orig_len;
    d.qual_off = a.qual_off;
    d.qual_len = a.qual_len;
    d.names = c.names;
    d.names_bytes = c.names_bytes;
    d.cname_off = c.name_off;
    d.cname_len = c.name_len;
    d.canon = c.canon;
    d.n_contigs = c.n;
    d.rg = rg;
    d.rg_n = rg_n;
    d.n1 = n1;
    d.paired = paired ? 1 : 0;
    d.sam = out;
    d.cap = cap;
    d.status = status;
    return d;
}

const char* sam_error(unsigned long long bits) {
    if (bits & 4) return "hit rid outside the contig table";
    if (bits & 8) return "arena or contig-name span outside its buffer";
    if (bits & 2) return "FASTQ SEQ/QUAL is not valid UTF-8";
    return "SAM batch buffer overflow";
}
}  // namespace

int ma_emit_sam_batch(ma_ctx* ctx, const ma_hits* hits, uint32_t n1, int paired, const ma_fastq_arena* arena,
                      const ma_sam_contigs* contigs, const uint8_t* rg, uint32_t rg_n, uint8_t* sam,
                      uint64_t sam_cap, uint64_t* sam_bytes, uint64_t* mapped) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        if (!sam_bytes || !mapped) fail(MA_ERR_ARG, "null argument");
        *sam_bytes = 0;
        *mapped = 0;
        const uint64_t n_seq = sam_lines_checked(hits, n1, paired, arena, contigs, rg, rg_n, sam, sam_cap);
        if (n_seq == 0) return;
        for (uint64_t i = 0; i < n_seq; ++i) {
            const uint64_t n = arena->data_bytes;
            const bool bad = arena->name_off[i] > n || arena->name_len[i] > n - arena->name_off[i] ||
                             arena->orig_off[i] > n || arena->orig_len[i] > n - arena->orig_off[i] ||
                             arena->qual_off[i] > n || arena->qual_len[i] > n - arena->qual_off[i];
            if (bad) fail(MA_ERR_ARG, "arena span of record " + std::to_string(i) + " lies outside the arena");
        }
        for (uint32_t i = 0; i < contigs->n; ++i)
            if (contigs->name_off[i] > contigs->names_bytes ||
                contigs->name_len[i] > contigs->names_bytes - contigs->name_off[i])
                fail(MA_ERR_ARG, "contig name span outside the name buffer");
        use_device(ctx);
        cudaStream_t st = ctx->stream;
        auto al = [](uint64_t n) { return (n + 255) & ~uint64_t(255); };
        const uint64_t hb = al(n_seq * 4), ob = al(n_seq * 8), cb4 = al(uint64_t(contigs->n) * 4),
                       cb8 = al(uint64_t(contigs->n) * 8);
        const uint64_t in_bytes = 6 * hb + 3 * ob + 3 * hb + cb8 + 2 * cb4 + al(contigs->names_bytes) + al(rg_n);
        ctx->sam_in.ensure(in_bytes);
        ctx->sam_arena.ensure(arena->data_bytes);
        uint8_t* d = ctx->sam_in.as<uint8_t>();
        auto put = [&](const void* src, uint64_t bytes, uint64_t slot) -> void* {
            void* dst = d;
            if (bytes) ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st), "H2D sam input");
            d += slot;
            return dst;
        };
        ma_hits dh{};
        dh.rid = static_cast<int32_t*>(put(hits->rid, n_seq * 4, hb));
        dh.pos = static_cast<uint32_t*>(put(hits->pos, n_seq * 4, hb));
        dh.mapq = static_cast<uint32_t*>(put(hits->mapq, n_seq * 4, hb));
        dh.flag = static_cast<int32_t*>(put(hits->flag, n_seq * 4, hb));
        dh.sl = static_cast<uint32_t*>(put(hits->sl, n_seq * 4, hb));
        dh.sr = static_cast<uint32_t*>(put(hits->sr, n_seq * 4, hb));
        ma_fastq_arena da{};
        da.data = ctx->sam_arena.as<uint8_t>();
        da.data_bytes = arena->data_bytes;
        if (arena->data_bytes)
            ck(cudaMemcpyAsync(ctx->sam_arena.p, arena->data, arena->data_bytes, cudaMemcpyHostToDevice, st),
               "H2D arena");
        da.name_off = static_cast<const uint64_t*>(put(arena->name_off, n_seq * 8, ob));
        da.orig_off = static_cast<const uint64_t*>(put(arena->orig_off, n_seq * 8, ob));
        da.qual_off = static_cast<const uint64_t*>(put(arena->qual_off, n_seq * 8, ob));
        da.name_len = static_cast<const uint32_t*>(put(arena->name_len, n_seq * 4, hb));
        da.orig_len = static_cast<const uint32_t*>(put(arena->orig_len, n_seq * 4, hb));
        da.qual_len = static_cast<const uint32_t*>(put(arena->qual_len, n_seq * 4, hb));
        ma_sam_contigs dc{};
        dc.n = contigs->n;
        dc.names_bytes = contigs->names_bytes;
        dc.name_off = static_cast<const uint64_t*>(put(contigs->name_off, uint64_t(contigs->n) * 8, cb8));
        dc.name_len = static_cast<const uint32_t*>(put(contigs->name_len, uint64_t(contigs->n) * 4, cb4));
        dc.canon = static_cast<const uint32_t*>(put(contigs->canon, uint64_t(contigs->n) * 4, cb4));
        dc.names = static_cast<const uint8_t*>(put(contigs->names, contigs->names_bytes, al(contigs->names_bytes)));
        const uint8_t* d_rg = static_cast<const uint8_t*>(put(rg, rg_n, al(rg_n)));
        ctx->sam_status.ensure(4 * sizeof(unsigned long long));
        unsigned long long* d_status = ctx->sam_status.as<unsigned long long>();
        ck(cudaMemsetAsync(d_status, 0, 3 * sizeof(unsigned long long), st), "memset");
        ctx->sam_out.ensure(sam_cap ? sam_cap : 1);
        const size_t scratch = sam_scratch_bytes(n_seq);
        ctx->sam_scratch.ensure(scratch);
        SamDev v = sam_view(dh, n1, paired, da, dc, d_rg, rg_n, ctx->sam_out.as<uint8_t>(), sam_cap, d_status);
        ctx->last_launches = enqueue_sam(v, ctx->sam_scratch.p, scratch, ctx->sm_count, st);
        unsigned long long status[3] = {0, 0, 0};
        ck(cudaMemcpyAsync(status, d_status, sizeof(status), cudaMemcpyDeviceToHost, st), "D2H sam status");
        ck(cudaStreamSynchronize(st), "sam");
        *sam_bytes = status[0];
        if (status[2]) fail(MA_ERR_ARG, sam_error(status[2]));
        if (status[0]) {
            ck(cudaMemcpyAsync(sam, ctx->sam_out.p, status[0], cudaMemcpyDeviceToHost, st), "D2H sam");
            ck(cudaStreamSynchronize(st), "D2H sam");
        }
        *mapped = status[1];
    });
}

int ma_emit_sam_batch_device(ma_ctx* ctx, const ma_hits* d_hits, uint32_t n1, int paired,
                             const ma_fastq_arena* d_arena, const ma_sam_contigs* d_contigs, const uint8_t* d_rg,
                             uint32_t rg_n, uint8_t* d_sam, uint64_t sam_cap, uint64_t* d_status, void* stream) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        if (!d_status) fail(MA_ERR_ARG, "null argument");
        const uint64_t n_seq = sam_lines_checked(d_hits, n1, paired, d_arena, d_contigs, d_rg, rg_n, d_sam, sam_cap);
        use_device(ctx);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
        unsigned long long* status = reinterpret_cast<unsigned long long*>(d_status);
        ck(cudaMemsetAsync(status, 0, 3 * sizeof(unsigned long long), st), "memset");
        if (n_seq == 0) return;
        const size_t scratch = sam_scratch_bytes(n_seq);
        ctx->sam_scratch.ensure(scratch);
        SamDev v = sam_view(*d_hits, n1, paired, *d_arena, *d_contigs, d_rg, rg_n, d_sam, sam_cap, status);
        ctx->last_launches = enqueue_sam(v, ctx->sam_scratch.p, scratch, ctx->sm_count, st);
    });
}

namespace {
const char* inflate_error(uint32_t code) {
    switch (code) {
        case 1: return "deflate data end early";
        case 2: return "invalid block type";
        case 3: return "invalid stored block lengths";
        case 4: return "invalid code lengths";
        case 5: return "invalid code";
        case 6: return "distance too far back";
        case 7: return "more data than ISIZE";
        case bgzf_inflate::S_SIZE: return "inflated size differs from ISIZE";
        case bgzf_inflate::S_CRC: return "CRC-32 mismatch";
        default: return "member span outside its buffer";
    }
}
}  // namespace

int ma_bgzf_inflate(ma_ctx* ctx, const uint8_t* in, uint64_t in_bytes, const uint64_t* src_off,
                    const uint32_t* src_len, const uint64_t* dst_off, const uint32_t* isize, const uint32_t* crc,
                    uint32_t n_members, uint8_t* out, uint64_t out_bytes, uint32_t* status) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        if (n_members == 0) return;
        if (!in || !src_off || !src_len || !dst_off || !isize || !crc || !status || (out_bytes && !out))
            fail(MA_ERR_ARG, "null argument");
        use_device(ctx);
        cudaStream_t st = ctx->stream;
        const uint64_t n = n_members, b8 = (n * 8 + 255) & ~uint64_t(255), b4 = (n * 4 + 255) & ~uint64_t(255);
        ctx->inf_in.ensure(in_bytes ? in_bytes : 1);
        ctx->inf_cols.ensure(2 * b8 + 4 * b4);
        ctx->inf_out.ensure(out_bytes ? out_bytes : 1);
        uint8_t* c = ctx->inf_cols.as<uint8_t>();
        bgzf_inflate::Job j{};
        j.in = ctx->inf_in.as<uint8_t>();
        j.in_bytes = in_bytes;
        j.src_off = reinterpret_cast<const uint64_t*>(c);
        j.dst_off = reinterpret_cast<const uint64_t*>(c + b8);
        j.src_len = reinterpret_cast<const uint32_t*>(c + 2 * b8);
        j.isize = reinterpret_cast<const uint32_t*>(c + 2 * b8 + b4);
        j.crc = reinterpret_cast<const uint32_t*>(c + 2 * b8 + 2 * b4);
        j.status = reinterpret_cast<uint32_t*>(c + 2 * b8 + 3 * b4);
        j.n = n_members;
        j.out = ctx->inf_out.as<uint8_t>();
        j.out_bytes = out_bytes;
        if (in_bytes) ck(cudaMemcpyAsync(ctx->inf_in.p, in, in_bytes, cudaMemcpyHostToDevice, st), "H2D inflate");
        ck(cudaMemcpyAsync(c, src_off, n * 8, cudaMemcpyHostToDevice, st), "H2D inflate");
        ck(cudaMemcpyAsync(c + b8, dst_off, n * 8, cudaMemcpyHostToDevice, st), "H2D inflate");
        ck(cudaMemcpyAsync(c + 2 * b8, src_len, n * 4, cudaMemcpyHostToDevice, st), "H2D inflate");
        ck(cudaMemcpyAsync(c + 2 * b8 + b4, isize, n * 4, cudaMemcpyHostToDevice, st), "H2D inflate");
        ck(cudaMemcpyAsync(c + 2 * b8 + 2 * b4, crc, n * 4, cudaMemcpyHostToDevice, st), "H2D inflate");
        ctx->last_launches = bgzf_inflate_enqueue(j, ctx->sm_count, st);
        ck(cudaMemcpyAsync(status, j.status, n * 4, cudaMemcpyDeviceToHost, st), "D2H inflate");
        if (out_bytes) ck(cudaMemcpyAsync(out, j.out, out_bytes, cudaMemcpyDeviceToHost, st), "D2H inflate");
        ck(cudaStreamSynchronize(st), "inflate");
        for (uint64_t m = 0; m < n; ++m)
            if (status[m])
                fail(MA_ERR_FORMAT, "BGZF member " + std::to_string(m) + ": " + inflate_error(status[m]));
    });
}

int ma_bgzf_inflate_device(ma_ctx* ctx, const uint8_t* d_in, uint64_t in_bytes, const uint64_t* d_src_off,
                           const uint32_t* d_src_len, const uint64_t* d_dst_off, const uint32_t* d_isize,
                           const uint32_t* d_crc, uint32_t n_members, uint8_t* d_out, uint64_t out_bytes,
                           uint32_t* d_status, void* stream) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        if (n_members == 0) return;
        if (!d_in || !d_src_off || !d_src_len || !d_dst_off || !d_isize || !d_crc || !d_status ||
            (out_bytes && !d_out))
            fail(MA_ERR_ARG, "null argument");
        use_device(ctx);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
        bgzf_inflate::Job j{d_in, in_bytes, d_src_off, d_src_len, d_dst_off, d_isize, d_crc, n_members, d_out,
                            out_bytes, d_status};
        ctx->last_launches = bgzf_inflate_enqueue(j, ctx->sm_count, st);
    });
}

uint64_t ma_bgzf_bound(uint64_t n) { return bgzf_bound(n); }

namespace {
uint64_t bgzf_on_device(ma_ctx* ctx, const uint8_t* d_in, uint64_t n, int level, int append_eof, uint8_t* d_out,
                        uint64_t out_cap, cudaStream_t st) {
    if (level < 0 || level > 9) fail(MA_ERR_ARG, "BGZF level must be in 0..9");
    const size_t scratch = bgzf_scratch_bytes(n, ctx->sm_count);
    ctx->bgzf_scratch.ensure(scratch);
    uint64_t need = 0;
    int launches = 0;
    const uint64_t got = bgzf_compress(d_in, n, level, d_out, out_cap, append_eof, ctx->bgzf_scratch.p, scratch,
                                       ctx->sm_count, st, &need, &launches, nullptr);
    ctx->last_launches = launches;
    if (!got && need) fail(MA_ERR_ARG, "BGZF output larger than the output buffer (" + std::to_string(need) + " bytes)");
    return got;
}
}  // namespace

int ma_bgzf_compress(ma_ctx* ctx, const uint8_t* in, uint64_t n, int level, int append_eof, uint8_t* out,
                     uint64_t out_cap, uint64_t* out_bytes) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        if (!out_bytes || (n && !in) || (out_cap && !out)) fail(MA_ERR_ARG, "null argument");
        *out_bytes = 0;
        use_device(ctx);
        cudaStream_t st = ctx->stream;
        ctx->bgzf_in.ensure(n + 16);
        if (n) ck(cudaMemcpyAsync(ctx->bgzf_in.p, in, n, cudaMemcpyHostToDevice, st), "H2D BGZF input");
        const uint64_t bound = bgzf_bound(n);
        ctx->bgzf_out.ensure(bound);
        const uint64_t got = bgzf_on_device(ctx, ctx->bgzf_in.as<uint8_t>(), n, level, append_eof,
                                            ctx->bgzf_out.as<uint8_t>(), bound, st);
        if (got > out_cap) fail(MA_ERR_ARG, "BGZF output larger than the output buffer (" + std::to_string(got) +
                                                " bytes)");
        if (got) ck(cudaMemcpyAsync(out, ctx->bgzf_out.p, got, cudaMemcpyDeviceToHost, st), "D2H BGZF");
        ck(cudaStreamSynchronize(st), "D2H BGZF");
        *out_bytes = got;
    });
}

int ma_bgzf_compress_device(ma_ctx* ctx, const uint8_t* d_in, uint64_t n, int level, int append_eof, uint8_t* d_out,
                            uint64_t out_cap, uint64_t* out_bytes, void* stream) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->last_launches = 0;
        if (!out_bytes || (n && !d_in) || (out_cap && !d_out)) fail(MA_ERR_ARG, "null argument");
        *out_bytes = 0;
        use_device(ctx);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
        *out_bytes = bgzf_on_device(ctx, d_in, n, level, append_eof, d_out, out_cap, st);
    });
}

int ma_last_launch_count(const ma_ctx* ctx) { return ctx ? ctx->last_launches : 0; }

int ma_ctx_set_profiling(ma_ctx* ctx, int flags) {
    if (!ctx) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        use_device(ctx);
        if ((flags & 1) && !ctx->ev[0])
            for (cudaEvent_t& e : ctx->ev) ck(cudaEventCreate(&e), "cudaEventCreate");
        if ((flags & 1) && !ctx->wave_timer.e[0])
            for (cudaEvent_t& e : ctx->wave_timer.e) ck(cudaEventCreate(&e), "cudaEventCreate");
        if ((flags & 1) && !ctx->wave_timer.s2[0])
            for (cudaEvent_t& e : ctx->wave_timer.s2) ck(cudaEventCreate(&e), "cudaEventCreate");
        ctx->profiling = flags;
    });
}

int ma_ctx_set_tuning(ma_ctx* ctx, const ma_tuning* t) {
    if (!ctx || !t) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        if (t->seed_kernel < 0 || t->seed_kernel > 4) fail(MA_ERR_ARG, "seed_kernel must be 0, 1, 2, 3 or 4");
        if (t->stage1_endpoints < 1) fail(MA_ERR_ARG, "stage1_endpoints must be >= 1");
        if (t->stage2_blocks_per_sm < 0 || t->stage2_blocks_per_sm > 64) fail(MA_ERR_ARG, "bad stage2_blocks_per_sm");
        if (t->reg_level < 0 || t->reg_level > 2) fail(MA_ERR_ARG, "reg_level must be 0, 1 or 2");
        if (t->stage1_max_rows < 1 || t->stage1_max_rows > 16) fail(MA_ERR_ARG, "stage1_max_rows must be in 1..16");
        if (t->stage2_first_wave < 1 || t->stage2_first_wave > 32)
            fail(MA_ERR_ARG, "stage2_first_wave must be in 1..32");
        if (t->wave_endpoints < 1 || t->wave_endpoints > 256) fail(MA_ERR_ARG, "wave_endpoints must be in 1..256");
        if (t->wave_loci_per_read < 1 || t->wave_loci_per_read > 64)
            fail(MA_ERR_ARG, "wave_loci_per_read must be in 1..64");
        if (t->wave_max_rounds < 0) fail(MA_ERR_ARG, "wave_max_rounds must be >= 0");
        if (t->wave_growth < 0 || t->wave_growth > 1) fail(MA_ERR_ARG, "wave_growth must be 0 or 1");
        ctx->tuning = *t;
    });
}

int ma_ctx_set_pipeline(ma_ctx* ctx, const ma_pipeline* p) {
    if (!ctx || !p) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        if (p->compute_streams < 1 || p->compute_streams > 3) fail(MA_ERR_ARG, "compute_streams must be 1..3");
        if (p->growth_percent > 1000) fail(MA_ERR_ARG, "growth_percent must be <= 1000");
        ctx->pipeline = *p;
    });
}

int ma_ctx_get_pipeline(const ma_ctx* ctx, ma_pipeline* p) {
    if (!ctx || !p) return MA_ERR_ARG;
    *p = ctx->pipeline;
    return MA_OK;
}

int ma_ctx_get_tuning(const ma_ctx* ctx, ma_tuning* t) {
    if (!ctx || !t) return MA_ERR_ARG;
    *t = ctx->tuning;
    return MA_OK;
}

int ma_ctx_wave_ms(const ma_ctx* ctx, float* out5) {
    if (!ctx || !out5) return MA_ERR_ARG;
    for (int i = 0; i < 5; ++i) out5[i] = ctx->wave_ms[i];
    return MA_OK;
}

int ma_ctx_traffic_stage2(const ma_ctx* ctx, uint64_t* out12) {
    if (!ctx || !out12) return MA_ERR_ARG;
    for (int i = 0; i < 12; ++i) out12[i] = ctx->traffic_stage2[i];
    return MA_OK;
}

int ma_ctx_kernel_ms(const ma_ctx* ctx, float* out4) {
    if (!ctx || !out4) return MA_ERR_ARG;
    for (int i = 0; i < 4; ++i) out4[i] = ctx->kernel_ms[i];
    return MA_OK;
}

int ma_ctx_traffic(const ma_ctx* ctx, uint64_t* out12) {
    if (!ctx || !out12) return MA_ERR_ARG;
    for (int i = 0; i < 12; ++i) out12[i] = ctx->traffic[i];
    return MA_OK;
}

int ma_bench_gather(ma_ctx* ctx, uint64_t buffer_bytes, int line_bytes, uint64_t n_loads, double* gbps) {
    if (!ctx || !gbps) return MA_ERR_ARG;
    return guarded(ctx, [&] {
        use_device(ctx);
        int sms = 0;
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device), "attribute");
        *gbps = run_gather_bench(buffer_bytes, line_bytes, n_loads, sms, ctx->stream);
    });
}

int ma_synth_reference(const char* fasta_out, uint64_t total_len, int n_contigs, double gc, double cpg,
                       uint64_t seed) {
    char err[512] = {0};
    int rc = ma_synth_reference_impl(fasta_out, total_len, n_contigs, gc, cpg, seed, err, sizeof err);
    if (rc != MA_OK) t_err = err;
    return rc;
}

int ma_synth_reference_model(const char* fasta_out, uint64_t total_len, int n_contigs, double gc, double cpg,
                             uint64_t seed, const ma_repeat_model* rm) {
    char err[512] = {0};
    int rc = ma_synth_reference_model_impl(fasta_out, total_len, n_contigs, gc, cpg, seed, rm, err, sizeof err);
    if (rc != MA_OK) t_err = err;
    return rc;
}

int ma_synth_reads(const char* fasta, const ma_read_model* m, uint32_t n1, int paired, uint32_t max_len,
                   uint64_t seed, uint8_t* bases, uint32_t* lens, uint64_t* truth_pos, uint8_t* truth_rev) {
    char err[512] = {0};
    int rc = ma_synth_reads_impl(fasta, m, n1, paired, max_len, seed, bases, lens, truth_pos, truth_rev, err,
                                 sizeof err);
    if (rc != MA_OK) t_err = err;
    return rc;
}

}  // extern "C"
