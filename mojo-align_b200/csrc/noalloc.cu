// noalloc.cu - a mapping entry point that allocates no device memory.
//
// Some callers of this library cannot let it call cudaMalloc: a framework
// whose caching allocator has already reserved the free HBM (a cudaMalloc
// would fail or fragment its pool), or a latency-bound serving loop that
// shares the GPU with other streams, where cudaMalloc's implicit device
// synchronisation would stall them.  ma_map_batch_device_noalloc serves
// them: it runs the same pack -> two-stage seed/extend -> rescue kernels as
// ma_map_batch_device, but takes its scratch (the packed reads, the stage-1
// to stage-2 hand-off and the device error flag) from one file-scope
// __device__ array of fixed size instead of the context's pool.
//
// The array belongs to this file's module.  Under CUDA's default lazy
// module loading (CUDA_MODULE_LOADING=LAZY) the module, and with it the
// array, is loaded on a device the first time this entry point runs there;
// with CUDA_MODULE_LOADING=EAGER it is loaded with the library.  Either way
// it stays on every device it was loaded on until the process exits.  The
// first call on a device is the set-up: with that device current it looks
// up the array's device address (cudaGetSymbolAddress) and loads the
// kernels the call runs, both of which can take device memory, as can the
// first launch of a kernel (the driver sizes its local memory then).  A call
// with n1 = 0 does the set-up and launches every kernel over zero reads, so a
// caller can make it before its caching allocator reserves the free HBM;
// make it before any stream capture too.  Each call is synchronous (it
// reads the device error word back) and puts the caller's current device
// back on return.  All calls share the array and it keeps the previous
// call's contents, so everything that must start at zero is cleared by each
// call, and calls whose kernels overlap on the GPU (different streams, or
// host threads without ordering) race on it.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "ma_device.cuh"
#include "ma_internal.h"

namespace ma {
const DevIndex* index_device_view(const ma_index* idx, int* device);
void set_thread_error(const std::string& msg);
int launch_pack(const uint8_t* d_bases, const uint32_t* d_lens, int64_t n_seq, int64_t n1, int max_len, int words,
                int bs_r1, int bs_r2, uint64_t* d_packed, int* d_err, cudaStream_t st);
size_t two_stage_scratch_bytes(int64_t n_seq);
int launch_seed_two_stage(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out,
                          int stage1_endpoints, int stage1_max_rows, int stage2_blocks, int level,
                          int first_wave, void* scratch, unsigned long long* d_tally, cudaEvent_t mid,
                          cudaStream_t st);
int stage2_blocks_per_sm(int level, bool counting);
int launch_rescue(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out, int64_t n_pairs,
                  cudaStream_t st);
void load_noalloc_kernels(int level);
}  // namespace ma

using namespace ma;

namespace {

// Largest batch the static scratch holds: one reference batch of 16384
// read pairs (METHYLGRAPHER_LINEAR_READ_BATCH default) with reads of up
// to 256 bases.
constexpr int64_t kMaxReads = 32768;
constexpr int kMaxLen = 256;
constexpr size_t kPackedBytes = static_cast<size_t>(kMaxReads) * 4 * (kMaxLen / 32) * 8;  // 8 MiB
constexpr size_t kHandoffBytes = 3u << 20;                                                 // >= 2.6 MiB needed
constexpr size_t kErrBytes = 256;
constexpr size_t kScratchBytes = kPackedBytes + kHandoffBytes + kErrBytes;  // about 11 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_addr[64] = {};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

constexpr int kLevel = 2;  // register budget of the seed kernels this entry point runs

// Set-up on `device` (which must be current), once: the device address of
// the scratch array and the kernels of the call, loaded now so that later
// calls load no module.
void* scratch_on(int device) {
    if (device < 0 || device >= 64) fail(MA_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        ck(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(static scratch)");
        load_noalloc_kernels(kLevel);
        ck(cudaGetLastError(), "loading the mapping kernels");
        g_scratch_addr[device] = p;
    }
    return g_scratch_addr[device];
}

// Makes `device` current for the call and puts the caller's device back.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int device) {
        ck(cudaGetDevice(&prev), "cudaGetDevice");
        if (prev != device) ck(cudaSetDevice(device), "cudaSetDevice");
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" int ma_map_batch_device_noalloc(const ma_index* idx, const uint8_t* d_bases, const uint32_t* d_lens,
                                           uint32_t n1, int paired, uint32_t max_len, int bs_r1, int bs_r2,
                                           const ma_params* p, ma_hits* d_out, ma_debug* d_dbg, void* stream) {
    try {
        int device = 0;
        const DevIndex* ix = index_device_view(idx, &device);
        if (!ix || !d_out || !p || (n1 && (!d_bases || !d_lens))) fail(MA_ERR_ARG, "null argument");
        if (p->seed_len < 1 || p->seed_len > MAX_READ_LEN || p->seed_stride < 1 || p->max_occ < 1)
            fail(MA_ERR_ARG, "seed_len must be in 1..1024, seed_stride and max_occ >= 1");
        if (bs_r1 < 0 || bs_r1 > 2 || bs_r2 < 0 || bs_r2 > 2) fail(MA_ERR_ARG, "bad bisulfite mode");
        if (max_len < 1 || max_len > static_cast<uint32_t>(kMaxLen))
            fail(MA_ERR_ARG, "max_len " + std::to_string(max_len) + " exceeds the static scratch maximum of " +
                                 std::to_string(kMaxLen) + " bases; use ma_map_batch_device");
        const int64_t n_seq = paired ? 2 * static_cast<int64_t>(n1) : n1;
        if (n_seq > kMaxReads)
            fail(MA_ERR_ARG, std::to_string(n_seq) + " reads exceed the static scratch maximum of " +
                                 std::to_string(kMaxReads) + " reads per call; split the batch");
        if (two_stage_scratch_bytes(n_seq) > kHandoffBytes) fail(MA_ERR_INTERNAL, "hand-off area too small");
        DeviceGuard on_device(device);
        char* base = static_cast<char*>(scratch_on(device));
        // a call with no reads still launches every kernel of a call (each
        // returns at once), so that the driver sizes their local memory in
        // the set-up call rather than in a later one
        const bool setup_only = n1 == 0;
        uint64_t* packed = reinterpret_cast<uint64_t*>(base);
        void* handoff = base + kPackedBytes;
        int* err = reinterpret_cast<int*>(base + kPackedBytes + kHandoffBytes);
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        int sms = 0;
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
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
        DevParams P{p->seed_len, p->seed_stride, p->max_occ, p->max_diff, p->max_soft, p->max_adj, p->rescue_win};
        const int words = static_cast<int>((max_len + 31) / 32);
        // the error flag and the hand-off counters keep the last call's
        // values: both are cleared on the stream before the kernels run
        ck(cudaMemsetAsync(err, 0, sizeof(int), st), "cudaMemsetAsync");
        launch_pack(d_bases, d_lens, n_seq, n1, static_cast<int>(max_len), words, bs_r1, bs_r2, packed, err, st);
        DevReads R{packed, d_lens, words, n_seq};
        const int level = kLevel;
        launch_seed_two_stage(*ix, R, P, o, 1, 2, stage2_blocks_per_sm(level, false) * sms, level, 32, handoff,
                              nullptr, nullptr, st);
        if (setup_only || (paired && p->rescue_win > 0)) launch_rescue(*ix, R, P, o, n1, st);
        ck(cudaGetLastError(), "kernel launch");
        int h = 0;
        ck(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H error flag");
        ck(cudaStreamSynchronize(st), "mapping kernels");
        if (h == 1) fail(MA_ERR_ARG, "a read length exceeds max_len");
        if (h) fail(MA_ERR_INTERNAL, "device error flag " + std::to_string(h));
        return MA_OK;
    } catch (const Error& e) {
        set_thread_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_thread_error(e.what());
        return MA_ERR_INTERNAL;
    }
}
