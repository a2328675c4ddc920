// serve.cu - the served form (ma_serve_*): a request loop over one resident
// index.
//
// Threads: callers submit requests into a FIFO; an issuer thread forms
// launch groups from the pending work (continuous batching), admits each
// against the reserved HBM range (serve_arena.h) and enqueues it on its
// slot's stream; a completer thread waits for groups in issue order,
// scatters their outputs into the callers' arrays and completes requests.
//
// Group layout in the reserved range (all 256-aligned): staged ASCII rows of
// every part, lens[n_seq], part table, packed reads, the 7 output arrays,
// error flag, seed scratch.  The host side of a slot (pinned) holds the
// lens + part table going in and the outputs + error flag coming back, so
// a group costs 2 copies per part (R1 rows, R2 rows) plus one copy each
// way, whatever its number of parts.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ma_device.cuh"
#include "ma_internal.h"
#include "serve_arena.h"

namespace ma {
const DevIndex* index_device_view(const ma_index* idx, int* device);
void ctx_launch_config(const ma_ctx* ctx, int* device, int* sm_count, ma_tuning* tuning);
void set_thread_error(const std::string& msg);
int launch_pack_parts(const uint8_t* d_bases, const uint32_t* d_lens, const PackPart* d_parts, int n_parts,
                      int64_t n_rows, int64_t n1_batch, int words, uint64_t* d_packed, int* d_err, cudaStream_t st);
int launch_seed_extend(const DevIndex& ix, const DevReads& R, const DevParams& P, const DevOut& out,
                       unsigned long long* d_tally, int level, cudaStream_t st);
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

using namespace ma;
using Clock = std::chrono::steady_clock;

namespace {

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

bool same_params(const ma_params& a, const ma_params& b) { return std::memcmp(&a, &b, sizeof a) == 0; }

struct Request {
    uint64_t id = 0;
    const uint8_t* bases = nullptr;
    const uint32_t* lens = nullptr;
    uint32_t n1 = 0, max_len = 0;
    bool paired = false;
    int bs_r1 = 0, bs_r2 = 0;
    ma_params p{};
    ma_hits out{};
    uint32_t issued = 0;  // pairs handed to groups
    uint32_t done = 0;    // pairs whose group has completed
    int status = MA_OK;
    bool complete = false;
    Clock::time_point t_submit, t_done;
    int mates() const { return paired ? 2 : 1; }
};
using RequestPtr = std::shared_ptr<Request>;

struct Part {
    RequestPtr rq;
    uint32_t a = 0, c = 0;  // request pairs [a, a + c)
    uint32_t dst = 0;       // batch pair offset
    uint64_t src = 0;       // offset of its staged rows in the bases area
};

// Byte layout of one launch group inside its arena block.
struct GroupLayout {
    uint64_t bases = 0, lens = 0, parts = 0, packed = 0, out[7] = {0, 0, 0, 0, 0, 0, 0}, scratch = 0, err = 0;
    uint64_t total = 0;
};

struct Group {
    uint64_t seq = 0;
    std::vector<Part> parts;
    uint32_t n1 = 0;
    bool paired = false;
    ma_params p{};
    int words = 1;
    uint64_t off = OffsetArena::kFail;  // arena block
    GroupLayout L;
    int slot = 0;
    int status = MA_OK;
    std::string err;
    int64_t n_seq() const { return paired ? 2 * static_cast<int64_t>(n1) : n1; }
};

uint64_t rnd(uint64_t n) { return OffsetArena::round_up(n); }

// Lays out a group of n1 pairs with `stage_bytes` of staged rows over
// `n_parts` parts.
GroupLayout layout_for(uint32_t n1, bool paired, int words, uint64_t stage_bytes, size_t n_parts,
                       const ma_tuning& t) {
    const int seed_kernel = t.seed_kernel;
    const uint64_t n_seq = paired ? 2ull * n1 : n1;
    GroupLayout L;
    uint64_t o = 0;
    L.bases = o;
    o += rnd(stage_bytes);
    L.lens = o;
    o += rnd(n_seq * 4);
    L.parts = o;
    o += rnd(n_parts * sizeof(PackPart));
    L.packed = o;
    o += rnd(n_seq * 4 * static_cast<uint64_t>(words) * 8);
    for (int f = 0; f < 7; ++f) {  // outputs then the error flag: one copy back
        L.out[f] = o;
        o += rnd(n_seq * 4);
    }
    L.err = o;
    o += OffsetArena::kAlign;
    L.scratch = o;
    if (seed_kernel == 1) o += rnd(two_stage_scratch_bytes(static_cast<int64_t>(n_seq)));
    if (seed_kernel >= 2) o += rnd(wavefront_scratch_bytes(static_cast<int64_t>(n_seq), t.wave_loci_per_read));
    L.total = o;
    return L;
}

// Host staging of one in-flight slot (pinned unless in scheduler-test
// mode): lens and part table in, outputs and error flag out.
struct HostSlot {
    char* in = nullptr;   // lens[n_seq] then PackPart[parts]
    char* out = nullptr;  // 7 x n_seq x 4 bytes, then the error flag
    size_t in_cap = 0, out_cap = 0;
};

}  // namespace

struct ma_server {
    bool test_mode = false;
    int device = 0, sm_count = 0;
    ma_tuning tuning{2, 1, 0, 2, 1, 1, 8, 4, 0, 1};
    const DevIndex* dix = nullptr;
    ma_serve_options opt{};
    char* base = nullptr;  // reserved device range (host memory in test mode)
    OffsetArena arena;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> done_ev;
    std::vector<HostSlot> hslot;

    std::mutex mu;
    std::condition_variable cv_issue, cv_complete, cv_done;
    std::deque<RequestPtr> pending;  // requests with pairs not yet issued, arrival order
    std::unordered_map<uint64_t, RequestPtr> reqs;
    std::deque<std::unique_ptr<Group>> inflight;  // issue order
    uint32_t n_inflight = 0;      // committed groups not yet completed
    uint64_t next_id = 1, group_seq = 0, groups_done = 0;
    uint64_t open_requests = 0;   // submitted, not complete
    bool stop = false;
    int broken = MA_OK;           // sticky device failure
    std::string err;
    ma_serve_stats stats{};
    std::vector<uint64_t> lat_id, lat_reads;
    std::vector<double> lat_ms;
    std::thread issuer, completer;

    int seed_kernel() const { return tuning.seed_kernel; }
};

namespace {

int words_for(uint32_t max_len) { return static_cast<int>((max_len + 31) / 32); }

// Next launch group from the pending work: requests in arrival order that
// match the oldest one's `paired` and parameters, up to `cap` pairs.  Does
// not change any request.
std::unique_ptr<Group> plan_group(ma_server* s, uint32_t cap) {
    auto g = std::make_unique<Group>();
    const RequestPtr& head = s->pending.front();
    g->paired = head->paired;
    g->p = head->p;
    uint64_t stage = 0;
    int words = 1;
    for (const RequestPtr& rq : s->pending) {
        if (rq->paired != head->paired || !same_params(rq->p, head->p)) continue;
        const uint32_t rem = rq->n1 - rq->issued;
        if (rem == 0) continue;
        const uint32_t c = std::min(rem, cap - g->n1);
        Part pt;
        pt.rq = rq;
        pt.a = rq->issued;
        pt.c = c;
        pt.dst = g->n1;
        pt.src = stage;
        stage += rnd(static_cast<uint64_t>(rq->mates()) * c * rq->max_len);
        words = std::max(words, words_for(rq->max_len));
        g->parts.push_back(pt);
        g->n1 += c;
        if (g->n1 == cap) break;
    }
    g->words = words;
    g->L = layout_for(g->n1, g->paired, words, stage, g->parts.size(), s->tuning);
    return g;
}

// FNV-1a of the converted read (scheduler-test mapping).
uint32_t fnv_converted(const uint8_t* row, int len, int mode) {
    uint32_t h = 2166136261u;
    for (int j = 0; j < len; ++j) {
        uint8_t c = row[j];
        if (mode == MA_BS_C2T && (c == 'C' || c == 'c')) c = 'T';
        if (mode == MA_BS_G2A && (c == 'G' || c == 'g')) c = 'A';
        h = (h ^ c) * 16777619u;
    }
    return h;
}

// Scheduler-test mode: the group's "kernels", run on the host over the same
// layout the device path uses.
void run_test_group(ma_server* s, Group& g, char* dev) {
    const int64_t n_seq = g.n_seq();
    const uint32_t* lens = reinterpret_cast<const uint32_t*>(dev + g.L.lens);
    const PackPart* parts = reinterpret_cast<const PackPart*>(dev + g.L.parts);
    std::vector<uint32_t> hash(static_cast<size_t>(n_seq), 0);
    std::vector<uint8_t> second(static_cast<size_t>(n_seq), 0);
    int* err = reinterpret_cast<int*>(dev + g.L.err);
    for (size_t j = 0; j < g.parts.size(); ++j) {
        const PackPart& pp = parts[j];
        const int64_t rows = static_cast<int64_t>(pp.c) * (g.paired ? 2 : 1);
        for (int64_t local = 0; local < rows; ++local) {
            const bool sec = local >= pp.c;
            const int64_t i = sec ? local - pp.c : local;
            const int64_t d = sec ? g.n1 + pp.dst + i : pp.dst + i;
            int len = static_cast<int>(lens[d]);
            if (len > static_cast<int>(pp.max_len)) {
                *err = 1;
                len = static_cast<int>(pp.max_len);
            }
            hash[d] = fnv_converted(reinterpret_cast<const uint8_t*>(dev + g.L.bases + pp.src) + local * pp.max_len,
                                    len, sec ? pp.bs_r2 : pp.bs_r1);
            second[d] = sec;
        }
    }
    for (int64_t d = 0; d < n_seq; ++d) {
        reinterpret_cast<int32_t*>(dev + g.L.out[0])[d] = static_cast<int32_t>(lens[d]);
        reinterpret_cast<uint32_t*>(dev + g.L.out[1])[d] = hash[d];
        reinterpret_cast<uint32_t*>(dev + g.L.out[2])[d] = static_cast<uint32_t>(g.p.seed_len);
        reinterpret_cast<int32_t*>(dev + g.L.out[3])[d] = second[d] ? 128 : 0;
        reinterpret_cast<uint32_t*>(dev + g.L.out[4])[d] = 0;
        reinterpret_cast<uint32_t*>(dev + g.L.out[5])[d] = 0;
        const int64_t mate = d < g.n1 ? d + g.n1 : d - g.n1;
        reinterpret_cast<uint32_t*>(dev + g.L.out[6])[d] = g.paired ? hash[mate] : 0;
    }
    (void)s;
}

DevParams dev_params(const ma_params& p) {
    DevParams d;
    d.seed_len = p.seed_len;
    d.seed_stride = p.seed_stride;
    d.max_occ = p.max_occ;
    d.max_diff = p.max_diff;
    d.max_soft = p.max_soft;
    d.max_adj = p.max_adj;
    d.rescue_win = p.rescue_win;
    return d;
}

// Enqueues one group: rows in, pack, seed/extend, rescue, outputs back.
// Test mode does the same moves on the host and runs run_test_group.
void issue_group(ma_server* s, Group& g) {
    HostSlot& hs = s->hslot[static_cast<size_t>(g.slot)];
    char* dev = s->base + g.off;
    const int64_t n_seq = g.n_seq();
    const uint64_t lens_bytes = rnd(static_cast<uint64_t>(n_seq) * 4);
    uint32_t* hl = reinterpret_cast<uint32_t*>(hs.in);
    PackPart* hp = reinterpret_cast<PackPart*>(hs.in + lens_bytes);
    const uint64_t in_bytes = lens_bytes + g.parts.size() * sizeof(PackPart);
    const uint64_t out_stride = rnd(static_cast<uint64_t>(n_seq) * 4);
    const uint64_t out_bytes = 7 * out_stride + sizeof(int);
    if (in_bytes > hs.in_cap || out_bytes > hs.out_cap) fail(MA_ERR_INTERNAL, "group exceeds its host staging");
    cudaStream_t st = s->test_mode ? nullptr : s->streams[static_cast<size_t>(g.slot)];
    int64_t row0 = 0;
    for (size_t j = 0; j < g.parts.size(); ++j) {
        const Part& pt = g.parts[j];
        const Request& rq = *pt.rq;
        const size_t rows_bytes = static_cast<size_t>(pt.c) * rq.max_len;
        std::memcpy(hl + pt.dst, rq.lens + pt.a, pt.c * 4ull);
        if (g.paired) std::memcpy(hl + g.n1 + pt.dst, rq.lens + rq.n1 + pt.a, pt.c * 4ull);
        PackPart pp{};
        pp.src = pt.src;
        pp.row0 = row0;
        pp.c = pt.c;
        pp.max_len = rq.max_len;
        pp.bs_r1 = rq.bs_r1;
        pp.bs_r2 = rq.bs_r2;
        pp.dst = pt.dst;
        hp[j] = pp;
        row0 += static_cast<int64_t>(pt.c) * rq.mates();
        const uint8_t* r1 = rq.bases + static_cast<size_t>(pt.a) * rq.max_len;
        const uint8_t* r2 = rq.bases + (static_cast<size_t>(rq.n1) + pt.a) * rq.max_len;
        if (s->test_mode) {
            std::memcpy(dev + g.L.bases + pt.src, r1, rows_bytes);
            if (g.paired) std::memcpy(dev + g.L.bases + pt.src + rows_bytes, r2, rows_bytes);
        } else {
            ck(cudaMemcpyAsync(dev + g.L.bases + pt.src, r1, rows_bytes, cudaMemcpyHostToDevice, st), "H2D rows");
            if (g.paired)
                ck(cudaMemcpyAsync(dev + g.L.bases + pt.src + rows_bytes, r2, rows_bytes, cudaMemcpyHostToDevice, st),
                   "H2D rows");
        }
    }
    if (s->test_mode) {
        std::memcpy(dev + g.L.lens, hs.in, in_bytes);
        std::memset(dev + g.L.err, 0, sizeof(int));
        run_test_group(s, g, dev);
        std::memcpy(hs.out, dev + g.L.out[0], out_bytes);
        return;
    }
    // lens and the part table are adjacent on both sides: one copy
    ck(cudaMemcpyAsync(dev + g.L.lens, hs.in, in_bytes, cudaMemcpyHostToDevice, st), "H2D lens");
    ck(cudaMemsetAsync(dev + g.L.err, 0, sizeof(int), st), "memset");
    uint64_t* packed = reinterpret_cast<uint64_t*>(dev + g.L.packed);
    const uint32_t* d_lens = reinterpret_cast<const uint32_t*>(dev + g.L.lens);
    int* d_err = reinterpret_cast<int*>(dev + g.L.err);
    launch_pack_parts(reinterpret_cast<const uint8_t*>(dev + g.L.bases), d_lens,
                      reinterpret_cast<const PackPart*>(dev + g.L.parts), static_cast<int>(g.parts.size()), row0, g.n1,
                      g.words, packed, d_err, st);
    DevReads R{packed, d_lens, g.words, n_seq};
    DevOut o{reinterpret_cast<int32_t*>(dev + g.L.out[0]), reinterpret_cast<uint32_t*>(dev + g.L.out[1]),
             reinterpret_cast<uint32_t*>(dev + g.L.out[2]), reinterpret_cast<int32_t*>(dev + g.L.out[3]),
             reinterpret_cast<uint32_t*>(dev + g.L.out[4]), reinterpret_cast<uint32_t*>(dev + g.L.out[5]),
             reinterpret_cast<uint32_t*>(dev + g.L.out[6]), nullptr, nullptr, nullptr, nullptr, nullptr};
    const DevParams P = dev_params(g.p);
    const ma_tuning& t = s->tuning;
    const int bps = t.stage2_blocks_per_sm > 0 ? t.stage2_blocks_per_sm : stage2_blocks_per_sm(t.reg_level, false);
    if (s->seed_kernel() == 1) {
        launch_seed_two_stage(*s->dix, R, P, o, t.stage1_endpoints, t.stage1_max_rows, bps * s->sm_count, t.reg_level,
                              t.stage2_first_wave, dev + g.L.scratch, nullptr, nullptr, st);
    } else if (s->seed_kernel() >= 2) {
        launch_seed_wavefront(*s->dix, R, P, o, 32 * g.words, t, bps * s->sm_count, dev + g.L.scratch, s->sm_count,
                              d_err, nullptr, nullptr, st);
    } else {
        launch_seed_extend(*s->dix, R, P, o, nullptr, t.reg_level, st);
    }
    if (g.paired && g.p.rescue_win > 0) launch_rescue(*s->dix, R, P, o, g.n1, st);
    ck(cudaGetLastError(), "kernel launch");
    ck(cudaMemcpyAsync(hs.out, dev + g.L.out[0], out_bytes, cudaMemcpyDeviceToHost, st), "D2H outputs");
    ck(cudaEventRecord(s->done_ev[static_cast<size_t>(g.slot)], st), "cudaEventRecord");
}

void finish_request(ma_server* s, Request& rq) {
    rq.complete = true;
    rq.t_done = Clock::now();
    --s->open_requests;
    if (rq.status == MA_OK) {
        ++s->stats.requests_completed;
        s->stats.reads_completed += static_cast<uint64_t>(rq.n1) * rq.mates();
    } else {
        ++s->stats.requests_failed;
    }
    s->lat_id.push_back(rq.id);
    s->lat_reads.push_back(static_cast<uint64_t>(rq.n1) * rq.mates());
    s->lat_ms.push_back(std::chrono::duration<double, std::milli>(rq.t_done - rq.t_submit).count());
}

// Marks the rest of a request failed (its pairs not yet issued are dropped).
// Caller holds the lock.
void fail_request(ma_server* s, Request& rq, int code, const std::string& msg) {
    if (rq.status == MA_OK) rq.status = code;
    s->err = msg;
    const uint32_t dropped = rq.n1 - rq.issued;
    rq.issued = rq.n1;
    rq.done += dropped;
}

void drop_exhausted(ma_server* s) {
    s->pending.erase(std::remove_if(s->pending.begin(), s->pending.end(),
                                    [](const RequestPtr& r) { return r->issued == r->n1; }),
                     s->pending.end());
}

void issuer_loop(ma_server* s) {
    if (!s->test_mode) cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_issue.wait(lk, [&] { return s->stop || (!s->pending.empty() && s->n_inflight < s->opt.max_inflight); });
        if (s->stop) return;
        uint32_t cap = s->opt.max_group_pairs;
        std::unique_ptr<Group> g;
        bool waited = false;
        while (!s->pending.empty()) {
            g = plan_group(s, cap);
            g->off = s->arena.alloc(g->L.total);
            if (g->off != OffsetArena::kFail) break;
            g.reset();
            if (s->n_inflight > 0) {
                // admission: wait for a group in flight to return its memory
                ++s->stats.admission_waits;
                const uint64_t before = s->groups_done;
                s->cv_issue.wait(lk, [&] { return s->stop || s->groups_done != before; });
                if (s->stop) return;
                waited = true;
                break;
            }
            if (cap > 1) {
                cap = std::max(1u, cap / 2);
                continue;
            }
            // nothing in flight and one pair does not fit (submit checks
            // this, so only a budget far below one pair's needs gets here)
            RequestPtr head = s->pending.front();
            fail_request(s, *head, MA_ERR_NOMEM, "one pair of a request exceeds the server's HBM budget");
            drop_exhausted(s);
            if (head->done == head->n1 && !head->complete) finish_request(s, *head);
            s->cv_done.notify_all();
        }
        if (waited || !g) continue;
        for (const Part& pt : g->parts) pt.rq->issued += pt.c;
        drop_exhausted(s);
        g->seq = s->group_seq++;
        g->slot = static_cast<int>(g->seq % s->opt.max_inflight);
        ++s->n_inflight;
        ++s->stats.groups_issued;
        s->stats.parts_issued += g->parts.size();
        s->stats.max_requests_in_group = std::max<uint64_t>(s->stats.max_requests_in_group, g->parts.size());
        s->stats.max_groups_in_flight = std::max<uint64_t>(s->stats.max_groups_in_flight, s->n_inflight);
        s->stats.peak_bytes = s->arena.peak();
        Group* gp = g.get();
        const int broken = s->broken;
        lk.unlock();
        try {
            if (broken != MA_OK) fail(broken, "server stopped after a device failure");
            issue_group(s, *gp);
        } catch (const Error& e) {
            gp->status = e.code;
            gp->err = e.what();
        } catch (const std::exception& e) {
            gp->status = MA_ERR_INTERNAL;
            gp->err = e.what();
        }
        lk.lock();
        if (gp->status == MA_ERR_CUDA) s->broken = MA_ERR_CUDA;
        s->inflight.push_back(std::move(g));
        s->cv_complete.notify_one();
    }
}

void completer_loop(ma_server* s) {
    if (!s->test_mode) cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_complete.wait(lk, [&] { return s->stop || !s->inflight.empty(); });
        if (s->inflight.empty()) return;  // stop with nothing in flight
        Group* g = s->inflight.front().get();
        lk.unlock();
        const HostSlot& hs = s->hslot[static_cast<size_t>(g->slot)];
        const uint64_t out_stride = rnd(static_cast<uint64_t>(g->n_seq()) * 4);
        if (g->status == MA_OK && !s->test_mode) {
            const cudaError_t e = cudaEventSynchronize(s->done_ev[static_cast<size_t>(g->slot)]);
            if (e != cudaSuccess) {
                g->status = MA_ERR_CUDA;
                g->err = std::string("mapping kernels: ") + cudaGetErrorString(e);
            }
        }
        if (g->status == MA_OK) {
            int flag = 0;
            std::memcpy(&flag, hs.out + 7 * out_stride, sizeof flag);
            if (flag == 1) {
                g->status = MA_ERR_ARG;
                g->err = "a read length exceeds max_len";
            } else if (flag) {
                g->status = MA_ERR_INTERNAL;
                g->err = "device error flag " + std::to_string(flag);
            }
        }
        if (g->status == MA_OK) {
            // scatter the batch rows back to each request's rows
            for (const Part& pt : g->parts) {
                Request& rq = *pt.rq;
                void* dst[7] = {rq.out.rid, rq.out.pos, rq.out.mapq, rq.out.flag, rq.out.sl, rq.out.sr, rq.out.nm};
                for (int f = 0; f < 7; ++f) {
                    const char* src = hs.out + f * out_stride;
                    std::memcpy(static_cast<char*>(dst[f]) + 4ull * pt.a, src + 4ull * pt.dst, 4ull * pt.c);
                    if (g->paired)
                        std::memcpy(static_cast<char*>(dst[f]) + 4ull * (static_cast<uint64_t>(rq.n1) + pt.a),
                                    src + 4ull * (static_cast<uint64_t>(g->n1) + pt.dst), 4ull * pt.c);
                }
            }
        }
        lk.lock();
        s->arena.release(g->off, g->L.total);
        for (const Part& pt : g->parts) {
            Request& rq = *pt.rq;
            if (g->status != MA_OK) fail_request(s, rq, g->status, g->err);
            rq.done += pt.c;
            if (rq.done == rq.n1 && !rq.complete) finish_request(s, rq);
        }
        if (g->status != MA_OK) drop_exhausted(s);
        if (g->status == MA_ERR_CUDA) s->broken = MA_ERR_CUDA;
        s->inflight.pop_front();
        --s->n_inflight;
        ++s->groups_done;
        s->cv_issue.notify_all();
        s->cv_done.notify_all();
    }
}

bool valid_hits(const ma_hits* o) {
    return o && o->rid && o->pos && o->mapq && o->flag && o->sl && o->sr && o->nm;
}

}  // namespace

namespace {
void destroy_resources(ma_server* s) {
    for (HostSlot& h : s->hslot) {
        if (s->test_mode) {
            std::free(h.in);
            std::free(h.out);
        } else {
            if (h.in) cudaFreeHost(h.in);
            if (h.out) cudaFreeHost(h.out);
        }
    }
    s->hslot.clear();
    for (cudaEvent_t e : s->done_ev)
        if (e) cudaEventDestroy(e);
    for (cudaStream_t st : s->streams)
        if (st) cudaStreamDestroy(st);
    if (s->base) {
        if (s->test_mode) std::free(s->base);
        else cudaFree(s->base);
    }
    s->base = nullptr;
}

template <typename F>
int serve_guarded(ma_server* s, F&& f) {
    try {
        f();
        return MA_OK;
    } catch (const Error& e) {
        if (s) {
            std::lock_guard<std::mutex> lk(s->mu);
            s->err = e.what();
        }
        set_thread_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_thread_error("host out of memory");
        return MA_ERR_NOMEM;
    } catch (const std::exception& e) {
        set_thread_error(e.what());
        return MA_ERR_INTERNAL;
    }
}
}  // namespace

extern "C" {

void ma_serve_options_default(ma_serve_options* o) {
    if (!o) return;
    o->hbm_budget_bytes = 0;
    o->max_group_pairs = 262144;
    o->max_inflight = 3;
    o->flags = 0;
}


int ma_serve_create(ma_ctx* ctx, const ma_index* idx, const ma_serve_options* opt, ma_server** out) {
    if (!out) return MA_ERR_ARG;
    *out = nullptr;
    auto* s = new ma_server();
    ma_serve_options_default(&s->opt);
    if (opt) s->opt = *opt;
    s->test_mode = (s->opt.flags & MA_SERVE_SCHEDULER_TEST) != 0;
    const int rc = serve_guarded(nullptr, [&] {
        if (s->opt.max_group_pairs < 1 || s->opt.max_group_pairs > (1u << 24))
            fail(MA_ERR_ARG, "max_group_pairs must be in 1..16777216");
        if (s->opt.max_inflight < 1 || s->opt.max_inflight > 8) fail(MA_ERR_ARG, "max_inflight must be in 1..8");
        const size_t G = s->opt.max_group_pairs;
        const size_t in_cap = rnd(2 * G * 4) + G * sizeof(PackPart);
        const size_t out_cap = 7 * rnd(2 * G * 4) + sizeof(int);
        if (s->test_mode) {
            if (s->opt.hbm_budget_bytes == 0) fail(MA_ERR_ARG, "scheduler-test mode needs an explicit budget");
            if (s->opt.hbm_budget_bytes > (1ull << 32)) fail(MA_ERR_ARG, "scheduler-test budget above 4 GiB");
            s->tuning.seed_kernel = 1;
            s->base = static_cast<char*>(std::malloc(s->opt.hbm_budget_bytes));
            if (!s->base) fail(MA_ERR_NOMEM, "host out of memory");
            s->arena.reset(s->opt.hbm_budget_bytes);
            s->hslot.resize(s->opt.max_inflight);
            for (HostSlot& h : s->hslot) {
                h.in = static_cast<char*>(std::malloc(in_cap));
                h.out = static_cast<char*>(std::malloc(out_cap));
                if (!h.in || !h.out) fail(MA_ERR_NOMEM, "host out of memory");
                h.in_cap = in_cap;
                h.out_cap = out_cap;
            }
        } else {
            if (!ctx || !idx) fail(MA_ERR_ARG, "null context or index");
            int idx_dev = -1;
            s->dix = index_device_view(idx, &idx_dev);
            ctx_launch_config(ctx, &s->device, &s->sm_count, &s->tuning);
            if (!s->dix || idx_dev != s->device) fail(MA_ERR_ARG, "index belongs to another device");
            ck(cudaSetDevice(s->device), "cudaSetDevice");
            size_t f = 0, t = 0;
            ck(cudaMemGetInfo(&f, &t), "cudaMemGetInfo");
            uint64_t budget = s->opt.hbm_budget_bytes;
            if (budget == 0) budget = std::min<uint64_t>(f / 4, 16ull << 30);
            if (budget + (256ull << 20) > f)
                fail(MA_ERR_NOMEM, "serving budget " + std::to_string(budget >> 20) + " MiB exceeds free HBM (" +
                                       std::to_string(f >> 20) + " MiB)");
            s->opt.hbm_budget_bytes = budget;
            ck(cudaMalloc(reinterpret_cast<void**>(&s->base), budget), "cudaMalloc serving budget");
            s->arena.reset(budget);
            s->streams.resize(s->opt.max_inflight, nullptr);
            s->done_ev.resize(s->opt.max_inflight, nullptr);
            s->hslot.resize(s->opt.max_inflight);
            for (uint32_t i = 0; i < s->opt.max_inflight; ++i) {
                ck(cudaStreamCreateWithFlags(&s->streams[i], cudaStreamNonBlocking), "cudaStreamCreate");
                ck(cudaEventCreateWithFlags(&s->done_ev[i], cudaEventDisableTiming), "cudaEventCreate");
                ck(cudaHostAlloc(reinterpret_cast<void**>(&s->hslot[i].in), in_cap, cudaHostAllocDefault),
                   "cudaHostAlloc");
                ck(cudaHostAlloc(reinterpret_cast<void**>(&s->hslot[i].out), out_cap, cudaHostAllocDefault),
                   "cudaHostAlloc");
                s->hslot[i].in_cap = in_cap;
                s->hslot[i].out_cap = out_cap;
            }
        }
        s->stats.budget_bytes = s->arena.capacity();
        s->issuer = std::thread(issuer_loop, s);
        s->completer = std::thread(completer_loop, s);
    });
    if (rc != MA_OK) {
        destroy_resources(s);
        delete s;
        return rc;
    }
    *out = s;
    return MA_OK;
}

int ma_serve_submit(ma_server* s, const uint8_t* bases, const uint32_t* lens, uint32_t n1, int paired,
                    uint32_t max_len, int bs_r1, int bs_r2, const ma_params* p, const ma_hits* out,
                    uint64_t* request_id) {
    if (!s || !request_id) return MA_ERR_ARG;
    return serve_guarded(s, [&] {
        if (!p) fail(MA_ERR_ARG, "params must not be NULL");
        if (p->seed_len < 1 || p->seed_len > MAX_READ_LEN) fail(MA_ERR_ARG, "seed_len must be in 1..1024");
        if (p->seed_stride < 1) fail(MA_ERR_ARG, "seed_stride must be >= 1");
        if (p->max_occ < 1) fail(MA_ERR_ARG, "max_occ must be >= 1");
        if (max_len < 1 || max_len > static_cast<uint32_t>(MAX_READ_LEN)) fail(MA_ERR_ARG, "max_len must be in 1..1024");
        if (bs_r1 < 0 || bs_r1 > 2 || bs_r2 < 0 || bs_r2 > 2) fail(MA_ERR_ARG, "bad bisulfite mode");
        if (!valid_hits(out)) fail(MA_ERR_ARG, "null output array");
        if (n1 && (!bases || !lens)) fail(MA_ERR_ARG, "null argument");
        const int mates = paired ? 2 : 1;
        const uint64_t n_seq = static_cast<uint64_t>(n1) * mates;
        for (uint64_t i = 0; i < n_seq; ++i)
            if (lens[i] > max_len) fail(MA_ERR_ARG, "read " + std::to_string(i) + " longer than max_len");
        const GroupLayout one = layout_for(1, paired != 0, words_for(max_len), rnd(static_cast<uint64_t>(mates) * max_len),
                                           1, s->tuning);
        if (one.total > s->arena.capacity())
            fail(MA_ERR_NOMEM, "one pair needs " + std::to_string(one.total) + " bytes, over the serving budget");
        auto rq = std::make_shared<Request>();
        rq->bases = bases;
        rq->lens = lens;
        rq->n1 = n1;
        rq->paired = paired != 0;
        rq->max_len = max_len;
        rq->bs_r1 = bs_r1;
        rq->bs_r2 = bs_r2;
        rq->p = *p;
        rq->out = *out;
        rq->t_submit = Clock::now();
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->broken != MA_OK) fail(s->broken, "server stopped after a device failure: " + s->err);
        if (s->stop) fail(MA_ERR_ARG, "server is shutting down");
        rq->id = s->next_id++;
        s->reqs[rq->id] = rq;
        ++s->stats.requests_submitted;
        ++s->open_requests;
        if (n1 == 0) {
            finish_request(s, *rq);
        } else {
            s->pending.push_back(rq);
            s->cv_issue.notify_one();
        }
        *request_id = rq->id;
    });
}

int ma_serve_poll(ma_server* s, uint64_t request_id, int* done) {
    if (!s || !done) return MA_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return MA_ERR_ARG;
    *done = it->second->complete ? 1 : 0;
    return it->second->complete ? it->second->status : MA_OK;
}

int ma_serve_wait(ma_server* s, uint64_t request_id, int timeout_ms) {
    if (!s) return MA_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return MA_ERR_ARG;
    RequestPtr rq = it->second;
    auto pred = [&] { return rq->complete; };
    if (timeout_ms < 0) s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) return MA_ERR_TIMEOUT;
    return rq->status;
}

int ma_serve_drain(ma_server* s, int timeout_ms) {
    if (!s) return MA_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto pred = [&] { return s->open_requests == 0; };
    if (timeout_ms < 0) s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) return MA_ERR_TIMEOUT;
    return s->stats.requests_failed ? MA_ERR_INTERNAL : MA_OK;
}

int ma_serve_get_stats(ma_server* s, ma_serve_stats* out) {
    if (!s || !out) return MA_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    out->peak_bytes = s->arena.peak();
    return MA_OK;
}

int ma_serve_latencies(ma_server* s, uint64_t* ids, uint64_t* reads, double* ms, uint64_t cap, uint64_t* count) {
    if (!s || !count) return MA_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    const uint64_t n = s->lat_ms.size();
    *count = n;
    const uint64_t m = std::min(cap, n);
    for (uint64_t i = 0; i < m; ++i) {
        if (ids) ids[i] = s->lat_id[i];
        if (reads) reads[i] = s->lat_reads[i];
        if (ms) ms[i] = s->lat_ms[i];
    }
    return MA_OK;
}

const char* ma_serve_last_error(const ma_server* s) { return s ? s->err.c_str() : ""; }

void ma_serve_destroy(ma_server* s) {
    if (!s) return;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_done.wait(lk, [&] { return s->open_requests == 0; });
        s->stop = true;
    }
    s->cv_issue.notify_all();
    s->cv_complete.notify_all();
    if (s->issuer.joinable()) s->issuer.join();
    if (s->completer.joinable()) s->completer.join();
    if (!s->test_mode) cudaSetDevice(s->device);
    destroy_resources(s);
    delete s;
}

}  // extern "C"
