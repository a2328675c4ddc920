// bgzf_inflate.cu - BGZF members inflated on the device (bgzf_inflate.cuh),
// one warp per member, a grid-stride loop over the members:
//   lane 0 decodes the member's deflate stream into a batch of tokens
//          (literal runs, back-references, stored spans; inflate.cuh) in the
//          warp's shared memory, with the Huffman tables there too;
//   the warp writes the batch's bytes, token by token, 32 bytes at a time
//          (a back-reference reads only bytes before its own start, so its
//          bytes are written in parallel);
//   the warp computes the member's CRC-32: each lane over 1/32 of the
//          bytes, the 32 partial values combined in GF(2).
// Every access is bounds-checked by the decoder before a token is emitted
// (distances within the output so far, lengths within the member's ISIZE,
// stored spans within the input).
#include <string>

#include "bgzf_inflate.cuh"
#include "ma_internal.h"

namespace ma {
namespace {

constexpr int THREADS = 128;
constexpr int WARPS = THREADS / 32;
constexpr uint32_t CRC_POLY = 0xEDB88320u;

struct __align__(16) WarpSmem {
    inflate::Tables t;
    inflate::Tok tok[inflate::BATCH_TOKENS];
    uint8_t lit[inflate::BATCH_LITERALS];
    uint32_t lane_crc[32];
    int ntok, status, done;
    uint32_t o0;
};

// a * b mod P in the reflected CRC-32 representation (bit 31 = x^0)
__device__ __forceinline__ uint32_t gf2_mul(uint32_t a, uint32_t b) {
    uint32_t r = 0;
    for (int i = 0; i < 32; ++i) {
        if (a & (0x80000000u >> i)) r ^= b;
        b = (b & 1u) ? (b >> 1) ^ CRC_POLY : b >> 1;
    }
    return r;
}

// x^k mod P
__device__ uint32_t gf2_xpow(uint64_t k) {
    uint32_t r = 0x80000000u, b = 0x40000000u;
    while (k) {
        if (k & 1) r = gf2_mul(r, b);
        b = gf2_mul(b, b);
        k >>= 1;
    }
    return r;
}

// CRC-32 of out[0, n) by the warp: lane l folds bytes [l*seg, (l+1)*seg)
// from a zero register; the parts are shifted by the bytes after them and
// added; the initial all-ones register and the final inversion are added
// last.  Lane 0 returns it.
__device__ uint32_t warp_crc(const uint8_t* out, uint32_t n, const uint32_t* crc_tab, WarpSmem& S, int lane) {
    const uint32_t seg = (n + 31) / 32;
    const uint32_t a = min(n, static_cast<uint32_t>(lane) * seg), b = min(n, a + seg);
    uint32_t c = 0;
    for (uint32_t i = a; i < b; ++i) c = (c >> 8) ^ crc_tab[(c ^ out[i]) & 255u];
    S.lane_crc[lane] = c;
    __syncwarp();
    uint32_t r = 0;
    if (lane == 0 && n) {
        const uint32_t x_seg = gf2_xpow(8ull * seg);
        for (int l = 0; l < 32; ++l) {
            const uint32_t la = min(n, static_cast<uint32_t>(l) * seg), lb = min(n, la + seg);
            if (lb > la) r = gf2_mul(r, lb - la == seg ? x_seg : gf2_xpow(8ull * (lb - la))) ^ S.lane_crc[l];
        }
    }
    if (lane == 0) r = r ^ gf2_mul(0xffffffffu, gf2_xpow(8ull * n)) ^ 0xffffffffu;
    __syncwarp();
    return r;
}

// Member m by the warp; returns its status (valid in lane 0).
__device__ uint32_t warp_member(const bgzf_inflate::Job& j, uint32_t m, WarpSmem& S, const uint32_t* crc_tab,
                                int lane) {
    const uint64_t so = j.src_off[m], sl = j.src_len[m], dof = j.dst_off[m], isz = j.isize[m];
    if (so > j.in_bytes || sl > j.in_bytes - so || dof > j.out_bytes || isz > j.out_bytes - dof)
        return bgzf_inflate::S_SPAN;
    const uint8_t* in = j.in + so;
    uint8_t* out = j.out + dof;
    inflate::Stream st;  // lane 0's decoder state
    if (lane == 0) inflate::stream_init(st, in, static_cast<uint32_t>(sl), static_cast<uint32_t>(isz));
    for (;;) {
        if (lane == 0) {
            S.o0 = st.o;
            S.ntok = inflate::decode_tokens(st, S.t, S.tok, inflate::BATCH_TOKENS, S.lit, inflate::BATCH_LITERALS);
            S.status = st.status;
            S.done = st.finished || st.status != inflate::OK;
        }
        __syncwarp();
        const int ntok = S.ntok;
        uint32_t o = S.o0;
        for (int i = 0; i < ntok; ++i) {
            const inflate::Tok k = S.tok[i];
            if (k.dist == inflate::TOK_LITERAL) {
                for (uint32_t x = lane; x < k.len; x += 32) out[o + x] = S.lit[k.src + x];
            } else if (k.dist == inflate::TOK_STORED) {
                for (uint32_t x = lane; x < k.len; x += 32) out[o + x] = in[k.src + x];
            } else {
                for (uint32_t x = lane; x < k.len; x += 32) out[o + x] = out[o - k.dist + x % k.dist];
            }
            o += k.len;
            __syncwarp();
        }
        const bool done = S.done;
        __syncwarp();
        if (done) break;
    }
    const int status = S.status;
    if (status != inflate::OK) return static_cast<uint32_t>(status);
    // the decoder stopped at the final block: the bytes written are its output
    uint32_t got = 0;
    if (lane == 0) got = st.o;
    got = __shfl_sync(0xFFFFFFFFu, got, 0);
    if (got != isz) return bgzf_inflate::S_SIZE;
    const uint32_t c = warp_crc(out, got, crc_tab, S, lane);
    return c == j.crc[m] ? 0u : bgzf_inflate::S_CRC;
}

__global__ void __launch_bounds__(THREADS) bgzf_inflate_kernel(bgzf_inflate::Job j) {
    __shared__ WarpSmem smem[WARPS];
    __shared__ uint32_t crc_tab[256];
    bgzf_inflate::crc_table(crc_tab, threadIdx.x, THREADS);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t nw = static_cast<uint64_t>(gridDim.x) * WARPS;
    for (uint64_t m = static_cast<uint64_t>(blockIdx.x) * WARPS + warp; m < j.n; m += nw) {
        const uint32_t s = warp_member(j, static_cast<uint32_t>(m), smem[warp], crc_tab, lane);
        if (lane == 0) j.status[m] = s;
        __syncwarp();
    }
}

void check_launch(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(MA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

int bgzf_inflate_enqueue(const bgzf_inflate::Job& j, int sm_count, cudaStream_t st) {
    if (!j.n) return 0;
    const uint64_t want = (j.n + WARPS - 1) / WARPS;
    const uint64_t cap = static_cast<uint64_t>(sm_count > 0 ? sm_count : 148) * 16;
    bgzf_inflate_kernel<<<static_cast<unsigned>(want < cap ? want : cap), THREADS, 0, st>>>(j);
    check_launch(cudaGetLastError(), "bgzf_inflate_kernel");
    return 1;
}

}  // namespace ma
