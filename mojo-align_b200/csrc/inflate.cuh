// inflate.cuh - a DEFLATE (RFC 1951) decoder for one raw deflate stream,
// compiled unchanged as host and device code.  The stream is decoded into
// batches of tokens (literal runs, back-references, stored spans) by one
// thread; the tokens' bytes are written by a whole warp on the device
// (bgzf_inflate.cu) or by write_tokens here.  Every read of the input and
// every write or back-reference of the output is checked against its
// buffer; a malformed stream ends with an error status, never with an
// access outside the buffers.
//
// Huffman decoding follows the canonical-code construction of RFC 1951
// section 3.2.2: a 9-bit lookup table for short codes (indexed by the next 9
// stream bits, codes stored bit-reversed since the stream is LSB first) and,
// for longer codes, a per-length walk over the count of codes of each length
// (the first code of a length is the previous first code plus the previous
// count, shifted left by one).  Code-length sets follow zlib's acceptance
// rules: an over-subscribed set is an error; an incomplete set is accepted
// only for literal/length and distance codes made of a single code of
// length 1.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define MA_HD __host__ __device__
#else
#define MA_HD
#endif

namespace ma {
namespace inflate {

enum Status : int {
    OK = 0,
    E_INPUT = 1,   // the stream ends before its final block does
    E_BLOCK = 2,   // block type 3
    E_STORED = 3,  // stored block: LEN != ~NLEN
    E_CODES = 4,   // invalid code lengths (over-subscribed, incomplete, too many, repeat with nothing before)
    E_SYMBOL = 5,  // a code that decodes to no symbol, or literal/length 286-287, distance 30-31
    E_DIST = 6,    // a distance before the start of the output
    E_OUTPUT = 7,  // more output than the buffer holds
};

constexpr int FAST_BITS = 9;
constexpr int MAX_BITS = 15;
constexpr int NLIT = 288, NDIST = 32;

struct Huff {
    uint16_t count[MAX_BITS + 1];   // codes of each length
    uint16_t symbol[NLIT];          // symbols ordered by (length, value)
    uint16_t fast[1 << FAST_BITS];  // length << 9 | symbol for codes <= FAST_BITS, 0 if longer
};

struct Tables {
    Huff lit, dist;
    uint8_t lens[NLIT + NDIST];
};

// Length and distance bases and extra bits (RFC 1951 section 3.2.5).
MA_HD inline uint32_t len_base(int i) {
    // symbols 257..285
    if (i < 8) return 3 + i;
    if (i == 28) return 258;
    const int e = (i - 4) >> 2;  // extra bits for i in 8..27
    return ((4 + ((i - 4) & 3)) << e) + 3;
}
MA_HD inline int len_extra(int i) { return (i < 8 || i == 28) ? 0 : ((i - 4) >> 2); }
MA_HD inline uint32_t dist_base(int i) {
    // symbols 0..29
    if (i < 4) return 1 + i;
    const int e = (i - 2) >> 1;
    return ((2 + (i & 1)) << e) + 1;
}
MA_HD inline int dist_extra(int i) { return i < 4 ? 0 : ((i - 2) >> 1); }

struct Bits {
    const uint8_t* in;
    uint32_t n, pos;  // input bytes, next byte to load
    uint64_t buf;     // pending bits, LSB first
    int cnt;          // pending bit count

    MA_HD void refill() {
        while (cnt <= 56 && pos < n) {
            buf |= static_cast<uint64_t>(in[pos++]) << cnt;
            cnt += 8;
        }
    }
    // k <= 32 bits; false when the stream has fewer left
    MA_HD bool get(int k, uint32_t& v) {
        if (cnt < k) refill();
        if (cnt < k) return false;
        v = static_cast<uint32_t>(buf & ((k == 32) ? 0xffffffffull : ((1ull << k) - 1)));
        buf >>= k;
        cnt -= k;
        return true;
    }
};

// Builds h from code lengths lens[0, n).  kind 0: code-length codes (must
// be complete), 1: literal/length or distance codes.
MA_HD inline int build(Huff& h, const uint8_t* lens, int n, int kind) {
    for (int l = 0; l <= MAX_BITS; ++l) h.count[l] = 0;
    for (int s = 0; s < n; ++s) h.count[lens[s]]++;
    const int used = n - h.count[0];
    int left = 1, max_len = 0;
    for (int l = 1; l <= MAX_BITS; ++l) {
        left <<= 1;
        left -= h.count[l];
        if (left < 0) return E_CODES;  // over-subscribed
        if (h.count[l]) max_len = l;
    }
    if (left > 0 && used > 0 && (kind == 0 || max_len != 1)) return E_CODES;  // incomplete
    uint16_t offs[MAX_BITS + 2];
    offs[1] = 0;
    for (int l = 1; l <= MAX_BITS; ++l) offs[l + 1] = static_cast<uint16_t>(offs[l] + h.count[l]);
    for (int s = 0; s < n; ++s)
        if (lens[s]) h.symbol[offs[lens[s]]++] = static_cast<uint16_t>(s);
    for (int i = 0; i < (1 << FAST_BITS); ++i) h.fast[i] = 0;
    // canonical codes, bit-reversed into the lookup table
    // first code of each length: first(1) = 0, first(l) = (first(l-1) + count(l-1)) << 1
    uint32_t next[MAX_BITS + 1];
    next[0] = 0;
    uint32_t code = 0;
    for (int l = 1; l <= MAX_BITS; ++l) {
        next[l] = code;
        code = (code + h.count[l]) << 1;
    }
    for (int s = 0; s < n; ++s) {
        const int l = lens[s];
        if (!l || l > FAST_BITS) {
            if (l) next[l]++;
            continue;
        }
        const uint32_t c = next[l]++;
        uint32_t r = 0;
        for (int b = 0; b < l; ++b) r |= ((c >> b) & 1u) << (l - 1 - b);
        for (uint32_t i = r; i < (1u << FAST_BITS); i += (1u << l)) h.fast[i] = static_cast<uint16_t>(l << 9 | s);
    }
    return OK;
}

// The next symbol of h, or -1 (no code matches / stream ends).
MA_HD inline int decode(Bits& b, const Huff& h) {
    if (b.cnt < FAST_BITS) b.refill();
    if (b.cnt >= FAST_BITS) {
        const uint16_t e = h.fast[b.buf & ((1u << FAST_BITS) - 1)];
        if (e) {
            const int l = e >> 9;
            b.buf >>= l;
            b.cnt -= l;
            return e & 511;
        }
    }
    // bit by bit: code grows MSB first; codes of length l span [first, first + count)
    int code = 0, first = 0, index = 0;
    for (int l = 1; l <= MAX_BITS; ++l) {
        uint32_t bit;
        if (!b.get(1, bit)) return -1;
        code |= static_cast<int>(bit);
        const int count = h.count[l];
        if (code - first < count) return h.symbol[index + (code - first)];
        index += count;
        first = (first + count) << 1;
        code <<= 1;
    }
    return -1;
}

// ---- resumable decoding into tokens ----
// The decoder turns the stream into tokens: a run of literal bytes (kept in
// a literal buffer), a back-reference (length, distance) or a stored span
// of the input.  Decoding and writing are separate so that one thread can
// decode while a warp writes the bytes (bgzf_inflate.cu); write_tokens is
// the sequential writer.
constexpr uint32_t TOK_LITERAL = 0;            // dist of a literal run: bytes at lit[src]
constexpr uint32_t TOK_STORED = 0xFFFFFFFFu;   // dist of a stored span: bytes at in[src]

struct Tok {
    uint32_t len, dist, src;
};

// Decoder state between batches of tokens.
struct Stream {
    Bits b;
    uint32_t o;      // bytes of output the tokens so far produce
    uint32_t cap;    // output buffer size
    uint32_t last;   // the current (or last) block is the final one
    int in_block;    // inside a compressed block (tables built)
    int status;      // Status; OK while decoding
    int finished;    // the final block has ended
};

MA_HD inline void stream_init(Stream& s, const uint8_t* in, uint32_t n, uint32_t cap) {
    s.b = Bits{in, n, 0, 0, 0};
    s.o = 0;
    s.cap = cap;
    s.last = 0;
    s.in_block = 0;
    s.status = OK;
    s.finished = 0;
}

// Decodes tokens into tok[0, max_tok) (literal bytes into lit[0, max_lit))
// until either buffer is full, the stream ends or an error sets s.status;
// returns the number of tokens.  max_tok >= 2, max_lit >= 8.
MA_HD inline int decode_tokens(Stream& s, Tables& t, Tok* tok, int max_tok, uint8_t* lit, int max_lit) {
    Bits& b = s.b;
    int nt = 0, nl = 0;
    while (s.status == OK && !s.finished) {
        if (!s.in_block) {
            if (s.last) {
                s.finished = 1;
                break;
            }
            // room for a stored block's head bytes and span
            if (nt + 2 > max_tok || nl + 8 > max_lit) break;
            uint32_t last, type;
            if (!b.get(1, last) || !b.get(2, type)) {
                s.status = E_INPUT;
                break;
            }
            s.last = last;
            if (type == 0) {
                // stored: skip to the byte boundary, LEN, NLEN, LEN bytes
                const int drop = b.cnt & 7;
                b.buf >>= drop;
                b.cnt -= drop;
                uint32_t len, nlen;
                if (!b.get(16, len) || !b.get(16, nlen)) {
                    s.status = E_INPUT;
                    break;
                }
                if (len != (~nlen & 0xffffu)) {
                    s.status = E_STORED;
                    break;
                }
                if (len > s.cap - s.o) {
                    s.status = E_OUTPUT;
                    break;
                }
                uint32_t k = 0;  // bytes already in the bit buffer (at most 4 here)
                while (k < len && b.cnt >= 8) {
                    lit[nl + static_cast<int>(k)] = static_cast<uint8_t>(b.buf);
                    b.buf >>= 8;
                    b.cnt -= 8;
                    ++k;
                }
                if (k) tok[nt++] = Tok{k, TOK_LITERAL, static_cast<uint32_t>(nl)};
                nl += static_cast<int>(k);
                const uint32_t rest = len - k;
                if (rest > b.n - b.pos) {
                    s.status = E_INPUT;
                    break;
                }
                if (rest) tok[nt++] = Tok{rest, TOK_STORED, b.pos};
                b.pos += rest;
                s.o += len;
                continue;
            }
            if (type == 3) {
                s.status = E_BLOCK;
                break;
            }
            int nlit, ndist;
            if (type == 1) {
                for (int v = 0; v < 144; ++v) t.lens[v] = 8;
                for (int v = 144; v < 256; ++v) t.lens[v] = 9;
                for (int v = 256; v < 280; ++v) t.lens[v] = 7;
                for (int v = 280; v < NLIT; ++v) t.lens[v] = 8;
                for (int v = 0; v < NDIST; ++v) t.lens[NLIT + v] = 5;
                nlit = NLIT;
                ndist = NDIST;
                if (build(t.lit, t.lens, nlit, 1) != OK || build(t.dist, t.lens + NLIT, ndist, 1) != OK) {
                    s.status = E_CODES;
                    break;
                }
            } else {
                uint32_t hlit, hdist, hclen;
                if (!b.get(5, hlit) || !b.get(5, hdist) || !b.get(4, hclen)) {
                    s.status = E_INPUT;
                    break;
                }
                nlit = static_cast<int>(hlit) + 257;
                ndist = static_cast<int>(hdist) + 1;
                if (nlit > 286 || ndist > 30) {
                    s.status = E_CODES;
                    break;
                }
                const uint8_t ORDER[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
                uint8_t cl[19];
                for (int i = 0; i < 19; ++i) cl[i] = 0;
                int st = OK;
                for (uint32_t i = 0; i < hclen + 4; ++i) {
                    uint32_t v;
                    if (!b.get(3, v)) {
                        st = E_INPUT;
                        break;
                    }
                    cl[ORDER[i]] = static_cast<uint8_t>(v);
                }
                if (st == OK && build(t.lit, cl, 19, 0) != OK) st = E_CODES;
                // literal/length then distance code lengths, one run-length sequence
                int i = 0;
                while (st == OK && i < nlit + ndist) {
                    const int sym = decode(b, t.lit);
                    if (sym < 0) {
                        st = b.cnt == 0 && b.pos >= b.n ? E_INPUT : E_CODES;
                        break;
                    }
                    if (sym < 16) {
                        t.lens[i++] = static_cast<uint8_t>(sym);
                        continue;
                    }
                    uint32_t rep;
                    uint8_t val = 0;
                    if (sym == 16) {
                        if (i == 0) {
                            st = E_CODES;
                            break;
                        }
                        val = t.lens[i - 1];
                        if (!b.get(2, rep)) {
                            st = E_INPUT;
                            break;
                        }
                        rep += 3;
                    } else if (sym == 17) {
                        if (!b.get(3, rep)) {
                            st = E_INPUT;
                            break;
                        }
                        rep += 3;
                    } else {
                        if (!b.get(7, rep)) {
                            st = E_INPUT;
                            break;
                        }
                        rep += 11;
                    }
                    if (i + static_cast<int>(rep) > nlit + ndist) {
                        st = E_CODES;
                        break;
                    }
                    while (rep--) t.lens[i++] = val;
                }
                if (st == OK && t.lens[256] == 0) st = E_CODES;  // no end-of-block code
                if (st == OK) {
                    // distance lengths sit right after the literal/length ones
                    uint8_t dl[NDIST];
                    for (int v = 0; v < ndist; ++v) dl[v] = t.lens[nlit + v];
                    if (build(t.lit, t.lens, nlit, 1) != OK || build(t.dist, dl, ndist, 1) != OK) st = E_CODES;
                }
                if (st != OK) {
                    s.status = st;
                    break;
                }
            }
            s.in_block = 1;
        }
        // the block's symbols, while there is room for one more token
        while (nt < max_tok && nl < max_lit) {
            const int sym = decode(b, t.lit);
            if (sym < 0) {
                s.status = b.cnt == 0 && b.pos >= b.n ? E_INPUT : E_SYMBOL;
                break;
            }
            if (sym < 256) {
                if (s.o >= s.cap) {
                    s.status = E_OUTPUT;
                    break;
                }
                if (nt > 0 && tok[nt - 1].dist == TOK_LITERAL &&
                    tok[nt - 1].src + tok[nt - 1].len == static_cast<uint32_t>(nl))
                    tok[nt - 1].len++;
                else
                    tok[nt++] = Tok{1, TOK_LITERAL, static_cast<uint32_t>(nl)};
                lit[nl++] = static_cast<uint8_t>(sym);
                s.o++;
                continue;
            }
            if (sym == 256) {
                s.in_block = 0;
                break;
            }
            const int li = sym - 257;
            if (li >= 29) {
                s.status = E_SYMBOL;
                break;
            }
            uint32_t e = 0;
            if (len_extra(li) && !b.get(len_extra(li), e)) {
                s.status = E_INPUT;
                break;
            }
            const uint32_t len = len_base(li) + e;
            const int ds = decode(b, t.dist);
            if (ds < 0) {
                s.status = b.cnt == 0 && b.pos >= b.n ? E_INPUT : E_SYMBOL;
                break;
            }
            if (ds >= 30) {
                s.status = E_SYMBOL;
                break;
            }
            e = 0;
            if (dist_extra(ds) && !b.get(dist_extra(ds), e)) {
                s.status = E_INPUT;
                break;
            }
            const uint32_t dist = dist_base(ds) + e;
            if (dist > s.o) {
                s.status = E_DIST;
                break;
            }
            if (len > s.cap - s.o) {
                s.status = E_OUTPUT;
                break;
            }
            tok[nt++] = Tok{len, dist, 0};
            s.o += len;
        }
        if (s.in_block) break;  // a token buffer is full
    }
    return nt;
}

// Writes the bytes of tok[0, ntok) to out from position o0, in order.  A
// back-reference of distance d copies byte k from o - d + k % d, which is
// before the token, so its bytes do not depend on one another.
MA_HD inline void write_tokens(const Tok* tok, int ntok, const uint8_t* lit, const uint8_t* in, uint8_t* out,
                               uint32_t o0) {
    uint32_t o = o0;
    for (int i = 0; i < ntok; ++i) {
        const Tok& k = tok[i];
        if (k.dist == TOK_LITERAL) {
            for (uint32_t j = 0; j < k.len; ++j) out[o + j] = lit[k.src + j];
        } else if (k.dist == TOK_STORED) {
            for (uint32_t j = 0; j < k.len; ++j) out[o + j] = in[k.src + j];
        } else {
            for (uint32_t j = 0; j < k.len; ++j) out[o + j] = out[o - k.dist + j % k.dist];
        }
        o += k.len;
    }
}

constexpr int BATCH_TOKENS = 64;   // tokens per decoding batch
constexpr int BATCH_LITERALS = 256;

// Inflates the raw deflate stream in[0, n) into out[0, cap); *out_len
// receives the bytes written.  t: scratch tables (may live in shared
// memory).  The token decoder and the sequential writer, batch by batch.
MA_HD inline int inflate_raw(const uint8_t* in, uint32_t n, uint8_t* out, uint32_t cap, uint32_t* out_len,
                             Tables& t) {
    Stream s;
    stream_init(s, in, n, cap);
    Tok tok[BATCH_TOKENS];
    uint8_t lit[BATCH_LITERALS];
    *out_len = 0;
    while (s.status == OK && !s.finished) {
        const uint32_t o0 = s.o;
        const int nt = decode_tokens(s, t, tok, BATCH_TOKENS, lit, BATCH_LITERALS);
        write_tokens(tok, nt, lit, in, out, o0);
    }
    if (s.status != OK) return s.status;
    *out_len = s.o;
    return OK;
}

}  // namespace inflate
}  // namespace ma
