// index_io.cpp - bwa 0.7 FM-index files: reading (the loader the reference
// uses) and writing (this library's own index builder).
//
// File formats follow what the reference reads
// (fq2bam-meth/src/linear_fm_index.mojo:88-175):
//   .bwt  u64 primary, u64 L2[1..4], then u32 words.  Every 128 BWT
//         positions start with 4 u64 counts (symbols before the block) and
//         continue with 8 u32 words of 2-bit symbols, most significant
//         first; one final block of 4 u64 totals closes the file.
//   .sa   u64 primary, L2[1..4], sa_intv, seq_len, then SA[i*sa_intv] for
//         i = 1..n_sa-1 as u64.
//   .pac  forward text, 4 bases per byte, most significant first, then the
//         bwa tail bytes (a zero byte when l_pac % 4 == 0, then l_pac % 4).
//   .ann  "l_pac n_seqs seed", then per contig "gi name anno" and
//         "offset len n_ambs".
//   .amb  "l_pac n_seqs n_holes", then per hole "offset len char".
// The BWT text is the forward pac followed by its reverse complement
// (seq_len = 2*l_pac), with the sentinel removed from the stored string at
// row `primary`.
#include <algorithm>
#include <array>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>
#include <thread>

#include "ma_internal.h"

namespace ma {

namespace {

std::vector<uint8_t> slurp(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) fail(MA_ERR_IO, "FmIndex missing " + path);
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<uint8_t> buf(n > 0 ? static_cast<size_t>(n) : 0);
    if (n > 0 && std::fread(buf.data(), 1, buf.size(), f) != buf.size()) {
        std::fclose(f);
        fail(MA_ERR_IO, "short read of " + path);
    }
    std::fclose(f);
    return buf;
}

uint64_t le64(const uint8_t* p) {
    uint64_t v = 0;
    for (int b = 0; b < 8; ++b) v |= static_cast<uint64_t>(p[b]) << (8 * b);
    return v;
}

void put64(std::vector<uint8_t>& out, uint64_t v) {
    for (int b = 0; b < 8; ++b) out.push_back(static_cast<uint8_t>(v >> (8 * b)));
}

void write_all(const std::string& path, const void* data, size_t n) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) fail(MA_ERR_IO, "cannot write " + path);
    if (n && std::fwrite(data, 1, n, f) != n) {
        std::fclose(f);
        fail(MA_ERR_IO, "short write of " + path);
    }
    if (std::fclose(f) != 0) fail(MA_ERR_IO, "close failed for " + path);
}

}  // namespace

BwaIndexHost load_bwa_index(const std::string& prefix) {
    BwaIndexHost ix;
    {
        std::vector<uint8_t> b = slurp(prefix + ".bwt");
        if (b.size() < 40 || (b.size() - 40) % 4 != 0) fail(MA_ERR_FORMAT, "FmIndex bad .bwt size");
        ix.primary = le64(b.data());
        ix.L2[0] = 0;
        for (int c = 1; c <= 4; ++c) ix.L2[c] = le64(b.data() + 8 * c);
        ix.seq_len = ix.L2[4];
        size_t nw = (b.size() - 40) / 4;
        ix.bwt.resize(nw + 2, 0);  // two spare words for 64-bit pair reads
        std::memcpy(ix.bwt.data(), b.data() + 40, nw * 4);
        uint64_t need = (ix.seq_len + 15) / 16 + 8 * ((ix.seq_len + 127) / 128 + 1);
        if (nw < need) fail(MA_ERR_FORMAT, "FmIndex .bwt shorter than seq_len implies");
    }
    for (int c = 0; c < 4; ++c)
        if (ix.L2[c] > ix.L2[c + 1]) fail(MA_ERR_FORMAT, "FmIndex L2 not monotone");
    if (ix.primary == 0 || ix.primary > ix.seq_len) fail(MA_ERR_FORMAT, "FmIndex bad primary");
    {
        std::vector<uint8_t> s = slurp(prefix + ".sa");
        if (s.size() < 56) fail(MA_ERR_FORMAT, "FmIndex bad .sa size");
        if (le64(s.data()) != ix.primary) fail(MA_ERR_FORMAT, "FmIndex SA/BWT primary mismatch");
        ix.sa_intv = static_cast<int64_t>(le64(s.data() + 40));
        if (le64(s.data() + 48) != ix.seq_len) fail(MA_ERR_FORMAT, "FmIndex SA/BWT seq_len mismatch");
        if (ix.sa_intv <= 0 || (ix.sa_intv & (ix.sa_intv - 1)) != 0)
            fail(MA_ERR_FORMAT, "FmIndex sa_intv must be a power of two");
        ix.n_sa = static_cast<int64_t>((ix.seq_len + ix.sa_intv) / ix.sa_intv);
        size_t nsa = static_cast<size_t>(ix.n_sa - 1);
        if (s.size() < 56 + nsa * 8) fail(MA_ERR_FORMAT, "FmIndex short .sa");
        ix.sa.resize(nsa);
        for (size_t i = 0; i < nsa; ++i) ix.sa[i] = le64(s.data() + 56 + 8 * i);
    }
    ix.pac = slurp(prefix + ".pac");
    {
        std::ifstream f(prefix + ".ann");
        if (!f) fail(MA_ERR_IO, "FmIndex missing " + prefix + ".ann");
        std::string line;
        if (!std::getline(f, line)) fail(MA_ERR_FORMAT, "FmIndex bad .ann header");
        std::istringstream h(line);
        long long lp = -1, nseq = -1;
        h >> lp >> nseq;
        if (lp < 0 || nseq < 0) fail(MA_ERR_FORMAT, "FmIndex bad .ann header");
        ix.l_pac = static_cast<uint64_t>(lp);
        uint64_t off = 0;
        for (long long i = 0; i < nseq; ++i) {
            std::string l1, l2;
            if (!std::getline(f, l1) || !std::getline(f, l2)) fail(MA_ERR_FORMAT, "FmIndex truncated .ann");
            std::istringstream a(l1), b(l2);
            long long gi = 0, o = 0, ln = -1;
            Contig c;
            a >> gi >> c.name;
            std::getline(a, c.anno);
            if (!c.anno.empty() && c.anno[0] == ' ') c.anno.erase(0, 1);
            b >> o >> ln >> c.n_ambs;
            if (c.name.empty() || ln < 0) fail(MA_ERR_FORMAT, "FmIndex truncated .ann");
            c.offset = off;  // offsets accumulate as in linear_fm_index.mojo:154-156
            c.len = static_cast<uint32_t>(ln);
            off += static_cast<uint64_t>(ln);
            ix.contigs.push_back(std::move(c));
        }
        if (off != ix.l_pac) fail(MA_ERR_FORMAT, "FmIndex .ann offsets != l_pac");
    }
    if (ix.seq_len != 2 * ix.l_pac) fail(MA_ERR_FORMAT, "FmIndex seq_len != 2*l_pac");
    if (ix.pac.size() < (ix.l_pac + 3) / 4) fail(MA_ERR_FORMAT, "FmIndex short .pac");
    return ix;
}

std::vector<FastaRecord> read_fasta(const std::string& path) {
    // the whole file in memory, lines split with memchr; sequence lines are
    // appended a line at a time (blanks and tabs inside them dropped)
    FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) fail(MA_ERR_IO, "cannot open FASTA " + path);
    std::fseek(fp, 0, SEEK_END);
    const long size = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    std::string text(size > 0 ? static_cast<size_t>(size) : 0, '\0');
    if (size > 0 && std::fread(&text[0], 1, text.size(), fp) != text.size()) {
        std::fclose(fp);
        fail(MA_ERR_IO, "short read of " + path);
    }
    std::fclose(fp);
    std::vector<FastaRecord> recs;
    const char* p = text.data();
    const char* end = p + text.size();
    // sequence bytes of each record, for one reserve() per record
    while (p < end) {
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', static_cast<size_t>(end - p)));
        const char* le = nl ? nl : end;
        const char* lend = le;
        if (lend > p && lend[-1] == '\r') --lend;
        if (lend > p) {
            if (*p == '>') {
                std::string line(p, lend);
                FastaRecord r;
                size_t sp = line.find_first_of(" \t", 1);
                r.name = line.substr(1, sp == std::string::npos ? std::string::npos : sp - 1);
                if (sp != std::string::npos) {
                    size_t st = line.find_first_not_of(" \t", sp);
                    if (st != std::string::npos) r.anno = line.substr(st);
                }
                if (r.name.empty()) fail(MA_ERR_FORMAT, "FASTA record without a name in " + path);
                // room for the record's bases: up to the next header
                const char* nh = static_cast<const char*>(std::memchr(le, '>', static_cast<size_t>(end - le)));
                r.seq.reserve(static_cast<size_t>((nh ? nh : end) - le));
                recs.push_back(std::move(r));
            } else {
                if (recs.empty()) fail(MA_ERR_FORMAT, "FASTA sequence before the first header in " + path);
                std::string& q = recs.back().seq;
                const char* a = p;
                for (const char* c = p; c < lend; ++c) {
                    if (*c == ' ' || *c == '\t') {
                        q.append(a, c);
                        a = c + 1;
                    }
                }
                q.append(a, lend);
            }
        }
        p = nl ? nl + 1 : end;
    }
    if (recs.empty()) fail(MA_ERR_FORMAT, "empty FASTA " + path);
    return recs;
}

namespace {

int nt4(char c) {
    switch (c) {
        case 'A': case 'a': return 0;
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': return 3;
        default: return 4;
    }
}

// bwa-meth's dual-strand text: per contig r<header> with G->A, then
// f<header> with C->T, upper-cased (bwameth.py convert_fasta).
std::vector<FastaRecord> bwameth_convert(const std::vector<FastaRecord>& in) {
    std::vector<FastaRecord> out;
    out.reserve(in.size() * 2);
    for (const auto& r : in) {
        std::string up(r.seq);
        for (auto& ch : up) ch = static_cast<char>(std::toupper(static_cast<unsigned char>(ch)));
        FastaRecord rr{"r" + r.name, r.anno, up}, ff{"f" + r.name, r.anno, up};
        for (auto& ch : rr.seq)
            if (ch == 'G') ch = 'A';
        for (auto& ch : ff.seq)
            if (ch == 'C') ch = 'T';
        out.push_back(std::move(rr));
        out.push_back(std::move(ff));
    }
    return out;
}

void write_fasta(const std::string& path, const std::vector<FastaRecord>& recs) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) fail(MA_ERR_IO, "cannot write " + path);
    std::string buf;
    for (const auto& r : recs) {  // one record's text at a time
        buf.clear();
        buf.reserve(r.seq.size() + r.seq.size() / 80 + r.name.size() + r.anno.size() + 8);
        buf += ">" + r.name;
        if (!r.anno.empty()) buf += " " + r.anno;
        buf += "\n";
        for (size_t i = 0; i < r.seq.size(); i += 80) {
            buf.append(r.seq, i, std::min<size_t>(80, r.seq.size() - i));
            buf += "\n";
        }
        if (std::fwrite(buf.data(), 1, buf.size(), f) != buf.size()) {
            std::fclose(f);
            fail(MA_ERR_IO, "short write of " + path);
        }
    }
    if (std::fclose(f) != 0) fail(MA_ERR_IO, "close failed for " + path);
}

}  // namespace

namespace {

// Runs f(t, nt) on nt host threads.
template <typename F>
void parallel(F f) {
    const unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t) pool.emplace_back(f, t, nt);
    for (auto& th : pool) th.join();
}

void put_u64_bytes(std::vector<uint8_t>& out, size_t at, uint64_t v) {
    for (int b = 0; b < 8; ++b) out[at + b] = static_cast<uint8_t>(v >> (8 * b));
}

}  // namespace

void build_index(const std::string& fasta, const std::string& out_prefix, bool bwameth_c2t, int sa_intv,
                 int device, uint64_t batch_limit) {
    if (sa_intv <= 0 || (sa_intv & (sa_intv - 1)) != 0) fail(MA_ERR_ARG, "sa_intv must be a power of two");
    std::vector<FastaRecord> recs = read_fasta(fasta);
    if (bwameth_c2t) {
        recs = bwameth_convert(recs);
        write_fasta(out_prefix, recs);
    }
    // ---- pac (forward), ambiguous bases replaced like bwa (seeded) ----
    uint64_t l_pac = 0;
    for (const auto& r : recs) l_pac += r.seq.size();
    if (l_pac == 0) fail(MA_ERR_FORMAT, "FASTA has no bases");
    const uint64_t n = 2 * l_pac;
    if (device < 0 && n + 1 >= 0xFFFFFFFFull)
        fail(MA_ERR_UNSUPPORTED, "the CPU index builder handles texts below 2^32 symbols; give a GPU");
    if (n > (1ull << 35) - 2) fail(MA_ERR_UNSUPPORTED, "index builder handles texts below 2^35 symbols");
    // forward text, one code per byte (codes of ambiguous bases drawn in
    // order from one seeded generator, as before)
    std::vector<uint8_t> fwd(l_pac);
    std::vector<Contig> contigs;
    std::vector<Hole> holes;
    std::vector<uint64_t> rec_off;
    {
        uint64_t pos = 0;
        for (const auto& r : recs) {
            rec_off.push_back(pos);
            pos += r.seq.size();
        }
    }
    std::vector<uint8_t> any_amb(recs.size(), 0);
    parallel([&](unsigned t, unsigned nt) {
        for (size_t ri = t; ri < recs.size(); ri += nt) {
            const std::string& q = recs[ri].seq;
            uint8_t* o = fwd.data() + rec_off[ri];
            uint8_t amb = 0;
            for (size_t i = 0; i < q.size(); ++i) {
                const int v = nt4(q[i]);
                o[i] = static_cast<uint8_t>(v);
                amb |= v > 3;
            }
            any_amb[ri] = amb;
        }
    });
    std::mt19937_64 rng(11);
    for (size_t ri = 0; ri < recs.size(); ++ri) {
        const auto& r = recs[ri];
        Contig c;
        c.name = r.name;
        c.anno = r.anno;
        c.offset = rec_off[ri];
        c.len = static_cast<uint32_t>(r.seq.size());
        if (any_amb[ri]) {
            for (size_t i = 0; i < r.seq.size(); ++i) {
                const uint64_t pos = rec_off[ri] + i;
                if (fwd[pos] <= 3) continue;
                if (!holes.empty() && holes.back().offset + holes.back().len == pos &&
                    holes.back().amb == std::toupper(r.seq[i])) {
                    holes.back().len++;
                } else {
                    holes.push_back(Hole{pos, 1, static_cast<char>(std::toupper(static_cast<unsigned char>(r.seq[i])))});
                    c.n_ambs++;
                }
                fwd[pos] = static_cast<uint8_t>(rng() & 3);
            }
        }
        contigs.push_back(std::move(c));
    }
    std::vector<FastaRecord>().swap(recs);
    uint64_t L2[5] = {0, 0, 0, 0, 0};
    {
        std::vector<std::array<uint64_t, 4>> part(64, {0, 0, 0, 0});
        parallel([&](unsigned t, unsigned nt) {
            const uint64_t a = l_pac * t / nt, b = l_pac * (t + 1) / nt;
            for (uint64_t i = a; i < b; ++i) part[t][fwd[i]]++;
        });
        uint64_t cf[4] = {0, 0, 0, 0};
        for (auto& pc : part)
            for (int c = 0; c < 4; ++c) cf[c] += pc[c];
        // the reverse complement holds each symbol's complement once more
        for (int c = 0; c < 4; ++c) L2[c + 1] = cf[c] + cf[3 - c];
        for (int c = 1; c <= 4; ++c) L2[c] += L2[c - 1];
    }

    uint64_t primary = 0;
    std::vector<uint32_t> bwt;
    std::vector<uint64_t> samples;
    if (device >= 0) {
        // T = pac + reverse complement, 32 symbols per word, LSB first
        const uint64_t n_words = n / 32 + 3;
        std::vector<uint64_t> tw(n_words, 0);
        parallel([&](unsigned t, unsigned nt) {
            const uint64_t w0 = (n / 32 + 1) * t / nt, w1 = (n / 32 + 1) * (t + 1) / nt;
            for (uint64_t w = w0; w < w1; ++w) {
                uint64_t v = 0;
                for (int j = 0; j < 32; ++j) {
                    const uint64_t i = 32 * w + j;
                    if (i >= n) break;
                    const uint64_t c = i < l_pac ? fwd[i] : 3u - fwd[n - 1 - i];
                    v |= c << (2 * j);
                }
                tw[w] = v;
            }
        });
        BwtBuild b = bwt_build_gpu(tw, n, sa_intv, batch_limit, device);
        primary = b.primary;
        bwt.swap(b.bwt);
        samples.swap(b.samples);
    } else {
        std::vector<uint8_t> text(n);
        std::memcpy(text.data(), fwd.data(), l_pac);
        for (uint64_t i = 0; i < l_pac; ++i) text[n - 1 - i] = static_cast<uint8_t>(3 - fwd[i]);
        std::vector<uint32_t> sa = suffix_array_cpu(text.data(), n);
        if (sa.size() != n + 1 || sa[0] != n) fail(MA_ERR_INTERNAL, "suffix array construction failed");
        // stored BWT: rows 0..n without the sentinel row
        const uint64_t n_occ = (n + 127) / 128 + 1;
        bwt.assign((n + 15) / 16 + 8 * n_occ, 0);
        uint64_t cnt[4] = {0, 0, 0, 0};
        uint64_t k = 0;      // stored position
        uint64_t wbase = 0;  // word index of current block start
        for (uint64_t row = 0; row <= n; ++row) {
            if (sa[row] == 0) {
                primary = row;
                continue;
            }
            const uint8_t c = text[sa[row] - 1];
            if (k % 128 == 0) {
                wbase = (k / 128) * 16;
                for (int cc = 0; cc < 4; ++cc) {
                    bwt[wbase + 2 * cc] = static_cast<uint32_t>(cnt[cc]);
                    bwt[wbase + 2 * cc + 1] = static_cast<uint32_t>(cnt[cc] >> 32);
                }
            }
            bwt[wbase + 8 + (k % 128) / 16] |= static_cast<uint32_t>(c) << ((15 - (k & 15)) << 1);
            cnt[c]++;
            k++;
        }
        // closing totals block
        uint64_t tb = ((n + 127) / 128) * 16;
        if (n % 128 != 0) tb = (n / 128) * 16 + 8 + ((n % 128) + 15) / 16;
        for (int cc = 0; cc < 4; ++cc) {
            bwt[tb + 2 * cc] = static_cast<uint32_t>(cnt[cc]);
            bwt[tb + 2 * cc + 1] = static_cast<uint32_t>(cnt[cc] >> 32);
        }
        const uint64_t n_sa = (n + static_cast<uint64_t>(sa_intv)) / static_cast<uint64_t>(sa_intv);
        samples.resize(n_sa - 1);
        for (uint64_t i = 1; i < n_sa; ++i) samples[i - 1] = sa[i * static_cast<uint64_t>(sa_intv)];
    }
    if (primary == 0) fail(MA_ERR_INTERNAL, "no primary row");

    // ---- write files ----
    {
        std::vector<uint8_t> out(40 + bwt.size() * 4);
        put_u64_bytes(out, 0, primary);
        for (int c = 1; c <= 4; ++c) put_u64_bytes(out, 8 * static_cast<size_t>(c), L2[c]);
        std::memcpy(out.data() + 40, bwt.data(), bwt.size() * 4);
        std::vector<uint32_t>().swap(bwt);
        write_all(out_prefix + ".bwt", out.data(), out.size());
    }
    {
        std::vector<uint8_t> out(56 + 8 * samples.size());
        put_u64_bytes(out, 0, primary);
        for (int c = 1; c <= 4; ++c) put_u64_bytes(out, 8 * static_cast<size_t>(c), L2[c]);
        put_u64_bytes(out, 40, static_cast<uint64_t>(sa_intv));
        put_u64_bytes(out, 48, n);
        std::memcpy(out.data() + 56, samples.data(), samples.size() * 8);  // little-endian host
        write_all(out_prefix + ".sa", out.data(), out.size());
    }
    {
        std::vector<uint8_t> pac((l_pac + 3) / 4, 0);
        parallel([&](unsigned t, unsigned nt) {
            const uint64_t nb = (l_pac + 3) / 4;
            const uint64_t b0 = nb * t / nt, b1 = nb * (t + 1) / nt;
            for (uint64_t b = b0; b < b1; ++b) {
                uint8_t v = 0;
                for (uint64_t i = 4 * b; i < 4 * b + 4 && i < l_pac; ++i)
                    v |= static_cast<uint8_t>(fwd[i] << ((~i & 3) << 1));
                pac[b] = v;
            }
        });
        if (l_pac % 4 == 0) pac.push_back(0);
        pac.push_back(static_cast<uint8_t>(l_pac % 4));
        write_all(out_prefix + ".pac", pac.data(), pac.size());
    }
    {
        std::string s = std::to_string(l_pac) + " " + std::to_string(contigs.size()) + " 11\n";
        for (const auto& c : contigs) {
            s += "0 " + c.name + " " + (c.anno.empty() ? std::string("(null)") : c.anno) + "\n";
            s += std::to_string(c.offset) + " " + std::to_string(c.len) + " " + std::to_string(c.n_ambs) + "\n";
        }
        write_all(out_prefix + ".ann", s.data(), s.size());
        std::string a = std::to_string(l_pac) + " " + std::to_string(contigs.size()) + " " +
                        std::to_string(holes.size()) + "\n";
        for (const auto& hh : holes)
            a += std::to_string(hh.offset) + " " + std::to_string(hh.len) + " " + std::string(1, hh.amb) + "\n";
        write_all(out_prefix + ".amb", a.data(), a.size());
    }
}

// ---------------------------------------------------------------------------
// CPU suffix array: prefix doubling that re-sorts only unresolved groups.
// Round 0 sorts suffixes by their first 21 symbols (3 bits each, the
// sentinel and past-the-end as 0); each later round sorts the members of a
// tied group by the rank of the suffix h symbols further on, h doubling.
std::vector<uint32_t> suffix_array_cpu(const uint8_t* text, uint64_t n) {
    const uint64_t N = n + 1;
    std::vector<uint64_t> key(N);
    for (uint64_t i = 0; i < N; ++i) {
        uint64_t k = 0;
        for (uint64_t j = 0; j < 21; ++j) {
            uint64_t p = i + j;
            k = (k << 3) | (p < n ? static_cast<uint64_t>(text[p]) + 1 : 0);
        }
        key[i] = k;
    }
    std::vector<uint32_t> sa(N);
    for (uint64_t i = 0; i < N; ++i) sa[i] = static_cast<uint32_t>(i);
    std::sort(sa.begin(), sa.end(), [&](uint32_t a, uint32_t b) {
        return key[a] != key[b] ? key[a] < key[b] : a < b;
    });
    std::vector<uint32_t> rank(N);
    std::vector<std::pair<uint32_t, uint32_t>> groups;  // [a, b) unresolved
    {
        uint64_t head = 0;
        for (uint64_t j = 0; j < N; ++j) {
            if (j > 0 && key[sa[j]] != key[sa[j - 1]]) {
                if (j - head > 1) groups.emplace_back(static_cast<uint32_t>(head), static_cast<uint32_t>(j));
                head = j;
            }
            rank[sa[j]] = static_cast<uint32_t>(head);
        }
        if (N - head > 1) groups.emplace_back(static_cast<uint32_t>(head), static_cast<uint32_t>(N));
    }
    std::vector<uint64_t>().swap(key);
    uint64_t h = 21;
    std::vector<uint32_t> k2;
    while (!groups.empty()) {
        if (h > N) fail(MA_ERR_INTERNAL, "suffix sort did not converge");
        // sort every group by the old rank h symbols on
        for (const auto& g : groups) {
            std::sort(sa.begin() + g.first, sa.begin() + g.second, [&](uint32_t a, uint32_t b) {
                return rank[a + h] < rank[b + h];
            });
        }
        // gather every member's key from the old ranks before any rank of
        // this round changes, then assign the new ranks
        k2.clear();
        for (const auto& g : groups)
            for (uint32_t j = g.first; j < g.second; ++j) k2.push_back(rank[sa[j] + h]);
        std::vector<std::pair<uint32_t, uint32_t>> next;
        size_t kp = 0;
        for (const auto& g : groups) {
            const uint32_t* kk = k2.data() + kp;
            uint32_t head = g.first;
            for (uint32_t j = g.first; j < g.second; ++j) {
                if (j > g.first && kk[j - g.first] != kk[j - 1 - g.first]) {
                    if (j - head > 1) next.emplace_back(head, j);
                    head = j;
                }
                rank[sa[j]] = head;
            }
            if (g.second - head > 1) next.emplace_back(head, g.second);
            kp += g.second - g.first;
        }
        groups.swap(next);
        h *= 2;
    }
    return sa;
}

}  // namespace ma
