// synth.cpp - seeded synthetic workloads for benchmarks and tests: a
// reference from a first-order base model and bisulfite-converted reads.
// No counterpart in the reference (which only runs on real samples).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "ma_internal.h"

namespace ma {
namespace {

// splitmix64: small, fast, reproducible across platforms
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uni() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
    uint64_t below(uint64_t n) { return n ? next() % n : 0; }
    double normal() {
        double u1 = uni(), u2 = uni();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

const char kBase[4] = {'A', 'C', 'G', 'T'};

char comp(char c) {
    switch (c) {
        case 'A': return 'T';
        case 'C': return 'G';
        case 'G': return 'C';
        case 'T': return 'A';
        default: return 'N';
    }
}

}  // namespace
}  // namespace ma

using namespace ma;

/*
 * First-order model: from A/G/T the next base is A,C,G,T with
 * (a, c, g, a); after a C, G is drawn with probability cpg/c_freq so that
 * CpG dinucleotides occur at about `cpg`, and the remaining mass keeps the
 * stationary GC fraction at `gc`.
 */
extern "C" int ma_synth_reference_impl(const char* fasta_out, uint64_t total_len, int n_contigs, double gc,
                                       double cpg, uint64_t seed, char* err, size_t err_cap) {
    try {
        if (!fasta_out || total_len == 0 || n_contigs <= 0 || gc <= 0 || gc >= 1 || cpg < 0)
            fail(MA_ERR_ARG, "bad synthetic reference arguments");
        const double pc = gc / 2, pa = (1 - gc) / 2;
        double g_after_c = pc > 0 ? cpg / pc : 0;
        if (g_after_c > 0.9) g_after_c = 0.9;
        // rows for A/G/T: (a, c, g, t); row for C: (a', c', g', t')
        const double g = (pc - pc * g_after_c) / (1 - pc);
        const double c = pc;
        const double at = (1 - c - g) / 2;
        const double at_c = (1 - c - g_after_c) / 2;
        double cum_other[4] = {at, at + c, at + c + g, 1.0};
        double cum_c[4] = {at_c, at_c + c, at_c + c + g_after_c, 1.0};
        (void)pa;
        Rng rng(seed);
        FILE* f = std::fopen(fasta_out, "wb");
        if (!f) fail(MA_ERR_IO, std::string("cannot write ") + fasta_out);
        std::string line;
        uint64_t per = total_len / static_cast<uint64_t>(n_contigs);
        int prev = static_cast<int>(rng.below(4));
        for (int ci = 0; ci < n_contigs; ++ci) {
            uint64_t len = (ci == n_contigs - 1) ? total_len - per * static_cast<uint64_t>(n_contigs - 1) : per;
            std::fprintf(f, ">chr%d synthetic\n", ci + 1);
            line.clear();
            for (uint64_t i = 0; i < len; ++i) {
                double u = rng.uni();
                const double* cum = prev == 1 ? cum_c : cum_other;
                int b = u < cum[0] ? 0 : u < cum[1] ? 1 : u < cum[2] ? 2 : 3;
                line.push_back(kBase[b]);
                prev = b;
                if (line.size() == 80) {
                    line.push_back('\n');
                    std::fwrite(line.data(), 1, line.size(), f);
                    line.clear();
                }
            }
            if (!line.empty()) {
                line.push_back('\n');
                std::fwrite(line.data(), 1, line.size(), f);
            }
        }
        if (std::fclose(f) != 0) fail(MA_ERR_IO, "close failed");
        return MA_OK;
    } catch (const Error& e) {
        std::snprintf(err, err_cap, "%s", e.what());
        return e.code;
    } catch (const std::exception& e) {
        std::snprintf(err, err_cap, "%s", e.what());
        return MA_ERR_INTERNAL;
    }
}

namespace {

// Bisulfite treatment of one strand (5'->3'): a C followed by G is
// retained with probability cpg_retain, any other C with 1 - conv.
void bisulfite(std::string& s, Rng& rng, double conv, double cpg_retain) {
    for (size_t i = 0; i < s.size(); ++i) {
        if (s[i] != 'C') continue;
        bool cpg = i + 1 < s.size() && s[i + 1] == 'G';
        bool keep = cpg ? rng.uni() < cpg_retain : rng.uni() >= conv;
        if (!keep) s[i] = 'T';
    }
}

std::string revcomp(const std::string& s) {
    std::string r(s.size(), 'N');
    for (size_t i = 0; i < s.size(); ++i) r[s.size() - 1 - i] = comp(s[i]);
    return r;
}

void substitute(std::string& s, Rng& rng, double rate) {
    if (rate <= 0) return;
    for (auto& ch : s) {
        if (rng.uni() < rate) {
            int cur = ch == 'A' ? 0 : ch == 'C' ? 1 : ch == 'G' ? 2 : 3;
            ch = kBase[(cur + 1 + static_cast<int>(rng.below(3))) & 3];
        }
    }
}

uint32_t draw_len(const ma_read_model* m, Rng& rng) {
    if (m->len_fixed) return m->len_fixed;
    double v = m->len_lognorm_median * std::exp(m->len_lognorm_sigma * rng.normal());
    uint32_t L = static_cast<uint32_t>(std::lround(v));
    if (L < m->len_min) L = m->len_min;
    if (L > m->len_max) L = m->len_max;
    return L;
}

}  // namespace

/*
 * Reads are drawn from uniform positions on the concatenated contigs (the
 * fragment stays within one contig).  Directional libraries give OT / OB:
 * R1 is the 5' end of the converted top (OT) or bottom (OB) strand, R2
 * the reverse complement of the fragment's other end on the same converted
 * strand.  Non-directional reads (CTOT / CTOB) are the reverse complements
 * of those.  Substitutions are applied after conversion; a random read is
 * uniform over ACGT.
 */
extern "C" int ma_synth_reads_impl(const char* fasta, const ma_read_model* m, uint32_t n1, int paired,
                                   uint32_t max_len, uint64_t seed, uint8_t* bases, uint32_t* lens,
                                   uint64_t* truth_pos, uint8_t* truth_rev, char* err, size_t err_cap) {
    try {
        if (!fasta || !m || !bases || !lens) fail(MA_ERR_ARG, "null argument");
        if (max_len == 0 || max_len > 1024) fail(MA_ERR_ARG, "max_len must be in 1..1024");
        std::vector<FastaRecord> recs = read_fasta(fasta);
        std::vector<std::string> seqs;
        std::vector<uint64_t> offs;
        uint64_t tot = 0;
        for (auto& r : recs) {
            for (auto& ch : r.seq) ch = static_cast<char>(std::toupper(static_cast<unsigned char>(ch)));
            offs.push_back(tot);
            tot += r.seq.size();
            seqs.push_back(std::move(r.seq));
        }
        const uint64_t n_seq = paired ? 2ull * n1 : n1;
        std::memset(bases, 'N', n_seq * max_len);
        // 16 fixed chunks, each with its own generator: the output depends on
        // the seed only, not on how many host threads run the chunks.
        constexpr uint32_t kChunks = 16;
        std::vector<std::string> errors(kChunks);
        auto work = [&](uint32_t chunk) {
          try {
            Rng rng(seed * 1000003ull + chunk);
            const uint32_t i0 = static_cast<uint32_t>(static_cast<uint64_t>(n1) * chunk / kChunks);
            const uint32_t i1 = static_cast<uint32_t>(static_cast<uint64_t>(n1) * (chunk + 1) / kChunks);
        for (uint32_t i = i0; i < i1; ++i) {
            uint32_t l1 = draw_len(m, rng), l2 = paired ? draw_len(m, rng) : 0;
            if (l1 > max_len) l1 = max_len;
            if (l2 > max_len) l2 = max_len;
            std::string r1, r2;
            uint64_t tp1 = UINT64_MAX, tp2 = UINT64_MAX;
            uint8_t tr1 = 0, tr2 = 0;
            if (rng.uni() < m->random_frac) {
                for (uint32_t j = 0; j < l1; ++j) r1.push_back(kBase[rng.below(4)]);
                for (uint32_t j = 0; j < l2; ++j) r2.push_back(kBase[rng.below(4)]);
            } else {
                uint32_t flen = l1;
                if (paired) {
                    double fl = m->frag_mean + m->frag_sd * rng.normal();
                    uint32_t need = l1 > l2 ? l1 : l2;
                    flen = fl < need ? need : static_cast<uint32_t>(fl);
                }
                // pick a contig weighted by length that fits the fragment
                uint64_t start = 0;
                size_t ci = 0;
                for (int tries = 0;; ++tries) {
                    uint64_t p = rng.below(tot);
                    ci = static_cast<size_t>(std::upper_bound(offs.begin(), offs.end(), p) - offs.begin()) - 1;
                    if (seqs[ci].size() >= flen) {
                        start = rng.below(seqs[ci].size() - flen + 1);
                        break;
                    }
                    if (tries > 1000) fail(MA_ERR_ARG, "no contig long enough for the fragment");
                }
                std::string top = seqs[ci].substr(start, flen);
                bool bottom = rng.uni() < 0.5;
                std::string strand = bottom ? revcomp(top) : top;
                bisulfite(strand, rng, m->conv_non_cpg, m->cpg_retain);
                bool nondir = rng.uni() < m->non_directional;
                std::string a = strand.substr(0, l1);
                std::string b = paired ? revcomp(strand.substr(flen - l2, l2)) : std::string();
                if (nondir) {
                    // complementary-to-original strands: R1 reads the other end
                    std::string t = paired ? b : revcomp(strand.substr(flen - l1, l1));
                    if (paired) b = a;
                    a = t;
                }
                r1 = a;
                r2 = b;
                // truth: forward text coordinate of the read's leftmost base
                uint64_t fs = offs[ci] + start;
                bool r1_rev = bottom != nondir;
                tr1 = r1_rev ? 1 : 0;
                tp1 = r1_rev ? fs + flen - l1 : fs;
                tr2 = paired ? (r1_rev ? 0 : 1) : 0;
                tp2 = paired ? (r1_rev ? fs : fs + flen - l2) : UINT64_MAX;
                if (nondir && !paired) tp1 = bottom ? fs : fs + flen - l1;
            }
            substitute(r1, rng, m->sub_rate);
            substitute(r2, rng, m->sub_rate);
            std::memcpy(bases + static_cast<uint64_t>(i) * max_len, r1.data(), r1.size());
            lens[i] = static_cast<uint32_t>(r1.size());
            if (truth_pos) truth_pos[i] = tp1;
            if (truth_rev) truth_rev[i] = tr1;
            if (paired) {
                uint64_t j = static_cast<uint64_t>(n1) + i;
                std::memcpy(bases + j * max_len, r2.data(), r2.size());
                lens[j] = static_cast<uint32_t>(r2.size());
                if (truth_pos) truth_pos[j] = tp2;
                if (truth_rev) truth_rev[j] = tr2;
            }
        }
          } catch (const std::exception& ex) {
            errors[chunk] = ex.what();
          }
        };
        std::vector<std::thread> pool;
        for (uint32_t c = 0; c < kChunks; ++c) pool.emplace_back(work, c);
        for (auto& t : pool) t.join();
        for (const auto& m : errors)
            if (!m.empty()) fail(MA_ERR_ARG, m);
        return MA_OK;
    } catch (const Error& e) {
        std::snprintf(err, err_cap, "%s", e.what());
        return e.code;
    } catch (const std::exception& e) {
        std::snprintf(err, err_cap, "%s", e.what());
        return MA_ERR_INTERNAL;
    }
}
