// synth.cpp - seeded synthetic workloads for benchmarks and tests: a
// reference from a first-order base model and bisulfite-converted reads.
// No counterpart in the reference (which only runs on real samples).
#include <algorithm>
#include <atomic>
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

// Seed of the independent stream `idx` of a generator seeded `seed`.  The
// seeds of Rng are mixed first: Rng(x) and Rng(x + 1) would give the same
// sequence one draw apart, since the state advances by the constant that
// multiplies the seed.
uint64_t stream_seed(uint64_t seed, uint64_t idx) {
    uint64_t z = seed * 0xD1B54A32D192ED03ull + idx * 0x9E3779B97F4A7C15ull + 0x8CB92BA72F3D8DD7ull;
    z = (z ^ (z >> 32)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 29)) * 0x94D049BB133111EBull;
    return z ^ (z >> 32);
}

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

// First-order base model of ma_synth_reference (rows for A/G/T and for C).
struct BaseModel {
    double cum_other[4], cum_c[4];
    BaseModel(double gc, double cpg) {
        const double pc = gc / 2;
        double g_after_c = pc > 0 ? cpg / pc : 0;
        if (g_after_c > 0.9) g_after_c = 0.9;
        const double g = (pc - pc * g_after_c) / (1 - pc);
        const double c = pc;
        const double at = (1 - c - g) / 2;
        const double at_c = (1 - c - g_after_c) / 2;
        const double o[4] = {at, at + c, at + c + g, 1.0};
        const double k[4] = {at_c, at_c + c, at_c + c + g_after_c, 1.0};
        for (int i = 0; i < 4; ++i) {
            cum_other[i] = o[i];
            cum_c[i] = k[i];
        }
    }
    int next(Rng& rng, int prev) const {
        const double u = rng.uni();
        const double* cum = prev == 1 ? cum_c : cum_other;
        return u < cum[0] ? 0 : u < cum[1] ? 1 : u < cum[2] ? 2 : 3;
    }
};

int code_of_base(char ch) { return ch == 'A' ? 0 : ch == 'C' ? 1 : ch == 'G' ? 2 : 3; }

// Element families of the repeat model: consensus sequences of the short
// and the long class, shared by every contig.
struct Families {
    std::vector<std::string> cls[2];
};

Families make_families(const ma_repeat_model& rm, const BaseModel& bm, uint64_t seed) {
    Families f;
    Rng rng(stream_seed(seed, 999));
    const uint32_t len[2] = {rm.short_len, rm.long_len};
    for (int c = 0; c < 2; ++c)
        for (uint32_t i = 0; i < rm.families; ++i) {
            std::string e;
            int prev = static_cast<int>(rng.below(4));
            for (uint32_t j = 0; j < len[c]; ++j) {
                prev = bm.next(rng, prev);
                e.push_back(kBase[prev]);
            }
            f.cls[c].push_back(std::move(e));
        }
    return f;
}

// One contig: background from the base model, interleaved (when rm is set)
// with copies of the family elements and with tandem runs, each kind
// emitted while its share of the bases emitted so far is below its target.
std::string make_contig(uint64_t len, const BaseModel& bm, Rng& rng, const ma_repeat_model* rm, const Families* fam) {
    std::string s;
    s.reserve(len);
    uint64_t rep = 0, tan = 0;
    int prev = static_cast<int>(rng.below(4));
    // probability that a copy is of the long class, so that long elements
    // give about long_share of the copied bases (long copies are 5'
    // truncated to 1/8..1 of the element, 9/16 of it on average)
    double q = 0;
    if (rm) {
        const double ls = rm->long_share, lmean = rm->long_len * 9.0 / 16.0;
        q = ls * rm->short_len / (ls * rm->short_len + (1 - ls) * lmean);
    }
    auto put = [&](char ch) {
        if (s.size() < len) s.push_back(ch);
    };
    while (s.size() < len) {
        const double at = static_cast<double>(s.size() + 1);
        const double need_r = rm ? rm->repeat_frac * at - static_cast<double>(rep) : -1;
        const double need_t = rm ? rm->tandem_frac * at - static_cast<double>(tan) : -1;
        const size_t before = s.size();
        if (need_r > 0 && need_r >= need_t && rm->families > 0) {
            // one copy: family element (or a 5' fragment of a long one),
            // substitutions at rate d, 1-bp insertions and deletions at d/20
            // each, either orientation
            const int c = rng.uni() < q ? 1 : 0;
            const std::string& e = fam->cls[c][rng.below(fam->cls[c].size())];
            size_t a = 0, n = e.size();
            if (c == 1) {
                n = static_cast<size_t>(e.size() / 8 + rng.below(e.size() - e.size() / 8 + 1));
                a = e.size() - n;
            }
            std::string cp = e.substr(a, n);
            if (rng.uni() < 0.5) {
                std::string r(cp.size(), 'N');
                for (size_t i = 0; i < cp.size(); ++i) r[cp.size() - 1 - i] = comp(cp[i]);
                cp.swap(r);
            }
            const double d = rm->div_min + (rm->div_max - rm->div_min) * rng.uni();
            for (char ch : cp) {
                const double u = rng.uni();
                if (u < d) {
                    put(kBase[(code_of_base(ch) + 1 + static_cast<int>(rng.below(3))) & 3]);
                } else if (u < d * 1.05) {
                    // deletion: the base is dropped
                } else if (u < d * 1.10) {
                    put(kBase[rng.below(4)]);
                    put(ch);
                } else {
                    put(ch);
                }
            }
            rep += s.size() - before;
        } else if (need_t > 0) {
            // tandem run: a unit of unit_min..unit_max bases repeated over
            // run_min..run_max bases, 2% of them substituted
            const uint32_t ul = rm->unit_min + static_cast<uint32_t>(rng.below(rm->unit_max - rm->unit_min + 1));
            const uint32_t rl = rm->run_min + static_cast<uint32_t>(rng.below(rm->run_max - rm->run_min + 1));
            std::string unit;
            int p = static_cast<int>(rng.below(4));
            for (uint32_t i = 0; i < ul; ++i) {
                p = bm.next(rng, p);
                unit.push_back(kBase[p]);
            }
            for (uint32_t i = 0; i < rl; ++i) {
                char ch = unit[i % ul];
                if (rng.uni() < 0.02) ch = kBase[(code_of_base(ch) + 1 + static_cast<int>(rng.below(3))) & 3];
                put(ch);
            }
            tan += s.size() - before;
        } else {
            // background: a run of geometric length, mean 300
            uint64_t n = 1 + static_cast<uint64_t>(-300.0 * std::log(1.0 - rng.uni() + 1e-300));
            for (uint64_t i = 0; i < n && s.size() < len; ++i) {
                prev = bm.next(rng, prev);
                s.push_back(kBase[prev]);
            }
        }
        if (!s.empty()) prev = code_of_base(s.back());
    }
    return s;
}

}  // namespace

/*
 * The reference model of ma_synth_reference_impl built contig by contig on
 * host threads (each contig with its own generator, so the output depends on
 * the seed only), optionally with the repeat model.  Contig lengths are
 * total_len / n_contigs (the last one takes the remainder).
 */
extern "C" int ma_synth_reference_model_impl(const char* fasta_out, uint64_t total_len, int n_contigs, double gc,
                                             double cpg, uint64_t seed, const ma_repeat_model* rm, char* err,
                                             size_t err_cap) {
    try {
        if (!fasta_out || total_len == 0 || n_contigs <= 0 || gc <= 0 || gc >= 1 || cpg < 0)
            fail(MA_ERR_ARG, "bad synthetic reference arguments");
        if (rm) {
            if (rm->repeat_frac < 0 || rm->tandem_frac < 0 || rm->repeat_frac + rm->tandem_frac >= 0.95 ||
                rm->short_len < 1 || rm->long_len < 8 || rm->div_min < 0 || rm->div_max < rm->div_min ||
                rm->div_max > 0.9 || rm->long_share < 0 || rm->long_share > 1 || rm->unit_min < 1 ||
                rm->unit_max < rm->unit_min || rm->run_min < 1 || rm->run_max < rm->run_min ||
                (rm->repeat_frac > 0 && rm->families < 1))
                fail(MA_ERR_ARG, "bad repeat model");
        }
        const BaseModel bm(gc, cpg);
        Families fam;
        if (rm) fam = make_families(*rm, bm, seed);
        const uint64_t per = total_len / static_cast<uint64_t>(n_contigs);
        std::vector<std::string> text(static_cast<size_t>(n_contigs));
        std::vector<std::string> errors(static_cast<size_t>(n_contigs));
        std::atomic<int> next{0};
        auto work = [&]() {
            for (int ci = next++; ci < n_contigs; ci = next++) {
                try {
                    const uint64_t len =
                        (ci == n_contigs - 1) ? total_len - per * static_cast<uint64_t>(n_contigs - 1) : per;
                    Rng rng(stream_seed(seed, 1000 + static_cast<uint64_t>(ci)));
                    std::string s = make_contig(len, bm, rng, rm, rm ? &fam : nullptr);
                    std::string& t = text[static_cast<size_t>(ci)];
                    t.reserve(s.size() + s.size() / 80 + 64);
                    t += ">chr" + std::to_string(ci + 1) + " synthetic\n";
                    for (size_t i = 0; i < s.size(); i += 80) {
                        t.append(s, i, std::min<size_t>(80, s.size() - i));
                        t.push_back('\n');
                    }
                } catch (const std::exception& ex) {
                    errors[static_cast<size_t>(ci)] = ex.what();
                }
            }
        };
        const unsigned nt = std::max(1u, std::min(static_cast<unsigned>(n_contigs),
                                                  std::min(64u, std::thread::hardware_concurrency())));
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nt; ++t) pool.emplace_back(work);
        for (auto& t : pool) t.join();
        for (const auto& m : errors)
            if (!m.empty()) fail(MA_ERR_INTERNAL, m);
        FILE* f = std::fopen(fasta_out, "wb");
        if (!f) fail(MA_ERR_IO, std::string("cannot write ") + fasta_out);
        for (const auto& t : text) {
            if (std::fwrite(t.data(), 1, t.size(), f) != t.size()) {
                std::fclose(f);
                fail(MA_ERR_IO, "short write of the synthetic reference");
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
            Rng rng(stream_seed(seed, chunk));
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
