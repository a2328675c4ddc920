/*
 * oracle_fm.c - CPU ORACLE for the linear bisulfite seed-and-extend path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: only tests/, the
 * smoke() entry and bench.py's CPU-baseline / reference arm may load it.
 * The product (mojo-align_b200/) never links, calls or falls back to it.
 *
 * It restates, line by line and on the CPU, the reference's own algorithm
 * (mojo-align; paths relative to its source tree):
 *   - bwa 0.7 index files as FmIndex.load reads them
 *       fq2bam-meth/src/linear_fm_index.mojo:88-175
 *   - FmIndex host methods pac_base / occ / inv_psi / sa_at / match_exact /
 *     depos                      linear_fm_index.mojo:206-320
 *   - _cvt (C->T / G->A)         fq2bam-meth/src/linear_fastq.mojo:29-46
 *   - pack_bases_kernel          fq2bam-meth/src/linear_gpu_fm.mojo:1136-1154
 *   - fm_seed_extend_kernel      linear_gpu_fm.mojo:1156-1837
 *   - fm_mate_rescue_kernel      linear_gpu_fm.mojo:1839-2011
 * with one thread per read (OpenMP) instead of one GPU thread per read.
 *
 * Behaviour the reference leaves undefined, and what this file does:
 *   - The 1-bp deletion probe of the seed kernel (L1735-1813) can index
 *     pac at a negative text position when b0 < 0 (a seed close to text
 *     position 0).  The reference then reads the byte before its pac
 *     buffer.  Here such a base reads as 4 ("not a base", a mismatch), the
 *     value FmIndex.pac_base returns off the text (linear_fm_index.mojo:
 *     206-208).
 * Parity status: the reference (Mojo, GPU-only for this path) cannot run
 * in this environment, and it publishes no per-read outputs.  This file is
 * pinned against the reference's own known-answer tests (FASTQ conversion
 * and pack vectors, convert_fastq vectors, the FM round-trip property and
 * the toy fixture; see tests/), not against reference outputs.
 */
#define _POSIX_C_SOURCE 200809L /* strdup */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct orc_index {
    uint64_t primary, seq_len, l_pac;
    uint64_t L2[5];
    int64_t sa_intv, n_sa;
    uint32_t *bwt;
    int64_t bwt_size; /* u32 words after the 40-byte header */
    uint64_t *sa;     /* sa[1..n_sa-1] of the file; element i holds SA[(i+1)*intv] */
    uint8_t *pac;
    int64_t pac_size;
    int64_t n_contigs;
    uint64_t *contig_off;
    uint32_t *contig_len;
    char **contig_name;
} orc_index;

/* Per-read traffic counters of the reference algorithm (64-B BWT lines). */
typedef struct orc_counters {
    uint64_t occ_lines;  /* distinct 64-B .bwt lines per backward step     */
    uint64_t lf_lines;   /* 64-B lines read by the sampled-SA walk          */
    uint64_t sa_loads;   /* 8-B sampled SA loads                            */
    uint64_t pac_sectors;/* 32-B pac sectors per extension / rescue compare */
    uint64_t endpoints;  /* right endpoints searched                         */
    uint64_t steps;      /* backward-search steps                            */
    uint64_t rows;       /* SA rows resolved                                 */
    uint64_t extends;    /* (locus, adj) candidates compared                 */
    uint64_t capped;     /* searches stopped by occ > max_occ (L1378-1379)   */
    uint64_t fallback;   /* seeds taken from the <= 16-row fallback (L1381-1385) */
} orc_counters;

static char g_err[512];
const char *orc_last_error(void) { return g_err; }

static void *read_file(const char *path, int64_t *size) {
    FILE *f = fopen(path, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    void *buf = malloc(n > 0 ? (size_t)n : 1);
    if (n > 0 && fread(buf, 1, (size_t)n, f) != (size_t)n) {
        free(buf);
        fclose(f);
        return NULL;
    }
    fclose(f);
    *size = n;
    return buf;
}

static uint64_t rd_u64(const uint8_t *p, int64_t idx) {
    /* FmIndex._u64: little-endian, linear_fm_index.mojo:177-186 */
    uint64_t v = 0;
    for (int b = 0; b < 8; ++b) v |= (uint64_t)p[idx * 8 + b] << (8 * b);
    return v;
}

void orc_index_free(orc_index *ix) {
    if (!ix) return;
    free(ix->bwt);
    free(ix->sa);
    free(ix->pac);
    free(ix->contig_off);
    free(ix->contig_len);
    if (ix->contig_name)
        for (int64_t i = 0; i < ix->n_contigs; ++i) free(ix->contig_name[i]);
    free(ix->contig_name);
    free(ix);
}

/* FmIndex.load, linear_fm_index.mojo:88-175.  Returns 0 or -1. */
int orc_index_load(const char *prefix, orc_index **out) {
    char path[4096];
    int64_t nb = 0, ns = 0, np = 0;
    orc_index *ix = (orc_index *)calloc(1, sizeof(orc_index));
    snprintf(path, sizeof path, "%s.bwt", prefix);
    uint8_t *bwt = (uint8_t *)read_file(path, &nb);
    snprintf(path, sizeof path, "%s.sa", prefix);
    uint8_t *sa = (uint8_t *)read_file(path, &ns);
    snprintf(path, sizeof path, "%s.pac", prefix);
    uint8_t *pac = (uint8_t *)read_file(path, &np);
    if (!bwt || !sa || !pac || nb < 40 || ns < 56) {
        snprintf(g_err, sizeof g_err, "FmIndex missing or short file under %s", prefix);
        free(bwt); free(sa); free(pac); free(ix);
        return -1;
    }
    ix->bwt_size = (nb - 40) / 4;                      /* L119 */
    ix->primary = rd_u64(bwt, 0);                      /* L120 */
    ix->L2[0] = 0;
    for (int c = 1; c <= 4; ++c) ix->L2[c] = rd_u64(bwt, c);
    ix->seq_len = ix->L2[4];                           /* L126 */
    if (rd_u64(sa, 0) != ix->primary) {                /* L128-130 */
        snprintf(g_err, sizeof g_err, "FmIndex SA/BWT primary mismatch");
        goto fail;
    }
    ix->sa_intv = (int64_t)rd_u64(sa, 5);              /* L131 */
    if (rd_u64(sa, 6) != ix->seq_len) {                /* L132-134 */
        snprintf(g_err, sizeof g_err, "FmIndex SA/BWT seq_len mismatch");
        goto fail;
    }
    if (ix->sa_intv <= 0) {
        snprintf(g_err, sizeof g_err, "FmIndex bad sa_intv");
        goto fail;
    }
    ix->n_sa = (int64_t)((ix->seq_len + (uint64_t)ix->sa_intv) / (uint64_t)ix->sa_intv); /* L135 */
    ix->bwt = (uint32_t *)malloc((size_t)(ix->bwt_size + 2) * 4);
    memcpy(ix->bwt, bwt + 40, (size_t)ix->bwt_size * 4);
    ix->bwt[ix->bwt_size] = ix->bwt[ix->bwt_size + 1] = 0;
    {
        int64_t nsa = ix->n_sa - 1;
        if (56 + nsa * 8 > ns) {
            snprintf(g_err, sizeof g_err, "FmIndex short .sa");
            goto fail;
        }
        ix->sa = (uint64_t *)malloc((size_t)(nsa > 0 ? nsa : 1) * 8);
        for (int64_t i = 0; i < nsa; ++i) ix->sa[i] = rd_u64(sa + 56, i);
    }
    ix->pac = pac;
    ix->pac_size = np;
    pac = NULL;
    free(bwt);
    free(sa);
    bwt = sa = NULL;
    /* .ann, L137-160 */
    {
        snprintf(path, sizeof path, "%s.ann", prefix);
        FILE *f = fopen(path, "r");
        if (!f) {
            snprintf(g_err, sizeof g_err, "FmIndex missing %.400s", path);
            goto fail;
        }
        char line[8192];
        unsigned long long lp = 0;
        long long nseq = 0;
        if (!fgets(line, sizeof line, f) || sscanf(line, "%llu %lld", &lp, &nseq) != 2) {
            fclose(f);
            snprintf(g_err, sizeof g_err, "FmIndex bad .ann header");
            goto fail;
        }
        ix->l_pac = lp;
        ix->n_contigs = nseq;
        ix->contig_off = (uint64_t *)calloc((size_t)(nseq > 0 ? nseq : 1), 8);
        ix->contig_len = (uint32_t *)calloc((size_t)(nseq > 0 ? nseq : 1), 4);
        ix->contig_name = (char **)calloc((size_t)(nseq > 0 ? nseq : 1), sizeof(char *));
        uint64_t off = 0;
        for (long long i = 0; i < nseq; ++i) {
            char l1[8192], l2[8192], nm[4096];
            long long a = 0, ln = 0;
            if (!fgets(l1, sizeof l1, f) || !fgets(l2, sizeof l2, f) ||
                sscanf(l1, "%lld %4095s", &a, nm) != 2 || sscanf(l2, "%lld %lld", &a, &ln) != 2) {
                fclose(f);
                snprintf(g_err, sizeof g_err, "FmIndex truncated .ann");
                goto fail;
            }
            ix->contig_name[i] = strdup(nm);
            ix->contig_len[i] = (uint32_t)ln;
            ix->contig_off[i] = off;
            off += (uint64_t)ln;
        }
        fclose(f);
        if (off != ix->l_pac) {
            snprintf(g_err, sizeof g_err, "FmIndex .ann offsets != l_pac");
            goto fail;
        }
    }
    *out = ix;
    return 0;
fail:
    free(bwt);
    free(sa);
    free(pac);
    orc_index_free(ix);
    return -1;
}

void orc_index_header(const orc_index *ix, uint64_t out[12]) {
    out[0] = ix->primary;
    out[1] = ix->seq_len;
    out[2] = ix->l_pac;
    for (int c = 0; c < 5; ++c) out[3 + c] = ix->L2[c];
    out[8] = (uint64_t)ix->sa_intv;
    out[9] = (uint64_t)ix->n_sa;
    out[10] = (uint64_t)ix->n_contigs;
    out[11] = (uint64_t)ix->bwt_size;
}

int64_t orc_contig(const orc_index *ix, int64_t i, uint64_t *off, uint32_t *len, char *name, int cap) {
    if (i < 0 || i >= ix->n_contigs) return -1;
    *off = ix->contig_off[i];
    *len = ix->contig_len[i];
    snprintf(name, (size_t)cap, "%s", ix->contig_name[i]);
    return 0;
}

/* ---------------- FmIndex host methods (linear_fm_index.mojo) ---------- */

/* pac_base, L206-212 */
int orc_pac_base(const orc_index *ix, int64_t pos) {
    if (pos < 0 || (uint64_t)pos >= ix->l_pac) return 4;
    uint8_t byte = ix->pac[pos >> 2];
    return (byte >> (((~pos) & 3) << 1)) & 3;
}

/* _occ_aux, L214-234 */
static inline uint64_t occ_aux(uint64_t y, int c) {
    uint64_t a = (c & 2) ? y : ~y;
    uint64_t b = (c & 1) ? y : ~y;
    y = (a >> 1) & b & 0x5555555555555555ULL;
    return (uint64_t)__builtin_popcountll(y);
}

/* Inline Occ of the kernels (L1261-1345), identical arithmetic to
 * FmIndex.occ (L242-275).  k_m is the signed row; returns count of c in
 * BWT[0..k_m]. */
static inline uint64_t occ_k(const orc_index *ix, int64_t k_m, int cc) {
    if (k_m < 0) return 0;
    if ((uint64_t)k_m == ix->seq_len) return ix->L2[cc + 1] - ix->L2[cc];
    uint64_t kko = (uint64_t)k_m;
    if (kko >= ix->primary) kko -= 1;
    int64_t baseo = (int64_t)((kko >> 7) << 4);
    const uint32_t *bwt = ix->bwt;
    uint64_t nocc = (uint64_t)bwt[baseo + cc * 2] | ((uint64_t)bwt[baseo + cc * 2 + 1] << 32);
    int64_t po = baseo + 8;
    int64_t endo = po + (int64_t)(((kko >> 5) - ((kko & 0xFFFFFFFFFFFFFF80ULL) >> 5)) << 1);
    while (po < endo) {
        uint64_t yo = ((uint64_t)bwt[po] << 32) | (uint64_t)bwt[po + 1];
        nocc += occ_aux(yo, cc);
        po += 2;
    }
    int64_t bitso = (int64_t)(((~(int64_t)kko) & 31) << 1);
    uint64_t masko = 0xFFFFFFFFFFFFFFFFULL;
    if (bitso > 0 && bitso < 64) masko = ~((1ULL << (uint64_t)bitso) - 1);
    uint64_t y5 = (((uint64_t)bwt[po] << 32) | (uint64_t)bwt[po + 1]) & masko;
    nocc += occ_aux(y5, cc);
    if (cc == 0) nocc -= (uint64_t)((~(int64_t)kko) & 31);
    return nocc;
}

uint64_t orc_occ(const orc_index *ix, int64_t k, int c) { return occ_k(ix, k, c); }

/* b0, L236-240: BWT symbol at (already primary-adjusted) position k */
static inline int bwt_b0(const orc_index *ix, uint64_t k) {
    int64_t kk = (int64_t)k;
    int64_t idx = ((kk >> 7) << 4) + 8 + ((kk & 0x7F) >> 4);
    uint32_t w = ix->bwt[idx];
    return (int)((w >> (((~kk) & 15) << 1)) & 3);
}

/* inv_psi, L277-284 */
uint64_t orc_inv_psi(const orc_index *ix, uint64_t k) {
    if (k == ix->primary) return 0;
    uint64_t x = k;
    if (k > ix->primary) x -= 1;
    int c = bwt_b0(ix, x);
    return ix->L2[c] + occ_k(ix, (int64_t)k, c);
}

/* sa_at, L286-293 (host variant: walks through primary via inv_psi) */
uint64_t orc_sa_at(const orc_index *ix, uint64_t k) {
    uint64_t kk = k, sa = 0;
    uint64_t mask = (uint64_t)(ix->sa_intv - 1);
    uint64_t guard = 0;
    while ((kk & mask) != 0) {
        sa += 1;
        kk = orc_inv_psi(ix, kk);
        if (++guard > ix->seq_len + 1) return UINT64_MAX; /* corrupt index */
    }
    int64_t idx = (int64_t)(kk / (uint64_t)ix->sa_intv);
    if (idx <= 0) return sa + UINT64_MAX; /* _sa_sample(0) = -1 */
    return sa + ix->sa[idx - 1];
}

/* match_exact, L295-313.  Returns occ (0 = no match). */
int64_t orc_match_exact(const orc_index *ix, const uint8_t *codes, int64_t length,
                        uint64_t *k_out, uint64_t *l_out) {
    uint64_t k = 0, l = ix->seq_len;
    for (int64_t i = length - 1; i >= 0; --i) {
        int c = codes[i];
        if (c > 3) return 0;
        uint64_t ok = occ_k(ix, (int64_t)k - 1, c);
        uint64_t ol = occ_k(ix, (int64_t)l, c);
        k = ix->L2[c] + ok + 1;
        l = ix->L2[c] + ol;
        if (k > l) return 0;
    }
    *k_out = k;
    *l_out = l;
    return (int64_t)(l - k + 1);
}

/* depos, L315-320 */
void orc_depos(const orc_index *ix, uint64_t pos, int64_t *fpos, int *is_rev) {
    if (pos >= ix->l_pac) {
        *fpos = (int64_t)(ix->l_pac * 2 - 1 - pos);
        *is_rev = 1;
    } else {
        *fpos = (int64_t)pos;
        *is_rev = 0;
    }
}

/* ---------------- read conversion and pack ----------------------------- */

/* _cvt, linear_fastq.mojo:37-46 */
static inline uint8_t cvt(uint8_t c, int mode) {
    if (mode == 1) return (c == 67 || c == 99) ? 84 : c;
    if (mode == 2) return (c == 71 || c == 103) ? 65 : c;
    return c;
}

void orc_convert(uint8_t *seq, int64_t n, int mode) {
    for (int64_t i = 0; i < n; ++i) seq[i] = cvt(seq[i], mode);
}

/* pack_bases_kernel, linear_gpu_fm.mojo:1136-1154 */
static inline uint8_t pack1(uint8_t b) {
    if (b == 65 || b == 97) return 0;
    if (b == 67 || b == 99) return 1;
    if (b == 71 || b == 103) return 2;
    if (b == 84 || b == 116) return 3;
    return 255;
}

void orc_pack_bases(const uint8_t *bases, uint8_t *codes, int64_t n) {
    for (int64_t i = 0; i < n; ++i) codes[i] = pack1(bases[i]);
}

/* ---------------- fm_seed_extend_kernel -------------------------------- */

static inline int64_t pac_rb(const orc_index *ix, int64_t ppos) {
    /* the kernel's inline pac read (e.g. L1569-1575); negative positions
     * are undefined in the reference and read as 4 here (file header). */
    if (ppos < 0) return 4;
    return (int64_t)((ix->pac[ppos >> 2] >> (((~ppos) & 3) << 1)) & 3);
}

static inline void count_pac(orc_counters *ct, int64_t a, int64_t b) {
    /* 32-B pac sectors covering text positions [a, b] */
    if (!ct || b < a) return;
    if (a < 0) a = 0;
    if (b < 0) return;
    ct->pac_sectors += (uint64_t)(((b >> 2) >> 5) - ((a >> 2) >> 5) + 1);
}

typedef struct orc_params {
    int64_t seed_len, seed_stride, max_occ, max_diff, max_soft, max_adj, rescue_win;
} orc_params;

static void seed_extend_one(const orc_index *ix, const uint8_t *codes, const uint32_t *read_lens,
                            int64_t max_len, int64_t rid, const orc_params *P,
                            int32_t *out_rid, uint32_t *out_pos, uint32_t *out_mapq,
                            int32_t *out_flag, uint32_t *out_sl, uint32_t *out_sr,
                            uint32_t *out_nm, uint64_t *d_uk, uint64_t *d_ul, int32_t *d_us,
                            int32_t *d_e, orc_counters *ct) {
    const uint64_t primary = ix->primary, seq_len = ix->seq_len, l_pac = ix->l_pac;
    const int64_t sa_intv = ix->sa_intv, n_sa = ix->n_sa, n_contigs = ix->n_contigs;
    const uint32_t *bwt = ix->bwt;
    const int64_t seed_len = P->seed_len, seed_stride = P->seed_stride, max_occ = P->max_occ;
    /* L1194-1200 */
    out_rid[rid] = -1;
    out_pos[rid] = 0;
    out_mapq[rid] = 0;
    out_flag[rid] = 4;
    out_sl[rid] = 0;
    out_sr[rid] = 0;
    out_nm[rid] = 0;
    if (d_us) { d_uk[rid] = 0; d_ul[rid] = 0; d_us[rid] = -1; d_e[rid] = -1; }
    int64_t qlen = (int64_t)read_lens[rid];
    if (qlen < seed_len) return;                       /* L1202-1203 */
    int64_t budget = P->max_diff;                      /* L1204-1216 */
    if (budget < 2) budget = 2;
    if (budget > qlen / 2) budget = qlen / 2;
    int64_t clip_cap = P->max_soft;
    if (clip_cap > qlen / 4) clip_cap = qlen / 4;
    int64_t adj_cap = P->max_adj;
    if (adj_cap < 0) adj_cap = 0;
    if (adj_cap > 12) adj_cap = 12;
    int64_t q_base = rid * max_len;
    const uint64_t *L2 = ix->L2;

    int64_t best_nm = 9999, best_rid = -1, best_pos = 0, best_sl = 0, best_sr = 0;
    uint32_t best_mq = 0;
    int64_t best_flag = 0;
    uint64_t b_uk = 0, b_ul = 0;
    int64_t b_us = -1, b_e = -1;

    int64_t e = seed_len - 1;                          /* L1233 */
    while (e < qlen) {
        uint64_t k = 0, l = seq_len, uk = 0, ul = 0, last_k = 0, last_l = 0;
        int64_t s = e, us = -1, last_s = -1;
        int found = 0;
        if (ct) ct->endpoints++;
        while (s >= 0) {                               /* L1245 */
            int64_t cc = (int64_t)codes[q_base + s];
            if (cc > 3) break;
            uint64_t ok = 0, ol = 0;
            /* pass 0 (k-1, skipped when k == 0) and pass 1 (l), L1251-1354 */
            if (k != 0) ok = occ_k(ix, (int64_t)(k - 1), (int)cc);
            ol = occ_k(ix, (int64_t)l, (int)cc);
            if (ct) {
                ct->steps++;
                int nl = 0;
                int64_t la = -1, lb = -1;
                if (k != 0 && (k - 1) != seq_len) {
                    uint64_t x = k - 1; if (x >= primary) x -= 1; la = (int64_t)(x >> 7); nl++;
                }
                if (l != seq_len) {
                    uint64_t x = l; if (x >= primary) x -= 1; lb = (int64_t)(x >> 7);
                    if (lb != la) nl++;
                }
                ct->occ_lines += (uint64_t)nl;
            }
            uint64_t Lc = L2[cc];                      /* L1355-1363 */
            k = Lc + ok + 1;
            l = Lc + ol;
            if (k > l) break;
            int64_t occ_n = (int64_t)(l - k + 1);
            int64_t mlen = e - s + 1;
            if (occ_n == 1 && mlen >= seed_len) {      /* L1368-1373 */
                uk = k; ul = l; us = s; found = 1;
                break;
            }
            if (occ_n >= 1 && occ_n <= 16 && mlen >= seed_len) { /* L1374-1377 */
                last_k = k; last_l = l; last_s = s;
            }
            if (occ_n > max_occ && mlen >= seed_len) {           /* L1378-1379 */
                if (ct) ct->capped++;
                break;
            }
            s -= 1;
        }
        if (!found && last_s >= 0) {                   /* L1381-1385 */
            uk = last_k; ul = last_l; us = last_s; found = 1;
            if (ct) ct->fallback++;
        }
        if (found) {
            uint64_t hi = uk;
            while (hi <= ul) {                         /* L1387-1388 */
                if (ct) ct->rows++;
                /* sampled-SA walk, L1390-1508 */
                uint64_t kk = hi, sa_v = 0;
                uint64_t smask = (uint64_t)(sa_intv - 1);
                int sa_ok = 1;
                while ((kk & smask) != 0) {
                    sa_v += 1;
                    if (kk == primary) { kk = 0; break; }
                    uint64_t xpsi = kk;
                    if (kk > primary) xpsi -= 1;
                    int64_t bi = (int64_t)xpsi;
                    int64_t bidx = ((bi >> 7) << 4) + 8 + ((bi & 0x7F) >> 4);
                    uint32_t w = bwt[bidx];
                    int64_t cc = (int64_t)((w >> (((~bi) & 15) << 1)) & 3);
                    uint64_t nocc = occ_k(ix, (int64_t)kk, (int)cc);
                    if (ct) ct->lf_lines++;
                    kk = L2[cc] + nocc;
                }
                int64_t sidx = (int64_t)(kk / (uint64_t)sa_intv);
                if (sidx <= 0 || sidx >= n_sa) sa_ok = 0;
                uint64_t sa_pos = sa_v;
                if (sa_ok) {
                    sa_pos = sa_v + ix->sa[sidx - 1];
                    if (ct) ct->sa_loads++;
                }
                if (sa_ok) {                           /* strand, L1509-1524 */
                    int64_t is_rev = 0, b0 = 0;
                    int64_t plen = e - us + 1;
                    if (sa_pos < l_pac) {
                        b0 = (int64_t)sa_pos - us;
                        is_rev = 0;
                    } else {
                        uint64_t seed_end = sa_pos + (uint64_t)plen - 1;
                        if (seed_end >= l_pac * 2) {
                            sa_ok = 0;
                        } else {
                            int64_t fp_end = (int64_t)(l_pac * 2 - 1 - sa_pos);
                            int64_t fp_start = fp_end - (plen - 1);
                            b0 = fp_start - (qlen - 1 - e);
                            is_rev = 1;
                        }
                    }
                    if (sa_ok) {
                        for (int64_t adj = -adj_cap; adj <= adj_cap; ++adj) { /* L1526-1527 */
                            int64_t bstart = b0 + adj;
                            int64_t probe = bstart;
                            if (probe < 0) probe = 0;
                            if ((uint64_t)probe >= l_pac) probe = (int64_t)l_pac - 1;
                            int64_t lo = 0, hi2 = n_contigs, crid = -1; /* L1536-1549 */
                            while (lo < hi2) {
                                int64_t mid = (lo + hi2) / 2;
                                int64_t off = (int64_t)ix->contig_off[mid];
                                int64_t ln = (int64_t)ix->contig_len[mid];
                                if (probe < off) hi2 = mid;
                                else if (probe >= off + ln) lo = mid + 1;
                                else { crid = mid; break; }
                            }
                            if (crid < 0) continue;
                            int64_t coff = (int64_t)ix->contig_off[crid];
                            int64_t clen = (int64_t)ix->contig_len[crid];
                            int64_t local = bstart - coff;
                            int64_t sl0 = 0, sr0 = 0;
                            if (local < 0) sl0 = -local;
                            if (local + qlen > clen) sr0 = local + qlen - clen;
                            if (!(sl0 + sr0 < qlen && sl0 <= clip_cap && sr0 <= clip_cap)) continue;
                            if (ct) ct->extends++;
                            int64_t nm_all = 0, j = sl0;  /* L1565-1587 */
                            while (j < qlen - sr0 && nm_all <= budget) {
                                int64_t ppos = bstart + j;
                                int64_t rb = pac_rb(ix, ppos);
                                int64_t qc = (int64_t)codes[q_base + j];
                                if (is_rev != 0) {
                                    int64_t qcr = (int64_t)codes[q_base + (qlen - 1 - j)];
                                    qc = qcr <= 3 ? 3 - qcr : 4;
                                }
                                if (rb > 3 || qc > 3 || rb != qc) nm_all += 1;
                                j += 1;
                            }
                            count_pac(ct, bstart + sl0, bstart + j - 1);
                            int64_t sl = sl0, sr = sr0, nm = nm_all;
                            if (nm_all > budget && clip_cap > 0) { /* L1591-1694 */
                                while (sl < clip_cap) {
                                    int64_t p0 = bstart + sl;
                                    if (p0 < coff || p0 >= coff + clen) { sl += 1; continue; }
                                    int64_t rb0 = pac_rb(ix, p0);
                                    int64_t qc0 = (int64_t)codes[q_base + sl];
                                    if (is_rev != 0) {
                                        int64_t q0r = (int64_t)codes[q_base + (qlen - 1 - sl)];
                                        qc0 = q0r <= 3 ? 3 - q0r : 4;
                                    }
                                    if (rb0 <= 3 && qc0 <= 3 && rb0 == qc0) break;
                                    sl += 1;
                                }
                                while (sr < clip_cap) {
                                    int64_t jr = qlen - 1 - sr;
                                    if (jr <= sl) break;
                                    int64_t p1 = bstart + jr;
                                    if (p1 < coff || p1 >= coff + clen) { sr += 1; continue; }
                                    int64_t rb1 = pac_rb(ix, p1);
                                    int64_t qc1 = (int64_t)codes[q_base + jr];
                                    if (is_rev != 0) {
                                        int64_t q1r = (int64_t)codes[q_base + (qlen - 1 - jr)];
                                        qc1 = q1r <= 3 ? 3 - q1r : 4;
                                    }
                                    if (rb1 <= 3 && qc1 <= 3 && rb1 == qc1) break;
                                    sr += 1;
                                }
                                nm = 0;
                                int64_t jm = sl;
                                while (jm < qlen - sr && nm <= budget) {
                                    int64_t pm = bstart + jm;
                                    int64_t rbm = pac_rb(ix, pm);
                                    int64_t qcm = (int64_t)codes[q_base + jm];
                                    if (is_rev != 0) {
                                        int64_t qmr = (int64_t)codes[q_base + (qlen - 1 - jm)];
                                        qcm = qmr <= 3 ? 3 - qmr : 4;
                                    }
                                    if (rbm > 3 || qcm > 3 || rbm != qcm) nm += 1;
                                    jm += 1;
                                }
                                count_pac(ct, bstart + sl, bstart + jm - 1);
                            }
                            int64_t alen = qlen - sl - sr;
                            if (nm <= budget && alen >= 24) { /* L1696-1728 */
                                if (nm < best_nm) {
                                    best_nm = nm;
                                    best_rid = crid;
                                    best_pos = local + sl;
                                    best_sl = sl;
                                    best_sr = sr;
                                    best_mq = nm == 0 ? 60 : 20;
                                    best_flag = is_rev * 16;
                                    b_uk = uk; b_ul = ul; b_us = us; b_e = e;
                                    if (best_nm == 0) {
                                        out_rid[rid] = (int32_t)best_rid;
                                        out_pos[rid] = (uint32_t)best_pos;
                                        out_mapq[rid] = best_mq;
                                        out_flag[rid] = (int32_t)best_flag;
                                        out_sl[rid] = (uint32_t)best_sl;
                                        out_sr[rid] = (uint32_t)best_sr;
                                        out_nm[rid] = (uint32_t)best_nm;
                                        if (d_us) { d_uk[rid] = b_uk; d_ul[rid] = b_ul; d_us[rid] = (int32_t)b_us; d_e[rid] = (int32_t)b_e; }
                                        return;
                                    }
                                }
                            } else if (adj == 0 && is_rev == 0 && (nm > budget || alen < 24)) {
                                /* 1bp deletion on a coarse g grid, L1729-1825 */
                                if (bstart + qlen + 1 <= coff + clen) {
                                    for (int64_t g = 0; g <= qlen; g += 4) {
                                        int64_t nm_d = 1, t = 0;
                                        while (t < g && nm_d <= budget) {
                                            int64_t rcd = pac_rb(ix, bstart + t);
                                            int64_t qcd = (int64_t)codes[q_base + t];
                                            if (rcd > 3 || qcd > 3 || rcd != qcd) nm_d += 1;
                                            t += 1;
                                        }
                                        while (t < qlen && nm_d <= budget) {
                                            int64_t rcd2 = pac_rb(ix, bstart + t + 1);
                                            int64_t qcd2 = (int64_t)codes[q_base + t];
                                            if (rcd2 > 3 || qcd2 > 3 || rcd2 != qcd2) nm_d += 1;
                                            t += 1;
                                        }
                                        count_pac(ct, bstart, bstart + t);
                                        if (nm_d <= budget && nm_d < best_nm) {
                                            best_nm = nm_d;
                                            best_rid = crid;
                                            best_pos = local;
                                            best_sl = 0;
                                            best_sr = 0;
                                            best_mq = 20;
                                            best_flag = 0;
                                            b_uk = uk; b_ul = ul; b_us = us; b_e = e;
                                        }
                                    }
                                }
                            }
                        }
                    }
                }
                hi += 1;
            }
        }
        e += seed_stride;                              /* L1828 */
    }
    if (best_rid >= 0) {                               /* L1830-1837 */
        out_rid[rid] = (int32_t)best_rid;
        out_pos[rid] = (uint32_t)best_pos;
        out_mapq[rid] = best_mq;
        out_flag[rid] = (int32_t)best_flag;
        out_sl[rid] = (uint32_t)best_sl;
        out_sr[rid] = (uint32_t)best_sr;
        out_nm[rid] = (uint32_t)best_nm;
        if (d_us) { d_uk[rid] = b_uk; d_ul[rid] = b_ul; d_us[rid] = (int32_t)b_us; d_e[rid] = (int32_t)b_e; }
    }
}

/* ---------------- fm_mate_rescue_kernel --------------------------------- */

static void mate_rescue_one(const orc_index *ix, const uint8_t *codes, const uint32_t *read_lens,
                            int64_t max_len, int64_t n_pairs, int64_t pi, const orc_params *P,
                            int32_t *out_rid, uint32_t *out_pos, uint32_t *out_mapq,
                            int32_t *out_flag, uint32_t *out_sl, uint32_t *out_sr,
                            uint32_t *out_nm, orc_counters *ct) {
    const int64_t n_contigs = ix->n_contigs;
    const uint64_t l_pac = ix->l_pac;
    int64_t i1 = pi, i2 = pi + n_pairs;                /* L1865-1870 */
    int m1 = (int64_t)out_rid[i1] >= 0;
    int m2 = (int64_t)out_rid[i2] >= 0;
    if (m1 == m2) return;
    int64_t src = i1, dst = i2;
    if (m2) { src = i2; dst = i1; }
    int64_t crid = (int64_t)out_rid[src];
    if (crid < 0 || crid >= n_contigs) return;
    int64_t qlen = (int64_t)read_lens[dst];
    if (qlen < 24) return;
    int64_t coff = (int64_t)ix->contig_off[crid];
    int64_t clen = (int64_t)ix->contig_len[crid];
    int64_t mate_pos = (int64_t)out_pos[src];
    int64_t win = P->rescue_win;                       /* L1885-1897 */
    if (win < 32) win = 32;
    if (win > 1024) win = 1024;
    int64_t lo = mate_pos - win;
    if (lo < 0) lo = 0;
    int64_t hi = mate_pos + win;
    if (hi > clen - 24) hi = clen - 24;
    if (hi <= lo) return;
    int64_t budget = P->max_diff;
    if (budget < 2) budget = 2;
    if (budget > qlen / 2) budget = qlen / 2;
    int64_t q_base = dst * max_len;
    int64_t best_nm = 9999, best_pos = 0, best_flag = 0;
    int64_t scan_nm = 9999, scan_local = lo, scan_rev = 0;
    int mate_rev = ((int64_t)out_flag[src] & 16) != 0;
    for (int64_t pass_s = 0; pass_s < 2; ++pass_s) {   /* L1911-1956 */
        int64_t is_rev;
        if (pass_s == 0) is_rev = mate_rev ? 0 : 1;
        else is_rev = mate_rev ? 1 : 0;
        for (int64_t local = lo; local <= hi; ++local) {
            int64_t bstart = coff + local;
            if (bstart < 0 || (uint64_t)(bstart + qlen) > l_pac) continue;
            int64_t nm = 0, j = 0;
            while (j < qlen && nm <= budget + 4) {
                int64_t ppos = bstart + j;
                int64_t rb = pac_rb(ix, ppos);
                int64_t qc = (int64_t)codes[q_base + j];
                if (is_rev != 0) {
                    int64_t qcr = (int64_t)codes[q_base + (qlen - 1 - j)];
                    qc = qcr <= 3 ? 3 - qcr : 4;
                }
                if (rb > 3 || qc > 3 || rb != qc) nm += 1;
                j += 1;
            }
            count_pac(ct, bstart, bstart + j - 1);
            if (nm < scan_nm) { scan_nm = nm; scan_local = local; scan_rev = is_rev; }
            if (nm <= budget && nm < best_nm) { best_nm = nm; best_pos = local; best_flag = is_rev * 16; }
        }
    }
    if (best_nm > budget && scan_nm < 9999) {           /* L1957-1998 */
        int64_t bstart = coff + scan_local;
        if (bstart >= 0 && (uint64_t)(bstart + qlen + 1) <= l_pac) {
            for (int64_t g = 0; g <= qlen; g += 4) {
                int64_t nm_d = 1, t = 0;
                while (t < g && nm_d <= budget) {
                    int64_t rb0 = pac_rb(ix, bstart + t);
                    int64_t qc0 = (int64_t)codes[q_base + t];
                    if (scan_rev != 0) {
                        int64_t q0r = (int64_t)codes[q_base + (qlen - 1 - t)];
                        qc0 = q0r <= 3 ? 3 - q0r : 4;
                    }
                    if (rb0 > 3 || qc0 > 3 || rb0 != qc0) nm_d += 1;
                    t += 1;
                }
                while (t < qlen && nm_d <= budget) {
                    int64_t rb1 = pac_rb(ix, bstart + t + 1);
                    int64_t qc1 = (int64_t)codes[q_base + t];
                    if (scan_rev != 0) {
                        int64_t q1r = (int64_t)codes[q_base + (qlen - 1 - t)];
                        qc1 = q1r <= 3 ? 3 - q1r : 4;
                    }
                    if (rb1 > 3 || qc1 > 3 || rb1 != qc1) nm_d += 1;
                    t += 1;
                }
                count_pac(ct, bstart, bstart + t);
                if (nm_d <= budget && nm_d < best_nm) {
                    best_nm = nm_d;
                    best_pos = scan_local;
                    best_flag = scan_rev * 16;
                }
            }
        }
    }
    if (best_nm <= budget) {                            /* L1999-2011 */
        uint32_t mq = 20;
        if (best_nm == 0) mq = 60;
        else if (best_nm <= 2) mq = 40;
        out_rid[dst] = (int32_t)crid;
        out_pos[dst] = (uint32_t)best_pos;
        out_mapq[dst] = mq;
        out_flag[dst] = (int32_t)best_flag;
        out_sl[dst] = 0;
        out_sr[dst] = 0;
        out_nm[dst] = (uint32_t)best_nm;
    }
}

/* ---------------- batch entry (_fm_fire_batch order, L2333-2416) -------- */

/*
 * bases: ASCII [n_seq][max_len] (R1 rows, then R2 rows when paired); the
 * conversion of linear_fastq.mojo:395 is applied to a copy first (R1 with
 * bs_r1, R2 with bs_r2), then pack, seed/extend, rescue.
 * params: seed_len, seed_stride, max_occ, max_diff, max_soft, max_adj,
 * rescue_win.  dbg arrays may be NULL.  score: NULL or [n_seq].
 * n_threads <= 0: all OpenMP threads.  Returns 0 or -1.
 */
int orc_map(const orc_index *ix, const uint8_t *bases, const uint32_t *lens, uint32_t n1,
            int paired, uint32_t max_len, int bs_r1, int bs_r2, const int32_t *params,
            int32_t *out_rid, uint32_t *out_pos, uint32_t *out_mapq, int32_t *out_flag,
            uint32_t *out_sl, uint32_t *out_sr, uint32_t *out_nm, uint64_t *d_uk,
            uint64_t *d_ul, int32_t *d_us, int32_t *d_e, int32_t *d_score,
            orc_counters *counters, int n_threads) {
    orc_params P;
    P.seed_len = params[0];
    P.seed_stride = params[1];
    P.max_occ = params[2];
    P.max_diff = params[3];
    P.max_soft = params[4];
    P.max_adj = params[5];
    P.rescue_win = params[6];
    if (P.seed_stride < 1) {
        snprintf(g_err, sizeof g_err, "seed_stride must be >= 1");
        return -1;
    }
    if (ix->sa_intv & (ix->sa_intv - 1)) {
        snprintf(g_err, sizeof g_err, "sa_intv must be a power of two");
        return -1;
    }
    int64_t n_seq = paired ? 2 * (int64_t)n1 : (int64_t)n1;
    int64_t n_bases = n_seq * (int64_t)max_len;
    uint8_t *codes = (uint8_t *)malloc((size_t)(n_bases > 0 ? n_bases : 1));
    for (int64_t r = 0; r < n_seq; ++r) {
        int mode = (r < (int64_t)n1) ? bs_r1 : bs_r2;
        if (lens[r] > max_len) {
            free(codes);
            snprintf(g_err, sizeof g_err, "read length exceeds max_len");
            return -1;
        }
        for (int64_t j = 0; j < (int64_t)max_len; ++j)
            codes[r * max_len + j] = pack1(cvt(bases[r * max_len + j], mode));
    }
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    orc_counters *tc = NULL;
    if (counters) tc = (orc_counters *)calloc((size_t)nt, sizeof(orc_counters));
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t r = 0; r < n_seq; ++r) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        seed_extend_one(ix, codes, lens, (int64_t)max_len, r, &P, out_rid, out_pos, out_mapq,
                        out_flag, out_sl, out_sr, out_nm, d_uk, d_ul, d_us, d_e,
                        tc ? &tc[tid] : NULL);
    }
    if (paired && P.rescue_win > 0) {
        int64_t n_pairs = n_seq / 2;
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t pi = 0; pi < n_pairs; ++pi) {
            int tid = 0;
#ifdef _OPENMP
            tid = omp_get_thread_num();
#endif
            mate_rescue_one(ix, codes, lens, (int64_t)max_len, n_pairs, pi, &P, out_rid, out_pos,
                            out_mapq, out_flag, out_sl, out_sr, out_nm, tc ? &tc[tid] : NULL);
        }
    }
    if (d_score) {
        for (int64_t r = 0; r < n_seq; ++r) {
            if (out_rid[r] < 0) d_score[r] = 0;
            else
                d_score[r] = (int32_t)((int64_t)lens[r] - (int64_t)out_sl[r] - (int64_t)out_sr[r] -
                                       5 * (int64_t)out_nm[r]);
        }
    }
    if (counters) {
        memset(counters, 0, sizeof *counters);
        for (int t = 0; t < nt; ++t) {
            counters->occ_lines += tc[t].occ_lines;
            counters->lf_lines += tc[t].lf_lines;
            counters->sa_loads += tc[t].sa_loads;
            counters->pac_sectors += tc[t].pac_sectors;
            counters->endpoints += tc[t].endpoints;
            counters->steps += tc[t].steps;
            counters->rows += tc[t].rows;
            counters->extends += tc[t].extends;
            counters->capped += tc[t].capped;
            counters->fallback += tc[t].fallback;
        }
        free(tc);
    }
    free(codes);
    return 0;
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
