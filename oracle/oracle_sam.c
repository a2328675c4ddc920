/*
 * ORACLE (test infrastructure only): CPU restatement of the SAM side of the
 * reference's FM path, used to check the device FASTQ split (pair-reader
 * rules) and the device SAM emitter.
 *
 * FASTQ, as the SAM path reads it (fq2bam-meth/python/fastq_batch.py):
 *   _qname                L18-28   drop every trailing '\r' / '\n', drop a
 *                                  leading '@', cut at the first ' ', then
 *                                  at the first '/'
 *   FastqPairReader._one  L250-263 four readline() calls per record; each
 *                                  line loses every trailing '\r' / '\n';
 *                                  only an empty header read ends the
 *                                  stream, later lines may be missing
 *                                  (they read as empty)
 *   read_batch            L265-317 up to n records
 * over one buffer of uncompressed FASTQ bytes.  When the buffer is not the
 * end of the stream (at_eof == 0) only records whose four lines all end in
 * '\n' are taken, and `consumed` is where the next buffer must start.
 *
 * SAM records (fq2bam-meth/src/linear_gpu_fm.mojo):
 *   _hit_from_fm          L987-1025  unmapped when rid < 0 or no base is
 *                                    left between the clips; CIGAR
 *                                    [slS]mM[srS]; SEQ is the original bases,
 *                                    reverse-complemented on flag 16
 *   SAM batch loop        L2787-2836 QUAL is the record's own; the mapped
 *                                    count is the records whose contig is
 *                                    not "*"
 *   _sam_with_rg_fm       L80-81     "\tRG:Z:" + the read group id
 * fq2bam-meth/src/linear_extend.mojo:
 *   pair_hits             L263-294   flags 1|64 / 1|128; same contig: 2,
 *                                    RNEXT "=", PNEXT the mate's POS, TLEN
 *                                    |pos2 - pos1| + len(SEQ2) (negated on
 *                                    R2); otherwise 8 on the mate of an
 *                                    unmapped record and RNEXT / PNEXT of a
 *                                    mapped mate
 *   hit_to_sam_line       L297-320   eleven tab-separated fields
 * methylgrapher/src/utility.mojo reverse_complement L28-49 (byte-wise, any
 * byte other than A/C/G/T becomes N), and linear_gpu_locate.mojo
 * _canonical_contig L156-162 (the caller passes the canonical names).
 *
 * Text conversions of the reference's Python/Mojo boundary
 * (_py_batch_to_recs, linear_gpu_fm.mojo:135-164): a name is decoded as
 * ASCII with replacement, so each byte >= 0x80 is written as U+FFFD
 * (EF BF BD); SEQ and QUAL are decoded as strict UTF-8, so a batch holding
 * an invalid sequence fails.
 */
#include <stdint.h>
#include <string.h>

/* readline(): the next line of buf[*pos, n) with its '\n'.  Returns 1 and
 * the content span without its trailing '\r' / '\n' run; 0 at the end of
 * the data, or for an unterminated line when !at_eof (it may continue in
 * the next buffer). */
static int pr_line(const uint8_t *buf, uint64_t n, int at_eof, uint64_t *pos, uint64_t *off, uint64_t *len) {
    const uint64_t s = *pos;
    if (s >= n) return 0;
    const uint8_t *nl = memchr(buf + s, '\n', n - s);
    uint64_t e;
    if (nl) {
        e = (uint64_t)(nl - buf);
        *pos = e + 1;
    } else {
        if (!at_eof) return 0;
        e = n;
        *pos = n;
    }
    while (e > s && buf[e - 1] == '\r') --e;
    *off = s;
    *len = e - s;
    return 1;
}

int64_t orc_fastq_parse_pr(const uint8_t *buf, uint64_t n, int at_eof, uint64_t max_records, uint64_t base,
                           uint64_t *name_off, uint32_t *name_len, uint64_t *seq_off, uint32_t *seq_len,
                           uint64_t *qual_off, uint32_t *qual_len, uint64_t *consumed, uint32_t *max_len) {
    uint64_t pos = 0, r = 0;
    uint32_t mx = 0;
    *consumed = 0;
    while (r < max_records) {
        uint64_t p = pos, off[4], len[4];
        int k = 0;
        for (; k < 4; ++k)
            if (!pr_line(buf, n, at_eof, &p, &off[k], &len[k])) break;
        if (k == 0) break;         /* no header line: end of the data */
        if (k < 4 && !at_eof) break;  /* the record may continue in the next buffer */
        for (; k < 4; ++k) {       /* lines past the end read as empty */
            off[k] = n;
            len[k] = 0;
        }
        uint64_t ns = off[0], ne = off[0] + len[0];
        if (ne > ns && buf[ns] == '@') ++ns;
        for (uint64_t i = ns; i < ne; ++i)
            if (buf[i] == ' ') {
                ne = i;
                break;
            }
        for (uint64_t i = ns; i < ne; ++i)
            if (buf[i] == '/') {
                ne = i;
                break;
            }
        name_off[r] = base + ns;
        name_len[r] = (uint32_t)(ne - ns);
        seq_off[r] = base + off[1];
        seq_len[r] = (uint32_t)len[1];
        qual_off[r] = base + off[3];
        qual_len[r] = (uint32_t)len[3];
        if (len[1] > mx) mx = (uint32_t)len[1];
        pos = p;
        ++r;
    }
    *consumed = pos;
    *max_len = mx;
    return (int64_t)r;
}

/* Strict UTF-8 (RFC 3629): no overlong forms, no surrogates, nothing above
 * U+10FFFF. */
static int utf8_ok(const uint8_t *p, uint64_t n) {
    uint64_t i = 0;
    while (i < n) {
        const uint8_t c = p[i];
        if (c < 0x80) {
            ++i;
            continue;
        }
        int k;
        uint8_t lo = 0x80, hi = 0xbf;
        if (c >= 0xc2 && c <= 0xdf) k = 1;
        else if (c >= 0xe0 && c <= 0xef) {
            k = 2;
            if (c == 0xe0) lo = 0xa0;
            if (c == 0xed) hi = 0x9f;
        } else if (c >= 0xf0 && c <= 0xf4) {
            k = 3;
            if (c == 0xf0) lo = 0x90;
            if (c == 0xf4) hi = 0x8f;
        } else return 0;
        if (n - i - 1 < (uint64_t)k) return 0;
        if (p[i + 1] < lo || p[i + 1] > hi) return 0;
        for (int j = 2; j <= k; ++j)
            if (p[i + j] < 0x80 || p[i + j] > 0xbf) return 0;
        i += (uint64_t)k + 1;
    }
    return 1;
}

typedef struct {
    int star;          /* contig "*": unmapped, or a canonical name "*" */
    int mapped;        /* placed by _hit_from_fm */
    int64_t flag, pos1, mapq, pnext, tlen;
    int64_t sl, m, sr;
    uint32_t canon;    /* canonical contig id */
    const uint8_t *contig;
    uint32_t contig_len;
    const uint8_t *rnext;
    uint32_t rnext_len;
} SamHit;

static const uint8_t STAR[1] = {'*'};
static const uint8_t EQ[1] = {'='};

static void hit_of(SamHit *h, int32_t rid, uint32_t pos, uint32_t mapq, int32_t flag, uint32_t sl, uint32_t sr,
                   uint32_t qlen, const uint8_t *names, const uint64_t *noff, const uint32_t *nlen,
                   const uint32_t *canon) {
    memset(h, 0, sizeof(*h));
    const int64_t m = (int64_t)qlen - (int64_t)sl - (int64_t)sr;
    h->rnext = STAR;
    h->rnext_len = 1;
    if (rid < 0 || m < 1) {
        h->star = 1;
        h->flag = 4;
        h->contig = STAR;
        h->contig_len = 1;
        return;
    }
    h->mapped = 1;
    h->flag = flag;
    h->pos1 = (int64_t)pos + 1;
    h->mapq = mapq;
    h->sl = sl;
    h->sr = sr;
    h->m = m;
    h->contig = names + noff[rid];
    h->contig_len = nlen[rid];
    h->canon = canon[rid];
    h->star = h->contig_len == 1 && h->contig[0] == '*';
}

static uint64_t put_int(uint8_t *o, int64_t v) {
    uint8_t t[24];
    int k = 0;
    uint64_t u = v < 0 ? (uint64_t)0 - (uint64_t)v : (uint64_t)v;
    do {
        t[k++] = (uint8_t)('0' + u % 10);
        u /= 10;
    } while (u);
    uint64_t w = 0;
    if (v < 0) o[w++] = '-';
    while (k) o[w++] = t[--k];
    return w;
}

/* One SAM line into o (NULL: only its length). */
static uint64_t sam_line(uint8_t *o, const SamHit *h, const uint8_t *data, uint64_t name_off, uint32_t name_len,
                         uint64_t seq_off, uint32_t seq_len, uint64_t qual_off, uint32_t qual_len,
                         const uint8_t *rg, uint32_t rg_len) {
    uint8_t tmp[160];
    uint64_t w = 0;
#define PUT(ptr, k)                                  \
    do {                                             \
        if (o) memcpy(o + w, (ptr), (k));            \
        w += (k);                                    \
    } while (0)
#define PUTC(c)                  \
    do {                         \
        if (o) o[w] = (uint8_t)(c); \
        ++w;                     \
    } while (0)
#define PUTI(v)                              \
    do {                                     \
        const uint64_t k_ = put_int(tmp, (v)); \
        PUT(tmp, k_);                        \
    } while (0)
    for (uint32_t i = 0; i < name_len; ++i) {
        const uint8_t c = data[name_off + i];
        if (c < 0x80) PUTC(c);
        else {
            PUTC(0xef);
            PUTC(0xbf);
            PUTC(0xbd);
        }
    }
    PUTC('\t');
    PUTI(h->flag);
    PUTC('\t');
    PUT(h->contig, h->contig_len);
    PUTC('\t');
    PUTI(h->pos1);
    PUTC('\t');
    PUTI(h->mapq);
    PUTC('\t');
    if (!h->mapped) PUTC('*');
    else {
        if (h->sl > 0) {
            PUTI(h->sl);
            PUTC('S');
        }
        PUTI(h->m);
        PUTC('M');
        if (h->sr > 0) {
            PUTI(h->sr);
            PUTC('S');
        }
    }
    PUTC('\t');
    PUT(h->rnext, h->rnext_len);
    PUTC('\t');
    PUTI(h->pnext);
    PUTC('\t');
    PUTI(h->tlen);
    PUTC('\t');
    const uint8_t *s = data + seq_off;
    if (h->mapped && (h->flag & 16)) {
        for (uint32_t i = 0; i < seq_len; ++i) {
            const uint8_t c = s[seq_len - 1 - i];
            PUTC(c == 'A' ? 'T' : c == 'T' ? 'A' : c == 'C' ? 'G' : c == 'G' ? 'C' : 'N');
        }
    } else PUT(s, seq_len);
    PUTC('\t');
    PUT(data + qual_off, qual_len);
    PUT("\tRG:Z:", 6);
    PUT(rg, rg_len);
    PUTC('\n');
#undef PUT
#undef PUTC
#undef PUTI
    return w;
}

/* SAM lines of one mapped batch (R1 rows then R2 rows in the hit arrays and
 * the arena columns; lines R1, R2 per pair).  Contig table per rid: the
 * canonical name (names + noff[rid], nlen[rid]) and canonical id.  Returns
 * the bytes written, or (checked in this order) -3 (rid outside the contig
 * table), -2 (SEQ / QUAL not valid UTF-8), -1 (cap too small: nothing
 * written). */
int64_t orc_emit_sam(const int32_t *rid, const uint32_t *pos, const uint32_t *mapq, const int32_t *flag,
                     const uint32_t *sl, const uint32_t *sr, uint64_t n1, int paired, const uint8_t *data,
                     const uint64_t *name_off, const uint32_t *name_len, const uint64_t *seq_off,
                     const uint32_t *seq_len, const uint64_t *qual_off, const uint32_t *qual_len,
                     const uint8_t *names, const uint64_t *noff, const uint32_t *nlen, const uint32_t *canon,
                     uint32_t n_contigs, const uint8_t *rg, uint32_t rg_len, uint8_t *out, uint64_t cap,
                     uint64_t *n_mapped) {
    const uint64_t n_seq = paired ? 2 * n1 : n1;
    for (uint64_t r = 0; r < n_seq; ++r)
        if (rid[r] >= 0 && (uint32_t)rid[r] >= n_contigs) return -3;
    for (uint64_t r = 0; r < n_seq; ++r)
        if (!utf8_ok(data + seq_off[r], seq_len[r]) || !utf8_ok(data + qual_off[r], qual_len[r])) return -2;
    uint64_t mapped = 0;
    for (int pass = 0; pass < 2; ++pass) {
        uint8_t *o = pass ? out : NULL;
        uint64_t w = 0;
        mapped = 0;
        for (uint64_t i = 0; i < n1; ++i) {
            SamHit h[2];
            const int k = paired ? 2 : 1;
            for (int m = 0; m < k; ++m) {
                const uint64_t r = i + (uint64_t)m * n1;
                hit_of(&h[m], rid[r], pos[r], mapq[r], flag[r], sl[r], sr[r], seq_len[r], names, noff, nlen, canon);
            }
            if (paired) {
                SamHit *a = &h[0], *b = &h[1];
                a->flag |= 1 | 64;
                b->flag |= 1 | 128;
                if (!a->star && !b->star && a->canon == b->canon) {
                    a->flag |= 2;
                    b->flag |= 2;
                    a->rnext = b->rnext = EQ;
                    a->pnext = b->pos1;
                    b->pnext = a->pos1;
                    int64_t t = b->pos1 - a->pos1;
                    if (t < 0) t = -t;
                    t += seq_len[i + n1];
                    a->tlen = t;
                    b->tlen = -t;
                } else {
                    if (a->star) b->flag |= 8;
                    if (b->star) a->flag |= 8;
                    if (!a->star) {
                        b->rnext = a->contig;
                        b->rnext_len = a->contig_len;
                        b->pnext = a->pos1;
                    }
                    if (!b->star) {
                        a->rnext = b->contig;
                        a->rnext_len = b->contig_len;
                        a->pnext = b->pos1;
                    }
                }
            }
            for (int m = 0; m < k; ++m) {
                const uint64_t r = i + (uint64_t)m * n1;
                mapped += !h[m].star;
                w += sam_line(o ? o + w : NULL, &h[m], data, name_off[r], name_len[r], seq_off[r], seq_len[r],
                              qual_off[r], qual_len[r], rg, rg_len);
            }
        }
        if (!pass && w > cap) return -1;
        if (pass) {
            *n_mapped = mapped;
            return (int64_t)w;
        }
    }
    return 0;
}
