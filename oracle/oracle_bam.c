/*
 * ORACLE (test infrastructure only): CPU restatement of the reference's BAM
 * record packing for the FM path, used to check the GPU packer byte for
 * byte.  Follows fq2bam-meth/src/linear_gpu_fm.mojo:
 *   _unclipped5       L371-386      _coord_key   L389-395
 *   _pack_end         L398-405      _nt16        L455-464
 *   _nt16_comp        L467-476      _reg2bin     L479-494
 *   _pack_bam_aln     L497-666      _emit_bam_from_batch  L669-984
 * Inputs are the batch's mapping outputs (R1 rows then R2 rows), the reads'
 * names, original bases and qualities as the FASTQ arena holds them, the
 * rid -> SAM tid table (_rid_to_tid_table, L423-435) and the RG id.
 */
#include <stdint.h>
#include <string.h>

typedef struct {
    uint32_t n1;
    int32_t paired;
    /* mapping outputs [n_seq], R1 rows then R2 rows */
    const int32_t *rid;
    const uint32_t *pos, *mapq;
    const int32_t *flag;
    const uint32_t *sl, *sr, *nm;
    /* FASTQ arena (FastqArena, linear_fastq.mojo:75-95): one byte array and,
     * per record, the offset and length of its name, original bases and
     * qualities; qual_off == NULL means no qualities */
    const uint8_t *arena;
    const uint64_t *name_off, *orig_off, *qual_off;
    const uint32_t *name_len, *orig_len, *qual_len;
    const int32_t *rid_to_tid;
    int32_t n_tid_map;
    const uint8_t *rg;
    uint32_t rg_n;
    uint64_t n_reads;  /* records already in the tile (n_reads) */
    uint64_t n_total;  /* records of flushed tiles (n_total) */
    uint64_t meta_cap; /* tile metadata capacity (meta_cap) */
    uint32_t chunk;    /* chunk index of this batch in the tile (tile_chunks) */
} orc_bam_in;

typedef struct {
    uint64_t *coord, *dhi, *dlo, *rec;
    uint32_t *len, *score, *pair;
} orc_bam_meta;

static int64_t unclipped5(int64_t flag, int64_t pos0, int64_t sl, int64_t sr, int64_t qlen) {
    if ((flag & 4) != 0 || qlen <= 0) return 0;
    if (sl < 0) sl = 0;
    if (sr < 0) sr = 0;
    if (sl + sr >= qlen) sl = sr = 0;
    const int64_t mid = qlen - sl - sr;
    if ((flag & 16) != 0) return pos0 + mid + sl - 1;
    return pos0 - sl;
}

static uint64_t coord_key(int64_t tid, int64_t pos0, int64_t orig) {
    if (tid < 0) return (UINT64_C(4294967295) << 32) | ((uint64_t)orig & UINT64_C(4294967295));
    if (pos0 < 0) pos0 = 0;
    return ((uint64_t)tid << 32) | (uint64_t)pos0;
}

static uint64_t pack_end(int64_t tid, int64_t u5, int64_t strand) {
    const uint64_t t = tid >= 0 ? (uint64_t)(tid + 1) : 0;
    int64_t u = u5 + 1073741824;
    if (u < 0) u = 0;
    return (t << 48) | ((uint64_t)(strand & 1) << 47) | ((uint64_t)u & UINT64_C(140737488355327));
}

static uint8_t nt16(uint8_t b) {
    if (b == 65 || b == 97) return 1;
    if (b == 67 || b == 99) return 2;
    if (b == 71 || b == 103) return 4;
    if (b == 84 || b == 116) return 8;
    return 15;
}

static uint8_t nt16_comp(uint8_t b) {
    if (b == 1) return 8;
    if (b == 8) return 1;
    if (b == 2) return 4;
    if (b == 4) return 2;
    return 15;
}

static int64_t reg2bin(int64_t beg, int64_t end) {
    if (end <= beg) end = beg + 1;
    end -= 1;
    if ((beg >> 14) == (end >> 14)) return 4681 + (beg >> 14);
    if ((beg >> 17) == (end >> 17)) return 585 + (beg >> 17);
    if ((beg >> 20) == (end >> 20)) return 73 + (beg >> 20);
    if ((beg >> 23) == (end >> 23)) return 9 + (beg >> 23);
    if ((beg >> 26) == (end >> 26)) return 1 + (beg >> 26);
    return 0;
}

static void put32(uint8_t *p, uint64_t off, uint32_t v) {
    p[off] = (uint8_t)(v & 255);
    p[off + 1] = (uint8_t)((v >> 8) & 255);
    p[off + 2] = (uint8_t)((v >> 16) & 255);
    p[off + 3] = (uint8_t)((v >> 24) & 255);
}

/* _pack_bam_aln: returns the offset after the record, or -1 on overflow. */
static int64_t pack_aln(uint8_t *p, uint64_t off0, uint64_t cap, const uint8_t *name, int64_t name_len,
                        int64_t flag, int64_t tid, int64_t pos0, int64_t mapq, int64_t sl, int64_t sr,
                        const uint8_t *seq, int64_t qlen, const uint8_t *qual, int64_t qual_len, int64_t ntid,
                        int64_t npos, int64_t tlen, int64_t nm, const uint8_t *rg, int64_t rg_n) {
    const int rev = (flag & 16) != 0;
    if (sl < 0) sl = 0;
    if (sr < 0) sr = 0;
    if (sl + sr >= qlen) sl = sr = 0;
    const int64_t mid = qlen - sl - sr;
    if (rev) {
        const int64_t t = sl;
        sl = sr;
        sr = t;
    }
    int64_t n_cigar = 0;
    if (tid >= 0 && (flag & 4) == 0) n_cigar = (sl > 0) + (mid > 0) + (sr > 0);
    const int64_t l_qname = name_len + 1;
    const int64_t block = 32 + l_qname + 4 * n_cigar + (qlen + 1) / 2 + qlen + (3 + rg_n + 1 + 4);
    if (off0 + 4 + (uint64_t)block > cap) return -1;
    int64_t bin = 4680, tid_w = -1, pos_w = -1;
    if (tid >= 0 && (flag & 4) == 0) {
        tid_w = tid;
        pos_w = pos0;
        int64_t end = pos0 + mid;
        if (end <= pos0) end = pos0 + 1;
        bin = reg2bin(pos0, end);
    }
    if (ntid < 0) ntid = npos = -1;
    if (mapq < 0) mapq = 0;
    if (mapq > 255) mapq = 255;
    put32(p, off0, (uint32_t)block);
    put32(p, off0 + 4, (uint32_t)tid_w);
    put32(p, off0 + 8, (uint32_t)pos_w);
    put32(p, off0 + 12, (uint32_t)((bin << 16) | (mapq << 8) | l_qname));
    put32(p, off0 + 16, (uint32_t)((flag << 16) | n_cigar));
    put32(p, off0 + 20, (uint32_t)qlen);
    put32(p, off0 + 24, (uint32_t)ntid);
    put32(p, off0 + 28, (uint32_t)npos);
    put32(p, off0 + 32, (uint32_t)tlen);
    uint64_t off = off0 + 36;
    memcpy(p + off, name, (size_t)name_len);
    p[off + name_len] = 0;
    off += l_qname;
    if (n_cigar > 0) {
        if (sl > 0) {
            put32(p, off, (uint32_t)((sl << 4) | 4));
            off += 4;
        }
        if (mid > 0) {
            put32(p, off, (uint32_t)(mid << 4));
            off += 4;
        }
        if (sr > 0) {
            put32(p, off, (uint32_t)((sr << 4) | 4));
            off += 4;
        }
    }
    int64_t si = 0;
    for (; si + 1 < qlen; si += 2) {
        const int64_t ia = rev ? qlen - 1 - si : si, ib = rev ? qlen - 2 - si : si + 1;
        uint8_t a = nt16(seq[ia]), b = nt16(seq[ib]);
        if (rev) {
            a = nt16_comp(a);
            b = nt16_comp(b);
        }
        p[off++] = (uint8_t)((a << 4) | b);
    }
    if (si < qlen) {
        uint8_t c = nt16(seq[rev ? 0 : si]);
        if (rev) c = nt16_comp(c);
        p[off++] = (uint8_t)(c << 4);
    }
    for (int64_t i = 0; i < qlen; ++i) {
        if (qual && qual_len == qlen) {
            const uint8_t q = qual[rev ? qlen - 1 - i : i];
            p[off + i] = q >= 33 ? (uint8_t)(q - 33) : 255;
        } else {
            p[off + i] = 255;
        }
    }
    off += qlen;
    p[off] = 82;
    p[off + 1] = 71;
    p[off + 2] = 90;
    off += 3;
    memcpy(p + off, rg, (size_t)rg_n);
    p[off + rg_n] = 0;
    off += rg_n + 1;
    p[off] = 78;
    p[off + 1] = 77;
    p[off + 2] = 67;
    if (nm < 0) nm = 0;
    if (nm > 255) nm = 255;
    p[off + 3] = (uint8_t)nm;
    off += 4;
    return (int64_t)off;
}

/* _pack_bam_aln alone, into p[0..cap): bytes written or -1. */
int64_t orc_pack_aln(uint8_t *p, uint64_t cap, const uint8_t *name, int64_t name_len, int64_t flag, int64_t tid,
                     int64_t pos0, int64_t mapq, int64_t sl, int64_t sr, const uint8_t *seq, int64_t qlen,
                     const uint8_t *qual, int64_t qual_len, int64_t ntid, int64_t npos, int64_t tlen, int64_t nm,
                     const uint8_t *rg, int64_t rg_n) {
    return pack_aln(p, 0, cap, name, name_len, flag, tid, pos0, mapq, sl, sr, seq, qlen, qual, qual_len, ntid, npos,
                    tlen, nm, rg, rg_n);
}

/* _emit_bam_from_batch (L669-984) for one batch.  Returns the bytes written
 * to `bam`, -1 when a record does not fit `cap` ("BAM batch buffer
 * overflow", L547-549) or -2 when the tile metadata is full ("FM sort cap
 * exceeded", L772-775 / L875-878).  Metadata arrays are the tile's, indexed
 * by the record's tile position n_reads + j like h_coord[n_reads]. */
int64_t orc_emit_bam(const orc_bam_in *in, uint8_t *bam, uint64_t cap, orc_bam_meta *m, uint64_t *n_mapped) {
    const uint32_t n1 = in->n1;
    uint64_t off = 0, nr = in->n_reads, mapped = 0;
    const uint64_t chunk_hi = (uint64_t)in->chunk << 32;
    for (uint32_t pj = 0; pj < n1; ++pj) {
        const int64_t rid1 = in->rid[pj];
        const int64_t pos1 = in->pos[pj], mq1 = in->mapq[pj], sl1 = in->sl[pj], sr1 = in->sr[pj], nm1 = in->nm[pj];
        int64_t fl1 = (int64_t)in->flag[pj] | 1 | 64;
        int64_t tid1 = -1;
        if (rid1 >= 0 && rid1 < in->n_tid_map) tid1 = in->rid_to_tid[rid1];
        else fl1 |= 4;
        const int64_t qlen1 = in->orig_len[pj];
        const uint8_t *s1 = in->arena + in->orig_off[pj];
        const uint8_t *q1 = in->qual_off ? in->arena + in->qual_off[pj] : NULL;
        const int64_t q1n = in->qual_len ? in->qual_len[pj] : 0;
        const uint8_t *name1 = in->arena + in->name_off[pj];
        if (!in->paired) {
            if (nr >= in->meta_cap) return -2;
            const uint64_t start = off;
            const int64_t o = pack_aln(bam, off, cap, name1, in->name_len[pj], fl1, tid1, pos1, mq1, sl1, sr1, s1,
                                       qlen1, q1, q1n, -1, -1, 0, nm1, in->rg, in->rg_n);
            if (o < 0) return -1;
            off = (uint64_t)o;
            m->coord[nr] = coord_key(tid1, pos1, (int64_t)nr);
            if (tid1 >= 0) {
                m->dhi[nr] = pack_end(tid1, unclipped5(fl1, pos1, sl1, sr1, qlen1), (fl1 >> 4) & 1);
                m->dlo[nr] = 0;
            } else {
                m->dhi[nr] = ~UINT64_C(0);
                m->dlo[nr] = nr;
            }
            m->rec[nr] = chunk_hi | start;
            m->len[nr] = (uint32_t)(off - start);
            const int64_t nmc = nm1 < 0 ? 0 : (nm1 > 255 ? 255 : nm1);
            m->score[nr] = (uint32_t)((mq1 << 8) | (255 - nmc));
            m->pair[nr] = (uint32_t)(in->n_total + nr);
            mapped += tid1 >= 0;
            ++nr;
            continue;
        }
        const uint64_t r2 = (uint64_t)n1 + pj;
        const int64_t rid2 = in->rid[r2];
        const int64_t pos2 = in->pos[r2], mq2 = in->mapq[r2], sl2 = in->sl[r2], sr2 = in->sr[r2], nm2 = in->nm[r2];
        int64_t fl2 = (int64_t)in->flag[r2] | 1 | 128;
        int64_t tid2 = -1;
        if (rid2 >= 0 && rid2 < in->n_tid_map) tid2 = in->rid_to_tid[rid2];
        else fl2 |= 4;
        if (tid1 < 0) fl2 |= 8;
        if (tid2 < 0) fl1 |= 8;
        int64_t ntid1 = -1, npos1 = -1, ntid2 = -1, npos2 = -1, tlen1 = 0, tlen2 = 0;
        const int64_t qlen2 = in->orig_len[r2];
        if (tid1 >= 0 && tid2 >= 0 && tid1 == tid2) {
            fl1 |= 2;
            fl2 |= 2;
            ntid1 = tid1;
            ntid2 = tid2;
            npos1 = pos2;
            npos2 = pos1;
            int64_t tl = pos2 - pos1;
            if (tl < 0) tl = -tl;
            tl += qlen2;
            tlen1 = pos1 <= pos2 ? tl : -tl;
            tlen2 = -tlen1;
        } else {
            if (tid1 >= 0) {
                ntid2 = tid1;
                npos2 = pos1;
            }
            if (tid2 >= 0) {
                ntid1 = tid2;
                npos1 = pos2;
            }
        }
        if (nr + 1 >= in->meta_cap) return -2;
        const uint8_t *q2 = in->qual_off ? in->arena + in->qual_off[r2] : NULL;
        const int64_t q2n = in->qual_len ? in->qual_len[r2] : 0;
        const uint64_t start1 = off;
        int64_t o = pack_aln(bam, off, cap, name1, in->name_len[pj], fl1, tid1, pos1, mq1, sl1, sr1, s1, qlen1, q1,
                             q1n, ntid1, npos1, tlen1, nm1, in->rg, in->rg_n);
        if (o < 0) return -1;
        off = (uint64_t)o;
        const uint64_t start2 = off;
        o = pack_aln(bam, off, cap, in->arena + in->name_off[r2], in->name_len[r2], fl2, tid2, pos2, mq2, sl2, sr2,
                     in->arena + in->orig_off[r2], qlen2, q2, q2n, ntid2, npos2, tlen2, nm2, in->rg, in->rg_n);
        if (o < 0) return -1;
        off = (uint64_t)o;
        const uint64_t i1 = nr, i2 = nr + 1;
        const uint32_t pid = (uint32_t)((in->n_total + nr) / 2);
        int64_t nms = nm1 + nm2;
        if (nms < 0) nms = 0;
        if (nms > 255) nms = 255;
        const uint32_t pscore = (uint32_t)(((mq1 + mq2) << 8) | (255 - nms));
        uint64_t dhi = ~UINT64_C(0), dlo = i1;
        if (tid1 >= 0 || tid2 >= 0) {
            const uint64_t e1 = pack_end(tid1, unclipped5(fl1, pos1, sl1, sr1, qlen1), (fl1 >> 4) & 1);
            const uint64_t e2 = pack_end(tid2, unclipped5(fl2, pos2, sl2, sr2, qlen2), (fl2 >> 4) & 1);
            if (tid1 < 0) {
                dhi = e2;
                dlo = 0;
            } else if (tid2 < 0) {
                dhi = e1;
                dlo = 0;
            } else if (e1 <= e2) {
                dhi = e1;
                dlo = e2;
            } else {
                dhi = e2;
                dlo = e1;
            }
        }
        m->coord[i1] = coord_key(tid1, pos1, (int64_t)i1);
        m->coord[i2] = coord_key(tid2, pos2, (int64_t)i2);
        m->dhi[i1] = m->dhi[i2] = dhi;
        m->dlo[i1] = m->dlo[i2] = dlo;
        m->rec[i1] = chunk_hi | start1;
        m->rec[i2] = chunk_hi | start2;
        m->len[i1] = (uint32_t)(start2 - start1);
        m->len[i2] = (uint32_t)(off - start2);
        m->score[i1] = m->score[i2] = pscore;
        m->pair[i1] = m->pair[i2] = pid;
        mapped += (tid1 >= 0) + (tid2 >= 0);
        nr += 2;
    }
    if (n_mapped) *n_mapped = mapped;
    return (int64_t)off;
}
