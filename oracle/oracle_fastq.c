/*
 * ORACLE (test infrastructure only): CPU restatement of the reference's
 * FASTQ record split, used to check the device parser.  Follows
 * fq2bam-meth/src/linear_fastq.mojo:
 *   _pipe_line    L233-280  a line ends at '\n', one trailing '\r' is
 *                           dropped; at the end of the stream an
 *                           unterminated rest is a line when it is not empty
 *                           after that strip
 *   _qname_span   L308-325  drop a leading '@', cut at the first ' ' or '/'
 *   _store_rec    L365-417  four lines per record; a record cut short raises
 *                           "truncated FASTQ (missing SEQ | + | QUAL)"
 *   fq_read_batch L437-451  up to n records
 * over one buffer of uncompressed FASTQ bytes.  When the buffer is not the
 * end of the stream (at_eof == 0) only records whose four lines all end in
 * '\n' are taken, and `consumed` is where the next buffer must start.
 */
#include <stdint.h>
#include <string.h>

/* Next line of buf[*pos, n): sets off / len, advances *pos.  Returns 1 for
 * a line, 0 when there is none (end of data, or an incomplete line when
 * !at_eof). */
static int next_line(const uint8_t *buf, uint64_t n, int at_eof, uint64_t *pos, uint64_t *off, uint64_t *len) {
    const uint64_t s = *pos;
    if (s >= n) return 0;
    const uint8_t *nl = memchr(buf + s, '\n', n - s);
    if (nl) {
        uint64_t e = (uint64_t)(nl - buf);
        *pos = e + 1;
        if (e > s && buf[e - 1] == '\r') --e;
        *off = s;
        *len = e - s;
        return 1;
    }
    if (!at_eof) return 0;
    uint64_t e = n;
    if (e > s && buf[e - 1] == '\r') --e;
    *pos = n;
    *off = s;
    *len = e - s;
    return e > s;
}

/* Returns the records parsed (<= max_records), or -1 / -2 / -3 for a
 * record missing its SEQ / + / QUAL line at the end of the stream.
 * Offsets are relative to buf plus `base`. */
int64_t orc_fastq_parse(const uint8_t *buf, uint64_t n, int at_eof, uint64_t max_records, uint64_t base,
                        uint64_t *name_off, uint32_t *name_len, uint64_t *seq_off, uint32_t *seq_len,
                        uint64_t *qual_off, uint32_t *qual_len, uint64_t *consumed, uint32_t *max_len) {
    uint64_t pos = 0, r = 0;
    uint32_t ml = 0;
    *consumed = 0;
    while (r < max_records) {
        uint64_t lo[4], ll[4];
        uint64_t p = pos;
        if (!next_line(buf, n, at_eof, &p, &lo[0], &ll[0])) break; /* end of records */
        int got = 1;
        while (got < 4 && next_line(buf, n, at_eof, &p, &lo[got], &ll[got])) ++got;
        if (got < 4) {
            if (at_eof) return -(int64_t)got; /* 1: missing SEQ, 2: missing +, 3: missing QUAL */
            break;                            /* wait for more bytes */
        }
        /* qname span of the header */
        uint64_t s = 0, e = ll[0];
        if (e > 0 && buf[lo[0]] == '@') s = 1;
        for (uint64_t i = s; i < e; ++i) {
            const uint8_t c = buf[lo[0] + i];
            if (c == ' ' || c == '/') {
                e = i;
                break;
            }
        }
        name_off[r] = base + lo[0] + s;
        name_len[r] = (uint32_t)(e > s ? e - s : 0);
        seq_off[r] = base + lo[1];
        seq_len[r] = (uint32_t)ll[1];
        qual_off[r] = base + lo[3];
        qual_len[r] = (uint32_t)ll[3];
        if (ll[1] > ml) ml = (uint32_t)ll[1];
        pos = p;
        ++r;
    }
    *consumed = pos;
    *max_len = ml;
    return (int64_t)r;
}
