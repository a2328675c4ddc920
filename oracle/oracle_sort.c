/*
 * ORACLE (test infrastructure only): CPU restatement of the reference's
 * coordinate sort + duplicate marking of the FM BAM path and of the sorted
 * record gather, used to check the GPU implementation bit for bit.
 *   gpu_sort_markdup       fq2bam-meth/src/linear_gpu_sort.mojo:24-560
 *     - LSD radix sort, 8-bit digits, 64-bit keys, u32 record indices
 *       (radix8, L149-245), on tiles of `tile` records (_sort_tile_size,
 *       L15-21; tile = n is the default);
 *     - duplicate order: radix on dlo, then dhi permuted into that order
 *       and radix on dhi (L311-360); tiles merged by (dhi, dlo, index)
 *       (L372-408);
 *     - Picard-style marking over that order (L409-466);
 *     - coordinate order: radix on coord, tiles merged by (coord, index)
 *       (L469-525).
 *   _gather_perm_to_writer fq2bam-meth/src/linear_gpu_fm.mojo:177-225 with
 *     _or_dup_flag L408-420: records concatenated in perm order, flag 0x400
 *     set on duplicates.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* radix8: stable LSD sort of keys[0..n) carrying idx, 8 passes of 8 bits.
 * keys and idx hold the result; tk / ti are scratch of n entries. */
static void radix8(uint64_t *keys, uint32_t *idx, uint64_t *tk, uint32_t *ti, uint64_t n) {
    uint64_t count[256];
    for (int p = 0; p < 8; ++p) {
        const int shift = 8 * p;
        uint64_t *ki = (p & 1) ? tk : keys, *ko = (p & 1) ? keys : tk;
        uint32_t *ii = (p & 1) ? ti : idx, *io = (p & 1) ? idx : ti;
        memset(count, 0, sizeof count);
        for (uint64_t i = 0; i < n; ++i) ++count[(ki[i] >> shift) & 255];
        uint64_t run = 0;
        for (int d = 0; d < 256; ++d) {
            const uint64_t c = count[d];
            count[d] = run;
            run += c;
        }
        for (uint64_t i = 0; i < n; ++i) {
            const uint64_t pos = count[(ki[i] >> shift) & 255]++;
            ko[pos] = ki[i];
            io[pos] = ii[i];
        }
    }
    /* eight passes end in keys / idx */
}

/* Sorts every tile; run_orig[b + i] = b + (tile-local sorted index). For
 * the duplicate order the tile is sorted on lo first, then on hi permuted
 * into that order. */
static void sort_tiles(uint64_t n, uint64_t tile, const uint64_t *lo, const uint64_t *hi, uint32_t *run_orig,
                       uint64_t *k, uint32_t *ix, uint64_t *tk, uint32_t *ti) {
    for (uint64_t b = 0; b < n; b += tile) {
        const uint64_t nt = b + tile > n ? n - b : tile;
        for (uint64_t i = 0; i < nt; ++i) {
            k[i] = lo[b + i];
            ix[i] = (uint32_t)i;
        }
        radix8(k, ix, tk, ti, nt);
        if (hi) {
            for (uint64_t i = 0; i < nt; ++i) k[i] = hi[b + ix[i]];
            radix8(k, ix, tk, ti, nt);
        }
        for (uint64_t i = 0; i < nt; ++i) run_orig[b + i] = (uint32_t)(b + ix[i]);
    }
}

/* k-way merge of the sorted tiles by (hi, lo, index) (hi == NULL: by
 * (lo, index)), into out[0..n). */
static void merge_tiles(uint64_t n, uint64_t tile, const uint64_t *lo, const uint64_t *hi, const uint32_t *run_orig,
                        uint32_t *out) {
    const uint64_t n_tiles = (n + tile - 1) / tile;
    uint64_t *head = calloc(n_tiles, sizeof *head);
    for (uint64_t o = 0; o < n; ++o) {
        int64_t best = -1;
        for (uint64_t t = 0; t < n_tiles; ++t) {
            const uint64_t len = (t + 1) * tile > n ? n - t * tile : tile;
            if (head[t] >= len) continue;
            if (best < 0) {
                best = (int64_t)t;
                continue;
            }
            const uint32_t a = run_orig[t * tile + head[t]], c = run_orig[(uint64_t)best * tile + head[best]];
            int take;
            if (hi) {
                take = hi[a] < hi[c] || (hi[a] == hi[c] && (lo[a] < lo[c] || (lo[a] == lo[c] && a < c)));
            } else {
                take = lo[a] < lo[c] || (lo[a] == lo[c] && a < c);
            }
            if (take) best = (int64_t)t;
        }
        out[o] = run_orig[(uint64_t)best * tile + head[best]];
        ++head[best];
    }
    free(head);
}

/* gpu_sort_markdup: is_dup in record order, perm = coordinate order,
 * dup_perm (optional) = duplicate-key order (identity without marking).
 * Returns the number of records marked, or -1 on allocation failure. */
int64_t orc_sort_markdup(uint64_t n, uint64_t tile, const uint64_t *coord, const uint64_t *dhi, const uint64_t *dlo,
                         const uint32_t *score, const uint32_t *pair, uint32_t *is_dup, uint32_t *perm,
                         int do_markdup, uint32_t *dup_perm) {
    if (n == 0) return 0;
    if (tile < 1 || tile >= n) tile = n;
    uint64_t *k = malloc(tile * sizeof *k), *tk = malloc(tile * sizeof *tk);
    uint32_t *ix = malloc(tile * sizeof *ix), *ti = malloc(tile * sizeof *ti);
    uint32_t *run_orig = malloc(n * sizeof *run_orig), *merged = malloc(n * sizeof *merged);
    if (!k || !tk || !ix || !ti || !run_orig || !merged) {
        free(k);
        free(tk);
        free(ix);
        free(ti);
        free(run_orig);
        free(merged);
        return -1;
    }
    int64_t marked = 0;
    memset(is_dup, 0, n * sizeof *is_dup);
    if (do_markdup) {
        sort_tiles(n, tile, dlo, dhi, run_orig, k, ix, tk, ti);
        merge_tiles(n, tile, dlo, dhi, run_orig, merged);
        const uint64_t sentinel = ~UINT64_C(0);
        uint64_t gi = 0;
        while (gi < n) {
            const uint32_t o0 = merged[gi];
            if (dhi[o0] == sentinel) {
                is_dup[o0] = 0;
                ++gi;
                continue;
            }
            uint64_t gj = gi + 1;
            while (gj < n && dhi[merged[gj]] == dhi[o0] && dlo[merged[gj]] == dlo[o0]) ++gj;
            uint32_t best_pair = pair[o0], best_score = score[o0];
            for (uint64_t g = gi; g < gj; ++g) {
                const uint32_t sc = score[merged[g]], pid = pair[merged[g]];
                if (sc > best_score || (sc == best_score && pid < best_pair)) {
                    best_score = sc;
                    best_pair = pid;
                }
            }
            for (uint64_t g = gi; g < gj; ++g) {
                const uint32_t d = pair[merged[g]] != best_pair;
                is_dup[merged[g]] = d;
                marked += d;
            }
            gi = gj;
        }
        if (dup_perm) memcpy(dup_perm, merged, n * sizeof *merged);
    } else if (dup_perm) {
        for (uint64_t i = 0; i < n; ++i) dup_perm[i] = (uint32_t)i;
    }
    sort_tiles(n, tile, coord, NULL, run_orig, k, ix, tk, ti);
    merge_tiles(n, tile, coord, NULL, run_orig, perm);
    free(k);
    free(tk);
    free(ix);
    free(ti);
    free(run_orig);
    free(merged);
    return marked;
}

/* _gather_perm_to_writer: the records of a tile in perm order, duplicates
 * flagged.  chunks[c] is the base of BAM chunk c; rec[i] = c << 32 | offset.
 * Returns the bytes written to out, or -1 when they exceed cap. */
int64_t orc_gather_sorted(uint64_t n, const uint8_t *const *chunks, const uint32_t *perm, const uint64_t *rec,
                          const uint32_t *len, const uint32_t *is_dup, int apply_dup, uint8_t *out, uint64_t cap) {
    uint64_t off = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const uint32_t o = perm[i];
        const uint64_t r = rec[o];
        const uint32_t rl = len[o];
        if (off + rl > cap) return -1;
        memcpy(out + off, chunks[r >> 32] + (r & UINT64_C(0xffffffff)), rl);
        if (apply_dup && is_dup[o] != 0) out[off + 19] |= 4; /* flag |= 1024 */
        off += rl;
    }
    return (int64_t)off;
}
