"""Seeded mapped batches for the SAM text tests, and the expected lines from
the per-record restatement of the reference's rules.

A batch is what the SAM loop of map_fastq_fm_gpu formats (fq2bam-meth/src/
linear_gpu_fm.mojo:2787-2836): the mapping outputs, the FASTQ arena (name,
original bases, qualities of every record, laid out in a shuffled order so
offsets are arbitrary) and the contig names.  Values range past what the
mapper emits (any flag bits, clips beyond the read, positions up to
2^32 - 1, MAPQ up to 2^32 - 1) and the text past plain ASCII (name bytes
>= 0x80, valid multi-byte UTF-8 in SEQ and QUAL, empty fields).
"""
from __future__ import annotations

import numpy as np

from mojoalign_b200.bam import BatchArena
from mojoalign_b200.linear_fm import hit_from_fm, hit_to_sam_line, pair_hits

# bwa-meth contigs (r/f pairs), a duplicate canonical name under another rid,
# a one-byte name that keeps its 'f', and a canonical name "*"
CONTIGS = ["rchr1", "fchr1", "rchr2", "fchr2", "chrM", "f", "r*", "fchr1", "rchrUn_KI270302v1"]

_UTF8 = [b"\xc3\xa9", b"\xe2\x82\xac", b"\xf0\x9f\x98\x80"]


def _bytes(rng, alphabet: bytes, n: int) -> bytes:
    return np.frombuffer(alphabet, np.uint8)[rng.integers(0, len(alphabet), size=n)].tobytes()


def random_sam_batch(seed: int, n1: int, paired: bool, *, mapped_frac: float = 0.8, n_contigs: int = len(CONTIGS),
                     odd_text: float = 0.04):
    rng = np.random.default_rng(seed)
    n_seq = n1 * (2 if paired else 1)
    recs = []
    for _ in range(n_seq):
        q = int(rng.choice([0, 1, 2, 36, 75, 100, 150, 151, 250]))
        seq = _bytes(rng, b"ACGTNacgtn" if rng.random() < 0.1 else b"ACGT", q)
        qual = _bytes(rng, bytes(range(33, 75)), q)
        if rng.random() < odd_text:  # a multi-byte character in SEQ / QUAL
            ch = _UTF8[int(rng.integers(0, 3))]
            k = int(rng.integers(0, len(seq) + 1))
            seq = seq[:k] + ch + seq[k:]
        if rng.random() < odd_text:
            qual = qual + _UTF8[int(rng.integers(0, 3))]
        if rng.random() < 0.02:
            qual = b""
        name = _bytes(rng, b"ABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789:_-", int(rng.choice([0, 1, 8, 20, 36, 60])))
        if rng.random() < odd_text:
            name = name + bytes([int(rng.integers(0x80, 0x100))]) + name[:3]
        recs.append((name, seq, qual))
    order = rng.permutation(n_seq)
    parts, pos = [], 0
    offs = np.zeros((3, n_seq), np.uint64)
    for i in order:
        for k in range(3):
            offs[k, i] = pos
            parts.append(recs[i][k])
            pos += len(recs[i][k])
        parts.append(b"\n")  # a separator byte that no span covers
        pos += 1
    data = np.frombuffer(b"".join(parts) + b"\0" * 7, np.uint8).copy()
    arena = BatchArena(data, offs[0].copy(), np.array([len(r[0]) for r in recs], np.uint32), offs[1].copy(),
                       np.array([len(r[1]) for r in recs], np.uint32), offs[2].copy(),
                       np.array([len(r[2]) for r in recs], np.uint32))
    mapped = rng.random(n_seq) < mapped_frac
    rid = np.where(mapped, rng.integers(0, n_contigs, size=n_seq), -1).astype(np.int32)
    flag = np.where(rng.random(n_seq) < 0.5, 16, 0).astype(np.int32)
    flag[~mapped] = 4
    odd = rng.random(n_seq) < 0.03
    flag[odd] = rng.integers(0, 1 << 12, size=int(odd.sum()))
    pos = rng.integers(0, 1 << 28, size=n_seq).astype(np.uint32)
    pos[rng.random(n_seq) < 0.02] = (1 << 32) - 1
    if paired:  # half the pairs on one contig, close together
        near = rng.random(n1) < 0.5
        rid[n1:][near & mapped[:n1]] = rid[:n1][near & mapped[:n1]]
        pos[n1:][near] = (pos[:n1][near].astype(np.int64) + rng.integers(-600, 600, size=int(near.sum()))).clip(
            0, (1 << 32) - 1).astype(np.uint32)
    mapq = rng.choice([0, 1, 20, 40, 60], size=n_seq).astype(np.uint32)
    mapq[rng.random(n_seq) < 0.01] = (1 << 32) - 1
    lens = arena.orig_len.astype(np.int64)
    sl = np.where(rng.random(n_seq) < 0.3, rng.integers(0, 21, size=n_seq), 0).astype(np.uint32)
    sr = np.where(rng.random(n_seq) < 0.3, rng.integers(0, 21, size=n_seq), 0).astype(np.uint32)
    over = rng.random(n_seq) < 0.02  # clips that leave no base
    sl[over] = (lens[over] // 2 + 1).astype(np.uint32)
    sr[over] = (lens[over] // 2 + 1).astype(np.uint32)
    hits = {"rid": rid, "pos": pos, "mapq": mapq, "flag": flag, "sl": sl, "sr": sr,
            "nm": rng.integers(0, 13, size=n_seq).astype(np.uint32)}
    return hits, arena, recs


def oracle_arena(a: BatchArena) -> dict:
    """The arena columns under the oracle's key names (SEQ = original bases)."""
    return {"data": a.data, "name_off": a.name_off, "name_len": a.name_len, "seq_off": a.orig_off,
            "seq_len": a.orig_len, "qual_off": a.qual_off, "qual_len": a.qual_len}


def expected_lines(hits: dict, n1: int, paired: bool, recs, contig_names, rg: str) -> tuple[bytes, int]:
    """The lines through the per-record restatement (hit_from_fm, pair_hits,
    hit_to_sam_line) with the reference's text conversions: names decoded as
    ASCII with replacement, SEQ / QUAL as UTF-8."""

    def hit(r):
        name, seq, qual = recs[r]
        s = seq.decode("utf-8")
        h = hit_from_fm(contig_names, name.decode("ascii", "replace"), s, s, int(hits["rid"][r]),
                        int(hits["pos"][r]), int(hits["mapq"][r]), int(hits["flag"][r]), int(hits["sl"][r]),
                        int(hits["sr"][r]))
        h.qual = qual.decode("utf-8")
        return h

    lines, mapped = [], 0
    for i in range(n1):
        hs = [hit(i)]
        if paired:
            hs = list(pair_hits(hs[0], hit(n1 + i)))
        for h in hs:
            mapped += h.contig != "*"
            lines.append(hit_to_sam_line(h) + "\tRG:Z:" + rg + "\n")
    return "".join(lines).encode("utf-8"), mapped
