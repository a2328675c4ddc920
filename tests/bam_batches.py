"""Seeded mapped batches for the BAM packing tests, and a BAM record reader.

A batch is the input of _emit_bam_from_batch (fq2bam-meth/src/
linear_gpu_fm.mojo:669-984): the seven mapping outputs, the FASTQ arena
(name / original bases / converted bases / qualities of every record, laid
out in the arena in a shuffled order so offsets are arbitrary) and a
rid -> tid table.  Values range past what the mapper emits (any flag bits,
clips beyond the read, positions up to 2^32 - 1, arbitrary base and quality
bytes) so the packer's clamping and truncation rules are all exercised.
"""
from __future__ import annotations

import struct

import numpy as np

from mojoalign_b200.bam import BatchArena

RID_TO_TID = np.array([0, 0, 1, 1, 2, 2, -1, 3], np.int32)


def random_batch(seed: int, n1: int, paired: bool, *, max_len: int = 300, long_frac: float = 0.0,
                 with_quals: bool = True, mapped_frac: float = 0.8):
    rng = np.random.default_rng(seed)
    n_seq = n1 * (2 if paired else 1)
    lens = rng.choice([0, 1, 2, 31, 75, 100, 101, 150, 151, 250, max_len], size=n_seq,
                      p=[0.01, 0.01, 0.02, 0.03, 0.1, 0.1, 0.1, 0.35, 0.12, 0.1, 0.06])
    if long_frac:
        longs = rng.random(n_seq) < long_frac
        lens[longs] = rng.integers(1500, 4000, size=int(longs.sum()))
    recs = []
    for i in range(n_seq):
        q = int(lens[i])
        if rng.random() < 0.05:
            seq = rng.integers(0, 256, size=q, dtype=np.uint8).tobytes()
        else:
            seq = np.frombuffer(b"ACGTNacgtn", np.uint8)[rng.choice(10, size=q, p=[.225, .225, .225, .225, .02,
                                                                             .015, .015, .015, .015, .02])].tobytes()
        u = rng.random()
        if u < 0.04:
            qual = rng.integers(0, 256, size=q, dtype=np.uint8).tobytes()
        elif u < 0.08:
            qual = rng.integers(33, 75, size=max(0, q + int(rng.choice([-2, -1, 1, 5]))), dtype=np.uint8).tobytes()
        else:
            qual = rng.integers(33, 75, size=q, dtype=np.uint8).tobytes()
        nl = int(rng.choice([0, 1, 8, 20, 36, 60, 255, 300], p=[0.01, 0.02, 0.2, 0.4, 0.3, 0.05, 0.01, 0.01]))
        name = np.frombuffer(b"ABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789:_", np.uint8)[
            rng.integers(0, 38, size=nl)].tobytes()
        recs.append((name, seq, qual))
    # arena: per record name, orig, converted, qual (the reference's push
    # order, linear_fastq.mojo:393-396), records in shuffled order
    order = rng.permutation(n_seq)
    parts, pos = [], 0
    offs = np.zeros((3, n_seq), np.uint64)
    for i in order:
        name, seq, qual = recs[i]
        for k, b in ((0, name), (1, seq), (None, seq.translate(bytes.maketrans(b"Cc", b"TT"))), (2, qual)):
            if k is not None:
                offs[k, i] = pos
            parts.append(b)
            pos += len(b)
    data = np.frombuffer(b"".join(parts) + b"\0" * 7, np.uint8).copy()
    arena = BatchArena(data, offs[0].copy(), np.array([len(r[0]) for r in recs], np.uint32), offs[1].copy(),
                       np.array([len(r[1]) for r in recs], np.uint32),
                       offs[2].copy() if with_quals else None,
                       np.array([len(r[2]) for r in recs], np.uint32) if with_quals else None)
    mapped = rng.random(n_seq) < mapped_frac
    rid = np.where(mapped, rng.integers(0, len(RID_TO_TID), size=n_seq), -1).astype(np.int32)
    rid[rng.random(n_seq) < 0.02] = len(RID_TO_TID) + 3  # past the table: unmapped
    flag = np.where(rng.random(n_seq) < 0.5, 16, 0).astype(np.int32)
    flag[~mapped] = 4
    odd = rng.random(n_seq) < 0.03
    flag[odd] = rng.integers(0, 1 << 12, size=int(odd.sum()))
    pos = rng.integers(0, 1 << 28, size=n_seq).astype(np.uint32)
    pos[rng.random(n_seq) < 0.05] = rng.integers(0, 40, size=1)[0]
    pos[rng.random(n_seq) < 0.02] = rng.integers(1 << 31, (1 << 32) - 1, dtype=np.uint64, size=1)[0]
    if paired:  # half the pairs close together, like proper pairs
        near = rng.random(n1) < 0.5
        pos[n1:][near] = (pos[:n1][near].astype(np.int64) + rng.integers(-600, 600, size=int(near.sum()))).clip(
            0, (1 << 32) - 1).astype(np.uint32)
        same = rng.random(n1) < 0.4
        rid[n1:][same & mapped[:n1]] = rid[:n1][same & mapped[:n1]]
    sl = rng.choice([0, 0, 0, 1, 3, 12, 20], size=n_seq).astype(np.uint32)
    sr = rng.choice([0, 0, 0, 2, 5, 19], size=n_seq).astype(np.uint32)
    big = rng.random(n_seq) < 0.02
    sl[big] = lens[big] + rng.integers(0, 3, size=int(big.sum()))
    sr[rng.random(n_seq) < 0.01] = (1 << 31) + 5
    hits = {
        "rid": rid, "pos": pos, "mapq": rng.choice([0, 1, 20, 60, 254, 300], size=n_seq).astype(np.uint32),
        "flag": flag, "sl": sl, "sr": sr, "nm": rng.choice([0, 0, 1, 2, 7, 255, 400], size=n_seq).astype(np.uint32),
    }
    return hits, arena, recs


def bam_cap_for(arena: BatchArena, rg_n: int) -> int:
    return int(arena.n_seq * (64 + rg_n) + int(arena.name_len.sum()) + 2 * int(arena.orig_len.sum()))


HEADER = struct.Struct("<iiiIIiiii")


def read_records(buf: bytes) -> list[dict]:
    """Splits BAM records and decodes their fixed fields."""
    out, off = [], 0
    while off < len(buf):
        block, tid, pos, bmn, fnc, l_seq, ntid, npos, tlen = HEADER.unpack_from(buf, off)
        l_qname = bmn & 255
        n_cigar = fnc & 0xFFFF
        p = off + 36
        name = buf[p:p + l_qname - 1]
        p += l_qname
        cigar = struct.unpack_from(f"<{n_cigar}I", buf, p)
        out.append({"off": off, "bytes": 4 + block, "tid": tid, "pos": pos, "bin": bmn >> 16, "mapq": (bmn >> 8) & 255,
                    "flag": fnc >> 16, "n_cigar": n_cigar, "l_seq": l_seq, "ntid": ntid, "npos": npos,
                    "tlen": tlen, "name": name, "cigar": cigar})
        off += 4 + block
    assert off == len(buf)
    return out


def random_tile_meta(seed: int, n: int, *, dup_rate: float = 0.3, unplaced: float = 0.05):
    """Sort/markdup inputs shaped like a tile's metadata: pairs share their
    duplicate key, score and pair id; a fraction of pairs repeat another
    pair's key (duplicates), some records are unplaced (dhi = ~0)."""
    rng = np.random.default_rng(seed)
    n_pairs = (n + 1) // 2
    tid = rng.integers(0, 4, size=n_pairs).astype(np.uint64)
    p5 = rng.integers(0, 1 << 20, size=n_pairs).astype(np.uint64)
    src = np.arange(n_pairs)
    dups = rng.random(n_pairs) < dup_rate
    src[dups] = rng.integers(0, n_pairs, size=int(dups.sum()))
    dhi = ((tid[src] + 1) << 48) | (p5[src] + (1 << 30))
    dlo = ((tid[src] + 1) << 48) | (np.uint64(1) << 47) | (p5[src] + (1 << 30) + 300)
    score = rng.integers(0, 4, size=n_pairs).astype(np.uint32) << 8
    pair = np.arange(n_pairs, dtype=np.uint32) + np.uint32(rng.integers(0, 1000))
    un = rng.random(n_pairs) < unplaced
    dhi[un] = ~np.uint64(0)
    rec = np.repeat(np.arange(n_pairs), 2)[:n]
    coord = (tid[rec] << 32) | (p5[rec] + np.uint64(rng.integers(0, 400, size=n)))
    idx = np.arange(n, dtype=np.uint64)
    coord[un[rec]] = (np.uint64(0xFFFFFFFF) << 32) | idx[un[rec]]
    dlo_r = dlo[rec].copy()
    dlo_r[un[rec]] = (2 * (idx[un[rec]] // 2))
    return {"coord": coord, "dhi": dhi[rec], "dlo": dlo_r, "score": score[rec], "pair": pair[rec]}
