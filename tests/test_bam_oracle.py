"""The BAM packing oracle (oracle/oracle_bam.c), pinned on the CPU.

- Record bytes against the reference's own Python BAM writer
  (fq2bam-meth/python/bam_emit.py) on the committed golden records, and the
  reference's unit vectors (tests/test_bam_emit.py:15-17).
- The batch rules of _emit_bam_from_batch (fq2bam-meth/src/
  linear_gpu_fm.mojo:669-984) on hand-built single-end and paired batches:
  flags, mate fields, TLEN, metadata keys, tile counters and the two
  failure modes.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from bam_batches import RID_TO_TID, read_records
from mojoalign_b200.bam import BatchArena

GOLDEN = Path(__file__).resolve().parent / "golden" / "bam_records.json"


def _golden():
    return json.loads(GOLDEN.read_text())


def test_records_match_reference_writer():
    g = _golden()
    rg = g["rg"].encode()
    assert len(g["records"]) >= 300
    for r in g["records"]:
        got = oracle.pack_aln(r["name"].encode(), r["flag"], r["tid"], r["pos"], r["mapq"], r["sl"], r["sr"],
                              r["seq"].encode(), None if r["qual"] is None else r["qual"].encode(), r["ntid"],
                              r["npos"], r["tlen"], r["nm"], rg)
        assert got.hex() == r["expect"], r


def test_reference_unit_vectors():
    u = _golden()["unit"]
    rec = read_records(oracle.pack_aln(b"r", 0, 0, 0, 0, 0, 0, b"ACGT", b"IIII", -1, -1, 0, 0, b"x"))[0]
    seq_off = rec["off"] + 36 + 2 + 4 * rec["n_cigar"]
    raw = oracle.pack_aln(b"r", 0, 0, 0, 0, 0, 0, b"ACGT", b"IIII", -1, -1, 0, 0, b"x")
    assert raw[seq_off:seq_off + 2].hex() == u["pack_seq_ACGT"] == "1248"
    for beg, end, want in u["reg2bin"]:
        if end - beg > 4096:
            continue
        qlen = max(end - beg, 0)
        rec = read_records(oracle.pack_aln(b"r", 0, 0, beg, 0, 0, 0, b"A" * qlen, None, -1, -1, 0, 0, b"x"))[0]
        assert rec["bin"] == want, (beg, end)


def _arena(records):
    return vars(BatchArena.from_records(records))


def _hits(rows):
    keys = ("rid", "pos", "mapq", "flag", "sl", "sr", "nm")
    return {k: np.array([r[i] for r in rows]) for i, k in enumerate(keys)}


def test_single_end_batch_rules():
    recs = [(b"a", b"ACGTACGTAC", b"I" * 10), (b"b", b"ACGTACGTAC", b"I" * 10), (b"c", b"ACGTACGTAC", b"I" * 10)]
    # rid, pos, mapq, flag, sl, sr, nm
    rows = [(1, 100, 60, 0, 2, 3, 1), (-1, 0, 0, 4, 0, 0, 0), (2, 200, 30, 16, 1, 4, 300)]
    bam, meta, mapped = oracle.emit_bam(_hits(rows), _arena(recs), 3, False, RID_TO_TID, b"rg1", n_reads=5,
                                        n_total=100, meta_cap=8, chunk=2)
    r = read_records(bam)
    assert [x["flag"] for x in r] == [65, 69, 81]
    assert [x["tid"] for x in r] == [0, -1, 1] and [x["pos"] for x in r] == [100, -1, 200]
    assert r[0]["cigar"] == ((2 << 4) | 4, 5 << 4, (3 << 4) | 4)
    assert r[2]["cigar"] == ((4 << 4) | 4, 5 << 4, (1 << 4) | 4)  # clips swap on the reverse strand
    assert r[1]["n_cigar"] == 0 and r[1]["bin"] == 4680
    assert mapped == 2
    assert list(meta["coord"]) == [100, (0xFFFFFFFF << 32) | 6, (1 << 32) | 200]
    # _pack_end: (tid + 1) << 48 | strand << 47 | (unclipped 5' + 2^30)
    assert meta["dhi"][0] == (1 << 48) | (98 + (1 << 30))
    assert meta["dhi"][2] == (2 << 48) | (1 << 47) | (200 + 5 + 1 - 1 + (1 << 30))
    assert meta["dhi"][1] == (1 << 64) - 1 and list(meta["dlo"]) == [0, 6, 0]
    assert list(meta["rec"]) == [(2 << 32) | x["off"] for x in r]
    assert list(meta["len"]) == [x["bytes"] for x in r]
    assert list(meta["score"]) == [(60 << 8) | 254, 255, (30 << 8) | 0]
    assert list(meta["pair"]) == [105, 106, 107]


def test_paired_batch_rules():
    recs = [(b"p%d" % i, b"ACGTACGTAC" + b"A" * (i % 3), b"I" * (10 + i % 3)) for i in range(8)]
    # R1 rows then R2 rows: proper pair, mate unmapped, different tids, both unmapped
    rows1 = [(1, 100, 60, 0, 0, 0, 1), (1, 500, 50, 16, 0, 0, 0), (1, 900, 40, 0, 0, 0, 0), (-1, 0, 0, 4, 0, 0, 0)]
    rows2 = [(0, 150, 60, 16, 0, 0, 2), (-1, 0, 0, 4, 0, 0, 0), (3, 70, 30, 16, 0, 0, 1), (-1, 0, 0, 4, 0, 0, 0)]
    bam, meta, mapped = oracle.emit_bam(_hits(rows1 + rows2), _arena(recs), 4, True, RID_TO_TID, b"rg1",
                                        n_reads=10, n_total=1000, meta_cap=18, chunk=0)
    r = read_records(bam)
    assert [x["name"] for x in r] == [b"p0", b"p4", b"p1", b"p5", b"p2", b"p6", b"p3", b"p7"]
    assert [x["flag"] for x in r] == [67, 147, 89, 133, 65, 145, 77, 141]
    qlen_r2 = 10 + 4 % 3
    assert (r[0]["tlen"], r[1]["tlen"]) == (50 + qlen_r2, -(50 + qlen_r2))
    assert (r[0]["ntid"], r[0]["npos"], r[1]["ntid"], r[1]["npos"]) == (0, 150, 0, 100)
    assert (r[2]["ntid"], r[2]["npos"], r[3]["ntid"], r[3]["npos"]) == (-1, -1, 0, 500)
    assert (r[4]["ntid"], r[4]["npos"], r[5]["ntid"], r[5]["npos"]) == (1, 70, 0, 900)
    assert all(x["tlen"] == 0 for x in r[2:])
    assert mapped == 5
    assert list(meta["pair"]) == [505, 505, 506, 506, 507, 507, 508, 508]
    assert meta["score"][0] == meta["score"][1] == (120 << 8) | 252
    assert meta["dhi"][0] <= meta["dlo"][0] and meta["dhi"][0] == meta["dhi"][1]
    assert meta["dlo"][2] == 0 and meta["dhi"][6] == (1 << 64) - 1 and meta["dlo"][6] == 16
    assert meta["coord"][7] == (0xFFFFFFFF << 32) | 17


def test_failure_modes():
    recs = [(b"a", b"ACGT", b"IIII")] * 4
    rows = [(0, 1, 1, 0, 0, 0, 0)] * 4
    with pytest.raises(RuntimeError, match="FM sort cap exceeded"):
        oracle.emit_bam(_hits(rows), _arena(recs), 4, False, RID_TO_TID, b"r", n_reads=1, meta_cap=4)
    with pytest.raises(RuntimeError, match="FM sort cap exceeded"):  # paired: n_reads + 1 >= cap
        oracle.emit_bam(_hits(rows), _arena(recs), 2, True, RID_TO_TID, b"r", n_reads=1, meta_cap=4)
    oracle.emit_bam(_hits(rows), _arena(recs), 2, True, RID_TO_TID, b"r", n_reads=0, meta_cap=4)
    with pytest.raises(RuntimeError, match="BAM batch buffer overflow"):
        oracle.emit_bam(_hits(rows), _arena(recs), 4, False, RID_TO_TID, b"r", cap=100)


def test_header_matches_reference_writer():
    from mojoalign_b200.fq2bam import bam_header
    from mojoalign_b200.mapper import Contig

    g = _golden()["header"]
    # bwa-meth contigs: f<name> / r<name> pairs collapse to one @SQ each
    contigs = [Contig("r" + n, 0, ln) for n, ln in zip(g["sq_names"], g["sq_lens"])]
    contigs += [Contig("f" + n, 0, ln) for n, ln in zip(g["sq_names"], g["sq_lens"])]
    assert bam_header(contigs, {}).hex() == g["blob"]
