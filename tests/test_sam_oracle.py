"""The SAM-side oracle (oracle/oracle_sam.c), pinned on the CPU.

- The FASTQ split under the SAM path's reader rules against records read by
  the reference's own FastqPairReader (fq2bam-meth/python/fastq_batch.py) on
  the committed golden texts (tests/golden/fastq_pair_reader.json).
- The SAM lines against the per-record restatement of _hit_from_fm,
  pair_hits and hit_to_sam_line (mojoalign_b200.linear_fm, itself pinned by
  the unit vectors of test_sam_emit.py) on seeded batches.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from sam_batches import CONTIGS, expected_lines, oracle_arena, random_sam_batch

GOLDEN = Path(__file__).resolve().parent / "golden" / "fastq_pair_reader.json"
_CVT = {"C2T": bytes.maketrans(b"Cc", b"Tt"), "G2A": bytes.maketrans(b"Gg", b"Aa")}


def _cases():
    return json.loads(GOLDEN.read_text())["cases"]


def _records(text: bytes, res: dict) -> list:
    """(name as the reader's str in UTF-8, original bases, qualities)."""
    out = []
    for i in range(res["n"]):
        nm = text[int(res["name_off"][i]):int(res["name_off"][i]) + int(res["name_len"][i])]
        sq = text[int(res["seq_off"][i]):int(res["seq_off"][i]) + int(res["seq_len"][i])]
        ql = text[int(res["qual_off"][i]):int(res["qual_off"][i]) + int(res["qual_len"][i])]
        out.append((nm.decode("ascii", "replace").encode("utf-8"), sq, ql))
    return out


def test_pair_reader_split_matches_reference_reader():
    cases = _cases()
    assert len(cases) >= 30
    for c in cases:
        for m in ("1", "2"):
            raw = c["r" + m]
            if raw is None:
                continue
            text = bytes.fromhex(raw)
            want = [(bytes.fromhex(r[0]), bytes.fromhex(r[1]), bytes.fromhex(r[3])) for r in c["records" + m]]
            res = oracle.fastq_parse_pr(text)
            got = _records(text, res)
            if c["error"]:  # R2 ended early: the reference returned nothing
                assert m == "1" or len(got) < len(_records(bytes.fromhex(c["r1"]),
                                                           oracle.fastq_parse_pr(bytes.fromhex(c["r1"]))))
                continue
            # the reader stops at the shorter file of a pair
            n = len(want)
            assert got[:n] == want, c["r1"][:80]
            if m == "1" or c["r2"] is None:
                assert len(got) == n
            # converted bases (the mapper's input) follow bs_r1 / bs_r2
            mode = c["bs_r" + m]
            for r, (_, sq, _) in zip(c["records" + m], got):
                assert bytes.fromhex(r[2]) == (sq.translate(_CVT[mode]) if mode in _CVT else sq)


def test_pair_reader_split_of_partial_buffers():
    for c in _cases():
        text = bytes.fromhex(c["r1"])
        full = oracle.fastq_parse_pr(text)
        for cut in sorted(set(np.linspace(0, len(text), num=min(len(text) + 1, 40), dtype=int).tolist())):
            part = oracle.fastq_parse_pr(text[:cut], at_eof=False, base=5)
            n = part["n"]
            assert n <= full["n"]
            for k in ("name_len", "seq_len", "qual_len"):
                np.testing.assert_array_equal(part[k], full[k][:n])
            for k in ("name_off", "seq_off", "qual_off"):
                np.testing.assert_array_equal(part[k], full[k][:n] + 5)
            # a record is taken only when its four lines end in '\n'
            assert text[:part["consumed"]].count(b"\n") == 4 * n
            rest = oracle.fastq_parse_pr(text[part["consumed"]:])
            assert part["n"] + rest["n"] == full["n"] or rest["n"] == full["n"] - n


@pytest.mark.parametrize("paired", [False, True])
@pytest.mark.parametrize("seed,n1", [(1, 1), (2, 9), (3, 1500)])
def test_sam_lines_match_record_restatement(seed, n1, paired):
    hits, arena, recs = random_sam_batch(seed, n1, paired)
    got, mapped = oracle.emit_sam(hits, n1, paired, oracle_arena(arena), CONTIGS, b"rg1")
    want, want_mapped = expected_lines(hits, n1, paired, recs, CONTIGS, "rg1")
    assert got == want
    assert mapped == want_mapped


def test_sam_unit_lines():
    recs = [(b"r1", b"ACGTAA", b"IIIIII"), (b"r2", b"TTGCA", b"")]
    from mojoalign_b200.bam import BatchArena

    a = oracle_arena(BatchArena.from_records(recs))
    hits = {"rid": np.array([1, 3]), "pos": np.array([99, 9]), "mapq": np.array([60, 20]),
            "flag": np.array([0, 16]), "sl": np.array([1, 0]), "sr": np.array([2, 0])}
    text, mapped = oracle.emit_sam(hits, 1, True, a, CONTIGS, b"g")
    # different canonical contigs: RNEXT / PNEXT of the mate, no flag 2
    assert text == (b"r1\t65\tchr1\t100\t60\t1S3M2S\tchr2\t10\t0\tACGTAA\tIIIIII\tRG:Z:g\n"
                    b"r2\t145\tchr2\t10\t20\t5M\tchr1\t100\t0\tTGCAA\t\tRG:Z:g\n")
    assert mapped == 2
    hits["rid"][1] = 7  # fchr1 again under another rid: the same canonical contig
    lines = oracle.emit_sam(hits, 1, True, a, CONTIGS, b"g")[0].split(b"\n")
    # |10 - 100| + len(SEQ2) = 95; flags gain 2
    assert lines[0] == b"r1\t67\tchr1\t100\t60\t1S3M2S\t=\t10\t95\tACGTAA\tIIIIII\tRG:Z:g"
    assert lines[1] == b"r2\t147\tchr1\t10\t20\t5M\t=\t100\t-95\tTGCAA\t\tRG:Z:g"
    hits["rid"][1] = 6  # canonical name "*": placed, but the pair sees it as unplaced
    lines = oracle.emit_sam(hits, 1, True, a, CONTIGS, b"g")[0].split(b"\n")
    assert lines[0] == b"r1\t73\tchr1\t100\t60\t1S3M2S\t*\t0\t0\tACGTAA\tIIIIII\tRG:Z:g"
    assert lines[1] == b"r2\t145\t*\t10\t20\t5M\tchr1\t100\t0\tTGCAA\t\tRG:Z:g"


def test_sam_errors():
    hits, arena, recs = random_sam_batch(5, 50, True, odd_text=0.0)
    a = oracle_arena(arena)
    text, _ = oracle.emit_sam(hits, 50, True, a, CONTIGS, b"x")
    with pytest.raises(RuntimeError, match="SAM batch buffer overflow"):
        oracle.emit_sam(hits, 50, True, a, CONTIGS, b"x", cap=len(text) - 1)
    assert oracle.emit_sam(hits, 50, True, a, CONTIGS, b"x", cap=len(text))[0] == text
    bad = dict(hits)
    bad["rid"] = hits["rid"].copy()
    bad["rid"][7] = len(CONTIGS)
    with pytest.raises(RuntimeError, match="rid outside"):
        oracle.emit_sam(bad, 50, True, a, CONTIGS, b"x")
    d = a["data"].copy()
    d[int(a["qual_off"][3])] = 0xff  # not UTF-8
    if a["qual_len"][3] == 0:
        d[int(a["seq_off"][3])] = 0xff
    with pytest.raises(RuntimeError, match="not valid UTF-8"):
        oracle.emit_sam(hits, 50, True, dict(a, data=d), CONTIGS, b"x")
