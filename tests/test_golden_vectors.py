"""The reference's own known answers for read conversion and packing.

- conversion_vectors.json comes from executing the reference's
  fq2bam-meth/python/fq2bam_meth.py (convert_fastq / convert_fasta_c2t /
  _convert_base) and from the assertions of
  fq2bam-meth/tests/test_linear_fastq.mojo:30-85 (see make_golden.py).
- pack codes restate pack_bases_kernel (linear_gpu_fm.mojo:1136-1154).
"""
from __future__ import annotations

import gzip
import json
from pathlib import Path

import numpy as np

import oracle
from mojoalign_b200 import fastq

GOLD = json.loads((Path(__file__).parent / "golden" / "conversion_vectors.json").read_text())


def codes(s: bytes) -> list[int]:
    return list(oracle.pack_bases(s))


def test_pack_codes_match_reference_kernel():
    expect = {ord("A"): 0, ord("a"): 0, ord("C"): 1, ord("c"): 1, ord("G"): 2, ord("g"): 2, ord("T"): 3,
              ord("t"): 3}
    allb = bytes(range(256))
    got = oracle.pack_bases(allb)
    for b in range(256):
        assert got[b] == expect.get(b, 255), b


def test_oracle_convert_matches_reference_convert_fastq():
    # The Mojo _cvt upper-cases the converted base ('c' -> 'T') where the
    # Python converter keeps case ('c' -> 't'); both pack to the same code.
    for row in GOLD["convert_fastq"]:
        s = row["seq"].encode()
        assert codes(oracle.convert(s, 1)) == codes(row["C2T"].encode())
        assert codes(oracle.convert(s, 2)) == codes(row["G2A"].encode())
        assert codes(fastq.convert(s, "C2T")) == codes(row["C2T"].encode())
        assert codes(fastq.convert(s, "G2A")) == codes(row["G2A"].encode())
        # upper-case inputs convert byte-identically
        if s == s.upper():
            assert oracle.convert(s, 1).decode() == row["C2T"]
            assert oracle.convert(s, 2).decode() == row["G2A"]


def test_convert_base_and_fasta_vectors():
    for row in GOLD["convert_base"]:
        for mode, m in (("C2T", 1), ("G2A", 2)):
            got = oracle.convert(row["base"].encode(), m).decode()
            assert got.upper() == row[mode].upper()
    row = GOLD["convert_fasta_c2t"][0]
    assert row["body"] == "ACGTCacgt" and row["out"].strip() == "ATGTTaTgt"
    assert codes(oracle.convert(b"ACGTCacgt", 1)) == codes(b"ATGTTaTgt")


def test_linear_fastq_known_answers(tmp_path):
    v = GOLD["linear_fastq_mojo"]
    r1, r2 = tmp_path / "r1.fq", tmp_path / "r2.fq"
    r1.write_text(v["r1"])
    r2.write_text(v["r2"])
    with fastq.FastqPairStream(str(r1), str(r2), "C2T", "G2A") as s:
        a = s.read_batch(8)
    assert a.n1 == v["n1"] and a.max_len == v["max_len"]
    assert a.name1[0] == v["name1_0"].encode()
    assert a.orig1[0][1] == v["orig1_0_byte1"]
    assert a.seq1[0][1] == v["seq1_0_byte1"]
    assert a.orig2[0][0] == v["orig2_0_byte0"]
    assert a.seq2[0][0] == v["seq2_0_byte0"]
    assert a.seq1[1][0] == v["seq1_1_byte0"] and len(a.seq1[1]) == v["seq1_1_len"]
    bases, lens = fastq.pack_bases(a, True, 8)
    flat = bases.reshape(-1)
    assert lens[0] == v["packed_len0"]
    assert flat[1] == v["packed_byte1"]
    assert flat[12] == v["packed_byte12"]
    assert flat[16] == v["packed_byte16"]
    # gzip input and EOF behaviour (test_linear_fastq.mojo:120-135)
    gz = tmp_path / "r1.fq.gz"
    with gzip.open(gz, "wb") as f:
        f.write(v["r1"].encode())
    with fastq.FastqPairStream(str(gz), "", "C2T", "") as s:
        ag = s.read_batch(8)
    assert ag.n1 == 2 and ag.seq1[0][1] == 84
    with fastq.FastqPairStream(str(r1)) as s:
        s.read_batch(1000)
        assert s.read_batch(8).n1 == 0


def test_fastq_errors(tmp_path):
    bad = tmp_path / "bad.fq"
    bad.write_text("@r1\nACGT\n+\n")
    with fastq.FastqPairStream(str(bad)) as s:
        try:
            s.read_batch(4)
            raise AssertionError("expected an error")
        except RuntimeError as e:
            assert "truncated FASTQ" in str(e)
    r1, r2 = tmp_path / "a.fq", tmp_path / "b.fq"
    r1.write_text("@x\nAC\n+\nII\n@y\nAC\n+\nII\n")
    r2.write_text("@x\nAC\n+\nII\n")
    with fastq.FastqPairStream(str(r1), str(r2)) as s:
        try:
            s.read_batch(4)
            raise AssertionError("expected an error")
        except RuntimeError as e:
            assert "R2 ended early" in str(e)


def test_qname_span():
    assert fastq.qname_span(b"@read1 extra/1") == b"read1"
    assert fastq.qname_span(b"@frag/1") == b"frag"
    assert fastq.qname_span(b"plain") == b"plain"
    assert fastq.qname_span(b"@") == b""


def test_pack_layout_is_reference_layout():
    a = fastq.FastqArena(n1=2, max_len=3, seq1=[b"AC", b"GTA"], orig1=[b"AC", b"GTA"], seq2=[b"T", b""],
                         orig2=[b"T", b""])
    bases, lens = fastq.pack_bases(a, True, 4)
    assert bases.shape == (4, 4)
    assert list(lens) == [2, 3, 1, 0]
    assert bytes(bases[0]) == b"ACNN" and bytes(bases[3]) == b"NNNN"
    assert np.all(bases[2, 1:] == 78)
