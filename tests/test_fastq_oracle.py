"""The FASTQ record-split oracle (oracle/oracle_fastq.c) on the CPU, pinned to
the reference's own unit test (fq2bam-meth/tests/test_linear_fastq.mojo:
30-85, vectors in tests/golden/conversion_vectors.json) and to the line rules
of _pipe_line (linear_fastq.mojo:233-280); and the package's host reader
(mojoalign_b200.fastq) against it."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from fastq_cases import random_fastq

GOLDEN = Path(__file__).resolve().parent / "golden" / "conversion_vectors.json"


def _span(buf, off, n):
    return bytes(buf[int(off):int(off) + int(n)])


def test_reference_unit_vectors():
    g = json.loads(GOLDEN.read_text())["linear_fastq_mojo"]
    r1, r2 = g["r1"].encode(), g["r2"].encode()
    a, b = oracle.fastq_parse(r1), oracle.fastq_parse(r2)
    assert a["n"] == b["n"] == g["n1"]
    assert max(a["max_len"], b["max_len"]) == g["max_len"]
    assert _span(r1, a["name_off"][0], a["name_len"][0]).decode() == g["name1_0"]
    assert r1[a["seq_off"][0] + 1] == g["orig1_0_byte1"]
    assert r2[b["seq_off"][0]] == g["orig2_0_byte0"]
    assert a["seq_len"][1] == g["seq1_1_len"]
    assert a["consumed"] == len(r1)


def test_line_rules():
    p = oracle.fastq_parse(b"@a b/1\r\nAC\r\n+\r\nII\r\n@c/2\nG\n+x\nJ")
    assert p["n"] == 2 and list(p["name_len"]) == [1, 1] and list(p["seq_len"]) == [2, 1]
    assert list(p["qual_len"]) == [2, 1] and p["consumed"] == 30
    # only one '\r' is dropped; an empty SEQ line is a line
    p = oracle.fastq_parse(b"r\nA\r\r\n+\n\n")
    assert p["n"] == 1 and p["seq_len"][0] == 2 and p["qual_len"][0] == 0 and p["name_len"][0] == 1
    # an unterminated rest that is empty after the strip is no line
    p = oracle.fastq_parse(b"@r\nA\n+\nI\n\r")
    assert p["n"] == 1 and p["consumed"] == 9
    # not at the end of the stream: incomplete records wait
    p = oracle.fastq_parse(b"@r\nA\n+\nI\n@s\nC\n+\nJ", at_eof=False)
    assert p["n"] == 1 and p["consumed"] == 9
    for text, msg in ((b"@r\nA\n+\nI\n@s", "SEQ"), (b"@r\nA\n+\nI\n@s\nC\n", "\\+"),
                      (b"@r\nA\n+\nI\n@s\nC\n+\n", "QUAL"), (b"@r\nA\n+\nI\n\n", "SEQ")):
        with pytest.raises(RuntimeError, match=f"truncated FASTQ \\(missing {msg}\\)"):
            oracle.fastq_parse(text)
    # the reference stops asking after max_records: no error then
    assert oracle.fastq_parse(b"@r\nA\n+\nI\n@s", max_records=1)["n"] == 1


def test_chunked_parse_equals_whole():
    text = random_fastq(3, 3000)
    whole = oracle.fastq_parse(text)
    got = {k: [] for k in ("name_off", "seq_off", "qual_off", "name_len", "seq_len", "qual_len")}
    start = 0
    rng = np.random.default_rng(0)
    while start < len(text):
        end = min(len(text), start + int(rng.integers(1, 50_000)))
        p = oracle.fastq_parse(text[start:end], at_eof=end == len(text), base=start)
        for k in got:
            got[k].append(p[k])
        if end == len(text):
            break
        start += p["consumed"]
    for k in got:
        np.testing.assert_array_equal(np.concatenate(got[k]), whole[k])


def test_host_reader_follows_the_oracle(tmp_path):
    from mojoalign_b200.fastq import FastqPairStream

    text = random_fastq(4, 500, crlf=0.3, terminated=False)
    f = tmp_path / "r.fq"
    f.write_bytes(text)
    with FastqPairStream(str(f)) as s:
        a = s.read_batch(10_000)
    p = oracle.fastq_parse(text)
    assert a.n1 == p["n"]
    for i in range(p["n"]):
        assert a.name1[i] == _span(text, p["name_off"][i], p["name_len"][i])
        assert a.orig1[i] == _span(text, p["seq_off"][i], p["seq_len"][i])
        assert a.qual1[i] == _span(text, p["qual_off"][i], p["qual_len"][i])
