"""FASTQ input files of the device pipelines: open_fastq() gives the bytes
the reference's readers see (gzip by suffix), with BGZF files inflated on a
thread pool.  Checked against Python's gzip module on BGZF files written by
the oracle's restatement of the reference's BGZF writer, plain and
multi-member gzip, mixed, padded, truncated and corrupted files."""
from __future__ import annotations

import gzip
import zlib

import numpy as np
import pytest

from fastq_cases import random_fastq
from mojoalign_b200.fqio import BgzfReader, is_bgzf, open_fastq
from oracle import bgzf_ref


def _read_all(f, step):
    out = bytearray()
    buf = bytearray(step)
    while True:
        k = f.readinto(buf)
        if not k:
            return bytes(out)
        out += buf[:k]


@pytest.fixture(scope="module")
def text():
    return random_fastq(3, 6000, crlf=0.3)


@pytest.mark.parametrize("level", [0, 1, 6])
@pytest.mark.parametrize("step", [1 << 20, 65280, 4097, 1])
def test_bgzf_files_read_like_gzip(tmp_path, text, level, step):
    if step == 1 and level != 1:
        pytest.skip("byte-at-a-time reads once")
    p = tmp_path / "r.fq.gz"
    p.write_bytes(bgzf_ref.compress(text, level))
    assert is_bgzf(str(p))
    with BgzfReader(str(p), threads=3, batch_bytes=200_000) as f:
        got = _read_all(f, step) if step > 1 else f.read(len(text) // 7) + f.read()
    assert got == gzip.decompress(p.read_bytes()) == text


def test_other_gzip_files_and_plain(tmp_path, text):
    one = tmp_path / "one.fq.gz"
    one.write_bytes(gzip.compress(text))
    multi = tmp_path / "multi.fastq.gzip"
    multi.write_bytes(gzip.compress(text[:1000]) + gzip.compress(text[1000:]))
    plain = tmp_path / "plain.fq"
    plain.write_bytes(text)
    for p in (one, multi, plain):
        assert not is_bgzf(str(p)) or p == plain
        with open_fastq(str(p)) as f:
            assert _read_all(f, 1 << 16) == text
    # BGZF members, then a plain gzip member, then zero padding
    mixed = tmp_path / "mixed.fq.gz"
    mixed.write_bytes(bgzf_ref.compress(text[:50_000], 1, eof=False) + gzip.compress(text[50_000:]) + b"\0" * 10)
    assert is_bgzf(str(mixed))
    with open_fastq(str(mixed), threads=2) as f:
        assert _read_all(f, 1 << 16) == gzip.decompress(mixed.read_bytes()) == text
    empty = tmp_path / "empty.fq.gz"
    empty.write_bytes(bgzf_ref.compress(b"", 1))
    with open_fastq(str(empty)) as f:
        assert _read_all(f, 100) == b""


def test_damaged_bgzf_files_fail_like_gzip(tmp_path, text):
    blob = bgzf_ref.compress(text, 1)
    cut = tmp_path / "cut.fq.gz"
    cut.write_bytes(blob[:len(blob) // 2])
    with pytest.raises(EOFError):
        gzip.decompress(cut.read_bytes())
    with pytest.raises(EOFError), open_fastq(str(cut), threads=2) as f:
        _read_all(f, 1 << 16)
    bad = bytearray(blob)
    m = bgzf_ref.members(bytes(blob))[1]
    bad[m["off"] + m["size"] - 5] ^= 0xFF  # the second member's ISIZE
    p = tmp_path / "bad.fq.gz"
    p.write_bytes(bytes(bad))
    with pytest.raises(gzip.BadGzipFile):
        gzip.decompress(bytes(bad))
    with pytest.raises(gzip.BadGzipFile), open_fastq(str(p), threads=2) as f:
        _read_all(f, 1 << 16)
    junk = tmp_path / "junk.fq.gz"
    junk.write_bytes(blob + b"xyz")
    with pytest.raises(gzip.BadGzipFile), open_fastq(str(junk)) as f:
        _read_all(f, 1 << 16)


def test_large_bgzf_file_many_batches(tmp_path):
    rng = np.random.default_rng(0)
    text = random_fastq(9, 40_000) + rng.integers(65, 70, size=3_000_000, dtype=np.uint8).tobytes()
    p = tmp_path / "big.fq.gz"
    p.write_bytes(bgzf_ref.compress(text, 1))
    with BgzfReader(str(p), threads=4, batch_bytes=1 << 20) as f:
        got = _read_all(f, 3 << 20)
    assert zlib.crc32(got) == zlib.crc32(text) and got == text


@pytest.mark.parametrize("threads,min_split", [(1, 1), (4, 1), (3, 1 << 20), (8, 7)])
def test_parallel_writer(tmp_path, threads, min_split):
    from mojoalign_b200.fqio import ParallelWriter

    rng = np.random.default_rng(threads)
    parts = [rng.integers(0, 256, size=n, dtype=np.uint8).tobytes() for n in (0, 1, 5, 4 << 20, 3, 1_000_001)]
    p = tmp_path / "out.bin"
    with ParallelWriter(p, threads=threads, min_split=min_split) as w:
        for b in parts:
            assert w.write(b) == len(b)
            assert w.write(memoryview(np.frombuffer(b, np.uint8))) == len(b)
    assert p.read_bytes() == b"".join(b + b for b in parts)
    with ParallelWriter(p, threads=threads) as w:  # truncates
        w.write(b"xy")
    assert p.read_bytes() == b"xy"


def test_bgzf_member_table(text):
    from mojoalign_b200.fqio import bgzf_members

    blob = bgzf_ref.compress(text, 1)
    t = bgzf_members(blob)
    ms = bgzf_ref.members(blob)
    assert t["src_off"].size == len(ms) and t["out_bytes"] == len(text)
    for i, m in enumerate(ms):
        payload = blob[int(t["src_off"][i]):int(t["src_off"][i]) + int(t["src_len"][i])]
        assert payload == m["payload"] and t["isize"][i] == m["isize"] and t["crc"][i] == m["crc"]
    assert list(t["dst_off"]) == list(np.concatenate([[0], np.cumsum(t["isize"][:-1].astype(np.uint64))]))
    with pytest.raises(gzip.BadGzipFile):
        bgzf_members(blob[:-5])  # the EOF member cut short
    with pytest.raises(gzip.BadGzipFile):
        bgzf_members(gzip.compress(text))  # not BGZF
    assert bgzf_members(b"")["out_bytes"] == 0
