"""Bulk FASTQ reader with the contract of fq2bam-meth/src/linear_fastq.mojo.

- `qname_span`  drops a leading '@' and cuts the name at the first space
                or '/' (_qname_span, L308-325).
- `convert`     R1 C/c -> T, R2 G/g -> A (_cvt, L37-46); other bytes stay.
- `FastqPairStream.read_batch` fills a `FastqArena` with up to n pairs,
                keeping name / original / converted / quality spans
                (_store_rec, L365-417; fq_read_batch, L437-451), raising
                "truncated FASTQ (...)" and "paired FASTQ length mismatch
                (R2 ended early)" like the reference.  gzip input is read
                through Python's gzip module instead of a pigz pipe.
- `pack_bases`  row-major n_seq x max_len bytes, R1 rows then R2 rows,
                padded with 'N' (78), plus u32 lengths (fq_pack_bases,
                L454-492).

On the mapping path the bases are packed unconverted and the conversion is
applied on the device (the bs modes of ma_map_batch); `convert` is the host
statement of the same rule.
"""
from __future__ import annotations

import gzip
from dataclasses import dataclass, field

import numpy as np

_BS = {"C2T": 1, "G2A": 2}
_C2T = bytes.maketrans(b"Cc", b"TT")
_G2A = bytes.maketrans(b"Gg", b"AA")


def bs_mode(mode: str) -> int:
    """_bs_mode, linear_fastq.mojo:29-34."""
    return _BS.get(mode, 0)


def convert(seq: bytes, mode) -> bytes:
    m = bs_mode(mode) if isinstance(mode, str) else mode
    if m == 1:
        return seq.translate(_C2T)
    if m == 2:
        return seq.translate(_G2A)
    return seq


def qname_span(header: bytes) -> bytes:
    s = 1 if header[:1] == b"@" else 0
    e = len(header)
    for i in range(s, e):
        if header[i] in (32, 47):
            e = i
            break
    return header[s:e]


@dataclass
class FastqArena:
    n1: int = 0
    max_len: int = 0
    name1: list = field(default_factory=list)
    orig1: list = field(default_factory=list)
    seq1: list = field(default_factory=list)
    qual1: list = field(default_factory=list)
    name2: list = field(default_factory=list)
    orig2: list = field(default_factory=list)
    seq2: list = field(default_factory=list)
    qual2: list = field(default_factory=list)


class _Pipe:
    def __init__(self, path: str, mode: int):
        self.path = path
        low = path.lower()
        self.fh = gzip.open(path, "rb") if (low.endswith(".gz") or low.endswith(".gzip")) else open(path, "rb")
        self.convert = mode

    def line(self):
        """_pipe_line: a line ends at '\\n' and loses one trailing '\\r'; an
        unterminated rest at the end of the stream is a line when it is not
        empty after that strip."""
        ln = self.fh.readline()
        if not ln:
            return None
        terminated = ln.endswith(b"\n")
        if terminated:
            ln = ln[:-1]
        if ln.endswith(b"\r"):
            ln = ln[:-1]
        if not terminated and not ln:
            return None
        return ln

    def record(self):
        h = self.line()
        if h is None:
            return None
        seq = self.line()
        if seq is None:
            raise RuntimeError("truncated FASTQ (missing SEQ)")
        plus = self.line()
        if plus is None:
            raise RuntimeError("truncated FASTQ (missing +)")
        qual = self.line()
        if qual is None:
            raise RuntimeError("truncated FASTQ (missing QUAL)")
        return qname_span(h), seq, convert(seq, self.convert), qual

    def close(self):
        self.fh.close()


class FastqPairStream:
    """fq_open / fq_read_batch / fq_close (linear_fastq.mojo:420-451)."""

    def __init__(self, fq1: str, fq2: str = "", bs_r1: str = "", bs_r2: str = ""):
        self.r1 = _Pipe(fq1, bs_mode(bs_r1))
        self.paired = len(fq2) > 0
        self.r2 = _Pipe(fq2, bs_mode(bs_r2)) if self.paired else None

    def read_batch(self, n_pairs: int) -> FastqArena:
        a = FastqArena()
        n = max(1, n_pairs)
        while a.n1 < n:
            rec = self.r1.record()
            if rec is None:
                break
            a.name1.append(rec[0]); a.orig1.append(rec[1]); a.seq1.append(rec[2]); a.qual1.append(rec[3])
            a.max_len = max(a.max_len, len(rec[1]))
            if self.paired:
                rec2 = self.r2.record()
                if rec2 is None:
                    raise RuntimeError("paired FASTQ length mismatch (R2 ended early)")
                a.name2.append(rec2[0]); a.orig2.append(rec2[1]); a.seq2.append(rec2[2]); a.qual2.append(rec2[3])
                a.max_len = max(a.max_len, len(rec2[1]))
            a.n1 += 1
        return a

    def close(self):
        self.r1.close()
        if self.r2:
            self.r2.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def pack_bases(a: FastqArena, paired: bool, max_len: int, converted: bool = True):
    """fq_pack_bases: (bases [n_seq, max_len] uint8 padded with 'N', lens uint32)."""
    n_seq = a.n1 * (2 if paired else 1)
    bases = np.full((n_seq, max_len), 78, dtype=np.uint8)
    lens = np.zeros(n_seq, dtype=np.uint32)
    rows1 = a.seq1 if converted else a.orig1
    rows2 = a.seq2 if converted else a.orig2
    for i, s in enumerate(rows1):
        lens[i] = len(s)
        if s:
            bases[i, : len(s)] = np.frombuffer(s, dtype=np.uint8)
    if paired:
        for i, s in enumerate(rows2):
            lens[a.n1 + i] = len(s)
            if s:
                bases[a.n1 + i, : len(s)] = np.frombuffer(s, dtype=np.uint8)
    return bases, lens
