"""SAM records of the drop-in, restating the reference's emit rules:
_hit_from_fm (fq2bam-meth/src/linear_gpu_fm.mojo:987-1025), pair_hits and
hit_to_sam_line (fq2bam-meth/src/linear_extend.mojo:263-320),
reverse_complement (methylgrapher/src/utility.mojo:28-49)."""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from mojoalign_b200.linear_fm import (canonical_contig, fm_prefix_from_ref, hit_from_fm, hit_to_sam_line,
                                      pair_hits, reverse_complement, sam_header, select_device)

NAMES = ["rchr1", "fchr1", "rchr2", "fchr2"]


def test_canonical_contig_and_revcomp():
    assert canonical_contig("fchr1") == "chr1" and canonical_contig("rchrX") == "chrX"
    assert canonical_contig("chr1") == "chr1"  # only a leading f or r is stripped
    assert canonical_contig("X") == "X"
    assert reverse_complement("ACGTN") == "NACGT"
    assert reverse_complement("acgt") == "NNNN"  # lower case is not complemented


def test_hit_records():
    h = hit_from_fm(NAMES, "r1", "ATGT", "ACGT", 1, 99, 60, 0, 0, 0)
    assert (h.flag, h.contig, h.pos, h.mapq, h.cigar, h.seq) == (0, "chr1", 100, 60, "4M", "ACGT")
    h = hit_from_fm(NAMES, "r1", "ATGTAA", "ACGTAA", 3, 9, 20, 16, 1, 2)
    assert (h.cigar, h.seq, h.pos, h.contig) == ("1S3M2S", "TTACGT", 10, "chr2")
    u = hit_from_fm(NAMES, "r1", "ATGT", "ACGT", -1, 0, 0, 4, 0, 0)
    assert hit_to_sam_line(u) == "r1\t4\t*\t0\t0\t*\t*\t0\t0\tACGT\t*"
    z = hit_from_fm(NAMES, "r1", "AT", "AC", 0, 5, 20, 0, 1, 1)  # nothing aligned
    assert z.flag == 4 and z.contig == "*"


def test_pair_flags_and_tlen():
    a = hit_from_fm(NAMES, "p", "A" * 10, "A" * 10, 1, 99, 60, 0, 0, 0)
    b = hit_from_fm(NAMES, "p", "T" * 8, "T" * 8, 0, 199, 60, 16, 0, 0)  # r/f of the same chromosome
    p1, p2 = pair_hits(a, b)
    assert (p1.flag, p2.flag) == (1 | 64 | 2, 1 | 128 | 2 | 16)
    assert (p1.rnext, p1.pnext, p1.tlen) == ("=", 200, 108)
    assert (p2.rnext, p2.pnext, p2.tlen) == ("=", 100, -108)
    u = hit_from_fm(NAMES, "p", "T" * 8, "T" * 8, -1, 0, 0, 4, 0, 0)
    q1, q2 = pair_hits(a, u)
    assert (q1.flag, q2.flag) == (1 | 64 | 8, 4 | 1 | 128)
    assert (q2.rnext, q2.pnext, q1.rnext, q1.pnext) == ("chr1", 100, "*", 0)


def test_header_and_prefix(tmp_path):
    cs = [SimpleNamespace(name=n, length=100 + i) for i, n in enumerate(NAMES)]
    h = sam_header(cs, {"METHYLGRAPHER_RG_ID": "rg7"}).splitlines()
    assert h[0] == "@HD\tVN:1.6\tSO:unsorted"
    assert h[1:3] == ["@SQ\tSN:chr1\tLN:100", "@SQ\tSN:chr2\tLN:102"]
    assert h[3] == "@RG\tID:rg7\tSM:sample\tLB:lib1\tPL:ILLUMINA\tPU:rg7"
    fa = tmp_path / "ref.fa"
    with pytest.raises(RuntimeError):
        fm_prefix_from_ref(fa)
    (tmp_path / "ref.fa.bwameth.c2t.bwt").write_bytes(b"")
    assert fm_prefix_from_ref(fa).endswith(".bwameth.c2t")
    with pytest.raises(RuntimeError):
        select_device("cpu")
    assert select_device("auto") == 0
