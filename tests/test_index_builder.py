"""Index builder output against brute force, and the reference's FM round trip.

The builder writes bwa 0.7 files that the oracle reads with its own parser
(a restatement of FmIndex.load, fq2bam-meth/src/linear_fm_index.mojo:88-175).
Bit-identity with files written by bwa itself cannot be checked here (bwa and
bwa-meth are absent); these tests pin the suffix array, BWT, counts, pac and
.ann contents against their definitions instead.
"""
from __future__ import annotations

import struct

import numpy as np
import pytest

import oracle
from mojoalign_b200 import MojoAlignError, build_index

COMP = {0: 3, 1: 2, 2: 1, 3: 0}
NT = {"A": 0, "C": 1, "G": 2, "T": 3}


def bwameth_text(contigs):
    recs = []
    for name, s in contigs:
        s = s.upper()
        recs.append(("r" + name, s.replace("G", "A")))
        recs.append(("f" + name, s.replace("C", "T")))
    return recs


def naive_index(recs):
    fwd = [NT[c] for _, s in recs for c in s]
    text = fwd + [COMP[c] for c in reversed(fwd)]
    n = len(text)
    sa = sorted(range(n + 1), key=lambda i: text[i:] + [-1])  # sentinel smallest
    return fwd, text, sa


def decode_bwt(prefix, seq_len):
    raw = open(str(prefix) + ".bwt", "rb").read()
    primary, *l2 = struct.unpack("<5Q", raw[:40])
    words = np.frombuffer(raw[40:], dtype="<u4")
    out = []
    for k in range(seq_len):
        w = words[((k >> 7) << 4) + 8 + ((k & 0x7F) >> 4)]
        out.append(int((w >> ((15 - (k & 15)) * 2)) & 3))
    return primary, [0] + l2, out, words


def write_fa(path, contigs):
    path.write_text("".join(f">{n} desc {i}\n{s}\n" for i, (n, s) in enumerate(contigs)))


CASES = [
    [("chr1", "ACGTACGTTTGACCA")],
    [("c1", "AAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAA"), ("c2", "ACACACACACACACACAC")],
    [("x", "GATTACA" * 9), ("y", "T"), ("z", "CCGGN" * 7)],
]


@pytest.mark.parametrize("contigs", CASES + ["random"])
@pytest.mark.parametrize("sa_intv", [1, 4, 32])
def test_builder_matches_definitions(tmp_path, contigs, sa_intv):
    if contigs == "random":
        rng = np.random.default_rng(sa_intv)
        contigs = [(f"r{i}", "".join(rng.choice(list("ACGT"), size=int(rng.integers(50, 300)))))
                   for i in range(4)]
    fa = tmp_path / "ref.fa"
    write_fa(fa, contigs)
    prefix = tmp_path / "ref.fa.bwameth.c2t"
    build_index(fa, prefix, bwameth_c2t=True, sa_intv=sa_intv)
    has_n = any("N" in s for _, s in contigs)
    recs = bwameth_text(contigs)
    ix = oracle.OracleIndex(prefix)
    l_pac = sum(len(s) for _, s in recs)
    assert ix.l_pac == l_pac and ix.seq_len == 2 * l_pac
    assert [c[0] for c in ix.contigs] == [r[0] for r in recs]
    assert [c[2] for c in ix.contigs] == [len(r[1]) for r in recs]
    # the bwameth text itself was written as the prefix FASTA
    txt = prefix.read_text().split(">")[1:]
    assert [t.split()[0] for t in txt] == [r[0] for r in recs]
    if has_n:
        # ambiguous bases become pseudo-random bases; use the pac as truth
        fwd = [ix.pac_base(i) for i in range(l_pac)]
        text = fwd + [COMP[c] for c in reversed(fwd)]
        n = len(text)
        sa = sorted(range(n + 1), key=lambda i: text[i:] + [-1])
    else:
        fwd, text, sa = naive_index(recs)
        assert [ix.pac_base(i) for i in range(l_pac)] == fwd
    n = len(text)
    primary, l2, bwt, words = decode_bwt(prefix, n)
    assert primary == sa.index(0) == ix.primary
    naive_bwt = [text[sa[i] - 1] for i in range(n + 1) if sa[i] != 0]
    assert bwt == naive_bwt
    for c in range(4):
        assert l2[c + 1] - l2[c] == text.count(c)
    # sampled SA
    raw = open(str(prefix) + ".sa", "rb").read()
    hdr = struct.unpack("<7Q", raw[:56])
    assert hdr[0] == primary and hdr[5] == sa_intv and hdr[6] == n
    samples = np.frombuffer(raw[56:], dtype="<u8")
    assert list(samples) == [sa[i * sa_intv] for i in range(1, (n + sa_intv) // sa_intv)]
    # Occ of the oracle (reference arithmetic) against direct counts
    rows = [text[sa[i] - 1] if sa[i] else -1 for i in range(n + 1)]
    for k in list(range(0, n + 1, max(1, n // 50))) + [n, primary, max(0, primary - 1)]:
        for c in range(4):
            assert ix.occ(k, c) == sum(1 for r in rows[: k + 1] if r == c), (k, c)
    # .pac tail bytes (bwa layout)
    pac = open(str(prefix) + ".pac", "rb").read()
    assert pac[-1] == l_pac % 4
    assert len(pac) == l_pac // 4 + 1 + 1


def test_match_exact_counts_against_brute_force(tmp_path):
    rng = np.random.default_rng(5)
    seq = "".join(rng.choice(list("ACGT"), size=400))
    fa = tmp_path / "ref.fa"
    write_fa(fa, [("chr1", seq + "ACGTACGTACGT" * 5)])
    prefix = tmp_path / "idx"
    build_index(fa, prefix, bwameth_c2t=False, sa_intv=8)
    ix = oracle.OracleIndex(prefix)
    fwd = [ix.pac_base(i) for i in range(ix.l_pac)]
    text = fwd + [COMP[c] for c in reversed(fwd)]
    for _ in range(200):
        L = int(rng.integers(1, 14))
        if rng.random() < 0.7:
            p = int(rng.integers(0, len(text) - L))
            pat = text[p:p + L]
        else:
            pat = [int(x) for x in rng.integers(0, 4, size=L)]
        want = sum(1 for i in range(len(text) - L + 1) if text[i:i + L] == pat)
        _, _, occ = ix.match_exact(pat)
        assert occ == want


def test_fm_roundtrip_property(small_ref):
    """fq2bam-meth/tests/fm_roundtrip.mojo:21-45 on the synthetic index, both strands."""
    _, prefix = small_ref
    ix = oracle.OracleIndex(prefix)
    rng = np.random.default_rng(0)
    seen = 0
    for _ in range(400):
        p = int(rng.integers(0, ix.l_pac - 32))
        fw = [ix.pac_base(p + i) for i in range(32)]
        for strand in (0, 1):
            pat = fw if strand == 0 else [COMP[c] for c in reversed(fw)]
            k, _, occ = ix.match_exact(pat)
            if occ != 1:
                continue
            seen += 1
            fpos, rev = ix.depos(ix.sa_at(k))
            assert rev == strand
            assert fpos == (p if strand == 0 else p + 31)
    assert seen > 600


def test_builder_errors(tmp_path):
    with pytest.raises(MojoAlignError) as e:
        build_index(tmp_path / "missing.fa", tmp_path / "x")
    assert e.value.code == -2
    fa = tmp_path / "a.fa"
    fa.write_text(">a\nACGT\n")
    with pytest.raises(MojoAlignError) as e:
        build_index(fa, tmp_path / "x", sa_intv=3)
    assert e.value.code == -1
    empty = tmp_path / "e.fa"
    empty.write_text("")
    with pytest.raises(MojoAlignError) as e:
        build_index(empty, tmp_path / "y")
    assert e.value.code == -3
