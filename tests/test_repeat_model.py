"""The repeat-heavy reference model and the oracle's view of it (CPU).

The repeat-heavy configuration asks for a reference with 45% of its bases in
copies of 300 bp and 6 kb family elements at 10-20% divergence plus 3%
low-complexity tandem runs, and for bit-exact multi-hit tie-breaking where
seeds have many occurrences: the reference's max_occ stop
(fq2bam-meth/src/linear_gpu_fm.mojo:1378-1379) and its <= 16-row fallback
(L1374-1385).  These tests check that the generator is deterministic, that it
puts the repeats there, and that reads on it drive the oracle through both
rules, so that the GPU parity tests on these references cover them.
"""
from __future__ import annotations

import collections

import numpy as np

import oracle
from mojoalign_b200 import BENCH_PARAMS, synth


def _seq(fa):
    return "".join(ln.strip() for ln in open(fa) if not ln.startswith(">"))


def test_generator_is_deterministic_and_sized(tmp_path):
    rm = synth.RepeatModel(families=8)
    a, b, c = tmp_path / "a.fa", tmp_path / "b.fa", tmp_path / "c.fa"
    synth.write_reference_model(a, 400_000, n_contigs=3, seed=9, repeats=rm)
    synth.write_reference_model(b, 400_000, n_contigs=3, seed=9, repeats=rm)
    synth.write_reference_model(c, 400_000, n_contigs=3, seed=10, repeats=rm)
    assert a.read_bytes() == b.read_bytes()
    assert a.read_bytes() != c.read_bytes()
    s = _seq(a)
    assert len(s) == 400_000 and set(s) <= set("ACGT")
    gc = (s.count("G") + s.count("C")) / len(s)
    assert 0.36 < gc < 0.46


def _multi_kmer_share(s, k=24):
    cnt = collections.Counter(s[i:i + k] for i in range(len(s) - k + 1))
    return sum(1 for i in range(len(s) - k + 1) if cnt[s[i:i + k]] > 1) / (len(s) - k + 1), cnt


def test_repeats_are_present_and_contigs_independent(tmp_path):
    plain, rep = tmp_path / "p.fa", tmp_path / "r.fa"
    synth.write_reference_model(plain, 600_000, n_contigs=4, seed=1)
    synth.write_reference_model(rep, 600_000, n_contigs=4, seed=1,
                                repeats=synth.RepeatModel(families=4, div_min=0.01, div_max=0.03))
    # contigs drawn from independent streams: no shared 24-mers by chance
    share_plain, _ = _multi_kmer_share(_seq(plain))
    assert share_plain < 0.001
    # young copies (1-3% divergence) keep most 24-mers of their family
    share_rep, cnt = _multi_kmer_share(_seq(rep))
    assert share_rep > 0.2
    # tandem runs give low-complexity k-mers with many occurrences
    assert cnt.most_common(1)[0][1] > 100


def test_oracle_hits_the_cap_and_the_fallback(repeat_ref, young_repeat_ref):
    for fa, prefix in (repeat_ref, young_repeat_ref):
        rb = synth.simulate_reads(fa, synth.ReadModel(len_fixed=250, conv_non_cpg=0.97), 4000, True, 250, seed=3)
        out = oracle.OracleIndex(prefix).map(rb.bases, rb.lens, rb.n1, True, 250, 1, 2, BENCH_PARAMS.as_list(),
                                             counters=True)
        ct = out["counters"]
        assert ct["capped"] > 0, ct
        assert ct["fallback"] > 0, ct
        # multi-row winners: the reported SA interval has several rows
        rows = out["ul"].astype(np.int64) - out["uk"].astype(np.int64) + 1
        assert ((out["rid"] >= 0) & (rows > 1)).any()
