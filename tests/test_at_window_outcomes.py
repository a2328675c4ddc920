"""The A/T window outcome table's exactness argument, on the CPU.

The kernels replace the backward search over an endpoint's last at_k bases,
when they are all A or T, by one table entry computed without max_occ at
index preparation (build_atw_kernel in csrc/device_index.cu), and apply
max_occ at run time (search_start in csrc/seed_core.cuh).  This test
restates both halves in Python over the oracle's Occ and checks, for every
A/T window of a small index and for windows inside random reads, that the
result is the reference's own search from that endpoint
(fq2bam-meth/src/linear_gpu_fm.mojo:1235-1385, restated in
oracle/oracle_fm.c seed_extend_one): the same seed interval and start, or no
seed, for several seed lengths and max_occ values, max_occ below 16
included.  Integer work: the tolerance is zero.
"""
from __future__ import annotations

import itertools

import numpy as np
import pytest

import oracle

A, T = 0, 3
COUNT_CAP = (1 << 29) - 1


def step(ix, k, l, c):
    ok = ix.occ(k - 1, c) if k else 0
    ol = ix.occ(l, c)
    return ix.L2[c] + ok + 1, ix.L2[c] + ol


def reference_search(ix, codes, e, sl, max_occ):
    """The seed of endpoint e: (k, l, s) or None (L1235-1385)."""
    k, l, s = 0, ix.seq_len, e
    last = None
    while s >= 0:
        c = int(codes[s])
        if c > 3:
            break
        k, l = step(ix, k, l, c)
        if k > l:
            break
        n, mlen = l - k + 1, e - s + 1
        if n == 1 and mlen >= sl:
            return (k, l, s)
        if n <= 16 and mlen >= sl:
            last = (k, l, s)
        if n > max_occ and mlen >= sl:
            break
        s -= 1
    return last


def table_entry(ix, window, sl):
    """build_atw_kernel: (kind, k, n, o, c_sl) of an A/T window (codes,
    first base first), the search over it with no max_occ stop."""
    K = len(window)
    k, l, c_sl = 0, ix.seq_len, 0
    kept = None
    for t in range(K):
        k, l = step(ix, k, l, int(window[K - 1 - t]))
        mlen = t + 1
        if k > l:
            return (1, kept[0], kept[1], kept[2], c_sl) if kept else (0, 0, 0, 0, c_sl)
        rows = l - k + 1
        if mlen == sl:
            c_sl = min(rows, COUNT_CAP)
        if mlen >= sl:
            if rows == 1:
                return (1, k, 1, mlen - 1, c_sl)
            if rows <= 16:
                kept = (k, rows, mlen - 1)
    return (2, k, l - k + 1, 0, c_sl)


def table_search(ix, codes, e, sl, max_occ, K, entry):
    """search_start's table path, then the ordinary steps of a continued
    search; None where the kernel takes the ordinary path from the start."""
    kind, k, n, o, c_sl = entry
    if c_sl > max_occ:
        return "steps" if c_sl <= 16 else None
    if kind == 0:
        return None
    if kind == 1:
        return (k, k + n - 1, e - o)
    l = k + n - 1
    s0 = e - K + 1
    last = (k, l, s0) if n <= 16 else None
    s = s0 - 1
    while s >= 0:
        c = int(codes[s])
        if c > 3:
            break
        k, l = step(ix, k, l, c)
        if k > l:
            break
        rows = l - k + 1
        if rows == 1:
            return (k, l, s)
        if rows <= 16:
            last = (k, l, s)
        if rows > max_occ:
            break
        s -= 1
    return last


def _check(ix, codes, e, sl, max_occ, K, cache):
    win = tuple(int(x) for x in codes[e - K + 1:e + 1])
    if win not in cache:
        cache[win] = table_entry(ix, win, sl)
    got = table_search(ix, codes, e, sl, max_occ, K, cache[win])
    if got == "steps":
        return 0
    assert got == reference_search(ix, codes, e, sl, max_occ), (win, e, sl, max_occ)
    return 1


@pytest.fixture(scope="module")
def ix(small_ref):
    return oracle.OracleIndex(small_ref[1])


@pytest.mark.parametrize("sl,K", [(8, 8), (8, 12), (10, 13)])
@pytest.mark.parametrize("max_occ", [1, 5, 16, 4096])
def test_every_window_alone(ix, sl, K, max_occ):
    """Every A/T window of K bases as a whole read (endpoint at its end)."""
    cache = {}
    used = 0
    for bits in itertools.product((A, T), repeat=K):
        codes = np.array(bits, np.uint8)
        used += _check(ix, codes, K - 1, sl, max_occ, K, cache)
    assert used > 0


@pytest.mark.parametrize("sl,K,max_occ", [(10, 14, 500), (11, 16, 8), (12, 18, 40), (9, 16, 3)])
def test_windows_inside_reads(ix, sl, K, max_occ):
    """A/T windows inside longer reads: the continued search steps past the
    window, through A/T bases, other bases and N, to the read start."""
    rng = np.random.default_rng(sl * 100 + K)
    ref = np.array([ix.pac_base(p) for p in range(0, 60000)], np.uint8)
    cache = {}
    used = 0
    for i in range(400):
        n = int(rng.integers(K, 90))
        if i % 2:  # text copied from the forward strand with A/T substituted in
            p = int(rng.integers(0, ref.size - n))
            codes = ref[p:p + n].copy()
            codes[rng.random(n) < 0.8] = A
        else:
            codes = rng.choice(np.array([A, T], np.uint8), n)
        codes[rng.random(n) < 0.02] = 4
        for e in range(K - 1, n):
            w = codes[e - K + 1:e + 1]
            if np.all((w == A) | (w == T)):
                used += _check(ix, codes, e, sl, max_occ, K, cache)
    assert used > 100
