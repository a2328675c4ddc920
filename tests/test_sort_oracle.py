"""The sort / duplicate-marking / gather oracle (oracle/oracle_sort.c) on the
CPU: the orders it must produce are the stable sorts the reference's LSD
radix yields (fq2bam-meth/src/linear_gpu_sort.mojo:149-245), its results do
not depend on the tile size (L15-21, L372-408, L500-525), and the marking
follows the reference's Picard-style rule (L409-466)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from bam_batches import RID_TO_TID, random_batch, random_tile_meta, read_records


def test_orders_are_stable_sorts():
    m = random_tile_meta(1, 20001)
    is_dup, perm, dp, marked = oracle.sort_markdup(**m)
    n = m["coord"].size
    np.testing.assert_array_equal(perm, np.argsort(m["coord"], kind="stable"))
    np.testing.assert_array_equal(dp, np.lexsort((np.arange(n), m["dlo"], m["dhi"])))
    assert marked == int(is_dup.sum()) > 0


@pytest.mark.parametrize("tile", [1, 7, 256, 4097, 19999])
def test_tile_size_does_not_change_results(tile):
    m = random_tile_meta(2, 20001)
    full = oracle.sort_markdup(**m)
    tiled = oracle.sort_markdup(**m, tile=tile)
    for a, b in zip(full[:3], tiled[:3]):
        np.testing.assert_array_equal(a, b)


def test_marking_rule():
    # one group of three pairs (6 records) + an unplaced pair + a singleton
    k = (1 << 48) | 5
    dhi = np.array([k, k, k, k, k, k, 2**64 - 1, 2**64 - 1, k + 1], np.uint64)
    dlo = np.array([9, 9, 9, 9, 9, 9, 6, 6, 0], np.uint64)
    score = np.array([10, 10, 30, 30, 30, 30, 0, 0, 1], np.uint32)
    pair = np.array([4, 4, 8, 8, 6, 6, 3, 3, 2], np.uint32)
    coord = np.arange(9, dtype=np.uint64)[::-1].copy()
    is_dup, perm, dp, marked = oracle.sort_markdup(coord, dhi, dlo, score, pair)
    # best score 30; tie between pairs 8 and 6 -> lowest pair id (6) kept
    assert list(is_dup) == [1, 1, 1, 1, 0, 0, 0, 0, 0] and marked == 4
    assert list(perm) == list(range(8, -1, -1))
    off = oracle.sort_markdup(coord, dhi, dlo, score, pair, do_markdup=False)
    assert not off[0].any() and list(off[2]) == list(range(9)) and off[3] == 0


def test_gather_and_duplicate_flag():
    hits, arena, _ = random_batch(5, 300, True)
    bam, meta, _ = oracle.emit_bam(hits, vars(arena), 300, True, RID_TO_TID, b"rg", cap=10**7)
    n = 600
    is_dup, perm, _, _ = oracle.sort_markdup(meta["coord"], meta["dhi"], meta["dlo"], meta["score"], meta["pair"])
    out = oracle.gather_sorted([bam], perm, meta["rec"], meta["len"], is_dup)
    recs = read_records(out)
    assert len(recs) == n and len(out) == len(bam)
    by_off = {int(r & 0xFFFFFFFF): i for i, r in enumerate(meta["rec"])}
    src = read_records(bam)
    for j, r in enumerate(recs):
        o = int(perm[j])
        assert by_off[src[o]["off"]] == o
        want_flag = src[o]["flag"] | (1024 if is_dup[o] else 0)
        assert r["flag"] == want_flag
    sc = meta["coord"][perm]
    assert (sc[1:] >= sc[:-1]).all()
    plain = oracle.gather_sorted([bam], perm, meta["rec"], meta["len"], is_dup, apply_dup=False)
    assert [r["flag"] for r in read_records(plain)] == [src[int(o)]["flag"] for o in perm]
