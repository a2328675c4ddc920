"""GPU coordinate sort + duplicate marking (ma_sort_markdup[_device]) and the
sorted record gather (ma_gather_sorted_bam[_device]) against the oracle's
restatement of gpu_sort_markdup / _gather_perm_to_writer: every output
identical."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from bam_batches import RID_TO_TID, bam_cap_for, random_batch, random_tile_meta
from mojoalign_b200 import GpuContext, MojoAlignError
from mojoalign_b200 import _lib
from mojoalign_b200.bam import BamTile, SortResult, emit_bam_from_batch, gather_sorted, sort_markdup

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = GpuContext(0)
    yield c
    c.close()


def _tile(m):
    n = m["coord"].size
    t = BamTile(meta_cap=n, n_reads=n)
    for k, v in m.items():
        t.meta[k][:] = v
    return t


@pytest.mark.parametrize("seed,n", [(1, 1), (2, 2), (3, 255), (4, 257), (5, 100_003), (6, 3_000_001)])
@pytest.mark.parametrize("do_markdup", [True, False])
def test_sort_markdup_matches_oracle(ctx, seed, n, do_markdup):
    m = random_tile_meta(seed, n, dup_rate=0.4)
    want = oracle.sort_markdup(**m, do_markdup=do_markdup)
    got = sort_markdup(ctx, _tile(m), do_markdup=do_markdup, dup_perm=True)
    np.testing.assert_array_equal(got.perm, want[1])
    np.testing.assert_array_equal(got.is_dup, want[0])
    np.testing.assert_array_equal(got.dup_perm, want[2])
    assert got.n_marked == want[3]


def _key_pattern(kind, n, rng):
    if kind == "all_equal":        # no digit varies: the input is copied
        return np.full(n, 0x0123456789ABCDEF, np.uint64)
    if kind == "one_digit":        # one active pass
        return (np.uint64(0x5500000000000000) | (rng.integers(0, 256, n, dtype=np.uint64) << np.uint64(24)))
    if kind == "top_bits":         # the sign bit and the top digit
        return rng.integers(0, 4, n, dtype=np.uint64) << np.uint64(62)
    if kind == "few_values":       # long runs of equal keys (stability)
        return rng.integers(0, 7, n, dtype=np.uint64) * np.uint64(0x0101010101010101)
    return rng.integers(0, 2**64 - 1, n, dtype=np.uint64, endpoint=True)  # every digit varies


@pytest.mark.parametrize("kind", ["all_equal", "one_digit", "top_bits", "few_values", "random"])
@pytest.mark.parametrize("n", [1, 4095, 4096, 4097, 1_000_003])
def test_coordinate_order_is_a_stable_sort(ctx, kind, n):
    """The radix passes give numpy's stable order for key patterns that
    skip no digit, some digits or all of them, at tile-size edges."""
    rng = np.random.default_rng(n)
    m = random_tile_meta(11, n, dup_rate=0.2)
    m["coord"] = _key_pattern(kind, n, rng)
    got = sort_markdup(ctx, _tile(m), do_markdup=True, dup_perm=True)
    np.testing.assert_array_equal(got.perm, np.argsort(m["coord"], kind="stable").astype(np.uint32))
    want = oracle.sort_markdup(**m, do_markdup=True)
    np.testing.assert_array_equal(got.is_dup, want[0])
    np.testing.assert_array_equal(got.dup_perm, want[2])


def test_deep_duplicate_group(ctx):
    n = 200_000
    m = random_tile_meta(7, n, dup_rate=0.0)
    m["dhi"][: n // 2] = (1 << 48) | 12345
    m["dlo"][: n // 2] = 77
    want = oracle.sort_markdup(**m)
    got = sort_markdup(ctx, _tile(m), dup_perm=True)
    np.testing.assert_array_equal(got.is_dup, want[0])
    np.testing.assert_array_equal(got.dup_perm, want[2])


def test_sort_markdup_device_form(ctx):
    import torch

    n = 500_000
    m = random_tile_meta(8, n)
    want = oracle.sort_markdup(**m)
    dev = torch.device("cuda", 0)
    d = {k: torch.from_numpy(v.view(np.int64 if v.dtype == np.uint64 else np.int32)).to(dev) for k, v in m.items()}
    out = {k: torch.zeros(n, dtype=torch.int32, device=dev) for k in ("is_dup", "perm", "dup_perm")}
    marked = torch.zeros(1, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    _lib.check(_lib.lib.ma_sort_markdup_device(
        ctx.handle, n, d["coord"].data_ptr(), d["dhi"].data_ptr(), d["dlo"].data_ptr(), d["score"].data_ptr(),
        d["pair"].data_ptr(), out["is_dup"].data_ptr(), out["perm"].data_ptr(), 1, out["dup_perm"].data_ptr(),
        marked.data_ptr(), None), ctx.handle)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out["perm"].cpu().numpy().view(np.uint32), want[1])
    np.testing.assert_array_equal(out["is_dup"].cpu().numpy().view(np.uint32), want[0])
    np.testing.assert_array_equal(out["dup_perm"].cpu().numpy().view(np.uint32), want[2])
    assert int(marked.item()) == want[3]


def test_map_emit_sort_gather_chain(ctx):
    """Three emitted batches (three chunks) of one tile, sorted, marked and
    gathered, against the same chain on the oracle."""
    rg = b"grp"
    tile = BamTile(meta_cap=3 * 2 * 4000)
    chunks, want_chunks = [], []
    want_meta = {k: [] for k in ("coord", "dhi", "dlo", "rec", "len", "score", "pair")}
    for c, seed in enumerate((31, 32, 33)):
        hits, arena, _ = random_batch(seed, 4000, True)
        cap = bam_cap_for(arena, len(rg))
        w, wm, _ = oracle.emit_bam(hits, vars(arena), 4000, True, RID_TO_TID, rg, n_reads=tile.n_reads,
                                   meta_cap=tile.meta_cap, chunk=c, cap=cap)
        tile.chunk = c
        got = emit_bam_from_batch(ctx, hits, 4000, True, arena, RID_TO_TID, rg, tile, cap)
        assert got.tobytes() == w
        chunks.append(got.copy())
        want_chunks.append(w)
        for k in want_meta:
            want_meta[k].append(wm[k])
    wm = {k: np.concatenate(v) for k, v in want_meta.items()}
    for k in wm:
        np.testing.assert_array_equal(tile.meta[k][: tile.n_reads], wm[k], err_msg=k)
    w_dup, w_perm, _, _ = oracle.sort_markdup(wm["coord"], wm["dhi"], wm["dlo"], wm["score"], wm["pair"])
    res = sort_markdup(ctx, tile)
    np.testing.assert_array_equal(res.perm, w_perm)
    np.testing.assert_array_equal(res.is_dup, w_dup)
    want = oracle.gather_sorted(want_chunks, w_perm, wm["rec"], wm["len"], w_dup)
    assert gather_sorted(ctx, chunks, tile, res).tobytes() == want
    plain = oracle.gather_sorted(want_chunks, w_perm, wm["rec"], wm["len"], w_dup, apply_dup=False)
    assert gather_sorted(ctx, chunks, tile, res, apply_dup=False).tobytes() == plain


def test_gather_rejects_out_of_range_records(ctx):
    hits, arena, _ = random_batch(41, 100, False)
    tile = BamTile(meta_cap=100)
    bam = emit_bam_from_batch(ctx, hits, 100, False, arena, RID_TO_TID, b"r", tile, bam_cap_for(arena, 1)).copy()
    res = SortResult(np.zeros(100, np.uint32), np.arange(100, dtype=np.uint32), None, 0)
    assert gather_sorted(ctx, [bam], tile, res).tobytes() == bam.tobytes()
    tile.meta["rec"][5] = (3 << 32)  # chunk 3 does not exist
    with pytest.raises(MojoAlignError, match="outside their chunks"):
        gather_sorted(ctx, [bam], tile, res)
    tile.meta["rec"][5] = len(bam) - 10  # span past the chunk end
    with pytest.raises(MojoAlignError, match="outside their chunks"):
        gather_sorted(ctx, [bam], tile, res)
