"""GPU BAM packing (ma_emit_bam_batch / ma_emit_bam_batch_device) against
the oracle's _emit_bam_from_batch restatement: record bytes, every metadata
array and the tile counters must be identical."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from bam_batches import RID_TO_TID, bam_cap_for, random_batch
from mojoalign_b200 import GpuContext, MojoAlignError
from mojoalign_b200.bam import META_FIELDS, BamTile, emit_bam_from_batch, emit_bam_device

pytestmark = pytest.mark.gpu

RG = b"mojo1"


@pytest.fixture(scope="module")
def ctx():
    c = GpuContext(0)
    yield c
    c.close()


def _check(ctx, seed, n1, paired, *, n_reads=0, n_total=0, chunk=0, **kw):
    hits, arena, _ = random_batch(seed, n1, paired, **kw)
    n_seq = arena.n_seq
    cap = bam_cap_for(arena, len(RG))
    want, want_meta, want_mapped = oracle.emit_bam(hits, vars(arena), n1, paired, RID_TO_TID, RG, n_reads=n_reads,
                                                   n_total=n_total, meta_cap=n_reads + n_seq, chunk=chunk, cap=cap)
    tile = BamTile(meta_cap=n_reads + n_seq, n_reads=n_reads, n_mapped=7, n_total=n_total, chunk=chunk)
    got = emit_bam_from_batch(ctx, hits, n1, paired, arena, RID_TO_TID, RG, tile, cap)
    assert got.tobytes() == want
    for k, _ in META_FIELDS:
        np.testing.assert_array_equal(tile.meta[k][n_reads:], want_meta[k], err_msg=k)
    assert tile.n_reads == n_reads + n_seq and tile.n_mapped == 7 + want_mapped
    return hits, arena, want, want_meta


@pytest.mark.parametrize("paired", [False, True])
@pytest.mark.parametrize("seed,n1", [(1, 1), (2, 7), (3, 1000), (4, 40000)])
def test_batch_matches_oracle(ctx, seed, n1, paired):
    _check(ctx, seed, n1, paired)


def test_tile_continuation_and_chunk(ctx):
    _check(ctx, 11, 3000, True, n_reads=12345, n_total=10 ** 9 + 7, chunk=5)
    _check(ctx, 12, 3000, False, n_reads=999, n_total=(1 << 32) + 3, chunk=(1 << 32) - 1)


def test_long_records_take_the_unstaged_path(ctx):
    _check(ctx, 21, 500, True, long_frac=0.2)
    _check(ctx, 22, 300, False, long_frac=1.0)


def test_without_qualities(ctx):
    _check(ctx, 31, 2000, True, with_quals=False)


def test_all_unmapped_and_all_mapped(ctx):
    _check(ctx, 41, 1500, True, mapped_frac=0.0)
    _check(ctx, 42, 1500, True, mapped_frac=1.0)


def _dev(a, dev):
    """numpy -> device tensor of the same bytes (unsigned views as signed)."""
    import torch

    a = np.ascontiguousarray(a)
    signed = {np.dtype(np.uint64): np.int64, np.dtype(np.uint32): np.int32}
    if a.dtype in signed:
        a = a.view(signed[a.dtype])
    return torch.from_numpy(a).to(dev)


def test_device_form_at_every_alignment(ctx):
    import torch

    n1, paired = 2500, True
    hits, arena, want, want_meta = _check(ctx, 51, n1, paired)
    dev = torch.device("cuda", 0)
    d_hits = {k: _dev(v, dev) for k, v in hits.items()}
    d_arena = {k: _dev(getattr(arena, k), dev)
               for k in ("data", "name_off", "name_len", "orig_off", "orig_len", "qual_off", "qual_len")}
    d_tids = torch.from_numpy(RID_TO_TID).to(dev)
    d_rg = torch.frombuffer(bytearray(RG), dtype=torch.uint8).to(dev)
    n_seq = arena.n_seq
    for shift in (0, 1, 7, 15):
        d_bam = torch.zeros(len(want) + 64, dtype=torch.uint8, device=dev)
        d_meta = {k: torch.zeros(n_seq + 3, dtype=torch.int64 if t == np.uint64 else torch.int32, device=dev)
                  for k, t in META_FIELDS}
        d_status = torch.zeros(3, dtype=torch.int64, device=dev)
        tile = BamTile(meta_cap=n_seq + 3, n_reads=3)
        torch.cuda.synchronize()  # the buffers were zeroed on torch's stream
        emit_bam_device(ctx, {k: v.data_ptr() for k, v in d_hits.items()}, n1, paired,
                        {k: v.data_ptr() for k, v in d_arena.items()}, int(arena.data.size), d_tids.data_ptr(),
                        int(RID_TO_TID.size), d_rg.data_ptr(), len(RG), d_bam.data_ptr() + shift, len(want),
                        {k: v.data_ptr() for k, v in d_meta.items()}, tile, d_status.data_ptr())
        torch.cuda.synchronize()
        status = d_status.cpu().numpy()
        assert status[0] == len(want) and status[2] == 0
        out = d_bam.cpu().numpy()
        assert out[shift:shift + len(want)].tobytes() == want
        assert not out[:shift].any() and not out[shift + len(want):].any()
        # the tile starts at 3 here: coord / dlo / pair of unplaced records
        # carry the tile index, so compare the offset-free arrays
        for k, t in META_FIELDS:
            if k in ("len", "score", "rec", "dhi"):
                got = d_meta[k].cpu().numpy().view(t)[3:]
                np.testing.assert_array_equal(got, want_meta[k], err_msg=k)
    # a buffer one byte short: nothing written, the total reported
    d_bam = torch.zeros(len(want), dtype=torch.uint8, device=dev)
    d_status = torch.zeros(3, dtype=torch.int64, device=dev)
    d_meta = {k: torch.zeros(n_seq, dtype=torch.int64 if t == np.uint64 else torch.int32, device=dev)
              for k, t in META_FIELDS}
    torch.cuda.synchronize()
    emit_bam_device(ctx, {k: v.data_ptr() for k, v in d_hits.items()}, n1, paired,
                    {k: v.data_ptr() for k, v in d_arena.items()}, int(arena.data.size), d_tids.data_ptr(),
                    int(RID_TO_TID.size), d_rg.data_ptr(), len(RG), d_bam.data_ptr(), len(want) - 1,
                    {k: v.data_ptr() for k, v in d_meta.items()}, BamTile(meta_cap=n_seq),
                    d_status.data_ptr())
    torch.cuda.synchronize()
    assert d_status.cpu().numpy()[0] == len(want)
    assert not d_bam.cpu().numpy().any()


def test_errors_leave_the_tile_unchanged(ctx):
    hits, arena, _ = random_batch(61, 100, True)
    cap = bam_cap_for(arena, len(RG))
    tile = BamTile(meta_cap=199, n_reads=0)
    with pytest.raises(MojoAlignError, match="FM sort cap exceeded"):
        emit_bam_from_batch(ctx, hits, 100, True, arena, RID_TO_TID, RG, tile, cap)
    assert tile.n_reads == 0 and tile.n_mapped == 0
    want, _, _ = oracle.emit_bam(hits, vars(arena), 100, True, RID_TO_TID, RG, cap=cap)
    tile = BamTile(meta_cap=200)
    with pytest.raises(MojoAlignError, match="BAM batch buffer overflow"):
        emit_bam_from_batch(ctx, hits, 100, True, arena, RID_TO_TID, RG, tile, len(want) - 1)
    assert tile.n_reads == 0
    assert emit_bam_from_batch(ctx, hits, 100, True, arena, RID_TO_TID, RG, tile, len(want)).tobytes() == want
    bad = random_batch(62, 10, False)[1]
    bad.orig_off[3] = bad.data.size + 1
    with pytest.raises(MojoAlignError, match="outside the arena"):
        emit_bam_from_batch(ctx, random_batch(62, 10, False)[0], 10, False, bad, RID_TO_TID, RG, BamTile(meta_cap=10),
                            10 ** 6)
    empty = emit_bam_from_batch(ctx, hits, 0, True, arena, RID_TO_TID, RG, BamTile(meta_cap=0), 0)
    assert empty.size == 0
