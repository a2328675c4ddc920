"""Device SAM text (ma_emit_sam_batch[_device]) and the FASTQ split under the
SAM path's reader rules (ma_fastq_parse_rules[_device], rules 1) against the
oracle: every byte, count and error identical."""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from fastq_cases import random_fastq
from mojoalign_b200 import GpuContext, MojoAlignError
from mojoalign_b200 import _lib
from mojoalign_b200.sam import HIT_FIELDS, SamContigs, emit_sam_device, emit_sam_from_batch, sam_bound
from sam_batches import CONTIGS, oracle_arena, random_sam_batch

pytestmark = pytest.mark.gpu

KEYS = ("name_off", "name_len", "seq_off", "seq_len", "qual_off", "qual_len")
GOLDEN = Path(__file__).resolve().parent / "golden" / "fastq_pair_reader.json"


@pytest.fixture(scope="module")
def ctx():
    c = GpuContext(0)
    yield c
    c.close()


@pytest.mark.parametrize("paired", [False, True])
@pytest.mark.parametrize("seed,n1", [(1, 1), (2, 7), (3, 1000), (4, 40000)])
def test_batch_matches_oracle(ctx, seed, n1, paired):
    hits, arena, _ = random_sam_batch(seed, n1, paired)
    want, want_mapped = oracle.emit_sam(hits, n1, paired, oracle_arena(arena), CONTIGS, b"mojo1")
    got, mapped = emit_sam_from_batch(ctx, hits, n1, paired, arena, SamContigs.from_names(CONTIGS), b"mojo1")
    assert got == want
    assert mapped == want_mapped


def test_all_unmapped_all_mapped_and_empty_rg(ctx):
    for frac, rg in ((0.0, b"r"), (1.0, b"")):
        hits, arena, _ = random_sam_batch(11, 3000, True, mapped_frac=frac)
        want = oracle.emit_sam(hits, 3000, True, oracle_arena(arena), CONTIGS, rg)
        assert emit_sam_from_batch(ctx, hits, 3000, True, arena, SamContigs.from_names(CONTIGS), rg) == want
    hits, arena, _ = random_sam_batch(12, 0, True)
    assert emit_sam_from_batch(ctx, hits, 0, True, arena, SamContigs.from_names(CONTIGS), b"r") == (b"", 0)


def _dev(a, dev):
    import torch

    a = np.ascontiguousarray(a)
    signed = {np.dtype(np.uint64): np.int64, np.dtype(np.uint32): np.int32}
    if a.dtype in signed:
        a = a.view(signed[a.dtype])
    return torch.from_numpy(a.copy()).to(dev)


def test_device_form_at_every_alignment(ctx):
    import torch

    n1, paired = 2500, True
    hits, arena, _ = random_sam_batch(21, n1, paired)
    want, want_mapped = oracle.emit_sam(hits, n1, paired, oracle_arena(arena), CONTIGS, b"grp")
    dev = torch.device("cuda", 0)
    d_h = {k: _dev(np.asarray(hits[k], dt), dev) for k, dt in HIT_FIELDS}
    hc = _lib.ma_hits(*[d_h[k].data_ptr() for k, _ in HIT_FIELDS])
    d_a = {k: _dev(getattr(arena, k), dev) for k in ("data", "name_off", "name_len", "orig_off", "orig_len",
                                                     "qual_off", "qual_len")}
    ac = _lib.ma_fastq_arena(d_a["data"].data_ptr(), int(arena.data.size), d_a["name_off"].data_ptr(),
                             d_a["name_len"].data_ptr(), d_a["orig_off"].data_ptr(), d_a["orig_len"].data_ptr(),
                             d_a["qual_off"].data_ptr(), d_a["qual_len"].data_ptr())
    contigs = SamContigs.from_names(CONTIGS).to_device(torch, dev)
    d_rg = torch.frombuffer(bytearray(b"grp"), dtype=torch.uint8).to(dev)
    for shift in (0, 1, 7, 15):
        d_out = torch.zeros(len(want) + 64, dtype=torch.uint8, device=dev)
        d_status = torch.zeros(3, dtype=torch.int64, device=dev)
        torch.cuda.synchronize()
        emit_sam_device(ctx, hc, n1, paired, ac, contigs, d_rg.data_ptr(), 3, d_out.data_ptr() + shift, len(want),
                        d_status.data_ptr())
        torch.cuda.synchronize()
        st = d_status.cpu().numpy()
        assert (st[0], st[1], st[2]) == (len(want), want_mapped, 0)
        out = d_out.cpu().numpy()
        assert out[shift:shift + len(want)].tobytes() == want
        assert not out[:shift].any() and not out[shift + len(want):].any()
    # one byte short: nothing written, the size and the overflow bit reported
    d_out = torch.zeros(len(want), dtype=torch.uint8, device=dev)
    d_status = torch.zeros(3, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    emit_sam_device(ctx, hc, n1, paired, ac, contigs, d_rg.data_ptr(), 3, d_out.data_ptr(), len(want) - 1,
                    d_status.data_ptr())
    torch.cuda.synchronize()
    st = d_status.cpu().numpy()
    assert st[0] == len(want) and st[2] == 1
    assert not d_out.cpu().numpy().any()
    # an arena span past the arena: error bit 8, nothing written
    bad_off = d_a["qual_off"].clone()
    bad_off[17] = int(arena.data.size)
    ac_bad = _lib.ma_fastq_arena(d_a["data"].data_ptr(), int(arena.data.size), d_a["name_off"].data_ptr(),
                                 d_a["name_len"].data_ptr(), d_a["orig_off"].data_ptr(), d_a["orig_len"].data_ptr(),
                                 bad_off.data_ptr(), d_a["qual_len"].data_ptr())
    if int(arena.qual_len[17]):
        d_out = torch.zeros(len(want), dtype=torch.uint8, device=dev)
        torch.cuda.synchronize()
        emit_sam_device(ctx, hc, n1, paired, ac_bad, contigs, d_rg.data_ptr(), 3, d_out.data_ptr(), len(want),
                        d_status.data_ptr())
        torch.cuda.synchronize()
        assert d_status.cpu().numpy()[2] & 8
        assert not d_out.cpu().numpy().any()


def test_errors_match_oracle(ctx):
    hits, arena, _ = random_sam_batch(31, 200, True, odd_text=0.0)
    contigs = SamContigs.from_names(CONTIGS)
    want, _ = oracle.emit_sam(hits, 200, True, oracle_arena(arena), CONTIGS, b"x")
    with pytest.raises(MojoAlignError, match="SAM batch buffer overflow"):
        emit_sam_from_batch(ctx, hits, 200, True, arena, contigs, b"x", cap=len(want) - 1)
    assert emit_sam_from_batch(ctx, hits, 200, True, arena, contigs, b"x", cap=len(want))[0] == want
    assert len(want) <= sam_bound(vars(arena), 400, contigs, 1)
    bad = dict(hits, rid=hits["rid"].copy())
    bad["rid"][5] = len(CONTIGS) + 2
    with pytest.raises(MojoAlignError, match="rid outside"):
        emit_sam_from_batch(ctx, bad, 200, True, arena, contigs, b"x")
    for seq_side in (False, True):
        a2 = type(arena)(**vars(arena))
        a2.data = arena.data.copy()
        r = int(np.argmax(arena.orig_len if seq_side else arena.qual_len))
        off = int((arena.orig_off if seq_side else arena.qual_off)[r])
        a2.data[off] = 0xc3  # a lead byte without its continuation (next byte is ASCII)
        with pytest.raises(RuntimeError, match="not valid UTF-8"):
            oracle.emit_sam(hits, 200, True, oracle_arena(a2), CONTIGS, b"x")
        with pytest.raises(MojoAlignError, match="not valid UTF-8"):
            emit_sam_from_batch(ctx, hits, 200, True, a2, contigs, b"x")


def _parse(ctx, text: bytes, at_eof=True, max_records=None, base=0, rules=1):
    b = np.frombuffer(text, np.uint8)
    cap = len(text) // 4 + 2 if max_records is None else max_records
    out = {k: np.zeros(max(cap, 1), np.uint64 if k.endswith("off") else np.uint32) for k in KEYS}
    rec = _lib.ma_fastq_records(*[out[k].ctypes.data for k in KEYS])
    o3 = (C.c_uint64 * 3)()
    _lib.check(_lib.lib.ma_fastq_parse_rules(ctx.handle, b.ctypes.data if b.size else None, b.size, int(at_eof), cap,
                                             base, rules, C.byref(rec), o3), ctx.handle)
    n = o3[0]
    res = {k: v[:n] for k, v in out.items()}
    res.update(n=n, consumed=o3[1], max_len=o3[2])
    return res


def _same(a, b):
    assert (a["n"], a["consumed"], a["max_len"]) == (b["n"], b["consumed"], b["max_len"])
    for k in KEYS:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_pair_reader_split_matches_oracle(ctx):
    for c in json.loads(GOLDEN.read_text())["cases"]:
        for raw in (c["r1"], c["r2"]):
            if raw is None:
                continue
            text = bytes.fromhex(raw)
            _same(_parse(ctx, text), oracle.fastq_parse_pr(text))
            for cut in range(0, len(text) + 1, max(1, len(text) // 23)):
                _same(_parse(ctx, text[:cut], at_eof=False, base=9),
                      oracle.fastq_parse_pr(text[:cut], at_eof=False, base=9))
                _same(_parse(ctx, text[:cut]), oracle.fastq_parse_pr(text[:cut]))
    for seed, n in ((1, 3), (2, 5000), (3, 200_000)):
        for terminated in (True, False):
            text = random_fastq(seed, n, terminated=terminated, crlf=0.3)
            _same(_parse(ctx, text), oracle.fastq_parse_pr(text))
            for mr in (1, n // 3 + 1):
                _same(_parse(ctx, text, max_records=mr), oracle.fastq_parse_pr(text, max_records=mr))


def test_pair_reader_split_device_form(ctx):
    import torch

    text = random_fastq(7, 30_000, crlf=0.5, terminated=False)
    want = oracle.fastq_parse_pr(text)
    dev = torch.device("cuda", 0)
    n = want["n"]
    d_buf = torch.zeros(len(text) + 32, dtype=torch.uint8, device=dev)
    d_buf[3:3 + len(text)] = torch.frombuffer(bytearray(text), dtype=torch.uint8).to(dev)
    d_out = {k: torch.zeros(n + 5, dtype=torch.int64 if k.endswith("off") else torch.int32, device=dev) for k in KEYS}
    rec = _lib.ma_fastq_records(*[d_out[k].data_ptr() for k in KEYS])
    o3 = (C.c_uint64 * 3)()
    torch.cuda.synchronize()
    _lib.check(_lib.lib.ma_fastq_parse_rules_device(ctx.handle, d_buf.data_ptr() + 3, len(text), 1, n + 5, 0, 1,
                                                    C.byref(rec), o3, None), ctx.handle)
    assert (o3[0], o3[1], o3[2]) == (n, want["consumed"], want["max_len"])
    for k in KEYS:
        got = d_out[k].cpu().numpy().view(np.uint64 if k.endswith("off") else np.uint32)[:n]
        np.testing.assert_array_equal(got, want[k], err_msg=k)
    with pytest.raises(MojoAlignError, match="unknown FASTQ rules"):
        _parse(ctx, b"@a\nA\n+\nI\n", rules=2)
