"""Device FASTQ record split (ma_fastq_parse[_device]) and row packing
(ma_fastq_rows_device) against the oracle's restatement of the reference's
reader: every span, count and error identical."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle
from fastq_cases import random_fastq
from mojoalign_b200 import GpuContext, MojoAlignError
from mojoalign_b200 import _lib

pytestmark = pytest.mark.gpu

KEYS = ("name_off", "name_len", "seq_off", "seq_len", "qual_off", "qual_len")


@pytest.fixture(scope="module")
def ctx():
    c = GpuContext(0)
    yield c
    c.close()


def parse_host(ctx, text: bytes, at_eof=True, max_records=None, base=0):
    b = np.frombuffer(text, np.uint8)
    cap = len(text) // 4 + 2 if max_records is None else max_records
    out = {k: np.zeros(cap, np.uint64 if k.endswith("off") else np.uint32) for k in KEYS}
    rec = _lib.ma_fastq_records(*[out[k].ctypes.data for k in KEYS])
    o3 = (C.c_uint64 * 3)()
    _lib.check(_lib.lib.ma_fastq_parse(ctx.handle, b.ctypes.data if b.size else None, b.size, int(at_eof), cap, base,
                                       C.byref(rec), o3), ctx.handle)
    n = o3[0]
    res = {k: v[:n] for k, v in out.items()}
    res.update(n=n, consumed=o3[1], max_len=o3[2])
    return res


def _same(a, b):
    assert (a["n"], a["consumed"], a["max_len"]) == (b["n"], b["consumed"], b["max_len"])
    for k in KEYS:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def _outcome(f, *a, **kw):
    try:
        return f(*a, **kw), None
    except (MojoAlignError, RuntimeError) as e:
        return None, str(e).split(": ")[-1]


@pytest.mark.parametrize("seed,n", [(1, 1), (2, 10), (3, 5000), (4, 200_000)])
@pytest.mark.parametrize("terminated", [True, False])
def test_whole_buffer_matches_oracle(ctx, seed, n, terminated):
    # an unterminated text whose last QUAL is empty loses that line: both
    # sides must then raise the same truncation error
    text = random_fastq(seed, n, terminated=terminated)
    got, gerr = _outcome(parse_host, ctx, text)
    want, werr = _outcome(oracle.fastq_parse, text)
    assert gerr == werr
    if want is not None:
        _same(got, want)


def test_limits_and_partial_buffers(ctx):
    text = random_fastq(5, 3000)
    for max_records in (1, 7, 2999, 3000, 5000):
        _same(parse_host(ctx, text, max_records=max_records), oracle.fastq_parse(text, max_records=max_records))
    rng = np.random.default_rng(1)
    for cut in rng.integers(1, len(text), size=20):
        part = text[:cut]
        _same(parse_host(ctx, part, at_eof=False, base=77), oracle.fastq_parse(part, at_eof=False, base=77))
    for text in (b"", b"\r", b"@r\nA\n+\nI\n\r", b"r\nA\r\r\n+\n\n", b"@a b/1\r\nAC\r\n+\r\nII\r\n@c/2\nG\n+x\nJ"):
        _same(parse_host(ctx, text), oracle.fastq_parse(text))


def test_truncated_records_raise(ctx):
    for text, msg in ((b"@r\nA\n+\nI\n@s", "SEQ"), (b"@r\nA\n+\nI\n@s\nC\n", "\\+"),
                      (b"@r\nA\n+\nI\n@s\nC\n+\n", "QUAL"), (b"@r\nA\n+\nI\n\n", "SEQ"), (b"\n", "SEQ")):
        with pytest.raises(MojoAlignError, match=f"truncated FASTQ \\(missing {msg}\\)"):
            parse_host(ctx, text)
    assert parse_host(ctx, b"@r\nA\n+\nI\n@s", max_records=1)["n"] == 1


def test_device_form_every_alignment_and_rows(ctx):
    import torch

    text = random_fastq(6, 20_000, crlf=0.5)
    want = oracle.fastq_parse(text)
    dev = torch.device("cuda", 0)
    n = want["n"]
    for shift in (0, 1, 3, 8, 15):
        d_buf = torch.zeros(len(text) + 32, dtype=torch.uint8, device=dev)
        d_buf[shift:shift + len(text)] = torch.frombuffer(bytearray(text), dtype=torch.uint8).to(dev)
        d_out = {k: torch.zeros(n + 5, dtype=torch.int64 if k.endswith("off") else torch.int32, device=dev)
                 for k in KEYS}
        rec = _lib.ma_fastq_records(*[d_out[k].data_ptr() for k in KEYS])
        o3 = (C.c_uint64 * 3)()
        torch.cuda.synchronize()
        _lib.check(_lib.lib.ma_fastq_parse_device(ctx.handle, d_buf.data_ptr() + shift, len(text), 1, n + 5, 0,
                                                  C.byref(rec), o3, None), ctx.handle)
        assert (o3[0], o3[1], o3[2]) == (n, want["consumed"], want["max_len"])
        for k in KEYS:
            got = d_out[k].cpu().numpy().view(np.uint64 if k.endswith("off") else np.uint32)[:n]
            np.testing.assert_array_equal(got, want[k], err_msg=k)
    # rows for the mapper: SEQ then 'N' to max_len
    ml = int(want["max_len"])
    rows = torch.empty(n * ml, dtype=torch.uint8, device=dev)
    lens = torch.empty(n, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    _lib.check(_lib.lib.ma_fastq_rows_device(ctx.handle, d_buf.data_ptr() + 15, d_out["seq_off"].data_ptr(),
                                             d_out["seq_len"].data_ptr(), n, ml, rows.data_ptr(), lens.data_ptr(),
                                             None), ctx.handle)
    torch.cuda.synchronize()
    r = rows.cpu().numpy().reshape(n, ml)
    for i in range(0, n, 97):
        s = text[int(want["seq_off"][i]):int(want["seq_off"][i]) + int(want["seq_len"][i])]
        assert r[i].tobytes() == s + b"N" * (ml - len(s))
    np.testing.assert_array_equal(lens.cpu().numpy().view(np.uint32), want["seq_len"])
