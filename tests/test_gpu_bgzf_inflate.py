"""BGZF members inflated on the device (ma_bgzf_inflate[_device]) against the
gzip module: the same bytes for every level, and the member-level errors
(size, CRC-32, damaged deflate data) the host-run member step reports."""
from __future__ import annotations

import ctypes as C
import gzip

import numpy as np
import pytest

from fastq_cases import random_fastq
from mojoalign_b200 import GpuContext, MojoAlignError, _lib
from mojoalign_b200.fqio import bgzf_inflate, bgzf_members
from oracle import bgzf_ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = GpuContext(0)
    yield c
    c.close()


@pytest.mark.parametrize("level", [0, 1, 6, 9])
def test_inflate_matches_gzip(ctx, level):
    text = random_fastq(21 + level, 20_000, crlf=0.2)
    blob = bgzf_ref.compress(text, level)
    assert bgzf_inflate(ctx, blob) == gzip.decompress(blob) == text


def test_empty_and_single_member(ctx):
    assert bgzf_inflate(ctx, bgzf_ref.compress(b"", 1)) == b""
    assert bgzf_inflate(ctx, bgzf_ref.compress(b"@r\nACGT\n+\nIIII\n", 6, eof=False)) == b"@r\nACGT\n+\nIIII\n"


def test_bad_members_are_reported(ctx):
    text = random_fastq(30, 3000)
    blob = bgzf_ref.compress(text, 1)
    t = bgzf_members(blob)
    bad = bytearray(blob)
    # the CRC-32 of member 1 (4 bytes before its ISIZE)
    end1 = int(t["src_off"][1] + t["src_len"][1])
    bad[end1] ^= 0xFF
    with pytest.raises(MojoAlignError, match="BGZF member 1: CRC-32 mismatch"):
        bgzf_inflate(ctx, bytes(bad))


def test_device_form_status(ctx):
    import torch

    text = random_fastq(31, 5000)
    blob = bgzf_ref.compress(text, 1)
    t = bgzf_members(blob)
    dev = torch.device("cuda", 0)

    def put(a):
        a = np.ascontiguousarray(a)
        sg = {np.dtype(np.uint64): np.int64, np.dtype(np.uint32): np.int32}
        return torch.from_numpy(a.view(sg.get(a.dtype, a.dtype)).copy()).to(dev)

    d_in = put(np.frombuffer(blob, np.uint8))
    cols = {k: put(t[k]) for k in ("src_off", "src_len", "dst_off", "isize", "crc")}
    cols["crc"][2] += 1  # member 2 fails its check, the others inflate
    n = int(t["src_off"].size)
    d_out = torch.zeros(t["out_bytes"] + 8, dtype=torch.uint8, device=dev)
    d_status = torch.zeros(n, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    _lib.check(_lib.lib.ma_bgzf_inflate_device(ctx.handle, d_in.data_ptr(), len(blob),
                                               *[cols[k].data_ptr() for k in ("src_off", "src_len", "dst_off",
                                                                              "isize", "crc")],
                                               n, d_out.data_ptr(), t["out_bytes"], d_status.data_ptr(), None),
               ctx.handle)
    torch.cuda.synchronize()
    status = d_status.cpu().numpy()
    assert status[2] == 9 and not np.delete(status, 2).any()
    out = d_out.cpu().numpy().tobytes()
    assert out[:t["out_bytes"]] == text and not any(out[t["out_bytes"]:])
