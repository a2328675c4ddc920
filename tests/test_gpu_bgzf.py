"""GPU BGZF (ma_bgzf_compress[_device]) against the oracle restatement of the
reference's writer: level 0 byte-identical; levels 1..9 member by member the
reference's framing (header fields, BSIZE, CRC-32, ISIZE, 65280-byte
pieces, EOF member) with deflate data that inflate to exactly the input."""
from __future__ import annotations

import ctypes as C
import gzip
import sys
import zlib
from pathlib import Path

import numpy as np
import pytest

from bam_batches import RID_TO_TID, bam_cap_for, random_batch
from mojoalign_b200 import GpuContext, MojoAlignError
from mojoalign_b200 import _lib
from oracle import bgzf_ref
import oracle

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from make_bgzf_golden import stream  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = GpuContext(0)
    yield c
    c.close()


def gpu_bgzf(ctx, data: bytes, level: int, eof: bool = True) -> bytes:
    b = np.frombuffer(data, np.uint8)
    cap = int(_lib.lib.ma_bgzf_bound(len(data)))
    out = np.empty(cap, np.uint8)
    got = C.c_uint64(0)
    _lib.check(_lib.lib.ma_bgzf_compress(ctx.handle, b.ctypes.data if b.size else None, len(data), level, int(eof),
                                         out.ctypes.data, cap, C.byref(got)), ctx.handle)
    return out[:got.value].tobytes()


def check_framing(out: bytes, data: bytes, eof: bool = True):
    ms = bgzf_ref.members(out)
    body = ms[:-1] if eof else ms
    if eof:
        assert out[ms[-1]["off"]:] == bgzf_ref.EOF_MEMBER
    assert len(body) == (len(data) + bgzf_ref.BLOCK - 1) // bgzf_ref.BLOCK
    pos = 0
    for m in body:
        assert m["fixed"] == (31, 139, 8, 4, 0, 0, 255, 6, 66, 67, 2)
        piece = data[pos:pos + bgzf_ref.BLOCK]
        assert bgzf_ref.inflate(m["payload"]) == piece
        assert m["crc"] == zlib.crc32(piece) & 0xFFFFFFFF and m["isize"] == len(piece)
        pos += len(piece)
    assert gzip.decompress(out) == data


def bam_stream(seed: int, n1: int) -> bytes:
    hits, arena, _ = random_batch(seed, n1, True)
    bam, _, _ = oracle.emit_bam(hits, vars(arena), n1, True, RID_TO_TID, b"mojo1", cap=bam_cap_for(arena, 5))
    return bam


CASES = [("ramp", 0), ("ramp", 1), ("ramp", 100), ("ramp", 32767), ("ramp", 32768), ("ramp", 65279),
         ("ramp", 65280), ("ramp", 65281), ("text", 200_000), ("zeros", 140_000)]


@pytest.mark.parametrize("kind,n", CASES)
def test_level0_is_byte_identical(ctx, kind, n):
    data = stream(kind, n)
    assert gpu_bgzf(ctx, data, 0) == bgzf_ref.compress(data, 0)


@pytest.mark.parametrize("kind,n", CASES)
@pytest.mark.parametrize("level", [1, 6, 9])
def test_levels_round_trip(ctx, kind, n, level):
    data = stream(kind, n)
    check_framing(gpu_bgzf(ctx, data, level), data)


def test_incompressible_and_bam_streams(ctx):
    rng = np.random.default_rng(3)
    noise = rng.integers(0, 256, size=300_000, dtype=np.uint8).tobytes()
    out = gpu_bgzf(ctx, noise, 1)
    check_framing(out, noise)
    assert len(out) <= len(bgzf_ref.compress(noise, 0))  # stored when coding does not pay
    bam = bam_stream(5, 20_000)
    out = gpu_bgzf(ctx, bam, 1, eof=False)
    check_framing(out, bam, eof=False)
    ref = bgzf_ref.compress(bam, 1, eof=False)
    # the coder's ratio on BAM records stays near zlib level 1's
    assert len(out) < 1.25 * len(ref), (len(out), len(ref), len(bam))


def test_device_form_and_errors(ctx):
    import torch

    data = bam_stream(6, 5_000)
    dev = torch.device("cuda", 0)
    d_in = torch.frombuffer(bytearray(data), dtype=torch.uint8).to(dev)
    cap = int(_lib.lib.ma_bgzf_bound(len(data)))
    d_out = torch.zeros(cap, dtype=torch.uint8, device=dev)
    got = C.c_uint64(0)
    torch.cuda.synchronize()
    _lib.check(_lib.lib.ma_bgzf_compress_device(ctx.handle, d_in.data_ptr(), len(data), 1, 1, d_out.data_ptr(), cap,
                                                C.byref(got), None), ctx.handle)
    out = d_out[:got.value].cpu().numpy().tobytes()
    check_framing(out, data)
    assert out == gpu_bgzf(ctx, data, 1)  # deterministic
    with pytest.raises(MojoAlignError, match="larger than the output buffer"):
        _lib.check(_lib.lib.ma_bgzf_compress_device(ctx.handle, d_in.data_ptr(), len(data), 1, 1, d_out.data_ptr(),
                                                    got.value - 1, C.byref(got), None), ctx.handle)
    with pytest.raises(MojoAlignError, match="level"):
        gpu_bgzf(ctx, data, 10)
