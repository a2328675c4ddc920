"""The DEFLATE decoder written for the device (csrc/inflate.cuh), compiled as
host code and checked against zlib: every compression level and strategy,
stored / fixed / dynamic blocks, BGZF members, and truncated or corrupted
streams (the same outcome as zlib: the same bytes, or an error), with an
AddressSanitizer build checking that no stream makes it read or write
outside its buffers."""
from __future__ import annotations

import ctypes as C
import subprocess
import zlib
from pathlib import Path

import numpy as np
import pytest

from fastq_cases import random_fastq
from oracle import bgzf_ref

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent / "mojo-align_b200" / "csrc"


def _build(tmp_path_factory, name, flags):
    d = tmp_path_factory.mktemp("inflate")
    so = d / name
    subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fPIC", "-shared", *flags, "-I", str(CSRC),
                    str(HERE / "inflate_harness.cpp"), "-o", str(so)], check=True)
    lib = C.CDLL(str(so))
    lib.harness_inflate.argtypes = [C.c_char_p, C.c_uint32, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]
    lib.harness_inflate.restype = C.c_int
    return lib


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    return _build(tmp_path_factory, "libinflate.so", ["-O2"])


def inflate(lib, data: bytes, cap: int):
    out = np.zeros(max(cap, 1), np.uint8)
    n = C.c_uint32(0)
    rc = lib.harness_inflate(data, len(data), out.ctypes.data, cap, C.byref(n))
    return rc, out[:n.value].tobytes()


def raw_deflate(data: bytes, level: int, strategy: int = zlib.Z_DEFAULT_STRATEGY, wbits: int = -15) -> bytes:
    c = zlib.compressobj(level, zlib.DEFLATED, wbits, 9, strategy)
    return c.compress(data) + c.flush()


def inputs():
    rng = np.random.default_rng(1)
    text = random_fastq(4, 400)
    return {
        "empty": b"",
        "one": b"A",
        "fastq": text[:65280],
        "fastq_small": text[:777],
        "random": rng.integers(0, 256, size=65280, dtype=np.uint8).tobytes(),
        "zeros": bytes(65280),
        "runs": b"".join(bytes([int(c)]) * int(k) for c, k in zip(rng.integers(0, 4, 3000) + 65,
                                                                rng.integers(1, 300, 3000)))[:65280],
        "long": text * 3,
    }


STRATEGIES = [zlib.Z_DEFAULT_STRATEGY, zlib.Z_FILTERED, zlib.Z_HUFFMAN_ONLY, zlib.Z_RLE, zlib.Z_FIXED]


@pytest.mark.parametrize("level", range(10))
def test_levels_and_strategies(lib, level):
    for name, data in inputs().items():
        for strategy in STRATEGIES:
            for wbits in (-15, -9):
                z = raw_deflate(data, level, strategy, wbits)
                rc, got = inflate(lib, z, len(data))
                assert rc == 0 and got == data, (name, strategy, wbits, rc)


def test_bgzf_members_and_output_cap(lib):
    text = random_fastq(5, 2000)
    for level in (0, 1, 6, 9):
        for m in bgzf_ref.members(bgzf_ref.compress(text, level)):
            rc, got = inflate(lib, m["payload"], m["isize"])
            assert rc == 0 and len(got) == m["isize"] and zlib.crc32(got) == m["crc"]
            if m["isize"]:
                rc, _ = inflate(lib, m["payload"], m["isize"] - 1)
                assert rc == 7  # E_OUTPUT


def _zlib_outcome(z: bytes):
    d = zlib.decompressobj(-15)
    try:
        out = d.decompress(z)
    except zlib.error:
        return None
    return out if d.eof else None


def test_truncated_and_corrupted_streams_match_zlib(lib):
    rng = np.random.default_rng(7)
    text = random_fastq(6, 60)
    streams = [raw_deflate(text, lv, st) for lv in (1, 6, 9) for st in STRATEGIES] + \
        [raw_deflate(b"ACGT" * 500, 6), raw_deflate(bytes(rng.integers(0, 256, 3000, dtype=np.uint8)), 0)]
    cases = 0
    for z in streams:
        for cut in sorted(set(rng.integers(0, len(z), size=25).tolist())):
            rc, _ = inflate(lib, z[:cut], 1 << 20)
            assert rc != 0
            cases += 1
        for _ in range(60):
            b = bytearray(z)
            for p in rng.integers(0, len(b), size=int(rng.integers(1, 4))):
                b[p] ^= 1 << int(rng.integers(0, 8))
            want = _zlib_outcome(bytes(b))
            rc, got = inflate(lib, bytes(b), 1 << 20)
            assert (rc == 0) == (want is not None), (rc, want is not None)
            if want is not None:
                assert got == want
            cases += 1
    assert cases > 1000


def test_no_access_outside_buffers_under_asan(tmp_path_factory):
    """Random and corrupted streams through an AddressSanitizer build, in a
    child process (the sanitizer runtime must be loaded first)."""
    d = tmp_path_factory.mktemp("inflate_asan")
    exe = d / "fuzz"
    src = d / "fuzz.cpp"
    src.write_text(r'''
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "inflate.cuh"
int main() {
    std::FILE* f = std::fopen("streams.bin", "rb");
    if (!f) return 2;
    ma::inflate::Tables* t = new ma::inflate::Tables;
    unsigned n;
    long ok = 0, bad = 0;
    while (std::fread(&n, 4, 1, f) == 1) {
        std::vector<uint8_t> in(n);
        if (n && std::fread(in.data(), 1, n, f) != n) return 3;
        for (unsigned cap : {0u, 1u, 100u, 70000u}) {
            std::vector<uint8_t> out(cap ? cap : 1);
            uint32_t got = 0;
            // exact-size buffers: an access past either end is a sanitizer error
            uint8_t* ib = n ? new uint8_t[n] : nullptr;
            for (unsigned i = 0; i < n; ++i) ib[i] = in[i];
            uint8_t* ob = cap ? new uint8_t[cap] : nullptr;
            int rc = ma::inflate::inflate_raw(ib, n, ob, cap, &got, *t);
            (rc == 0 ? ok : bad)++;
            delete[] ib;
            delete[] ob;
        }
    }
    delete t;
    std::fclose(f);
    std::printf("%ld %ld\n", ok, bad);
    return 0;
}
''')
    subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
                    "-I", str(CSRC), str(src), "-o", str(exe)], check=True)
    rng = np.random.default_rng(11)
    text = random_fastq(8, 80)
    base = [raw_deflate(text, lv, st) for lv in (0, 1, 9) for st in STRATEGIES]
    blobs = []
    for z in base:
        blobs.append(z)
        for _ in range(40):
            b = bytearray(z)
            for p in rng.integers(0, len(b), size=int(rng.integers(1, 6))):
                b[p] = int(rng.integers(0, 256))
            blobs.append(bytes(b[: int(rng.integers(0, len(b) + 1))]))
    blobs += [rng.integers(0, 256, size=int(rng.integers(0, 3000)), dtype=np.uint8).tobytes() for _ in range(300)]
    with open(d / "streams.bin", "wb") as f:
        for b in blobs:
            f.write(len(b).to_bytes(4, "little") + b)
    r = subprocess.run([str(exe)], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    ok, bad = map(int, r.stdout.split())
    assert ok > 0 and bad > 0


def members_on_host(lib, blob: bytes, table=None):
    """harness_inflate_members: the kernel's per-member step over a BGZF file."""
    from mojoalign_b200.fqio import bgzf_members

    t = table or bgzf_members(blob)
    lib.harness_inflate_members.argtypes = [C.c_char_p, C.c_uint64] + [C.c_void_p] * 5 + \
        [C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p]
    out = np.zeros(max(t["out_bytes"], 1), np.uint8)
    status = np.zeros(max(t["src_off"].size, 1), np.uint32)
    lib.harness_inflate_members(blob, len(blob), *[t[k].ctypes.data for k in ("src_off", "src_len", "dst_off",
                                                                               "isize", "crc")],
                                int(t["src_off"].size), out.ctypes.data, t["out_bytes"], status.ctypes.data)
    return out[:t["out_bytes"]].tobytes(), status[:t["src_off"].size]


def test_member_step_inflates_bgzf_files(lib):
    import gzip

    from mojoalign_b200.fqio import bgzf_members

    text = random_fastq(12, 3000, crlf=0.2)
    for level in (0, 1, 5, 9):
        blob = bgzf_ref.compress(text, level)
        got, status = members_on_host(lib, blob)
        assert not status.any() and got == gzip.decompress(blob) == text
    blob = bgzf_ref.compress(text, 1)
    t = bgzf_members(blob)
    assert t["out_bytes"] == len(text) and t["isize"][-1] == 0  # the EOF member
    # a wrong CRC, a wrong ISIZE, a damaged payload, spans outside the buffers
    bad = dict(t, crc=t["crc"].copy(), isize=t["isize"].copy(), src_off=t["src_off"].copy())
    bad["crc"][1] ^= 1
    bad["isize"][2] -= 1
    bad["src_off"][3] = len(blob)
    _, status = members_on_host(lib, blob, bad)
    assert status[1] == 9 and status[2] == 7 and status[3] == 10 and not status[4:].any()
    dmg = bytearray(blob)
    dmg[int(t["src_off"][0]) + 5] ^= 0x55
    _, status = members_on_host(lib, bytes(dmg), t)
    assert status[0] != 0 and not status[1:].any()
