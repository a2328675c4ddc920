"""File input and output of the device pipelines.

The reference reads `.gz` / `.gzip` files through `pigz -dc` (or Python's
gzip module when pigz is absent: fq2bam-meth/python/fastq_batch.py:31-46,
linear_fastq.mojo _looks_gz L49-51) and anything else as plain bytes.  The
same bytes come out of open_fastq().  A gzip file made of BGZF members (the
blocked gzip of bgzip / htslib: every member carries a "BC" extra field
with its size) is inflated on a thread pool, many members at once; any other
gzip file is read by the gzip module, one member after another.
"""
from __future__ import annotations

import gzip
import io
import os
import struct
import zlib
from collections import deque
from concurrent.futures import ThreadPoolExecutor

_MAGIC = b"\x1f\x8b\x08"
JOB_BYTES = 1 << 20  # compressed bytes per inflate job


def _bgzf_size(head: bytes) -> int:
    """Total size of the BGZF member whose first bytes are `head` (at least
    18 bytes), or 0 when it is not a BGZF member."""
    if len(head) < 18 or head[:3] != _MAGIC or not (head[3] & 4):
        return 0
    xlen = struct.unpack_from("<H", head, 10)[0]
    if len(head) < 12 + xlen:
        return 0
    i = 12
    while i + 4 <= 12 + xlen:
        slen = struct.unpack_from("<H", head, i + 2)[0]
        if head[i:i + 2] == b"BC" and slen == 2:
            return struct.unpack_from("<H", head, i + 4)[0] + 1
        i += 4 + slen
    return 0


def _inflate_members(blob: bytes, sizes: list) -> bytes:
    """The members of `blob` (consecutive BGZF members of the given sizes)
    inflated and checked (CRC-32, ISIZE), concatenated."""
    out = []
    pos = 0
    for n in sizes:
        m = memoryview(blob)[pos:pos + n]
        xlen = struct.unpack_from("<H", m, 10)[0]
        crc, isize = struct.unpack_from("<II", m, n - 8)
        # one inflate call into a buffer of the stored size (the GIL is
        # released for the whole member)
        data = zlib.decompress(m[12 + xlen:n - 8], -15, max(isize, 1))
        if len(data) != isize or zlib.crc32(data) != crc:
            raise gzip.BadGzipFile("BGZF member fails its CRC-32 / size check")
        out.append(data)
        pos += n
    return b"".join(out)


class _Prefixed(io.RawIOBase):
    """A raw binary reader: the bytes `head`, then the rest of file `fh`
    (which stays open: its owner closes it)."""

    def __init__(self, head: bytes, fh):
        super().__init__()
        self._head = memoryview(head)
        self._fh = fh

    def readable(self) -> bool:
        return True

    def readinto(self, b) -> int:
        if len(self._head):
            k = min(len(b), len(self._head))
            b[:k] = self._head[:k]
            self._head = self._head[k:]
            return k
        return self._fh.readinto(b)


class BgzfReader:
    """A binary file object over a BGZF file: its members are inflated by a
    thread pool in batches of about `batch_bytes` compressed bytes, in order.
    A member that is not BGZF (a plain gzip member appended to the file)
    switches the rest of the file to the gzip module."""

    def __init__(self, path: str, threads: int | None = None, batch_bytes: int = 16 << 20):
        self._fh = open(path, "rb")
        self._threads = max(1, threads or (os.cpu_count() or 1))
        self._pool = ThreadPoolExecutor(max_workers=self._threads)
        self._batch = batch_bytes
        self._jobs: deque = deque()
        self._raw = b""  # compressed bytes read but not yet split into members
        self._done = False  # no more compressed bytes to schedule
        self._tail = None  # gzip.GzipFile over a non-BGZF remainder
        self._cur = memoryview(b"")

    def _read_batch(self) -> None:
        """Reads about batch_bytes of whole members and schedules them."""
        if len(self._raw) < self._batch:
            self._raw += self._fh.read(self._batch - len(self._raw))
        sizes, pos = [], 0
        while True:
            n = _bgzf_size(self._raw[pos:pos + 18 + 256])
            if n == 0 or pos + n > len(self._raw):
                break
            sizes.append(n)
            pos += n
        if sizes:
            blob, self._raw = self._raw[:pos], self._raw[pos:]
            # jobs of about JOB_BYTES compressed bytes, so that all threads work
            first_byte = first_member = off = 0
            for i, n in enumerate(sizes):
                off += n
                if off - first_byte >= JOB_BYTES or i == len(sizes) - 1:
                    self._jobs.append(self._pool.submit(_inflate_members, blob[first_byte:off],
                                                        sizes[first_member:i + 1]))
                    first_byte, first_member = off, i + 1
            return
        # no whole BGZF member at the front
        n = _bgzf_size(self._raw[:18 + 256])
        if n and len(self._raw) < n:
            # a BGZF member cut by the batch boundary: read the rest of it
            more = self._fh.read(n - len(self._raw))
            if not more:
                raise EOFError("Compressed file ended before the end-of-stream marker was reached")
            self._raw += more
            return
        # zero padding (gzip allows it between and after members) is skipped
        head = self._raw.lstrip(b"\0")
        while not head:
            chunk = self._fh.read(1 << 16)
            if not chunk:
                self._done = True
                self._raw = b""
                return
            head = chunk.lstrip(b"\0")
        if len(head) < 18 + 256:
            head += self._fh.read(18 + 256 - len(head))
        if _bgzf_size(head[:18 + 256]):
            self._raw = head  # BGZF members go on after the padding
            return
        if head[:2] != _MAGIC[:2]:
            raise gzip.BadGzipFile("Not a gzipped file (%r)" % head[:2])
        # a member that is not BGZF: the gzip module reads the rest of the
        # file from here, straight from the open file
        self._done = True
        self._raw = b""
        self._tail = gzip.GzipFile(fileobj=io.BufferedReader(_Prefixed(head, self._fh)))

    def _fill_jobs(self) -> None:
        while not self._done and len(self._jobs) < 4 * self._threads:
            self._read_batch()

    def readinto(self, b) -> int:
        mv = memoryview(b).cast("B")
        got = 0
        while got < len(mv):
            if len(self._cur):
                k = min(len(self._cur), len(mv) - got)
                mv[got:got + k] = self._cur[:k]
                self._cur = self._cur[k:]
                got += k
                continue
            self._fill_jobs()
            if self._jobs:
                self._cur = memoryview(self._jobs.popleft().result())
                continue
            if self._tail is not None:
                k = self._tail.readinto(mv[got:])
                if k:
                    got += k
                    continue
            break
        return got

    def read(self, n: int = -1) -> bytes:
        if n is None or n < 0:
            parts = []
            while True:
                chunk = bytearray(1 << 20)
                k = self.readinto(chunk)
                if not k:
                    return b"".join(parts)
                parts.append(bytes(chunk[:k]))
        buf = bytearray(n)
        return bytes(buf[:self.readinto(buf)])

    def close(self) -> None:
        for j in self._jobs:
            j.cancel()
        self._pool.shutdown(wait=True)
        self._fh.close()
        if self._tail is not None:
            self._tail.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def bgzf_members(blob: bytes) -> dict:
    """The member table of a BGZF file held in memory: per member the offset
    and length of its deflate payload, the offset of its bytes in the
    inflated stream, ISIZE and CRC-32 (numpy arrays), and the inflated size.
    Raises gzip.BadGzipFile when a member is not BGZF or runs past the end."""
    import numpy as np

    so, sl, do, isz, crc = [], [], [], [], []
    pos, out = 0, 0
    while pos < len(blob):
        n = _bgzf_size(blob[pos:pos + 18 + 256])
        if n == 0 or pos + n > len(blob) or n < 26:
            raise gzip.BadGzipFile(f"no whole BGZF member at byte {pos}")
        xlen = struct.unpack_from("<H", blob, pos + 10)[0]
        c, s_ = struct.unpack_from("<II", blob, pos + n - 8)
        so.append(pos + 12 + xlen)
        sl.append(n - 12 - xlen - 8)
        do.append(out)
        isz.append(s_)
        crc.append(c)
        out += s_
        pos += n
    return {"src_off": np.array(so, np.uint64), "src_len": np.array(sl, np.uint32), "dst_off": np.array(do, np.uint64),
            "isize": np.array(isz, np.uint32), "crc": np.array(crc, np.uint32), "out_bytes": out}


def bgzf_inflate(ctx, blob: bytes) -> bytes:
    """A BGZF file inflated on the device (ma_bgzf_inflate): the same bytes as
    the gzip module gives; MojoAlignError names the first bad member."""
    import ctypes as C

    import numpy as np

    from ._lib import check, lib

    t = bgzf_members(blob)
    src = np.frombuffer(blob, np.uint8)
    out = np.empty(max(t["out_bytes"], 1), np.uint8)
    status = np.zeros(max(t["src_off"].size, 1), np.uint32)
    p = lambda a: a.ctypes.data  # noqa: E731
    check(lib.ma_bgzf_inflate(ctx.handle, p(src) if src.size else None, src.size, p(t["src_off"]), p(t["src_len"]),
                              p(t["dst_off"]), p(t["isize"]), p(t["crc"]), int(t["src_off"].size), p(out),
                              t["out_bytes"], p(status)), ctx.handle)
    return out[:t["out_bytes"]].tobytes()


def is_bgzf(path: str) -> bool:
    with open(path, "rb") as fh:
        return _bgzf_size(fh.read(18 + 256)) > 0


def open_fastq(path: str, threads: int | None = None):
    """A binary file object with the uncompressed FASTQ bytes of `path`
    (gzip by the .gz / .gzip suffix, like the reference)."""
    low = str(path).lower()
    if low.endswith(".gz") or low.endswith(".gzip"):
        if is_bgzf(path):
            return BgzfReader(str(path), threads)
        return gzip.open(path, "rb")
    return open(path, "rb")


WRITE_THREADS = 4  # the page-cache copy of one writer thread tops out well below the disk's


class ParallelWriter:
    """Writes byte buffers at increasing offsets of one file, each buffer
    split over a few threads (os.pwrite), so that the copy into the page
    cache is not bound by one core.  Buffers are written in call order;
    write() returns once the buffer is on its way to the file (the data may
    be reused after it returns)."""

    def __init__(self, path, threads: int = WRITE_THREADS, min_split: int = 8 << 20):
        self.fd = os.open(str(path), os.O_WRONLY | os.O_CREAT | os.O_TRUNC, 0o644)
        self.off = 0
        self.threads = max(1, threads)
        self.min_split = min_split
        self._pool = ThreadPoolExecutor(max_workers=self.threads) if self.threads > 1 else None

    def _put(self, mv, off: int) -> None:
        done = 0
        while done < len(mv):
            done += os.pwrite(self.fd, mv[done:], off + done)

    def write(self, data) -> int:
        mv = memoryview(data).cast("B")
        n = len(mv)
        if self._pool is None or n < self.min_split:
            self._put(mv, self.off)
        else:
            step = (n + self.threads - 1) // self.threads
            futs = [self._pool.submit(self._put, mv[i:i + step], self.off + i) for i in range(0, n, step)]
            for f in futs:
                f.result()
        self.off += n
        return n

    def close(self) -> None:
        if self._pool is not None:
            self._pool.shutdown(wait=True)
        if self.fd >= 0:
            os.close(self.fd)
            self.fd = -1

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
