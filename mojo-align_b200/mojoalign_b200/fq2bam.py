"""FASTQ to coordinate-sorted, duplicate-marked BAM with every stage on the GPU.

The .bam destination of map_fastq_fm_gpu (fq2bam-meth/src/linear_gpu_fm.mojo:
1028-3341 with emit_bam, L2084): the reference parses FASTQ on the host
(linear_fastq.mojo), maps each batch on the GPU, copies the outputs back,
packs BAM records on the host (_emit_bam_from_batch), sorts and marks
duplicates (gpu_sort_markdup, with host round trips), gathers the records in
coordinate order and compresses them with zlib threads (bam_emit.BamWriter).
Here the uncompressed FASTQ bytes are copied to the device once and nothing
but the finished BGZF file comes back:

    host: read / gunzip FASTQ  ->  HBM: split records (ma_fastq_parse_device)
      -> mapper rows (ma_fastq_rows_device) -> map (ma_map_batch_device)
      -> BAM records + tile metadata (ma_emit_bam_batch_device; the FASTQ
         bytes of the batch are the arena) ... for every batch, then
      -> sort + markdup (ma_sort_markdup_device)
      -> header + sorted records (ma_gather_sorted_bam_device)
      -> BGZF (ma_bgzf_compress_device)  ->  host: write the file.

The file is the reference's: same header (BamWriter.__init__, bam_emit.py:
312-356, with the canonical @SQ list of _open_bam_writer,
linear_gpu_fm.mojo:91-125), same records in the same order and flags, BGZF
pieces cut at the same 65280-byte boundaries.  At METHYLGRAPHER_BAM_LEVEL=0 the
bytes are identical; at levels 1..9 the deflate data come from this library's
coder and the members inflate to the same bytes.  The result does not depend
on the batch size.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import gzip
import os
import struct
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import pinned
from .fqio import ParallelWriter, open_fastq
from ._lib import (MA_FASTQ_RULES_STREAM, check, lib, ma_bam_meta, ma_bam_tile, ma_fastq_arena, ma_fastq_records,
                   ma_hits)
from .bam import META_FIELDS, canonical_rid_to_tid
from .linear_fm import canonical_contig, fm_prefix_from_ref, select_device
from .mapper import GpuContext, GpuIndex, MapResult, bs_mode
from .params import FmParams

SORT_CAP_ENV = ("METHYLGRAPHER_FM_SORT_CAP", 67108864)
MAX_LEN_CAP = 1024
REC_KEYS = ("name_off", "name_len", "seq_off", "seq_len", "qual_off", "qual_len")


def _env(env, name, default):
    v = env.get(name, "")
    return v if v else default


def bam_header(contigs, env=None) -> bytes:
    """The uncompressed BAM header BamWriter writes (bam_emit.py:312-356) for
    the canonical @SQ list of _open_bam_writer (linear_gpu_fm.mojo:91-125)."""
    env = os.environ if env is None else env
    names, lens, seen = [], [], set()
    for c in contigs:
        canon = canonical_contig(c.name)
        if canon not in seen:
            seen.add(canon)
            names.append(canon)
            lens.append(int(c.length))
    rg = _env(env, "METHYLGRAPHER_RG_ID", "mojo1")
    sm = _env(env, "METHYLGRAPHER_RG_SM", "sample")
    lb = _env(env, "METHYLGRAPHER_RG_LB", "lib1")
    pl = _env(env, "METHYLGRAPHER_RG_PL", "ILLUMINA")
    lines = ["@HD\tVN:1.6\tSO:coordinate"]
    lines += [f"@SQ\tSN:{n}\tLN:{ln}" for n, ln in zip(names, lens)]
    lines.append(f"@RG\tID:{rg}\tSM:{sm}\tLB:{lb}\tPL:{pl}\tPU:{rg}")
    lines.append("@PG\tID:MojoFq2bamMeth\tPN:MojoFq2bamMeth\tVN:0.1.0-mojo-fm")
    text = ("\n".join(lines) + "\n").encode("ascii")
    blob = bytearray(b"BAM\x01") + struct.pack("<i", len(text)) + text + struct.pack("<i", len(names))
    for n, ln in zip(names, lens):
        nb = n.encode("ascii") + b"\x00"
        blob += struct.pack("<i", len(nb)) + nb + struct.pack("<i", ln)
    return bytes(blob)


class _Feed:
    """Uncompressed bytes of one FASTQ file in a pinned host buffer (gzip by
    suffix, like _looks_gz, linear_fastq.mojo:49-51; BGZF files inflated on
    a thread pool): fill() tops the buffer up to its capacity, consume(n)
    drops the first n bytes."""

    def __init__(self, path: str, chunk: int, torch):
        self.fh = open_fastq(path)
        self._buf = pinned.take(chunk)
        self.pin = self._buf[:chunk].numpy()
        self.len = 0
        self.eof = False

    def fill(self):
        mv = memoryview(self.pin)
        while not self.eof and self.len < self.pin.size:
            k = self.fh.readinto(mv[self.len:])
            if not k:
                self.eof = True
                break
            self.len += k

    def consume(self, n: int):
        rest = self.len - n
        if rest > 0 and n > 0:
            self.pin[:rest] = self.pin[n:self.len].copy()
        self.len = max(rest, 0)

    def close(self):
        self.fh.close()
        pinned.give(self._buf)
        self._buf = None


class _DeviceFeed:
    """Uncompressed bytes of one BGZF FASTQ file in HBM, inflated on the
    device: fill() reads whole members (their compressed bytes only cross
    PCIe) into a pinned buffer, copies them to the device and inflates them
    behind the bytes left from the last piece (ma_bgzf_inflate_device, one
    warp per member); consume(n) drops the first n bytes, moving the rest to
    the front on the device.  Same interface as _Feed, with `dev` in place
    of `pin`.  A member that is not BGZF (an appended plain gzip member) is
    inflated on the host and copied in."""

    def __init__(self, path: str, chunk: int, torch, ctx):
        self.torch, self.ctx = torch, ctx
        self.fh = open(path, "rb")
        self.cap = chunk
        self.dev = torch.empty(chunk + 16, dtype=torch.uint8, device=torch.device("cuda", ctx.device))
        self.stream = torch.cuda.Stream(device=self.dev.device)
        # compressed bytes of one fill at most a quarter of the piece (BGZF
        # members inflate to at most 64 KB; FASTQ compresses 2-4x)
        self._cbuf = pinned.take(max(chunk // 4, 1 << 20))
        self.cpin = self._cbuf.numpy()
        self.craw = b""  # compressed bytes read but not yet inflated
        self.len = 0
        self.eof = False
        self.h2d_bytes = 0
        self._tail = None  # host reader over a non-BGZF remainder

    def _more(self, need: int) -> bool:
        """Reads until craw holds `need` bytes; False at the end of the file."""
        while len(self.craw) < need:
            more = self.fh.read(max(1 << 20, need - len(self.craw)))
            if not more:
                return False
            self.craw += more
        return True

    def _members(self):
        """Whole BGZF members from the file (compressed bytes; as many as fit
        the pinned buffer and the room left in the device buffer), skipping
        zero padding between them: their table, compressed and inflated
        sizes, and why it stopped ("room", "end" of the file, or "other": a
        member that is not BGZF)."""
        from .fqio import _bgzf_size

        room = self.cap - self.len
        so, sl, do, isz, crc = [], [], [], [], []
        used = out = 0
        why = "end"
        while True:
            self._more(18 + 256)
            if self.craw[:1] == b"\0":  # gzip allows zero padding between members
                self.craw = self.craw.lstrip(b"\0")
                continue
            if not self.craw:
                break
            n = _bgzf_size(self.craw[:18 + 256])
            if n == 0:
                why = "other"
                break
            if not self._more(n):
                raise EOFError("Compressed file ended before the end-of-stream marker was reached")
            isize = struct.unpack_from("<I", self.craw, n - 4)[0]
            if out + isize > room or used + n > self.cpin.size:
                why = "room"
                break
            xlen = struct.unpack_from("<H", self.craw, 10)[0]
            self.cpin[used:used + n] = np.frombuffer(self.craw, np.uint8, n)
            so.append(used + 12 + xlen)
            sl.append(n - 12 - xlen - 8)
            do.append(out)
            isz.append(isize)
            crc.append(struct.unpack_from("<I", self.craw, n - 8)[0])
            used += n
            out += isize
            self.craw = self.craw[n:]
        return why, used, out, (so, sl, do, isz, crc)

    def fill(self):
        torch = self.torch
        if self._tail is not None:
            self._fill_host()
            return
        why, used, out, table = self._members()
        if used:
            so = table[0]
            with torch.cuda.stream(self.stream):
                d_in = torch.empty(used, dtype=torch.uint8, device=self.dev.device)
                d_in.copy_(torch.from_numpy(self.cpin[:used]), non_blocking=True)
                tab = [torch.from_numpy(np.asarray(v, dt)).to(self.dev.device)
                       for v, dt in zip(table, (np.uint64, np.uint32, np.uint64, np.uint32, np.uint32))]
                status = torch.zeros(len(so), dtype=torch.int32, device=self.dev.device)
                check(lib.ma_bgzf_inflate_device(self.ctx.handle, d_in.data_ptr(), used, *[t.data_ptr() for t in tab],
                                                 len(so), self.dev.data_ptr() + self.len, self.cap - self.len,
                                                 status.data_ptr(), self.stream.cuda_stream), self.ctx.handle)
                bad = torch.nonzero(status).flatten().cpu()
            self.stream.synchronize()
            if bad.numel():
                m = int(bad[0])
                raise gzip.BadGzipFile(f"BGZF member {m} of a piece fails to inflate (status {int(status[m])})")
            self.h2d_bytes += used
            self.len += out
        if why == "other":
            # a member that is not BGZF: the gzip module reads the rest
            import io

            from .fqio import _Prefixed

            self._tail = gzip.GzipFile(fileobj=io.BufferedReader(_Prefixed(self.craw, self.fh)))
            self.craw = b""
            self._fill_host()
            return
        self.eof = why == "end"

    def _fill_host(self):
        torch = self.torch
        room = self.cap - self.len
        if room <= 0:
            return
        data = self._tail.read(room)
        if not data:
            self.eof = True
            return
        t = torch.from_numpy(np.frombuffer(data, np.uint8).copy())
        self.dev[self.len:self.len + len(data)].copy_(t)
        self.h2d_bytes += len(data)
        self.len += len(data)
        self.eof = False

    def consume(self, n: int):
        rest = self.len - n
        if rest > 0 and n > 0:
            with self.torch.cuda.stream(self.stream):
                self.dev[:rest].copy_(self.dev[n:self.len].clone())
            self.stream.synchronize()
        self.len = max(rest, 0)

    def close(self):
        self.fh.close()
        if self._tail is not None:
            self._tail.close()
        pinned.give(self._cbuf)
        self._cbuf = None


class _Grow:
    """A device array that keeps its contents when it grows."""

    def __init__(self, torch, dtype, dev):
        self.torch, self.dtype, self.dev = torch, dtype, dev
        self.t = torch.empty(0, dtype=dtype, device=dev)

    def ensure(self, n):
        if self.t.numel() >= n:
            return self.t
        new = self.torch.empty(max(n, 2 * self.t.numel()), dtype=self.dtype, device=self.dev)
        if self.t.numel():
            new[: self.t.numel()] = self.t
        self.t = new
        return new


class MappedChunk:
    """One chunk of the FASTQ files in HBM, split into records and mapped:
    the bytes of both mates (the arena), the record columns (R1 records then
    R2 records) and the mapping outputs."""

    def __init__(self, d_buf, n_bytes, n1, n_seq, max_len, cols, out):
        self.d_buf, self.n_bytes, self.n1, self.n_seq, self.max_len = d_buf, n_bytes, n1, n_seq, max_len
        self.cols, self.out = cols, out
        self.hits = ma_hits(*[out[f].data_ptr() for f in MapResult.FIELDS])
        self.arena = ma_fastq_arena(d_buf.data_ptr(), n_bytes, cols["name_off"].data_ptr(),
                                    cols["name_len"].data_ptr(), cols["seq_off"].data_ptr(),
                                    cols["seq_len"].data_ptr(), cols["qual_off"].data_ptr(),
                                    cols["qual_len"].data_ptr())


def _feed(path: str, chunk: int, torch, ctx, device_inflate: bool):
    """The feed of one FASTQ file: BGZF files (by the gzip suffix and the
    first member) inflated on the device when device_inflate is set, others
    through the host reader."""
    from .fqio import is_bgzf

    low = path.lower()
    if device_inflate and (low.endswith(".gz") or low.endswith(".gzip")) and is_bgzf(path):
        return _DeviceFeed(path, chunk, torch, ctx)
    return _Feed(path, chunk, torch)


def mapped_chunks(ctx, index, params, fq1, fq2, bs_r1, bs_r2, rules, batch_pairs, chunk_bytes, stream, tm,
                  before_map=None, device_inflate: bool = True):
    """Yields MappedChunk for consecutive pieces of the FASTQ file(s): the
    uncompressed bytes go to HBM once (the next piece is read on a host
    thread meanwhile), records are split under `rules` (MA_FASTQ_RULES_*),
    at most batch_pairs per piece, and mapped on `stream`.  Pairs follow the
    reference's readers: R2 running out first is "paired FASTQ length
    mismatch (R2 ended early)", extra R2 records are ignored.
    before_map(n_seq), when given, runs before a piece is mapped (it may
    raise).  tm["read_wait"] accumulates the seconds spent waiting for
    bytes."""
    import time

    import torch

    paired = len(str(fq2)) > 0
    dev = torch.device("cuda", ctx.device)
    sh = stream.cuda_stream
    p = params.to_c()
    feeds = [_feed(str(fq1), chunk_bytes, torch, ctx, device_inflate)] + (
        [_feed(str(fq2), chunk_bytes, torch, ctx, device_inflate)] if paired else [])
    tm.setdefault("fastq_h2d_bytes", 0)
    pool = ThreadPoolExecutor(max_workers=1)  # reads the next piece while the GPU maps this one
    pending = None
    o3 = (C.c_uint64 * 3)()
    try:
        for f in feeds:
            f.fill()
        while True:
            t0 = time.perf_counter()
            if pending is not None:
                pending.result()
                pending = None
            tm["read_wait"] += time.perf_counter() - t0
            if not feeds[0].len:
                return
            # both mates' bytes in one device buffer: the piece's arena
            sizes = [f.len for f in feeds]
            d_buf = torch.empty(sum(sizes) + 16, dtype=torch.uint8, device=dev)
            off = 0
            for f in feeds:
                if isinstance(f, _DeviceFeed):
                    d_buf[off:off + f.len].copy_(f.dev[: f.len])
                else:
                    d_buf[off:off + f.len].copy_(torch.from_numpy(f.pin[: f.len]), non_blocking=True)
                    tm["fastq_h2d_bytes"] += f.len
                off += f.len
            recs, rcs, counts = [], [], []
            for m, f in enumerate(feeds):
                base = sum(sizes[:m])
                r = {k: torch.empty(batch_pairs, dtype=torch.int64 if k.endswith("off") else torch.int32,
                                    device=dev) for k in REC_KEYS}
                rc = ma_fastq_records(*[r[k].data_ptr() for k in REC_KEYS])
                check(lib.ma_fastq_parse_rules_device(ctx.handle, d_buf.data_ptr() + base, sizes[m], int(f.eof),
                                                      batch_pairs, base, rules, C.byref(rc), o3, sh), ctx.handle)
                recs.append(r)
                rcs.append(rc)
                counts.append((int(o3[0]), int(o3[1]), int(o3[2])))
            n1 = counts[0][0]
            if paired and counts[1][0] < n1:
                if feeds[1].eof:
                    raise RuntimeError("paired FASTQ length mismatch (R2 ended early)")
                n1 = counts[1][0]  # R2's piece ended first: take the pairs both hold
            if n1 == 0:
                if feeds[0].eof:
                    return
                raise RuntimeError("FASTQ record larger than the read chunk")
            # bytes to drop from each feed: the span of its first n1 records;
            # the host buffers are free once the copies above are done
            used = []
            for m, f in enumerate(feeds):
                u = counts[m][1]
                if counts[m][0] != n1:
                    check(lib.ma_fastq_parse_rules_device(ctx.handle, d_buf.data_ptr() + sum(sizes[:m]), sizes[m],
                                                          int(f.eof), n1, sum(sizes[:m]), rules, C.byref(rcs[m]),
                                                          o3, sh), ctx.handle)
                    u = int(o3[1])
                used.append(u)
            stream.synchronize()

            def refill(used=used):
                for f, u in zip(feeds, used):
                    f.consume(u)
                    f.fill()

            pending = pool.submit(refill)
            max_len = max(max(c[2] for c in counts), params.seed_len)
            if max_len > MAX_LEN_CAP:
                raise RuntimeError("read longer than FM base cap (1024)")
            n_seq = n1 * (2 if paired else 1)
            if before_map is not None:
                before_map(n_seq)
            # mapper rows, R1 rows then R2 rows
            rows = torch.empty(n_seq * max_len, dtype=torch.uint8, device=dev)
            lens = torch.empty(n_seq, dtype=torch.int32, device=dev)
            for m, r in enumerate(recs):
                check(lib.ma_fastq_rows_device(ctx.handle, d_buf.data_ptr(), r["seq_off"].data_ptr(),
                                               r["seq_len"].data_ptr(), n1, max_len,
                                               rows.data_ptr() + m * n1 * max_len, lens.data_ptr() + m * n1 * 4,
                                               sh), ctx.handle)
            out = {f: torch.empty(n_seq, dtype=torch.int32, device=dev) for f in MapResult.FIELDS}
            chunk = MappedChunk(d_buf, int(sum(sizes)), n1, n_seq, max_len,
                                {k: torch.cat([r[k][:n1] for r in recs]) for k in REC_KEYS}, out)
            check(lib.ma_map_batch_device(ctx.handle, index.handle, rows.data_ptr(), lens.data_ptr(), n1,
                                          int(paired), max_len, bs_mode(bs_r1), bs_mode(bs_r2), C.byref(p),
                                          C.byref(chunk.hits), None, sh), ctx.handle)
            del recs, rcs
            yield chunk
            del chunk, d_buf, rows, lens, out
    finally:
        if pending is not None:
            pending.exception()
        pool.shutdown(wait=True)
        for f in feeds:
            if isinstance(f, _DeviceFeed):
                tm["fastq_h2d_bytes"] += f.h2d_bytes
            f.close()


def map_fastq_to_bam(ref_fa, fq1, out_bam, device: str = "auto", fq2: str = "", bs_r1: str = "",
                     bs_r2: str = "", params: FmParams | None = None, environ=None, kmer_k: int = 12,
                     kmer3_k: int | None = None, ctx: GpuContext | None = None, index: GpuIndex | None = None,
                     batch_pairs: int = 1 << 20, chunk_bytes: int = 512 << 20, level: int | None = None,
                     stats: dict | None = None, device_inflate: bool = True) -> int:
    """FASTQ -> sorted, duplicate-marked BGZF BAM; returns the mapped records.
    `stats`, when given, receives seconds spent per phase (waiting for FASTQ
    bytes, the per-batch device work, sort + gather, BGZF, writing) and the
    FASTQ bytes copied to the device (fastq_h2d_bytes: the compressed bytes
    of BGZF inputs inflated on the device, device_inflate)."""
    import time

    import torch

    tm = {"read_wait": 0.0, "batches": 0.0, "sort_gather": 0.0, "bgzf": 0.0, "write": 0.0}
    t_start = time.perf_counter()

    env = os.environ if environ is None else environ
    params = params or FmParams.from_env(env)
    level = int(_env(env, "METHYLGRAPHER_BAM_LEVEL", "1")) if level is None else level
    md_raw = _env(env, "METHYLGRAPHER_LINEAR_MARKDUP", "1").lower()
    do_markdup = md_raw not in ("0", "false", "no", "off")
    meta_cap = int(_env(env, SORT_CAP_ENV[0], str(SORT_CAP_ENV[1])))
    own_ctx = ctx is None
    ctx = ctx or GpuContext(select_device(device))
    own_index = index is None
    if index is None:
        k3 = min(params.seed_len, 18) if kmer3_k is None else kmer3_k
        index = GpuIndex(ctx, fm_prefix_from_ref(ref_fa), kmer_k=min(kmer_k, params.seed_len), kmer3_k=k3)
    paired = len(str(fq2)) > 0
    dev = torch.device("cuda", ctx.device)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    rg = _env(env, "METHYLGRAPHER_RG_ID", "mojo1").encode("ascii")
    d_rg = torch.tensor(list(rg) or [0], dtype=torch.uint8, device=dev)
    tids = canonical_rid_to_tid([c.name for c in index.contigs])
    d_tids = torch.from_numpy(tids).to(dev)
    header = bam_header(index.contigs, env)
    meta = {k: _Grow(torch, torch.int64 if t == np.uint64 else torch.int32, dev) for k, t in META_FIELDS}
    chunks, chunk_len = [], []
    n_reads = n_mapped = 0
    status = torch.zeros(3, dtype=torch.int64, device=dev)
    scope = contextlib.ExitStack()
    scope.enter_context(torch.cuda.stream(stream))  # torch work shares the pipeline's stream

    def cap_check(n_seq):
        if n_reads + n_seq > meta_cap:
            raise RuntimeError("FM sort cap exceeded; set METHYLGRAPHER_FM_SORT_CAP")

    pieces = mapped_chunks(ctx, index, params, fq1, fq2, bs_r1, bs_r2, MA_FASTQ_RULES_STREAM, batch_pairs,
                           chunk_bytes, stream, tm, cap_check, device_inflate=device_inflate)
    try:
        t_loop = time.perf_counter()
        for ch in pieces:
            n_seq = ch.n_seq
            dm = {k: meta[k].ensure(n_reads + n_seq) for k, _ in META_FIELDS}
            dmeta = ma_bam_meta(*[dm[k].data_ptr() for k, _ in META_FIELDS])
            seq_total = int(ch.cols["seq_len"].sum().item())
            name_total = int(ch.cols["name_len"].sum().item())
            cap = n_seq * (64 + len(rg)) + name_total + 2 * seq_total
            d_chunk = torch.empty(cap, dtype=torch.uint8, device=dev)
            tile = ma_bam_tile(n_reads, n_mapped, 0, meta_cap, len(chunks))
            check(lib.ma_emit_bam_batch_device(ctx.handle, C.byref(ch.hits), ch.n1, int(paired), C.byref(ch.arena),
                                               d_tids.data_ptr(), int(tids.size), d_rg.data_ptr(), len(rg),
                                               d_chunk.data_ptr(), cap, C.byref(dmeta), C.byref(tile),
                                               status.data_ptr(), sh), ctx.handle)
            stream.synchronize()
            st = status.cpu().numpy()
            if st[2] or st[0] > cap:
                raise RuntimeError("BAM batch buffer overflow")
            chunks.append(d_chunk)
            chunk_len.append(int(st[0]))
            n_reads += n_seq
            n_mapped += int(st[1])
            del ch
        tm["batches"] = time.perf_counter() - t_loop - tm["read_wait"]
        # ---- sort, mark, gather, compress ----
        t0 = time.perf_counter()
        total_records = int(sum(chunk_len))
        d_stream = torch.empty(len(header) + total_records + 16, dtype=torch.uint8, device=dev)
        d_stream[: len(header)].copy_(torch.frombuffer(bytearray(header), dtype=torch.uint8))
        if n_reads:
            perm = torch.empty(n_reads, dtype=torch.int32, device=dev)
            is_dup = torch.empty(n_reads, dtype=torch.int32, device=dev)
            mt = {k: meta[k].t for k, _ in META_FIELDS}
            check(lib.ma_sort_markdup_device(ctx.handle, n_reads, mt["coord"].data_ptr(), mt["dhi"].data_ptr(),
                                             mt["dlo"].data_ptr(), mt["score"].data_ptr(), mt["pair"].data_ptr(),
                                             is_dup.data_ptr(), perm.data_ptr(), int(do_markdup), None, None, sh),
                  ctx.handle)
            d_ptrs = torch.tensor([c.data_ptr() for c in chunks], dtype=torch.int64, device=dev)
            d_lens = torch.tensor(chunk_len, dtype=torch.int64, device=dev)
            gst = torch.zeros(2, dtype=torch.int64, device=dev)
            check(lib.ma_gather_sorted_bam_device(ctx.handle, n_reads, perm.data_ptr(), mt["rec"].data_ptr(),
                                                  mt["len"].data_ptr(), is_dup.data_ptr(), int(do_markdup),
                                                  d_ptrs.data_ptr(), d_lens.data_ptr(), len(chunks),
                                                  d_stream.data_ptr() + len(header), total_records,
                                                  gst.data_ptr(), sh), ctx.handle)
            stream.synchronize()
            g = gst.cpu().numpy()
            if g[1] or int(g[0]) != total_records:
                raise RuntimeError("sorted record stream does not match the tile")
            del chunks
        tm["sort_gather"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        n_stream = len(header) + total_records
        cap = int(lib.ma_bgzf_bound(n_stream))
        d_out = torch.empty(cap, dtype=torch.uint8, device=dev)
        got = C.c_uint64(0)
        check(lib.ma_bgzf_compress_device(ctx.handle, d_stream.data_ptr(), n_stream, level, 1, d_out.data_ptr(), cap,
                                          C.byref(got), sh), ctx.handle)
        tm["bgzf"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        host_out = pinned.take(got.value)
        try:
            host_out[: got.value].copy_(d_out[: got.value])
            with ParallelWriter(out_bam) as fw:
                fw.write(memoryview(host_out.numpy())[: got.value])
        finally:
            pinned.give(host_out)
        tm["write"] = time.perf_counter() - t0
        tm["total"] = time.perf_counter() - t_start
        if stats is not None:
            stats.update({k: round(v, 4) for k, v in tm.items()})
    finally:
        pieces.close()
        stream.synchronize()
        scope.close()
        if own_index:
            index.close()
        if own_ctx:
            ctx.close()
    return n_mapped
