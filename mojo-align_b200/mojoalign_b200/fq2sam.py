"""FASTQ to SAM text with every per-read stage on the GPU.

The .sam destination of map_fastq_fm_gpu (fq2bam-meth/src/linear_gpu_fm.mojo:
1028-3341 without emit_bam): the reference reads FASTQ with its Python
FastqPairReader (fq2bam-meth/python/fastq_batch.py), maps each batch on the
GPU, copies the outputs back and formats one LinearHit per read on the host
(_hit_from_fm, pair_hits, hit_to_sam_line).  Here the uncompressed FASTQ
bytes are copied to the device once and the finished text comes back:

    host: read / gunzip FASTQ  ->  HBM: split records under the pair
      reader's rules (ma_fastq_parse_rules_device)
      -> mapper rows (ma_fastq_rows_device) -> map (ma_map_batch_device)
      -> SAM lines (ma_emit_sam_batch_device; the FASTQ bytes are the arena)
      -> host: write the text (a writer thread, overlapped with the next
         chunk's device work).

The file is the reference's: the header of _write_sam_header_fm (L40-76),
then the lines in input order (R1, R2 per pair).  The text does not depend on
the chunk or batch sizes.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
from concurrent.futures import ThreadPoolExecutor

from . import pinned
from ._lib import MA_FASTQ_RULES_PAIR_READER, check, lib, ma_fastq_arena, ma_fastq_records, ma_hits
from .fq2bam import MAX_LEN_CAP, REC_KEYS, _Feed
from .fqio import ParallelWriter
from .linear_fm import _env_str, fm_prefix_from_ref, sam_header, select_device
from .mapper import GpuContext, GpuIndex, MapResult, bs_mode
from .params import FmParams
from .sam import LINE_FIXED, SamContigs, sam_error


def map_fastq_to_sam(ref_fa, fq1, out_sam, device: str = "auto", fq2: str = "", bs_r1: str = "", bs_r2: str = "",
                     params: FmParams | None = None, environ=None, kmer_k: int = 12, kmer3_k: int | None = None,
                     ctx: GpuContext | None = None, index: GpuIndex | None = None, batch_pairs: int = 1 << 20,
                     chunk_bytes: int = 256 << 20, stats: dict | None = None) -> int:
    """FASTQ -> SAM; returns the mapped records.  `stats`, when given,
    receives seconds per phase (waiting for FASTQ bytes, device work per
    chunk, waiting for the writer) and the SAM emitter's device time
    (CUDA events on the pipeline's stream) with the lines, text bytes and
    arena bytes (name + SEQ + QUAL) it handled."""
    import time

    import torch

    tm = {"read_wait": 0.0, "batches": 0.0, "write_wait": 0.0, "emit_kernel_s": 0.0, "emit_lines": 0,
          "emit_text_bytes": 0, "emit_arena_bytes": 0}
    t_start = time.perf_counter()
    env = os.environ if environ is None else environ
    params = params or FmParams.from_env(env)
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
    rg = _env_str("METHYLGRAPHER_RG_ID", "mojo1", env).encode()
    d_rg = torch.tensor(list(rg) or [0], dtype=torch.uint8, device=dev)
    contigs = SamContigs.from_names([c.name for c in index.contigs])
    d_contigs = contigs.to_device(torch, dev)
    p = params.to_c()
    feeds = [_Feed(str(fq1), chunk_bytes, torch)] + ([_Feed(str(fq2), chunk_bytes, torch)] if paired else [])
    reader = ThreadPoolExecutor(max_workers=1)  # reads the next chunk while the GPU maps this one
    writer = ThreadPoolExecutor(max_workers=1)  # writes chunk k while chunk k+1 maps
    pending = None
    host_out = [None, None]  # pinned text buffers, alternating between chunks
    writes = [None, None]
    n_mapped = 0
    k_chunk = 0
    status = torch.zeros(3, dtype=torch.int64, device=dev)
    o3 = (C.c_uint64 * 3)()
    scope = contextlib.ExitStack()
    scope.enter_context(torch.cuda.stream(stream))
    fh = ParallelWriter(out_sam)
    try:
        fh.write(sam_header(index.contigs, env).encode())
        for f in feeds:
            f.fill()
        while True:
            t0 = time.perf_counter()
            if pending is not None:
                pending.result()
                pending = None
            tm["read_wait"] += time.perf_counter() - t0
            t0 = time.perf_counter()
            if not feeds[0].len:
                break
            sizes = [f.len for f in feeds]
            d_buf = torch.empty(sum(sizes) + 16, dtype=torch.uint8, device=dev)
            off = 0
            for f in feeds:
                d_buf[off:off + f.len].copy_(torch.from_numpy(f.pin[: f.len]), non_blocking=True)
                off += f.len
            recs, rcs, counts = [], [], []
            for m, f in enumerate(feeds):
                base = sum(sizes[:m])
                r = {k: torch.empty(batch_pairs, dtype=torch.int64 if k.endswith("off") else torch.int32,
                                    device=dev) for k in REC_KEYS}
                rc = ma_fastq_records(*[r[k].data_ptr() for k in REC_KEYS])
                check(lib.ma_fastq_parse_rules_device(ctx.handle, d_buf.data_ptr() + base, sizes[m], int(f.eof),
                                                      batch_pairs, base, MA_FASTQ_RULES_PAIR_READER, C.byref(rc), o3,
                                                      sh), ctx.handle)
                recs.append(r)
                rcs.append(rc)
                counts.append((int(o3[0]), int(o3[1]), int(o3[2])))
            n1 = counts[0][0]
            if paired and counts[1][0] < n1:
                if feeds[1].eof:  # FastqPairReader.read_batch, fastq_batch.py:296-298
                    raise RuntimeError("paired FASTQ length mismatch (R2 ended early)")
                n1 = counts[1][0]  # R2's chunk ended first: take the pairs both hold
            if n1 == 0:
                if feeds[0].eof:
                    break
                raise RuntimeError("FASTQ record larger than the read chunk")
            used = []
            for m, f in enumerate(feeds):
                u = counts[m][1]
                if counts[m][0] != n1:
                    check(lib.ma_fastq_parse_rules_device(ctx.handle, d_buf.data_ptr() + sum(sizes[:m]), sizes[m],
                                                          int(f.eof), n1, sum(sizes[:m]), MA_FASTQ_RULES_PAIR_READER,
                                                          C.byref(rcs[m]), o3, sh), ctx.handle)
                    u = int(o3[1])
                used.append(u)
            stream.synchronize()

            def refill(used=used):
                for f, u in zip(feeds, used):
                    f.consume(u)
                    f.fill()

            pending = reader.submit(refill)
            max_len = max(max(c[2] for c in counts), params.seed_len)
            if max_len > MAX_LEN_CAP:
                raise RuntimeError("read longer than FM base cap (1024)")
            n_seq = n1 * (2 if paired else 1)
            rows = torch.empty(n_seq * max_len, dtype=torch.uint8, device=dev)
            lens = torch.empty(n_seq, dtype=torch.int32, device=dev)
            for m, r in enumerate(recs):
                check(lib.ma_fastq_rows_device(ctx.handle, d_buf.data_ptr(), r["seq_off"].data_ptr(),
                                               r["seq_len"].data_ptr(), n1, max_len,
                                               rows.data_ptr() + m * n1 * max_len, lens.data_ptr() + m * n1 * 4,
                                               sh), ctx.handle)
            out = {f: torch.empty(n_seq, dtype=torch.int32, device=dev) for f in MapResult.FIELDS}
            hits = ma_hits(*[out[f].data_ptr() for f in MapResult.FIELDS])
            check(lib.ma_map_batch_device(ctx.handle, index.handle, rows.data_ptr(), lens.data_ptr(), n1,
                                          int(paired), max_len, bs_mode(bs_r1), bs_mode(bs_r2), C.byref(p),
                                          C.byref(hits), None, sh), ctx.handle)
            cols = {k: torch.cat([r[k][:n1] for r in recs]) for k in REC_KEYS}
            arena = ma_fastq_arena(d_buf.data_ptr(), int(sum(sizes)), cols["name_off"].data_ptr(),
                                   cols["name_len"].data_ptr(), cols["seq_off"].data_ptr(),
                                   cols["seq_len"].data_ptr(), cols["qual_off"].data_ptr(),
                                   cols["qual_len"].data_ptr())
            # the text of the chunk fits in: per line the fixed fields and
            # contig names, three bytes per name byte, SEQ, QUAL
            cap = n_seq * (LINE_FIXED + len(rg) + 2 * contigs.max_name) + 3 * int(
                cols["name_len"].sum().item()) + sum(sizes)
            d_text = torch.empty(cap, dtype=torch.uint8, device=dev)
            if stats is not None:
                ev = [torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)]
                ev[0].record(stream)
            check(lib.ma_emit_sam_batch_device(ctx.handle, C.byref(hits), n1, int(paired), C.byref(arena),
                                               C.byref(d_contigs.c), d_rg.data_ptr(), len(rg), d_text.data_ptr(),
                                               cap, status.data_ptr(), sh), ctx.handle)
            if stats is not None:
                ev[1].record(stream)
            st = status.cpu().numpy()  # synchronizes the stream
            if stats is not None:
                tm["emit_kernel_s"] += ev[0].elapsed_time(ev[1]) / 1000.0
                tm["emit_lines"] += n_seq
                tm["emit_text_bytes"] += int(st[0])
                tm["emit_arena_bytes"] += sum(int(cols[k].sum().item()) for k in ("name_len", "seq_len", "qual_len"))
            if st[2]:
                raise RuntimeError(sam_error(int(st[2])))
            n_text = int(st[0])
            n_mapped += int(st[1])
            slot = k_chunk & 1
            t1 = time.perf_counter()
            if writes[slot] is not None:
                writes[slot].result()
                writes[slot] = None
            tm["write_wait"] += time.perf_counter() - t1
            if host_out[slot] is None or host_out[slot].numel() < n_text:
                pinned.give(host_out[slot])
                host_out[slot] = None
                host_out[slot] = pinned.take(n_text)
            host_out[slot][:n_text].copy_(d_text[:n_text], non_blocking=True)
            stream.synchronize()
            writes[slot] = writer.submit(fh.write, memoryview(host_out[slot].numpy())[:n_text])
            k_chunk += 1
            del d_buf, rows, out, cols, d_text
            tm["batches"] += time.perf_counter() - t0
        t1 = time.perf_counter()
        for w in writes:
            if w is not None:
                w.result()
        tm["write_wait"] += time.perf_counter() - t1
        tm["total"] = time.perf_counter() - t_start
        if stats is not None:
            stats.update({k: round(v, 6) if isinstance(v, float) else v for k, v in tm.items()})
    finally:
        if pending is not None:
            pending.exception()
        reader.shutdown(wait=True)
        writer.shutdown(wait=True)
        fh.close()
        for t in host_out:
            pinned.give(t)
        stream.synchronize()
        scope.close()
        for f in feeds:
            f.close()
        if own_index:
            index.close()
        if own_ctx:
            ctx.close()
    return n_mapped
