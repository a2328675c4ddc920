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
from ._lib import MA_FASTQ_RULES_PAIR_READER, check, lib
from .fq2bam import mapped_chunks
from .fqio import ParallelWriter
from .linear_fm import _env_str, fm_prefix_from_ref, sam_header, select_device
from .mapper import GpuContext, GpuIndex
from .params import FmParams
from .sam import LINE_FIXED, SamContigs, sam_error


def map_fastq_to_sam(ref_fa, fq1, out_sam, device: str = "auto", fq2: str = "", bs_r1: str = "", bs_r2: str = "",
                     params: FmParams | None = None, environ=None, kmer_k: int = 12, kmer3_k: int | None = None,
                     ctx: GpuContext | None = None, index: GpuIndex | None = None, batch_pairs: int = 1 << 20,
                     chunk_bytes: int = 256 << 20, stats: dict | None = None, device_inflate: bool = True) -> int:
    """FASTQ -> SAM; returns the mapped records.  `stats`, when given,
    receives seconds per phase (waiting for FASTQ bytes, device work per
    chunk, waiting for the writer), the SAM emitter's device time (CUDA
    events on the pipeline's stream) with the lines, text bytes and arena
    bytes (name + SEQ + QUAL) it handled, and the FASTQ bytes copied to the
    device (fastq_h2d_bytes: the compressed bytes of BGZF inputs inflated on
    the device, device_inflate)."""
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
    writer = ThreadPoolExecutor(max_workers=1)  # writes chunk k while chunk k+1 maps
    host_out = [None, None]  # pinned text buffers, alternating between chunks
    writes = [None, None]
    n_mapped = 0
    k_chunk = 0
    status = torch.zeros(3, dtype=torch.int64, device=dev)
    scope = contextlib.ExitStack()
    scope.enter_context(torch.cuda.stream(stream))
    fh = ParallelWriter(out_sam)
    pieces = mapped_chunks(ctx, index, params, fq1, fq2, bs_r1, bs_r2, MA_FASTQ_RULES_PAIR_READER, batch_pairs,
                           chunk_bytes, stream, tm, device_inflate=device_inflate)
    try:
        fh.write(sam_header(index.contigs, env).encode())
        t_loop = time.perf_counter()
        for ch in pieces:
            n_seq = ch.n_seq
            cols = ch.cols
            # the text of the chunk fits in: per line the fixed fields and
            # contig names, three bytes per name byte, SEQ, QUAL
            cap = n_seq * (LINE_FIXED + len(rg) + 2 * contigs.max_name) + 3 * int(
                cols["name_len"].sum().item()) + ch.n_bytes
            d_text = torch.empty(cap, dtype=torch.uint8, device=dev)
            if stats is not None:
                ev = [torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)]
                ev[0].record(stream)
            check(lib.ma_emit_sam_batch_device(ctx.handle, C.byref(ch.hits), ch.n1, int(paired), C.byref(ch.arena),
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
            del ch, cols, d_text
        tm["batches"] = time.perf_counter() - t_loop - tm["read_wait"] - tm["write_wait"]
        t1 = time.perf_counter()
        for w in writes:
            if w is not None:
                w.result()
        tm["write_wait"] += time.perf_counter() - t1
        tm["total"] = time.perf_counter() - t_start
        if stats is not None:
            stats.update({k: round(v, 6) if isinstance(v, float) else v for k, v in tm.items()})
    finally:
        pieces.close()
        writer.shutdown(wait=True)
        fh.close()
        for t in host_out:
            pinned.give(t)
        stream.synchronize()
        scope.close()
        if own_index:
            index.close()
        if own_ctx:
            ctx.close()
    return n_mapped
