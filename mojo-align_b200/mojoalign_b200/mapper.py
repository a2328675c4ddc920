"""GPU mapping through the C ABI: contexts, resident indexes, batches.

This is the function-level drop-in for the FM engine's batch step
(_fm_fire_batch, fq2bam-meth/src/linear_gpu_fm.mojo:2279-2417): one call
converts + packs the reads on the device, runs seed/extend and (paired)
mate rescue, and returns the seven per-read output arrays of
fm_seed_extend_kernel (L1183-1189) plus optional side outputs.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import MA_BS_C2T, MA_BS_G2A, MA_BS_NONE, check, fspath, lib, ma_debug, ma_hits, ma_index_info, ptr
from .params import FmParams

BS_MODES = {"": MA_BS_NONE, "C2T": MA_BS_C2T, "G2A": MA_BS_G2A}


def bs_mode(mode) -> int:
    """_bs_mode (fq2bam-meth/src/linear_fastq.mojo:29-34); ints pass through."""
    if isinstance(mode, int):
        return mode
    return BS_MODES.get(mode, MA_BS_NONE)


class GpuContext:
    """One CUDA device context (one per host thread)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib.ma_ctx_create(device, C.byref(h)))
        self.handle = h
        self.device = device

    def hbm_info(self) -> tuple[int, int]:
        f, t = C.c_uint64(), C.c_uint64()
        check(lib.ma_hbm_info(self.handle, C.byref(f), C.byref(t)), self.handle)
        return f.value, t.value

    def last_launch_count(self) -> int:
        return lib.ma_last_launch_count(self.handle)

    def set_tuning(self, seed_kernel: int = 2, stage1_endpoints: int = 1, stage2_blocks_per_sm: int = 0,
                   reg_level: int = 2, stage1_max_rows: int = 1, stage2_first_wave: int = 1,
                   wave_endpoints: int = 8, wave_loci_per_read: int = 4, wave_max_rounds: int = 0,
                   wave_growth: int = 1) -> None:
        """Result-neutral kernel choices (see ma_tuning in the C header)."""
        t = _lib.ma_tuning(seed_kernel, stage1_endpoints, stage2_blocks_per_sm, reg_level, stage1_max_rows,
                           stage2_first_wave, wave_endpoints, wave_loci_per_read, wave_max_rounds, wave_growth)
        check(lib.ma_ctx_set_tuning(self.handle, C.byref(t)), self.handle)

    def set_graphs(self, enable: bool = True) -> None:
        """Device mapping calls replay a captured CUDA graph while their
        arguments repeat (see ma_ctx_set_graphs)."""
        check(lib.ma_ctx_set_graphs(self.handle, int(enable)), self.handle)

    def set_pipeline(self, first_chunk_pairs: int = 0, growth_percent: int = 50, max_chunk_pairs: int = 0,
                     compute_streams: int = 3) -> None:
        """Chunking of map_batch's copy / compute pipeline (see ma_pipeline)."""
        p = _lib.ma_pipeline(first_chunk_pairs, growth_percent, max_chunk_pairs, compute_streams)
        check(lib.ma_ctx_set_pipeline(self.handle, C.byref(p)), self.handle)

    def pipeline(self) -> dict:
        p = _lib.ma_pipeline()
        check(lib.ma_ctx_get_pipeline(self.handle, C.byref(p)), self.handle)
        return {f: getattr(p, f) for f, _ in p._fields_}

    def tuning(self) -> dict:
        t = _lib.ma_tuning()
        check(lib.ma_ctx_get_tuning(self.handle, C.byref(t)), self.handle)
        return {f: getattr(t, f) for f, _ in t._fields_}

    def set_profiling(self, flags: int) -> None:
        check(lib.ma_ctx_set_profiling(self.handle, flags), self.handle)

    def kernel_ms(self) -> list[float]:
        v = (C.c_float * 4)()
        check(lib.ma_ctx_kernel_ms(self.handle, v), self.handle)
        return list(v)

    def wave_ms(self) -> list[float]:
        """Wavefront search, eval, finalize ms of the last profiled call, the
        rounds timed and the stage-2 ms (see ma_ctx_wave_ms)."""
        v = (C.c_float * 5)()
        check(lib.ma_ctx_wave_ms(self.handle, v), self.handle)
        return list(v)

    def traffic_stage2(self) -> list[int]:
        """The stage-2 part of traffic() (see ma_ctx_traffic_stage2)."""
        v = (C.c_uint64 * 12)()
        check(lib.ma_ctx_traffic_stage2(self.handle, v), self.handle)
        return list(v)

    def traffic(self) -> list[int]:
        v = (C.c_uint64 * 12)()
        check(lib.ma_ctx_traffic(self.handle, v), self.handle)
        return list(v)

    def gather_gbps(self, buffer_bytes: int, line_bytes: int, n_loads: int = 1 << 30) -> float:
        g = C.c_double()
        check(lib.ma_bench_gather(self.handle, buffer_bytes, line_bytes, n_loads, C.byref(g)), self.handle)
        return g.value

    def close(self) -> None:
        if self.handle:
            lib.ma_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Contig:
    name: str
    offset: int
    length: int


class GpuIndex:
    """A bwa 0.7 FM-index made resident in HBM (FmIndex.load + upload)."""

    def __init__(self, ctx: GpuContext, prefix, kmer_k: int = 12, kmer3_k: int = 0, hbm_budget_bytes: int = 0,
                 wide_rows: bool = False, occ_super_shift: int = 0, prep_chunk_rows: int = 0, at_k: int = 0,
                 at_seed_len: int = 0):
        """Layout options (result-neutral): wide_rows stores 40-bit SA rows
        even for short texts, occ_super_shift sets the Occ superblock
        (log2 positions, 0 = 31), prep_chunk_rows the SA rows per
        preparation pass (0 = 2^30), at_k / at_seed_len the A/T window
        outcome table (windows of at_k bases, used by calls with seed_len
        at_seed_len; 0 = none)."""
        h = C.c_void_p()
        opt = _lib.ma_index_options(kmer_k, kmer3_k, hbm_budget_bytes, int(wide_rows), occ_super_shift,
                                    prep_chunk_rows, at_k, at_seed_len)
        check(lib.ma_index_open(ctx.handle, fspath(prefix), C.byref(opt), C.byref(h)), ctx.handle)
        self.handle = h
        self.ctx = ctx
        info = ma_index_info()
        check(lib.ma_index_get_info(h, C.byref(info)))
        self.info = info
        self.contigs = []
        for i in range(info.n_contigs):
            nm, off, ln = C.c_char_p(), C.c_uint64(), C.c_uint64()
            check(lib.ma_index_contig(h, i, C.byref(nm), C.byref(off), C.byref(ln)))
            self.contigs.append(Contig(nm.value.decode(), off.value, ln.value))

    def close(self) -> None:
        if self.handle:
            lib.ma_index_close(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def page_locked(n: int, dtype) -> np.ndarray:
    """A page-locked host array of n elements (its memory stays valid while
    the array, or a view of it, lives)."""
    import torch

    dt = np.dtype(dtype)
    t = torch.empty(n * dt.itemsize, dtype=torch.uint8, pin_memory=True)
    a = t.numpy().view(dt)
    return a


@dataclass
class MapResult:
    rid: np.ndarray
    pos: np.ndarray
    mapq: np.ndarray
    flag: np.ndarray
    sl: np.ndarray
    sr: np.ndarray
    nm: np.ndarray
    uk: np.ndarray | None = None
    ul: np.ndarray | None = None
    us: np.ndarray | None = None
    e: np.ndarray | None = None
    score: np.ndarray | None = None

    FIELDS = ("rid", "pos", "mapq", "flag", "sl", "sr", "nm")
    DEBUG = ("uk", "ul", "us", "e", "score")

    @classmethod
    def empty(cls, n: int, debug: bool, pinned: bool = False) -> "MapResult":
        """Output arrays for n reads; pinned=True allocates them page-locked,
        so that map_batch copies the results straight into them."""
        alloc = page_locked if pinned else np.empty
        r = cls(alloc(n, np.int32), alloc(n, np.uint32), alloc(n, np.uint32), alloc(n, np.int32),
                alloc(n, np.uint32), alloc(n, np.uint32), alloc(n, np.uint32))
        if debug:
            r.uk = alloc(n, np.uint64)
            r.ul = alloc(n, np.uint64)
            r.us = alloc(n, np.int32)
            r.e = alloc(n, np.int32)
            r.score = alloc(n, np.int32)
        return r

    def hits(self) -> ma_hits:
        return ma_hits(*[ptr(getattr(self, f)) for f in self.FIELDS])

    def debug(self) -> ma_debug | None:
        if self.uk is None:
            return None
        return ma_debug(*[ptr(getattr(self, f)) for f in self.DEBUG])


def map_batch(ctx: GpuContext, index: GpuIndex, bases: np.ndarray, lens: np.ndarray, n1: int, paired: bool,
              max_len: int, bs_r1="C2T", bs_r2="G2A", params: FmParams | None = None, debug: bool = False,
              out: MapResult | None = None) -> MapResult:
    """Maps one batch of padded ASCII reads (R1 rows, then R2 rows)."""
    params = params or FmParams()
    n_seq = n1 * (2 if paired else 1)
    bases = np.ascontiguousarray(bases, dtype=np.uint8)
    lens = np.ascontiguousarray(lens, dtype=np.uint32)
    if bases.size < n_seq * max_len or lens.size < n_seq:
        raise ValueError("bases / lens smaller than the batch")
    res = out if out is not None else MapResult.empty(n_seq, debug)
    p = params.to_c()
    hits = res.hits()
    dbg = res.debug()
    rc = lib.ma_map_batch(ctx.handle, index.handle, ptr(bases), ptr(lens), n1, int(paired), max_len,
                          bs_mode(bs_r1), bs_mode(bs_r2), C.byref(p), C.byref(hits),
                          C.byref(dbg) if dbg is not None else None)
    check(rc, ctx.handle)
    return res


def map_batch_device(ctx: GpuContext, index: GpuIndex, d_bases: int, d_lens: int, n1: int, paired: bool,
                     max_len: int, d_out: dict, bs_r1="C2T", bs_r2="G2A", params: FmParams | None = None,
                     d_debug: dict | None = None, stream: int | None = None) -> None:
    """Same on device pointers (ints); d_out / d_debug map field -> pointer."""
    params = params or FmParams()
    p = params.to_c()
    hits = ma_hits(*[d_out[f] for f in MapResult.FIELDS])
    dbg = ma_debug(*[d_debug[f] for f in MapResult.DEBUG]) if d_debug else None
    rc = lib.ma_map_batch_device(ctx.handle, index.handle, d_bases, d_lens, n1, int(paired), max_len,
                                 bs_mode(bs_r1), bs_mode(bs_r2), C.byref(p), C.byref(hits),
                                 C.byref(dbg) if dbg is not None else None, stream)
    check(rc, ctx.handle)


def probe_index(prefix, kmer_k: int = 12, kmer3_k: int = 0, at_k: int = 0) -> ma_index_info:
    """Validates a bwa index on the host (no GPU) and reports its HBM need,
    with the A/T window outcome table of at_k bases (2^at_k entries of 16
    bytes) when at_k > 0."""
    if at_k < 0 or at_k > 30:
        raise _lib.MojoAlignError(_lib.MA_ERR_ARG, "at_k must be in 0..30")
    info = ma_index_info()
    check(lib.ma_index_probe(fspath(prefix), kmer_k, kmer3_k, C.byref(info)))
    if at_k:
        info.device_bytes += (1 << at_k) * 16
    return info


def build_index(fasta, out_prefix, bwameth_c2t: bool = True, sa_intv: int = 32, device: int = -1,
                batch_suffixes: int = 0) -> None:
    """Writes a bwa-0.7 FM-index (optionally of the bwa-meth c2t text).
    device >= 0 builds the BWT on that GPU, at most batch_suffixes suffixes
    sorted at once (0 = what fits); -1 sorts on the host."""
    if batch_suffixes:
        check(lib.ma_index_build_batched(fspath(fasta), fspath(out_prefix), int(bwameth_c2t), sa_intv, device,
                                         batch_suffixes))
    else:
        check(lib.ma_index_build(fspath(fasta), fspath(out_prefix), int(bwameth_c2t), sa_intv, device))


__all__ = ["GpuContext", "GpuIndex", "MapResult", "map_batch", "map_batch_device", "build_index", "probe_index",
           "bs_mode", "_lib"]
