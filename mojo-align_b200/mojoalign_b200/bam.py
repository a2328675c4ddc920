"""BAM records of mapped batches, packed on the GPU.

Host side of ma_emit_bam_batch / ma_emit_bam_batch_device, with the
contract of fq2bam-meth/src/linear_gpu_fm.mojo:
- `BatchArena`     the FASTQ arena of a batch as fq_export_ptrs
                   (linear_fastq.mojo:518-544) exposes it: one byte array and
                   per-record (offset, length) of name, original bases and
                   qualities, R1 records then R2 records.
- `BamTile`        the tile metadata arrays h_coord .. h_pair
                   (L2133-2139) and the n_reads / n_mapped / n_total /
                   tile_chunks counters _emit_bam_from_batch advances.
- `emit_bam_from_batch`  one batch (L669-984): returns the packed records
                   and advances the tile; raises MojoAlignError with the
                   reference's messages ("FM sort cap exceeded", "BAM batch
                   buffer overflow").
- `rid_to_tid_table`  contig index -> SAM tid over canonical contig names
                   (_rid_to_tid_table, L423-435).
- `sort_markdup`   gpu_sort_markdup (linear_gpu_sort.mojo:24-560) on a tile's
                   metadata: coordinate permutation, duplicate flags and the
                   duplicate-key order.
- `gather_sorted`  the record gather of _gather_perm_to_writer (L177-225):
                   the tile's records in coordinate order, duplicates flagged.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._lib import check, lib, ma_bam_meta, ma_bam_tile, ma_fastq_arena, ma_hits, ptr
from .fastq import FastqArena

META_FIELDS = (("coord", np.uint64), ("dhi", np.uint64), ("dlo", np.uint64), ("rec", np.uint64),
               ("len", np.uint32), ("score", np.uint32), ("pair", np.uint32))
HIT_FIELDS = (("rid", np.int32), ("pos", np.uint32), ("mapq", np.uint32), ("flag", np.int32),
              ("sl", np.uint32), ("sr", np.uint32), ("nm", np.uint32))


@dataclass
class BatchArena:
    data: np.ndarray
    name_off: np.ndarray
    name_len: np.ndarray
    orig_off: np.ndarray
    orig_len: np.ndarray
    qual_off: np.ndarray | None
    qual_len: np.ndarray | None

    @property
    def n_seq(self) -> int:
        return int(self.name_off.size)

    @classmethod
    def from_records(cls, records, with_quals: bool = True) -> "BatchArena":
        """records: (name, original bases, qualities) byte strings, R1 then R2."""
        n = len(records)
        offs = np.zeros((3, n), np.uint64)
        lens = np.zeros((3, n), np.uint32)
        parts = []
        pos = 0
        for i, rec in enumerate(records):
            for k in range(3 if with_quals else 2):
                b = bytes(rec[k])
                offs[k, i] = pos
                lens[k, i] = len(b)
                parts.append(b)
                pos += len(b)
        data = np.frombuffer(b"".join(parts), np.uint8).copy() if pos else np.zeros(0, np.uint8)
        return cls(data, offs[0].copy(), lens[0].copy(), offs[1].copy(), lens[1].copy(),
                   offs[2].copy() if with_quals else None, lens[2].copy() if with_quals else None)

    @classmethod
    def from_fastq(cls, a: FastqArena, paired: bool) -> "BatchArena":
        recs = list(zip(a.name1, a.orig1, a.qual1))
        if paired:
            recs += list(zip(a.name2, a.orig2, a.qual2))
        return cls.from_records(recs)

    def to_c(self) -> ma_fastq_arena:
        return ma_fastq_arena(ptr(self.data), int(self.data.size), ptr(self.name_off), ptr(self.name_len),
                              ptr(self.orig_off), ptr(self.orig_len), ptr(self.qual_off), ptr(self.qual_len))


@dataclass
class BamTile:
    """Tile state of the FM BAM path: counters and, unless the metadata lives
    elsewhere (host_meta=False: the device forms), the host metadata arrays."""
    meta_cap: int
    n_reads: int = 0
    n_mapped: int = 0
    n_total: int = 0
    chunk: int = 0
    meta: dict = field(default_factory=dict)
    host_meta: bool = True

    def __post_init__(self):
        if not self.meta and self.host_meta:
            self.meta = {k: np.zeros(self.meta_cap, t) for k, t in META_FIELDS}

    def to_c(self) -> ma_bam_tile:
        return ma_bam_tile(self.n_reads, self.n_mapped, self.n_total, self.meta_cap, self.chunk)

    def meta_c(self) -> ma_bam_meta:
        return ma_bam_meta(*[ptr(self.meta[k]) for k, _ in META_FIELDS])


def _hits_c(hits) -> tuple[ma_hits, list]:
    keep = [np.ascontiguousarray(getattr(hits, k) if not isinstance(hits, dict) else hits[k], dtype=t)
            for k, t in HIT_FIELDS]
    return ma_hits(*[ptr(a) for a in keep]), keep


def emit_bam_from_batch(ctx, hits, n1: int, paired: bool, arena: BatchArena, rid_to_tid, rg: bytes,
                        tile: BamTile, bam_cap: int, out: np.ndarray | None = None) -> np.ndarray:
    """Packs one mapped batch; returns the records (a view of `out`)."""
    h, keep = _hits_c(hits)
    tids = np.ascontiguousarray(rid_to_tid, dtype=np.int32)
    rgb = np.frombuffer(bytes(rg), np.uint8) if rg else np.zeros(0, np.uint8)
    if out is None or out.size < bam_cap:
        out = np.empty(max(bam_cap, 1), np.uint8)
    n = C.c_uint64(0)
    ca = arena.to_c()
    meta = tile.meta_c()
    t = tile.to_c()
    rc = lib.ma_emit_bam_batch(ctx.handle, C.byref(h), n1, int(paired), C.byref(ca), ptr(tids), int(tids.size),
                               ptr(rgb), int(rgb.size), ptr(out), bam_cap, C.byref(n), C.byref(meta), C.byref(t))
    check(rc, ctx.handle)
    del keep
    tile.n_reads, tile.n_mapped = t.n_reads, t.n_mapped
    return out[: n.value]


def emit_bam_device(ctx, d_hits: dict, n1: int, paired: bool, d_arena: dict, arena_bytes: int, d_rid_to_tid: int,
                    n_tid: int, d_rg: int, rg_n: int, d_bam: int, bam_cap: int, d_meta: dict, tile: BamTile,
                    d_status: int, stream: int | None = None) -> None:
    """Device form: every argument named d_* is a device pointer (int)."""
    h = ma_hits(*[d_hits[k] for k, _ in HIT_FIELDS])
    ca = ma_fastq_arena(d_arena["data"], arena_bytes, d_arena["name_off"], d_arena["name_len"],
                        d_arena["orig_off"], d_arena["orig_len"], d_arena.get("qual_off"), d_arena.get("qual_len"))
    meta = ma_bam_meta(*[d_meta[k] for k, _ in META_FIELDS])
    t = tile.to_c()
    rc = lib.ma_emit_bam_batch_device(ctx.handle, C.byref(h), n1, int(paired), C.byref(ca), d_rid_to_tid, n_tid,
                                      d_rg, rg_n, d_bam, bam_cap, C.byref(meta), C.byref(t), d_status, stream)
    check(rc, ctx.handle)


def canonical_rid_to_tid(contig_names) -> np.ndarray:
    """_rid_to_tid_table: one tid per distinct canonical contig name, in
    order of first appearance."""
    from .linear_fm import canonical_contig
    seen: dict[str, int] = {}
    out = []
    for name in contig_names:
        c = canonical_contig(name)
        if c not in seen:
            seen[c] = len(seen)
        out.append(seen[c])
    return np.asarray(out, np.int32)


rid_to_tid_table = canonical_rid_to_tid


@dataclass
class SortResult:
    is_dup: np.ndarray
    perm: np.ndarray
    dup_perm: np.ndarray | None
    n_marked: int


def sort_markdup(ctx, tile: BamTile, do_markdup: bool = True, dup_perm: bool = False) -> SortResult:
    """Sorts the tile's first n_reads records (host arrays in, host out)."""
    n = tile.n_reads
    m = {k: np.ascontiguousarray(tile.meta[k][:n]) for k in ("coord", "dhi", "dlo", "score", "pair")}
    is_dup = np.empty(n, np.uint32)
    perm = np.empty(n, np.uint32)
    dp = np.empty(n, np.uint32) if dup_perm else None
    marked = C.c_uint64(0)
    rc = lib.ma_sort_markdup(ctx.handle, n, ptr(m["coord"]), ptr(m["dhi"]), ptr(m["dlo"]), ptr(m["score"]),
                             ptr(m["pair"]), ptr(is_dup), ptr(perm), int(do_markdup), ptr(dp), C.byref(marked))
    check(rc, ctx.handle)
    return SortResult(is_dup, perm, dp, marked.value)


def gather_sorted(ctx, chunks, tile: BamTile, res: SortResult, apply_dup: bool = True,
                  out: np.ndarray | None = None) -> np.ndarray:
    """The tile's records in res.perm order; chunks are the BAM chunks the
    tile's `rec` entries point into (chunk index = position in the list).
    Returns a view of `out` (allocated when missing or too small)."""
    n = tile.n_reads
    bufs = [np.ascontiguousarray(np.frombuffer(c, np.uint8) if not isinstance(c, np.ndarray) else c, dtype=np.uint8)
            for c in chunks]
    ptrs = (C.c_void_p * max(1, len(bufs)))(*[ptr(b) for b in bufs])
    lens = np.array([b.size for b in bufs] or [0], np.uint64)
    rec = np.ascontiguousarray(tile.meta["rec"][:n])
    length = np.ascontiguousarray(tile.meta["len"][:n])
    cap = int(length.sum(dtype=np.uint64))
    if out is None or out.size < cap:
        out = np.empty(max(cap, 1), np.uint8)
    got = C.c_uint64(0)
    rc = lib.ma_gather_sorted_bam(ctx.handle, n, ptr(res.perm), ptr(rec), ptr(length), ptr(res.is_dup),
                                  int(apply_dup), C.cast(ptrs, C.c_void_p), ptr(lens), len(bufs), ptr(out), cap,
                                  C.byref(got))
    check(rc, ctx.handle)
    return out[: got.value]
