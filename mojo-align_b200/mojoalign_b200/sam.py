"""SAM text of mapped batches on the GPU (ma_emit_sam_batch[_device]).

The SAM lines of a batch are what map_fastq_fm_gpu's SAM loop writes
(fq2bam-meth/src/linear_gpu_fm.mojo:2787-2836): _hit_from_fm (L987-1025),
pair_hits / hit_to_sam_line (fq2bam-meth/src/linear_extend.mojo:263-320) and
the RG tag (_sam_with_rg_fm, L80-81).  The contig field carries the canonical
name (_canonical_contig, linear_gpu_locate.mojo:156-162).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import check, lib, ma_fastq_arena, ma_hits, ma_sam_contigs, ptr
from .bam import BatchArena

HIT_FIELDS = (("rid", np.int32), ("pos", np.uint32), ("mapq", np.uint32), ("flag", np.int32), ("sl", np.uint32),
              ("sr", np.uint32), ("nm", np.uint32))
LINE_FIXED = 128  # bytes of a line besides name, SEQ, QUAL, contig names and RG id


def canonical_name(name: bytes) -> bytes:
    """_canonical_contig: a leading f / r dropped from names of two or more bytes."""
    return name[1:] if len(name) >= 2 and name[:1] in (b"f", b"r") else name


@dataclass
class SamContigs:
    """Per rid: canonical name span and canonical id (equal ids exactly for
    equal canonical names)."""
    names: np.ndarray
    name_off: np.ndarray
    name_len: np.ndarray
    canon: np.ndarray

    @classmethod
    def from_names(cls, contig_names) -> "SamContigs":
        blob, off, ln, canon, ids = bytearray(), [], [], [], {}
        for n in contig_names:
            c = canonical_name(n.encode() if isinstance(n, str) else bytes(n))
            off.append(len(blob))
            ln.append(len(c))
            blob += c
            canon.append(ids.setdefault(c, len(ids)))
        return cls(np.frombuffer(bytes(blob) or b"\0", np.uint8).copy(), np.array(off, np.uint64),
                   np.array(ln, np.uint32), np.array(canon, np.uint32))

    @property
    def max_name(self) -> int:
        return int(self.name_len.max(initial=1))

    def to_c(self) -> ma_sam_contigs:
        return ma_sam_contigs(ptr(self.names), int(self.names.size), ptr(self.name_off), ptr(self.name_len),
                              ptr(self.canon), int(self.canon.size))

    def to_device(self, torch, dev) -> "DeviceSamContigs":
        return DeviceSamContigs(self, torch, dev)


class DeviceSamContigs:
    """The contig table in device memory (keeps its tensors alive)."""

    def __init__(self, host: SamContigs, torch, dev):
        def put(a):
            a = np.ascontiguousarray(a)
            signed = {np.dtype(np.uint64): np.int64, np.dtype(np.uint32): np.int32}
            return torch.from_numpy(a.view(signed.get(a.dtype, a.dtype)).copy()).to(dev)

        self.host = host
        self.t = [put(host.names), put(host.name_off), put(host.name_len), put(host.canon)]
        self.c = ma_sam_contigs(self.t[0].data_ptr(), int(host.names.size), self.t[1].data_ptr(), self.t[2].data_ptr(),
                                self.t[3].data_ptr(), int(host.canon.size))


def sam_bound(arena_cols: dict, n_seq: int, contigs: SamContigs, rg_n: int) -> int:
    """Bytes enough for the lines of n_seq records: per line the fixed fields,
    twice the longest canonical name, the RG tag, up to three bytes per name
    byte, SEQ and QUAL."""
    s = lambda k: int(np.asarray(arena_cols[k][:n_seq], dtype=np.uint64).sum())  # noqa: E731
    return n_seq * (LINE_FIXED + rg_n + 2 * contigs.max_name) + 3 * s("name_len") + s("orig_len") + s("qual_len")


def emit_sam_from_batch(ctx, hits: dict, n1: int, paired: bool, arena: BatchArena, contigs: SamContigs, rg: bytes,
                        cap: int | None = None) -> tuple[bytes, int]:
    """Host form: SAM text and mapped-record count of one batch."""
    n_seq = n1 * (2 if paired else 1)
    h = {k: np.ascontiguousarray(hits[k], dt) for k, dt in HIT_FIELDS if k in hits}
    if "nm" not in h:
        h["nm"] = np.zeros(n_seq, np.uint32)
    if arena.qual_off is None:
        raise ValueError("SAM lines need the qualities")
    if cap is None:
        cap = sam_bound(vars(arena), n_seq, contigs, len(rg))
    out = np.zeros(max(cap, 1), np.uint8)
    got, mapped = C.c_uint64(0), C.c_uint64(0)
    hc = ma_hits(*[ptr(h[k]) for k, _ in HIT_FIELDS])
    ac = arena.to_c()
    cc = contigs.to_c()
    rgb = np.frombuffer(rg or b"\0", np.uint8)
    check(lib.ma_emit_sam_batch(ctx.handle, C.byref(hc), n1, int(paired), C.byref(ac), C.byref(cc), ptr(rgb), len(rg),
                                ptr(out), cap, C.byref(got), C.byref(mapped)), ctx.handle)
    return out[:got.value].tobytes(), int(mapped.value)


def emit_sam_device(ctx, d_hits: ma_hits, n1: int, paired: bool, d_arena: ma_fastq_arena,
                    d_contigs: DeviceSamContigs, d_rg: int, rg_n: int, d_out: int, cap: int, d_status: int,
                    stream: int | None = None) -> None:
    """Device form, asynchronous: d_status (3 x u64) receives the text size,
    the mapped records and the error bits."""
    check(lib.ma_emit_sam_batch_device(ctx.handle, C.byref(d_hits), n1, int(paired), C.byref(d_arena),
                                       C.byref(d_contigs.c), d_rg, rg_n, d_out, cap, d_status, stream), ctx.handle)


SAM_ERRORS = {4: "hit rid outside the contig table", 8: "arena or contig-name span outside its buffer",
              2: "FASTQ SEQ/QUAL is not valid UTF-8", 1: "SAM batch buffer overflow"}


def sam_error(bits: int) -> str:
    for b in (4, 8, 2, 1):
        if bits & b:
            return SAM_ERRORS[b]
    return ""
