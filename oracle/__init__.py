"""ORACLE (test infrastructure): ctypes wrapper of liboracle_fm.so.

A CPU restatement of the reference's FM path (see oracle_fm.c for the
reference file:line map).  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference arm may import this package, and only to check or
time the reference algorithm; the product never routes through it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle_fm.so"


def build() -> Path:
    newest = max((HERE / f).stat().st_mtime for f in ("oracle_fm.c", "oracle_bam.c", "oracle_sort.c", "oracle_fastq.c", "Makefile"))
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        subprocess.run(["make", "-s", "-C", str(HERE), "liboracle_fm.so"], check=True)
    return LIB


class Counters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in
                ("occ_lines", "lf_lines", "sa_loads", "pac_sectors", "endpoints", "steps", "rows", "extends",
                 "capped", "fallback")]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class BamIn(C.Structure):
    _fields_ = [("n1", C.c_uint32), ("paired", C.c_int32)] + \
        [(n, C.c_void_p) for n in ("rid", "pos", "mapq", "flag", "sl", "sr", "nm", "arena", "name_off", "orig_off",
                                   "qual_off", "name_len", "orig_len", "qual_len", "rid_to_tid")] + \
        [("n_tid_map", C.c_int32), ("rg", C.c_void_p), ("rg_n", C.c_uint32), ("n_reads", C.c_uint64),
         ("n_total", C.c_uint64), ("meta_cap", C.c_uint64), ("chunk", C.c_uint32)]


BAM_META_FIELDS = (("coord", np.uint64), ("dhi", np.uint64), ("dlo", np.uint64), ("rec", np.uint64),
                   ("len", np.uint32), ("score", np.uint32), ("pair", np.uint32))


class BamMeta(C.Structure):
    _fields_ = [(n, C.c_void_p) for n, _ in BAM_META_FIELDS]


def _load():
    build()
    lib = C.CDLL(str(LIB))
    vp = C.c_void_p
    lib.orc_index_load.argtypes = [C.c_char_p, C.POINTER(vp)]
    lib.orc_index_load.restype = C.c_int
    lib.orc_index_free.argtypes = [vp]
    lib.orc_last_error.restype = C.c_char_p
    lib.orc_index_header.argtypes = [vp, C.POINTER(C.c_uint64)]
    lib.orc_contig.argtypes = [vp, C.c_int64, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.c_char_p, C.c_int]
    lib.orc_contig.restype = C.c_int64
    lib.orc_pac_base.argtypes = [vp, C.c_int64]
    lib.orc_pac_base.restype = C.c_int
    lib.orc_occ.argtypes = [vp, C.c_int64, C.c_int]
    lib.orc_occ.restype = C.c_uint64
    lib.orc_inv_psi.argtypes = [vp, C.c_uint64]
    lib.orc_inv_psi.restype = C.c_uint64
    lib.orc_sa_at.argtypes = [vp, C.c_uint64]
    lib.orc_sa_at.restype = C.c_uint64
    lib.orc_match_exact.argtypes = [vp, vp, C.c_int64, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    lib.orc_match_exact.restype = C.c_int64
    lib.orc_depos.argtypes = [vp, C.c_uint64, C.POINTER(C.c_int64), C.POINTER(C.c_int)]
    lib.orc_convert.argtypes = [vp, C.c_int64, C.c_int]
    lib.orc_pack_bases.argtypes = [vp, vp, C.c_int64]
    lib.orc_map.argtypes = [vp, vp, vp, C.c_uint32, C.c_int, C.c_uint32, C.c_int, C.c_int, vp,
                            vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, C.POINTER(Counters), C.c_int]
    lib.orc_map.restype = C.c_int
    lib.orc_max_threads.restype = C.c_int
    lib.orc_emit_bam.argtypes = [C.POINTER(BamIn), vp, C.c_uint64, C.POINTER(BamMeta), C.POINTER(C.c_uint64)]
    lib.orc_emit_bam.restype = C.c_int64
    lib.orc_pack_aln.argtypes = [vp, C.c_uint64, C.c_char_p] + [C.c_int64] * 7 + [C.c_char_p, C.c_int64, C.c_char_p] + \
        [C.c_int64] * 5 + [C.c_char_p, C.c_int64]
    lib.orc_pack_aln.restype = C.c_int64
    lib.orc_sort_markdup.argtypes = [C.c_uint64, C.c_uint64] + [vp] * 7 + [C.c_int, vp]
    lib.orc_sort_markdup.restype = C.c_int64
    lib.orc_gather_sorted.argtypes = [C.c_uint64] + [vp] * 5 + [C.c_int, vp, C.c_uint64]
    lib.orc_gather_sorted.restype = C.c_int64
    lib.orc_fastq_parse.argtypes = [vp, C.c_uint64, C.c_int, C.c_uint64, C.c_uint64] + [vp] * 6 + \
        [C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]
    lib.orc_fastq_parse.restype = C.c_int64
    lib.orc_fastq_parse_pr.argtypes = lib.orc_fastq_parse.argtypes
    lib.orc_fastq_parse_pr.restype = C.c_int64
    lib.orc_emit_sam.argtypes = [vp] * 6 + [C.c_uint64, C.c_int] + [vp] * 7 + [vp] * 4 + \
        [C.c_uint32, C.c_char_p, C.c_uint32, vp, C.c_uint64, C.POINTER(C.c_uint64)]
    lib.orc_emit_sam.restype = C.c_int64
    return lib


lib = _load()


def _p(a):
    return None if a is None else a.ctypes.data


class OracleIndex:
    """bwa 0.7 index as FmIndex.load reads it (linear_fm_index.mojo:88-175)."""

    def __init__(self, prefix):
        h = C.c_void_p()
        if lib.orc_index_load(os.fsencode(os.fspath(prefix)), C.byref(h)) != 0:
            raise RuntimeError(lib.orc_last_error().decode())
        self.h = h
        hdr = (C.c_uint64 * 12)()
        lib.orc_index_header(h, hdr)
        (self.primary, self.seq_len, self.l_pac, *l2, self.sa_intv, self.n_sa, self.n_contigs,
         self.bwt_size) = list(hdr)
        self.L2 = l2
        self.contigs = []
        for i in range(self.n_contigs):
            off, ln, nm = C.c_uint64(), C.c_uint32(), C.create_string_buffer(4096)
            lib.orc_contig(h, i, C.byref(off), C.byref(ln), nm, 4096)
            self.contigs.append((nm.value.decode(), off.value, ln.value))

    def close(self):
        if self.h:
            lib.orc_index_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # FmIndex host methods, linear_fm_index.mojo:206-320
    def pac_base(self, pos: int) -> int:
        return lib.orc_pac_base(self.h, pos)

    def occ(self, k: int, c: int) -> int:
        return lib.orc_occ(self.h, k, c)

    def inv_psi(self, k: int) -> int:
        return lib.orc_inv_psi(self.h, k)

    def sa_at(self, k: int) -> int:
        return lib.orc_sa_at(self.h, k)

    def match_exact(self, codes) -> tuple[int, int, int]:
        a = np.ascontiguousarray(codes, dtype=np.uint8)
        k, l = C.c_uint64(), C.c_uint64()
        occ = lib.orc_match_exact(self.h, _p(a), a.size, C.byref(k), C.byref(l))
        return (k.value, l.value, occ) if occ else (0, 0, 0)

    def depos(self, pos: int) -> tuple[int, int]:
        fp, rev = C.c_int64(), C.c_int()
        lib.orc_depos(self.h, pos, C.byref(fp), C.byref(rev))
        return fp.value, rev.value

    def map(self, bases, lens, n1: int, paired: bool, max_len: int, bs_r1: int, bs_r2: int, params,
            threads: int = 0, counters: bool = False) -> dict:
        """orc_map: convert + pack + seed/extend + rescue, like _fm_fire_batch."""
        n_seq = n1 * (2 if paired else 1)
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        lens = np.ascontiguousarray(lens, dtype=np.uint32)
        out = {
            "rid": np.empty(n_seq, np.int32), "pos": np.empty(n_seq, np.uint32), "mapq": np.empty(n_seq, np.uint32),
            "flag": np.empty(n_seq, np.int32), "sl": np.empty(n_seq, np.uint32), "sr": np.empty(n_seq, np.uint32),
            "nm": np.empty(n_seq, np.uint32), "uk": np.empty(n_seq, np.uint64), "ul": np.empty(n_seq, np.uint64),
            "us": np.empty(n_seq, np.int32), "e": np.empty(n_seq, np.int32), "score": np.empty(n_seq, np.int32),
        }
        prm = (C.c_int32 * 7)(*params)
        ct = Counters()
        rc = lib.orc_map(self.h, _p(bases), _p(lens), n1, int(paired), max_len, bs_r1, bs_r2, prm,
                         *[_p(out[k]) for k in ("rid", "pos", "mapq", "flag", "sl", "sr", "nm", "uk", "ul", "us",
                                                "e", "score")],
                         C.byref(ct) if counters else None, threads)
        if rc != 0:
            raise RuntimeError(lib.orc_last_error().decode())
        if counters:
            out["counters"] = ct.as_dict()
        return out


HIT_FIELDS = (("rid", np.int32), ("pos", np.uint32), ("mapq", np.uint32), ("flag", np.int32),
              ("sl", np.uint32), ("sr", np.uint32), ("nm", np.uint32))


def emit_bam(hits, arena, n1: int, paired: bool, rid_to_tid, rg: bytes, *, n_reads: int = 0,
             n_total: int = 0, meta_cap: int | None = None, chunk: int = 0, cap: int | None = None):
    """orc_emit_bam: _emit_bam_from_batch (linear_gpu_fm.mojo:669-984) on one batch.

    hits: mapping outputs by field name, [n_seq] (R1 rows then R2 rows).
    arena: dict with "data" (uint8) and "name_off"/"orig_off"/"qual_off"
    (uint64, qual_off may be None) and "name_len"/"orig_len"/"qual_len"
    (uint32), [n_seq].  Returns (bam bytes, metadata arrays of the batch's
    records, mapped count); raises on overflow like the reference.
    """
    n_seq = n1 * (2 if paired else 1)
    h = {k: np.ascontiguousarray(hits[k], dtype=t) for k, t in HIT_FIELDS}
    data = np.ascontiguousarray(arena["data"], dtype=np.uint8)
    offs = {k: (None if arena.get(k) is None else np.ascontiguousarray(arena[k], dtype=np.uint64))
            for k in ("name_off", "orig_off", "qual_off")}
    lens = {k: (None if arena.get(k) is None else np.ascontiguousarray(arena[k], dtype=np.uint32))
            for k in ("name_len", "orig_len", "qual_len")}
    tids = np.ascontiguousarray(rid_to_tid, dtype=np.int32)
    rgb = np.frombuffer(bytes(rg) + b"\0", dtype=np.uint8)
    if meta_cap is None:
        meta_cap = n_reads + n_seq + 1
    if cap is None:
        cap = sum(int(x) for x in (n_seq * 64, lens["name_len"].sum(dtype=np.uint64),
                                   2 * lens["orig_len"].sum(dtype=np.uint64), n_seq * len(rg)))
    bam = np.zeros(max(cap, 1), np.uint8)
    meta = {k: np.zeros(meta_cap, t) for k, t in BAM_META_FIELDS}
    bi = BamIn(n1=n1, paired=int(paired), **{k: _p(v) for k, v in h.items()}, arena=_p(data),
               **{k: _p(v) for k, v in offs.items()}, **{k: _p(v) for k, v in lens.items()},
               rid_to_tid=_p(tids), n_tid_map=len(tids), rg=_p(rgb), rg_n=len(rg), n_reads=n_reads,
               n_total=n_total, meta_cap=meta_cap, chunk=chunk)
    bm = BamMeta(**{k: _p(v) for k, v in meta.items()})
    mapped = C.c_uint64(0)
    n = lib.orc_emit_bam(C.byref(bi), _p(bam), cap, C.byref(bm), C.byref(mapped))
    if n == -1:
        raise RuntimeError("BAM batch buffer overflow")
    if n == -2:
        raise RuntimeError("FM sort cap exceeded")
    return bam[:n].tobytes(), {k: v[n_reads:n_reads + n_seq].copy() for k, v in meta.items()}, mapped.value


def pack_aln(name: bytes, flag: int, tid: int, pos0: int, mapq: int, sl: int, sr: int, seq: bytes, qual,
             ntid: int, npos: int, tlen: int, nm: int, rg: bytes) -> bytes:
    """orc_pack_aln: one record of _pack_bam_aln (linear_gpu_fm.mojo:497-666).
    qual None = no qualities; sl/sr are in read orientation (swapped on the
    reverse strand inside)."""
    cap = 64 + len(name) + 2 * len(seq) + len(rg) + 16
    buf = np.zeros(cap, np.uint8)
    n = lib.orc_pack_aln(_p(buf), cap, name, len(name), flag, tid, pos0, mapq, sl, sr, seq, len(seq),
                         qual, len(qual) if qual is not None else 0, ntid, npos, tlen, nm, rg, len(rg))
    if n < 0:
        raise RuntimeError("BAM batch buffer overflow")
    return buf[:n].tobytes()


def sort_markdup(coord, dhi, dlo, score, pair, do_markdup: bool = True, tile: int = 0, dup_perm: bool = True):
    """orc_sort_markdup: gpu_sort_markdup (linear_gpu_sort.mojo:24-560).
    Returns (is_dup, perm, dup_perm or None, marked)."""
    coord, dhi, dlo = (np.ascontiguousarray(a, dtype=np.uint64) for a in (coord, dhi, dlo))
    score, pair = (np.ascontiguousarray(a, dtype=np.uint32) for a in (score, pair))
    n = coord.size
    is_dup = np.zeros(n, np.uint32)
    perm = np.zeros(n, np.uint32)
    dp = np.zeros(n, np.uint32) if dup_perm else None
    m = lib.orc_sort_markdup(n, tile, _p(coord), _p(dhi), _p(dlo), _p(score), _p(pair), _p(is_dup), _p(perm),
                             int(do_markdup), _p(dp))
    if m < 0:
        raise MemoryError("orc_sort_markdup")
    return is_dup, perm, dp, int(m)


def gather_sorted(chunks, perm, rec, length, is_dup, apply_dup: bool = True) -> bytes:
    """orc_gather_sorted: _gather_perm_to_writer (linear_gpu_fm.mojo:177-225)
    as one byte stream.  chunks: list of bytes-like BAM chunks."""
    bufs = [np.frombuffer(bytes(c), np.uint8) for c in chunks]
    ptrs = (C.c_void_p * max(1, len(bufs)))(*[b.ctypes.data for b in bufs])
    perm = np.ascontiguousarray(perm, dtype=np.uint32)
    rec = np.ascontiguousarray(rec, dtype=np.uint64)
    length = np.ascontiguousarray(length, dtype=np.uint32)
    is_dup = np.ascontiguousarray(is_dup, dtype=np.uint32)
    cap = int(length.sum(dtype=np.uint64))
    out = np.zeros(max(cap, 1), np.uint8)
    k = lib.orc_gather_sorted(perm.size, C.cast(ptrs, C.c_void_p), _p(perm), _p(rec), _p(length), _p(is_dup),
                              int(apply_dup), _p(out), cap)
    if k < 0:
        raise RuntimeError("BAM record larger than batch buffer")
    return out[:k].tobytes()


FASTQ_ERRORS = {-1: "truncated FASTQ (missing SEQ)", -2: "truncated FASTQ (missing +)",
                -3: "truncated FASTQ (missing QUAL)"}


def fastq_parse(buf, at_eof: bool = True, max_records: int | None = None, base: int = 0) -> dict:
    """orc_fastq_parse: the record split of fq_read_batch / _store_rec /
    _pipe_line / _qname_span (linear_fastq.mojo:233-451) over one buffer.
    Returns name/seq/qual offsets and lengths, `n`, `consumed`, `max_len`;
    raises RuntimeError with the reference's message on a truncated record."""
    b = np.frombuffer(bytes(buf), np.uint8)
    cap = b.size // 4 + 2 if max_records is None else max_records
    out = {k: np.zeros(cap, np.uint64 if k.endswith("off") else np.uint32)
           for k in ("name_off", "name_len", "seq_off", "seq_len", "qual_off", "qual_len")}
    consumed, ml = C.c_uint64(0), C.c_uint32(0)
    n = lib.orc_fastq_parse(_p(b) if b.size else None, b.size, int(at_eof), cap, base,
                            *[_p(out[k]) for k in ("name_off", "name_len", "seq_off", "seq_len", "qual_off",
                                                   "qual_len")], C.byref(consumed), C.byref(ml))
    if n < 0:
        raise RuntimeError(FASTQ_ERRORS[n])
    res = {k: v[:n].copy() for k, v in out.items()}
    res.update(n=int(n), consumed=consumed.value, max_len=ml.value)
    return res


def pack_bases(ascii_bytes) -> np.ndarray:
    """pack_bases_kernel (linear_gpu_fm.mojo:1136-1154)."""
    a = np.frombuffer(bytes(ascii_bytes), dtype=np.uint8).copy()
    out = np.empty_like(a)
    lib.orc_pack_bases(_p(a), _p(out), a.size)
    return out


def convert(seq: bytes, mode: int) -> bytes:
    """_cvt (linear_fastq.mojo:37-46): mode 1 C->T, 2 G->A."""
    a = np.frombuffer(bytes(seq), dtype=np.uint8).copy()
    lib.orc_convert(_p(a), a.size, mode)
    return a.tobytes()


def max_threads() -> int:
    return lib.orc_max_threads()


REC_KEYS = ("name_off", "name_len", "seq_off", "seq_len", "qual_off", "qual_len")


def fastq_parse_pr(buf, at_eof: bool = True, max_records: int | None = None, base: int = 0) -> dict:
    """orc_fastq_parse_pr: the record split of FastqPairReader (fq2bam-meth/
    python/fastq_batch.py:18-317), the reader of the SAM path, over one
    buffer.  Same result keys as fastq_parse; never raises."""
    b = np.frombuffer(bytes(buf), np.uint8)
    cap = b.size // 4 + 2 if max_records is None else max_records
    out = {k: np.zeros(max(cap, 1), np.uint64 if k.endswith("off") else np.uint32) for k in REC_KEYS}
    consumed, ml = C.c_uint64(0), C.c_uint32(0)
    n = lib.orc_fastq_parse_pr(_p(b) if b.size else None, b.size, int(at_eof), cap, base,
                               *[_p(out[k]) for k in REC_KEYS], C.byref(consumed), C.byref(ml))
    res = {k: v[:n].copy() for k, v in out.items()}
    res.update(n=int(n), consumed=consumed.value, max_len=ml.value)
    return res


def sam_contigs(contig_names) -> dict:
    """Per rid: the canonical name (_canonical_contig, linear_gpu_locate.mojo:
    156-162, a leading f/r dropped from names of two or more bytes) and a
    canonical id, equal exactly when the canonical names are equal."""
    blob, off, ln, canon, ids = bytearray(), [], [], [], {}
    for name in contig_names:
        nb = name.encode() if isinstance(name, str) else bytes(name)
        c = nb[1:] if len(nb) >= 2 and nb[:1] in (b"f", b"r") else nb
        off.append(len(blob))
        ln.append(len(c))
        blob += c
        canon.append(ids.setdefault(c, len(ids)))
    return {"names": np.frombuffer(bytes(blob) or b"\0", np.uint8).copy(), "off": np.array(off, np.uint64),
            "len": np.array(ln, np.uint32), "canon": np.array(canon, np.uint32)}


SAM_ERRORS = {-1: "SAM batch buffer overflow", -2: "FASTQ SEQ/QUAL is not valid UTF-8",
              -3: "hit rid outside the contig table"}


def emit_sam(hits: dict, n1: int, paired: bool, arena: dict, contig_names, rg: bytes, cap: int | None = None):
    """orc_emit_sam: the SAM lines of one mapped batch (_hit_from_fm, pair_hits,
    hit_to_sam_line, _sam_with_rg_fm).  `hits`: rid/pos/mapq/flag/sl/sr rows
    (R1 then R2); `arena`: data + the REC_KEYS columns in the same order.
    Returns (text bytes, mapped records); raises RuntimeError on the errors of
    SAM_ERRORS."""
    t = sam_contigs(contig_names)
    h = {k: np.ascontiguousarray(hits[k], dt) for k, dt in
         (("rid", np.int32), ("pos", np.uint32), ("mapq", np.uint32), ("flag", np.int32), ("sl", np.uint32),
          ("sr", np.uint32))}
    a = {k: np.ascontiguousarray(arena[k], np.uint64 if k.endswith("off") else np.uint32) for k in REC_KEYS}
    data = np.ascontiguousarray(np.frombuffer(bytes(arena["data"]), np.uint8) if not isinstance(arena["data"], np.ndarray)
                                else arena["data"], np.uint8)
    if cap is None:
        n_seq = n1 * (2 if paired else 1)
        cap = n_seq * (160 + len(rg)) + 3 * int(a["name_len"][:n_seq].sum()) + int(a["seq_len"][:n_seq].sum()) + \
            int(a["qual_len"][:n_seq].sum()) + 2 * n_seq * int(t["len"].max(initial=1))
    out = np.zeros(max(cap, 1), np.uint8)
    mapped = C.c_uint64(0)
    k = lib.orc_emit_sam(*[_p(h[x]) for x in ("rid", "pos", "mapq", "flag", "sl", "sr")], n1, int(paired),
                         _p(data) if data.size else None, *[_p(a[x]) for x in REC_KEYS], _p(t["names"]), _p(t["off"]),
                         _p(t["len"]), _p(t["canon"]), int(t["canon"].size), rg, len(rg), _p(out), cap,
                         C.byref(mapped))
    if k < 0:
        raise RuntimeError(SAM_ERRORS[int(k)])
    return out[:k].tobytes(), int(mapped.value)
