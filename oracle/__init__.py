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
    src = HERE / "oracle_fm.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE), "liboracle_fm.so"], check=True)
    return LIB


class Counters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in
                ("occ_lines", "lf_lines", "sa_loads", "pac_sectors", "endpoints", "steps", "rows", "extends")]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


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
