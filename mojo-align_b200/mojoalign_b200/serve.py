"""Served form: a request loop over one resident index (ma_serve_* C ABI).

Requests are read batches in the ma_map_batch layout (padded ASCII rows, R1
rows then R2 rows) from any number of samples.  The native server admits
them against a reserved HBM budget, merges the pending work of several
requests into each launch group (continuous batching), keeps up to
`max_inflight` groups in flight on their own streams, and completes each
request with exactly the outputs ma_map_batch gives it alone.

No counterpart in the reference, whose map_fastq_fm_gpu maps one FASTQ
stream in fixed 16384-pair batches (fq2bam-meth/src/linear_gpu_fm.mojo:2074,
2438-3094).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import (MA_ERR_TIMEOUT, MA_OK, MA_SERVE_SCHEDULER_TEST, MojoAlignError, check, lib, ma_serve_options,
                   ma_serve_stats, ptr)
from .mapper import GpuContext, GpuIndex, MapResult, bs_mode
from .params import FmParams


@dataclass
class Ticket:
    id: int
    result: MapResult
    bases: np.ndarray  # kept alive until the request completes
    lens: np.ndarray


class Server:
    """Python handle of an ma_server.

    scheduler_test=True runs the scheduler with no device work at all (the
    outputs are a host function of each read, not alignments; see the C
    header); ctx and index may then be None.
    """

    def __init__(self, ctx: GpuContext | None, index: GpuIndex | None, hbm_budget_bytes: int = 0,
                 max_group_pairs: int = 262144, max_inflight: int = 3, scheduler_test: bool = False):
        o = ma_serve_options()
        lib.ma_serve_options_default(C.byref(o))
        o.hbm_budget_bytes = hbm_budget_bytes
        o.max_group_pairs = max_group_pairs
        o.max_inflight = max_inflight
        o.flags = MA_SERVE_SCHEDULER_TEST if scheduler_test else 0
        h = C.c_void_p()
        check(lib.ma_serve_create(ctx.handle if ctx else None, index.handle if index else None, C.byref(o),
                                  C.byref(h)))
        self.handle = h
        self._live: dict[int, Ticket] = {}

    def _error(self, rc: int) -> MojoAlignError:
        msg = lib.ma_serve_last_error(self.handle)
        return MojoAlignError(rc, msg.decode() if msg else "")

    def submit(self, bases: np.ndarray, lens: np.ndarray, n1: int, paired: bool, max_len: int, bs_r1="C2T",
               bs_r2="G2A", params: FmParams | None = None) -> Ticket:
        params = params or FmParams()
        n_seq = n1 * (2 if paired else 1)
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        lens = np.ascontiguousarray(lens, dtype=np.uint32)
        if bases.size < n_seq * max_len or lens.size < n_seq:
            raise ValueError("bases / lens smaller than the request")
        res = MapResult.empty(n_seq, debug=False)
        p = params.to_c()
        hits = res.hits()
        rid = C.c_uint64()
        rc = lib.ma_serve_submit(self.handle, ptr(bases), ptr(lens), n1, int(paired), max_len, bs_mode(bs_r1),
                                 bs_mode(bs_r2), C.byref(p), C.byref(hits), C.byref(rid))
        if rc != MA_OK:
            raise self._error(rc)
        t = Ticket(rid.value, res, bases, lens)
        self._live[t.id] = t
        return t

    def done(self, t: Ticket) -> bool:
        d = C.c_int()
        rc = lib.ma_serve_poll(self.handle, t.id, C.byref(d))
        if d.value and rc != MA_OK:
            raise self._error(rc)
        return bool(d.value)

    def wait(self, t: Ticket, timeout_ms: int = -1) -> MapResult:
        rc = lib.ma_serve_wait(self.handle, t.id, timeout_ms)
        if rc == MA_ERR_TIMEOUT:
            raise TimeoutError(f"request {t.id} still running after {timeout_ms} ms")
        self._live.pop(t.id, None)
        if rc != MA_OK:
            raise self._error(rc)
        return t.result

    def drain(self, timeout_ms: int = -1) -> None:
        rc = lib.ma_serve_drain(self.handle, timeout_ms)
        if rc == MA_ERR_TIMEOUT:
            raise TimeoutError("server still busy")
        self._live.clear()
        if rc != MA_OK:
            raise self._error(rc)

    def stats(self) -> dict:
        s = ma_serve_stats()
        check(lib.ma_serve_get_stats(self.handle, C.byref(s)))
        return {f: getattr(s, f) for f, _ in ma_serve_stats._fields_}

    def latencies(self):
        """(ids, reads, ms) of completed requests, in completion order."""
        n = C.c_uint64()
        check(lib.ma_serve_latencies(self.handle, None, None, None, 0, C.byref(n)))
        ids = np.empty(n.value, np.uint64)
        reads = np.empty(n.value, np.uint64)
        ms = np.empty(n.value, np.float64)
        check(lib.ma_serve_latencies(self.handle, ptr(ids), ptr(reads), ptr(ms), n.value, C.byref(n)))
        return ids, reads, ms

    def close(self) -> None:
        if self.handle:
            lib.ma_serve_destroy(self.handle)
            self.handle = None
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def percentiles(ms: np.ndarray, qs=(50, 99, 99.9)) -> dict:
    if ms.size == 0:
        return {f"p{q:g}": None for q in qs}
    return {f"p{q:g}": float(np.percentile(ms, q)) for q in qs}
