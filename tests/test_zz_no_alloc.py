"""The no-allocation mapping entry point against the allocating one.

ma_map_batch_device_noalloc serves callers that must not let the library
call cudaMalloc (for instance a framework whose caching allocator already
holds the free HBM, or a latency-bound loop that cannot absorb cudaMalloc's
implicit device synchronisation).  It takes its scratch from a fixed
device array instead of the context's pool.  Its outputs must equal those
of ma_map_batch_device on the same reads, exactly (integer outputs), on two
calls in a row, since the array keeps the previous call's contents, and
the device's free memory must be the same after each of those calls as
before it (after the set-up call with no reads).

This file is named to be collected last, so a run that stops at the first
failure has run every other test before it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from mojoalign_b200 import BENCH_PARAMS, GpuContext, GpuIndex, MapResult, map_batch_device, synth
from mojoalign_b200 import _lib

pytestmark = pytest.mark.gpu

FIELDS = MapResult.FIELDS + MapResult.DEBUG


def _device_outputs(torch, n, dev):
    return {f: torch.empty(n, dtype=torch.int64 if f in ("uk", "ul") else torch.int32, device=dev)
            for f in FIELDS}


def test_noalloc_matches_allocating_entry_point(small_ref):
    torch = pytest.importorskip("torch")
    fa, prefix = small_ref
    ctx = GpuContext(0)
    gi = GpuIndex(ctx, prefix, kmer_k=12, kmer3_k=12)
    dev = torch.device("cuda:0")
    rb = synth.simulate_reads(fa, synth.ReadModel(sub_rate=0.02), 4000, True, 150, seed=21)
    d_bases = torch.from_numpy(rb.bases.reshape(-1)).to(dev)
    d_lens = torch.from_numpy(rb.lens.view(np.int32)).to(dev)
    n = rb.n_seq
    stream = torch.cuda.current_stream(dev)

    ref = _device_outputs(torch, n, dev)
    map_batch_device(ctx, gi, d_bases.data_ptr(), d_lens.data_ptr(), rb.n1, True, 150,
                     {f: ref[f].data_ptr() for f in MapResult.FIELDS}, "C2T", "G2A", BENCH_PARAMS,
                     d_debug={f: ref[f].data_ptr() for f in MapResult.DEBUG}, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    want = {f: ref[f].cpu().numpy() for f in FIELDS}

    p = BENCH_PARAMS.to_c()
    outs = [_device_outputs(torch, n, dev) for _ in range(2)]
    args = []
    for out in outs:
        for t in out.values():
            t.fill_(-7)
        args.append((_lib.ma_hits(*[out[f].data_ptr() for f in MapResult.FIELDS]),
                     _lib.ma_debug(*[out[f].data_ptr() for f in MapResult.DEBUG])))
    # set-up call (no reads): places the scratch array and loads the kernels
    _lib.check(_lib.lib.ma_map_batch_device_noalloc(gi.handle, d_bases.data_ptr(), d_lens.data_ptr(), 0, 1, 150,
                                                    1, 2, C.byref(p), C.byref(args[0][0]), None,
                                                    stream.cuda_stream))
    torch.cuda.synchronize()
    for call, (out, (hits, dbg)) in enumerate(zip(outs, args)):
        free_before = torch.cuda.mem_get_info(dev)[0]
        rc = _lib.lib.ma_map_batch_device_noalloc(gi.handle, d_bases.data_ptr(), d_lens.data_ptr(), rb.n1, 1, 150,
                                                  1, 2, C.byref(p), C.byref(hits), C.byref(dbg),
                                                  stream.cuda_stream)
        _lib.check(rc)
        torch.cuda.synchronize()
        # the property the entry point exists for: the device's free memory
        # is the same after the call as before it
        assert torch.cuda.mem_get_info(dev)[0] == free_before, f"call {call} changed the free device memory"
        for f in FIELDS:
            got = out[f].cpu().numpy()
            assert np.array_equal(got, want[f]), f"call {call}: field {f} differs from ma_map_batch_device"
    hits = args[0][0]

    # a batch beyond the fixed scratch size is refused with a clear error
    big = 20000  # pairs -> 40000 reads > 32768
    rc = _lib.lib.ma_map_batch_device_noalloc(gi.handle, d_bases.data_ptr(), d_lens.data_ptr(), big, 1, 150, 1, 2,
                                              C.byref(p), C.byref(hits), None, stream.cuda_stream)
    assert rc == _lib.MA_ERR_ARG
    assert "static scratch maximum" in _lib.last_error()
    gi.close()
    ctx.close()
