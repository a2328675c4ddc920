"""Device mapping calls replayed from a captured CUDA graph.

With ma_ctx_set_graphs(ctx, 1) the second call with the same arguments
captures the launch sequence (pack, the wavefront rounds, stage 2, rescue)
into a graph and later calls launch it.  The outputs must not change: every
call equals the uncaptured call and the oracle, also after the arguments
change (a new batch size: the graph is rebuilt) and back.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from mojoalign_b200 import BENCH_PARAMS, GpuContext, GpuIndex, MapResult, map_batch_device, synth

pytestmark = pytest.mark.gpu


def test_graph_replay_equals_plain_calls(small_ref):
    torch = pytest.importorskip("torch")
    fa, prefix = small_ref
    ctx = GpuContext(0)
    gi = GpuIndex(ctx, prefix, kmer_k=12, kmer3_k=12)
    dev = torch.device("cuda:0")
    rb = synth.simulate_reads(fa, synth.ReadModel(sub_rate=0.01), 6000, True, 150, seed=41)
    o = oracle.OracleIndex(prefix).map(rb.bases, rb.lens, rb.n1, True, 150, 1, 2, BENCH_PARAMS.as_list())
    d_b = torch.from_numpy(rb.bases.reshape(-1)).to(dev)
    d_l = torch.from_numpy(rb.lens.view(np.int32)).to(dev)
    stream = torch.cuda.Stream(dev)  # the calls and the torch work share one stream
    torch.cuda.set_stream(stream)
    out = {f: torch.empty(rb.n_seq, dtype=torch.int32, device=dev) for f in MapResult.FIELDS}
    ptrs = {f: x.data_ptr() for f, x in out.items()}

    def call(n1):
        for x in out.values():
            x.fill_(-9)
        map_batch_device(ctx, gi, d_b.data_ptr(), d_l.data_ptr(), n1, True, 150, ptrs, "C2T", "G2A", BENCH_PARAMS,
                         stream=stream.cuda_stream)
        torch.cuda.synchronize()
        return {f: x.cpu().numpy() for f, x in out.items()}

    plain = call(rb.n1)
    plain_launches = ctx.last_launch_count()
    ctx.set_graphs(True)
    for n1 in (rb.n1, rb.n1, rb.n1, rb.n1 // 2, rb.n1 // 2, rb.n1 // 2, rb.n1, rb.n1):
        got = call(n1)
        n = 2 * n1
        if n1 == rb.n1:
            for f in MapResult.FIELDS:
                assert np.array_equal(got[f], plain[f]), f
                assert np.array_equal(got[f].view(o[f].dtype), o[f]), f
            assert ctx.last_launch_count() == plain_launches
        else:
            # half the pairs: the call's rows are the first 2 * n1 rows of
            # the buffer (its R2 rows are rows n1 .. 2 * n1 - 1)
            oh = oracle.OracleIndex(prefix).map(rb.bases[:n], rb.lens[:n], n1, True, 150, 1, 2,
                                                BENCH_PARAMS.as_list())
            for f in MapResult.FIELDS:
                assert np.array_equal(got[f][:n].view(oh[f].dtype), oh[f]), f
            assert (got["rid"][n:] == -9).all()  # nothing written past the call's reads
    ctx.set_graphs(False)
    torch.cuda.synchronize()
    torch.cuda.set_stream(torch.cuda.default_stream(dev))
    gi.close()
    ctx.close()
