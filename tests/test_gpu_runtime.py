"""Runtime behaviour on the GPU: HBM admission (the analogue of
gpu_mem.require_index_capacity, gpu-common/python/gpu_mem.py:203-329),
determinism and launch accounting."""
from __future__ import annotations

import numpy as np
import pytest

from mojoalign_b200 import BENCH_PARAMS, GpuContext, GpuIndex, MojoAlignError, map_batch, probe_index, synth
from mojoalign_b200 import _lib

pytestmark = pytest.mark.gpu


def test_hbm_admission_fails_closed(small_ref):
    _, prefix = small_ref
    with GpuContext(0) as ctx:
        free, total = ctx.hbm_info()
        assert 0 < free <= total
        with pytest.raises(MojoAlignError) as e:
            GpuIndex(ctx, prefix, kmer_k=12, kmer3_k=12, hbm_budget_bytes=1 << 20)
        assert e.value.code == _lib.MA_ERR_NOMEM and "MiB" in str(e.value)
        need = probe_index(prefix, 12, 12).device_bytes
        with GpuIndex(ctx, prefix, kmer_k=12, kmer3_k=12, hbm_budget_bytes=need + (64 << 20)) as gi:
            assert gi.info.device_bytes <= need


def test_repeatable_and_launch_count(small_ref):
    fa, prefix = small_ref
    rb = synth.simulate_reads(fa, synth.ReadModel(), 3000, True, 150, seed=41)
    with GpuContext(0) as ctx, GpuIndex(ctx, prefix, kmer_k=12, kmer3_k=12) as gi:
        ctx.set_tuning(1, 1, 0, 2, 1, 1)  # the two-stage form
        a = map_batch(ctx, gi, rb.bases, rb.lens, rb.n1, True, 150, "C2T", "G2A", BENCH_PARAMS, debug=True)
        assert ctx.last_launch_count() == 4  # pack, stage 1, stage 2, rescue
        b = map_batch(ctx, gi, rb.bases, rb.lens, rb.n1, True, 150, "C2T", "G2A", BENCH_PARAMS, debug=True)
        for f in a.FIELDS + a.DEBUG:
            assert np.array_equal(getattr(a, f), getattr(b, f)), f
        se = map_batch(ctx, gi, rb.bases[: rb.n1], rb.lens[: rb.n1], rb.n1, False, 150, "C2T", "", BENCH_PARAMS)
        assert ctx.last_launch_count() == 3  # no rescue for single-end reads
        assert se.rid.size == rb.n1


@pytest.mark.parametrize("pipeline", [(1000, 0, 1000, 1), (1000, 50, 2500, 2), (700, 100, 0, 3), (0, 50, 0, 1)])
def test_pipeline_chunking_is_result_neutral(small_ref, pipeline):
    """Chunk sizes, growth and compute lanes of map_batch's copy / compute
    pipeline change no output (pairs are never split across chunks)."""
    fa, prefix = small_ref
    rb = synth.simulate_reads(fa, synth.ReadModel(), 9000, True, 150, seed=43)
    with GpuContext(0) as ctx, GpuIndex(ctx, prefix, kmer_k=12, kmer3_k=12) as gi:
        ctx.set_tuning(2, 1, 0, 2, 1, 1, 8, 4, 0, 1)
        ctx.set_pipeline(9000, 0, 9000, 1)  # one chunk
        a = map_batch(ctx, gi, rb.bases, rb.lens, rb.n1, True, 150, "C2T", "G2A", BENCH_PARAMS, debug=True)
        ctx.set_pipeline(*pipeline)
        for _ in range(2):
            b = map_batch(ctx, gi, rb.bases, rb.lens, rb.n1, True, 150, "C2T", "G2A", BENCH_PARAMS, debug=True)
            for f in a.FIELDS + a.DEBUG:
                assert np.array_equal(getattr(a, f), getattr(b, f)), (pipeline, f)
        with pytest.raises(MojoAlignError):
            ctx.set_pipeline(0, 50, 0, 4)
