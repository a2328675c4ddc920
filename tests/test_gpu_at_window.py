"""The A/T window outcome table (index options at_k / at_seed_len) against
the oracle, bit-exact.

With the table, a search whose last at_k bases are all A or T takes its
outcome (a seed, no seed, or the interval to continue from) from one lookup
instead of the backward steps of fm_seed_extend_kernel
(fq2bam-meth/src/linear_gpu_fm.mojo:1235-1385).  The outputs must not
change: all 12 outputs are compared with the oracle in every kernel form of
TUNINGS, on references where A/T windows are common (an A/T-rich genome, a
repeat-heavy genome), with reads from both strand origins, with max_occ
below 16 (the stop at seed_len that the table defers to the steps), with a
seed length the table was not built for (table unused), and with windows
long enough to run past the read start.  Integer work: the tolerance is
zero.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import oracle
from mojoalign_b200 import BENCH_PARAMS, FmParams, GpuContext, GpuIndex, map_batch, synth
from test_gpu_parity import FIELDS, TUNINGS

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = GpuContext(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def at_rich_ref(tmp_path_factory):
    """A 1 Mbp reference with GC 0.12 in 4 contigs: most converted windows
    of 20-28 bases hold only A and T, so every outcome kind occurs."""
    from mojoalign_b200 import build_index

    d = tmp_path_factory.mktemp("at_rich_ref")
    fa = d / "ref.fa"
    synth.write_reference(fa, 1_000_000, n_contigs=4, gc=0.12, seed=21)
    prefix = Path(str(fa) + ".bwameth.c2t")
    build_index(fa, prefix, bwameth_c2t=True, sa_intv=32, device=-1)
    return fa, prefix


def _reads(fa, n1, paired, max_len, seed, **model):
    return synth.simulate_reads(fa, synth.ReadModel(**model), n1, paired, max_len, seed=seed)


UNEVEN = dict(len_fixed=0, len_lognorm_median=120.0, len_lognorm_sigma=0.35, len_min=36, len_max=300,
              non_directional=0.5)


def _compare(ctx, prefix, rb, paired, max_len, params, at_k, at_seed_len, k3=19, tunings=TUNINGS):
    """Every tuning's 12 outputs with the table equal the oracle's."""
    o = oracle.OracleIndex(prefix).map(rb.bases, rb.lens, rb.n1, paired, max_len, 1, 2, params.as_list())
    with GpuIndex(ctx, prefix, kmer_k=12, kmer3_k=min(k3, params.seed_len), at_k=at_k,
                  at_seed_len=at_seed_len) as gi:
        for tu in tunings:
            ctx.set_tuning(*tu)
            g = map_batch(ctx, gi, rb.bases, rb.lens, rb.n1, paired, max_len, 1, 2, params, debug=True)
            for f in FIELDS:
                a, b = getattr(g, f), o[f]
                bad = np.nonzero(a != b)[0]
                assert bad.size == 0, (
                    f"at_k {at_k} tuning {tu} {f}: {bad.size} of {a.size} reads differ; first read {bad[0]}: "
                    + ", ".join(f"{x}=({getattr(g, x)[bad[0]]},{o[x][bad[0]]})" for x in FIELDS))
    ctx.set_tuning()
    return o


def _occ_lines(ctx, prefix, rb, paired, max_len, params, **opts):
    """Occ lines the counting kernels tally for one call."""
    with GpuIndex(ctx, prefix, kmer_k=12, kmer3_k=min(19, params.seed_len), **opts) as gi:
        ctx.set_profiling(2)
        try:
            map_batch(ctx, gi, rb.bases, rb.lens, rb.n1, paired, max_len, 1, 2, params)
            return ctx.traffic()[0]
        finally:
            ctx.set_profiling(0)


@pytest.mark.parametrize("at_k", [20, 24, 28])
def test_uneven_reads_both_strand_origins(ctx, at_rich_ref, at_k):
    fa, prefix = at_rich_ref
    rb = _reads(fa, 12000, False, 300, 31, **UNEVEN)
    o = _compare(ctx, prefix, rb, False, 300, BENCH_PARAMS, at_k, BENCH_PARAMS.seed_len)
    assert (o["rid"] >= 0).mean() > 0.3


def test_table_replaces_backward_steps(ctx, at_rich_ref):
    """The table is used: the same call takes fewer Occ lines with it."""
    fa, prefix = at_rich_ref
    rb = _reads(fa, 20000, False, 300, 32, **UNEVEN)
    without = _occ_lines(ctx, prefix, rb, False, 300, BENCH_PARAMS)
    with_table = _occ_lines(ctx, prefix, rb, False, 300, BENCH_PARAMS, at_k=24, at_seed_len=19)
    assert with_table < 0.8 * without, (with_table, without)


def test_pairs_2x150(ctx, at_rich_ref):
    fa, prefix = at_rich_ref
    rb = _reads(fa, 6000, True, 150, 33, sub_rate=0.01)
    _compare(ctx, prefix, rb, True, 150, BENCH_PARAMS, 24, 19)


@pytest.mark.parametrize("params,at_k", [
    (FmParams(seed_len=14, max_occ=8), 18),                  # max_occ < 16: the seed_len stop keeps an interval
    (FmParams(seed_len=14, max_occ=40, seed_stride=1), 20),  # many capped searches, stride 1
    (FmParams(seed_len=12, max_occ=500, max_diff=6), 12),    # window = seed length
    (FmParams(seed_len=19, max_occ=500), 30),                # longest window
])
def test_parameter_sweep(ctx, at_rich_ref, params, at_k):
    fa, prefix = at_rich_ref
    rb = _reads(fa, 6000, False, 300, 34, **UNEVEN)
    _compare(ctx, prefix, rb, False, 300, params, at_k, params.seed_len, k3=19, tunings=TUNINGS[::2])


def test_seed_length_the_table_was_not_built_for(ctx, at_rich_ref):
    fa, prefix = at_rich_ref
    rb = _reads(fa, 6000, False, 300, 35, **UNEVEN)
    _compare(ctx, prefix, rb, False, 300, FmParams(seed_len=18, max_occ=500), 24, 19, tunings=TUNINGS[::4])


def test_short_reads_and_windows_at_the_read_start(ctx, at_rich_ref):
    """Reads of 20-40 bases: windows that end where the read starts."""
    fa, prefix = at_rich_ref
    rb = _reads(fa, 8000, False, 64, 36, len_fixed=0, len_lognorm_median=30, len_lognorm_sigma=0.3, len_min=20,
                len_max=64, non_directional=0.5)
    _compare(ctx, prefix, rb, False, 64, FmParams(seed_len=16, max_occ=500), 20, 16, tunings=TUNINGS[::2])


def test_repeat_heavy_reference(ctx, repeat_ref):
    fa, prefix = repeat_ref
    rb = _reads(fa, 8000, False, 300, 37, **UNEVEN)
    _compare(ctx, prefix, rb, False, 300, BENCH_PARAMS, 26, 19)


def test_bad_options_fail_closed(ctx, at_rich_ref):
    from mojoalign_b200 import MojoAlignError

    _, prefix = at_rich_ref
    for at_k, sl in ((31, 19), (18, 19), (20, 0)):
        with pytest.raises(MojoAlignError):
            GpuIndex(ctx, prefix, kmer_k=12, at_k=at_k, at_seed_len=sl)
