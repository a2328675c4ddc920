"""GPU path against the oracle on repeat-heavy references, bit-exact.

The kernels reach the reference's answer through exactness arguments (locus
memo, duplicate prediction from the seed summary, the early stop for
nm <= 2 from unique segments, the shift filter).  Those arguments are most
at risk where the text repeats: seeds with many occurrences, the max_occ
stop (fq2bam-meth/src/linear_gpu_fm.mojo:1378-1379), the <= 16-row fallback
(L1374-1385), many candidate loci per read and near-ties between copies.
These tests map reads of the repeat-heavy configuration (2x250 pairs,
non-CpG conversion 0.97) and uneven single-end reads on such references, in
every kernel form of TUNINGS and with the interval tables up to k = 19, and
compare all 12 outputs with the oracle.  Integer work: the tolerance is zero.
"""
from __future__ import annotations

import pytest

import oracle
from mojoalign_b200 import BENCH_PARAMS, FmParams, GpuContext, synth
from test_gpu_parity import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = GpuContext(0)
    yield c
    c.close()


def _reads(fa, n1, paired, max_len, seed, **model):
    return synth.simulate_reads(fa, synth.ReadModel(**model), n1, paired, max_len, seed=seed)


def _assert_stressed(prefix, rb, paired, max_len, params):
    """The oracle on these reads meets the cap and the fallback."""
    ct = oracle.OracleIndex(prefix).map(rb.bases, rb.lens, rb.n1, paired, max_len, 1, 2, params.as_list(),
                                        counters=True)["counters"]
    assert ct["capped"] > 0 and ct["fallback"] > 0, ct


@pytest.mark.parametrize("k,k3", [(12, 19), (12, 12), (0, 0)])
def test_repeat_heavy_pairs_2x250(ctx, repeat_ref, k, k3):
    fa, prefix = repeat_ref
    rb = _reads(fa, 6000, True, 250, 11, len_fixed=250, conv_non_cpg=0.97)
    _assert_stressed(prefix, rb, True, 250, BENCH_PARAMS)
    g = compare(prefix, ctx, rb.bases, rb.lens, rb.n1, True, 250, BENCH_PARAMS, k=k, k3=k3)
    assert (g.rid >= 0).mean() > 0.8


def test_repeat_heavy_uneven_single_end(ctx, repeat_ref):
    fa, prefix = repeat_ref
    rb = _reads(fa, 12000, False, 300, 12, len_fixed=0, len_lognorm_median=120, len_lognorm_sigma=0.35,
                len_min=36, len_max=300, non_directional=0.5)
    compare(prefix, ctx, rb.bases, rb.lens, rb.n1, False, 300, BENCH_PARAMS, k=12, k3=19)


@pytest.mark.parametrize("k3", [19, 12])
def test_young_repeats_pairs(ctx, young_repeat_ref, k3):
    fa, prefix = young_repeat_ref
    rb = _reads(fa, 6000, True, 150, 13, sub_rate=0.01)
    _assert_stressed(prefix, rb, True, 150, BENCH_PARAMS)
    compare(prefix, ctx, rb.bases, rb.lens, rb.n1, True, 150, BENCH_PARAMS, k=12, k3=k3)


@pytest.mark.parametrize("params", [FmParams(seed_len=19, max_occ=50), FmParams(seed_len=17, seed_stride=1,
                                                                                 max_occ=20, max_diff=6),
                                    FmParams(seed_len=22, seed_stride=3, max_occ=4096)])
def test_young_repeats_parameter_sweep(ctx, young_repeat_ref, params):
    fa, prefix = young_repeat_ref
    rb = _reads(fa, 3000, True, 250, 14, len_fixed=250, conv_non_cpg=0.97, sub_rate=0.01)
    compare(prefix, ctx, rb.bases, rb.lens, rb.n1, True, 250, params, k=12, k3=19)
