"""Resident-layout choices are result-neutral (GPU against the oracle).

Texts of 2^32 symbols or more store SA rows as 40-bit values and count Occ
symbols from 2^31-position superblocks; the k-mer tables and the seed
summary are prepared in chunks of SA rows.  Those paths are forced here on
small references (40-bit rows, superblocks of 2^8..2^12 positions, chunks
of a few thousand rows) and every output must equal the oracle's.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from mojoalign_b200 import BENCH_PARAMS, GpuContext, GpuIndex, map_batch, synth

pytestmark = pytest.mark.gpu

FIELDS = ("rid", "pos", "mapq", "flag", "sl", "sr", "nm", "uk", "ul", "us", "e", "score")
LAYOUTS = [dict(wide_rows=True), dict(occ_super_shift=8), dict(occ_super_shift=12, prep_chunk_rows=4096),
           dict(wide_rows=True, occ_super_shift=7, prep_chunk_rows=1000)]


@pytest.fixture(scope="module")
def ctx():
    c = GpuContext(0)
    yield c
    c.close()


def _check(ctx, fa, prefix, layout, paired, max_len, seed, **model):
    rb = synth.simulate_reads(fa, synth.ReadModel(**model), 4000, paired, max_len, seed=seed)
    o = oracle.OracleIndex(prefix).map(rb.bases, rb.lens, rb.n1, paired, max_len, 1, 2, BENCH_PARAMS.as_list())
    for tuning in ((0, 1, 0, 0, 16, 32), (2, 1, 0, 1, 2, 32, 8, 4, 0, 1), (3, 1, 0, 1, 2, 32, 8, 16, 0, 1),
                   (4, 1, 0, 1, 2, 32, 8, 16, 0, 1)):
        ctx.set_tuning(*tuning)
        with GpuIndex(ctx, prefix, kmer_k=12, kmer3_k=19, **layout) as gi:
            g = map_batch(ctx, gi, rb.bases, rb.lens, rb.n1, paired, max_len, 1, 2, BENCH_PARAMS, debug=True)
        for f in FIELDS:
            bad = np.nonzero(getattr(g, f) != o[f])[0]
            assert bad.size == 0, f"layout {layout} tuning {tuning} {f}: {bad.size} reads differ"
    ctx.set_tuning()


@pytest.mark.parametrize("layout", LAYOUTS)
def test_layouts_small_reference(ctx, small_ref, layout):
    fa, prefix = small_ref
    _check(ctx, fa, prefix, layout, True, 150, 31, sub_rate=0.01)


@pytest.mark.parametrize("layout", LAYOUTS[1:])
def test_layouts_repeat_reference(ctx, repeat_ref, layout):
    fa, prefix = repeat_ref
    _check(ctx, fa, prefix, layout, True, 250, 32, len_fixed=250, conv_non_cpg=0.97)
