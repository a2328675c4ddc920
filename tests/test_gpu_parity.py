"""GPU path (through the C ABI) against the oracle, bit-exact.

Every output of the reference kernel (rid, pos, mapq, flag, sl, sr, nm) and
the side outputs (uk, ul, us, e, score) must be identical to the oracle's
restatement of fm_seed_extend_kernel + fm_mate_rescue_kernel
(fq2bam-meth/src/linear_gpu_fm.mojo:1156-2011) on the same reads.  Integer
work: the tolerance is zero.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from mojoalign_b200 import BENCH_PARAMS, FmParams, GpuContext, GpuIndex, MojoAlignError, map_batch, synth

pytestmark = pytest.mark.gpu

FIELDS = ("rid", "pos", "mapq", "flag", "sl", "sr", "nm", "uk", "ul", "us", "e", "score")


@pytest.fixture(scope="module")
def ctx():
    c = GpuContext(0)
    yield c
    c.close()


_INDEX_CACHE = {}


def gpu_index(ctx, prefix, k, k3=0):
    key = (str(prefix), k, k3)
    if key not in _INDEX_CACHE:
        _INDEX_CACHE[key] = GpuIndex(ctx, prefix, kmer_k=k, kmer3_k=k3)
    return _INDEX_CACHE[key]


# Result-neutral kernel forms (seed_kernel, stage1_endpoints,
# stage2_blocks_per_sm, reg_level, stage1_max_rows, stage2_first_wave, wave_endpoints, wave_loci_per_read,
# wave_max_rounds): one thread per read; two stages with the first 1, 2 or 3 right endpoints in stage 1, at
# each register budget; wavefront rounds of several widths, with a locus list too small for the batch (reads
# overflow to the stage-2 warps), with the rounds cut short (the rest finished by stage 2) and with doubling
# round widths; the same with lane refill in the search pass and staged eval (seed_kernel 3), and with the
# staged eval alone (seed_kernel 4).
TUNINGS = [(0, 1, 0, 0, 16, 32), (1, 1, 0, 1, 2, 32), (1, 3, 1, 2, 1, 1), (1, 2, 0, 0, 16, 4), (1, 1, 0, 2, 1, 7),
           (2, 1, 0, 1, 2, 32, 32, 4, 0), (2, 2, 0, 2, 1, 1, 5, 1, 0), (2, 1, 0, 0, 2, 32, 3, 4, 2),
           (2, 1, 0, 1, 1, 1, 4, 2, 0, 1), (3, 1, 0, 1, 2, 32, 32, 4, 0), (3, 2, 0, 2, 1, 1, 5, 1, 0),
           (3, 1, 0, 0, 2, 32, 3, 4, 2), (3, 1, 0, 1, 1, 1, 8, 16, 0, 1), (4, 1, 0, 1, 2, 32, 32, 4, 0),
           (4, 2, 0, 2, 1, 1, 5, 1, 0), (4, 1, 0, 0, 2, 32, 3, 4, 2), (4, 2, 0, 1, 1, 1, 8, 16, 0, 1)]


def compare(prefix, ctx, bases, lens, n1, paired, max_len, params, k=12, bs=(1, 2), tunings=TUNINGS, k3=12):
    gi = gpu_index(ctx, prefix, k, k3)
    o = oracle.OracleIndex(prefix).map(bases, lens, n1, paired, max_len, bs[0], bs[1], params.as_list())
    g = None
    for tu in tunings:
        ctx.set_tuning(*tu)
        g = map_batch(ctx, gi, bases, lens, n1, paired, max_len, bs[0], bs[1], params, debug=True)
        for f in FIELDS:
            a, b = getattr(g, f), o[f]
            bad = np.nonzero(a != b)[0]
            assert bad.size == 0, (
                f"tuning {tu} {f}: {bad.size} of {a.size} reads differ; first read {bad[0]}: "
                f"gpu {a[bad[0]]} oracle {b[bad[0]]}; "
                + ", ".join(f"{x}=({getattr(g, x)[bad[0]]},{o[x][bad[0]]})" for x in FIELDS)
            )
    ctx.set_tuning()
    return g


def sim(fa, n1, paired, max_len=150, seed=1, **model):
    return synth.simulate_reads(fa, synth.ReadModel(**model), n1, paired, max_len, seed=seed)


def test_single_end_default_model(ctx, small_ref):
    fa, prefix = small_ref
    rb = sim(fa, 20000, False)
    g = compare(prefix, ctx, rb.bases, rb.lens, rb.n1, False, 150, BENCH_PARAMS)
    assert (g.rid >= 0).mean() > 0.9


def test_paired_end_with_rescue(ctx, small_ref):
    fa, prefix = small_ref
    rb = sim(fa, 10000, True, seed=2, sub_rate=0.02)
    compare(prefix, ctx, rb.bases, rb.lens, rb.n1, True, 150, BENCH_PARAMS)


@pytest.mark.parametrize("k,k3", [(0, 0), (10, 0), (12, 0), (0, 12), (12, 9), (0, 19)])
def test_kmer_tables_are_exact(ctx, small_ref, k, k3):
    fa, prefix = small_ref
    rb = sim(fa, 5000, True, seed=3, sub_rate=0.01)
    compare(prefix, ctx, rb.bases, rb.lens, rb.n1, True, 150, BENCH_PARAMS, k=k, k3=k3)


def test_high_error_soft_clips_and_deletions(ctx, small_ref):
    fa, prefix = small_ref
    rb = sim(fa, 8000, True, seed=4, sub_rate=0.04, conv_non_cpg=0.9)
    g = compare(prefix, ctx, rb.bases, rb.lens, rb.n1, True, 150, FmParams(seed_len=19, max_occ=500, max_diff=8))
    assert (g.sl > 0).any() or (g.sr > 0).any()


def test_contig_edges(ctx, edgy_ref):
    fa, prefix = edgy_ref
    for paired in (False, True):
        rb = sim(fa, 6000, paired, seed=5, sub_rate=0.01, frag_mean=300)
        compare(prefix, ctx, rb.bases, rb.lens, rb.n1, paired, 150, BENCH_PARAMS)


def test_uneven_and_short_reads(ctx, small_ref):
    fa, prefix = small_ref
    rb = sim(fa, 8000, False, max_len=300, seed=6, len_fixed=0, len_lognorm_median=60, len_lognorm_sigma=0.8,
             len_min=1, len_max=300)
    assert rb.lens.min() < 19
    compare(prefix, ctx, rb.bases, rb.lens, rb.n1, False, 300, BENCH_PARAMS)


def test_long_reads_max_len(ctx, small_ref):
    fa, prefix = small_ref
    rb = sim(fa, 1500, False, max_len=1024, seed=7, len_fixed=0, len_lognorm_median=700, len_lognorm_sigma=0.3,
             len_min=300, len_max=1024, sub_rate=0.01)
    assert rb.lens.max() == 1024 or rb.lens.max() > 900
    compare(prefix, ctx, rb.bases, rb.lens, rb.n1, False, 1024, BENCH_PARAMS)


def test_reads_with_ambiguous_bases(ctx, small_ref):
    fa, prefix = small_ref
    rb = sim(fa, 6000, True, seed=8)
    rng = np.random.default_rng(8)
    for r in rng.choice(rb.n_seq, size=rb.n_seq // 4, replace=False):
        L = int(rb.lens[r])
        for p in rng.integers(0, L, size=int(rng.integers(1, 8))):
            rb.bases[r, p] = rng.choice([ord("N"), ord("n"), ord("R"), ord(".")])
    compare(prefix, ctx, rb.bases, rb.lens, rb.n1, True, 150, BENCH_PARAMS)


PARAM_SETS = [
    FmParams(),
    FmParams(seed_len=12, seed_stride=1, max_occ=5),
    FmParams(seed_len=25, seed_stride=3, max_occ=4096, max_diff=30),
    FmParams(seed_len=19, max_occ=500, max_diff=2, max_soft=0, max_adj=0),
    FmParams(seed_len=19, max_occ=500, max_soft=300, max_adj=12, rescue_win=5000),
    FmParams(seed_len=8, seed_stride=5, max_occ=64, max_adj=20, rescue_win=10),
    FmParams(seed_len=19, max_occ=1, max_diff=1, max_soft=5, max_adj=3, rescue_win=32),
]


@pytest.mark.parametrize("params", PARAM_SETS, ids=lambda p: "-".join(map(str, p.as_list())))
def test_parameter_sweep(ctx, edgy_ref, params):
    fa, prefix = edgy_ref
    rb = sim(fa, 3000, True, seed=9, sub_rate=0.02)
    compare(prefix, ctx, rb.bases, rb.lens, rb.n1, True, 150, params)


def test_unconverted_reads_all_modes(ctx, small_ref):
    fa, prefix = small_ref
    rb = sim(fa, 4000, True, seed=10, conv_non_cpg=0.0, cpg_retain=1.0)
    for bs in ((0, 0), (2, 1), (1, 1)):
        compare(prefix, ctx, rb.bases, rb.lens, rb.n1, True, 150, BENCH_PARAMS, bs=bs)


def _ref_text(fa):
    seqs = []
    for block in open(fa).read().split(">")[1:]:
        lines = block.splitlines()
        seqs.append("".join(lines[1:]).upper())
    return seqs


def test_deletions_and_text_start(ctx, small_ref):
    """Reads with a 1-bp deletion (deletion probe) and reads overhanging the
    first contig's start (negative text positions in the probe)."""
    fa, prefix = small_ref
    chrom = _ref_text(fa)[0].replace("C", "T")  # f-strand-like reads (C->T)
    rng = np.random.default_rng(11)
    reads = []
    for _ in range(3000):
        p = int(rng.integers(0, len(chrom) - 200))
        s = chrom[p:p + 151]
        g = int(rng.integers(10, 140))
        reads.append(s[:g] + s[g + 1:])
    for _ in range(600):
        pre = "".join(rng.choice(list("AGT"), size=int(rng.integers(1, 30))))
        reads.append((pre + chrom[: 150])[:150])
    n = len(reads)
    bases = np.full((n, 150), ord("N"), np.uint8)
    lens = np.zeros(n, np.uint32)
    for i, s in enumerate(reads):
        bases[i, : len(s)] = np.frombuffer(s.encode(), np.uint8)
        lens[i] = len(s)
    for params in (BENCH_PARAMS, FmParams(seed_len=19, max_occ=500, max_diff=3, max_soft=30)):
        compare(prefix, ctx, bases, lens, n, False, 150, params)


def test_empty_batch_and_errors(ctx, small_ref):
    fa, prefix = small_ref
    gi = gpu_index(ctx, prefix, 12)
    bases = np.zeros((0, 150), np.uint8)
    lens = np.zeros(0, np.uint32)
    r = map_batch(ctx, gi, bases, lens, 0, False, 150)
    assert r.rid.size == 0
    bases = np.full((2, 8), ord("A"), np.uint8)
    with pytest.raises(MojoAlignError) as e:
        map_batch(ctx, gi, bases, np.array([8, 9], np.uint32), 2, False, 8)
    assert e.value.code == -1
    with pytest.raises(MojoAlignError):
        map_batch(ctx, gi, bases, np.array([8, 8], np.uint32), 2, False, 8, params=FmParams(seed_stride=0))
    # the context still works after a rejected call
    rb = sim(fa, 500, False, seed=12)
    compare(prefix, ctx, rb.bases, rb.lens, rb.n1, False, 150, BENCH_PARAMS)


def test_toy_fixture_shape(ctx, tmp_path):
    """The reference's toy fixture shape (fq2bam-meth/tests/data/fq2bam_fixture):
    a 64-bp A/T-alternating chr1 and two exact 32-bp PE reads."""
    from mojoalign_b200 import build_index

    fa = tmp_path / "ref.fa"
    fa.write_text(">chr1\n" + "AT" * 32 + "\n")
    prefix = tmp_path / "ref.fa.bwameth.c2t"
    build_index(fa, prefix, bwameth_c2t=True, sa_intv=32)
    read = np.frombuffer(("AT" * 16).encode(), np.uint8)
    bases = np.stack([read, read])
    lens = np.array([32, 32], np.uint32)
    for p in (FmParams(), FmParams(seed_len=19), FmParams(seed_len=8, max_occ=4096)):
        compare(prefix, ctx, bases, lens, 1, True, 32, p, k=0, k3=0)
        compare(prefix, ctx, bases, lens, 1, True, 32, p, k=4, k3=8)


def test_host_batch_pipeline_matches_device_batch(ctx, small_ref):
    """ma_map_batch pipelines large batches in chunks of pairs over two
    streams; its outputs must equal one device-resident launch."""
    torch = pytest.importorskip("torch")
    from mojoalign_b200 import MapResult, map_batch_device

    fa, prefix = small_ref
    gi = gpu_index(ctx, prefix, 12, 12)
    rb = sim(fa, 300_000, True, seed=31, sub_rate=0.01)
    host = map_batch(ctx, gi, rb.bases, rb.lens, rb.n1, True, 150, "C2T", "G2A", BENCH_PARAMS, debug=True)
    dev = torch.device("cuda:0")
    d_bases = torch.from_numpy(rb.bases.reshape(-1)).to(dev)
    d_lens = torch.from_numpy(rb.lens.view(np.int32)).to(dev)
    out = {f: torch.empty(rb.n_seq, dtype=torch.int64 if f in ("uk", "ul") else torch.int32, device=dev)
           for f in FIELDS}
    map_batch_device(ctx, gi, d_bases.data_ptr(), d_lens.data_ptr(), rb.n1, True, 150,
                     {f: out[f].data_ptr() for f in MapResult.FIELDS}, "C2T", "G2A", BENCH_PARAMS,
                     d_debug={f: out[f].data_ptr() for f in MapResult.DEBUG},
                     stream=torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize()
    for f in FIELDS:
        assert np.array_equal(out[f].cpu().numpy(), getattr(host, f).view(out[f].cpu().numpy().dtype)), f


@pytest.mark.parametrize("chunking", [(0, 50, 0, 3), (7000, 0, 7000, 1), (5000, 50, 60000, 2), (1, 100, 3, 3)])
def test_host_batch_pinned_and_pageable_arrays(ctx, small_ref, chunking):
    """ma_map_batch with page-locked lengths and outputs (copied directly)
    and with pageable ones (staged through the context's page-locked
    buffers): equal outputs for every chunking of the pipeline, pairs and
    single-end, the staged outputs of every slot delivered."""
    torch = pytest.importorskip("torch")
    from mojoalign_b200 import MapResult, map_batch_device

    fa, prefix = small_ref
    gi = gpu_index(ctx, prefix, 12, 12)
    dev = torch.device("cuda:0")
    for paired, n in ((True, 20_000), (False, 30_011)):
        rb = sim(fa, n, paired, seed=41 + paired, sub_rate=0.01)
        if chunking[2] == 3:
            rb = sim(fa, 40, paired, seed=43, sub_rate=0.01)  # chunks of 1, 2, 3 pairs
        # the device-resident call is the reference
        d_bases = torch.from_numpy(rb.bases.reshape(-1)).to(dev)
        d_lens = torch.from_numpy(rb.lens.view(np.int32)).to(dev)
        d_out = {f: torch.empty(rb.n_seq, dtype=torch.int64 if f in ("uk", "ul") else torch.int32, device=dev)
                 for f in FIELDS}
        map_batch_device(ctx, gi, d_bases.data_ptr(), d_lens.data_ptr(), rb.n1, paired, 150,
                         {f: d_out[f].data_ptr() for f in MapResult.FIELDS}, "C2T", "G2A", BENCH_PARAMS,
                         d_debug={f: d_out[f].data_ptr() for f in MapResult.DEBUG},
                         stream=torch.cuda.current_stream(dev).cuda_stream)
        torch.cuda.synchronize()
        ref = {f: d_out[f].cpu().numpy() for f in FIELDS}
        ctx.set_pipeline(*chunking)
        try:
            want = map_batch(ctx, gi, rb.bases, rb.lens, rb.n1, paired, 150, "C2T", "G2A", BENCH_PARAMS, debug=True)
            pin = MapResult.empty(rb.n_seq, debug=True)
            for f in FIELDS:
                a = getattr(pin, f)
                t = torch.empty(a.size, dtype=torch.int64 if a.itemsize == 8 else torch.int32, pin_memory=True)
                setattr(pin, f, t.numpy().view(a.dtype))
            lens = torch.from_numpy(rb.lens.view(np.int32).copy()).pin_memory().numpy().view(np.uint32)
            bases = torch.from_numpy(rb.bases.copy()).pin_memory().numpy()
            got = map_batch(ctx, gi, bases, lens, rb.n1, paired, 150, "C2T", "G2A", BENCH_PARAMS, out=pin)
        finally:
            ctx.set_pipeline()
        for f in FIELDS:
            assert np.array_equal(getattr(want, f).view(ref[f].dtype), ref[f]), ("pageable", paired, f)
            assert np.array_equal(getattr(got, f).view(ref[f].dtype), ref[f]), ("page-locked", paired, f)


@pytest.fixture(scope="module")
def config0_ref(tmp_path_factory):
    """The reference's CPU-runnable case: synthetic 4 Mbp, GC 0.41, CpG ~1%, seed 0."""
    from pathlib import Path

    from mojoalign_b200 import build_index

    d = tmp_path_factory.mktemp("config0")
    fa = d / "ref.fa"
    synth.write_reference(fa, 4_000_000, n_contigs=1, gc=0.41, cpg=0.01, seed=0)
    prefix = Path(str(fa) + ".bwameth.c2t")
    build_index(fa, prefix, bwameth_c2t=True, sa_intv=32, device=-1)
    return fa, prefix


def test_config0_in_full(ctx, config0_ref):
    """100 k single-end 150 bp reads from both strands (conversion 0.99, CpG
    retention 0.75, 0.5% substitutions, 5% random reads, seed 1), seeds of
    19 bp with at most 500 occurrences: every output, the SA intervals and
    scores included, equal to the oracle's, in the reference's launch shape
    and in the wavefront form."""
    fa, prefix = config0_ref
    rb = sim(fa, 100_000, False)
    g = compare(prefix, ctx, rb.bases, rb.lens, rb.n1, False, 150, BENCH_PARAMS, bs=(1, 0),
                tunings=[TUNINGS[0], TUNINGS[5]])
    assert 0.9 < (g.rid >= 0).mean() < 0.97  # the 5% random reads stay unmapped
