"""End to end: FASTQ files -> sorted, duplicate-marked BAM on the GPU
(map_fastq_to_bam / map_fastq_fm_gpu with a .bam destination) against the
same path restated on the CPU from the oracle (tests/fq2bam_oracle.py):
byte-identical files at BGZF level 0, identical content at level 1, for
paired and single-end input, gzip input, several batch and chunk sizes,
with and without duplicate marking."""
from __future__ import annotations

import gzip

import numpy as np
import pytest

import fq2bam_oracle
from mojoalign_b200 import FmParams, GpuContext, GpuIndex, synth
from mojoalign_b200.fq2bam import bam_header, map_fastq_to_bam
from mojoalign_b200.linear_fm import map_fastq_fm_gpu

pytestmark = pytest.mark.gpu

PARAMS = FmParams(seed_len=19, max_occ=500)


def write_fastq(path, rb, rows, mate, seed, dup_every=0, gz=False):
    rng = np.random.default_rng(seed)
    out = []
    for k, i in enumerate(rows):
        j = i if not dup_every or k % dup_every else rows[max(0, k - 1)]  # repeat the previous read: a duplicate
        seq = rb.bases[j, :rb.lens[j]].tobytes()
        qual = rng.integers(35, 75, size=len(seq), dtype=np.uint8).tobytes()
        out.append(b"@r%07d %d:N:0:ACGT\n%s\n+\n%s\n" % (k, mate, seq, qual))
    data = b"".join(out)
    if gz:
        with gzip.open(path, "wb") as fh:
            fh.write(data)
    else:
        path.write_bytes(data)


@pytest.fixture(scope="module")
def reads(small_ref, tmp_path_factory):
    fa, prefix = small_ref
    d = tmp_path_factory.mktemp("fq2bam")
    model = synth.ReadModel(len_fixed=0, len_lognorm_median=110, len_min=36, len_max=250, non_directional=0.3)
    n1 = 6000
    rb = synth.simulate_reads(fa, model, n1, True, 250, seed=9)
    r1, r2 = d / "r1.fq", d / "r2.fq"
    write_fastq(r1, rb, list(range(n1)), 1, 1, dup_every=7)
    write_fastq(r2, rb, list(range(n1, 2 * n1)), 2, 2, dup_every=7)
    r1gz = d / "r1.fq.gz"
    write_fastq(r1gz, rb, list(range(n1)), 1, 1, dup_every=7, gz=True)
    return fa, prefix, d, r1, r2, r1gz


@pytest.fixture(scope="module")
def gi(small_ref):
    fa, prefix = small_ref
    ctx = GpuContext(0)
    g = GpuIndex(ctx, prefix, kmer_k=12, kmer3_k=PARAMS.seed_len)
    yield ctx, g
    g.close()
    ctx.close()


def _want(prefix, r1, r2, contigs, level, markdup=True):
    header = bam_header(contigs, {})
    return fq2bam_oracle.fq2bam(prefix, r1, r2, PARAMS.as_list(), 1, 2, header, b"mojo1", level, markdup)


@pytest.mark.parametrize("batch_pairs,chunk", [(1 << 20, 256 << 20), (1000, 100_000), (777, 1 << 20)])
def test_paired_level0_byte_identical(reads, gi, tmp_path, batch_pairs, chunk):
    fa, prefix, d, r1, r2, _ = reads
    ctx, g = gi
    out = tmp_path / "o.bam"
    n = map_fastq_to_bam(fa, r1, out, fq2=r2, bs_r1="C2T", bs_r2="G2A", params=PARAMS, environ={}, ctx=ctx,
                         index=g, batch_pairs=batch_pairs, chunk_bytes=chunk, level=0)
    want = _want(prefix, r1, r2, g.contigs, 0)
    got = out.read_bytes()
    assert got == want
    assert n > 0


def test_level1_content_and_options(reads, gi, tmp_path):
    fa, prefix, d, r1, r2, r1gz = reads
    ctx, g = gi
    out = tmp_path / "o.bam"
    map_fastq_to_bam(fa, r1, out, fq2=r2, bs_r1="C2T", bs_r2="G2A", params=PARAMS, environ={}, ctx=ctx, index=g,
                     batch_pairs=2500, level=1)
    assert gzip.decompress(out.read_bytes()) == gzip.decompress(_want(prefix, r1, r2, g.contigs, 0))
    # single-end, gzip input, no duplicate marking
    map_fastq_to_bam(fa, r1gz, out, bs_r1="C2T", params=PARAMS, environ={"METHYLGRAPHER_LINEAR_MARKDUP": "0"},
                     ctx=ctx, index=g, batch_pairs=1500, level=0)
    assert out.read_bytes() == _want(prefix, r1, None, g.contigs, 0, markdup=False)


def test_drop_in_bam_destination(reads, gi, tmp_path):
    fa, prefix, d, r1, r2, _ = reads
    ctx, g = gi
    out = tmp_path / "drop.bam"
    n = map_fastq_fm_gpu(fa, r1, out, fq2=r2, bs_r1="C2T", bs_r2="G2A", params=PARAMS,
                         environ={"METHYLGRAPHER_BAM_LEVEL": "0"}, ctx=ctx, index=g)
    assert out.read_bytes() == _want(prefix, r1, r2, g.contigs, 0)
    assert n > 0
