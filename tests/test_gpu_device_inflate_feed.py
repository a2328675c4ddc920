"""BGZF FASTQ inputs inflated on the device inside the file pipelines.

The reference decompresses gzip FASTQ on the host (`pigz -dc` or the gzip
module: fq2bam-meth/src/linear_fastq.mojo:131-230,
fq2bam-meth/python/fastq_batch.py:31-46).  For BGZF inputs (bgzip / htslib)
the pipelines here copy the compressed members to the device and inflate
them there, one warp per member, carrying the partial record at the end of
each piece to the next piece on the device.  The BAM and SAM files must be
the same as with the host reader, and only the compressed bytes cross PCIe.
"""
from __future__ import annotations

import pytest

from mojoalign_b200 import FmParams, GpuContext, GpuIndex, synth
from mojoalign_b200.fq2bam import map_fastq_to_bam
from mojoalign_b200.fq2sam import map_fastq_to_sam
from oracle import bgzf_ref
from test_gpu_fq2bam import write_fastq

pytestmark = pytest.mark.gpu

PARAMS = FmParams(seed_len=19, max_occ=500)


@pytest.fixture(scope="module")
def bgzf_reads(small_ref, tmp_path_factory):
    fa, prefix = small_ref
    d = tmp_path_factory.mktemp("devinflate")
    model = synth.ReadModel(len_fixed=0, len_lognorm_median=110, len_min=36, len_max=250)
    n1 = 8000
    rb = synth.simulate_reads(fa, model, n1, True, 250, seed=19)
    plain = []
    for m, rows in ((1, range(n1)), (2, range(n1, 2 * n1))):
        p = d / f"r{m}.fq"
        write_fastq(p, rb, list(rows), m, m)
        plain.append(p)
    gz = []
    for k, p in enumerate(plain):
        data = p.read_bytes()
        blob = bgzf_ref.compress(data, 1 if k == 0 else 6)
        q = d / f"r{k + 1}.fq.gz"
        q.write_bytes(blob)
        gz.append(q)
    # R1 again with zero padding between members and a plain gzip member at the end
    import gzip

    data = plain[0].read_bytes()
    cut = len(data) // 2
    cut = data.index(b"\n@", cut) + 1
    mixed = d / "r1_mixed.fq.gz"
    mixed.write_bytes(bgzf_ref.compress(data[:cut], 1)[:-28] + b"\0" * 5 + gzip.compress(data[cut:]))
    return fa, prefix, plain, gz, mixed


@pytest.fixture(scope="module")
def gi(small_ref):
    fa, prefix = small_ref
    ctx = GpuContext(0)
    g = GpuIndex(ctx, prefix, kmer_k=12, kmer3_k=PARAMS.seed_len)
    yield ctx, g
    g.close()
    ctx.close()


@pytest.mark.parametrize("chunk", [300_000, 64 << 20])
def test_bam_from_device_inflated_bgzf(bgzf_reads, gi, tmp_path, chunk):
    fa, prefix, plain, gz, _ = bgzf_reads
    ctx, g = gi
    outs, stats = [], []
    for dev_inflate, fqs in ((False, plain), (True, gz)):
        out = tmp_path / f"o{int(dev_inflate)}.bam"
        st = {}
        map_fastq_to_bam(fa, fqs[0], out, fq2=fqs[1], bs_r1="C2T", bs_r2="G2A", params=PARAMS, environ={},
                         ctx=ctx, index=g, batch_pairs=3000, chunk_bytes=chunk, level=0, stats=st,
                         device_inflate=dev_inflate)
        outs.append(out.read_bytes())
        stats.append(st)
    assert outs[0] == outs[1]
    # each compressed member crossed once; the host reader copies the text
    assert stats[1]["fastq_h2d_bytes"] == sum(q.stat().st_size for q in gz)
    assert stats[0]["fastq_h2d_bytes"] >= sum(q.stat().st_size for q in plain)


def test_sam_from_device_inflated_bgzf(bgzf_reads, gi, tmp_path):
    fa, prefix, plain, gz, mixed = bgzf_reads
    ctx, g = gi
    outs = []
    for dev_inflate, fqs in ((False, plain), (True, gz), (True, [mixed, gz[1]])):
        out = tmp_path / f"s{len(outs)}.sam"
        map_fastq_to_sam(fa, fqs[0], out, fq2=fqs[1], bs_r1="C2T", bs_r2="G2A", params=PARAMS, environ={},
                         ctx=ctx, index=g, batch_pairs=2500, chunk_bytes=400_000, device_inflate=dev_inflate)
        outs.append(out.read_bytes())
    assert outs[0] == outs[1] == outs[2]
