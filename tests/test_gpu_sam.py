"""map_fastq_fm_gpu end to end: FASTQ in, SAM out, on the GPU.

The expected records are built from the oracle's outputs on the same reads
with the reference's emit rules (_hit_from_fm, pair_hits, hit_to_sam_line:
fq2bam-meth/src/linear_gpu_fm.mojo:987-1025, linear_extend.mojo:263-320).
Several FASTQ batches of different max lengths go through one call.
"""
from __future__ import annotations

import numpy as np
import pytest

import fq2sam_oracle
import oracle
from mojoalign_b200 import FmParams, synth
from mojoalign_b200.linear_fm import hit_from_fm, hit_to_sam_line, map_fastq_fm_gpu, pair_hits, sam_header

pytestmark = pytest.mark.gpu


def write_fastq(path, names, rows, mate):
    with open(path, "w") as fh:
        for nm, s in zip(names, rows):
            q = "".join(chr(33 + (i * 7 + len(s)) % 41) for i in range(len(s)))
            fh.write(f"@{nm}/{mate} comment\n{s}\n+\n{q}\n")


def expected_sam(prefix, names, rows1, rows2, params, contigs, rg="mojo1"):
    paired = rows2 is not None
    allrows = rows1 + (rows2 or [])
    max_len = max(max(len(s) for s in allrows), params.seed_len)
    bases = np.full((len(allrows), max_len), 78, dtype=np.uint8)
    for i, s in enumerate(allrows):
        bases[i, :len(s)] = np.frombuffer(s.encode(), dtype=np.uint8)
    lens = np.array([len(s) for s in allrows], dtype=np.uint32)
    n1 = len(rows1)
    o = oracle.OracleIndex(prefix).map(bases, lens, n1, paired, max_len, 1, 2, params.as_list())
    cn = [c.name for c in contigs]

    def hit(i, name, s):
        h = hit_from_fm(cn, name, s, s, int(o["rid"][i]), int(o["pos"][i]), int(o["mapq"][i]), int(o["flag"][i]),
                        int(o["sl"][i]), int(o["sr"][i]))
        h.qual = "".join(chr(33 + (k * 7 + len(s)) % 41) for k in range(len(s)))
        return h

    lines, mapped = [], 0
    for i in range(n1):
        h1 = hit(i, names[i], rows1[i])
        if not paired:
            lines.append(hit_to_sam_line(h1) + "\tRG:Z:" + rg)
            mapped += h1.contig != "*"
            continue
        p1, p2 = pair_hits(h1, hit(n1 + i, names[i], rows2[i]))
        mapped += (p1.contig != "*") + (p2.contig != "*")
        lines += [hit_to_sam_line(p1) + "\tRG:Z:" + rg, hit_to_sam_line(p2) + "\tRG:Z:" + rg]
    return lines, mapped


def reads(fa, n1, paired, seed):
    rb = synth.simulate_reads(fa, synth.ReadModel(len_fixed=0, len_max=180, random_frac=0.08), n1, paired, 180,
                              seed=seed)
    rows = [bytes(rb.bases[i, :rb.lens[i]]).decode() for i in range(rb.n_seq)]
    # lower-case and N bases reach the emit path (reverse_complement maps them to N)
    rows[3] = rows[3][:10].lower() + rows[3][10:]
    rows[5] = rows[5][:40] + "NN" + rows[5][42:]
    return rows


@pytest.mark.parametrize("paired", [True, False])
def test_map_fastq_fm_gpu_matches_oracle_records(small_ref, tmp_path, paired, monkeypatch):
    fa, prefix = small_ref
    n1 = 2500
    rows = reads(fa, n1, paired, seed=11 + paired)
    names = [f"read{i}" for i in range(n1)]
    fq1, fq2 = tmp_path / "r1.fq", tmp_path / "r2.fq"
    write_fastq(fq1, names, rows[:n1], 1)
    if paired:
        write_fastq(fq2, names, rows[n1:], 2)
    monkeypatch.setenv("METHYLGRAPHER_LINEAR_READ_BATCH", "700")  # 4 batches, the last one short
    monkeypatch.setenv("METHYLGRAPHER_RG_ID", "rgX")
    out = tmp_path / "out.sam"
    n_mapped = map_fastq_fm_gpu(fa, fq1, out, "auto", str(fq2) if paired else "", "C2T", "G2A")
    params = FmParams.from_env()
    from mojoalign_b200 import GpuContext, GpuIndex
    ctx = GpuContext(0)
    gi = GpuIndex(ctx, prefix, kmer_k=12)
    contigs = gi.contigs
    gi.close()
    ctx.close()
    exp, exp_mapped = expected_sam(prefix, names, rows[:n1], rows[n1:] if paired else None, params, contigs, "rgX")
    text = out.read_text().splitlines()
    hdr = sam_header(contigs, {"METHYLGRAPHER_RG_ID": "rgX"}).splitlines()
    assert text[:len(hdr)] == hdr
    body = text[len(hdr):]
    assert len(body) == len(exp)
    bad = [i for i, (a, b) in enumerate(zip(body, exp)) if a != b]
    assert not bad, f"{len(bad)} records differ; first:\n{body[bad[0]]}\n{exp[bad[0]]}"
    assert n_mapped == exp_mapped and 0 < n_mapped <= len(exp)


def messy_fastq(rows, names, mate, seed):
    """FASTQ text with mixed line ends (LF, CRLF, CR CR LF), names with
    comments and bytes >= 0x80, and a last record cut after its SEQ line."""
    rng = np.random.default_rng(seed)
    out = []
    for i, (nm, s) in enumerate(zip(names, rows)):
        eol = [b"\n", b"\r\n", b"\r\r\n"][int(rng.integers(0, 3))]
        q = bytes(33 + (k * 7 + len(s)) % 41 for k in range(len(s)))
        head = b"@" + nm.encode() + (b"\xe9" if i % 97 == 5 else b"") + b"/%d x" % mate
        out.append(head + eol + s.encode() + eol + b"+" + eol + q + eol)
    out.append(b"@cut/%d\n" % mate + rows[0][:30].encode() + b"\n")
    return b"".join(out)


@pytest.mark.parametrize("paired", [True, False])
def test_sam_path_on_messy_fastq_in_small_chunks(small_ref, tmp_path, paired):
    from mojoalign_b200 import GpuContext, GpuIndex
    from mojoalign_b200.fq2sam import map_fastq_to_sam

    fa, prefix = small_ref
    n1 = 1800
    rows = reads(fa, n1, paired, seed=21 + paired)
    names = [f"m{i}" for i in range(n1)]
    t1 = messy_fastq(rows[:n1], names, 1, 5)
    t2 = messy_fastq(rows[n1:], names, 2, 6) if paired else None
    fq1, fq2 = tmp_path / "m1.fq", tmp_path / "m2.fq"
    fq1.write_bytes(t1)
    if paired:
        fq2.write_bytes(t2)
    params = FmParams.from_env({})
    ctx = GpuContext(0)
    gi = GpuIndex(ctx, prefix, kmer_k=12)
    try:
        out = tmp_path / "m.sam"
        stats = {}
        n_mapped = map_fastq_to_sam(fa, fq1, out, "auto", str(fq2) if paired else "", "C2T", "G2A", params, {},
                                    ctx=ctx, index=gi, batch_pairs=700, chunk_bytes=64 << 10, stats=stats)
        want, want_mapped = fq2sam_oracle.fq2sam(prefix, None, None, params.as_list(), 1, 2,
                                                 [c.name for c in gi.contigs], b"mojo1", texts=(t1, t2))
        hdr = sam_header(gi.contigs, {}).encode()
    finally:
        gi.close()
        ctx.close()
    got = out.read_bytes()
    assert got[:len(hdr)] == hdr
    body = got[len(hdr):]
    if body != want:
        a, b = body.split(b"\n"), want.split(b"\n")
        bad = [i for i, (x, y) in enumerate(zip(a, b)) if x != y]
        raise AssertionError(f"{len(a)} vs {len(b)} lines, {len(bad)} differ; first:\n{a[bad[0]] if bad else ''}\n"
                             f"{b[bad[0]] if bad else ''}")
    assert n_mapped == want_mapped
    assert b"\xef\xbf\xbd" in body  # a name byte >= 0x80 became U+FFFD


def test_sam_path_r2_ending_early_fails(small_ref, tmp_path):
    fa, _ = small_ref
    rows = reads(fa, 50, True, seed=3)
    names = [f"e{i}" for i in range(50)]
    (tmp_path / "a1.fq").write_bytes(messy_fastq(rows[:50], names, 1, 1))
    (tmp_path / "a2.fq").write_bytes(messy_fastq(rows[50:90], names[:40], 2, 2))
    with pytest.raises(RuntimeError, match="R2 ended early"):
        map_fastq_fm_gpu(fa, tmp_path / "a1.fq", tmp_path / "a.sam", "auto", str(tmp_path / "a2.fq"), "C2T", "G2A")
