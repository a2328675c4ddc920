"""Function-level drop-in for map_fastq_fm_gpu (SAM output).

map_fastq_fm_gpu(ref_fa, fq1, out_sam, device, fq2, bs_r1, bs_r2) -> int
follows fq2bam-meth/src/linear_gpu_fm.mojo:1028-3341 on its SAM path:

- the index prefix is resolved like fm_prefix_from_ref
  (fq2bam-meth/src/linear_fm_index.mojo:350-358);
- FASTQ batches of METHYLGRAPHER_LINEAR_READ_BATCH pairs are mapped on the
  GPU (conversion by bs_r1 / bs_r2 on the device);
- records are written as the reference writes them: _hit_from_fm
  (linear_gpu_fm.mojo:987-1025), pair_hits and hit_to_sam_line
  (fq2bam-meth/src/linear_extend.mojo:263-320), the RG tag of
  _sam_with_rg_fm (L80-81) and the header of _write_sam_header_fm (L40-76);
- the return value is the number of mapped records.

A .bam destination takes the reference's BAM path on the GPU end to end
(mojoalign_b200.fq2bam.map_fastq_to_bam): record packing, coordinate sort,
duplicate marking and BGZF.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, replace
from pathlib import Path

from .fastq import FastqPairStream, pack_bases
from .mapper import GpuContext, GpuIndex, map_batch
from .params import READ_BATCH_ENV, FmParams, env_int

_RC = bytes.maketrans(b"ACGT", b"TGCA")


def canonical_contig(name: str) -> str:
    """_canonical_contig (linear_gpu_locate.mojo:156-162): drop bwa-meth's f/r."""
    if len(name) >= 2 and name[0] in "fr":
        return name[1:]
    return name


def reverse_complement(seq: str) -> str:
    """utility.reverse_complement (methylgrapher/src/utility.mojo:28-49):
    A<->T, C<->G, any other byte (lower case included) -> N."""
    b = seq.encode("ascii", "replace")
    out = bytearray(b.translate(_RC)[::-1])
    src = b[::-1]
    for i, ch in enumerate(src):
        if ch not in b"ACGT":
            out[i] = ord("N")
    return out.decode("ascii")


@dataclass
class LinearHit:
    """linear_extend.mojo:11-48."""
    query_name: str
    flag: int
    contig: str
    pos: int  # 1-based
    mapq: int
    cigar: str
    seq: str
    qual: str = "*"
    rnext: str = "*"
    pnext: int = 0
    tlen: int = 0


def hit_from_fm(contig_names, name: str, align_seq: str, original_seq: str, rid: int, start0: int, mapq: int,
                flag: int, soft_l: int, soft_r: int) -> LinearHit:
    """_hit_from_fm, linear_gpu_fm.mojo:987-1025."""
    qlen = len(align_seq)
    emit = original_seq if original_seq else align_seq
    if rid < 0:
        return LinearHit(name, 4, "*", 0, 0, "*", emit, "*")
    m = qlen - soft_l - soft_r
    if m < 1:
        return LinearHit(name, 4, "*", 0, 0, "*", emit, "*")
    cigar = (f"{soft_l}S" if soft_l > 0 else "") + f"{m}M" + (f"{soft_r}S" if soft_r > 0 else "")
    if flag & 16:
        emit = reverse_complement(emit)
    return LinearHit(name, flag, canonical_contig(contig_names[rid]), start0 + 1, mapq, cigar, emit, "*")


def pair_hits(h1: LinearHit, h2: LinearHit) -> tuple[LinearHit, LinearHit]:
    """pair_hits, linear_extend.mojo:263-294."""
    a = replace(h1, flag=h1.flag | 1 | 64)
    b = replace(h2, flag=h2.flag | 1 | 128)
    if a.contig != "*" and b.contig != "*" and a.contig == b.contig:
        a.flag |= 2
        b.flag |= 2
        a.rnext = b.rnext = "="
        a.pnext = b.pos
        b.pnext = a.pos
        tlen = abs(b.pos - a.pos) + len(b.seq)
        a.tlen = tlen
        b.tlen = -tlen
    else:
        if a.contig == "*":
            b.flag |= 8
        if b.contig == "*":
            a.flag |= 8
        if a.contig != "*":
            b.rnext = a.contig
            b.pnext = a.pos
        if b.contig != "*":
            a.rnext = b.contig
            a.pnext = b.pos
    return a, b


def hit_to_sam_line(h: LinearHit) -> str:
    """hit_to_sam_line, linear_extend.mojo:297-320."""
    return "\t".join([h.query_name, str(h.flag), h.contig, str(h.pos), str(h.mapq), h.cigar, h.rnext, str(h.pnext),
                      str(h.tlen), h.seq, h.qual])


def _env_str(name: str, default: str, environ) -> str:
    v = environ.get(name, default)
    return v if v else default


def sam_header(contigs, environ=None) -> str:
    """_write_sam_header_fm, linear_gpu_fm.mojo:40-76."""
    env = os.environ if environ is None else environ
    lines = ["@HD\tVN:1.6\tSO:unsorted"]
    seen = set()
    for c in contigs:
        canon = canonical_contig(c.name)
        if canon not in seen:
            seen.add(canon)
            lines.append(f"@SQ\tSN:{canon}\tLN:{c.length}")
    rg = _env_str("METHYLGRAPHER_RG_ID", "mojo1", env)
    sm = _env_str("METHYLGRAPHER_RG_SM", "sample", env)
    lb = _env_str("METHYLGRAPHER_RG_LB", "lib1", env)
    pl = _env_str("METHYLGRAPHER_RG_PL", "ILLUMINA", env)
    lines.append(f"@RG\tID:{rg}\tSM:{sm}\tLB:{lb}\tPL:{pl}\tPU:{rg}")
    lines.append("@PG\tID:MojoFq2bamMeth\tPN:MojoFq2bamMeth\tVN:0.1.0-mojo-fm")
    return "\n".join(lines) + "\n"


def fm_prefix_from_ref(ref_fa) -> str:
    """fm_prefix_from_ref, linear_fm_index.mojo:350-358."""
    ref_fa = str(ref_fa)
    if Path(ref_fa + ".bwt").is_file():
        return ref_fa
    bw = ref_fa + ".bwameth.c2t"
    if Path(bw + ".bwt").is_file():
        return bw
    raise RuntimeError("No BWA FM-index (.bwt) beside " + ref_fa)


def select_device(device: str) -> int:
    """The FM engine needs an NVIDIA device here ("auto" / "nvidia" / an
    ordinal); "cpu" and "amd" fail closed like the reference's
    `map_fastq_fm_gpu needs DeviceContext cuda/hip` (L1053-1062)."""
    d = (device or "auto").lower()
    if d in ("auto", "nvidia", "gpu", "cuda"):
        return 0
    if d.isdigit():
        return int(d)
    raise RuntimeError(f"MojoLinear GPU-fm needs an NVIDIA device, got {device!r}")


def map_fastq_fm_gpu(ref_fa, fq1, out_sam, device: str = "auto", fq2: str = "", bs_r1: str = "", bs_r2: str = "",
                     params: FmParams | None = None, environ=None, kmer_k: int = 12, kmer3_k: int | None = None,
                     ctx: GpuContext | None = None, index: GpuIndex | None = None) -> int:
    env = os.environ if environ is None else environ
    if str(out_sam).lower().endswith(".bam"):  # _path_is_bam, linear_gpu_fm.mojo:84-88
        from .fq2bam import map_fastq_to_bam

        return map_fastq_to_bam(ref_fa, fq1, out_sam, device, fq2, bs_r1, bs_r2, params, env, kmer_k, kmer3_k,
                                ctx, index)
    params = params or FmParams.from_env(env)
    batch = env_int(READ_BATCH_ENV[0], READ_BATCH_ENV[1], env)
    own_ctx = ctx is None
    ctx = ctx or GpuContext(select_device(device))
    own_index = index is None
    if index is None:
        k3 = min(params.seed_len, 18) if kmer3_k is None else kmer3_k
        index = GpuIndex(ctx, fm_prefix_from_ref(ref_fa), kmer_k=min(kmer_k, params.seed_len), kmer3_k=k3)
    paired = len(str(fq2)) > 0
    names = [c.name for c in index.contigs]
    rg = _env_str("METHYLGRAPHER_RG_ID", "mojo1", env)
    n_mapped = 0
    try:
        with open(out_sam, "w") as fh, FastqPairStream(str(fq1), str(fq2), "", "") as stream:
            fh.write(sam_header(index.contigs, env))
            while True:
                a = stream.read_batch(batch)
                if a.n1 == 0:
                    break
                max_len = max(a.max_len, params.seed_len)
                if max_len > 1024:
                    raise RuntimeError("read longer than FM base cap (1024)")
                bases, lens = pack_bases(a, paired, max_len, converted=False)
                r = map_batch(ctx, index, bases, lens, a.n1, paired, max_len, bs_r1, bs_r2, params)
                out = []
                for i in range(a.n1):
                    h1 = hit_from_fm(names, a.name1[i].decode(), a.seq1[i].decode(), a.orig1[i].decode(),
                                     int(r.rid[i]), int(r.pos[i]), int(r.mapq[i]), int(r.flag[i]), int(r.sl[i]),
                                     int(r.sr[i]))
                    h1.qual = a.qual1[i].decode()
                    if not paired:
                        n_mapped += h1.contig != "*"
                        out.append(hit_to_sam_line(h1) + "\tRG:Z:" + rg)
                        continue
                    j = a.n1 + i
                    h2 = hit_from_fm(names, a.name2[i].decode(), a.seq2[i].decode(), a.orig2[i].decode(),
                                     int(r.rid[j]), int(r.pos[j]), int(r.mapq[j]), int(r.flag[j]), int(r.sl[j]),
                                     int(r.sr[j]))
                    h2.qual = a.qual2[i].decode()
                    p1, p2 = pair_hits(h1, h2)
                    n_mapped += (p1.contig != "*") + (p2.contig != "*")
                    out.append(hit_to_sam_line(p1) + "\tRG:Z:" + rg)
                    out.append(hit_to_sam_line(p2) + "\tRG:Z:" + rg)
                fh.write("\n".join(out) + "\n")
    finally:
        if own_index:
            index.close()
        if own_ctx:
            ctx.close()
    return n_mapped
