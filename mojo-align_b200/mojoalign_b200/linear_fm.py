"""Function-level drop-in for map_fastq_fm_gpu (SAM output).

map_fastq_fm_gpu(ref_fa, fq1, out_sam, device, fq2, bs_r1, bs_r2) -> int
follows fq2bam-meth/src/linear_gpu_fm.mojo:1028-3341 on its SAM path:

- the index prefix is resolved like fm_prefix_from_ref
  (fq2bam-meth/src/linear_fm_index.mojo:350-358);
- FASTQ is split on the device under the rules of the SAM path's reader
  (fastq_batch.FastqPairReader), mapped on the GPU (conversion by bs_r1 /
  bs_r2 on the device), and the SAM lines are built on the device
  (mojoalign_b200.fq2sam.map_fastq_to_sam, ma_emit_sam_batch_device) as the
  reference writes them: _hit_from_fm (linear_gpu_fm.mojo:987-1025),
  pair_hits and hit_to_sam_line (fq2bam-meth/src/linear_extend.mojo:263-320),
  the RG tag of _sam_with_rg_fm (L80-81), after the header of
  _write_sam_header_fm (L40-76);
- the return value is the number of mapped records.

The per-record functions below (hit_from_fm, pair_hits, hit_to_sam_line,
reverse_complement) restate the reference's record rules for Python callers;
the drop-in's own SAM text comes from the device.

A .bam destination takes the reference's BAM path on the GPU end to end
(mojoalign_b200.fq2bam.map_fastq_to_bam): record packing, coordinate sort,
duplicate marking and BGZF.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, replace
from pathlib import Path

from .mapper import GpuContext, GpuIndex
from .params import FmParams

_RC_BYTES = bytes(ord({"A": "T", "T": "A", "C": "G", "G": "C"}.get(chr(c), "N")) for c in range(256))


def canonical_contig(name: str) -> str:
    """_canonical_contig (linear_gpu_locate.mojo:156-162): drop bwa-meth's f/r."""
    if len(name) >= 2 and name[0] in "fr":
        return name[1:]
    return name


def reverse_complement(seq: str) -> str:
    """utility.reverse_complement (methylgrapher/src/utility.mojo:28-49):
    byte-wise over the UTF-8 bytes, A<->T, C<->G, any other byte (lower case
    included) -> N."""
    return bytes(_RC_BYTES[c] for c in reversed(seq.encode("utf-8"))).decode("ascii")


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
    """_hit_from_fm, linear_gpu_fm.mojo:987-1025 (lengths in bytes)."""
    qlen = len(align_seq.encode("utf-8"))
    emit = original_seq if original_seq.encode("utf-8") else align_seq
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
        tlen = abs(b.pos - a.pos) + len(b.seq.encode("utf-8"))
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
    from .fq2sam import map_fastq_to_sam

    return map_fastq_to_sam(ref_fa, fq1, out_sam, device, fq2, bs_r1, bs_r2, params, env, kmer_k, kmer3_k, ctx, index)
