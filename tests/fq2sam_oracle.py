"""The FASTQ -> SAM path of map_fastq_fm_gpu restated on the CPU from the
oracle's pieces, for the end-to-end tests and the bench's CPU baseline:
oracle.fastq_parse_pr (the SAM path's FastqPairReader), OracleIndex.map (the
mapping kernels) and oracle.emit_sam (_hit_from_fm, pair_hits,
hit_to_sam_line, _sam_with_rg_fm).  Returns the SAM body (no header)."""
from __future__ import annotations

import numpy as np

import oracle
from fq2bam_oracle import read_fastq


def fq2sam(prefix, fq1, fq2, params, bs_r1: int, bs_r2: int, contig_names, rg: bytes, texts=None):
    """`params`: FmParams.as_list(); `texts`: the FASTQ bytes when already in
    memory.  Returns (SAM body bytes, mapped records)."""
    t1 = texts[0] if texts else read_fastq(fq1)
    paired = fq2 is not None or (texts is not None and texts[1] is not None)
    t2 = (texts[1] if texts else read_fastq(fq2)) if paired else None
    p1 = oracle.fastq_parse_pr(t1)
    n1 = p1["n"]
    parts = [(p1, 0)]
    if paired:
        p2 = oracle.fastq_parse_pr(t2)
        if p2["n"] < n1:
            raise RuntimeError("paired FASTQ length mismatch (R2 ended early)")
        parts.append((p2, len(t1)))
    data = t1 + (t2 or b"")
    cols = {k: np.concatenate([p[k][:n1] + (b if k.endswith("off") else 0) for p, b in parts]).astype(
        np.uint64 if k.endswith("off") else np.uint32) for k in oracle.REC_KEYS}
    n_seq = int(cols["seq_len"].size)
    if n_seq == 0:
        return b"", 0
    max_len = max(int(cols["seq_len"].max()), params[0])
    bases = np.full((n_seq, max_len), 78, dtype=np.uint8)
    for i in range(n_seq):
        o, ln = int(cols["seq_off"][i]), int(cols["seq_len"][i])
        bases[i, :ln] = np.frombuffer(data[o:o + ln], np.uint8)
    ix = oracle.OracleIndex(prefix)
    try:
        o = ix.map(bases, cols["seq_len"].copy(), n1, paired, max_len, bs_r1, bs_r2, params)
    finally:
        ix.close()
    arena = dict(cols, data=np.frombuffer(data, np.uint8))
    return oracle.emit_sam({k: o[k] for k in ("rid", "pos", "mapq", "flag", "sl", "sr")}, n1, paired, arena,
                           contig_names, rg)
