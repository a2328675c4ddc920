"""The FASTQ -> sorted BAM path of map_fastq_fm_gpu restated on the CPU from
the oracle's pieces, for the end-to-end tests: oracle.fastq_parse (the
reference's reader), OracleIndex.map (the mapping kernels), oracle.emit_bam
(_emit_bam_from_batch), oracle.sort_markdup (gpu_sort_markdup),
oracle.gather_sorted (_gather_perm_to_writer) and oracle.bgzf_ref (the BGZF
writer), behind the header BamWriter writes."""
from __future__ import annotations

import gzip

import numpy as np

import oracle
from oracle import bgzf_ref

KEYS = ("name_off", "name_len", "seq_off", "seq_len", "qual_off", "qual_len")


def canonical(name: str) -> str:
    return name[1:] if len(name) >= 2 and name[0] in "fr" else name


def rid_to_tid(names) -> np.ndarray:
    seen, out = {}, []
    for n in names:
        c = canonical(n)
        seen.setdefault(c, len(seen))
        out.append(seen[c])
    return np.asarray(out, np.int32)


def read_fastq(path) -> bytes:
    path = str(path)
    opener = gzip.open if path.lower().endswith((".gz", ".gzip")) else open
    with opener(path, "rb") as fh:
        return fh.read()


def fq2bam(prefix, fq1, fq2, params, bs_r1: int, bs_r2: int, header: bytes, rg: bytes, level: int,
           markdup: bool = True) -> bytes:
    ix = oracle.OracleIndex(prefix)
    try:
        t1 = read_fastq(fq1)
        p1 = oracle.fastq_parse(t1)
        paired = fq2 is not None
        if paired:
            t2 = read_fastq(fq2)
            p2 = oracle.fastq_parse(t2, base=len(t1))
            if p2["n"] < p1["n"]:
                raise RuntimeError("paired FASTQ length mismatch (R2 ended early)")
            n1 = p1["n"]
            data = t1 + t2
            cols = {k: np.concatenate([p1[k], p2[k][:n1]]) for k in KEYS}
        else:
            n1 = p1["n"]
            data = t1
            cols = {k: p1[k] for k in KEYS}
        n_seq = n1 * (2 if paired else 1)
        max_len = max(int(cols["seq_len"].max()) if n_seq else 0, params[0])
        rows = np.full((n_seq, max_len), 78, np.uint8)
        buf = np.frombuffer(data, np.uint8)
        for i in range(n_seq):
            o, l = int(cols["seq_off"][i]), int(cols["seq_len"][i])
            rows[i, :l] = buf[o:o + l]
        hits = ix.map(rows, cols["seq_len"], n1, paired, max_len, bs_r1, bs_r2, params) if n_seq else None
        if not n_seq:
            return bgzf_ref.compress(header, level)
        arena = {"data": buf, "name_off": cols["name_off"], "name_len": cols["name_len"],
                 "orig_off": cols["seq_off"], "orig_len": cols["seq_len"], "qual_off": cols["qual_off"],
                 "qual_len": cols["qual_len"]}
        tids = rid_to_tid([c[0] for c in ix.contigs])
        cap = n_seq * (64 + len(rg)) + int(cols["name_len"].sum()) + 2 * int(cols["seq_len"].sum())
        bam, meta, _ = oracle.emit_bam(hits, arena, n1, paired, tids, rg, meta_cap=n_seq, cap=cap)
        is_dup, perm, _, _ = oracle.sort_markdup(meta["coord"], meta["dhi"], meta["dlo"], meta["score"],
                                                 meta["pair"], do_markdup=markdup, dup_perm=False)
        stream = oracle.gather_sorted([bam], perm, meta["rec"], meta["len"], is_dup, apply_dup=markdup)
        return bgzf_ref.compress(header + stream, level)
    finally:
        ix.close()
