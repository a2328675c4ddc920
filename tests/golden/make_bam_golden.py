"""Regenerates tests/golden/bam_records.json from the reference.

Run from the repository root where the mojo-align source tree is available
(its path is the one required argument).  The reference's Python BAM writer,
fq2bam-meth/python/bam_emit.py (BamWriter.write_batch, L358-475), is
imported and run on seeded random alignments; its BGZF layer is replaced by
a byte sink so the raw records can be kept.  The records it packs follow
the same BAM layout as the Mojo packer _pack_bam_aln
(fq2bam-meth/src/linear_gpu_fm.mojo:497-666) on the inputs drawn here:
bases from ACGTN in both cases (the two differ on IUPAC codes), positions
below 2^29 (the BAM binning range; BamWriter rejects larger bins), qualities
'!'..'~' (they differ below '!'), and clips handed to BamWriter in the
stored-strand orientation, since _pack_bam_aln swaps them itself on the
reverse strand (L531-534).  The fixture stores the clips as _pack_bam_aln
receives them.  Also records the reference's own unit vectors
(tests/test_bam_emit.py:15-17) and the uncompressed header BamWriter writes
for a two-contig reference with the default read group (BamWriter.__init__,
L312-356, as _open_bam_writer calls it, linear_gpu_fm.mojo:91-125).
"""
from __future__ import annotations

import importlib.util
import json
import random
import sys
from pathlib import Path

OUT = Path(__file__).resolve().parent / "bam_records.json"
RG = "mojo1"


def load_bam_emit(root: Path):
    path = root / "fq2bam-meth" / "python" / "bam_emit.py"
    spec = importlib.util.spec_from_file_location("bam_emit_reference", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class Sink:
    def __init__(self, *_a, **_k):
        self.parts = []

    def write(self, data):
        self.parts.append(bytes(data))

    def close(self):
        pass


def draw(rng: random.Random, i: int) -> dict:
    qlen = rng.choice([0, 1, 2, 3, 17, 50, 75, 100, 101, 150, 151, 250, 301])
    seq = "".join(rng.choice("ACGTNacgtn" if rng.random() < 0.2 else "ACGT") for _ in range(qlen))
    kind = rng.random()
    if kind < 0.1:
        qual = None
    elif kind < 0.2:
        qual = "".join(chr(rng.randint(33, 126)) for _ in range(max(0, qlen + rng.choice([-1, 1, 3]))))
    else:
        qual = "".join(chr(rng.randint(33, 126)) for _ in range(qlen))
    name_n = rng.choice([1, 5, 12, 30, 48, 80]) if i % 37 else rng.choice([254, 255, 300])
    name = "".join(rng.choice("ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789:_-") for _ in range(name_n))
    flag = rng.choice([0, 16]) | rng.choice([0, 0, 0, 4]) | rng.choice([1, 0]) | rng.choice([64, 128, 0]) | \
        rng.choice([0, 2]) | rng.choice([0, 8])
    tid = rng.choice([-1, 0, 0, 1, 2, 7])
    big = rng.random() < 0.3
    pos = rng.choice([0, 1, 16383, 16384, 131071, (1 << 20) - 3, (1 << 23) - 5, (1 << 26) - 7]) if big else \
        rng.randint(0, (1 << 29) - 1 - 1000)
    sl = rng.choice([0, 0, 0, 1, 5, 20, qlen, qlen + 3])
    sr = rng.choice([0, 0, 0, 2, 7, 19, qlen // 2])
    return {
        "name": name, "flag": flag, "tid": tid, "pos": pos, "mapq": rng.choice([0, 1, 37, 60, 255, 256, 999]),
        "sl": sl, "sr": sr, "seq": seq, "qual": qual, "ntid": rng.choice([-1, -2, 0, 1, 3]),
        "npos": rng.randint(-1, (1 << 31) - 1), "tlen": rng.randint(-(1 << 31), (1 << 31) - 1),
        "nm": rng.choice([0, 1, 2, 12, 255, 256, 1000]),
    }


def main(root: Path) -> None:
    mod = load_bam_emit(root)
    mod._BgzfWriter = Sink
    rng = random.Random(20240611)
    recs = [draw(rng, i) for i in range(400)]
    w = mod.BamWriter("unused.bam", ["chr1", "chr2"], [1000, 2000], rg_id=RG, level=1, sort_order="coordinate")
    header_parts = len(w._bgzf.parts)
    for r in recs:
        rev = bool(r["flag"] & 16)
        # BamWriter takes the clips of the stored strand
        sl, sr = (r["sr"], r["sl"]) if rev else (r["sl"], r["sr"])
        w.write_batch(qnames=[r["name"]], flags=[r["flag"]], tids=[r["tid"]], pos0s=[r["pos"]], mapqs=[r["mapq"]],
                      sls=[sl], srs=[sr], seqs=[r["seq"]], quals=[r["qual"] if r["qual"] is not None else ""],
                      next_tids=[r["ntid"]], next_pos0s=[r["npos"]], tlens=[r["tlen"]], nms=[r["nm"]])
    body = w._bgzf.parts[header_parts:]
    assert len(body) == len(recs)
    for r, b in zip(recs, body):
        r["expect"] = b.hex()
    unit = {
        "pack_seq_ACGT": mod._pack_seq(b"ACGT").hex(),
        "reg2bin": [[b, e, mod._reg2bin(b, e)] for b, e in
                    [(0, 1), (0, 0), (16383, 16385), (100, 200), (1 << 17, (1 << 17) + 5), (0, 1 << 20),
                     (5, (1 << 23) + 1), (1 << 26, (1 << 26) + 1), (0, 1 << 29)]],
    }
    header = b"".join(w._bgzf.parts[:header_parts])
    OUT.write_text(json.dumps({"rg": RG, "unit": unit, "header": {"sq_names": ["chr1", "chr2"], "sq_lens": [1000, 2000],
                                                               "blob": header.hex()},
                               "records": recs}, indent=0) + "\n")
    print(f"wrote {OUT} ({len(recs)} records)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <mojo-align source tree>")
    main(Path(sys.argv[1]))
