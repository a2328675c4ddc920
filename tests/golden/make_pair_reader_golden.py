"""Regenerates tests/golden/fastq_pair_reader.json from the reference.

Run from the repository root where the mojo-align source tree is available
(its path is the one required argument).  The reference's FASTQ reader of the
SAM path, fq2bam-meth/python/fastq_batch.py (FastqPairReader, L230-325, and
_qname, L18-28), is imported and run over hand-made FASTQ texts: line-ending
variants, records cut short at the end, blank lines, names with and without
'@', ' ' and '/', bytes >= 0x80 in names, and seeded random files.  For each
text the fixture keeps every record the reader returns (name as the UTF-8
of the str it builds, original bases, converted bases and qualities as hex)
and, for the paired cases, the error the reader raises when R2 ends first.
"""
from __future__ import annotations

import importlib.util
import json
import random
import sys
import tempfile
from pathlib import Path

OUT = Path(__file__).resolve().parent / "fastq_pair_reader.json"


def load_reader(root: Path):
    path = root / "fq2bam-meth" / "python" / "fastq_batch.py"
    spec = importlib.util.spec_from_file_location("fastq_batch_reference", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


HAND = [
    b"",
    b"\n",
    b"\n\n\n\n\n",
    b"@r1/1 comment\nACGT\n+\nIIII\n",
    b"@r1\r\nACGT\r\n+\r\nIIII\r\n@r2 x/y\r\nGGCC\r\n+\r\nJJJJ",
    b"@a\r\r\nAC\r\r\n+\r\r\nII\r\r\n@b\nT\r\n+\n\r\n",
    b"@a\nAC\n+\nII\n@b",
    b"@a\nAC\n+\nII\n@b\n",
    b"@a\nAC\n+\nII\n@b\nGG",
    b"@a\nAC\n+\nII\n@b\nGG\n+",
    b"@a\nAC\n+\nII\n@b\nGG\n+\n",
    b"@a\nAC\n+\nII\n@b\nGG\n+\nJ",
    b"@a\nAC\n+\nII\n\n@b\nGG\n+\nJJ\n",
    b"@a\nAC\n+\nII\n\n\n",
    b"noat name\nACGT\n+\nIIII\n",
    b"@x/y z\nA\n+\nI\n@x y/z\nA\n+\nI\n@/\nA\n+\nI\n@ \nA\n+\nI\n@@d\nA\n+\nI\n",
    b"@\xc3\xa9t\xff/1\nACGT\n+\nIIII\n",
    b"@r\tt\nAC\tG\n+\nI\x01I\n",
    b"\r\n\r\n\r\n\r",
    b"@q\nacgtnACGTN\n+\n!!!!!!!!!!\n",
    b"@only header",
    b"@r\nACGT\n+\nIIII\n\r",
]


def random_text(seed: int, n: int) -> bytes:
    rng = random.Random(seed)
    out = []
    for i in range(n):
        eol = rng.choice([b"\n", b"\n", b"\r\n", b"\r\r\n"])
        name = "".join(rng.choice("ABCxyz0123:_-") for _ in range(rng.randint(0, 12))).encode()
        if rng.random() < 0.3:
            name += rng.choice([b"/1", b"/2", b" comment", b" a/b", b"/3 c"])
        L = rng.choice([0, 1, 36, 100, 150, 151])
        seq = bytes(rng.choice(b"ACGTNacgt") for _ in range(L))
        qual = bytes(rng.randint(33, 126) for _ in range(L))
        out.append((b"@" if rng.random() < 0.95 else b"") + name + eol + seq + eol + b"+" + eol + qual + eol)
    text = b"".join(out)
    cut = rng.choice([0, 0, 1, 2, 5])
    return text[:len(text) - cut] if cut else text


def run(mod, tmp: Path, t1: bytes, t2: bytes | None, bs_r1: str, bs_r2: str, batch: int) -> dict:
    f1 = tmp / "r1.fq"
    f1.write_bytes(t1)
    f2 = ""
    if t2 is not None:
        (tmp / "r2.fq").write_bytes(t2)
        f2 = str(tmp / "r2.fq")
    r = mod.FastqPairReader(str(f1), f2, bs_r1, bs_r2)
    recs = {"1": [], "2": []}
    err = None
    try:
        while True:
            b = r.read_batch(batch)
            if b.n1 == 0:
                break
            for m in ("1", "2"):
                names = getattr(b, "names" + m)
                for i in range(len(names)):
                    recs[m].append([names[i].encode("utf-8").hex(), bytes(getattr(b, "orig" + m)[i]).hex(),
                                    bytes(getattr(b, "seq" + m)[i]).hex(), bytes(getattr(b, "qual" + m)[i]).hex()])
    except RuntimeError as e:
        err = str(e)
    finally:
        r.close()
    return {"r1": t1.hex(), "r2": None if t2 is None else t2.hex(), "bs_r1": bs_r1, "bs_r2": bs_r2, "batch": batch,
            "records1": recs["1"], "records2": recs["2"], "error": err}


def main(root: Path) -> None:
    mod = load_reader(root)
    cases = []
    with tempfile.TemporaryDirectory() as d:
        tmp = Path(d)
        for t in HAND:
            cases.append(run(mod, tmp, t, None, "C2T", "", 1000))
        for seed in range(6):
            cases.append(run(mod, tmp, random_text(seed, 60), None, "G2A" if seed % 2 else "C2T", "", 7 + seed))
        # paired: equal files, R2 longer (extra records ignored), R2 shorter (error)
        a, b = random_text(10, 30), random_text(11, 30)
        cases.append(run(mod, tmp, a, b, "C2T", "G2A", 16))
        cases.append(run(mod, tmp, random_text(12, 25), random_text(13, 28), "C2T", "G2A", 1000))
        cases.append(run(mod, tmp, random_text(14, 28), random_text(15, 25), "C2T", "G2A", 1000))
    OUT.write_text(json.dumps({"cases": cases}, indent=0) + "\n")
    print(f"wrote {OUT} ({len(cases)} cases)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <mojo-align source tree>")
    main(Path(sys.argv[1]))
