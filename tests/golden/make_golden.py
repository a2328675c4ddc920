"""Regenerates tests/golden/conversion_vectors.json from the reference.

Run from the repository root in an environment where the mojo-align source
tree is available (its path is the one required argument).  The reference's
orchestrator module fq2bam-meth/python/fq2bam_meth.py is plain Python and is
imported and executed to produce its conversion outputs.  The Mojo FASTQ
path (fq2bam-meth/src/linear_fastq.mojo) cannot run without the Mojo
toolchain; its expected values are the ones asserted by the reference's own
test, fq2bam-meth/tests/test_linear_fastq.mojo:30-85, restated here.
"""
from __future__ import annotations

import importlib.util
import json
import sys
import tempfile
from pathlib import Path

OUT = Path(__file__).resolve().parent / "conversion_vectors.json"


def load_reference(root: Path):
    path = root / "fq2bam-meth" / "python" / "fq2bam_meth.py"
    spec = importlib.util.spec_from_file_location("fq2bam_meth_reference", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


SEQS = [
    "ACGT",  # test_fq2bam_meth.py:33-42
    "ACGTACGT", "GGTAGGTA", "CCCC", "GGGG",  # test_linear_fastq.mojo:31-34
    "ACGTNacgtn", "NNNN", "cCgGaAtT", "ACGTRYKMSWBDHVN.-",
    "TTTTTTTTTTTTTTTTTTTTTTTTTTTTTTTT", "",
]


def main(root: Path) -> None:
    ref = load_reference(root)
    vectors = {"convert_fastq": [], "convert_fasta_c2t": [], "convert_base": [], "linear_fastq_mojo": {}}
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        for i, s in enumerate(SEQS):
            src = td / f"r{i}.fq"
            src.write_text(f"@r{i}\n{s}\n+\n{'I' * len(s)}\n")
            row = {"seq": s}
            for mode in ("C2T", "G2A"):
                dst = td / f"r{i}.{mode}.fq"
                ref.convert_fastq(src, dst, mode)
                row[mode] = dst.read_text().splitlines()[1]
            vectors["convert_fastq"].append(row)
        for s in ("ACGTCacgt", "NNNNcccc", "ACGT\nacgt"):
            src = td / "in.fa"
            dst = td / "out.fa"
            src.write_text(">chr1\n" + s + "\n")
            ref.convert_fasta_c2t(src, dst)
            vectors["convert_fasta_c2t"].append({"body": s, "out": dst.read_text().split("\n", 1)[1]})
    for ch in "ACGTNacgtnRY":
        vectors["convert_base"].append(
            {"base": ch, "C2T": ref._convert_base(ch, "C2T"), "G2A": ref._convert_base(ch, "G2A")}
        )
    # test_linear_fastq.mojo:31-85 (R1 C2T, R2 G2A, pack stride 8)
    vectors["linear_fastq_mojo"] = {
        "r1": "@read1 extra/1\nACGTACGT\n+\nIIIIIIII\n@read2\nCCCC\n+\nJJJJ\n",
        "r2": "@read1 extra/2\nGGTAGGTA\n+\nKKKKKKKK\n@read2\nGGGG\n+\nLLLL\n",
        "n1": 2,
        "max_len": 8,
        "name1_0": "read1",
        "orig1_0_byte1": 67,
        "seq1_0_byte1": 84,
        "orig2_0_byte0": 71,
        "seq2_0_byte0": 65,
        "seq1_1_byte0": 84,
        "seq1_1_len": 4,
        "packed_len0": 8,
        "packed_byte1": 84,
        "packed_byte12": 78,
        "packed_byte16": 65,
    }
    OUT.write_text(json.dumps(vectors, indent=1) + "\n")
    print(f"wrote {OUT}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <mojo-align source tree>")
    main(Path(sys.argv[1]))
