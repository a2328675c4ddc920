"""The GPU index builder against the host builder, byte for byte.

`bwa index` (third-party, absent) builds the reference's index files; this
library's builder writes the same bwa 0.7 layout.  The host builder is pinned
against brute-force suffix arrays in test_index_builder.py; here the GPU
construction (suffixes sorted in bucket batches, ties refined 31 symbols at
a time) must write identical .bwt / .sa / .pac / .ann / .amb files, with
small batch limits so that many batches run, on texts with long runs and
repeat copies (deep refinements).
"""
from __future__ import annotations

import numpy as np
import pytest

from mojoalign_b200 import build_index, synth

pytestmark = pytest.mark.gpu

EXTS = (".bwt", ".sa", ".pac", ".ann", ".amb")


def _same_files(a, b):
    for ext in EXTS:
        x = open(str(a) + ext, "rb").read()
        y = open(str(b) + ext, "rb").read()
        assert x == y, f"{ext} differs ({len(x)} vs {len(y)} bytes)"


def _both(fa, tmp_path, batch, c2t=True, sa_intv=32):
    cpu, gpu = tmp_path / "cpu", tmp_path / "gpu"
    build_index(fa, cpu, bwameth_c2t=c2t, sa_intv=sa_intv, device=-1)
    build_index(fa, gpu, bwameth_c2t=c2t, sa_intv=sa_intv, device=0, batch_suffixes=batch)
    _same_files(cpu, gpu)


@pytest.mark.parametrize("sa_intv", [1, 4, 32])
def test_small_texts(tmp_path, sa_intv):
    rng = np.random.default_rng(sa_intv)
    cases = [
        [("chr1", "ACGTACGTTTGACCA")],
        [("c1", "A" * 36), ("c2", "AC" * 9)],
        [("x", "GATTACA" * 9), ("y", "T"), ("z", "CCGGN" * 7)],
        [(f"r{i}", "".join(rng.choice(list("ACGT"), size=int(rng.integers(50, 300))))) for i in range(4)],
    ]
    for i, contigs in enumerate(cases):
        fa = tmp_path / f"c{i}.fa"
        fa.write_text("".join(f">{n} d\n{s}\n" for n, s in contigs))
        d = tmp_path / f"d{i}"
        d.mkdir()
        for batch in (0, 300):
            _both(fa, d, batch, sa_intv=sa_intv)
        _both(fa, d, 0, c2t=False, sa_intv=sa_intv)


def test_random_reference_many_batches(small_ref, tmp_path):
    fa, _ = small_ref
    _both(fa, tmp_path, 20_000)


def test_repeat_references(repeat_ref, young_repeat_ref, tmp_path):
    for k, (fa, _) in enumerate((repeat_ref, young_repeat_ref)):
        d = tmp_path / f"r{k}"
        d.mkdir()
        _both(fa, d, 400_000)


def test_tandem_heavy_text(tmp_path):
    """Long tandem runs tie suffixes for hundreds of symbols."""
    fa = tmp_path / "t.fa"
    rm = synth.RepeatModel(repeat_frac=0.0, tandem_frac=0.6, families=1, unit_min=1, unit_max=3, run_min=500,
                           run_max=3000)
    synth.write_reference_model(fa, 200_000, n_contigs=2, seed=2, repeats=rm)
    _both(fa, tmp_path, 100_000)
