"""Shared fixtures.  `gpu` marks tests that need a B200 (run with -m gpu)."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "mojo-align_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def small_ref(tmp_path_factory):
    """A 300 kbp synthetic reference in 3 contigs and its bwa-meth index."""
    from mojoalign_b200 import build_index, synth

    d = tmp_path_factory.mktemp("small_ref")
    fa = d / "ref.fa"
    synth.write_reference(fa, 300_000, n_contigs=3, seed=0)
    prefix = Path(str(fa) + ".bwameth.c2t")
    build_index(fa, prefix, bwameth_c2t=True, sa_intv=32, device=-1)
    return fa, prefix


@pytest.fixture(scope="session")
def edgy_ref(tmp_path_factory):
    """Many short contigs (edge clips, contig crossings), bwa-meth index."""
    from mojoalign_b200 import build_index, synth

    d = tmp_path_factory.mktemp("edgy_ref")
    fa = d / "ref.fa"
    synth.write_reference(fa, 60_000, n_contigs=40, seed=3)
    prefix = Path(str(fa) + ".bwameth.c2t")
    build_index(fa, prefix, bwameth_c2t=True, sa_intv=16, device=-1)
    return fa, prefix


@pytest.fixture(scope="session")
def repeat_ref(tmp_path_factory):
    """A 3 Mbp repeat-heavy reference (the repeat-heavy configuration's
    model: 45% of the bases in copies of 300 bp / 6 kb family elements at
    10-20% divergence, 3% in tandem runs; 16 families per length class) and
    its bwa-meth index."""
    from mojoalign_b200 import build_index, synth

    d = tmp_path_factory.mktemp("repeat_ref")
    fa = d / "ref.fa"
    synth.write_reference_model(fa, 3_000_000, n_contigs=3, seed=4, repeats=synth.RepeatModel(families=16))
    prefix = Path(str(fa) + ".bwameth.c2t")
    build_index(fa, prefix, bwameth_c2t=True, sa_intv=32, device=-1)
    return fa, prefix


@pytest.fixture(scope="session")
def young_repeat_ref(tmp_path_factory):
    """A 2 Mbp reference where half the bases are copies of 4 families per
    class at 1-3% divergence (young repeats: seeds with hundreds of exact
    occurrences, the max_occ cap and the 16-row fallback on most reads)."""
    from mojoalign_b200 import build_index, synth

    d = tmp_path_factory.mktemp("young_repeat_ref")
    fa = d / "ref.fa"
    rm = synth.RepeatModel(repeat_frac=0.5, tandem_frac=0.03, families=4, div_min=0.01, div_max=0.03)
    synth.write_reference_model(fa, 2_000_000, n_contigs=2, seed=5, repeats=rm)
    prefix = Path(str(fa) + ".bwameth.c2t")
    build_index(fa, prefix, bwameth_c2t=True, sa_intv=32, device=-1)
    return fa, prefix
