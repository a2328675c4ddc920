"""Seeded synthetic references and bisulfite reads (benchmarks and tests)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import check, fspath, lib, ma_read_model, ma_repeat_model, ptr


def write_reference(path, total_len: int, n_contigs: int = 1, gc: float = 0.41, cpg: float = 0.01,
                    seed: int = 0) -> None:
    """FASTA from a first-order base model (GC fraction gc, CpG rate cpg)."""
    check(lib.ma_synth_reference(fspath(path), total_len, n_contigs, gc, cpg, seed))


@dataclass
class RepeatModel:
    """Repeat content of a synthetic reference.  The defaults are the
    repeat-heavy configuration: 45% of the bases in copies of 300 bp and
    6 kb family elements at 10-20% divergence, 3% in low-complexity tandem
    runs."""
    repeat_frac: float = 0.45
    tandem_frac: float = 0.03
    families: int = 64
    short_len: int = 300
    long_len: int = 6000
    long_share: float = 0.5
    div_min: float = 0.10
    div_max: float = 0.20
    unit_min: int = 1
    unit_max: int = 6
    run_min: int = 20
    run_max: int = 400

    def to_c(self) -> ma_repeat_model:
        return ma_repeat_model(self.repeat_frac, self.tandem_frac, self.families, self.short_len, self.long_len,
                               self.long_share, self.div_min, self.div_max, self.unit_min, self.unit_max,
                               self.run_min, self.run_max)


def write_reference_model(path, total_len: int, n_contigs: int = 1, gc: float = 0.41, cpg: float = 0.01,
                          seed: int = 0, repeats: RepeatModel | None = None) -> None:
    """FASTA from the same base model as write_reference, generated contig by
    contig on host threads, with the repeat model when `repeats` is given."""
    rm = repeats.to_c() if repeats is not None else None
    check(lib.ma_synth_reference_model(fspath(path), total_len, n_contigs, gc, cpg, seed,
                                       None if rm is None else C.byref(rm)))


@dataclass
class ReadModel:
    len_fixed: int = 150
    len_lognorm_median: float = 120.0
    len_lognorm_sigma: float = 0.35
    len_min: int = 36
    len_max: int = 300
    frag_mean: float = 350.0
    frag_sd: float = 50.0
    conv_non_cpg: float = 0.99
    cpg_retain: float = 0.75
    sub_rate: float = 0.005
    random_frac: float = 0.05
    non_directional: float = 0.0

    def to_c(self) -> ma_read_model:
        return ma_read_model(self.len_fixed, self.len_lognorm_median, self.len_lognorm_sigma, self.len_min,
                             self.len_max, self.frag_mean, self.frag_sd, self.conv_non_cpg, self.cpg_retain,
                             self.sub_rate, self.random_frac, self.non_directional)


@dataclass
class ReadBatch:
    """Padded row-major ASCII reads: R1 rows, then R2 rows when paired."""
    bases: np.ndarray  # uint8 [n_seq, max_len]
    lens: np.ndarray   # uint32 [n_seq]
    n1: int
    paired: bool
    max_len: int
    truth_pos: np.ndarray | None = None
    truth_rev: np.ndarray | None = None

    @property
    def n_seq(self) -> int:
        return self.n1 * (2 if self.paired else 1)


def simulate_reads(fasta, model: ReadModel, n1: int, paired: bool, max_len: int, seed: int = 1,
                   bases_out: np.ndarray | None = None) -> ReadBatch:
    n_seq = n1 * (2 if paired else 1)
    bases = bases_out if bases_out is not None else np.empty((n_seq, max_len), dtype=np.uint8)
    lens = np.empty(n_seq, dtype=np.uint32)
    tp = np.empty(n_seq, dtype=np.uint64)
    tr = np.empty(n_seq, dtype=np.uint8)
    m = model.to_c()
    check(lib.ma_synth_reads(fspath(fasta), m, n1, int(paired), max_len, seed, ptr(bases), ptr(lens), ptr(tp),
                             ptr(tr)))
    return ReadBatch(bases, lens, n1, paired, max_len, tp, tr)
