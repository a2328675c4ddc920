"""Mapping parameters of the FM path and their env knobs.

Mirrors the knob block of map_fastq_fm_gpu
(fq2bam-meth/src/linear_gpu_fm.mojo:2074-2082) and the parser _env_int
(fq2bam-meth/src/linear_gpu_locate.mojo:139-145): an unset variable gives the
default, a value below 1 gives the default, a non-integer raises.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, fields

from ._lib import ma_params

ENV_NAMES = {
    "seed_len": ("METHYLGRAPHER_FM_SEED_LEN", 18),
    "seed_stride": ("METHYLGRAPHER_FM_SEED_STRIDE", 2),
    "max_occ": ("METHYLGRAPHER_FM_MAX_OCC", 4096),
    "max_diff": ("METHYLGRAPHER_FM_MAX_DIFF", 12),
    "max_soft": ("METHYLGRAPHER_FM_MAX_SOFT", 20),
    "max_adj": ("METHYLGRAPHER_FM_ADJ", 8),
    "rescue_win": ("METHYLGRAPHER_FM_RESCUE_WIN", 512),
}
READ_BATCH_ENV = ("METHYLGRAPHER_LINEAR_READ_BATCH", 16384)


def env_int(name: str, default: int, environ=None) -> int:
    env = os.environ if environ is None else environ
    n = int(env.get(name, str(default)))
    return default if n < 1 else n


@dataclass(frozen=True)
class FmParams:
    seed_len: int = 18
    seed_stride: int = 2
    max_occ: int = 4096
    max_diff: int = 12
    max_soft: int = 20
    max_adj: int = 8
    rescue_win: int = 512

    @classmethod
    def from_env(cls, environ=None) -> "FmParams":
        return cls(**{f: env_int(n, d, environ) for f, (n, d) in ENV_NAMES.items()})

    def to_c(self) -> ma_params:
        return ma_params(*[getattr(self, f.name) for f in fields(self)])

    def as_list(self) -> list[int]:
        return [getattr(self, f.name) for f in fields(self)]


# The workload parameters of the benchmark configurations: the reference
# defaults with seed_len 19 and max_occ 500.
BENCH_PARAMS = FmParams(seed_len=19, max_occ=500)
