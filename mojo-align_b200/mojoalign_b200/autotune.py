"""Autotuner for the result-neutral execution choices of the seed kernels.

Sweeps the kernel form (one thread per read, two stages, or wavefront
rounds), the number of right endpoints stage 1 (or the first round)
covers, the round width, the seed kernels' register budget and the
persistent stage-2 grid, on a sample batch.  Every candidate must produce
identical outputs (checked here); the fastest by device time wins.

In the wavefront form a round gives every active read `wave_endpoints`
search threads, so the round width is the warps-per-read choice: 4, 8 and
16 endpoints pack 8, 4 and 2 reads per warp (64, 32, 16 reads per 256-thread
CTA), 32, 64 and 128 endpoints give each read 1, 2 and 4 warps (8, 4 and 2
reads per CTA).  The stage-2 warps take one read each.  seed_kernel 3 is the
wavefront with lane refill in the search pass (each lane takes a new
endpoint when its search ends) and staged shifts in the eval pass (the live
shifts of a warp's loci evaluated 32 at a time); seed_kernel 4 combines the
plain search pass with the staged eval pass.

The seed stride is not swept: it decides which right endpoints are tried
(linear_gpu_fm.mojo:1828) and so changes results.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mapper import GpuContext, GpuIndex, MapResult, map_batch
from .params import FmParams

DEFAULT_CANDIDATES = [
    (0, 1, 0, 1, 16, 32, 32),
    (1, 1, 0, 2, 1, 1, 32),
    (2, 1, 0, 0, 1, 1, 8, 4, 0, 1),
    (2, 1, 0, 1, 1, 1, 8, 4, 0, 1),
    (2, 1, 0, 2, 1, 1, 8, 4, 0, 1),
    (2, 1, 0, 0, 1, 1, 16, 4, 0, 0),
    (2, 1, 0, 1, 1, 1, 16, 4, 0, 0),
    (2, 1, 0, 0, 1, 1, 4, 4, 0, 1),
    (2, 1, 0, 1, 1, 1, 4, 4, 0, 1),
    (2, 2, 0, 1, 1, 1, 8, 4, 0, 1),
    (2, 1, 0, 1, 1, 1, 8, 8, 0, 1),    # larger locus lists (many multi-row seeds: genome scale)
    (2, 1, 0, 1, 1, 1, 8, 16, 0, 1),
    (2, 2, 0, 1, 1, 1, 8, 16, 0, 1),
    (2, 1, 0, 2, 1, 1, 8, 16, 0, 1),
    (2, 1, 0, 1, 1, 1, 32, 4, 0, 0),   # one warp per read and round
    (2, 1, 0, 1, 1, 1, 64, 4, 0, 0),   # two warps per read
    (2, 1, 0, 1, 1, 1, 128, 4, 0, 0),  # four warps per read
    (3, 1, 0, 1, 1, 1, 8, 4, 0, 1),    # lane refill in the search pass
    (3, 1, 0, 2, 1, 1, 8, 4, 0, 1),
    (3, 1, 0, 1, 1, 1, 8, 16, 0, 1),
    (3, 2, 0, 1, 1, 1, 8, 16, 0, 1),
    (3, 1, 0, 2, 1, 1, 8, 16, 0, 1),
    (3, 1, 0, 1, 1, 1, 32, 16, 0, 0),
    (4, 1, 0, 1, 1, 1, 8, 4, 0, 1),    # plain search, staged eval
    (4, 1, 0, 1, 1, 1, 8, 16, 0, 1),
    (4, 2, 0, 1, 1, 1, 8, 16, 0, 1),
    (4, 2, 0, 2, 1, 1, 8, 16, 0, 1),
    (2, 2, 0, 1, 1, 1, 8, 32, 0, 1),   # locus lists of 32 per read
    (4, 2, 0, 1, 1, 1, 8, 32, 0, 1),
]
FIELDS = ("seed_kernel", "stage1_endpoints", "stage2_blocks_per_sm", "reg_level", "stage1_max_rows",
          "stage2_first_wave", "wave_endpoints", "wave_loci_per_read", "wave_max_rounds", "wave_growth")


DEFAULTS = (2, 1, 0, 2, 1, 1, 8, 4, 0, 1)


@dataclass
class TuneResult:
    tuning: dict
    seed_ms: float
    all_ms: list


def autotune(ctx: GpuContext, index: GpuIndex, bases: np.ndarray, lens: np.ndarray, n1: int, paired: bool,
             max_len: int, bs_r1="C2T", bs_r2="G2A", params: FmParams | None = None, candidates=None,
             reps: int = 2, run=None) -> TuneResult:
    """`run()`, when given, maps the sample once with the context's current
    tuning and returns (outputs as a dict of arrays, seed/extend ms); by
    default the sample goes through map_batch from host memory."""
    params = params or FmParams()
    candidates = candidates or DEFAULT_CANDIDATES
    n_seq = n1 * (2 if paired else 1)
    ref = None
    timings = []

    def host_run():
        res = MapResult.empty(n_seq, debug=True)
        map_batch(ctx, index, bases, lens, n1, paired, max_len, bs_r1, bs_r2, params, out=res)
        return {f: getattr(res, f) for f in MapResult.FIELDS + MapResult.DEBUG}, ctx.kernel_ms()[1]

    run = run or host_run
    ctx.set_profiling(1)
    try:
        for cand in candidates:
            ctx.set_tuning(*cand)
            out, _ = run()
            if ref is None:
                ref = out
            else:
                for f in ref:
                    if not np.array_equal(out[f], ref[f]):
                        raise AssertionError(f"tuning {cand} changed output {f}; the kernels are not result-neutral")
            timings.append((min(run()[1] for _ in range(reps)), cand))
    finally:
        ctx.set_profiling(0)
    best_ms, best = min(timings)
    ctx.set_tuning(*best)
    best = tuple(best) + tuple(DEFAULTS[len(best):])
    return TuneResult(dict(zip(FIELDS, best)), best_ms,
                      [{"tuning": dict(zip(FIELDS, c)), "seed_ms": round(t, 3)} for t, c in timings])
