"""Measured random-gather roofline of this GPU.

    python -m mojoalign_b200.roofline [device]

Times uniformly random, independent loads of aligned 32- and 64-byte lines
over buffers from 16 MiB (L2-resident) to 32 GiB (HBM) with
ma_bench_gather and prints one JSON object of GB/s per buffer size and
line size.  The seed/extend kernels gather 32-byte Occ lines, k-mer table
entries and SA entries at random: this is their ceiling, far below the
sequential copy bandwidth.
"""
from __future__ import annotations

import json
import sys

from .mapper import GpuContext

SIZES_MB = (16, 64, 256, 1024, 4096, 8192, 16384, 32768)


def sweep(device: int = 0, sizes_mb=SIZES_MB, loads: int = 1 << 30) -> dict:
    ctx = GpuContext(device)
    try:
        out = {}
        for mb in sizes_mb:
            for lb in (32, 64):
                out[f"{mb}MiB_{lb}B_GBs"] = round(ctx.gather_gbps(mb << 20, lb, loads), 1)
        return out
    finally:
        ctx.close()


if __name__ == "__main__":
    print(json.dumps(sweep(int(sys.argv[1]) if len(sys.argv) > 1 else 0)))
