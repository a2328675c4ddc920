"""The process boundary of the FM engine: `python -m mojoalign_b200.linear_mapper`.

Mirrors the command line the orchestrator runs (fq2bam-meth/python/
fq2bam_meth.py:582-608, `mojo fq2bam-meth/src/linear_mapper.mojo ...`):

    -ref <fasta or bwameth.c2t prefix> -fq1 <R1> [-fq2 <R2>] -out_sam <.sam|.bam>
    [-device nvidia|amd|auto] [-k N] [-cache_dir D] [-bs_r1 C2T] [-bs_r2 G2A]
    [-build_cache_only]

with the parser of run_mojo_linear_cli (linear_mapper.mojo:314-346; `-key
value` pairs read by utility.get_kv_value) and the engine choice of its
map_fastq_to_sam (L129-166): METHYLGRAPHER_LINEAR_ENGINE=fm (or bwa-mem /
bwamem), METHYLGRAPHER_LINEAR_GPU_LOCATE on, a GPU device and no
-build_cache_only run map_fastq_fm_gpu, the engine this library implements.
The k-mer engines (parity, dense) are not part of it: asking for one fails,
and so does every other error, with a message on stderr and exit status 1,
which is what makes the orchestrator fall back to BWA (unless GPU_REQUIRE=1).
-k and -cache_dir belong to the k-mer engines; the FM path ignores them, as
the reference's does.
"""
from __future__ import annotations

import os
import sys
import time

FM_ENGINES = ("fm", "bwa-mem", "bwamem")


def get_kv_value(args: list, key: str, default: str) -> str:
    """utility.get_kv_value (methylgrapher/src/utility.mojo:151-165): the
    argument after the first `-<key>`, or `default` (also when `-<key>` is
    the last argument)."""
    for i, a in enumerate(args):
        if len(a) > 1 and a.startswith("-") and a[1:] == key:
            return args[i + 1] if i + 1 < len(args) else default
    return default


def run_mojo_linear_cli(args: list, environ=None) -> int:
    """run_mojo_linear_cli: returns the exit status; raises on errors."""
    env = os.environ if environ is None else environ
    ref_fa = get_kv_value(args, "ref", "")
    fq1 = get_kv_value(args, "fq1", "")
    fq2 = get_kv_value(args, "fq2", "")
    out_sam = get_kv_value(args, "out_sam", "aligned.sam")
    device = get_kv_value(args, "device", "auto")
    int(get_kv_value(args, "k", "15"))  # parsed like the reference (a bad -k fails)
    bs_r1 = get_kv_value(args, "bs_r1", "")
    bs_r2 = get_kv_value(args, "bs_r2", "")
    build_cache_only = any(a in ("-build_cache_only", "--build_cache_only") for a in args)
    if not ref_fa:
        raise RuntimeError("MojoLinearMap requires -ref")
    if not build_cache_only and not fq1:
        raise RuntimeError("MojoLinearMap requires -fq1 (or pass -build_cache_only)")
    engine = env.get("METHYLGRAPHER_LINEAR_ENGINE", "parity").lower()
    locate = env.get("METHYLGRAPHER_LINEAR_GPU_LOCATE", "1").lower()
    locate_on = locate in ("", "1", "true", "yes")
    if not (engine in FM_ENGINES and locate_on and device.lower() in ("nvidia", "amd", "auto")
            and not build_cache_only):
        raise RuntimeError(f"MojoLinear engine {engine!r} (device {device!r}"
                           f"{', -build_cache_only' if build_cache_only else ''}) is not part of this build; "
                           "it runs the FM engine: METHYLGRAPHER_LINEAR_ENGINE=fm, "
                           "METHYLGRAPHER_LINEAR_GPU_LOCATE=1, -device nvidia|auto")
    from .linear_fm import map_fastq_fm_gpu

    print("MojoLinear engine=fm (opt-in FM-index / BWA-MEM-style)", flush=True)
    t0 = time.perf_counter()
    n_mapped = map_fastq_fm_gpu(ref_fa, fq1, out_sam, device, fq2, bs_r1, bs_r2, environ=env)
    print(f"wrote records -> {out_sam} mapped_records= {n_mapped} backend=gpu-fm", flush=True)
    print(f"MojoLinear GPU-fm map_wall_s= {time.perf_counter() - t0:.3f}", flush=True)
    return 0


def main(argv=None) -> int:
    args = list(sys.argv[1:] if argv is None else argv)
    try:
        return run_mojo_linear_cli(args)
    except Exception as e:  # fail closed: message, status 1
        print(f"MojoLinearMap error: {e}", file=sys.stderr, flush=True)
        return 1


if __name__ == "__main__":
    sys.exit(main())
