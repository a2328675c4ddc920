#!/usr/bin/env python
"""Benchmark of the linear bisulfite seed-and-extend path (reads/s).

Default workload (`--workload genome`, per GPU): a synthetic 3.1 Gbp
reference (GC 0.41, CpG ~1%, seed 0) indexed as the bwa-meth dual-strand
text (12.4 G symbols, the index built on the GPU), and 50 M single-end
bisulfite reads with lengths lognormal (median 120) clipped to 36-300, half
of them non-directional (seed 1 + rank).  One step maps every read through
the batched form (the autotuned wavefront kernels, one device call per 8 M
reads, each call replayed from a captured CUDA graph).  Beside it: the plain
single-launch form (the reference's launch shape) and the served form on the
same reads, a served stream of 8 samples with p50 / p99 / p99.9 latency,
the oracle on a 1 M-read parity sample, and the file stages (BAM, sort,
BGZF, FASTQ -> BAM / SAM) on a 250 Mbp reference.

`--workload chromosome`: 250 Mbp, 10 M pairs 2x150, the plain single-launch
call; `--workload repeats`: 3.1 Gbp with 45% repeats, 10 M pairs 2x250 at
non-CpG conversion 0.97.  Parameters: the reference defaults with seed_len
19 and max_occ 500; each mate counts as one read.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload ...]

Prints one JSON line (rank 0).  `value` is measured with the reads already
in HBM; `e2e` through the host API (ma_map_batch) with pinned host buffers,
copies included.  `--impl reference` times the CPU restatement of the
reference kernels (the oracle; the Mojo reference cannot run here) on all
host cores over a bounded sample of the same workload.  Progress lines go
to stderr.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for p in (ROOT, ROOT / "mojo-align_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

import numpy as np  # noqa: E402

METRIC = "reads/s seed+extend"
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the seed
# kernels (wf_init through seed_stage2, pack excluded) per read of one timed
# step of the default genome workload (3100 Mbp, 50 M uneven single-end
# reads), from a one-pass ncu capture of that step on this build with the
# tuning below; roofline.traffic reports it for runs of that workload and
# tuning, and null otherwise.
GENOME_SEED_DRAM_BYTES_PER_READ = 24660
GENOME_SEED_DRAM_TUNING = (4, 2, 0, 1, 1, 1, 8, 32, 0, 1)
GENOME_SEED_DRAM_AT_K = 28  # the capture's A/T window table (0: none)
# The workload parameters: the reference defaults with seed_len 19 and
# max_occ 500 (mojoalign_b200.params.BENCH_PARAMS holds the same values; the
# reference arm takes them from here so that it loads nothing of the
# package).
BENCH_PARAM_VALUES = {"seed_len": 19, "seed_stride": 2, "max_occ": 500, "max_diff": 12, "max_soft": 20,
                      "max_adj": 8, "rescue_win": 512}
SEED_KERNELS = {
    0: "seed/extend: seed_stage1_kernel over every endpoint (one thread per read)",
    1: "seed/extend: seed_stage1_kernel + seed_stage2_kernel (thread per read, then warp per read)",
    2: "seed/extend: wavefront rounds (wf_search_kernel + wf_eval_kernel + wf_finalize_kernel per round, "
       "seed_stage2_kernel for reads left over)",
    3: "seed/extend: wavefront rounds with lane refill (wf_search_refill_kernel + wf_eval_staged_kernel + "
       "wf_finalize_kernel per round, seed_stage2_kernel for reads left over)",
    4: "seed/extend: wavefront rounds with staged eval (wf_search_kernel + wf_eval_staged_kernel + "
       "wf_finalize_kernel per round, seed_stage2_kernel for reads left over)",
}
READ_LEN = 150


_T0 = time.time()


def log(msg: str) -> None:
    """One progress line on stderr (the JSON line alone goes to stdout)."""
    sys.stderr.write(f"[bench +{time.time() - _T0:7.1f}s] {msg}\n")
    sys.stderr.flush()


def profiled_region(start: bool) -> None:
    """cudaProfilerStart / cudaProfilerStop around the timed mapping steps:
    `ncu --profile-from-start off` then captures exactly those launches (no
    effect without a profiler)."""
    import torch

    if start:
        torch.cuda.profiler.start()
    else:
        torch.cuda.profiler.stop()


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--genome-mb", type=int, default=250)
    ap.add_argument("--pairs", type=int, default=10_000_000, help="read pairs per GPU")
    ap.add_argument("--kmer", type=int, default=12)
    ap.add_argument("--kmer3", type=int, default=19, help="converted-alphabet k-mer tables (<= seed_len)")
    ap.add_argument("--at-k", type=int, default=28, help="A/T window outcome table: window length (0 = none); "
                    "built for the workload's seed length")
    ap.add_argument("--workdir", default=os.environ.get("MOJOALIGN_BENCH_DIR", tempfile.gettempdir()))
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU time of the baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the oracle timing (profiling runs)")
    ap.add_argument("--no-forms", action="store_true", help="skip the plain / batched / served comparison")
    ap.add_argument("--no-stages", action="store_true", help="genome workloads: skip the file stages (BAM, sort, "
                    "BGZF, FASTQ -> BAM / SAM, FASTQ split) on the chromosome-scale reference")
    ap.add_argument("--forms-reads", type=int, default=4_000_000, help="uneven-length reads of the comparison")
    ap.add_argument("--forms-ref-batches", type=int, default=64, help="16384-read batches timed in the "
                    "reference-loop form")
    ap.add_argument("--serve-pool", type=int, default=2_000_000, help="reads per simulated sample")
    ap.add_argument("--serve-burst", type=int, default=160, help="requests of the saturation burst")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="Poisson phase duration")
    ap.add_argument("--serve-group", type=int, default=262144, help="reads (pairs) per launch group")
    ap.add_argument("--serve-budget-gb", type=int, default=8, help="serving HBM budget")
    ap.add_argument("--bam-pairs", type=int, default=1_000_000, help="read pairs of the BAM-packing batch "
                    "(0 = skip that stage)")
    ap.add_argument("--sort-batches", type=int, default=4, help="BAM batches (of --bam-pairs pairs) in the "
                    "tile of the sort / duplicate-marking / gather stage (0 = skip)")
    ap.add_argument("--fastq-pairs", type=int, default=2_000_000, help="read pairs of the FASTQ-split stage "
                    "(its R1 file; 0 = skip)")
    ap.add_argument("--bgzf-level", type=int, default=1, help="BGZF level of the compression stage "
                    "(the reference's default, METHYLGRAPHER_BAM_LEVEL=1; -1 = skip)")
    ap.add_argument("--fq2bam-pairs", type=int, default=2_000_000, help="read pairs of the FASTQ -> sorted BAM "
                    "stage (0 = skip)")
    ap.add_argument("--fq2sam-pairs", type=int, default=2_000_000, help="read pairs of the FASTQ -> SAM stage "
                    "(0 = skip)")
    ap.add_argument("--workload", choices=["chromosome", "genome", "repeats"], default="genome",
                    help="chromosome: 250 Mbp, 10 M pairs 2x150, plain single-launch (and the file stages); "
                    "genome: 3.1 Gbp, 50 M uneven single-end reads, batched / plain / served forms and the served "
                    "stream; repeats: 3.1 Gbp with 45%% repeats, 10 M pairs 2x250 at conversion 0.97")
    ap.add_argument("--genome-mb-large", type=int, default=0, help="reference size of the genome workloads "
                    "(0 = 3100)")
    ap.add_argument("--genome-reads", type=int, default=0, help="reads (pairs) of the genome workloads "
                    "(0 = the workload's)")
    ap.add_argument("--genome-chunk", type=int, default=8_000_000, help="reads per device call (a wavefront "
                    "round lists at most 2^31-1 loci: smaller calls leave room for more loci per read)")
    ap.add_argument("--parity-reads", type=int, default=1_000_000, help="reads checked against the oracle")
    ap.add_argument("--serve-stream-budget-mb", type=int, default=512, help="HBM budget of the served stream "
                    "(below what max_inflight groups need, so that admission waits)")
    ap.add_argument("--gather-sweep", action="store_true", help="print the measured random-gather roofline "
                    "(32- and 64-byte lines, 16 MiB to 32 GiB buffers) as one JSON object and exit")
    ap.add_argument("--prepare-sample", default="", help=argparse.SUPPRESS)
    ap.add_argument("--tuning", default="", help="fixed kernel choice 'seed_kernel,stage1_endpoints,"
                    "stage2_blocks_per_sm,reg_level,stage1_max_rows,stage2_first_wave[,wave_endpoints,"
                    "wave_loci_per_read,wave_max_rounds,wave_growth]' instead of the autotuner")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Dist:
    """Barrier / max-reduce over ranks (torch.distributed when world > 1)."""

    def __init__(self, world: int, backend: str):
        self.world = world
        self.pg = None
        if world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=1800))
            self.dist = dist
            self.pg = True
        self.backend = backend

    def barrier(self):
        if self.pg:
            if self.backend == "nccl":
                import torch

                self.dist.barrier(device_ids=[torch.cuda.current_device()])
            else:
                self.dist.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch

        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.dist.destroy_process_group()


def aggregate_reads_per_s(reads_per_rank: int, world: int, ms_max: float) -> float:
    """Weak scaling: every rank maps its own batch; the job's rate is all
    ranks' reads over the slowest rank's step time."""
    return reads_per_rank * world / (ms_max / 1000.0)


def shard_seed(rank: int) -> int:
    """Read-simulation seed of a rank: each rank maps different reads."""
    return 1 + rank


def prepare_reference(args, rank, dist: Dist, device: int, genome_mb: int | None = None, repeats=None,
                      tag: str = ""):
    """Synthetic reference + bwa-meth index, built once per node by rank 0
    (the index on the GPU).  `repeats` (a synth.RepeatModel) adds the
    repeat-heavy model."""
    from mojoalign_b200 import build_index, synth

    genome_mb = genome_mb or args.genome_mb
    d = Path(args.workdir) / f"mojoalign_bench_{genome_mb}mb{tag}"
    d.mkdir(parents=True, exist_ok=True)
    fa = d / "ref.fa"
    prefix = Path(str(fa) + ".bwameth.c2t")
    done = d / "index.ok"
    t0 = time.time()
    if rank == 0 and not done.exists():
        try:
            import torch

            device = device if torch.cuda.is_available() else -1
        except ImportError:
            device = -1
        n_contigs = max(1, min(24, genome_mb // 50))
        log(f"synthetic reference: {genome_mb} Mbp")
        synth.write_reference_model(fa, genome_mb * 1_000_000, n_contigs=n_contigs, gc=0.41, cpg=0.01, seed=0,
                                    repeats=repeats)
        log("index build")
        build_index(fa, prefix, bwameth_c2t=True, sa_intv=32, device=device)
        log("index built")
        done.write_text("ok\n")
    dist.barrier()
    return fa, prefix, time.time() - t0


def simulate(args, fa, rank, bases_out=None):
    from mojoalign_b200 import synth

    model = synth.ReadModel(len_fixed=READ_LEN, frag_mean=350, frag_sd=50, conv_non_cpg=0.99, cpg_retain=0.75,
                            sub_rate=0.005, random_frac=0.05)
    return synth.simulate_reads(fa, model, args.pairs, True, READ_LEN, seed=shard_seed(rank), bases_out=bases_out)


def sample_pairs(rb, n):
    """First n pairs of a paired batch, as a smaller paired batch."""
    b = np.concatenate([rb.bases[:n], rb.bases[rb.n1:rb.n1 + n]])
    l = np.concatenate([rb.lens[:n], rb.lens[rb.n1:rb.n1 + n]])
    return b, l


def time_oracle(prefix, rb, params, target_s, probe_pairs=20000, min_pairs=500_000):
    """Times the oracle on a bounded sample sized to about target_s seconds,
    at least min_pairs pairs (the parity sample: 1 M reads or more)."""
    import oracle

    ix = oracle.OracleIndex(prefix)
    b, l = sample_pairs(rb, probe_pairs)
    t = time.perf_counter()
    ix.map(b, l, probe_pairs, True, READ_LEN, 1, 2, params.as_list())
    rate = 2 * probe_pairs / (time.perf_counter() - t)
    n = int(min(rb.n1, max(probe_pairs, min_pairs, rate * target_s / 2)))
    b, l = sample_pairs(rb, n)
    t = time.perf_counter()
    out = ix.map(b, l, n, True, READ_LEN, 1, 2, params.as_list())
    dt = time.perf_counter() - t
    return ix, out, n, 2 * n / dt, dt


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = Path(tempfile.mkstemp(prefix="clocks_", suffix=".csv")[1])

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        rows = [r.split(",") for r in self.path.read_text().splitlines() if r.count(",") >= 8]
        self.path.unlink(missing_ok=True)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        busy = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


BAM_RG = b"mojo1"
BAM_NAME_LEN = 20


def bam_batch(rb, res, n1: int, first: int = 0, seed: int = 7):
    """The BAM packer's input for pairs [first, first + n1) of the mapped
    workload: their mapping outputs and a FASTQ arena of 20-byte names, the
    original bases and phred+33 qualities 2..41, records of equal size back
    to back (name, bases, qualities per record, the reference arena's
    order)."""
    from mojoalign_b200.bam import HIT_FIELDS, BatchArena

    sel = np.concatenate([first + np.arange(n1), rb.n1 + first + np.arange(n1)])
    n_seq = 2 * n1
    hits = {k: np.ascontiguousarray(getattr(res, k)[sel]).astype(t, copy=False) for k, t in HIT_FIELDS}
    rec = BAM_NAME_LEN + 2 * READ_LEN
    data = np.empty((n_seq, rec), np.uint8)
    idx = np.arange(n_seq)
    digits = np.array([(first + idx % n1) // 10 ** k % 10 for k in range(9, -1, -1)], np.uint8).T + 48
    data[:, :10] = np.frombuffer(b"B200:7:FC:", np.uint8)
    data[:, 10:20] = digits
    data[:, BAM_NAME_LEN:BAM_NAME_LEN + READ_LEN] = rb.bases[sel, :READ_LEN]
    data[:, BAM_NAME_LEN + READ_LEN:] = np.random.default_rng(seed + first).integers(35, 75, size=(n_seq, READ_LEN),
                                                                                      dtype=np.uint8)
    base = idx.astype(np.uint64) * rec
    arena = BatchArena(data.reshape(-1), base, np.full(n_seq, BAM_NAME_LEN, np.uint32),
                       base + BAM_NAME_LEN, rb.lens[sel].astype(np.uint32),
                       base + BAM_NAME_LEN + READ_LEN, rb.lens[sel].astype(np.uint32))
    return hits, arena


def device_copy(a, dev):
    """numpy -> device tensor holding the same bytes (unsigned integer
    arrays travel as the signed type of their width)."""
    import torch

    a = np.ascontiguousarray(a)
    signed = {np.dtype(np.uint64): np.int64, np.dtype(np.uint32): np.int32}
    if a.dtype in signed:
        a = a.view(signed[a.dtype])
    if not a.flags.writeable:
        a = a.copy()
    return torch.from_numpy(a).to(dev)


def run_bam_stage(args, ctx, rb, res, local, peaks):
    """BAM record packing of one mapped batch: device-resident throughput,
    the host API end to end, the oracle on one core, and byte parity."""
    import torch

    import oracle
    from mojoalign_b200.bam import META_FIELDS, BamTile, emit_bam_device, emit_bam_from_batch

    n1 = min(args.bam_pairs, rb.n1)
    hits, arena = bam_batch(rb, res, n1)
    n_seq = 2 * n1
    tids = np.arange(16, dtype=np.int32) // 2  # f<name> / r<name> contigs share a tid
    # parity at full size and the CPU baseline (one core)
    t = time.perf_counter()
    want, want_meta, want_mapped = oracle.emit_bam(hits, vars(arena), n1, True, tids, BAM_RG, meta_cap=n_seq,
                                                   cap=n_seq * 512)
    cpu_s = time.perf_counter() - t
    bam_bytes = len(want)
    dev = torch.device("cuda", local)
    d_hits = {k: device_copy(v, dev) for k, v in hits.items()}
    d_arena = {k: device_copy(getattr(arena, k), dev)
               for k in ("data", "name_off", "name_len", "orig_off", "orig_len", "qual_off", "qual_len")}
    d_tids = device_copy(tids, dev)
    d_rg = device_copy(np.frombuffer(BAM_RG, np.uint8), dev)
    d_bam = torch.empty(bam_bytes + 16, dtype=torch.uint8, device=dev)
    d_meta = {k: torch.empty(n_seq, dtype=torch.int64 if t_ == np.uint64 else torch.int32, device=dev)
              for k, t_ in META_FIELDS}
    d_status = torch.zeros(3, dtype=torch.int64, device=dev)
    tile = BamTile(meta_cap=n_seq, host_meta=False)
    torch.cuda.synchronize()
    stream = torch.cuda.Stream(device=dev)  # a handle of 0 would select the context's own stream

    def step():
        emit_bam_device(ctx, {k: v.data_ptr() for k, v in d_hits.items()}, n1, True,
                        {k: v.data_ptr() for k, v in d_arena.items()}, int(arena.data.size), d_tids.data_ptr(),
                        int(tids.size), d_rg.data_ptr(), len(BAM_RG), d_bam.data_ptr(), bam_bytes,
                        {k: v.data_ptr() for k, v in d_meta.items()}, tile, d_status.data_ptr(),
                        stream.cuda_stream)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    launches = ctx.last_launch_count()
    status = d_status.cpu().numpy()
    same = d_bam[:bam_bytes].cpu().numpy().tobytes() == want and int(status[1]) == want_mapped
    for k, t_ in META_FIELDS:
        same = same and np.array_equal(d_meta[k].cpu().numpy().view(t_), want_meta[k])
    del d_hits, d_arena, d_bam, d_meta
    # end to end: pinned host buffers in, records and metadata out
    pin = {k: torch.from_numpy(v.view(np.int32) if v.dtype == np.uint32 else v).pin_memory().numpy().view(v.dtype)
           for k, v in hits.items()}
    pin_arena = type(arena)(*[None if v is None else torch.from_numpy(
        v.view({8: np.int64, 4: np.int32, 1: np.uint8}[v.itemsize])).pin_memory().numpy().view(v.dtype)
        for v in (arena.data, arena.name_off, arena.name_len, arena.orig_off, arena.orig_len, arena.qual_off,
                  arena.qual_len)])
    out = torch.empty(bam_bytes, dtype=torch.uint8, pin_memory=True).numpy()
    host_tile = BamTile(meta_cap=n_seq, meta={k: torch.empty(n_seq, dtype=torch.int64 if t_ == np.uint64 else
                                                             torch.int32, pin_memory=True).numpy().view(t_)
                                              for k, t_ in META_FIELDS})
    emit_bam_from_batch(ctx, pin, n1, True, pin_arena, tids, BAM_RG, host_tile, bam_bytes, out=out)
    t = time.perf_counter()
    for _ in range(args.steps):
        host_tile.n_reads = 0
        emit_bam_from_batch(ctx, pin, n1, True, pin_arena, tids, BAM_RG, host_tile, bam_bytes, out=out)
    e2e_s = (time.perf_counter() - t) / args.steps
    same = same and out.tobytes() == want
    in_bytes = int(arena.name_len.sum()) + int(arena.orig_len.sum()) + int(arena.qual_len.sum())
    alg = n_seq * (28 + 36 + 44) + in_bytes + bam_bytes
    achieved = alg / (ms / 1000.0) / 1e9
    return {
        "metric": "records/s BAM pack", "value": round(n_seq / (ms / 1000.0), 1), "unit": "records/s",
        "ms_per_batch": round(ms, 3),
        "config": {"workload": f"BAM records of the first {n1} pairs of the mapped workload (PE 2x{READ_LEN}, "
                               f"{BAM_NAME_LEN}-byte names, qualities, RG {BAM_RG.decode()})",
                   "records": n_seq, "bam_bytes": bam_bytes, "mapped_records": want_mapped},
        "e2e": {"value": round(n_seq / e2e_s, 1), "unit": "records/s",
                "h2d_bytes_per_step": int(arena.data.size + n_seq * (28 + 36)),
                "d2h_bytes_per_step": int(bam_bytes + n_seq * 44)},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                     "frac": round(achieved / peaks.get("hbm_gbs"), 4), "traffic": None,
                     "alg_bytes_per_launch": alg,
                     "kernel": "bam_layout_kernel + record-size scan + bam_records_kernel (one emit call)"},
        "gpu_launches": launches * args.steps,
        "cpu_baseline": {"value": round(n_seq / cpu_s, 1), "unit": "records/s", "cores": 1, "kind": "port",
                         "sample": f"the whole batch ({n_seq} records), {cpu_s:.2f} s"},
        "parity": {"records": n_seq, "bytes_and_metadata_identical": bool(same)},
    }


def fastq_text(rb, n: int, mate: int = 1, seed: int = 11) -> bytes:
    """FASTQ text of n reads of the workload (mate 1: the R1 rows): Illumina-
    style headers with a comment, the original bases, '+' and phred+33
    qualities, LF line ends."""
    rows = rb.bases[(mate - 1) * rb.n1:(mate - 1) * rb.n1 + n, :READ_LEN]
    comment = b" %d:N:0:ACGTACGT\n" % mate
    c = len(comment)
    rec = np.empty((n, 21 + c + 2 * READ_LEN + 4), np.uint8)
    rec[:, :11] = np.frombuffer(b"@B200:7:FC:", np.uint8)
    idx = np.arange(n)
    rec[:, 11:21] = np.array([idx // 10 ** k % 10 for k in range(9, -1, -1)], np.uint8).T + 48
    rec[:, 21:21 + c] = np.frombuffer(comment, np.uint8)
    q = 21 + c + READ_LEN
    rec[:, 21 + c:q] = rows
    rec[:, q:q + 3] = np.frombuffer(b"\n+\n", np.uint8)
    rec[:, q + 3:q + 3 + READ_LEN] = np.random.default_rng(seed).integers(35, 75, size=(n, READ_LEN), dtype=np.uint8)
    rec[:, -1] = 10
    return rec.tobytes()


def run_fastq_stage(args, ctx, rb, local, peaks):
    """Record split + mapper rows of one FASTQ buffer on the device, the
    host-bytes path end to end, and the oracle's split on one core."""
    import ctypes as C

    import torch

    import oracle
    from mojoalign_b200 import _lib

    n = min(args.fastq_pairs, rb.n1)
    text = fastq_text(rb, n)
    nb = len(text)
    dev = torch.device("cuda", local)
    keys = ("name_off", "name_len", "seq_off", "seq_len", "qual_off", "qual_len")
    d_out = {k: torch.empty(n, dtype=torch.int64 if k.endswith("off") else torch.int32, device=dev) for k in keys}
    rec = _lib.ma_fastq_records(*[d_out[k].data_ptr() for k in keys])
    pin = torch.from_numpy(np.frombuffer(text, np.uint8).copy()).pin_memory()
    d_buf = pin.to(dev)
    d_rows = torch.empty(n * READ_LEN, dtype=torch.uint8, device=dev)
    d_lens = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    o3 = (C.c_uint64 * 3)()

    def device_step():
        _lib.check(_lib.lib.ma_fastq_parse_device(ctx.handle, d_buf.data_ptr(), nb, 1, n, 0, C.byref(rec), o3,
                                                  stream.cuda_stream), ctx.handle)
        launches = ctx.last_launch_count()
        _lib.check(_lib.lib.ma_fastq_rows_device(ctx.handle, d_buf.data_ptr(), d_out["seq_off"].data_ptr(),
                                                 d_out["seq_len"].data_ptr(), n, int(o3[2]), d_rows.data_ptr(),
                                                 d_lens.data_ptr(), stream.cuda_stream), ctx.handle)
        return launches + ctx.last_launch_count()

    torch.cuda.synchronize()
    for _ in range(max(args.warmup, 3)):
        device_step()
    stream.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    ev0.record(stream)
    for _ in range(args.steps):
        launches += device_step()
    ev1.record(stream)
    stream.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps

    def e2e_step():
        d_buf.copy_(pin, non_blocking=True)  # host bytes -> HBM on torch's stream
        torch.cuda.current_stream().synchronize()
        return device_step()

    e2e_step()
    stream.synchronize()
    t = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    stream.synchronize()
    e2e_s = (time.perf_counter() - t) / args.steps
    got = {k: d_out[k].cpu().numpy().view(np.uint64 if k.endswith("off") else np.uint32) for k in keys}
    rows = d_rows.cpu().numpy().reshape(n, READ_LEN)
    t = time.perf_counter()
    want = oracle.fastq_parse(text, max_records=n)
    cpu_s = time.perf_counter() - t
    same = int(o3[0]) == want["n"] == n and all(np.array_equal(got[k], want[k]) for k in keys)
    same = same and np.array_equal(rows, rb.bases[:n, :READ_LEN])
    alg = nb + n * (3 * 8 + 3 * 4) + n * (READ_LEN + 4)
    achieved = alg / (ms / 1000.0) / 1e9
    return {
        "metric": "records/s FASTQ split + mapper rows", "value": round(n / (ms / 1000.0), 1), "unit": "records/s",
        "ms_per_buffer": round(ms, 3), "gb_per_s_of_fastq": round(nb / (ms / 1000.0) / 1e9, 1),
        "config": {"workload": f"R1 FASTQ text of {n} reads of the workload ({READ_LEN} bp, 40-byte headers, LF)",
                   "records": n, "fastq_bytes": nb},
        "e2e": {"value": round(n / e2e_s, 1), "unit": "records/s", "h2d_bytes_per_step": nb,
                "d2h_bytes_per_step": 48},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                     "frac": round(achieved / peaks.get("hbm_gbs"), 4), "traffic": None,
                     "alg_bytes_per_launch": alg,
                     "alg": "FASTQ bytes read once + 36 B of spans and the row + length written per record"},
        "gpu_launches": launches,
        "cpu_baseline": {"value": round(n / cpu_s, 1), "unit": "records/s", "cores": 1, "kind": "port",
                         "sample": f"the whole buffer ({n} records, {nb} bytes), {cpu_s:.2f} s"},
        "parity": {"records": n, "spans_and_rows_identical": bool(same)},
    }


def run_bgzf_stage(args, ctx, stream_bytes, local, peaks):
    """BGZF of the sorted record stream: device throughput, the host API end
    to end, the oracle's zlib writer on the host cores, the size against
    zlib at the same level, and the round trip."""
    import concurrent.futures as cf
    import ctypes as C
    import zlib

    import torch

    from mojoalign_b200 import _lib
    from oracle import bgzf_ref

    data = np.ascontiguousarray(stream_bytes)
    n = int(data.size)
    level = args.bgzf_level
    dev = torch.device("cuda", local)
    d_in = torch.from_numpy(data).to(dev)
    cap = int(_lib.lib.ma_bgzf_bound(n))
    d_out = torch.empty(cap, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(device=dev)
    got = C.c_uint64(0)

    def device_step():
        _lib.check(_lib.lib.ma_bgzf_compress_device(ctx.handle, d_in.data_ptr(), n, level, 1, d_out.data_ptr(), cap,
                                                    C.byref(got), stream.cuda_stream), ctx.handle)
        return ctx.last_launch_count()

    torch.cuda.synchronize()
    for _ in range(max(args.warmup, 3)):
        device_step()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    ev0.record(stream)
    for _ in range(args.steps):
        launches += device_step()
    ev1.record(stream)
    stream.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    out = d_out[:got.value].cpu().numpy().tobytes()
    # round trip and framing of every member
    ms_ = bgzf_ref.members(out)
    ok = out[ms_[-1]["off"]:] == bgzf_ref.EOF_MEMBER and len(ms_) - 1 == (n + bgzf_ref.BLOCK - 1) // bgzf_ref.BLOCK
    mv = memoryview(data)
    for i, m in enumerate(ms_[:-1]):
        piece = mv[i * bgzf_ref.BLOCK:(i + 1) * bgzf_ref.BLOCK]
        ok = ok and m["isize"] == len(piece) and m["crc"] == (zlib.crc32(piece) & 0xFFFFFFFF)
        ok = ok and m["fixed"] == (31, 139, 8, 4, 0, 0, 255, 6, 66, 67, 2)
        if i % 16 == 0:
            ok = ok and bgzf_ref.inflate(m["payload"]) == bytes(piece)
    # end to end: pinned host stream in, BGZF bytes out
    pin_in = torch.from_numpy(data).pin_memory().numpy()
    pin_out = torch.empty(cap, dtype=torch.uint8, pin_memory=True).numpy()

    def host_step():
        _lib.check(_lib.lib.ma_bgzf_compress(ctx.handle, pin_in.ctypes.data, n, level, 1, pin_out.ctypes.data, cap,
                                             C.byref(got)), ctx.handle)

    host_step()
    t = time.perf_counter()
    for _ in range(args.steps):
        host_step()
    e2e_s = (time.perf_counter() - t) / args.steps
    ok = ok and pin_out[:got.value].tobytes() == out
    # the oracle (the reference's zlib writer) on all host cores over a sample
    sample = bytes(mv[:min(n, 256 * bgzf_ref.BLOCK)])
    cores = os.cpu_count() or 1
    pieces = [sample[i:i + bgzf_ref.BLOCK] for i in range(0, len(sample), bgzf_ref.BLOCK)]
    t = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=cores) as ex:
        zparts = list(ex.map(lambda c: bgzf_ref.member(c, level), pieces))
    cpu_s = time.perf_counter() - t
    zsize = sum(len(z) for z in zparts)
    gsize = sum(m["size"] for m in ms_[:len(pieces)])
    return {
        "metric": "GB/s BGZF (uncompressed bytes)", "value": round(n / (ms / 1000.0) / 1e9, 2), "unit": "GB/s",
        "ms_per_stream": round(ms, 3),
        "config": {"workload": "the sorted, duplicate-marked record stream of the sort stage", "bytes": n,
                   "level": level, "bgzf_bytes": len(out),
                   "ratio": round(n / len(out), 3),
                   "size_vs_zlib_same_level": round(gsize / zsize, 4)},
        "e2e": {"value": round(n / e2e_s / 1e9, 2), "unit": "GB/s", "h2d_bytes_per_step": n,
                "d2h_bytes_per_step": len(out)},
        "roofline": {"bound": "hbm", "achieved": round((n + len(out)) / (ms / 1000.0) / 1e9, 1),
                     "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                     "frac": round((n + len(out)) / (ms / 1000.0) / 1e9 / peaks.get("hbm_gbs"), 4),
                     "traffic": None, "alg_bytes_per_launch": n + len(out),
                     "alg": "input read once + members written once; the coder is bound by shared-memory "
                            "matching, not HBM"},
        "gpu_launches": launches,
        "cpu_baseline": {"value": round(len(sample) / cpu_s / 1e9, 3), "unit": "GB/s", "cores": cores,
                         "kind": "port", "sample": f"first {len(pieces)} pieces ({len(sample)} bytes) through the "
                                                   f"reference writer's zlib member code, {cores} threads, "
                                                   f"{cpu_s:.2f} s"},
        "parity": {"members": len(ms_) - 1, "framing_crc_isize_and_round_trip": bool(ok)},
    }


def run_fq2bam_stage(args, ctx, gi, rb, local, params):
    """FASTQ files of the workload -> sorted, duplicate-marked BAM file through
    map_fastq_to_bam (every stage on the GPU, files read and written on the
    host), against the same path restated on the CPU from the oracle on a
    sample (its mapping step dominates)."""
    import shutil
    import sys as _sys

    from mojoalign_b200 import _lib
    from mojoalign_b200.fq2bam import bam_header, map_fastq_to_bam

    n = min(args.fq2bam_pairs, rb.n1)
    d = Path(tempfile.mkdtemp(prefix="fq2bam_", dir=args.workdir))
    try:
        r1, r2 = d / "r1.fq", d / "r2.fq"
        r1.write_bytes(fastq_text(rb, n, 1))
        r2.write_bytes(fastq_text(rb, n, 2))
        out = d / "out.bam"
        fq_bytes = r1.stat().st_size + r2.stat().st_size
        map_fastq_to_bam(None, r1, out, fq2=r2, bs_r1="C2T", bs_r2="G2A", params=params, environ={}, ctx=ctx,
                         index=gi, level=args.bgzf_level if args.bgzf_level >= 0 else 1)
        times, phases = [], {}
        for _ in range(max(1, min(args.steps, 3))):
            t = time.perf_counter()
            mapped = map_fastq_to_bam(None, r1, out, fq2=r2, bs_r1="C2T", bs_r2="G2A", params=params, environ={},
                                      ctx=ctx, index=gi, level=args.bgzf_level if args.bgzf_level >= 0 else 1,
                                      stats=phases)
            times.append(time.perf_counter() - t)
        wall = statistics.median(times)
        bam_size = out.stat().st_size
        # the same FASTQ as BGZF files (bgzip's format, level 1): inflated on
        # the device, only the compressed members cross PCIe
        gz = []
        for src in (r1, r2):
            raw = np.fromfile(src, dtype=np.uint8)
            cap = int(_lib.lib.ma_bgzf_bound(raw.size))
            buf = np.empty(cap, np.uint8)
            size = _lib.C.c_uint64()
            _lib.check(_lib.lib.ma_bgzf_compress(ctx.handle, raw.ctypes.data, raw.size, 1, 1, buf.ctypes.data, cap,
                                                 _lib.C.byref(size)), ctx.handle)
            q = Path(str(src) + ".gz")
            buf[:size.value].tofile(q)
            gz.append(q)
        out_gz = d / "out_gz.bam"
        lvl = args.bgzf_level if args.bgzf_level >= 0 else 1
        map_fastq_to_bam(None, gz[0], out_gz, fq2=gz[1], bs_r1="C2T", bs_r2="G2A", params=params, environ={},
                         ctx=ctx, index=gi, level=lvl)
        gz_times, gz_phases = [], {}
        for _ in range(max(1, min(args.steps, 3))):
            t = time.perf_counter()
            map_fastq_to_bam(None, gz[0], out_gz, fq2=gz[1], bs_r1="C2T", bs_r2="G2A", params=params, environ={},
                             ctx=ctx, index=gi, level=lvl, stats=gz_phases)
            gz_times.append(time.perf_counter() - t)
        gz_wall = statistics.median(gz_times)
        gz_bytes = sum(q.stat().st_size for q in gz)
        gz_same = gzip_content(out_gz) == gzip_content(out)
        # parity on a sample: the first pairs through both paths at level 0
        ns = 20_000
        s1, s2 = d / "s1.fq", d / "s2.fq"
        s1.write_bytes(fastq_text(rb, ns, 1))
        s2.write_bytes(fastq_text(rb, ns, 2))
        so = d / "s.bam"
        map_fastq_to_bam(None, s1, so, fq2=s2, bs_r1="C2T", bs_r2="G2A", params=params, environ={}, ctx=ctx,
                         index=gi, level=0)
        _sys.path.insert(0, str(ROOT / "tests"))
        import fq2bam_oracle

        t = time.perf_counter()
        want = fq2bam_oracle.fq2bam(args._prefix, s1, s2, params.as_list(), 1, 2, bam_header(gi.contigs, {}),
                                    b"mojo1", 0)
        cpu_s = time.perf_counter() - t
        same = so.read_bytes() == want
        records = 2 * n
        return {
            "metric": "reads/s FASTQ -> sorted, duplicate-marked BAM", "value": round(records / wall, 1),
            "unit": "reads/s", "s_per_run": round(wall, 3), "phases_s": phases,
            "config": {"workload": f"{n} PE 2x{READ_LEN} pairs of the workload as two FASTQ files "
                                   f"({fq_bytes} bytes) -> one BAM file", "bam_bytes": bam_size,
                       "bgzf_level": args.bgzf_level if args.bgzf_level >= 0 else 1, "mapped_records": mapped},
            "e2e": {"value": round(records / wall, 1), "unit": "reads/s", "h2d_bytes_per_step": fq_bytes,
                    "d2h_bytes_per_step": bam_size,
                    "timing": "host wall clock of the whole call: file reads, every GPU stage, the file write"},
            "cpu_baseline": {"value": round(2 * ns / cpu_s, 1), "unit": "reads/s", "cores": os.cpu_count(),
                             "kind": "port", "sample": f"the first {ns} pairs through the oracle pipeline "
                                                       f"(mapping on all cores), {cpu_s:.2f} s"},
            "parity": {"reads": 2 * ns, "bam_file_identical_at_level0": bool(same)},
            "bgzf_input": {"value": round(records / gz_wall, 1), "unit": "reads/s", "s_per_run": round(gz_wall, 3),
                           "phases_s": gz_phases, "input_bytes": gz_bytes,
                           "e2e": {"h2d_bytes_per_step": int(gz_phases.get("fastq_h2d_bytes", gz_bytes)),
                                   "d2h_bytes_per_step": out_gz.stat().st_size},
                           "inflate": "BGZF members copied to the device and inflated there (one warp per member)",
                           "parity": {"bam_content_equals_plain_input": bool(gz_same)}},
        }
    finally:
        shutil.rmtree(d, ignore_errors=True)


def gzip_content(path) -> bytes:
    """The inflated content of a BGZF file, its members inflated on a host
    thread pool (gzip.decompress copies the rest of the buffer for every
    member, quadratic in the member count)."""
    from mojoalign_b200.fqio import BgzfReader

    with BgzfReader(str(path)) as fh:
        return fh.read()


def run_fq2sam_stage(args, ctx, gi, rb, local, params, peaks):
    """FASTQ files of the workload -> SAM text through map_fastq_to_sam (split,
    mapping and SAM lines on the GPU; files read and the text written on the
    host), the SAM emitter's device time inside it, and the same path
    restated on the CPU from the oracle on a sample (mapping dominates)."""
    import shutil
    import sys as _sys

    from mojoalign_b200.fq2sam import map_fastq_to_sam
    from mojoalign_b200.linear_fm import sam_header

    n = min(args.fq2sam_pairs, rb.n1)
    d = Path(tempfile.mkdtemp(prefix="fq2sam_", dir=args.workdir))
    try:
        r1, r2 = d / "r1.fq", d / "r2.fq"
        r1.write_bytes(fastq_text(rb, n, 1))
        r2.write_bytes(fastq_text(rb, n, 2))
        out = d / "out.sam"
        fq_bytes = r1.stat().st_size + r2.stat().st_size
        kw = dict(fq2=r2, bs_r1="C2T", bs_r2="G2A", params=params, environ={}, ctx=ctx, index=gi)
        map_fastq_to_sam(None, r1, out, **kw)
        times, phases = [], {}
        for _ in range(max(1, min(args.steps, 3))):
            ph = {}
            t = time.perf_counter()
            mapped = map_fastq_to_sam(None, r1, out, stats=ph, **kw)
            times.append(time.perf_counter() - t)
            if not phases or ph["emit_kernel_s"] < phases["emit_kernel_s"]:
                phases = ph
        wall = statistics.median(times)
        sam_size = out.stat().st_size
        # the emitter: algorithmic bytes = arena spans read once, 24 B of hit
        # fields and 36 B of span columns per line, the text written once
        emit_s = phases["emit_kernel_s"]
        lines = phases["emit_lines"]
        alg = phases["emit_arena_bytes"] + 60 * lines + phases["emit_text_bytes"]
        achieved = alg / emit_s / 1e9
        # parity + CPU baseline on a sample of the same reads
        ns = 20_000
        t1, t2 = fastq_text(rb, ns, 1), fastq_text(rb, ns, 2)
        s1, s2 = d / "s1.fq", d / "s2.fq"
        s1.write_bytes(t1)
        s2.write_bytes(t2)
        so = d / "s.sam"
        map_fastq_to_sam(None, s1, so, fq2=s2, bs_r1="C2T", bs_r2="G2A", params=params, environ={}, ctx=ctx,
                         index=gi)
        _sys.path.insert(0, str(ROOT / "tests"))
        import fq2sam_oracle

        t = time.perf_counter()
        want, _ = fq2sam_oracle.fq2sam(args._prefix, None, None, params.as_list(), 1, 2,
                                       [c.name for c in gi.contigs], b"mojo1", texts=(t1, t2))
        cpu_s = time.perf_counter() - t
        same = so.read_bytes() == sam_header(gi.contigs, {}).encode() + want
        records = 2 * n
        return {
            "metric": "reads/s FASTQ -> SAM", "value": round(records / wall, 1), "unit": "reads/s",
            "s_per_run": round(wall, 3), "phases_s": phases,
            "config": {"workload": f"{n} PE 2x{READ_LEN} pairs of the workload as two FASTQ files "
                                   f"({fq_bytes} bytes) -> one SAM file", "sam_bytes": sam_size,
                       "mapped_records": mapped},
            "e2e": {"value": round(records / wall, 1), "unit": "reads/s", "h2d_bytes_per_step": fq_bytes,
                    "d2h_bytes_per_step": sam_size,
                    "timing": "host wall clock of the whole call: file reads, every GPU stage, the file write"},
            "emitter": {"lines_per_s": round(lines / emit_s, 1), "ms": round(emit_s * 1e3, 3),
                        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks.get("hbm_gbs"),
                                     "unit": "GB/s", "frac": round(achieved / peaks.get("hbm_gbs"), 4),
                                     "traffic": None, "alg_bytes": alg,
                                     "alg": "name + SEQ + QUAL spans read once, 60 B of hit and span fields per "
                                            "line, the text written once"}},
            "cpu_baseline": {"value": round(2 * ns / cpu_s, 1), "unit": "reads/s", "cores": os.cpu_count(),
                             "kind": "port", "sample": f"the first {ns} pairs through the oracle pipeline "
                                                       f"(mapping on all cores), {cpu_s:.2f} s"},
            "parity": {"reads": 2 * ns, "sam_file_identical": bool(same)},
        }
    finally:
        shutil.rmtree(d, ignore_errors=True)


def run_sort_stage(args, ctx, rb, res, local, peaks):
    """Coordinate sort + duplicate marking + sorted gather of one BAM tile
    made of --sort-batches emitted batches: device-resident throughput, the
    host API end to end, the oracle on one core, and parity."""
    import torch

    import oracle
    from mojoalign_b200 import _lib
    from mojoalign_b200.bam import META_FIELDS, BamTile, emit_bam_device

    bp = min(args.bam_pairs, rb.n1 // max(1, args.sort_batches))
    nb = args.sort_batches
    n = 2 * bp * nb
    dev = torch.device("cuda", local)
    tids = np.arange(16, dtype=np.int32) // 2
    d_tids = device_copy(tids, dev)
    d_rg = device_copy(np.frombuffer(BAM_RG, np.uint8), dev)
    d_meta = {k: torch.empty(n, dtype=torch.int64 if t_ == np.uint64 else torch.int32, device=dev)
              for k, t_ in META_FIELDS}
    d_status = torch.zeros(3, dtype=torch.int64, device=dev)
    tile = BamTile(meta_cap=n, host_meta=False)
    chunks, chunk_len = [], []
    rec_cap = 4 + 32 + BAM_NAME_LEN + 1 + 12 + (READ_LEN + 1) // 2 + READ_LEN + 8 + len(BAM_RG)
    for c in range(nb):
        hits, arena = bam_batch(rb, res, bp, first=c * bp)
        d_hits = {k: device_copy(v, dev) for k, v in hits.items()}
        d_arena = {k: device_copy(getattr(arena, k), dev)
                   for k in ("data", "name_off", "name_len", "orig_off", "orig_len", "qual_off", "qual_len")}
        d_chunk = torch.empty(2 * bp * rec_cap, dtype=torch.uint8, device=dev)
        tile.n_reads, tile.chunk = 2 * bp * c, c
        torch.cuda.synchronize()
        emit_bam_device(ctx, {k: v.data_ptr() for k, v in d_hits.items()}, bp, True,
                        {k: v.data_ptr() for k, v in d_arena.items()}, int(arena.data.size), d_tids.data_ptr(),
                        int(tids.size), d_rg.data_ptr(), len(BAM_RG), d_chunk.data_ptr(), d_chunk.numel(),
                        {k: v.data_ptr() for k, v in d_meta.items()}, tile, d_status.data_ptr())
        torch.cuda.synchronize()
        st = d_status.cpu().numpy()
        assert st[0] <= d_chunk.numel() and st[2] == 0
        chunks.append(d_chunk)
        chunk_len.append(int(st[0]))
        del d_hits, d_arena
    meta = {k: d_meta[k].cpu().numpy().view(t_) for k, t_ in META_FIELDS}
    d_chunk_ptrs = device_copy(np.array([c.data_ptr() for c in chunks], np.uint64), dev)
    d_chunk_len = device_copy(np.array(chunk_len, np.uint64), dev)
    total = int(sum(chunk_len))
    d_out = {k: torch.empty(n, dtype=torch.int32, device=dev) for k in ("is_dup", "perm")}
    d_marked = torch.zeros(1, dtype=torch.int64, device=dev)
    d_sorted = torch.empty(total, dtype=torch.uint8, device=dev)
    d_gstat = torch.zeros(2, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    stream = torch.cuda.Stream(device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]

    def step(timed=False):
        if timed:
            ev[0].record(stream)
        _lib.check(_lib.lib.ma_sort_markdup_device(
            ctx.handle, n, d_meta["coord"].data_ptr(), d_meta["dhi"].data_ptr(), d_meta["dlo"].data_ptr(),
            d_meta["score"].data_ptr(), d_meta["pair"].data_ptr(), d_out["is_dup"].data_ptr(),
            d_out["perm"].data_ptr(), 1, None, d_marked.data_ptr(), stream.cuda_stream), ctx.handle)
        sort_launches = ctx.last_launch_count()
        if timed:
            ev[1].record(stream)
        _lib.check(_lib.lib.ma_gather_sorted_bam_device(
            ctx.handle, n, d_out["perm"].data_ptr(), d_meta["rec"].data_ptr(), d_meta["len"].data_ptr(),
            d_out["is_dup"].data_ptr(), 1, d_chunk_ptrs.data_ptr(), d_chunk_len.data_ptr(), nb,
            d_sorted.data_ptr(), total, d_gstat.data_ptr(), stream.cuda_stream), ctx.handle)
        if timed:
            ev[2].record(stream)
        return sort_launches + ctx.last_launch_count()

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    sort_ms, gather_ms = [], []
    launches = 0
    for _ in range(args.steps):
        launches += step(timed=True)
        stream.synchronize()
        sort_ms.append(ev[0].elapsed_time(ev[1]))
        gather_ms.append(ev[1].elapsed_time(ev[2]))
    g_is_dup = d_out["is_dup"].cpu().numpy().view(np.uint32)
    g_perm = d_out["perm"].cpu().numpy().view(np.uint32)
    g_sorted = d_sorted.cpu().numpy()
    gst = d_gstat.cpu().numpy()
    host_chunks = [c[:l].cpu().numpy() for c, l in zip(chunks, chunk_len)]
    del chunks, d_sorted
    # the oracle (one core) on the same tile: CPU baseline and parity
    t = time.perf_counter()
    w_dup, w_perm, _, w_marked = oracle.sort_markdup(meta["coord"], meta["dhi"], meta["dlo"], meta["score"],
                                                     meta["pair"], dup_perm=False)
    w_sorted = oracle.gather_sorted(host_chunks, w_perm, meta["rec"], meta["len"], w_dup)
    cpu_s = time.perf_counter() - t
    same = (np.array_equal(g_perm, w_perm) and np.array_equal(g_is_dup, w_dup) and int(gst[0]) == total
            and g_sorted.tobytes() == w_sorted and int(d_marked.item()) == w_marked)
    del w_sorted
    # end to end through the host API: pinned metadata and chunks in, perm /
    # flags / sorted stream out
    from mojoalign_b200.bam import gather_sorted, sort_markdup

    pin_meta = {k: torch.from_numpy(v.view(np.int64 if v.dtype == np.uint64 else np.int32)).pin_memory().numpy()
                .view(v.dtype) for k, v in meta.items()}
    pin_chunks = [torch.from_numpy(c).pin_memory().numpy() for c in host_chunks]
    host_tile = BamTile(meta_cap=n, n_reads=n, meta=pin_meta)
    pin_out = torch.empty(total, dtype=torch.uint8, pin_memory=True).numpy()
    res_ = sort_markdup(ctx, host_tile)
    gather_sorted(ctx, pin_chunks, host_tile, res_, out=pin_out)
    t = time.perf_counter()
    for _ in range(args.steps):
        res_ = sort_markdup(ctx, host_tile)
        out = gather_sorted(ctx, pin_chunks, host_tile, res_, out=pin_out)
    e2e_s = (time.perf_counter() - t) / args.steps
    same = same and np.array_equal(res_.perm, w_perm) and len(out) == total
    args._sorted_stream = g_sorted
    ms = statistics.mean(sort_ms) + statistics.mean(gather_ms)
    sort_alg = n * (3 * 8 + 2 * 4 + 2 * 4)
    gather_alg = 2 * total + n * (4 + 8 + 4 + 4)
    s_ach = sort_alg / (statistics.mean(sort_ms) / 1000.0) / 1e9
    g_ach = gather_alg / (statistics.mean(gather_ms) / 1000.0) / 1e9
    return {
        "metric": "records/s sort+markdup+gather", "value": round(n / (ms / 1000.0), 1), "unit": "records/s",
        "ms_per_tile": round(ms, 3), "sort_markdup_ms": round(statistics.mean(sort_ms), 3),
        "gather_ms": round(statistics.mean(gather_ms), 3),
        "config": {"workload": f"one BAM tile of {nb} emitted batches x {bp} PE 2x{READ_LEN} pairs of the mapped "
                               f"workload", "records": n, "bam_bytes": total, "duplicates_marked": int(w_marked)},
        "e2e": {"value": round(n / e2e_s, 1), "unit": "records/s",
                "h2d_bytes_per_step": int(n * 32 + total + n * 24), "d2h_bytes_per_step": int(n * 8 + total)},
        "roofline": {"bound": "hbm", "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                     "sort_markdup": {"achieved": round(s_ach, 1), "frac": round(s_ach / peaks.get("hbm_gbs"), 4),
                                      "alg_bytes_per_launch": sort_alg,
                                      "alg": "read coord/dhi/dlo (8 B each) + score/pair (4 B each), write perm "
                                             "and is_dup (4 B each)"},
                     "gather": {"achieved": round(g_ach, 1), "frac": round(g_ach / peaks.get("hbm_gbs"), 4),
                                "alg_bytes_per_launch": gather_alg,
                                "alg": "read and write every record byte once + perm/rec/len/is_dup per record"},
                     "traffic": None},
        "gpu_launches": launches,
        "cpu_baseline": {"value": round(n / cpu_s, 1), "unit": "records/s", "cores": 1, "kind": "port",
                         "sample": f"the whole tile ({n} records), {cpu_s:.2f} s"},
        "parity": {"records": n, "perm_flags_and_stream_identical": bool(same)},
    }


def workload_config(args) -> dict:
    """The `config` block: the workload only, the same in both arms."""
    return {"workload": f"plain single-launch, {args.genome_mb} Mbp synthetic bisulfite reference "
                        f"(bwa-meth c2t index), {args.pairs} PE 2x{READ_LEN} read pairs per GPU",
            "form": "plain single-launch", "genome_bp": args.genome_mb * 1_000_000,
            "reads_per_gpu": 2 * args.pairs, "read_len": READ_LEN, "paired": True,
            "params": dict(BENCH_PARAM_VALUES),
            "l2": "inputs larger than L2 (reads and index several GB)"}


LINE_HEAD = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
             "vs_baseline", "dtype", "data", "impl", "parity_failures", "parity_sample", "config", "e2e",
             "gpu_launches", "cpu_baseline")


def ordered_line(line: dict) -> dict:
    """The JSON line with the contract keys and the parity record first, so
    that a reader that keeps only the head of the line still sees them."""
    out = {k: line[k] for k in LINE_HEAD if k in line}
    out.update(line)
    return out


def parity_failures(obj, path="") -> list:
    """Every parity check of the line that failed: a sample with mismatched
    fields, a `parity` record with a false flag, a form not equal to plain."""
    bad = []
    if isinstance(obj, dict):
        for k, v in obj.items():
            here = f"{path}.{k}" if path else k
            if k == "mismatched_fields" and isinstance(v, int) and v > 0:
                bad.append(f"{here}={v}")
            elif k == "equals_plain" and v is False:
                bad.append(here)
            elif path.endswith("parity") and v is False:
                bad.append(here)
            else:
                bad += parity_failures(v, here)
    return bad


def seeding_roofline(tally, wave, tally2=None, n_seq=0, seed_kernel=2) -> dict:
    """The seeding kernel alone (wavefront search: k-mer table, Occ and SA
    gathers) from the counting pass's tallies (the rounds' part: the
    stage-2 warps' tallies, tally2, taken out) and the per-round search
    times; the stage-2 warps reported beside it."""
    if not wave or not any(w[0] for w in wave):
        return {}
    tally2 = tally2 or [0] * 12
    search_ms = statistics.mean(w[0] for w in wave)
    seed_bytes = 32 * sum(tally[i] - tally2[i] for i in range(3))
    name = "wf_search_refill_kernel" if seed_kernel == 3 else "wf_search_kernel"
    out = {"seeding": {"kernel": f"{name} (all rounds)", "ms": round(search_ms, 3),
                       "eval_ms": round(statistics.mean(w[1] for w in wave), 3),
                       "finalize_ms": round(statistics.mean(w[2] for w in wave), 3),
                       "alg_bytes": int(seed_bytes),
                       "alg": "32-B sectors of the Occ lines, k-mer table entries and SA entries the rounds' "
                              "search gathers (this implementation's accesses)",
                       "achieved_GBs": round(seed_bytes / (search_ms / 1000) / 1e9, 1)}}
    if len(wave[0]) > 4:
        out["seeding"]["stage2_ms"] = round(statistics.mean(w[4] for w in wave), 3)
        if n_seq:
            out["seeding"]["stage2_reads_per_read"] = round(tally2[9] / n_seq, 4)
    return out


def add_gather_fractions(line) -> None:
    """Fractions of the measured random-gather rooflines for the seeding
    figure (32- and 64-byte lines)."""
    sd = line["roofline"].get("seeding")
    g = line.get("gather_roofline") or {}
    if sd and g:
        sd["frac_of_gather32"] = round(sd["achieved_GBs"] / g["hbm_32B_GBs"], 4)
        sd["frac_of_gather64"] = round(sd["achieved_GBs"] / g["hbm_64B_GBs"], 4)


def reference_algorithm_bytes(line, ix, bases, lens, n1, paired, max_len, params, n_seq, bs2=2) -> None:
    """Bytes the reference algorithm moves per read, from the oracle's
    counters on (up to 100 k pairs of) the given reads: 64-B BWT lines per
    backward step and per LF-walk step, 8-B SA samples, 32-B pac sectors,
    packed reads in, 28 B of outputs; and as GB/s over the seed kernels'
    and the search kernel's times for the whole call."""
    k = min(n1, 100_000)
    if paired:
        b = np.concatenate([bases[:k], bases[n1:n1 + k]])
        l_ = np.concatenate([lens[:k], lens[n1:n1 + k]])
    else:
        b, l_ = bases[:k], lens[:k]
    ct = ix.map(b, l_, k, paired, max_len, 1, bs2, params.as_list(), counters=True)["counters"]
    nr = int(l_.size)
    seed_ref = 64 * (ct["occ_lines"] + ct["lf_lines"]) + 8 * ct["sa_loads"]
    total = seed_ref + 32 * ct["pac_sectors"] + int(((l_.astype(np.int64) + 3) // 4).sum()) + 28 * nr
    r = line["roofline"]
    r["reference_algorithm"] = {
        "bytes_per_read": round(total / nr, 1), "seeding_bytes_per_read": round(seed_ref / nr, 1),
        "source": f"oracle counters (orc_counters) on {nr} reads of the workload",
        "oracle_capped_searches_per_read": round(ct["capped"] / nr, 4),
        "oracle_fallback_seeds_per_read": round(ct["fallback"] / nr, 4),
        "GBs_over_seed_kernels": round(total / nr * n_seq / (r["kernel_ms"] / 1000) / 1e9, 1)}
    if r.get("seeding"):
        r["reference_algorithm"]["seeding_GBs_over_search_kernel"] = round(
            seed_ref / nr * n_seq / (r["seeding"]["ms"] / 1000) / 1e9, 1)


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "_fallback": True}


def run_ours(args, rank, world, local):
    import torch

    torch.cuda.set_device(local)
    dist = Dist(world, "nccl")
    from mojoalign_b200 import BENCH_PARAMS, GpuContext, GpuIndex, MapResult, map_batch, map_batch_device
    from mojoalign_b200 import _lib

    params = BENCH_PARAMS
    assert dict(zip(BENCH_PARAM_VALUES, params.as_list())) == BENCH_PARAM_VALUES
    fa, prefix, prep_s = prepare_reference(args, rank, dist, local)
    n_seq = 2 * args.pairs
    pinned = torch.empty((n_seq, READ_LEN), dtype=torch.uint8, pin_memory=True)
    t = time.time()
    log("reads")
    rb = simulate(args, fa, rank, bases_out=pinned.numpy())
    sim_s = time.time() - t
    lens_pinned = torch.from_numpy(rb.lens.view(np.int32)).pin_memory()

    ctx = GpuContext(local)
    t = time.time()
    log("index open")
    gi = GpuIndex(ctx, prefix, kmer_k=args.kmer, kmer3_k=args.kmer3, at_k=args.at_k,
                  at_seed_len=params.seed_len if args.at_k else 0)
    open_s = time.time() - t
    log("autotune")

    # ---- result-neutral kernel choices picked on a sample of the batch ----
    from mojoalign_b200.autotune import autotune

    ns = min(args.pairs, 1_000_000)
    tb = np.concatenate([rb.bases[:ns], rb.bases[args.pairs:args.pairs + ns]])
    tl = np.concatenate([rb.lens[:ns], rb.lens[args.pairs:args.pairs + ns]])
    if args.tuning:
        from mojoalign_b200.autotune import FIELDS, TuneResult

        fixed = [int(x) for x in args.tuning.split(",")]
        fixed += [2, 1, 0, 2, 1, 1, 8, 4, 0, 1][len(fixed):]
        ctx.set_tuning(*fixed)
        tune = TuneResult(dict(zip(FIELDS, fixed)), float("nan"), [])
        ns = 0
    else:
        # the sample as one device-resident call, like the timed steps
        dev = f"cuda:{local}"
        d_tb = torch.from_numpy(tb).to(dev).reshape(-1)
        d_tl = torch.from_numpy(tl.view(np.int32)).to(dev)
        t_out = {f: torch.empty(2 * ns, dtype=torch.int32, device=dev) for f in MapResult.FIELDS}
        t_dbg = {f: torch.empty(2 * ns, dtype=torch.int64 if f in ("uk", "ul") else torch.int32, device=dev)
                 for f in MapResult.DEBUG}

        def run_sample():
            map_batch_device(ctx, gi, d_tb.data_ptr(), d_tl.data_ptr(), ns, True, READ_LEN,
                             {f: x.data_ptr() for f, x in t_out.items()}, "C2T", "G2A", params,
                             d_debug={f: x.data_ptr() for f, x in t_dbg.items()},
                             stream=torch.cuda.current_stream().cuda_stream)
            outs = {f: x.cpu().numpy() for f, x in list(t_out.items()) + list(t_dbg.items())}
            return outs, ctx.kernel_ms()[1]

        tune = autotune(ctx, gi, tb, tl, ns, True, READ_LEN, "C2T", "G2A", params, run=run_sample)
        del d_tb, d_tl, t_out, t_dbg
    del tb, tl

    # ---- device-resident inputs and outputs ----
    d_bases = pinned.to(f"cuda:{local}").reshape(-1)
    d_lens = lens_pinned.to(f"cuda:{local}")
    d_out = {f: torch.empty(n_seq, dtype=torch.int32, device=f"cuda:{local}") for f in MapResult.FIELDS}
    out_ptrs = {f: t_.data_ptr() for f, t_ in d_out.items()}
    stream = torch.cuda.Stream()  # the calls launch on the stream they are given: time them there
    torch.cuda.set_stream(stream)

    def step():
        map_batch_device(ctx, gi, d_bases.data_ptr(), d_lens.data_ptr(), args.pairs, True, READ_LEN, out_ptrs,
                         "C2T", "G2A", params, stream=stream.cuda_stream)

    log(f"tuning {tune.tuning}; counting pass")
    # traffic accounting: one untimed pass of the counting kernel
    _lib.check(_lib.lib.ma_ctx_set_profiling(ctx.handle, 2), ctx.handle)
    step()
    tally = (_lib.C.c_uint64 * 12)()
    _lib.lib.ma_ctx_traffic(ctx.handle, tally)
    tally = list(tally)
    tally2 = ctx.traffic_stage2()
    _lib.check(_lib.lib.ma_ctx_set_profiling(ctx.handle, 1), ctx.handle)

    log("timed steps")
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    seed_ms, stage1_ms, other_ms = [], [], []
    kms = (_lib.C.c_float * 4)()
    torch.cuda.synchronize()
    profiled_region(True)
    ev0.record(stream)
    wave = []
    for _ in range(args.steps):
        step()
        _lib.lib.ma_ctx_kernel_ms(ctx.handle, kms)
        seed_ms.append(float(kms[1]))
        stage1_ms.append(float(kms[3]))
        other_ms.append((float(kms[0]), float(kms[2])))
        wave.append(ctx.wave_ms())
    ev1.record(stream)
    torch.cuda.synchronize()
    profiled_region(False)
    ms = ev0.elapsed_time(ev1) / args.steps
    clk = clocks.stop()
    dist.barrier()
    launches = ctx.last_launch_count() * args.steps
    ms_max = dist.max(ms)
    value = aggregate_reads_per_s(n_seq, world, ms_max)

    log("end to end")
    # ---- end to end through the host API (pinned host in, host out) ----
    _lib.check(_lib.lib.ma_ctx_set_profiling(ctx.handle, 0), ctx.handle)  # per-chunk timing would serialise
    from mojoalign_b200.mapper import page_locked

    res = MapResult.empty(n_seq, debug=False, pinned=True)
    bases_np = pinned.numpy()
    lens_np = page_locked(n_seq, np.uint32)
    lens_np[:] = rb.lens
    map_batch(ctx, gi, bases_np, lens_np, args.pairs, True, READ_LEN, "C2T", "G2A", params, out=res)
    dist.barrier()
    t = time.perf_counter()
    for _ in range(args.steps):
        map_batch(ctx, gi, bases_np, lens_np, args.pairs, True, READ_LEN, "C2T", "G2A", params, out=res)
    e2e_s = dist.max((time.perf_counter() - t) / args.steps)
    e2e_value = aggregate_reads_per_s(n_seq, world, e2e_s * 1000.0)
    mapped = float((res.rid >= 0).mean())

    # ---- roofline of the dominant kernel (seed/extend) ----
    peaks = measured_peaks()
    words = (READ_LEN + 31) // 32
    alg_bytes = 32 * (tally[0] + tally[1] + tally[2] + tally[3]) + n_seq * (4 * words * 8 + 4) + n_seq * 28
    seed_avg_ms = statistics.mean(seed_ms)
    achieved = alg_bytes / (seed_avg_ms / 1000.0) / 1e9
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
            "frac": round(achieved / peaks.get("hbm_gbs"), 4),
            "traffic": None,
            "traffic_source": "not captured for this workload; the genome workload's line carries the measured "
                              "DRAM bytes",
            "peak_source": "fallback" if peaks.get("_fallback") else "measured (MEASURED_PEAKS.json hbm_gbs)",
            "kernel": SEED_KERNELS.get(tune.tuning.get("seed_kernel", 1), "seed/extend"),
            "kernel_ms": round(seed_avg_ms, 3), "stage1_ms": round(statistics.mean(stage1_ms), 3),
            "pack_ms": round(statistics.mean(x[0] for x in other_ms), 3),
            "rescue_ms": round(statistics.mean(x[1] for x in other_ms), 3),
            "alg_bytes_per_launch": int(alg_bytes),
            "tally_per_read": {k: round(v / n_seq, 3) for k, v in zip(
                ["occ_lines_32B", "kmer_loads", "sa_loads", "pac_sectors_32B", "backward_steps", "endpoints",
                 "loci_evaluated", "read_words", "endpoints_skipped", "stage2_reads", "stage2_groups",
                 "shift_evals"], tally)}}
    roof.update(seeding_roofline(tally, wave, tally2, n_seq, tune.tuning.get("seed_kernel", 2)))
    line = {"metric": METRIC, "value": round(value, 1), "unit": "reads/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": workload_config(args),
            "run": {"tuning": tune.tuning, "autotune_sample_reads": 2 * ns, "kmer_k": args.kmer,
                    "kmer3_k": args.kmer3, "at_k": args.at_k, "index_hbm_bytes": int(gi.info.device_bytes),
                    "mapped_frac": round(mapped, 4)},
            "e2e": {"value": round(e2e_value, 1), "unit": "reads/s",
                    "h2d_bytes_per_step": int(n_seq * READ_LEN + n_seq * 4),
                    "d2h_bytes_per_step": int(n_seq * 28)},
            "gpu_launches": launches, "roofline": roof, "clocks": clk,
            "setup_s": {"reference_and_index": round(prep_s, 1), "reads": round(sim_s, 1),
                        "index_open": round(open_s, 1)}}
    line["autotune"] = tune.all_ms
    if rank == 0:
        line["gather_roofline"] = {}
        for lb in (32, 64):
            g = _lib.C.c_double()
            _lib.check(_lib.lib.ma_bench_gather(ctx.handle, 8 << 30, lb, 1 << 30, _lib.C.byref(g)), ctx.handle)
            line["gather_roofline"][f"hbm_{lb}B_GBs"] = round(g.value, 1)
        g = _lib.C.c_double()
        _lib.check(_lib.lib.ma_bench_gather(ctx.handle, 64 << 20, 32, 1 << 30, _lib.C.byref(g)), ctx.handle)
        line["gather_roofline"]["l2_32B_GBs"] = round(g.value, 1)
        line["roofline"]["frac_of_gather32"] = round(achieved / line["gather_roofline"]["hbm_32B_GBs"], 4)
        add_gather_fractions(line)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        log("oracle sample")
        ix, o, n, rate, dt = time_oracle(prefix, rb, params, args.cpu_seconds)
        import oracle

        line["cpu_baseline"] = {"value": round(rate, 1), "unit": "reads/s", "cores": oracle.max_threads(),
                                "kind": "port", "sample": f"first {n} pairs ({2 * n} reads) of the GPU workload, "
                                                          f"{dt:.1f} s", "cpu": _cpu_model()}
        # full-size parity: the GPU's outputs for those reads against the oracle
        bad = 0
        for f in MapResult.FIELDS:
            g = getattr(res, f)
            g = np.concatenate([g[:n], g[args.pairs:args.pairs + n]])
            bad += int((g != o[f]).sum())
        line["parity_sample"] = {"reads": 2 * n, "mismatched_fields": bad}
        reference_algorithm_bytes(line, ix, rb.bases, rb.lens, rb.n1, True, READ_LEN, params, n_seq)
    if rank == 0 and world == 1:
        stages = stage_block(args, ctx, gi, rb, res, prefix, local, peaks, params)
        if stages:
            line["stages"] = stages
    if rank == 0 and world == 1 and not args.no_forms:
        from mojoalign_b200.autotune import FIELDS as TFIELDS

        best = tuple(tune.tuning[f] for f in TFIELDS if f in tune.tuning)
        del d_bases, d_lens, d_out
        torch.cuda.empty_cache()
        log("forms")
        line["forms"] = run_forms(args, ctx, gi, params, fa, local, best)
    bad = parity_failures(line)
    line["parity_failures"] = bad
    if rank == 0:
        print(json.dumps(ordered_line(line)), flush=True)
    gi.close()
    ctx.close()
    dist.close()
    if bad:
        sys.stderr.write("parity check failed: " + ", ".join(bad) + "\n")
        sys.exit(3)


def stage_block(args, ctx, gi, rb, res, prefix, local, peaks, params) -> dict:
    """The stages either side of the mapping kernels (BAM records, sort +
    duplicate marking + gather, BGZF, FASTQ -> BAM, FASTQ -> SAM, FASTQ
    split) on the pairs `rb` and their mapping outputs `res`."""
    import torch

    stages = {}
    if args.bam_pairs > 0:
        log("stage: BAM pack")
        stages["bam_pack"] = run_bam_stage(args, ctx, rb, res, local, peaks)
        if args.sort_batches > 0:
            torch.cuda.empty_cache()
            log("stage: sort")
            stages["sort_markdup_gather"] = run_sort_stage(args, ctx, rb, res, local, peaks)
            if args.bgzf_level >= 0 and getattr(args, "_sorted_stream", None) is not None:
                torch.cuda.empty_cache()
                log("stage: BGZF")
                stages["bgzf"] = run_bgzf_stage(args, ctx, args._sorted_stream, local, peaks)
                del args._sorted_stream
    args._prefix = prefix
    if args.fq2bam_pairs > 0:
        torch.cuda.empty_cache()
        log("stage: FASTQ -> BAM")
        stages["fq2bam"] = run_fq2bam_stage(args, ctx, gi, rb, local, params)
    if args.fq2sam_pairs > 0:
        torch.cuda.empty_cache()
        log("stage: FASTQ -> SAM")
        stages["fq2sam"] = run_fq2sam_stage(args, ctx, gi, rb, local, params, peaks)
    if args.fastq_pairs > 0:
        torch.cuda.empty_cache()
        log("stage: FASTQ split")
        stages["fastq_split"] = run_fastq_stage(args, ctx, rb, local, peaks)
    return stages


def chromosome_stages(args, local, params, peaks) -> dict:
    """The file stages measured beside a genome workload: the chromosome
    workload's reference (args.genome_mb, 250 Mbp by default) and index,
    and as many of its 2x150 pairs as the stages use, mapped first."""
    import torch
    from mojoalign_b200 import GpuContext, GpuIndex, MapResult, map_batch

    class _Solo(Dist):
        def __init__(self):
            super().__init__(1, "gloo")

    fa, prefix, _ = prepare_reference(args, 0, _Solo(), local)
    pairs = max(args.bam_pairs * max(1, args.sort_batches), args.fq2bam_pairs, args.fq2sam_pairs,
                args.fastq_pairs, 1)
    sub = argparse.Namespace(**vars(args))
    sub.pairs = pairs
    log(f"stages: {pairs} pairs on the {args.genome_mb} Mbp reference")
    rb = simulate(sub, fa, 0)
    ctx = GpuContext(local)
    gi = GpuIndex(ctx, prefix, kmer_k=args.kmer, kmer3_k=args.kmer3, at_k=args.at_k,
                  at_seed_len=params.seed_len if args.at_k else 0)
    res = MapResult.empty(rb.n_seq, debug=False)
    map_batch(ctx, gi, rb.bases, rb.lens, rb.n1, True, READ_LEN, "C2T", "G2A", params, out=res)
    try:
        out = stage_block(args, ctx, gi, rb, res, prefix, local, peaks, params)
        out["reference"] = f"{args.genome_mb} Mbp synthetic bisulfite reference, {pairs} PE 2x{READ_LEN} pairs"
        return out
    finally:
        gi.close()
        ctx.close()
        torch.cuda.empty_cache()


UNEVEN_MODEL = dict(len_fixed=0, len_lognorm_median=120.0, len_lognorm_sigma=0.35, len_min=36, len_max=300,
                    non_directional=0.5)
UNEVEN_MAX = 300


def serving_samples():
    """Eight simulated samples: CpG retention 0.4-0.9 and three length
    profiles (fixed 150; lognormal median 120 in 36-300; lognormal median 90,
    sigma 0.5, in 36-250), mixed directional / non-directional."""
    out = []
    for k in range(8):
        prof = k % 3
        m = dict(cpg_retain=0.4 + 0.5 * k / 7, non_directional=0.25 * (k % 2))
        if prof == 0:
            m.update(len_fixed=150)
            ml = 150
        elif prof == 1:
            m.update(len_fixed=0, len_lognorm_median=120.0, len_lognorm_sigma=0.35, len_min=36, len_max=300)
            ml = 300
        else:
            m.update(len_fixed=0, len_lognorm_median=90.0, len_lognorm_sigma=0.5, len_min=36, len_max=250)
            ml = 250
        out.append((m, ml))
    return out


def sample_pools(args, fa) -> list:
    """The 8 simulated samples' read pools (pinned host rows), simulated on
    8 host threads at once (each simulation reads the reference itself)."""
    import concurrent.futures as cf

    import torch
    from mojoalign_b200 import synth

    specs = serving_samples()
    bufs = [torch.empty((args.serve_pool, ml), dtype=torch.uint8, pin_memory=True) for _, ml in specs]

    def one(k):
        m, ml = specs[k]
        r = synth.simulate_reads(fa, synth.ReadModel(**m), args.serve_pool, False, ml, seed=200 + k,
                                 bases_out=bufs[k].numpy())
        return (bufs[k], bufs[k].numpy(), r.lens, ml)

    with cf.ThreadPoolExecutor(max_workers=len(specs)) as ex:
        return list(ex.map(one, range(len(specs))))


def log_uniform_sizes(rng, n, lo, hi):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.int64)


def run_forms(args, ctx, gi, params, fa, local, best_tuning):
    """Plain single-launch vs batched vs served on uneven-length reads.

    - plain_1launch: the reference's launch shape (one thread per read over
      every right endpoint, seed_kernel 0), one launch over all reads, inputs
      resident in HBM (device time);
    - plain_reference_batches: the same kernel through ma_map_batch in the
      reference's fixed 16384-read batches, one synchronous call per batch
      (host time, copies included);
    - batched: the autotuned two-stage persistent kernel (work queue), one
      call over all reads, inputs resident (device time);
    - served: the request loop (ma_serve_*), host buffers, copies included:
      saturation throughput over a burst of requests from 8 samples
      (log-uniform 1k-2M reads), then p50/p99/p99.9 request latency under
      Poisson arrivals at half that throughput.
    Every form's outputs for the uneven batch are compared with plain's.
    """
    import torch
    from mojoalign_b200 import MapResult, map_batch, map_batch_device, synth
    from mojoalign_b200.serve import Server, percentiles

    n = args.forms_reads
    dev = f"cuda:{local}"
    pinned = torch.empty((n, UNEVEN_MAX), dtype=torch.uint8, pin_memory=True)
    rb = synth.simulate_reads(fa, synth.ReadModel(**UNEVEN_MODEL), n, False, UNEVEN_MAX, seed=101,
                              bases_out=pinned.numpy())
    bases_np, lens_np = pinned.numpy(), rb.lens
    d_bases = pinned.to(dev).reshape(-1)
    d_lens = torch.from_numpy(lens_np.view(np.int32)).to(dev)
    stream = torch.cuda.Stream()  # the calls launch on the stream they are given: time them there
    torch.cuda.set_stream(stream)
    forms = {"workload": f"{n} single-end reads, lengths lognormal (median 120, sigma 0.35) clipped to 36-300, "
                         f"half non-directional, on the {args.genome_mb} Mbp index",
             "mean_len": round(float(lens_np.mean()), 1)}

    def device_form(tuning, reps=3):
        ctx.set_tuning(*tuning)
        d_out = {f: torch.empty(n, dtype=torch.int32, device=dev) for f in MapResult.FIELDS}
        ptrs = {f: t.data_ptr() for f, t in d_out.items()}

        def go():
            map_batch_device(ctx, gi, d_bases.data_ptr(), d_lens.data_ptr(), n, False, UNEVEN_MAX, ptrs, "C2T", "",
                             params, stream=stream.cuda_stream)
        go()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            go()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        return n / (ms / 1000.0), {f: t.cpu().numpy().view(np.uint32) for f, t in d_out.items()}

    plain_tuning = (0, 1, 0, 1, 16, 32, 32, 4, 0, 0)
    plain_rate, plain_out = device_form(plain_tuning)
    batched_rate, batched_out = device_form(best_tuning)
    same = all(np.array_equal(plain_out[f], batched_out[f]) for f in MapResult.FIELDS)
    forms["mapped_frac"] = round(float((plain_out["rid"].view(np.int32) >= 0).mean()), 4)
    forms["plain_1launch"] = {"reads_per_s": round(plain_rate, 1), "tuning": "seed_kernel 0 (thread per read)",
                              "timing": "device, inputs resident"}
    from mojoalign_b200.autotune import FIELDS as TFIELDS

    forms["batched"] = {"reads_per_s": round(batched_rate, 1), "tuning": dict(zip(TFIELDS, best_tuning)),
                        "timing": "device, inputs resident", "equals_plain": same}

    # the reference's loop: 16384-read synchronous batches of the same kernel
    ctx.set_tuning(*plain_tuning)
    res = MapResult.empty(n, debug=False)
    nb = min(n, args.forms_ref_batches * 16384)
    t = time.perf_counter()
    for a in range(0, nb, 16384):
        c = min(16384, nb - a)
        sub = MapResult(*[getattr(res, f)[a:a + c] for f in MapResult.FIELDS])
        map_batch(ctx, gi, bases_np[a:a + c], lens_np[a:a + c], c, False, UNEVEN_MAX, "C2T", "", params, out=sub)
    ref_rate = nb / (time.perf_counter() - t)
    forms["plain_reference_batches"] = {"reads_per_s": round(ref_rate, 1), "reads": nb, "batch": 16384,
                                        "timing": "host, pinned host buffers, copies included",
                                        "equals_plain": all(np.array_equal(getattr(res, f)[:nb].view(np.uint32), plain_out[f][:nb])
                                                            for f in MapResult.FIELDS)}
    ctx.set_tuning(*best_tuning)

    # ---- served ----
    rng = np.random.default_rng(7)
    budget = args.serve_budget_gb << 30
    with Server(ctx, gi, hbm_budget_bytes=budget, max_group_pairs=args.serve_group, max_inflight=3) as srv:
        # the uneven batch itself as a request stream: equality with plain
        sizes = log_uniform_sizes(rng, 4096, 1000, 2_000_000)
        cuts, a = [], 0
        for sz in sizes:
            if a >= n:
                break
            cuts.append((a, int(min(sz, n - a))))
            a += cuts[-1][1]
        def stream_uneven():
            t0 = time.perf_counter()
            ts = [srv.submit(bases_np[a:a + c], lens_np[a:a + c], c, False, UNEVEN_MAX, "C2T", "", params)
                  for a, c in cuts]
            srv.drain()
            return ts, n / (time.perf_counter() - t0)

        stream_uneven()  # warm-up
        tickets, same_reads_rate = stream_uneven()
        served_same = all(np.array_equal(getattr(t_.result, f).view(np.uint32), plain_out[f][a:a + c])
                          for t_, (a, c) in zip(tickets, cuts) for f in MapResult.FIELDS)
        del tickets

        # 8 samples, each a pool of reads; requests are slices of a pool
        pools = sample_pools(args, fa)

        def request(k, size):
            _, b, l, ml = pools[k]
            size = int(min(size, args.serve_pool))
            a = int(rng.integers(0, args.serve_pool - size + 1))
            return b[a:a + size], l[a:a + size], size, ml

        def burst(count):
            reqs = [request(int(rng.integers(0, 8)), s) for s in log_uniform_sizes(rng, count, 1000, 2_000_000)]
            t0 = time.perf_counter()
            for b, l, c, ml in reqs:
                srv.submit(b, l, c, False, ml, "C2T", "", params)
            srv.drain()
            return sum(r[2] for r in reqs) / (time.perf_counter() - t0)

        burst(16)  # warm-up
        g0 = srv.stats()
        sat = burst(args.serve_burst)
        g1 = srv.stats()
        # Poisson arrivals at half the saturation rate
        mean_size = (2_000_000 - 1000) / np.log(2_000_000 / 1000)
        lam = 0.5 * sat / mean_size
        _, _, before = srv.latencies()
        n0 = before.size
        t0 = time.perf_counter()
        t_next = t0
        sent = 0
        while t_next - t0 < args.serve_seconds:
            now = time.perf_counter()
            if now < t_next:
                time.sleep(t_next - now)
            b, l, c, ml = request(int(rng.integers(0, 8)), log_uniform_sizes(rng, 1, 1000, 2_000_000)[0])
            srv.submit(b, l, c, False, ml, "C2T", "", params)
            sent += c
            t_next += rng.exponential(1.0 / lam)
        srv.drain()
        wall = time.perf_counter() - t0
        _, reads, ms = srv.latencies()
        ms, reads = ms[n0:], reads[n0:]
        st = srv.stats()
    small = ms[reads <= 10_000]
    forms["served"] = {
        "reads_per_s": round(same_reads_rate, 1),
        "timing": "host, submit to last completion, copies included",
        "same_reads": f"the {n} uneven reads above as {len(cuts)} requests of log-uniform 1k-2M reads",
        "equals_plain": bool(served_same),
        "samples_burst": {"reads_per_s": round(sat, 1), "requests": args.serve_burst,
                          "groups": g1["groups_issued"] - g0["groups_issued"]},
        "poisson": {"offered_reads_per_s": round(0.5 * sat, 1), "achieved_reads_per_s": round(sent / wall, 1),
                    "seconds": round(wall, 1), "requests": int(ms.size),
                    "latency_ms": {k: (round(v, 2) if v is not None else None)
                                   for k, v in percentiles(ms).items()},
                    "latency_ms_requests_le_10k_reads": {k: (round(v, 2) if v is not None else None)
                                                         for k, v in percentiles(small).items()}},
        "options": {"hbm_budget_bytes": budget, "max_group_pairs": args.serve_group, "max_inflight": 3},
        "stats": {k: st[k] for k in ("groups_issued", "parts_issued", "max_requests_in_group",
                                     "max_groups_in_flight", "peak_bytes", "admission_waits")},
        "samples": "8 (CpG retention 0.4-0.9; fixed 150 / lognormal 120 / lognormal 90 length profiles), "
                   f"pools of {args.serve_pool} reads, request sizes log-uniform 1k-2M reads"}
    forms["served_over_plain_1launch"] = round(same_reads_rate / plain_rate, 3)
    forms["served_over_batched_1call"] = round(same_reads_rate / batched_rate, 3)
    forms["served_over_plain_reference_batches"] = round(same_reads_rate / ref_rate, 3)
    forms["batched_over_plain_1launch"] = round(batched_rate / plain_rate, 3)
    del d_bases, d_lens, pools
    return forms


GENOME_WORKLOADS = {
    # configs[2]/[3]: 3.1 Gbp reference, 50 M uneven single-end reads, then
    # the served stream against the same resident index
    "genome": dict(genome_mb=3100, repeats=False, n1=50_000_000, paired=False, max_len=UNEVEN_MAX,
                   model=UNEVEN_MODEL, bs=("C2T", ""),
                   text="{n1} single-end reads, lengths lognormal (median 120, sigma 0.35) clipped to 36-300, "
                        "half non-directional, on a {mb} Mbp synthetic bisulfite reference (bwa-meth c2t index)"),
    # 3.1 Gbp reference with 45% repeats + 3% tandem runs,
    # 20 M pairs 2x250 at non-CpG conversion 0.97
    "repeats": dict(genome_mb=3100, repeats=True, n1=10_000_000, paired=True, max_len=250,
                    model=dict(len_fixed=250, frag_mean=500, frag_sd=60, conv_non_cpg=0.97),
                    bs=("C2T", "G2A"),
                    text="{n1} PE 2x250 read pairs (non-CpG conversion 0.97) on a {mb} Mbp synthetic bisulfite "
                         "reference with 45% repeats (300 bp / 6 kb families, 10-20% divergence) and 3% tandem "
                         "runs (bwa-meth c2t index)"),
}


def host_capped_reads(n1: int, bytes_per_unit: int, world: int) -> int:
    """n1, or fewer when `world` ranks' pinned reads would take more than
    half of the host's memory."""
    try:
        total = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES")
    except (ValueError, OSError):
        return n1
    cap = int(total // 2 // max(1, world) // bytes_per_unit)
    return max(1, min(n1, cap))


def genome_config(args, spec, n1: int | None = None) -> dict:
    mb = args.genome_mb_large or spec["genome_mb"]
    n1 = n1 or args.genome_reads or spec["n1"]
    n_seq = n1 * (2 if spec["paired"] else 1)
    return {"workload": spec["text"].format(n1=n1, mb=mb), "form": "batched (one device call per chunk)",
            "genome_bp": mb * 1_000_000, "reads_per_gpu": n_seq, "paired": spec["paired"],
            "max_len": spec["max_len"], "params": dict(BENCH_PARAM_VALUES),
            "l2": "inputs larger than L2 (reads and index tens of GB)"}


def run_genome(args, rank, world, local):
    """Genome scale: the batched (autotuned) form over the whole read set
    per step, the plain single-launch form and the served form on the same
    reads, a served stream of 8 samples, parity against the oracle."""
    import torch
    from mojoalign_b200 import BENCH_PARAMS, GpuContext, GpuIndex, MapResult, map_batch, map_batch_device, synth
    from mojoalign_b200 import _lib

    spec = GENOME_WORKLOADS[args.workload]
    torch.cuda.set_device(local)
    dist = Dist(world, "nccl")
    params = BENCH_PARAMS
    mb = args.genome_mb_large or spec["genome_mb"]
    n1 = args.genome_reads or spec["n1"]
    paired, max_len = spec["paired"], spec["max_len"]
    per = 2 if paired else 1
    # every rank's reads stay pinned on the host: with several ranks on one
    # node, at most half of the host memory goes to them
    n1 = host_capped_reads(n1, per * max_len, world)
    n_seq = n1 * per
    bs1, bs2 = spec["bs"]
    dev = f"cuda:{local}"
    timings = {}
    t = time.time()
    fa, prefix, timings["reference_and_index"] = prepare_reference(
        args, rank, dist, local, genome_mb=mb, repeats=synth.RepeatModel() if spec["repeats"] else None,
        tag="_repeats" if spec["repeats"] else "")
    t = time.time()
    pinned = torch.empty((n_seq, max_len), dtype=torch.uint8, pin_memory=True)
    log(f"reads: {n1} x {per}")
    rb = synth.simulate_reads(fa, synth.ReadModel(**spec["model"]), n1, paired, max_len, seed=shard_seed(rank),
                              bases_out=pinned.numpy())
    timings["reads"] = time.time() - t
    ctx = GpuContext(local)
    # the ranks of a node open the index one after another: loading the
    # files holds ~11 GB of host memory per rank for a while
    for turn in range(world):
        if turn == rank:
            log("index open")
            t = time.time()
            gi = GpuIndex(ctx, prefix, kmer_k=args.kmer, kmer3_k=args.kmer3, at_k=args.at_k,
                          at_seed_len=params.seed_len if args.at_k else 0)
            timings["index_open"] = time.time() - t
        dist.barrier()
    bases_np, lens_np = pinned.numpy(), rb.lens

    # one stream for the torch copies and the library's calls (the calls
    # launch on the stream they are given), so that they stay ordered
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    d_bases = pinned.to(dev).reshape(-1)
    d_lens = torch.from_numpy(lens_np.view(np.int32)).to(dev)
    d_out = {f: torch.empty(n_seq, dtype=torch.int32, device=dev) for f in MapResult.FIELDS}
    # pairs (or reads) per device call: the packed reads and the seed
    # scratch of one call stay a few GB
    chunk = max(1, min(n1, args.genome_chunk // (2 if paired else 1)))

    def call(a, c):
        """One device call over single-end reads [a, a + c)."""
        offs = {f: x.data_ptr() + 4 * a for f, x in d_out.items()}
        map_batch_device(ctx, gi, d_bases.data_ptr() + a * max_len, d_lens.data_ptr() + 4 * a, c, False,
                         max_len, offs, bs1, bs2, params, stream=stream.cuda_stream)

    if paired:
        # the pairs as one call each chunk: the R1 and R2 rows of a chunk of
        # pairs are not adjacent in the full batch, so each chunk is staged
        # as its own batch (R1 rows, then R2 rows)
        rows = d_bases.view(n_seq, max_len)
        chunk_rows = torch.empty((2 * chunk, max_len), dtype=torch.uint8, device=dev)
        chunk_lens = torch.empty(2 * chunk, dtype=torch.int32, device=dev)
        chunk_out = {f: torch.empty(2 * chunk, dtype=torch.int32, device=dev) for f in MapResult.FIELDS}

        def call(a, c):  # noqa: F811
            chunk_rows[:c].copy_(rows[a:a + c])
            chunk_rows[c:2 * c].copy_(rows[n1 + a:n1 + a + c])
            chunk_lens[:c].copy_(d_lens[a:a + c])
            chunk_lens[c:2 * c].copy_(d_lens[n1 + a:n1 + a + c])
            map_batch_device(ctx, gi, chunk_rows.data_ptr(), chunk_lens.data_ptr(), c, True, max_len,
                             {f: x.data_ptr() for f, x in chunk_out.items()}, bs1, bs2, params,
                             stream=stream.cuda_stream)
            for f, x in d_out.items():
                x[a:a + c].copy_(chunk_out[f][:c])
                x[n1 + a:n1 + a + c].copy_(chunk_out[f][c:2 * c])

    def step():
        for a in range(0, n1, chunk):
            call(a, min(chunk, n1 - a))

    # ---- kernel form picked by the autotuner on a sample ----
    from mojoalign_b200.autotune import FIELDS as TFIELDS
    from mojoalign_b200.autotune import TuneResult, autotune

    ns = min(n1, 1_000_000 if paired else 2_000_000)
    log("autotune")
    if args.tuning:
        fixed = [int(x) for x in args.tuning.split(",")]
        fixed += [2, 1, 0, 2, 1, 1, 8, 4, 0, 1][len(fixed):]
        ctx.set_tuning(*fixed)
        tune = TuneResult(dict(zip(TFIELDS, fixed)), float("nan"), [])
    else:
        if paired:
            sb = np.concatenate([bases_np[:ns], bases_np[n1:n1 + ns]])
            sl = np.concatenate([lens_np[:ns], lens_np[n1:n1 + ns]])
        else:
            sb, sl = bases_np[:ns], lens_np[:ns]
        d_sb = torch.from_numpy(sb).to(dev).reshape(-1)
        d_sl = torch.from_numpy(sl.view(np.int32)).to(dev)
        n_s = sl.size
        s_out = {f: torch.empty(n_s, dtype=torch.int32, device=dev) for f in MapResult.FIELDS}
        s_dbg = {f: torch.empty(n_s, dtype=torch.int64 if f in ("uk", "ul") else torch.int32, device=dev)
                 for f in MapResult.DEBUG}

        def run_sample():
            map_batch_device(ctx, gi, d_sb.data_ptr(), d_sl.data_ptr(), ns, paired, max_len,
                             {f: x.data_ptr() for f, x in s_out.items()}, bs1, bs2, params,
                             d_debug={f: x.data_ptr() for f, x in s_dbg.items()}, stream=stream.cuda_stream)
            outs = {f: x.cpu().numpy() for f, x in list(s_out.items()) + list(s_dbg.items())}
            return outs, ctx.kernel_ms()[1]

        tune = autotune(ctx, gi, sb, sl, ns, paired, max_len, bs1, bs2, params, run=run_sample)
        del d_sb, d_sl, s_out, s_dbg, sb, sl
    best = tuple(tune.tuning[f] for f in TFIELDS if f in tune.tuning)

    log(f"tuning {tune.tuning}; counting pass")
    # ---- traffic tally: one untimed pass of the counting kernels ----
    _lib.check(_lib.lib.ma_ctx_set_profiling(ctx.handle, 2), ctx.handle)
    tally, tally2 = [0] * 12, [0] * 12
    for a in range(0, n1, chunk):
        call(a, min(chunk, n1 - a))
        tt = (_lib.C.c_uint64 * 12)()
        _lib.lib.ma_ctx_traffic(ctx.handle, tt)
        tally = [x + y for x, y in zip(tally, tt)]
        tally2 = [x + y for x, y in zip(tally2, ctx.traffic_stage2())]
    _lib.check(_lib.lib.ma_ctx_set_profiling(ctx.handle, 1), ctx.handle)

    # ---- per-kernel times of the seed kernels (events around each kernel
    # group; one profiled step, not the timed one) ----
    seed_ms, wave = [], []
    kms = (_lib.C.c_float * 4)()
    for _ in range(2):
        sm, wv = 0.0, [0.0] * 5
        for a in range(0, n1, chunk):
            call(a, min(chunk, n1 - a))
            _lib.lib.ma_ctx_kernel_ms(ctx.handle, kms)
            sm += float(kms[1])
            wv = [x + y for x, y in zip(wv, ctx.wave_ms())]
        seed_ms.append(sm)
        wave.append(wv)
    seed_ms, wave = seed_ms[1:], wave[1:]
    _lib.check(_lib.lib.ma_ctx_set_profiling(ctx.handle, 0), ctx.handle)

    log("timed steps")
    # ---- timed steps: the batched form over every read, each device call
    # replayed from its captured CUDA graph ----
    ctx.set_graphs(True)
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    torch.cuda.synchronize()
    profiled_region(True)
    ev0.record(stream)
    for _ in range(args.steps):
        for a in range(0, n1, chunk):
            call(a, min(chunk, n1 - a))
            launches += ctx.last_launch_count()
    ev1.record(stream)
    torch.cuda.synchronize()
    profiled_region(False)
    ms = ev0.elapsed_time(ev1) / args.steps
    clk = clocks.stop()
    dist.barrier()
    ctx.set_graphs(False)
    ms_max = dist.max(ms)
    value = aggregate_reads_per_s(n_seq, world, ms_max)
    batched_out = {f: x.cpu().numpy() for f, x in d_out.items()}

    log("end to end")
    # ---- end to end from pinned host buffers (copies inside) ----
    _lib.check(_lib.lib.ma_ctx_set_profiling(ctx.handle, 0), ctx.handle)
    from mojoalign_b200.mapper import page_locked

    res = MapResult.empty(n_seq, debug=False, pinned=True)
    lens_pin = page_locked(n_seq, np.uint32)
    lens_pin[:] = lens_np
    map_batch(ctx, gi, bases_np, lens_pin, n1, paired, max_len, bs1, bs2, params, out=res)
    dist.barrier()
    t = time.perf_counter()
    for _ in range(args.steps):
        map_batch(ctx, gi, bases_np, lens_pin, n1, paired, max_len, bs1, bs2, params, out=res)
    e2e_s = dist.max((time.perf_counter() - t) / args.steps)
    e2e_same = all(np.array_equal(getattr(res, f).view(np.int32), batched_out[f]) for f in MapResult.FIELDS)

    # ---- roofline of the seed kernels ----
    peaks = measured_peaks()
    words = (max_len + 31) // 32
    alg_bytes = 32 * (tally[0] + tally[1] + tally[2] + tally[3]) + n_seq * (4 * words * 8 + 4) + n_seq * 28
    seed_avg_ms = statistics.mean(seed_ms)
    achieved = alg_bytes / (seed_avg_ms / 1000.0) / 1e9
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
            "frac": round(achieved / peaks.get("hbm_gbs"), 4), "traffic": None,
            "peak_source": "fallback" if peaks.get("_fallback") else "measured (MEASURED_PEAKS.json hbm_gbs)",
            "kernel": SEED_KERNELS.get(tune.tuning.get("seed_kernel", 2), "seed/extend"),
            "kernel_ms": round(seed_avg_ms, 3), "alg_bytes_per_launch": int(alg_bytes),
            "tally_per_read": {k: round(v / n_seq, 3) for k, v in zip(
                ["occ_lines_32B", "kmer_loads", "sa_loads", "pac_sectors_32B", "backward_steps", "endpoints",
                 "loci_evaluated", "read_words", "endpoints_skipped", "stage2_reads", "stage2_groups",
                 "shift_evals"], tally)}}
    roof.update(seeding_roofline(tally, wave, tally2, n_seq, tune.tuning.get("seed_kernel", 2)))
    if (GENOME_SEED_DRAM_BYTES_PER_READ and spec is GENOME_WORKLOADS["genome"] and mb == spec["genome_mb"]
            and n1 == spec["n1"] and tuple(best) == GENOME_SEED_DRAM_TUNING and args.at_k == GENOME_SEED_DRAM_AT_K):
        roof["traffic"] = int(GENOME_SEED_DRAM_BYTES_PER_READ * n_seq)
        roof["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the seed kernels of one timed "
                                  "step of this workload and tuning (one-pass capture of this build), per read x reads")
        roof["traffic_over_alg"] = round(roof["traffic"] / alg_bytes, 3)

    line = {"metric": METRIC, "value": round(value, 1), "unit": "reads/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": genome_config(args, spec, n1),
            "run": {"tuning": tune.tuning, "autotune": tune.all_ms, "kmer_k": args.kmer, "kmer3_k": args.kmer3,
                    "at_k": args.at_k, "index_hbm_bytes": int(gi.info.device_bytes), "calls_per_step": -(-n1 // chunk),
                    "cuda_graphs": "each device call replays its captured graph (one host launch per call)",
                    "mapped_frac": round(float((batched_out["rid"] >= 0).mean()), 4)},
            "e2e": {"value": round(aggregate_reads_per_s(n_seq, world, e2e_s * 1000.0), 1), "unit": "reads/s",
                    "h2d_bytes_per_step": int(n_seq * max_len + n_seq * 4), "d2h_bytes_per_step": int(n_seq * 28),
                    "equals_device": bool(e2e_same)},
            "gpu_launches": launches, "roofline": roof, "clocks": clk,
            "setup_s": {k: round(v, 1) for k, v in timings.items()}}
    if rank == 0:
        line["gather_roofline"] = {}
        for lb in (32, 64):
            g = _lib.C.c_double()
            _lib.check(_lib.lib.ma_bench_gather(ctx.handle, 8 << 30, lb, 1 << 30, _lib.C.byref(g)), ctx.handle)
            line["gather_roofline"][f"hbm_{lb}B_GBs"] = round(g.value, 1)
        line["roofline"]["frac_of_gather32"] = round(achieved / line["gather_roofline"]["hbm_32B_GBs"], 4)
        line["roofline"]["frac_of_gather64"] = round(achieved / line["gather_roofline"]["hbm_64B_GBs"], 4)
        add_gather_fractions(line)
    if rank == 0 and world == 1 and not args.no_forms and not paired:
        del d_bases
        torch.cuda.empty_cache()
        log("forms")
        line["forms"] = genome_forms(args, ctx, gi, params, fa, local, best, bases_np, lens_np, n1, max_len,
                                     batched_out, value, stream)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle

        log("oracle sample")
        t = time.perf_counter()
        ix = oracle.OracleIndex(prefix)
        load_s = time.perf_counter() - t
        n = min(n1, args.parity_reads // (2 if paired else 1))
        if paired:
            b = np.concatenate([bases_np[:n], bases_np[n1:n1 + n]])
            l_ = np.concatenate([lens_np[:n], lens_np[n1:n1 + n]])
        else:
            b, l_ = bases_np[:n], lens_np[:n]
        t = time.perf_counter()
        o = ix.map(b, l_, n, paired, max_len, 1, 2 if paired else 0, params.as_list())
        dt = time.perf_counter() - t
        bad = 0
        for f in MapResult.FIELDS:
            g = batched_out[f]
            g = np.concatenate([g[:n], g[n1:n1 + n]]) if paired else g[:n]
            bad += int((g.view(o[f].dtype) != o[f]).sum())
        nr = n * (2 if paired else 1)
        line["parity_sample"] = {"reads": nr, "mismatched_fields": bad}
        line["cpu_baseline"] = {"value": round(nr / dt, 1), "unit": "reads/s", "cores": oracle.max_threads(),
                                "kind": "port", "cpu": _cpu_model(),
                                "sample": f"the parity sample ({nr} reads), {dt:.1f} s, index load {load_s:.1f} s"}
        reference_algorithm_bytes(line, ix, bases_np, lens_np, n1, paired, max_len, params, n_seq,
                                  bs2=2 if paired else 0)
    gi.close()
    ctx.close()
    torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not args.no_stages:
        line["stages"] = chromosome_stages(args, local, params, peaks)
    bad = parity_failures(line)
    line["parity_failures"] = bad
    if rank == 0:
        print(json.dumps(ordered_line(line)), flush=True)
    dist.close()
    if bad:
        sys.stderr.write("parity check failed: " + ", ".join(bad) + "\n")
        sys.exit(3)


def genome_forms(args, ctx, gi, params, fa, local, best, bases_np, lens_np, n, max_len, batched_out, batched_rate,
                 stream):
    """Plain single-launch, batched and served forms on the same single-end
    reads (equal outputs), then the served stream of 8 samples."""
    import torch
    from mojoalign_b200 import MapResult, map_batch_device, synth
    from mojoalign_b200.autotune import FIELDS as TFIELDS
    from mojoalign_b200.serve import Server, percentiles

    dev = f"cuda:{local}"
    forms = {}
    # plain single-launch (the reference's launch shape) on the first reads
    # of the batch, one call, inputs resident
    m = min(n, args.forms_reads)
    d_b = torch.from_numpy(bases_np[:m]).to(dev).reshape(-1)
    d_l = torch.from_numpy(lens_np[:m].view(np.int32)).to(dev)

    def device_form(tuning, reps=2):
        ctx.set_tuning(*tuning)
        d_o = {f: torch.empty(m, dtype=torch.int32, device=dev) for f in MapResult.FIELDS}
        ptrs = {f: x.data_ptr() for f, x in d_o.items()}

        def go():
            map_batch_device(ctx, gi, d_b.data_ptr(), d_l.data_ptr(), m, False, max_len, ptrs, "C2T", "", params,
                             stream=stream.cuda_stream)
        go()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            go()
        e1.record(stream)
        torch.cuda.synchronize()
        return m / (e0.elapsed_time(e1) / reps / 1000.0), {f: x.cpu().numpy() for f, x in d_o.items()}

    plain_rate, plain_out = device_form((0, 1, 0, 1, 16, 32, 32, 4, 0, 0))
    wave_rate, wave_out = device_form(best)
    same = all(np.array_equal(plain_out[f], batched_out[f][:m]) and np.array_equal(wave_out[f], plain_out[f])
               for f in MapResult.FIELDS)
    forms["reads"] = m
    forms["plain_1launch"] = {"reads_per_s": round(plain_rate, 1), "tuning": "seed_kernel 0 (thread per read)",
                              "timing": "device, inputs resident, one call"}
    forms["wavefront_1call"] = {"reads_per_s": round(wave_rate, 1), "tuning": dict(zip(TFIELDS, best)),
                                "timing": "device, inputs resident, one call", "equals_plain": bool(same)}
    ctx.set_tuning(*best)
    del d_b, d_l
    torch.cuda.empty_cache()

    # served: the same m reads as requests of log-uniform 1k-2M reads
    rng = np.random.default_rng(7)
    sizes = log_uniform_sizes(rng, 1 << 16, 1000, 2_000_000)
    cuts, a = [], 0
    for sz in sizes:
        if a >= m:
            break
        cuts.append((a, int(min(sz, m - a))))
        a += cuts[-1][1]
    group = args.serve_group
    with Server(ctx, gi, hbm_budget_bytes=args.serve_budget_gb << 30, max_group_pairs=group, max_inflight=3) as srv:
        def stream_same():
            t0 = time.perf_counter()
            ts = [srv.submit(bases_np[a:a + c], lens_np[a:a + c], c, False, max_len, "C2T", "", params)
                  for a, c in cuts]
            srv.drain()
            return ts, m / (time.perf_counter() - t0)

        stream_same()
        tickets, served_rate = stream_same()
        served_same = all(np.array_equal(getattr(t_.result, f).view(np.uint32), plain_out[f][a:a + c].view(np.uint32))
                          for t_, (a, c) in zip(tickets, cuts) for f in MapResult.FIELDS)
        del tickets
    forms["served"] = {"reads_per_s": round(served_rate, 1), "requests": len(cuts),
                       "timing": "host, submit to last completion, copies included",
                       "equals_plain": bool(served_same)}
    forms["batched_all_reads"] = {"reads_per_s": round(batched_rate, 1),
                                  "timing": "device, inputs resident, the headline step"}
    forms["served_over_plain_1launch"] = round(served_rate / plain_rate, 3)
    forms["served_over_wavefront_1call"] = round(served_rate / wave_rate, 3)
    forms["batched_over_plain_1launch"] = round(batched_rate / plain_rate, 3)

    # served stream: 8 samples, Poisson arrivals at half the burst rate, an
    # HBM budget that admission has to wait on
    pools = sample_pools(args, fa)

    def request(k, size):
        _, b, l, ml = pools[k]
        size = int(min(size, args.serve_pool))
        a = int(rng.integers(0, args.serve_pool - size + 1))
        return b[a:a + size], l[a:a + size], size, ml

    log("served stream")
    budget = args.serve_stream_budget_mb << 20
    with Server(ctx, gi, hbm_budget_bytes=budget, max_group_pairs=group, max_inflight=3) as srv:
        def burst(count):
            reqs = [request(int(rng.integers(0, 8)), s) for s in log_uniform_sizes(rng, count, 1000, 2_000_000)]
            t0 = time.perf_counter()
            for b, l, c, ml in reqs:
                srv.submit(b, l, c, False, ml, "C2T", "", params)
            srv.drain()
            return sum(r[2] for r in reqs) / (time.perf_counter() - t0)

        burst(16)
        sat = burst(args.serve_burst)
        mean_size = (2_000_000 - 1000) / np.log(2_000_000 / 1000)
        lam = 0.5 * sat / mean_size
        _, _, before = srv.latencies()
        n0 = before.size
        t0 = time.perf_counter()
        t_next = t0
        sent = 0
        while t_next - t0 < args.serve_seconds:
            now = time.perf_counter()
            if now < t_next:
                time.sleep(t_next - now)
            b, l, c, ml = request(int(rng.integers(0, 8)), log_uniform_sizes(rng, 1, 1000, 2_000_000)[0])
            srv.submit(b, l, c, False, ml, "C2T", "", params)
            sent += c
            t_next += rng.exponential(1.0 / lam)
        srv.drain()
        wall = time.perf_counter() - t0
        _, reads, lat = srv.latencies()
        lat, reads = lat[n0:], reads[n0:]
        st = srv.stats()
    forms["serving"] = {
        "samples": "8 (CpG retention 0.4-0.9; fixed 150 / lognormal 120 / lognormal 90 length profiles), pools of "
                   f"{args.serve_pool} reads, request sizes log-uniform 1k-2M reads",
        "burst_reads_per_s": round(sat, 1),
        "poisson": {"offered_reads_per_s": round(0.5 * sat, 1), "achieved_reads_per_s": round(sent / wall, 1),
                    "seconds": round(wall, 1), "requests": int(lat.size),
                    "latency_ms": {k: (round(v, 2) if v is not None else None) for k, v in percentiles(lat).items()}},
        "options": {"hbm_budget_bytes": budget, "max_group_pairs": group, "max_inflight": 3},
        "stats": {k: st[k] for k in ("groups_issued", "parts_issued", "max_requests_in_group",
                                     "max_groups_in_flight", "peak_bytes", "admission_waits")}}
    del pools
    return forms


def _cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


REF_SAMPLE_PAIRS = 1_000_000  # pairs handed to the reference arm (its steps time a part of them)


def prepare_sample(args, out: str) -> None:
    """Data preparation of the reference arm, run in a child process: the
    synthetic reference and its index (built by this package, on the GPU
    when there is one), the workload's reads, and the first reads of the
    batch saved to `out` (R1 rows, R2 rows when paired, lengths) with the
    index prefix."""
    from mojoalign_b200 import synth

    class _Solo(Dist):
        def __init__(self):
            super().__init__(1, "gloo")

    _, _, local = dist_env()
    if args.workload == "chromosome":
        fa, prefix, _ = prepare_reference(args, 0, _Solo(), local)
        rb = simulate(args, fa, 0)
        max_len = READ_LEN
    else:
        spec = GENOME_WORKLOADS[args.workload]
        mb = args.genome_mb_large or spec["genome_mb"]
        fa, prefix, _ = prepare_reference(args, 0, _Solo(), local, genome_mb=mb,
                                          repeats=synth.RepeatModel() if spec["repeats"] else None,
                                          tag="_repeats" if spec["repeats"] else "")
        n1 = min(args.genome_reads or spec["n1"], REF_SAMPLE_PAIRS)
        max_len = spec["max_len"]
        rb = synth.simulate_reads(fa, synth.ReadModel(**spec["model"]), n1, spec["paired"], max_len, seed=1)
    n = min(rb.n1, REF_SAMPLE_PAIRS)
    r2 = rb.bases[rb.n1:rb.n1 + n] if rb.paired else rb.bases[:0]
    l2 = rb.lens[rb.n1:rb.n1 + n] if rb.paired else rb.lens[:0]
    np.savez(out, r1=rb.bases[:n], r2=r2, l1=rb.lens[:n], l2=l2, prefix=np.array(str(prefix)),
             paired=np.array(rb.paired), max_len=np.array(max_len))


def run_reference(args, rank, world, local):
    """The reference algorithm on the host cores: the oracle (the CPU
    restatement of the reference kernels; the Mojo reference cannot run
    here).  The inputs are made by a child process, so this process loads
    only the oracle's library."""
    if rank != 0:
        return
    with tempfile.TemporaryDirectory(prefix="mojoalign_ref_") as td:
        sample = Path(td) / "sample.npz"
        cmd = [sys.executable, str(Path(__file__).resolve()), "--prepare-sample", str(sample),
               "--genome-mb", str(args.genome_mb), "--pairs", str(args.pairs), "--workdir", args.workdir,
               "--workload", args.workload, "--genome-mb-large", str(args.genome_mb_large),
               "--genome-reads", str(args.genome_reads)]
        subprocess.run(cmd, check=True)
        z = np.load(sample)
        r1, r2, l1, l2, prefix = z["r1"], z["r2"], z["l1"], z["l2"], str(z["prefix"])
        paired, max_len = bool(z["paired"]), int(z["max_len"])
    import oracle

    plist = list(BENCH_PARAM_VALUES.values())
    ix = oracle.OracleIndex(prefix)
    per = 2 if paired else 1
    bs2 = 2 if paired else 0

    def batch(n):
        if not paired:
            return r1[:n], l1[:n]
        return np.concatenate([r1[:n], r2[:n]]), np.concatenate([l1[:n], l2[:n]])

    # size one step to about cpu_seconds / (steps + warmup) * 2
    probe = min(10000, len(l1))
    b, l = batch(probe)
    t = time.perf_counter()
    ix.map(b, l, probe, paired, max_len, 1, bs2, plist)
    rate = per * probe / (time.perf_counter() - t)
    per_step_s = max(2.0, 60.0 / max(1, args.steps + args.warmup))
    n = int(min(len(l1), max(probe, rate * per_step_s / per)))
    b, l = batch(n)
    for _ in range(args.warmup):
        ix.map(b, l, n, paired, max_len, 1, bs2, plist)
    t = time.perf_counter()
    for _ in range(args.steps):
        ix.map(b, l, n, paired, max_len, 1, bs2, plist)
    dt = (time.perf_counter() - t) / args.steps
    value = per * n / dt
    config = workload_config(args) if args.workload == "chromosome" else genome_config(
        args, GENOME_WORKLOADS[args.workload])
    line = {"metric": METRIC, "value": round(value, 1), "unit": "reads/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dt * 1000, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic", "impl": "reference",
            "config": config,
            "cpu_baseline": {"value": round(value, 1), "unit": "reads/s", "cores": oracle.max_threads(),
                             "kind": "port", "cpu": _cpu_model(),
                             "sample": f"first {per * n} reads of the workload per step"},
            "e2e": {"value": round(value, 1), "unit": "reads/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(ordered_line(line)), flush=True)


def gather_sweep(device: int = 0, sizes_mb=(16, 64, 256, 1024, 4096, 8192, 16384, 32768),
                 loads: int = 1 << 30) -> dict:
    """Measured random-gather roofline of this GPU: uniformly random,
    independent loads of aligned 32- and 64-byte lines over buffers from
    16 MiB (L2-resident) to 32 GiB (HBM), GB/s per buffer and line size.
    The seed/extend kernels gather Occ lines, k-mer table entries and SA
    entries at random: this is their ceiling, far below the copy bandwidth."""
    from mojoalign_b200 import GpuContext

    ctx = GpuContext(device)
    try:
        return {f"{mb}MiB_{lb}B_GBs": round(ctx.gather_gbps(mb << 20, lb, loads), 1)
                for mb in sizes_mb for lb in (32, 64)}
    finally:
        ctx.close()


def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.prepare_sample:
        prepare_sample(args, args.prepare_sample)
    elif args.gather_sweep:
        print(json.dumps(gather_sweep(local)), flush=True)
    elif args.impl == "reference":
        run_reference(args, rank, world, local)
    elif args.workload == "chromosome":
        run_ours(args, rank, world, local)
    else:
        run_genome(args, rank, world, local)


if __name__ == "__main__":
    main()
