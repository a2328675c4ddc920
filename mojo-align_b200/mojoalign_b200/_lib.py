"""ctypes binding of libmojoalign_b200.so (the C ABI in include/mojoalign_b200.h).

The shared library is the only compute path: importing this module fails
loudly when it is missing, and every mapping call fails when no sm_100 GPU
is present.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmojoalign_b200.so"

MA_OK = 0
MA_ERR_ARG = -1
MA_ERR_IO = -2
MA_ERR_FORMAT = -3
MA_ERR_CUDA = -4
MA_ERR_NOMEM = -5
MA_ERR_UNSUPPORTED = -6
MA_ERR_TIMEOUT = -7
MA_ERR_INTERNAL = -8

MA_BS_NONE, MA_BS_C2T, MA_BS_G2A = 0, 1, 2

ERR_NAMES = {
    MA_ERR_ARG: "MA_ERR_ARG",
    MA_ERR_IO: "MA_ERR_IO",
    MA_ERR_FORMAT: "MA_ERR_FORMAT",
    MA_ERR_CUDA: "MA_ERR_CUDA",
    MA_ERR_NOMEM: "MA_ERR_NOMEM",
    MA_ERR_UNSUPPORTED: "MA_ERR_UNSUPPORTED",
    MA_ERR_TIMEOUT: "MA_ERR_TIMEOUT",
    MA_ERR_INTERNAL: "MA_ERR_INTERNAL",
}


class MojoAlignError(RuntimeError):
    """A failed C ABI call; `code` is the MA_ERR_* status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {message}")
        self.code = code


class ma_params(C.Structure):
    _fields_ = [
        ("seed_len", C.c_int32),
        ("seed_stride", C.c_int32),
        ("max_occ", C.c_int32),
        ("max_diff", C.c_int32),
        ("max_soft", C.c_int32),
        ("max_adj", C.c_int32),
        ("rescue_win", C.c_int32),
    ]


class ma_hits(C.Structure):
    _fields_ = [
        ("rid", C.c_void_p),
        ("pos", C.c_void_p),
        ("mapq", C.c_void_p),
        ("flag", C.c_void_p),
        ("sl", C.c_void_p),
        ("sr", C.c_void_p),
        ("nm", C.c_void_p),
    ]


class ma_debug(C.Structure):
    _fields_ = [
        ("uk", C.c_void_p),
        ("ul", C.c_void_p),
        ("us", C.c_void_p),
        ("e", C.c_void_p),
        ("score", C.c_void_p),
    ]


class ma_index_info(C.Structure):
    _fields_ = [
        ("seq_len", C.c_uint64),
        ("l_pac", C.c_uint64),
        ("primary", C.c_uint64),
        ("L2", C.c_uint64 * 5),
        ("sa_intv", C.c_int64),
        ("n_sa", C.c_int64),
        ("n_contigs", C.c_int64),
        ("sa_reject_below", C.c_uint64),
        ("kmer_k", C.c_int32),
        ("kmer3_k", C.c_int32),
        ("device_bytes", C.c_uint64),
    ]


class ma_index_options(C.Structure):
    _fields_ = [("kmer_k", C.c_int32), ("kmer3_k", C.c_int32), ("hbm_budget_bytes", C.c_uint64),
                ("wide_rows", C.c_int32), ("occ_super_shift", C.c_int32), ("prep_chunk_rows", C.c_uint64),
                ("at_k", C.c_int32), ("at_seed_len", C.c_int32)]


class ma_tuning(C.Structure):
    _fields_ = [("seed_kernel", C.c_int32), ("stage1_endpoints", C.c_int32), ("stage2_blocks_per_sm", C.c_int32),
                ("reg_level", C.c_int32), ("stage1_max_rows", C.c_int32), ("stage2_first_wave", C.c_int32),
                ("wave_endpoints", C.c_int32), ("wave_loci_per_read", C.c_int32), ("wave_max_rounds", C.c_int32),
                ("wave_growth", C.c_int32)]


class ma_pipeline(C.Structure):
    _fields_ = [("first_chunk_pairs", C.c_uint32), ("growth_percent", C.c_uint32), ("max_chunk_pairs", C.c_uint32),
                ("compute_streams", C.c_uint32)]


class ma_repeat_model(C.Structure):
    _fields_ = [
        ("repeat_frac", C.c_double),
        ("tandem_frac", C.c_double),
        ("families", C.c_uint32),
        ("short_len", C.c_uint32),
        ("long_len", C.c_uint32),
        ("long_share", C.c_double),
        ("div_min", C.c_double),
        ("div_max", C.c_double),
        ("unit_min", C.c_uint32),
        ("unit_max", C.c_uint32),
        ("run_min", C.c_uint32),
        ("run_max", C.c_uint32),
    ]


class ma_read_model(C.Structure):
    _fields_ = [
        ("len_fixed", C.c_uint32),
        ("len_lognorm_median", C.c_double),
        ("len_lognorm_sigma", C.c_double),
        ("len_min", C.c_uint32),
        ("len_max", C.c_uint32),
        ("frag_mean", C.c_double),
        ("frag_sd", C.c_double),
        ("conv_non_cpg", C.c_double),
        ("cpg_retain", C.c_double),
        ("sub_rate", C.c_double),
        ("random_frac", C.c_double),
        ("non_directional", C.c_double),
    ]


class ma_serve_options(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_group_pairs", C.c_uint32), ("max_inflight", C.c_uint32),
                ("flags", C.c_uint32)]


class ma_serve_stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "requests_submitted", "requests_completed", "requests_failed", "reads_completed", "groups_issued",
        "parts_issued", "max_requests_in_group", "max_groups_in_flight", "budget_bytes", "peak_bytes",
        "admission_waits")]


MA_SERVE_SCHEDULER_TEST = 1


class ma_fastq_arena(C.Structure):
    _fields_ = [("data", C.c_void_p), ("data_bytes", C.c_uint64), ("name_off", C.c_void_p), ("name_len", C.c_void_p),
                ("orig_off", C.c_void_p), ("orig_len", C.c_void_p), ("qual_off", C.c_void_p),
                ("qual_len", C.c_void_p)]


class ma_fastq_records(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("name_off", "name_len", "seq_off", "seq_len", "qual_off", "qual_len")]


class ma_sam_contigs(C.Structure):
    _fields_ = [("names", C.c_void_p), ("names_bytes", C.c_uint64), ("name_off", C.c_void_p), ("name_len", C.c_void_p),
                ("canon", C.c_void_p), ("n", C.c_uint32)]


MA_FASTQ_RULES_STREAM = 0
MA_FASTQ_RULES_PAIR_READER = 1


class ma_bam_meta(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("coord", "dhi", "dlo", "rec", "len", "score", "pair")]


class ma_bam_tile(C.Structure):
    _fields_ = [("n_reads", C.c_uint64), ("n_mapped", C.c_uint64), ("n_total", C.c_uint64), ("meta_cap", C.c_uint64),
                ("chunk", C.c_uint32)]

# (name, restype, argtypes) of every exported entry point of the header.
SIGNATURES = [
    ("ma_params_default", None, [C.POINTER(ma_params)]),
    ("ma_ctx_create", C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    ("ma_ctx_destroy", None, [C.c_void_p]),
    ("ma_last_error", C.c_char_p, [C.c_void_p]),
    ("ma_hbm_info", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("ma_index_build", C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int]),
    ("ma_index_build_batched", C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_uint64]),
    ("ma_index_options_default", None, [C.POINTER(ma_index_options)]),
    ("ma_index_open", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(ma_index_options), C.POINTER(C.c_void_p)]),
    ("ma_index_close", None, [C.c_void_p]),
    ("ma_index_probe", C.c_int, [C.c_char_p, C.c_int, C.c_int, C.POINTER(ma_index_info)]),
    ("ma_index_get_info", C.c_int, [C.c_void_p, C.POINTER(ma_index_info)]),
    ("ma_index_contig", C.c_int,
     [C.c_void_p, C.c_int64, C.POINTER(C.c_char_p), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("ma_map_batch", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_uint32, C.c_int, C.c_int,
      C.POINTER(ma_params), C.POINTER(ma_hits), C.POINTER(ma_debug)]),
    ("ma_map_batch_device", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_uint32, C.c_int, C.c_int,
      C.POINTER(ma_params), C.POINTER(ma_hits), C.POINTER(ma_debug), C.c_void_p]),
    ("ma_map_batch_device_noalloc", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_uint32, C.c_int, C.c_int,
      C.POINTER(ma_params), C.POINTER(ma_hits), C.POINTER(ma_debug), C.c_void_p]),
    ("ma_last_launch_count", C.c_int, [C.c_void_p]),
    ("ma_ctx_set_profiling", C.c_int, [C.c_void_p, C.c_int]),
    ("ma_ctx_set_graphs", C.c_int, [C.c_void_p, C.c_int]),
    ("ma_ctx_set_tuning", C.c_int, [C.c_void_p, C.POINTER(ma_tuning)]),
    ("ma_ctx_get_tuning", C.c_int, [C.c_void_p, C.POINTER(ma_tuning)]),
    ("ma_ctx_set_pipeline", C.c_int, [C.c_void_p, C.POINTER(ma_pipeline)]),
    ("ma_ctx_get_pipeline", C.c_int, [C.c_void_p, C.POINTER(ma_pipeline)]),
    ("ma_ctx_kernel_ms", C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    ("ma_ctx_wave_ms", C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    ("ma_ctx_traffic_stage2", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    ("ma_ctx_traffic", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    ("ma_bench_gather", C.c_int, [C.c_void_p, C.c_uint64, C.c_int, C.c_uint64, C.POINTER(C.c_double)]),
    ("ma_serve_options_default", None, [C.POINTER(ma_serve_options)]),
    ("ma_serve_create", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(ma_serve_options), C.POINTER(C.c_void_p)]),
    ("ma_serve_submit", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_uint32, C.c_int, C.c_int, C.POINTER(ma_params),
      C.POINTER(ma_hits), C.POINTER(C.c_uint64)]),
    ("ma_serve_poll", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_int)]),
    ("ma_serve_wait", C.c_int, [C.c_void_p, C.c_uint64, C.c_int]),
    ("ma_serve_drain", C.c_int, [C.c_void_p, C.c_int]),
    ("ma_serve_get_stats", C.c_int, [C.c_void_p, C.POINTER(ma_serve_stats)]),
    ("ma_serve_latencies", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("ma_serve_last_error", C.c_char_p, [C.c_void_p]),
    ("ma_serve_destroy", None, [C.c_void_p]),
    ("ma_emit_bam_batch", C.c_int,
     [C.c_void_p, C.POINTER(ma_hits), C.c_uint32, C.c_int, C.POINTER(ma_fastq_arena), C.c_void_p, C.c_int32,
      C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(ma_bam_meta),
      C.POINTER(ma_bam_tile)]),
    ("ma_emit_bam_batch_device", C.c_int,
     [C.c_void_p, C.POINTER(ma_hits), C.c_uint32, C.c_int, C.POINTER(ma_fastq_arena), C.c_void_p, C.c_int32,
      C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.POINTER(ma_bam_meta), C.POINTER(ma_bam_tile),
      C.c_void_p, C.c_void_p]),
    ("ma_sort_markdup", C.c_int,
     [C.c_void_p, C.c_uint64] + [C.c_void_p] * 7 + [C.c_int, C.c_void_p, C.POINTER(C.c_uint64)]),
    ("ma_sort_markdup_device", C.c_int,
     [C.c_void_p, C.c_uint64] + [C.c_void_p] * 7 + [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("ma_gather_sorted_bam", C.c_int,
     [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
      C.c_uint32, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("ma_gather_sorted_bam_device", C.c_int,
     [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
      C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    ("ma_fastq_parse", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_uint32, C.c_uint64, C.POINTER(ma_fastq_records),
      C.POINTER(C.c_uint64)]),
    ("ma_fastq_parse_device", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_uint32, C.c_uint64, C.POINTER(ma_fastq_records),
      C.POINTER(C.c_uint64), C.c_void_p]),
    ("ma_fastq_parse_rules", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_uint32, C.c_uint64, C.c_int, C.POINTER(ma_fastq_records),
      C.POINTER(C.c_uint64)]),
    ("ma_fastq_parse_rules_device", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_uint32, C.c_uint64, C.c_int, C.POINTER(ma_fastq_records),
      C.POINTER(C.c_uint64), C.c_void_p]),
    ("ma_emit_sam_batch", C.c_int,
     [C.c_void_p, C.POINTER(ma_hits), C.c_uint32, C.c_int, C.POINTER(ma_fastq_arena), C.POINTER(ma_sam_contigs),
      C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("ma_emit_sam_batch_device", C.c_int,
     [C.c_void_p, C.POINTER(ma_hits), C.c_uint32, C.c_int, C.POINTER(ma_fastq_arena), C.POINTER(ma_sam_contigs),
      C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    ("ma_fastq_rows_device", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("ma_bgzf_compress", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("ma_bgzf_compress_device", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64),
      C.c_void_p]),
    ("ma_bgzf_bound", C.c_uint64, [C.c_uint64]),
    ("ma_bgzf_inflate", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_uint64] + [C.c_void_p] * 5 + [C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p]),
    ("ma_bgzf_inflate_device", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_uint64] + [C.c_void_p] * 5 + [C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p,
                                                                C.c_void_p]),
    ("ma_synth_reference", C.c_int, [C.c_char_p, C.c_uint64, C.c_int, C.c_double, C.c_double, C.c_uint64]),
    ("ma_synth_reference_model", C.c_int,
     [C.c_char_p, C.c_uint64, C.c_int, C.c_double, C.c_double, C.c_uint64, C.POINTER(ma_repeat_model)]),
    ("ma_synth_reads", C.c_int,
     [C.c_char_p, C.POINTER(ma_read_model), C.c_uint32, C.c_int, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p,
      C.c_void_p, C.c_void_p]),
]


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python mojo-align_b200/build_lib.py` "
            "(or __graft_entry__.build()); there is no fallback implementation"
        )
    lib = C.CDLL(str(LIB_PATH))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error(ctx=None) -> str:
    msg = lib.ma_last_error(ctx)
    return msg.decode() if msg else ""


def check(rc: int, ctx=None) -> None:
    if rc != MA_OK:
        raise MojoAlignError(rc, last_error(ctx))


def ptr(a) -> int | None:
    """Address of a numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data


def fspath(p) -> bytes:
    return os.fsencode(os.fspath(p))
