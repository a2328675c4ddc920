"""The C ABI on the host: exported symbols, defaults, host-only index
checks and their failure modes (fail closed like FmIndex.load,
fq2bam-meth/src/linear_fm_index.mojo:88-175).  No GPU needed."""
from __future__ import annotations

import re
import shutil
import struct
from pathlib import Path

import pytest

import oracle
from mojoalign_b200 import MojoAlignError, probe_index
from mojoalign_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "mojoalign_b200.h"


def declared_functions() -> set[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return set(re.findall(r"\b(ma_[a-z0-9_]+)\s*\(", text))


def test_every_declared_entry_point_is_exported():
    names = declared_functions()
    assert len(names) >= 20
    for n in sorted(names):
        assert hasattr(_lib.lib, n), f"{n} declared in the header but not exported"
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert names <= bound, f"entry points without a ctypes signature: {sorted(names - bound)}"


def declared_arity() -> dict[str, int]:
    """Parameter count of every prototype in the header."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(ma_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_ctypes_signatures_match_the_header():
    arity = declared_arity()
    assert len(arity) >= 20
    for name, _, args in _lib.SIGNATURES:
        if name in arity:
            assert len(args) == arity[name], f"{name}: {len(args)} ctypes arguments, header declares {arity[name]}"


def declared_struct_fields(name: str) -> list[str]:
    """Field names of `typedef struct name { ... } name;` in the header."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    m = re.search(r"typedef struct " + name + r"\s*\{(.*?)\}\s*" + name + r"\s*;", text, flags=re.S)
    assert m, name
    return [re.sub(r"\[.*\]", "", d.split()[-1]) for d in m.group(1).split(";") if d.strip()]


@pytest.mark.parametrize("name", ["ma_index_options", "ma_index_info", "ma_params", "ma_tuning"])
def test_ctypes_structs_match_the_header(name):
    assert [f[0] for f in getattr(_lib, name)._fields_] == declared_struct_fields(name)


def test_index_options_default():
    o = _lib.ma_index_options()
    _lib.lib.ma_index_options_default(o)
    assert (o.kmer_k, o.kmer3_k, o.hbm_budget_bytes, o.wide_rows, o.occ_super_shift, o.prep_chunk_rows,
            o.at_k, o.at_seed_len) == (12, 0, 0, 0, 0, 0, 0, 0)


def test_params_default_are_the_reference_defaults():
    p = _lib.ma_params()
    _lib.lib.ma_params_default(p)
    # METHYLGRAPHER_FM_* defaults, linear_gpu_fm.mojo:2074-2082
    assert [p.seed_len, p.seed_stride, p.max_occ, p.max_diff, p.max_soft, p.max_adj, p.rescue_win] == \
        [18, 2, 4096, 12, 20, 8, 512]


def test_context_without_sm100_gpu_fails_closed():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = _lib.C.c_void_p()
    rc = _lib.lib.ma_ctx_create(0, _lib.C.byref(h))
    assert rc == _lib.MA_ERR_CUDA
    assert _lib.last_error()


def test_probe_counts_the_at_window_table(small_ref):
    _, prefix = small_ref
    base = probe_index(prefix, kmer_k=10, kmer3_k=9).device_bytes
    assert probe_index(prefix, kmer_k=10, kmer3_k=9, at_k=20).device_bytes == base + (1 << 20) * 16
    with pytest.raises(MojoAlignError):
        probe_index(prefix, at_k=31)


def test_probe_matches_oracle_header(small_ref):
    _, prefix = small_ref
    info = probe_index(prefix, kmer_k=10, kmer3_k=9)
    ix = oracle.OracleIndex(prefix)
    assert (info.seq_len, info.l_pac, info.primary) == (ix.seq_len, ix.l_pac, ix.primary)
    assert list(info.L2) == list(ix.L2)
    assert (info.sa_intv, info.n_sa, info.n_contigs) == (ix.sa_intv, ix.n_sa, ix.n_contigs)
    assert 0 < info.sa_reject_below <= info.seq_len
    assert info.device_bytes > 4 * info.seq_len


def _copy_index(src_prefix, dst_dir: Path) -> Path:
    dst = dst_dir / "idx"
    for ext in (".bwt", ".sa", ".pac", ".ann", ".amb"):
        shutil.copy(str(src_prefix) + ext, str(dst) + ext)
    return dst


@pytest.mark.parametrize("corruption,code", [
    ("missing_sa", _lib.MA_ERR_IO),
    ("short_bwt", _lib.MA_ERR_FORMAT),
    ("primary_mismatch", _lib.MA_ERR_FORMAT),
    ("seq_len_mismatch", _lib.MA_ERR_FORMAT),
    ("ann_offsets", _lib.MA_ERR_FORMAT),
    ("truncated_ann", _lib.MA_ERR_FORMAT),
    ("bad_sa_intv", _lib.MA_ERR_FORMAT),
])
def test_corrupt_index_fails_closed(small_ref, tmp_path, corruption, code):
    _, prefix = small_ref
    p = _copy_index(prefix, tmp_path)
    if corruption == "missing_sa":
        Path(str(p) + ".sa").unlink()
    elif corruption == "short_bwt":
        b = Path(str(p) + ".bwt").read_bytes()
        Path(str(p) + ".bwt").write_bytes(b[: len(b) // 2 // 4 * 4])
    elif corruption in ("primary_mismatch", "seq_len_mismatch", "bad_sa_intv"):
        b = bytearray(Path(str(p) + ".sa").read_bytes())
        word = {"primary_mismatch": 0, "seq_len_mismatch": 6, "bad_sa_intv": 5}[corruption]
        v = struct.unpack_from("<Q", b, 8 * word)[0]
        struct.pack_into("<Q", b, 8 * word, v + 3 if corruption != "bad_sa_intv" else 24)
        Path(str(p) + ".sa").write_bytes(bytes(b))
    elif corruption == "ann_offsets":
        lines = Path(str(p) + ".ann").read_text().splitlines()
        off, ln, amb = lines[2].split()
        lines[2] = f"{off} {int(ln) + 1} {amb}"
        Path(str(p) + ".ann").write_text("\n".join(lines) + "\n")
    elif corruption == "truncated_ann":
        lines = Path(str(p) + ".ann").read_text().splitlines()
        Path(str(p) + ".ann").write_text("\n".join(lines[:-1]) + "\n")
    with pytest.raises(MojoAlignError) as e:
        probe_index(p)
    assert e.value.code == code, str(e.value)


def test_probe_argument_errors(small_ref):
    _, prefix = small_ref
    with pytest.raises(MojoAlignError) as e:
        probe_index(prefix, kmer_k=15)
    assert e.value.code == _lib.MA_ERR_ARG
