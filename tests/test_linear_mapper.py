"""The FM engine's command line (python -m mojoalign_b200.linear_mapper),
mirroring run_mojo_linear_cli (fq2bam-meth/src/linear_mapper.mojo:314-346)
and the engine choice of its map_fastq_to_sam (L129-166): argument parsing,
dispatch to map_fastq_fm_gpu, fail-closed exit status."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import pytest

import mojoalign_b200.linear_fm as linear_fm
from mojoalign_b200.linear_mapper import get_kv_value, main, run_mojo_linear_cli

FM_ENV = {"METHYLGRAPHER_LINEAR_ENGINE": "fm"}
ARGS = ["-ref", "ref.fa", "-fq1", "r1.fq", "-fq2", "r2.fq", "-out_sam", "out.bam", "-device", "nvidia", "-k", "15",
        "-cache_dir", "cache", "-bs_r1", "C2T", "-bs_r2", "G2A"]


def test_get_kv_value():
    a = ["-ref", "x.fa", "-fq1", "-k", "7", "--fq2", "b", "-out_sam"]
    assert get_kv_value(a, "ref", "") == "x.fa"
    assert get_kv_value(a, "fq1", "") == "-k"  # the next argument, whatever it is
    assert get_kv_value(a, "k", "15") == "7"
    assert get_kv_value(a, "fq2", "") == ""  # "--fq2" is not "-fq2"
    assert get_kv_value(a, "out_sam", "aligned.sam") == "aligned.sam"  # last argument: the default
    assert get_kv_value(["-", "v"], "", "d") == "d"


@pytest.fixture
def fake_map(monkeypatch):
    calls = []

    def fake(*a, **kw):
        calls.append((a, kw))
        return 42

    monkeypatch.setattr(linear_fm, "map_fastq_fm_gpu", fake)
    return calls


def test_fm_engine_dispatch(fake_map, capsys):
    for eng in ("fm", "FM", "bwa-mem", "bwamem"):
        assert run_mojo_linear_cli(ARGS, {"METHYLGRAPHER_LINEAR_ENGINE": eng}) == 0
    a, kw = fake_map[0]
    assert a == ("ref.fa", "r1.fq", "out.bam", "nvidia", "r2.fq", "C2T", "G2A")
    assert kw["environ"]["METHYLGRAPHER_LINEAR_ENGINE"] == "fm"
    out = capsys.readouterr().out
    assert "MojoLinear engine=fm" in out and "mapped_records= 42" in out
    # defaults: out_sam aligned.sam, device auto, no mate, no conversion
    assert main(["-ref", "r.fa", "-fq1", "a.fq"]) == 1  # engine parity by default
    assert run_mojo_linear_cli(["-ref", "r.fa", "-fq1", "a.fq"], dict(FM_ENV, METHYLGRAPHER_LINEAR_GPU_LOCATE="")) == 0
    assert fake_map[-1][0] == ("r.fa", "a.fq", "aligned.sam", "auto", "", "", "")


@pytest.mark.parametrize("args,env,msg", [
    (["-fq1", "a.fq"], FM_ENV, "requires -ref"),
    (["-ref", "r.fa"], FM_ENV, "requires -fq1"),
    (["-ref", "r.fa", "-fq1", "a.fq"], {}, "engine 'parity'"),
    (["-ref", "r.fa", "-fq1", "a.fq", "-device", "cpu"], FM_ENV, "device 'cpu'"),
    (["-ref", "r.fa", "-fq1", "a.fq"], dict(FM_ENV, METHYLGRAPHER_LINEAR_GPU_LOCATE="0"), "not part of this build"),
    (["-ref", "r.fa", "-build_cache_only"], FM_ENV, "-build_cache_only"),
    (["-ref", "r.fa", "-fq1", "a.fq", "-k", "x"], FM_ENV, "invalid literal"),
])
def test_errors_exit_1(fake_map, monkeypatch, capsys, args, env, msg):
    monkeypatch.setattr(os, "environ", dict(env))
    assert main(args) == 1
    assert msg in capsys.readouterr().err
    assert not fake_map


def test_module_entry_point(tmp_path):
    root = Path(__file__).resolve().parent.parent
    env = dict(os.environ, PYTHONPATH=str(root / "mojo-align_b200"), METHYLGRAPHER_LINEAR_ENGINE="fm")
    r = subprocess.run([sys.executable, "-m", "mojoalign_b200.linear_mapper", "-fq1", "a.fq"], env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 1 and "requires -ref" in r.stderr
