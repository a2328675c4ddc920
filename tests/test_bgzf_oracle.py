"""The BGZF oracle (oracle/bgzf_ref.py) against what the reference's own
writer (fq2bam-meth/python/bam_emit.py, _BgzfWriter / _bgzf_block) wrote for
the same streams (tests/golden/bgzf_vectors.json), and its member reader."""
from __future__ import annotations

import gzip
import hashlib
import json
import sys
from pathlib import Path

import pytest

from oracle import bgzf_ref

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
from make_bgzf_golden import stream  # noqa: E402


def _cases():
    return json.loads((GOLDEN / "bgzf_vectors.json").read_text())


def test_constants():
    g = _cases()
    assert g["block"] == bgzf_ref.BLOCK
    assert g["eof"] == bgzf_ref.EOF_MEMBER.hex()


@pytest.mark.parametrize("level", [0, 1])
def test_files_match_reference_writer(level):
    for c in _cases()["cases"]:
        data = stream(c["kind"], c["n"])
        out = bgzf_ref.compress(data, level)
        want = c["levels"][str(level)]
        assert len(out) == want["size"] and hashlib.sha256(out).hexdigest() == want["sha256"], (c["kind"], c["n"])
        ms = bgzf_ref.members(out)
        assert [m["size"] for m in ms] == want["member_sizes"]
        assert gzip.decompress(out) == data
        body = b"".join(bgzf_ref.inflate(m["payload"]) for m in ms[:-1])
        assert body == data
