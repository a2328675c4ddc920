"""Regenerates tests/golden/bgzf_vectors.json from the reference.

Run from the repository root where the mojo-align source tree is available
(its path is the one required argument).  Imports the reference's BAM writer,
fq2bam-meth/python/bam_emit.py, and records what its BGZF layer
(_bgzf_block L77-98 through _BgzfWriter L101-186) writes for deterministic
inputs: per level, the SHA-256 and size of the file and of each member, for
streams cut at and around the 65280-byte block size.  The inputs are
regenerated by the tests from the same rule (`stream(kind, n)` below)."""
from __future__ import annotations

import hashlib
import importlib.util
import json
import sys
import tempfile
from pathlib import Path

OUT = Path(__file__).resolve().parent / "bgzf_vectors.json"
CASES = [("ramp", 0), ("ramp", 1), ("ramp", 100), ("ramp", 32767), ("ramp", 32768), ("ramp", 65280),
         ("ramp", 65281), ("text", 200_000), ("zeros", 140_000)]


def stream(kind: str, n: int) -> bytes:
    if kind == "ramp":
        return bytes((i * 7 + (i >> 8)) & 255 for i in range(n))
    if kind == "zeros":
        return bytes(n)
    words = [b"chr1", b"ACGT", b"mojo1", b"NM", b"RG", b"IIIII", b"read:", b"0001"]
    out = bytearray()
    i = 0
    while len(out) < n:
        out += words[(i * 5 + i // 3) % len(words)]
        i += 1
    return bytes(out[:n])


def main(root: Path) -> None:
    spec = importlib.util.spec_from_file_location("bam_emit_reference", root / "fq2bam-meth" / "python" / "bam_emit.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    res = {"block": mod._MAX_UNCOMPRESSED, "eof": mod._BGZF_EOF.hex(), "cases": []}
    for kind, n in CASES:
        data = stream(kind, n)
        entry = {"kind": kind, "n": n, "levels": {}}
        for level in (0, 1):
            with tempfile.TemporaryDirectory() as d:
                w = mod._BgzfWriter(str(Path(d) / "o.bgzf"), level=level, threads=1)
                w.write(data)
                w.close()
                blob = (Path(d) / "o.bgzf").read_bytes()
            entry["levels"][str(level)] = {"size": len(blob), "sha256": hashlib.sha256(blob).hexdigest(),
                                           "member_sizes": []}
            off = 0
            while off < len(blob):
                bsize = int.from_bytes(blob[off + 16:off + 18], "little")
                entry["levels"][str(level)]["member_sizes"].append(bsize + 1)
                off += bsize + 1
        res["cases"].append(entry)
    OUT.write_text(json.dumps(res, indent=0) + "\n")
    print(f"wrote {OUT}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <mojo-align source tree>")
    main(Path(sys.argv[1]))
