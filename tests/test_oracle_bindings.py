"""The oracle's ctypes bindings (oracle/__init__.py) against the C
definitions in oracle/*.c: every bound function exists with the declared
number of parameters."""
from __future__ import annotations

import re
from pathlib import Path

import oracle

ORACLE = Path(__file__).resolve().parents[1] / "oracle"


def defined_arity() -> dict[str, int]:
    out = {}
    for f in ORACLE.glob("*.c"):
        text = re.sub(r"/\*.*?\*/", "", f.read_text(), flags=re.S)
        for m in re.finditer(r"^[a-z_0-9 ]*?\b(orc_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*\{", text, flags=re.S | re.M):
            args = m.group(2).strip()
            out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_bindings_match_definitions():
    arity = defined_arity()
    assert len(arity) >= 15
    checked = 0
    for name, n in arity.items():
        fn = getattr(oracle.lib, name, None)
        assert fn is not None, name
        if fn.argtypes is not None:
            assert len(fn.argtypes) == n, f"{name}: {len(fn.argtypes)} ctypes arguments, C defines {n}"
            checked += 1
    assert checked >= 10
