"""Seeded FASTQ texts for the record-split tests: names with and without '@',
spaces and '/', CRLF and LF line ends (and doubled '\\r'), empty SEQ lines,
reads up to a few kb, arbitrary quality bytes, optionally an unterminated
last line."""
from __future__ import annotations

import numpy as np


def random_fastq(seed: int, n: int, *, crlf: float = 0.2, max_len: int = 400, terminated: bool = True) -> bytes:
    rng = np.random.default_rng(seed)
    out = []
    letters = np.frombuffer(b"ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789:_-.", np.uint8)
    for i in range(n):
        nl = b"\r\n" if rng.random() < crlf else (b"\r\r\n" if rng.random() < 0.01 else b"\n")
        name = letters[rng.integers(0, letters.size, size=int(rng.integers(0, 40)))].tobytes()
        u = rng.random()
        if u < 0.1:
            name += b" " + letters[rng.integers(0, letters.size, size=8)].tobytes()
        elif u < 0.2:
            name += b"/" + bytes([49 + (i & 1)])
        elif u < 0.25:
            name += b"\t1:N:0"
        head = (b"@" if rng.random() < 0.97 else b"") + name
        q = int(rng.choice([0, 1, 36, 100, 150, 151, 250, max_len], p=[.02, .01, .07, .2, .4, .1, .15, .05]))
        if rng.random() < 0.01:
            q = int(rng.integers(1000, 5000))
        seq = np.frombuffer(b"ACGTNacgt", np.uint8)[rng.integers(0, 9, size=q)].tobytes()
        qual = rng.integers(33, 127, size=q, dtype=np.uint8).tobytes()
        if rng.random() < 0.02:
            qual = qual[: max(0, q - 3)]
        plus = b"+" if rng.random() < 0.9 else b"+" + name
        out.append(head + nl + seq + nl + plus + nl + qual + nl)
    text = b"".join(out)
    if not terminated and text.endswith(b"\n"):
        text = text[:-1]
    return text
