"""A process-wide pool of page-locked host buffers for the file pipelines.

Pinning memory costs far more than copying it (a few hundred ms per GB), and
the FASTQ -> SAM / BAM pipelines need GB-sized pinned buffers for their
FASTQ feeds and their output text on every call.  Buffers returned to the
pool are kept for the next call, up to `limit` bytes in total; `release()`
unpins them all.  Thread-safe: a buffer is owned by one caller between
take() and give().
"""
from __future__ import annotations

import threading

_LOCK = threading.Lock()
_FREE: list = []  # torch uint8 tensors, pinned
_LIMIT = [8 << 30]


def take(nbytes: int):
    """A pinned uint8 tensor of at least nbytes (the smallest free one that
    fits, else a new one)."""
    import torch

    nbytes = max(int(nbytes), 1)
    with _LOCK:
        best = None
        for i, t in enumerate(_FREE):
            if t.numel() >= nbytes and (best is None or t.numel() < _FREE[best].numel()):
                best = i
        if best is not None:
            return _FREE.pop(best)
    return torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)


def give(t) -> None:
    """Returns a buffer from take(); the largest free buffers beyond the
    pool's limit are dropped."""
    if t is None:
        return
    with _LOCK:
        _FREE.append(t)
        _FREE.sort(key=lambda x: x.numel())
        while _FREE and sum(x.numel() for x in _FREE) > _LIMIT[0]:
            _FREE.pop()


def set_limit(nbytes: int) -> None:
    with _LOCK:
        _LIMIT[0] = int(nbytes)
    give(None)


def release() -> None:
    """Unpins every free buffer."""
    with _LOCK:
        _FREE.clear()
