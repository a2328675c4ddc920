"""The pinned host buffer pool of the file pipelines (mojoalign_b200.pinned):
reuse of the smallest free buffer that fits, ownership between take() and
give(), the size limit.  Page-locking needs a GPU driver, so the allocation
is replaced by a plain one here."""
from __future__ import annotations

import threading

import pytest
import torch

from mojoalign_b200 import pinned


@pytest.fixture
def pool(monkeypatch):
    made = []
    real_empty = torch.empty

    def fake_empty(n, dtype=None, pin_memory=False):
        assert pin_memory
        t = real_empty(n, dtype=dtype)
        made.append(t)
        return t

    monkeypatch.setattr(torch, "empty", fake_empty)
    pinned.release()
    pinned.set_limit(8 << 30)
    yield made
    pinned.release()
    pinned.set_limit(8 << 30)


def test_reuse_smallest_fit(pool):
    a, b = pinned.take(100), pinned.take(1000)
    assert len(pool) == 2 and a.numel() == 100 and b.numel() == 1000
    pinned.give(b)
    pinned.give(a)
    c = pinned.take(50)  # the 100-byte buffer, not the 1000-byte one
    assert c is a and len(pool) == 2
    d = pinned.take(500)
    assert d is b
    e = pinned.take(500)  # nothing free fits: a new buffer
    assert len(pool) == 3 and e.numel() == 500
    pinned.give(None)  # ignored


def test_limit_drops_the_largest(pool):
    pinned.set_limit(1500)
    bufs = [pinned.take(n) for n in (400, 700, 900)]
    for t in bufs:
        pinned.give(t)
    free = [t.numel() for t in pinned._FREE]
    assert sum(free) <= 1500 and 400 in free and 900 not in free


def test_threads_never_share_a_buffer(pool):
    pinned.give(pinned.take(10))
    got, lock = [], threading.Lock()

    def work():
        for _ in range(200):
            t = pinned.take(10)
            with lock:
                assert all(t is not x for x in got)
                got.append(t)
            with lock:
                got.remove(t)
            pinned.give(t)

    ts = [threading.Thread(target=work) for _ in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
