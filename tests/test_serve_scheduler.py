"""The served form's host logic, on CPU (scheduler-test mode: no device).

In this mode a launch group's "mapping" is a host function of each read in
the merged batch (rid = length, pos = FNV-1a of the converted read, nm = the
mate's hash, flag = 128 for second mates, mapq = seed_len), so these tests
check what the GPU path shares with it: admission against the budget,
merging of requests into groups, splitting of large requests, the batch
layout (a mate's row is found across the merge), and the scatter of every
result back to its own request's rows.
"""
from __future__ import annotations

import threading

import numpy as np
import pytest

from mojoalign_b200 import FmParams, MojoAlignError
from mojoalign_b200._lib import MA_ERR_ARG, MA_ERR_NOMEM
from mojoalign_b200.fastq import convert
from mojoalign_b200.serve import Server


def fnv(b: bytes) -> int:
    h = 2166136261
    for c in b:
        h = ((h ^ c) * 16777619) & 0xFFFFFFFF
    return h


def make_request(rng, n1, paired, max_len, min_len=20):
    n_seq = n1 * (2 if paired else 1)
    lens = rng.integers(min_len, max_len + 1, n_seq).astype(np.uint32)
    alphabet = np.frombuffer(b"ACGTNacgt", dtype=np.uint8)
    bases = alphabet[rng.integers(0, alphabet.size, (n_seq, max_len))].astype(np.uint8)
    return bases, lens


def expected(bases, lens, n1, paired, bs_r1, bs_r2, params):
    n_seq = n1 * (2 if paired else 1)
    h = np.array([fnv(convert(bytes(bases[i, :lens[i]]), bs_r1 if i < n1 else bs_r2)) for i in range(n_seq)],
                 dtype=np.uint32)
    e = {
        "rid": lens.astype(np.int32),
        "pos": h,
        "mapq": np.full(n_seq, params.seed_len, np.uint32),
        "flag": np.where(np.arange(n_seq) >= n1, 128, 0).astype(np.int32),
        "sl": np.zeros(n_seq, np.uint32),
        "sr": np.zeros(n_seq, np.uint32),
        "nm": (np.concatenate([h[n1:], h[:n1]]) if paired else np.zeros(n_seq, np.uint32)).astype(np.uint32),
    }
    return e


def check_result(res, exp):
    for f, v in exp.items():
        np.testing.assert_array_equal(getattr(res, f), v, err_msg=f)


def test_merge_split_and_scatter():
    rng = np.random.default_rng(5)
    p1 = FmParams()
    p2 = FmParams(seed_len=21)
    shapes = [(1, True, 150, "C2T", "G2A", p1), (37, True, 100, "C2T", "G2A", p1), (5000, True, 300, "G2A", "C2T", p1),
              (700, False, 64, "C2T", "", p1), (3, True, 40, "", "", p1), (2600, True, 151, "C2T", "G2A", p2),
              (1, False, 1024, "C2T", "", p2), (999, True, 33, "C2T", "G2A", p1)]
    with Server(None, None, hbm_budget_bytes=64 << 20, max_group_pairs=1024, max_inflight=3,
                scheduler_test=True) as srv:
        subs = []
        for n1, paired, ml, b1, b2, prm in shapes:
            bases, lens = make_request(rng, n1, paired, ml)
            subs.append((srv.submit(bases, lens, n1, paired, ml, b1, b2, prm), (bases, lens, n1, paired, b1, b2, prm)))
        for t, (bases, lens, n1, paired, b1, b2, prm) in subs:
            check_result(srv.wait(t, 60_000), expected(bases, lens, n1, paired, b1, b2, prm))
        st = srv.stats()
    assert st["requests_completed"] == len(shapes) and st["requests_failed"] == 0
    assert st["reads_completed"] == sum(n * (2 if p else 1) for n, p, *_ in shapes)
    assert st["parts_issued"] > len(shapes)  # large requests were split over groups
    assert st["max_requests_in_group"] >= 2  # and small ones merged
    assert st["peak_bytes"] <= st["budget_bytes"]


def test_alone_equals_mixed():
    rng = np.random.default_rng(11)
    p = FmParams()
    target = make_request(rng, 3000, True, 150)
    with Server(None, None, hbm_budget_bytes=32 << 20, max_group_pairs=4096, scheduler_test=True) as srv:
        alone = srv.wait(srv.submit(*target, 3000, True, 150, "C2T", "G2A", p))
    with Server(None, None, hbm_budget_bytes=32 << 20, max_group_pairs=2048, scheduler_test=True) as srv:
        others = [srv.submit(*make_request(rng, n, True, ml), n, True, ml, "C2T", "G2A", p)
                  for n, ml in ((500, 100), (10, 250), (1200, 150))]
        t = srv.submit(*target, 3000, True, 150, "C2T", "G2A", p)
        others += [srv.submit(*make_request(rng, n, True, ml), n, True, ml, "C2T", "G2A", p)
                   for n, ml in ((77, 90), (4000, 120))]
        mixed = srv.wait(t)
        srv.drain(60_000)
        assert srv.stats()["max_requests_in_group"] >= 2
    for f in mixed.FIELDS:
        np.testing.assert_array_equal(getattr(mixed, f), getattr(alone, f), err_msg=f)


def test_admission_waits_for_memory():
    rng = np.random.default_rng(2)
    p = FmParams()
    # a budget that holds one 512-pair group of 300-base pairs (about 0.75 MiB), not two
    with Server(None, None, hbm_budget_bytes=1 << 20, max_group_pairs=512, max_inflight=3,
                scheduler_test=True) as srv:
        reqs = [make_request(rng, 2000, True, 300) for _ in range(3)]
        ts = [srv.submit(b, l, 2000, True, 300, "C2T", "G2A", p) for b, l in reqs]
        for t, (b, l) in zip(ts, reqs):
            check_result(srv.wait(t), expected(b, l, 2000, True, "C2T", "G2A", p))
        st = srv.stats()
    assert st["peak_bytes"] <= st["budget_bytes"] == 1 << 20
    assert st["max_groups_in_flight"] == 1 and st["groups_issued"] >= 12


def test_submit_from_threads_and_latencies():
    p = FmParams()
    results = {}
    with Server(None, None, hbm_budget_bytes=32 << 20, max_group_pairs=2048, scheduler_test=True) as srv:
        def worker(k):
            rng = np.random.default_rng(100 + k)
            for j in range(6):
                n1 = int(rng.integers(1, 1500))
                b, l = make_request(rng, n1, True, 120)
                t = srv.submit(b, l, n1, True, 120, "C2T", "G2A", p)
                results[(k, j)] = (t, b, l, n1)

        th = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        srv.drain(60_000)
        for t, b, l, n1 in results.values():
            check_result(t.result, expected(b, l, n1, True, "C2T", "G2A", p))
        ids, reads, ms = srv.latencies()
    assert ids.size == 24 and np.all(ms >= 0)
    assert int(reads.sum()) == sum(2 * r[3] for r in results.values())


def test_errors():
    rng = np.random.default_rng(3)
    p = FmParams()
    with Server(None, None, hbm_budget_bytes=1 << 20, scheduler_test=True) as srv:
        b, l = make_request(rng, 4, True, 50)
        l[3] = 51
        with pytest.raises(MojoAlignError) as e:
            srv.submit(b, l, 4, True, 50)
        assert e.value.code == MA_ERR_ARG
        srv.wait(srv.submit(*make_request(rng, 1, True, 1024), 1, True, 1024))
        t = srv.submit(np.zeros((0, 10), np.uint8), np.zeros(0, np.uint32), 0, True, 10)
        assert srv.done(t)
    with Server(None, None, hbm_budget_bytes=4096, scheduler_test=True) as srv:
        with pytest.raises(MojoAlignError) as e:
            srv.submit(*make_request(rng, 1, True, 1024), 1, True, 1024)
        assert e.value.code == MA_ERR_NOMEM
    with pytest.raises(MojoAlignError):
        Server(None, None, hbm_budget_bytes=0, scheduler_test=True)
