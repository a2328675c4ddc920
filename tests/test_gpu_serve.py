"""Served form on the GPU: every request's outputs equal the oracle's for it
alone, whatever it was merged with, split into, or overlapped by.

Requests come from several simulated samples (different CpG retention,
fixed and lognormal length profiles, paired and single-end, different
bisulfite modes) and are submitted together so that launch groups merge
requests and split the large ones over several groups.  Integer work: the
tolerance is zero.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from mojoalign_b200 import FmParams, GpuContext, GpuIndex, map_batch, synth
from mojoalign_b200.serve import Server

pytestmark = pytest.mark.gpu

FIELDS = ("rid", "pos", "mapq", "flag", "sl", "sr", "nm")


@pytest.fixture(scope="module")
def ctx():
    c = GpuContext(0)
    yield c
    c.close()


def sample_requests(fa):
    out = []
    specs = [  # (n1, paired, max_len, model, bs_r1, bs_r2, seed)
        (1500, True, 150, synth.ReadModel(cpg_retain=0.4), "C2T", "G2A", 21),
        (37, True, 150, synth.ReadModel(cpg_retain=0.9), "C2T", "G2A", 22),
        (2200, False, 300, synth.ReadModel(len_fixed=0, non_directional=0.5), "C2T", "", 23),
        (5, False, 120, synth.ReadModel(len_fixed=0, len_max=120), "G2A", "", 24),
        (900, True, 250, synth.ReadModel(len_fixed=250, sub_rate=0.02), "C2T", "G2A", 25),
        (1, True, 150, synth.ReadModel(), "C2T", "G2A", 26),
        (3100, True, 100, synth.ReadModel(len_fixed=100, cpg_retain=0.6), "C2T", "G2A", 27),
    ]
    for n1, paired, ml, model, b1, b2, seed in specs:
        rb = synth.simulate_reads(fa, model, n1, paired, ml, seed=seed)
        out.append((rb.bases, rb.lens, n1, paired, ml, b1, b2))
    return out


def oracle_map(prefix, req, params):
    bases, lens, n1, paired, ml, b1, b2 = req
    bsm = {"": 0, "C2T": 1, "G2A": 2}
    return oracle.OracleIndex(prefix).map(bases, lens, n1, paired, ml, bsm[b1], bsm[b2], params.as_list())


@pytest.mark.parametrize("tuning", [None, (0, 1, 0, 1, 16, 32), (2, 1, 0, 1, 1, 1, 32, 4, 0),
                                    (3, 1, 0, 2, 1, 1, 8, 4, 0, 1), (4, 1, 0, 2, 1, 1, 8, 4, 0, 1)])
def test_served_requests_match_oracle(ctx, small_ref, tuning):
    fa, prefix = small_ref
    gi = GpuIndex(ctx, prefix, kmer_k=12, kmer3_k=12)
    params = FmParams()
    reqs = sample_requests(fa)
    if tuning:
        ctx.set_tuning(*tuning)
    try:
        with Server(ctx, gi, hbm_budget_bytes=256 << 20, max_group_pairs=1024, max_inflight=3) as srv:
            tickets = [srv.submit(b, l, n1, pr, ml, b1, b2, params) for b, l, n1, pr, ml, b1, b2 in reqs]
            srv.drain(120_000)
            st = srv.stats()
            for t, req in zip(tickets, reqs):
                got = srv.wait(t)
                exp = oracle_map(prefix, req, params)
                for f in FIELDS:
                    bad = np.nonzero(getattr(got, f) != exp[f])[0]
                    assert bad.size == 0, f"request {t.id} {f}: {bad.size} reads differ, first {bad[0]}"
    finally:
        ctx.set_tuning()
        gi.close()
    assert st["requests_completed"] == len(reqs) and st["requests_failed"] == 0
    assert st["max_requests_in_group"] >= 2 and st["parts_issued"] > len(reqs)


def test_alone_equals_mixed_and_plain(ctx, small_ref):
    fa, prefix = small_ref
    gi = GpuIndex(ctx, prefix, kmer_k=12, kmer3_k=12)
    params = FmParams()
    reqs = sample_requests(fa)
    target = reqs[0]
    try:
        with Server(ctx, gi, hbm_budget_bytes=128 << 20, max_group_pairs=4096) as srv:
            alone = srv.wait(srv.submit(*target[:5], target[5], target[6], params))
        with Server(ctx, gi, hbm_budget_bytes=128 << 20, max_group_pairs=700, max_inflight=2) as srv:
            ts = [srv.submit(b, l, n1, pr, ml, b1, b2, params) for b, l, n1, pr, ml, b1, b2 in reqs[::-1]]
            mixed = srv.wait(ts[-1])
            srv.drain(120_000)
        plain = map_batch(ctx, gi, *target[:5], target[5], target[6], params)
    finally:
        gi.close()
    for f in FIELDS:
        np.testing.assert_array_equal(getattr(mixed, f), getattr(alone, f), err_msg=f)
        np.testing.assert_array_equal(getattr(plain, f), getattr(alone, f), err_msg=f)
