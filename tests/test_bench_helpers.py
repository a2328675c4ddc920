"""The bench's own bookkeeping (CPU): parity failures stop the run, the
contract keys lead the JSON line, the seeding roofline arithmetic, and the
per-rank read cap."""
from __future__ import annotations

import importlib.util
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
spec = importlib.util.spec_from_file_location("bench", ROOT / "bench.py")
bench = importlib.util.module_from_spec(spec)
spec.loader.exec_module(bench)


def test_parity_failures_found_anywhere():
    line = {"parity_sample": {"reads": 10, "mismatched_fields": 0},
            "forms": {"batched": {"equals_plain": True}, "served": {"equals_plain": False}},
            "stages": {"bam": {"parity": {"records": 5, "bytes_identical": True}},
                       "sam": {"parity": {"sam_file_identical": False}}}}
    bad = bench.parity_failures(line)
    assert "forms.served.equals_plain" in bad
    assert "stages.sam.parity.sam_file_identical" in bad
    assert len(bad) == 2
    line["parity_sample"]["mismatched_fields"] = 3
    assert "parity_sample.mismatched_fields=3" in bench.parity_failures(line)


def test_line_order_puts_contract_and_parity_first():
    line = {"forms": {}, "roofline": {}, "value": 1.0, "metric": "m", "parity_sample": {"reads": 1},
            "parity_failures": [], "unit": "u"}
    keys = list(bench.ordered_line(line))
    assert keys[:3] == ["metric", "value", "unit"]
    assert keys.index("parity_sample") < keys.index("roofline")
    assert set(keys) == set(line)


def test_seeding_roofline_arithmetic():
    tally = [10 ** 9, 5 * 10 ** 8, 2 * 10 ** 8] + [0] * 9
    tally2 = [10 ** 8, 0, 0] + [0] * 6 + [500] + [0] * 2
    wave = [[20.0, 10.0, 5.0, 5.0, 3.0], [20.0, 10.0, 5.0, 5.0, 3.0]]
    r = bench.seeding_roofline(tally, wave, tally2, 1000)["seeding"]
    assert r["alg_bytes"] == 32 * 16 * 10 ** 8  # the stage-2 warps' gathers are not the rounds'
    assert abs(r["achieved_GBs"] - 32 * 16 * 10 ** 8 / 0.020 / 1e9) < 0.1
    assert r["stage2_ms"] == 3.0 and r["stage2_reads_per_read"] == 0.5
    line = {"roofline": {"seeding": r}, "gather_roofline": {"hbm_32B_GBs": 800.0, "hbm_64B_GBs": 900.0}}
    bench.add_gather_fractions(line)
    assert line["roofline"]["seeding"]["frac_of_gather32"] == round(r["achieved_GBs"] / 800.0, 4)
    assert bench.seeding_roofline(tally, []) == {}


def test_host_capped_reads():
    assert bench.host_capped_reads(1000, 300, 1) == 1000
    assert bench.host_capped_reads(10 ** 15, 300, 8) < 10 ** 15
    assert bench.host_capped_reads(10 ** 15, 300, 8) >= 1
