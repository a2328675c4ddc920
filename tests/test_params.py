"""Env knobs of the FM engine (linear_gpu_fm.mojo:2074-2082) parsed like
_env_int (linear_gpu_locate.mojo:139-145)."""
from __future__ import annotations

import pytest

from mojoalign_b200.params import BENCH_PARAMS, ENV_NAMES, FmParams, env_int


def test_defaults_and_overrides():
    assert FmParams.from_env({}) == FmParams()
    env = {"METHYLGRAPHER_FM_SEED_LEN": "19", "METHYLGRAPHER_FM_MAX_OCC": "500"}
    assert FmParams.from_env(env) == BENCH_PARAMS


def test_values_below_one_mean_default():
    for field, (name, default) in ENV_NAMES.items():
        assert getattr(FmParams.from_env({name: "0"}), field) == default
        assert getattr(FmParams.from_env({name: "-5"}), field) == default


def test_non_integer_raises():
    with pytest.raises(ValueError):
        env_int("X", 3, {"X": "abc"})


def test_c_struct_order():
    p = FmParams(1, 2, 3, 4, 5, 6, 7).to_c()
    assert [p.seed_len, p.seed_stride, p.max_occ, p.max_diff, p.max_soft, p.max_adj, p.rescue_win] == \
        [1, 2, 3, 4, 5, 6, 7]
