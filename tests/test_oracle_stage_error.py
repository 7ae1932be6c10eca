"""Bounds on the error of every distance stage against exact FP64 (measured in
stage_error.py on nearest-neighbour pairs at the benchmark mixtures' full
density)."""
import numpy as np
import pytest

import stage_error


@pytest.mark.parametrize("name", stage_error.WORKLOAD_NAMES)
def test_distance_stage_errors(name):
    r = stage_error.distance_errors(name, queries=60)
    assert r["pairs"] > 1000
    d = {"blobs_10m_d12": 12, "blobs_20m_d128": 128, "blobs_50m_d96": 96}[name]
    u = 2.0 ** -24
    # sequential FP32 sum of d rounded squares: at most about d units in the
    # last place of the sum; measured far below
    assert r["fp32_diffsum"]["max"] <= d * u
    assert r["fp32_diffsum"]["p99"] <= 1e-6
    # float accumulation of exact double squares, then sqrtf: half the
    # relative error of the sum plus one rounding
    assert r["sqrt_l2"]["max"] <= d * u
    # the 16-bit forms lose accuracy in proportion to (|a|^2 + |c|^2) / |a - c|^2;
    # FP16's three extra mantissa bits give about 8x less error
    assert r["fp16_form"]["median"] < r["bf16_form"]["median"] / 4
    assert r["bf16_form"]["max"] < 0.25
    assert r["cancellation"]["median"] > 10


def test_fix_distances_and_clique_share_the_recipe(oracle):
    rng = np.random.default_rng(3)
    X = (rng.normal(size=(300, 24)) * 5).astype(np.float32)
    ids = np.stack([rng.choice(np.delete(np.arange(300), i), 8, replace=False)
                    for i in range(300)]).astype(np.int32)
    fd = oracle.fix_distances(X, ids)
    for i in range(0, 300, 37):
        for j in range(8):
            assert np.float32(oracle.euclid_ref(X[i], X[ids[i, j]])) == fd[i, j]


def test_stability_fp32_against_fp64():
    s = stage_error.stability_errors("blobs_10m_d12", n=6000)
    assert s["clusters"] >= 10
    assert s["stability_rel_max"] < 1e-4
    assert s["label_diffs"] <= s["points"] // 100
