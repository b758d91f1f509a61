"""StatisticsSensor in the oracle (src/detector.cpp:1569-1888).

The reference's own histograms (tests/golden/ref_*_stats_*.npz, made by
``make_golden.py statistics``) pin the restatement bit for bit on both streams: all
six histograms with time windows beside a FarFieldCBS sensor, a non-absorbing sensor
inside the sample that a photon may cross many times (backward crossings only), and
theta / event filters.
"""
import os

import numpy as np
import pytest

from oracle import pyoracle as O
from tests.golden.make_golden import statistics_scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
SCENES = {s["name"]: s for s in statistics_scenes()}


@pytest.mark.parametrize("name", sorted(SCENES))
@pytest.mark.parametrize("stream", ["xoshiro", "philox"])
def test_oracle_statistics_reproduce_reference_bit_for_bit(name, stream):
    spec = SCENES[name]
    g = np.load(os.path.join(GOLDEN, f"ref_{stream}_{name}.npz"))
    rng = "xoshiro" if stream == "xoshiro" else "philox_u53"
    res = O.Oracle(spec).run(spec["n_photons"], spec["seed"], rng=rng)
    for i, t in enumerate(res.tallies):
        np.testing.assert_array_equal(t.ravel(), g[f"sensor{i}"].ravel(), err_msg=f"sensor {i}")
    np.testing.assert_array_equal(res.hits.astype(np.int64), g["hits"])


def test_statistics_layout_and_counts():
    """Each counted hit adds one to bin 0 of every time-resolved histogram it falls in;
    the time windows hold the hits that arrived before len_t."""
    spec = SCENES["stats_bilayer"]
    res = O.Oracle(spec).run(800, 9)
    h = res.tallies[1]
    n_t = 11                                   # ceil(20 / 2) + 1
    ev = h[:n_t * 200].reshape(n_t, 200)
    th = h[n_t * 200:n_t * 230].reshape(n_t, 30)
    assert th[0].sum() == res.hits[1]          # every exit at z = 0 has theta < pi / 2
    assert ev[0].sum() <= res.hits[1]          # longer paths fall past 200 events
    assert ev[1:].sum() <= ev[0].sum() and th[1:].sum() <= th[0].sum()
    assert h.size == n_t * (200 + 30 + 12 + 30) + 30 + 20
    inner = res.tallies[2]
    assert inner[:60].sum() <= res.hits[2] and inner.size == 100
