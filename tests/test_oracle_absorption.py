"""The Absorption recorder in the oracle (src/absortion.cpp:54-91, called from
src/simulation.cpp:589-592).

The reference's own grids (tests/golden/ref_*_absorption_*.npz, made by
``make_golden.py absorption``) pin the restatement bit for bit on both streams: a
time-resolved grid over the two-layer slab and a time-integrated one over the
mixture slab.  A semi-infinite medium also checks the energy balance the deposits
close: absorbed + reflected weight per photon is 1 within its Monte Carlo error.
"""
import copy
import os

import numpy as np
import pytest

from luminis_mc_b200 import workloads as W
from oracle import pyoracle as O
from tests.golden.make_golden import absorption_scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
SCENES = {s["name"]: s for s in absorption_scenes()}


@pytest.mark.parametrize("name", sorted(SCENES))
@pytest.mark.parametrize("stream", ["xoshiro", "philox"])
def test_oracle_absorption_reproduces_reference_bit_for_bit(name, stream):
    spec = SCENES[name]
    g = np.load(os.path.join(GOLDEN, f"ref_{stream}_{name}.npz"))
    rng = "xoshiro" if stream == "xoshiro" else "philox_u53"
    res = O.Oracle(spec).run(spec["n_photons"], spec["seed"], rng=rng)
    np.testing.assert_array_equal(res.absorption, g["absorption"])
    for i, t in enumerate(res.tallies):
        np.testing.assert_array_equal(t, g[f"sensor{i}"], err_msg=f"sensor {i}")


def test_time_slices_partition_the_integrated_slice():
    spec = SCENES["absorption_bilayer"]
    res = O.Oracle(spec).run(400, 3)
    a = res.absorption
    assert a.shape == (11, 21, 31)
    # every deposit of this scene arrives before t_max, so slices 1.. sum to slice 0
    np.testing.assert_allclose(a[1:].sum(axis=0), a[0], rtol=1e-12, atol=1e-15)


def test_absorbed_plus_reflected_weight_is_one():
    """Semi-infinite Mie medium with albedo ~0.91: every photon's weight ends as
    deposits or as the weight it carries out through the absorbing plane at z = 0.
    Russian roulette keeps that balance in expectation, and the weights it plays
    with are below 1e-4, so the sum is 1 to ~1e-5 per photon."""
    spec = copy.deepcopy(W.mie_cbs_small(4000, 77))
    spec["media"][0].update(mu_a=1.0)
    spec["sensors"] = [{"kind": "planar_fluence", "z": 0.0, "len_x": 400.0, "len_y": 400.0,
                        "len_t": 0.0, "dx": 400.0, "dy": 400.0, "d_t": 0.0, "absorb": True}]
    spec["absorption"] = {"radius": 200.0, "depth": 200.0, "d_r": 200.0, "d_z": 200.0}
    n = spec["n_photons"]
    res = O.Oracle(spec).run(n, spec["seed"], records=True)
    r = res.records
    absorbed = float(res.absorption.sum())
    reflected = float(r["weight"][r["fate"] == 1].sum())
    assert res.stats["cap"] == 0 and res.stats["detected"] + res.stats["roulette"] == n
    assert abs((absorbed + reflected) / n - 1.0) < 1e-4
