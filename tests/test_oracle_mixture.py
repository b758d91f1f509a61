"""MixtureLayer in the oracle (src/sample.cpp:41-104, src/simulation.cpp:297-614).

The reference's own tallies on mixture scenes (tests/golden/ref_*_mixture*.npz and
ref_philox_estimator_mixture.npz, made by ``make_golden.py mixture``) pin the
restatement: species drawn per vertex on the selection CDF, free paths with the
aggregate mean free path, interface crossings rescaled by the aggregate mu_t,
weights by the layer's albedo, and in estimator mode the layer albedo at the first
vertex and the species' own albedo afterwards.
"""
import copy
import os

import numpy as np
import pytest

from oracle import pyoracle as O
from tests.golden.make_golden import mixture_scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
SCENES = {s["name"]: s for s in mixture_scenes()}


@pytest.mark.parametrize("name,stream", [("mixture_bilayer_small", "xoshiro"),
                                         ("mixture_bilayer_small", "philox"),
                                         ("mixture_cbs_small", "xoshiro"),
                                         ("mixture_cbs_small", "philox"),
                                         ("estimator_mixture", "philox")])
def test_oracle_mixture_reproduces_reference_bit_for_bit(name, stream):
    spec = SCENES[name]
    g = np.load(os.path.join(GOLDEN, f"ref_{stream}_{name}.npz"))
    rng = "xoshiro" if stream == "xoshiro" else "philox_u53"
    res = O.Oracle(spec).run(spec["n_photons"], spec["seed"], rng=rng)
    for i, t in enumerate(res.tallies):
        np.testing.assert_array_equal(t, g[f"sensor{i}"], err_msg=f"sensor {i}")
    np.testing.assert_array_equal(res.hits.astype(np.int64), g["hits"])


def test_mixture_draws_one_uniform_per_vertex():
    """A one-species mixture draws a species uniform at every vertex that a
    HomogeneousLayer of the same medium does not: more draws, other histories."""
    spec = copy.deepcopy(SCENES["mixture_cbs_small"])
    spec["layers"] = [{"species": [0], "densities": [3.0e6], "z_min": 0.0, "z_max": float("inf")}]
    mix = O.Oracle(spec).run(300, 5)
    homo = dict(spec, layers=[{"medium": 0, "z_min": 0.0, "z_max": float("inf")}])
    hom = O.Oracle(homo).run(300, 5)
    # per vertex: species, theta and at least one (phi, accept) pair; per step: a path
    assert mix.stats["draws"] >= 4 * mix.stats["events"] + mix.stats["steps"]
    assert not all(np.array_equal(a, b) for a, b in zip(mix.tallies, hom.tallies))


def test_mixture_rejects_species_without_cross_section():
    spec = copy.deepcopy(SCENES["mixture_cbs_small"])
    spec["phases"][0] = {"kind": "hg", "g": 0.8}
    with pytest.raises(ValueError, match="scattering_cross_section"):
        O.Oracle(spec)


def test_mixture_rejects_nonpositive_total():
    spec = copy.deepcopy(SCENES["mixture_cbs_small"])
    spec["layers"][0]["densities"] = [0.0, 0.0]
    with pytest.raises(ValueError, match="total mu_s"):
        O.Oracle(spec)


def test_mixture_adjoint_is_refused():
    spec = SCENES["mixture_cbs_small"]
    with pytest.raises(ValueError):
        O.Oracle(spec).run_adjoint(10, 1)
