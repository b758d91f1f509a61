"""The likelihood-ratio estimator of the oracle (oracle/lmc_oracle.c, adjoint
outputs) against central finite differences with common random numbers.

Scene: the two-layer HG slab (g = 0.8 over g = 0.9, mu_a raised to 0.5/mm to keep
paths short) with a FarFieldCBS and a PlanarFluence sensor at z = 0.  Outputs: the
total S0 of the fluence grid, its radial profile and the CBS S0 grids.  For each of
the 8 parameters (mu_a, mu_s, mean free path, g of both media) the replica mean of
the LR derivative must agree with the replica mean of (T(p+h) - T(p-h)) / 2h,
h = 1 % of the parameter, within the combined standard error: both are unbiased
for the same derivative (the O(h^2) bias of the difference is far below the noise).
"""
import copy

import numpy as np
import pytest

from luminis_mc_b200 import workloads as W
from oracle import pyoracle as O

R, N, H = 8, 4000, 0.01


def adjoint_scene():
    spec = W.bilayer_hg(0, 1)
    spec["name"] = "adjoint_bilayer_hg"
    spec["sensors"] = [
        {"kind": "farfield_cbs", "theta_max": 0.5, "phi_max": 2 * W.PI, "len_t": 0.0,
         "d_theta": 0.1, "d_phi": 2 * W.PI, "d_t": 0.0, "theta_limit": (0.0, 0.5)},
        {"kind": "planar_fluence", "z": 0.0, "len_x": 10.0, "len_y": 10.0, "len_t": 0.0,
         "dx": 0.5, "dy": 0.5, "d_t": 0.0, "absorb": True}]
    for m in spec["media"]:
        m["mu_a"] = 0.5
    return spec


def perturbed(spec, medium, name, factor):
    sp = copy.deepcopy(spec)
    if name == "g":
        ph = sp["media"][medium]["phase"]
        sp["phases"][ph]["g"] *= factor
    else:
        sp["media"][medium][name] *= factor
    return sp


def base_value(spec, medium, name):
    if name == "g":
        return spec["phases"][spec["media"][medium]["phase"]]["g"]
    return spec["media"][medium][name]


def outputs(spec, seed):
    return O.Oracle(spec).run_adjoint(N, seed, radial_sensor=1, radial_bins=10,
                                      radial_max=5.0)[1] / N


def test_adjoint_layout():
    spec = adjoint_scene()
    res, out = O.Oracle(spec).run_adjoint(500, 3, radial_sensor=1, radial_bins=10, radial_max=5.0)
    assert out.shape == (1 + 4 * 2, 1 + 10 + 2 * 5)
    # the total is the sum of the fluence sensor's time-integrated S0 grid
    np.testing.assert_allclose(out[0, 0], res.tallies[1][0, 0].sum(), rtol=1e-12)
    # S0 coherent / incoherent rows are the CBS sensor's own S0 grids
    np.testing.assert_allclose(out[0, 11:16], res.tallies[0][0].ravel(), rtol=1e-12)
    np.testing.assert_allclose(out[0, 16:21], res.tallies[0][4].ravel(), rtol=1e-12)
    # the radial profile partitions the hits with r < 5 mm
    assert out[0, 1:11].sum() <= out[0, 0] * (1 + 1e-12)


def test_adjoint_without_sensors_is_rejected():
    spec = adjoint_scene()
    with pytest.raises(ValueError):
        O.Oracle(spec).run_adjoint(10, 1, radial_sensor=0)     # sensor 0 is not a fluence sensor


@pytest.mark.parametrize("name", ["mu_a", "mu_s", "mfp", "g"])
def test_lr_matches_crn_finite_differences(name):
    spec = adjoint_scene()
    zs = []
    for medium in range(2):
        v = base_value(spec, medium, name)
        plus, minus = perturbed(spec, medium, name, 1 + H), perturbed(spec, medium, name, 1 - H)
        lr, fd = [], []
        for r in range(R):
            seed = 100 + r
            lr.append(outputs(spec, seed)[1 + 4 * medium + ("mu_a", "mu_s", "mfp", "g").index(name)])
            fd.append((outputs(plus, seed)[0] - outputs(minus, seed)[0]) / (2 * H * v))
        lr, fd = np.array(lr), np.array(fd)
        for idx in (0, 1, 2, 4, 11):          # total, radial bins 0, 1, 3, CBS S0 coherent bin 0
            a, b = lr[:, idx], fd[:, idx]
            se = np.sqrt(a.var(ddof=1) / R + b.var(ddof=1) / R)
            if se == 0:
                assert a.mean() == pytest.approx(b.mean(), abs=1e-12)
                continue
            zs.append((a.mean() - b.mean()) / se)
    zs = np.array(zs)
    assert np.all(np.abs(zs) < 4.5), zs
    assert np.mean(zs ** 2) < 3.0, zs
