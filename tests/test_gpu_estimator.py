"""Estimator-mode FarFieldCBS on the GPU: the last-flight CBS estimate at every
scattering vertex (FarFieldCBSSensor::process_estimation).

* FP64 against the reference's own tallies on the Philox stream
  (tests/golden/ref_philox_estimator_*.npz: one Mie medium with the 100-bin grid; the
  two-layer slab with time bins, a 2-D grid and a theta cap), 1e-9 of each sensor's
  largest bin, hit counts exact.
* FP32 transport (the estimate itself is binary64) against the oracle on the u24
  stream: 5 % of the largest bin, the FP32 tally tolerance of the parity tests.
* The public API accumulates the estimator tallies like the reference.
"""
import os

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.device import DeviceRun
from oracle import pyoracle as O
from tests.golden.make_golden import estimator_scenes

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("spec", estimator_scenes(), ids=lambda s: s["name"])
def test_gpu_fp64_estimator_reproduces_reference(spec, cuda):
    g = np.load(os.path.join(GOLDEN, f"ref_philox_{spec['name']}.npz"))
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    st, _ = run.run(spec["n_photons"], spec["seed"], precision="fp64")
    assert st["error_flags"] == 0
    for i, t in enumerate(run.host_tallies()):
        ref = g[f"sensor{i}"]
        np.testing.assert_allclose(t, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max(),
                                   err_msg=f"sensor {i}")
        assert st["hits"][i] == g["hits"][i]
    run.close()


@pytest.mark.parametrize("spec", estimator_scenes(), ids=lambda s: s["name"])
def test_gpu_fp32_estimator_matches_oracle(spec, cuda):
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    run.run(spec["n_photons"], spec["seed"], precision="fp32")
    ref = O.Oracle(spec).run(spec["n_photons"], spec["seed"], rng="philox_u24")
    for t, o in zip(run.host_tallies(), ref.tallies):
        scale = max(float(np.abs(o).max()), 1e-300)
        assert float(np.abs(t - o).max()) <= 5e-2 * scale
    run.close()


def test_public_api_estimator_accumulates(cuda):
    spec = estimator_scenes()[0]
    cfg, hs, keep = W.build(lm, spec)
    lm.run_simulation_parallel(cfg, precision="fp64")
    g = np.load(os.path.join(GOLDEN, f"ref_philox_{spec['name']}.npz"))
    got = W.tally_arrays(hs[0], "farfield_cbs")
    np.testing.assert_allclose(got, g["sensor0"], rtol=1e-9, atol=1e-9 * np.abs(g["sensor0"]).max())
    assert hs[0].hits == g["hits"][0]
