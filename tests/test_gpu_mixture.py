"""MixtureLayer on the GPU (src/sample.cpp:41-104, src/simulation.cpp:297-614).

* FP64 against the reference's own tallies on the Philox stream
  (tests/golden/ref_philox_mixture_*.npz, ref_philox_estimator_mixture.npz: a
  three-species slab over the Mie medium, a semi-infinite two-species mixture and
  estimator-mode FarFieldCBS in it), 1e-9 of each sensor's largest bin, hit counts
  exact.
* FP32 against the oracle on the u24 stream, 5 % of the largest bin (the FP32 tally
  tolerance of the parity tests); the species draw compares in binary64, so the
  photon histories stay those of the oracle.
* A sweep holding a mixture scene equals the lone run; likelihood-ratio outputs
  refuse mixtures (their scores model HomogeneousLayers only).
"""
import os

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.device import DeviceRun
from oracle import pyoracle as O
from tests.golden.make_golden import mixture_scenes

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("spec", mixture_scenes(), ids=lambda s: s["name"])
def test_gpu_fp64_mixture_reproduces_reference(spec, cuda):
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


@pytest.mark.parametrize("spec", mixture_scenes(), ids=lambda s: s["name"])
def test_gpu_fp32_mixture_matches_oracle(spec, cuda):
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    st, _ = run.run(spec["n_photons"], spec["seed"], precision="fp32")
    ref = O.Oracle(spec).run(spec["n_photons"], spec["seed"], rng="philox_u24")
    for t, o in zip(run.host_tallies(), ref.tallies):
        scale = max(float(np.abs(o).max()), 1e-300)
        assert float(np.abs(t - o).max()) <= 5e-2 * scale
    run.close()


def test_sweep_with_mixture_equals_lone_run(cuda):
    from luminis_mc_b200.sweep import SweepRun
    specs = [W.mixture_bilayer(0, 5), W.mie_cbs_small(0, 5), W.mixture_cbs_small(0, 5)]
    counts = [1200, 900, 1500]
    sw = SweepRun([W.build(lm, s)[0] for s in specs])
    sw.set_photons(counts)
    st = sw.run(17, precision="fp64")
    assert st["error_flags"] == 0
    for k, (spec, n, p0) in enumerate(zip(specs, counts, sw.offsets())):
        cfg, _, keep = W.build(lm, spec)
        run = DeviceRun(cfg)
        run.run(n, 17, int(p0), precision="fp64")
        for a, b in zip(sw.host_tallies(k), run.host_tallies()):
            np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12 * max(np.abs(b).max(), 1e-300))
        run.close()
    sw.close()


def test_adjoint_refuses_mixture_layers(cuda):
    from luminis_mc_b200.adjoint import AdjointTransport
    cfg, _, keep = W.build(lm, W.mixture_cbs_small(10, 1))
    with pytest.raises(NotImplementedError):
        AdjointTransport(cfg, radial_sensor=1)
