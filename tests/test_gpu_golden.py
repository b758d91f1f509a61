"""The GPU path against the reference's own tallies (tests/golden): the
unmodified reference drew the same Philox stream through the replay seam, so the
FP64 kernel must reproduce its tallies and hit counts (1e-9; 1e-6 for the
phase-sensitive speckle field)."""
import os

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.device import DeviceRun
from tests.golden.make_golden import golden_scenes

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("spec", golden_scenes(), ids=lambda s: s["name"])
def test_gpu_fp64_reproduces_reference_golden(spec, cuda):
    g = dict(np.load(os.path.join(GOLDEN, f"ref_philox_{spec['name']}.npz")))
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    stats, _ = run.run(spec["n_photons"], spec["seed"], precision="fp64")
    for i, (t, s) in enumerate(zip(run.host_tallies(), spec["sensors"])):
        ref = g[f"sensor{i}"]
        tol = 1e-6 if s["kind"] == "planar_field" else 1e-9
        np.testing.assert_allclose(t, ref, rtol=tol, atol=tol * np.abs(ref).max())
        assert stats["hits"][i] == g["hits"][i]
    run.close()


def test_gpu_farfield_fluence_matches_reference_records(cuda):
    """FarFieldFluence (no reference class) against its definition applied to the
    reference's own photon records (tests/golden/ref_farfield_fluence_small.npz)."""
    from tests.golden.make_golden import farfield_scene
    spec = farfield_scene()
    ref = np.load(os.path.join(GOLDEN, "ref_farfield_fluence_small.npz"))["sensor0"]
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    run.run(spec["n_photons"], spec["seed"], precision="fp64")
    got = run.host_tallies()[0]
    np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())
    run.close()
