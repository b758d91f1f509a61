"""The reference's own objects, run on the GPU through the reference-side binding.

Each scene is built with the reference's Python API (its pybind module, built from its
sources under oracle/_ref), transported on the GPU by luminis_mc_b200.refbind in FP64
on the Philox stream, and its tallies are read back FROM THE REFERENCE'S OWN SENSOR
OBJECTS.  They must equal the tallies the unmodified reference produced on the same
stream through the replay seam (tests/golden/ref_philox_*.npz) to 1e-9 (1e-6 for the
phase-sensitive speckle field), with the same hit counts.  The reference's own
postprocess_farfield_cbs then runs on the GPU-filled sensor.
"""
import os
import sys

import numpy as np
import pytest

from luminis_mc_b200 import refbind
from luminis_mc_b200 import workloads as W
from oracle import pyoracle as O
from tests.golden.make_golden import (absorption_scenes, estimator_scenes, golden_scenes,
                                      mixture_scenes, statistics_scenes)

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def reference():
    loaded = sys.modules.get("luminis_mc")
    return loaded if loaded is not None else O.reference_module("pin")


def _cases():
    scenes = (golden_scenes() + mixture_scenes() + absorption_scenes() + statistics_scenes()
              + estimator_scenes())
    out = [(s, f"ref_philox_{s['name']}.npz") for s in scenes]
    missing = [f for _, f in out if not os.path.exists(os.path.join(GOLDEN, f))]
    assert not missing, missing
    return out


@pytest.mark.parametrize("spec,fixture", _cases(), ids=lambda c: c["name"] if isinstance(c, dict) else "")
def test_reference_objects_on_the_gpu_reproduce_the_reference(spec, fixture, cuda):
    ref = reference()
    ref.set_log_level(ref.LogLevel.off)
    g = dict(np.load(os.path.join(GOLDEN, fixture)))
    cfg, hs, keep = W.build(ref, spec)
    stats = refbind.run_simulation_parallel(cfg, precision="fp64")
    assert stats["photons"] == spec["n_photons"]
    for i, (h, s) in enumerate(zip(hs, spec["sensors"])):
        got = W.tally_arrays(h, s["kind"])
        want = g[f"sensor{i}"]
        tol = 1e-6 if s["kind"] == "planar_field" else 1e-9
        np.testing.assert_allclose(got, want, rtol=tol, atol=tol * max(np.abs(want).max(), 1e-300))
        assert h.hits == g["hits"][i], f"sensor {i} hits"
    if cfg.absorption is not None and "absorption" in g:
        got = np.stack([np.array(m, copy=True) for m in cfg.absorption.time_slices])
        np.testing.assert_allclose(got, g["absorption"], rtol=1e-9,
                                   atol=1e-9 * np.abs(g["absorption"]).max())


def test_reference_postprocess_runs_on_gpu_tallies(cuda):
    """postprocess_farfield_cbs of the reference (src/results.cpp:61-101) on a sensor the
    GPU filled: S0 coherent per photon per solid angle, from the reference's own code."""
    ref = reference()
    ref.set_log_level(ref.LogLevel.off)
    spec = golden_scenes()[0]                           # mie_cbs_small, FarFieldCBS 100 x 1
    g = dict(np.load(os.path.join(GOLDEN, f"ref_philox_{spec['name']}.npz")))
    cfg, hs, keep = W.build(ref, spec)
    refbind.run_simulation_parallel(cfg, precision="fp64")
    # a second call adds into the same sensors, as the reference's merge does
    refbind.run_simulation_parallel(cfg, precision="fp64")
    n = spec["n_photons"]
    out = ref.postprocess_farfield_cbs(hs[0], 2 * n)
    coh = np.array(out.coherent[0].S0, copy=True)
    dom = np.array(out.dOmega, copy=True)
    want = np.where(dom > 1e-30, g["sensor0"][0, 0] / n / np.where(dom > 1e-30, dom, 1.0), 0.0)
    np.testing.assert_allclose(coh, want, rtol=1e-9, atol=1e-9 * np.abs(want).max())
    assert hs[0].hits == 2 * g["hits"][0]
