"""StatisticsSensor on the GPU (src/detector.cpp:1569-1888).

* FP64 against the reference's own histograms on the Philox stream
  (tests/golden/ref_philox_stats_*.npz): all six histograms with time windows at
  z = 0 beside a FarFieldCBS sensor, a non-absorbing sensor inside the sample (the
  in-kernel tally path, many crossings per photon), and theta / event filters.
  Counts are exact.
* FP32 against the oracle on the u24 stream: every histogram within 5 % of its
  largest bin plus 3 counts.
* run_simulation_parallel fills the sensor's histograms; a sweep counts as a lone
  lmc_run (lmc_run_noalloc: tests/test_zz_no_alloc.py).
"""
import os

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.device import DeviceRun
from oracle import pyoracle as O
from tests.golden.make_golden import statistics_scenes

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("spec", statistics_scenes(), ids=lambda s: s["name"])
def test_gpu_fp64_statistics_reproduce_reference(spec, cuda):
    g = np.load(os.path.join(GOLDEN, f"ref_philox_{spec['name']}.npz"))
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    st, _ = run.run(spec["n_photons"], spec["seed"], precision="fp64")
    assert st["error_flags"] == 0
    for i, (t, s) in enumerate(zip(run.host_tallies(), spec["sensors"])):
        ref = g[f"sensor{i}"]
        if s["kind"] == "statistics":
            np.testing.assert_array_equal(t.ravel(), ref.ravel(), err_msg=f"sensor {i}")
        else:
            np.testing.assert_allclose(t, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())
        assert st["hits"][i] == g["hits"][i]
    run.close()


@pytest.mark.parametrize("spec", statistics_scenes(), ids=lambda s: s["name"])
def test_gpu_fp32_statistics_match_oracle(spec, cuda):
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    run.run(spec["n_photons"], spec["seed"], precision="fp32")
    ref = O.Oracle(spec).run(spec["n_photons"], spec["seed"], rng="philox_u24")
    for t, o, s in zip(run.host_tallies(), ref.tallies, spec["sensors"]):
        if s["kind"] != "statistics":
            continue
        assert float(np.abs(t.ravel() - o.ravel()).max()) <= 5e-2 * float(np.abs(o).max()) + 3
    run.close()


def test_public_api_fills_histograms(cuda):
    spec = statistics_scenes()[1]
    cfg, hs, keep = W.build(lm, spec)
    lm.run_simulation_parallel(cfg, precision="fp64")
    g = np.load(os.path.join(GOLDEN, f"ref_philox_{spec['name']}.npz"))
    np.testing.assert_array_equal(W.tally_arrays(hs[0], "statistics"), g["sensor0"].ravel())
    assert hs[0].hits == g["hits"][0]
    assert len(hs[0].events_histogram) == 1 and len(hs[0].events_histogram[0]) == 100
    assert hs[0].phi_histogram == [] and len(hs[0].weight_histogram) == 25


def test_sweep_counts_as_lone_runs(cuda):
    from luminis_mc_b200.sweep import SweepRun
    specs = [statistics_scenes()[1], W.mie_cbs_small(0, 3)]
    counts = [1500, 700]
    sw = SweepRun([W.build(lm, s)[0] for s in specs])
    sw.set_photons(counts)
    sw.run(29, precision="fp64")
    for k, (spec, n, p0) in enumerate(zip(specs, counts, sw.offsets())):
        cfg, _, keep = W.build(lm, spec)
        run = DeviceRun(cfg)
        run.run(n, 29, int(p0), precision="fp64")
        want = run.host_tallies()
        for a, b in zip(sw.host_tallies(k), want):
            np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12 * max(np.abs(b).max(), 1e-300))
        run.close()
    sw.close()
