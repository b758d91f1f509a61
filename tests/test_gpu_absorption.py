"""The Absorption recorder on the GPU (src/absortion.cpp:54-91).

* FP64 against the reference's own grids on the Philox stream
  (tests/golden/ref_philox_absorption_*.npz): a time-resolved grid over the two-layer
  slab and a time-integrated one over the mixture slab, 1e-9 of the largest cell.
* FP32 against the oracle on the u24 stream, 5 % of the largest cell.
* run_simulation_parallel adds the grid into config.absorption.time_slices; a sweep
  holds the same grid as a lone lmc_run (lmc_run_noalloc: tests/test_zz_no_alloc.py).
"""
import os

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.device import DeviceRun
from oracle import pyoracle as O
from tests.golden.make_golden import absorption_scenes

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("spec", absorption_scenes(), ids=lambda s: s["name"])
def test_gpu_fp64_absorption_reproduces_reference(spec, cuda):
    g = np.load(os.path.join(GOLDEN, f"ref_philox_{spec['name']}.npz"))
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    st, _ = run.run(spec["n_photons"], spec["seed"], precision="fp64")
    assert st["error_flags"] == 0
    ref = g["absorption"]
    np.testing.assert_allclose(run.host_absorption(), ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())
    for i, t in enumerate(run.host_tallies()):
        r = g[f"sensor{i}"]
        np.testing.assert_allclose(t, r, rtol=1e-9, atol=1e-9 * np.abs(r).max())
        assert st["hits"][i] == g["hits"][i]
    run.close()


@pytest.mark.parametrize("spec", absorption_scenes(), ids=lambda s: s["name"])
def test_gpu_fp32_absorption_matches_oracle(spec, cuda):
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    run.run(spec["n_photons"], spec["seed"], precision="fp32")
    ref = O.Oracle(spec).run(spec["n_photons"], spec["seed"], rng="philox_u24").absorption
    got = run.host_absorption()
    assert float(np.abs(got - ref).max()) <= 5e-2 * float(np.abs(ref).max())
    assert abs(float(got.sum()) / float(ref.sum()) - 1.0) < 1e-3
    run.close()


def test_public_api_accumulates_absorption(cuda):
    spec = absorption_scenes()[0]
    cfg, _, keep = W.build(lm, spec)
    lm.run_simulation_parallel(cfg, precision="fp64")
    lm.run_simulation_parallel(cfg, precision="fp64")
    g = np.load(os.path.join(GOLDEN, f"ref_philox_{spec['name']}.npz"))["absorption"]
    got = np.stack([np.asarray(m) for m in cfg.absorption.time_slices])
    np.testing.assert_allclose(got, 2 * g, rtol=1e-9, atol=1e-9 * np.abs(g).max())


def test_sweep_holds_the_lone_run_grid(cuda):
    from luminis_mc_b200.sweep import SweepRun
    specs = absorption_scenes()
    counts = [700, 500]
    sw = SweepRun([W.build(lm, s)[0] for s in specs])
    sw.set_photons(counts)
    sw.run(23, precision="fp64")
    for k, (spec, n, p0) in enumerate(zip(specs, counts, sw.offsets())):
        cfg, _, keep = W.build(lm, spec)
        run = DeviceRun(cfg)
        run.run(n, 23, int(p0), precision="fp64")
        want = run.host_absorption()
        np.testing.assert_allclose(sw.host_absorption(k), want, rtol=1e-12,
                                   atol=1e-12 * np.abs(want).max())
        run.close()
    sw.close()


def test_adjoint_refuses_absorption(cuda):
    """Likelihood-ratio runs carry no Absorption grid: refused, not silently dropped."""
    from luminis_mc_b200.adjoint import AdjointTransport
    spec = absorption_scenes()[0]
    cfg, _, keep = W.build(lm, spec)
    tr = AdjointTransport(cfg)
    with pytest.raises(NotImplementedError):
        tr.run(100, 1, precision="fp64")
    tr.close()
