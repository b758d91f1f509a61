"""Sweeps (lmc_create_sweep / lmc_run_sweep): many scenes in one launch.

Scene s of a sweep owns photons [P_s, P_s + n_s) of the (seed, photon) stream, so its
tallies and hit counts must equal those of a lone run of that scene over the same
photon range (lmc_run with photon_begin = P_s).  FP64 and FP32, scenes of different
shapes in one sweep, and a CUDA-graph replay of a run.  FP64 agrees to 1e-12; FP32 to
1e-5 of each sensor's largest bin: the sweep kernel is a separate compilation whose
binary32 operations may round differently (different fused multiply-adds), while
every photon keeps its discrete history (hit counts stay equal).
"""
import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.device import DeviceRun
from luminis_mc_b200.sweep import SweepRun

pytestmark = pytest.mark.gpu
RTOL = 1e-12
FP32_TOL = 1e-5


def _specs():
    out = [W.mie_sweep(i, seed=7) for i in (0, 5, 17, 200)]
    b = W.bilayer_rgd_mie(0, 7)
    b["sensors"][1].update(len_x=4.0, len_y=4.0, dx=0.25, dy=0.25, len_t=15.0, d_t=1.0)
    out.append(b)
    return out


def _sequential(spec, n, seed, begin, precision):
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    st, _ = run.run(n, seed, begin, precision=precision)
    t = [x.copy() for x in run.host_tallies()]
    run.close()
    return t, st["hits"][:len(spec["sensors"])]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_sweep_equals_sequential_runs(precision, cuda):
    specs = _specs()
    counts = [3000, 500, 2200, 1, 2500]
    cfgs = [W.build(lm, s)[0] for s in specs]
    sw = SweepRun(cfgs)
    sw.set_photons(counts)
    st = sw.run(11, precision=precision)
    assert st["photons"] == sum(counts) and st["error_flags"] == 0
    hits = sw.hits()
    for k, (spec, n, p0) in enumerate(zip(specs, counts, sw.offsets())):
        want, want_hits = _sequential(spec, n, 11, int(p0), precision)
        got = sw.host_tallies(k)
        tol = RTOL if precision == "fp64" else FP32_TOL
        for g, w in zip(got, want):
            np.testing.assert_allclose(g, w, rtol=tol, atol=tol * max(np.abs(w).max(), 1e-300))
        assert list(hits[k][:len(spec["sensors"])]) == list(want_hits)
    sw.close()


def test_sweep_graph_replay_adds_runs(cuda):
    import torch
    specs = _specs()[:4]
    cfgs = [W.build(lm, s)[0] for s in specs]
    sw = SweepRun(cfgs)
    sw.set_photons([4000, 1000, 3000, 500])
    sw.run(3, precision="fp64")                 # grows the hit queue outside the capture
    once = [sw.host_tallies(k) for k in range(4)]
    g = sw.capture(3, precision="fp64")
    sw.zero()
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    for k in range(4):
        for a, b in zip(sw.host_tallies(k), once[k]):
            np.testing.assert_allclose(a, 2 * b, rtol=RTOL, atol=RTOL * max(np.abs(b).max(), 1e-300))
    sw.close()


def test_sweep_rejects_planes_inside_the_sample(cuda):
    spec = W.bilayer_rgd_mie(0, 1)
    spec["sensors"][1]["z"] = 0.25
    with pytest.raises(NotImplementedError):
        SweepRun([W.build(lm, s)[0] for s in (_specs()[0], spec)])


def _lone_adjoint(spec, n, seed, begin, precision, **radial):
    from luminis_mc_b200.adjoint import AdjointTransport
    cfg, _, keep = W.build(lm, spec)
    tr = AdjointTransport(cfg, **radial)
    out, jac, _ = tr.run(n, seed, precision=precision, begin=begin)
    tr.close()
    return out.cpu().numpy() * n, jac.cpu().numpy() * n      # sums over the photons


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_sweep_adjoint_equals_lone_adjoint_runs(precision, cuda):
    """Each scene's block of lmc_run_sweep_adjoint (its CBS S0 grids and their
    derivatives with respect to its medium's mu_a, mu_s, mfp, g) equals
    lmc_run_adjoint on that scene alone over its photon range."""
    specs = [W.mie_sweep(i, seed=7) for i in (0, 5, 17, 200)]
    counts = [3000, 1200, 2200, 900]
    sw = SweepRun([W.build(lm, s)[0] for s in specs])
    sw.set_photons(counts)
    blocks, st = sw.run_adjoint(13, precision=precision)
    assert st["error_flags"] == 0
    tol = RTOL if precision == "fp64" else FP32_TOL
    for k, (spec, n, p0) in enumerate(zip(specs, counts, sw.offsets())):
        out, jac = blocks[k]
        want_out, want_jac = _lone_adjoint(spec, n, 13, int(p0), precision)
        assert jac.shape == want_jac.shape == (4, want_out.size)
        np.testing.assert_allclose(out.cpu().numpy(), want_out, rtol=tol,
                                   atol=tol * np.abs(want_out).max())
        for r in range(4):
            np.testing.assert_allclose(jac[r].cpu().numpy(), want_jac[r], rtol=tol,
                                       atol=tol * max(np.abs(want_jac[r]).max(), 1e-300))
    sw.close()


def test_sweep_adjoint_radial_outputs_and_media_counts(cuda):
    """Scenes with different media counts (K = 4 and 8) and the radial reflectance
    profile of a PlanarFluenceSensor, added globally in a sweep."""
    from tests.test_oracle_adjoint import adjoint_scene
    a = adjoint_scene()
    b = W.bilayer_hg(0, 5)
    b["sensors"][1].update(len_x=4.0, len_y=4.0, dx=0.25, dy=0.25, len_t=0.0, d_t=0.0)
    b["sensors"].pop(2)
    c = W.mie_cbs_small(0, 5)
    c["sensors"].append({"kind": "planar_fluence", "z": 0.0, "len_x": 4.0, "len_y": 4.0,
                         "len_t": 0.0, "dx": 0.5, "dy": 0.5, "d_t": 0.0, "absorb": True})
    specs, counts = [a, b, c], [1500, 1000, 1200]
    radial = dict(radial_sensor=1, radial_bins=10, radial_max=5.0)
    sw = SweepRun([W.build(lm, s)[0] for s in specs])
    sw.set_photons(counts)
    blocks, st = sw.run_adjoint(3, precision="fp64", **radial)
    for k, (spec, n, p0) in enumerate(zip(specs, counts, sw.offsets())):
        out, jac = blocks[k]
        want_out, want_jac = _lone_adjoint(spec, n, 3, int(p0), "fp64", **radial)
        assert jac.shape[0] == 4 * len(spec["media"])
        np.testing.assert_allclose(out.cpu().numpy(), want_out, rtol=RTOL,
                                   atol=RTOL * np.abs(want_out).max())
        np.testing.assert_allclose(jac.cpu().numpy(), want_jac, rtol=RTOL,
                                   atol=RTOL * np.abs(want_jac).max())
    sw.close()


def test_autotune_picks_a_shape_and_keeps_results(cuda):
    """lmc_autotune times its candidate launch shapes on a scaled-down sweep, restores the
    photon counts, and the tuned shape gives the same FP64 tallies (results do not
    depend on the launch shape)."""
    specs = _specs()[:4]
    counts = [30000, 5000, 22000, 900]
    sw = SweepRun([W.build(lm, s)[0] for s in specs])
    sw.set_photons(counts)
    st0 = sw.run(5, precision="fp64")
    base = [sw.host_tallies(k) for k in range(4)]
    r = sw.autotune(5, precision="fp64", sample_photons=20000)
    assert r["block_size"] in (128, 256) and r["blocks_per_sm"] in (0, 1, 2)
    assert r["n_tried"] >= 6 and r["photons_per_s"] > 0 and 4 <= r["sample_photons"] <= 25000
    sw.zero()
    st = sw.run(5, precision="fp64")
    assert st["photons"] == st0["photons"] == sum(counts)
    for k in range(4):
        for a, b in zip(sw.host_tallies(k), base[k]):
            np.testing.assert_allclose(a, b, rtol=RTOL, atol=RTOL * max(np.abs(b).max(), 1e-300))
    sw.close()
    from luminis_mc_b200.simulation import Transport
    t = Transport(W.build(lm, W.mie_cbs_small(0, 1))[0])
    r = t.autotune(1, precision="fp32", sample_photons=50000)
    assert r["sample_photons"] == 50000 and r["photons_per_s"] > 0
    t.close()
