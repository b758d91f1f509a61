"""GPU parity: the CUDA transport against the CPU oracle on the same Philox stream.

(a) per-photon replay: every photon's final state (events, draws, fate, position,
    direction, frame, Jones vector, weight, path length, reverse field at CBS
    detection) from the GPU record buffer against the oracle's record;
(b) tallies: every sensor bin against the oracle's tallies.
FP64 transport must match to 1e-9 relative with all event counts exact; FP32
transport (draws "u24") must agree on the discrete history (events, draws, fate)
for every photon of these scenes and on positions to 1e-5 of the path length, on
weights to 1e-12 (the weight is binary64 in both modes), on directions and frames to
1e-6 sqrt(events + 1) and on Jones vectors to 1e-5 sqrt(events + 1) (the 1/sqrt(F)
renormalisation amplifies rounding, as the FP64 comparison shows: 1e-13 against
1e-16 ulps).
"""
import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.device import DeviceRun
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-9
# The speckle field sums exp(i k L) with k L ~ 1e6 rad over 100 mm paths, which
# turns 1e-13 path differences (FMA contraction, libm ulps) into ~1e-7 rad.
FP64_FIELD_RTOL = 1e-6
FP32_RTOL = {"weight": 1e-12, "opticalpath": 1e-5}
# Rounding of the frame and Jones updates accumulates as a random walk over the
# photon's events, so those bounds scale with sqrt(events + 1): 1e-6 * sqrt(n)
# for directions (2e-5 at 400 events), 1e-5 * sqrt(n) for Jones vectors.  Measured on
# these scenes: at most 3.4e-7 * sqrt(n) for directions, 3.6e-6 * sqrt(n) for Jones
# vectors (Henyey-Greenstein bilayer).
FP32_PER_SQRT_EVENT = {"dir": 1e-6, "m": 1e-6, "n": 1e-6, "E": 1e-5, "Er": 2e-5}
FP32_POS_OF_PATH = 1e-5       # positions: |difference| / path length
# every photon of these scenes (fixed seeds) follows the binary64 discrete history
FP32_MAX_DIVERGED = 0.0


def small_specs():
    yield W.mie_cbs_small(3000, 20240)
    yield W.bilayer_rgd_mie(3000, 77)
    yield W.bilayer_hg(3000, 5)
    spec = W.mie_long_paths(300, 9)
    spec["max_events"] = 20000
    yield spec


def _relerr(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.maximum(np.abs(b), 1.0)
    return np.abs(a - b) / scale


def _compare_records(gpu, ora, rtol):
    """Indices of photons whose discrete history agrees, and the max relative
    error of their continuous state."""
    assert np.array_equal(gpu["photon"], ora["photon"])
    same = ((gpu["events"] == ora["events"]) & (gpu["draws"] == ora["draws"]) &
            (gpu["fate"] == ora["fate"]) & (gpu["n_hits"] == ora["n_hits"]))
    worst = {}
    for f in ("weight", "opticalpath", "pos", "dir", "m", "n", "E", "r1", "rn", "Er", "hit"):
        if f in FP32_PER_SQRT_EVENT and rtol is None:
            continue
        e = _relerr(gpu[f][same], ora[f][same])
        worst[f] = float(e.max()) if e.size else 0.0
    return same, worst


@pytest.mark.parametrize("spec", list(small_specs()), ids=lambda s: s["name"])
def test_replay_fp64_exact(spec, cuda):
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    n = cfg.n_photons
    stats, rec = run.run(n, cfg.seed, precision="fp64", records=True)
    ref = O.Oracle(spec).run(n, cfg.seed, rng="philox_u53", records=True)
    same, worst = _compare_records(rec, ref.records, FP64_RTOL)
    assert same.all(), f"{(~same).sum()} photons differ in events/draws/fate"
    for f, e in worst.items():
        assert e < FP64_RTOL, f"{f}: {e}"
    assert stats["events"] == ref.stats["events"]
    assert stats["steps"] == ref.stats["steps"]
    assert stats["draws"] == ref.stats["draws"]
    for s_idx, (g, o) in enumerate(zip(run.host_tallies(), ref.tallies)):
        # Stokes S1..S3 bins can cancel to ~0, so the floor scales with the sensor
        tol = FP64_FIELD_RTOL if spec["sensors"][s_idx]["kind"] == "planar_field" else FP64_RTOL
        np.testing.assert_allclose(g, o, rtol=tol, atol=tol * np.abs(o).max(),
                                   err_msg=f"sensor {s_idx}")
        assert stats["hits"][s_idx] == ref.hits[s_idx]
    run.close()


@pytest.mark.parametrize("spec", list(small_specs()), ids=lambda s: s["name"])
def test_replay_fp32_tolerance(spec, cuda):
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    n = cfg.n_photons
    stats, rec = run.run(n, cfg.seed, precision="fp32", records=True)
    ref = O.Oracle(spec).run(n, cfg.seed, rng="philox_u24", records=True)
    same, worst = _compare_records(rec, ref.records, None)
    diverged = 1.0 - same.mean()
    assert diverged <= FP32_MAX_DIVERGED, f"diverged fraction {diverged}"
    for f, tol in FP32_RTOL.items():
        assert worst[f] < tol, f"{f}: max relative error {worst[f]} over {same.sum()} photons"
    g, o = rec[same], ref.records[same]
    root_n = np.sqrt(o["events"].astype(np.float64) + 1.0)[:, None]
    for f, tol in FP32_PER_SQRT_EVENT.items():
        e = float((_relerr(g[f], o[f]) / root_n).max()) if g.size else 0.0
        assert e < tol, f"{f}: {e} per sqrt(event)"
    path = np.maximum(o["opticalpath"], 1.0)[:, None]
    for f in ("pos", "r1", "rn", "hit"):
        e = float((np.abs(g[f] - o[f]) / path).max())
        assert e < FP32_POS_OF_PATH, f"{f}: {e} of the path length"
    # tallies: binary32 transport against the binary64 oracle, bin by bin.  Intensity
    # totals agree to 1e-3; the CBS coherent grids carry the interference phase
    # k (s_out + s_in).(r_n - r_1), which binary32 positions perturb by ~1e-2 rad.
    for s_idx, (gt, ot) in enumerate(zip(run.host_tallies(), ref.tallies)):
        kind = spec["sensors"][s_idx]["kind"]
        if kind == "planar_field":
            # The speckle phase k n L needs the path to the exit plane to ~lambda/100
            # after ~100 mm; binary32 directions move the last crossing by ~1e-4 mm,
            # i.e. ~1 rad, so only the binary64 mode reproduces the realisation bin by
            # bin.  binary32 must still deposit the same field energy per photon.
            e_g = float((gt ** 2).sum())
            e_o = float((ot ** 2).sum())
            assert abs(e_g - e_o) <= 0.1 * e_o, (e_g, e_o)
            continue
        scale = np.abs(ot).max()
        assert np.abs(gt - ot).max() <= 0.05 * scale + 1e-300, f"sensor {s_idx}"
        plane = 4 if kind == "farfield_cbs" else 0          # incoherent S0 for CBS
        assert abs(gt[plane].sum() - ot[plane].sum()) <= 1e-3 * abs(ot[plane].sum()) + 1e-300
        if kind == "farfield_cbs":
            assert abs(gt[0].sum() - ot[0].sum()) <= 1e-2 * abs(ot[0].sum()) + 1e-300
    run.close()


def test_launch_shape_independence(cuda):
    """Results depend on (seed, photon index) only, like the reference's per-photon
    seeding makes them independent of n_threads (src/simulation.cpp:172-197)."""
    spec = W.bilayer_rgd_mie(2000, 31)
    cfg, _, keep = W.build(lm, spec)
    a = DeviceRun(cfg)
    _, ra = a.run(2000, 31, precision="fp64", records=True, block_size=256)
    b = DeviceRun(cfg)
    _, rb = b.run(2000, 31, precision="fp64", records=True, block_size=64, blocks_per_sm=1)
    assert ra.tobytes() == rb.tobytes()
    a.close()
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_records_over_several_batches(precision, cuda):
    """A run split into hit-queue batches writes every photon's record at its own slot
    (photon begin + i at records[i]), exactly as a one-batch run does."""
    spec = W.bilayer_rgd_mie(2000, 37)
    cfg, _, keep = W.build(lm, spec)
    a = DeviceRun(cfg)
    _, ra = a.run(2000, 37, 500, precision=precision, records=True)
    b = DeviceRun(cfg)
    _, rb = b.run(2000, 37, 500, precision=precision, records=True, batch_photons=300)
    assert np.array_equal(rb["photon"], np.arange(500, 2500, dtype=rb["photon"].dtype))
    assert ra.tobytes() == rb.tobytes()
    for ga, gb in zip(a.host_tallies(), b.host_tallies()):
        np.testing.assert_allclose(gb, ga, rtol=1e-12, atol=1e-12 * max(np.abs(ga).max(), 1e-300))
    a.close()
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("make", [W.mie_cbs_small, W.bilayer_rgd_mie, W.mixture_bilayer],
                         ids=["mie_cbs_small", "bilayer_rgd_mie", "mixture_bilayer"])
def test_cbs_replay_equals_tracked_history(make, precision, cuda):
    """By default a queued run keeps no reverse-path history in the transport and
    replays the photons a FarFieldCBS grid reads; with no_replay every photon's history
    is tracked event by event.  Both give the same tallies and counts: the replay
    rebuilds exactly the history the tracked run keeps (same stream, same arithmetic)."""
    spec = make(20000, 53)
    cfg, _, keep = W.build(lm, spec)
    a = DeviceRun(cfg)
    sa, _ = a.run(20000, 53, precision=precision)                    # replayed
    b = DeviceRun(cfg)
    sb, _ = b.run(20000, 53, precision=precision, no_replay=True)    # tracked
    assert sa["replay_launches"] > 0 and sa["replayed"] > 0
    assert sb["replay_launches"] == 0
    assert sa["error_flags"] == 0 and sb["error_flags"] == 0
    for ga, gb in zip(a.host_tallies(), b.host_tallies()):
        np.testing.assert_allclose(ga, gb, rtol=1e-12, atol=1e-12 * max(np.abs(gb).max(), 1e-300))
    assert sa["hits"] == sb["hits"] and sa["events"] == sb["events"]
    a.close()
    b.close()


def test_photon_ranges_compose(cuda):
    """Two runs over [0, n/2) and [n/2, n) tally the same as one run over [0, n)."""
    spec = W.mie_cbs_small(4000, 99)
    cfg, _, keep = W.build(lm, spec)
    one = DeviceRun(cfg)
    one.run(4000, 99, precision="fp64")
    two = DeviceRun(cfg)
    two.run(2000, 99, 0, precision="fp64")
    two.run(2000, 99, 2000, precision="fp64")
    for x, y in zip(one.host_tallies(), two.host_tallies()):
        np.testing.assert_allclose(x, y, rtol=1e-11, atol=1e-13)
    one.close()
    two.close()


def test_zero_photons(cuda):
    cfg, hs, keep = W.build(lm, W.mie_cbs_small(0, 1))
    lm.run_simulation_parallel(cfg)
    assert hs[0].hits == 0
    assert np.all(np.asarray(hs[0].S0_coh[0]) == 0)


def test_public_api_matches_oracle(cuda):
    """run_simulation_parallel through host buffers equals the oracle's tallies, and
    accumulates into existing tallies like the reference's merge_from."""
    spec = W.bilayer_rgd_mie(3000, 123)
    cfg, hs, keep = W.build(lm, spec)
    lm.run_simulation_parallel(cfg, precision="fp64")
    ref = O.Oracle(spec).run(3000, 123, rng="philox_u53")
    for i, (h, s) in enumerate(zip(hs, spec["sensors"])):
        got = W.tally_arrays(h, s["kind"])
        np.testing.assert_allclose(got, ref.tallies[i], rtol=FP64_RTOL,
                                   atol=FP64_RTOL * np.abs(ref.tallies[i]).max())
        assert h.hits == ref.hits[i]
    lm.run_simulation_parallel(cfg, precision="fp64")
    for i, (h, s) in enumerate(zip(hs, spec["sensors"])):
        np.testing.assert_allclose(W.tally_arrays(h, s["kind"]), 2 * ref.tallies[i],
                                   rtol=FP64_RTOL, atol=2 * FP64_RTOL * np.abs(ref.tallies[i]).max())
        assert h.hits == 2 * ref.hits[i]


def test_public_api_scene_kept_between_calls(cuda):
    """The scene run_simulation_parallel keeps between calls: alternating scenes, a
    changed photon budget and MAX_EVENTS on an unchanged scene, and a changed laser
    each give the tallies of a fresh call."""
    def fresh(spec, **cfg_kw):
        lm.release_gpu_cache()
        cfg, hs, keep = W.build(lm, spec)
        for k, v in cfg_kw.items():
            setattr(cfg, k, v)
        lm.run_simulation_parallel(cfg, precision="fp64")
        return [W.tally_arrays(h, s["kind"]).copy() for h, s in zip(hs, spec["sensors"])]

    a, b = W.bilayer_rgd_mie(1500, 31), W.mie_cbs_small(1500, 32)
    want_a, want_b = fresh(a), fresh(b)
    want_a_short = fresh(a, MAX_EVENTS=7)
    cfg_a, hs_a, keep_a = W.build(lm, a)
    cfg_b, hs_b, keep_b = W.build(lm, b)
    lm.release_gpu_cache()
    for cfg in (cfg_a, cfg_b, cfg_a):
        lm.run_simulation_parallel(cfg, precision="fp64")
    for h, s, w in zip(hs_a, a["sensors"], want_a):
        np.testing.assert_allclose(W.tally_arrays(h, s["kind"]), 2 * w, rtol=1e-12,
                                   atol=1e-12 * np.abs(w).max())
    for h, s, w in zip(hs_b, b["sensors"], want_b):
        np.testing.assert_allclose(W.tally_arrays(h, s["kind"]), w, rtol=1e-12,
                                   atol=1e-12 * np.abs(w).max())
    cfg_a, hs_a, keep_a = W.build(lm, a)
    lm.run_simulation_parallel(cfg_a, precision="fp64")
    cfg_a.MAX_EVENTS = 7
    before = [W.tally_arrays(h, s["kind"]).copy() for h, s in zip(hs_a, a["sensors"])]
    lm.run_simulation_parallel(cfg_a, precision="fp64")
    for h, s, w, b0 in zip(hs_a, a["sensors"], want_a_short, before):
        np.testing.assert_allclose(W.tally_arrays(h, s["kind"]) - b0, w, rtol=1e-9,
                                   atol=1e-12 * max(np.abs(w).max(), 1.0))
    cfg_a.MAX_EVENTS = a.get("max_events", cfg_a.MAX_EVENTS)
    cfg_a.laser.position = lm.Vec3(0.3, -0.2, 1e-9)
    lm.run_simulation_parallel(cfg_a, precision="fp64")
    spec = dict(a)
    got = [W.tally_arrays(h, s["kind"]).copy() for h, s in zip(hs_a, a["sensors"])]
    lm.release_gpu_cache()
    cfg_c, hs_c, keep_c = W.build(lm, spec)
    cfg_c.laser.position = lm.Vec3(0.3, -0.2, 1e-9)
    lm.run_simulation_parallel(cfg_c, precision="fp64")
    moved = False
    for g, h, s, b0, w, w0 in zip(got, hs_c, a["sensors"], before, want_a_short, want_a):
        shifted = W.tally_arrays(h, s["kind"])
        np.testing.assert_allclose(g - b0 - w, shifted, rtol=1e-9,
                                   atol=1e-9 * max(np.abs(g).max(), 1.0))
        moved |= not np.allclose(shifted, w0)
    assert moved, "moving the source must change the tallies"
    lm.release_gpu_cache()


def test_device_then_host_run_on_one_handle(cuda):
    """lmc_run (grows the hit queue) followed by lmc_run_host on the same handle:
    the host path's staging buffer must not disturb the queue the next run reuses."""
    import torch
    spec = W.mie_cbs_small(2000, 57)
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    run.run(2000, 57, precision="fp64")
    host = np.zeros(run.transport.tally_size)
    run.transport.run_host(host, 2000, 57, precision="fp64")
    run.run(2000, 57, precision="fp64")
    torch.cuda.synchronize()
    for d, h in zip(run.host_tallies(), run.transport.split(host)):
        np.testing.assert_allclose(d, 2 * h, rtol=FP64_RTOL, atol=FP64_RTOL * np.abs(h).max())
    run.close()


@pytest.mark.parametrize("spec", list(small_specs())[:3], ids=lambda s: s["name"])
def test_fp64_on_the_u24_stream_replays_the_oracle(spec, cuda):
    """stream_format=1: binary64 transport on the binary32 run's numbers (u24) is the
    oracle's binary64 replay of that stream, so FP32-vs-FP64 comparisons on it measure
    precision alone."""
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    n = cfg.n_photons
    stats, rec = run.run(n, cfg.seed, precision="fp64", records=True, stream_format=1)
    ref = O.Oracle(spec).run(n, cfg.seed, rng="philox_u24", records=True)
    same, worst = _compare_records(rec, ref.records, FP64_RTOL)
    assert same.all(), f"{(~same).sum()} photons differ in events/draws/fate"
    for f, e in worst.items():
        assert e < FP64_RTOL, f"{f}: {e}"
    assert stats["draws"] == ref.stats["draws"]
    run.close()
