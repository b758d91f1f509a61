"""The Python API mirrors the reference's (python/python_module.cpp): names,
arguments, error behaviour, post-processing; checked on CPU."""
import math

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.simulation import Transport, scene_desc
from oracle import pyoracle as O


def reference():
    try:
        return O.reference_module("pin")
    except ImportError as e:
        pytest.skip(str(e))


def test_run_rejects_missing_pointers_like_the_reference():
    cfg = lm.SimConfig()
    with pytest.raises(ValueError, match="sample"):
        lm.run_simulation_parallel(cfg)
    cfg2, _, keep = W.build(lm, W.mie_cbs_small(10, 1))
    cfg2.laser = None
    with pytest.raises(ValueError, match="laser"):
        lm.run_simulation_parallel(cfg2)
    cfg2, _, keep = W.build(lm, W.mie_cbs_small(10, 1))
    cfg2.detector = None
    with pytest.raises(ValueError, match="detector"):
        lm.run_simulation_parallel(cfg2)


def test_sample_validation_messages():
    s = lm.Sample(1.33)
    med = lm.MieMedium(lm.HenyeyGreensteinPhaseFunction(0.9), 0.5e-3, 1.59, 1.33, 0.633e-3)
    with pytest.raises(ValueError, match="first layer must start at z = 0"):
        s.add_layer(med, 0.1, 1.0)
    s.add_layer(med, 0.0, 1.0)
    with pytest.raises(ValueError, match="does not match previous"):
        s.add_layer(med, 2.0, 3.0)
    s.add_layer(med, 1.0, math.inf)
    with pytest.raises(ValueError, match="infinite top layer"):
        s.add_layer(med, 5.0, 6.0)
    assert s.size() == 2 and s.interfaces == [1.0]
    assert s.is_inside(lm.Vec3(0, 0, 5.0)) and not s.is_inside(lm.Vec3(0, 0, -1e-9))


def test_photon_record_sensor_raises_before_any_launch():
    cfg, _, keep = W.build(lm, W.mie_cbs_small(10, 1))
    cfg.detector.add_detector(lm.PhotonRecordSensor(0.0))
    with pytest.raises(NotImplementedError):
        scene_desc(cfg)


def test_statistics_sensor_settings_and_packing():
    """StatisticsSensor (src/detector.cpp:1802-1888): histogram sizes follow the
    set_* calls (time-resolved ones get N_t = ceil(len_t/dt)+1 slices) and pack into
    the C description with the set bits and bin parameters."""
    s = lm.StatisticsSensor(0.0)
    assert not s.absorb_photons and s._tally.size == 0
    s.set_events_histogram_bins(50)
    s.set_time_resolution(10.0, 2.5)
    s.set_theta_histogram_bins(0.0, 1.0, 10)
    s.set_time_histogram_bins(20.0, 8)
    assert s.N_t == 5 and s._tally.size == 5 * 50 + 5 * 10 + 8
    assert len(s.events_histogram) == 5 and len(s.events_histogram[0]) == 50
    assert s.time_histogram == [0] * 8 and s.weight_histogram == []
    assert s.dtheta == 0.1 and s.h_dtime == 2.5 and s.n_bins_time == 8
    cfg, _, keep = W.build(lm, W.mie_cbs_small(10, 1))
    h = cfg.detector.add_detector(s)
    h.set_direction_limit(lm.CrossingDirection.Backward)
    sc, _, sensors = scene_desc(cfg)
    d = sc.sensors[1]
    assert d.kind == 4 and d.stats.set == 1 | 2 | 16
    assert (d.stats.n_events, d.stats.n_theta, d.stats.n_time) == (50, 10, 8)
    assert (d.len_t, d.dt, d.f_dir) == (10.0, 2.5, 1)


def test_absorption_recorder_host_api():
    """Absorption (src/absortion.cpp): grid shapes, host-side deposits into slice 0 and
    the arrival-time slice, clone/merge and the mirrored per-volume image."""
    a = lm.Absorption(1.0, 0.5, 0.25, 0.1, 2.0, 9.0)
    assert a.n_t == 6 and a.time_slices[0].shape == (5, 6)

    class P:
        pos = lm.Vec3(0.3, 0.4, 0.25)          # r = 0.5 -> i_r = 2, i_z = 2
        launch_time, opticalpath, velocity = 0.0, 5.0, 1.0

    a.record_absorption(P, 0.75)
    assert a.time_slices[0][2, 2] == 0.75 and a.time_slices[3][2, 2] == 0.75
    P.pos = lm.Vec3(2.0, 0.0, 0.1)            # outside the radius
    a.record_absorption(P, 1.0)
    assert sum(float(m.sum()) for m in a.time_slices) == 1.5
    b = a.clone()
    assert float(b.time_slices[0].sum()) == 0.0
    b.merge_from(a)
    b.merge_from(a)
    assert b.time_slices[0][2, 2] == 1.5
    img = a.get_total_image(10)
    assert img.shape == (10, 6)
    vox = math.pi * (0.75 ** 2 - 0.5 ** 2) * 0.1
    assert img[5 - 2, 2] == 0.75 / (10.0 * vox) and img[5 + 2, 2] == img[3, 2]
    assert a.get_absorption_image(10, 7).shape == (0, 0)


def test_absorption_packs_into_the_scene():
    cfg, _, keep = W.build(lm, W.mie_cbs_small(10, 1))
    cfg.absorption = lm.Absorption(2.0, 1.0, 0.1, 0.05, 0.5, 10.0)
    sc, _, _ = scene_desc(cfg)
    A = sc.absorption
    assert A.enabled == 1 and (A.radius, A.depth, A.d_r, A.d_z, A.d_t, A.t_max) == (
        2.0, 1.0, 0.1, 0.05, 0.5, 10.0)


def test_mixture_layer_aggregates_and_packing():
    """MixtureLayer (src/sample.cpp:41-88): mu_s_i = n_i sigma_i, albedo-preserving
    absorption, mfp_total, the selection CDF; packed as species + densities with each
    species' cross-section in its medium description."""
    spec = W.mixture_bilayer(10, 1)
    cfg, _, keep = W.build(lm, spec)
    layer = cfg.sample.get_layer(0)
    assert isinstance(layer, lm.MixtureLayer)
    sig = [sp.scattering_cross_section() for sp in layer.species]
    mu_s_i = [n * s for n, s in zip(layer.number_densities, sig)]
    assert layer.mu_s_i == mu_s_i
    assert layer.mu_s_total == sum(mu_s_i)
    mu_a = sum(m * (sp.mu_a / sp.mu_s) for m, sp in zip(mu_s_i, layer.species))
    assert layer.mu_a_total == pytest.approx(mu_a, rel=1e-15)
    assert layer.mu_t_total == layer.mu_s_total + layer.mu_a_total
    assert layer.mfp_total == 1.0 / layer.mu_s_total
    assert layer.selection_cdf[-1] == 1.0
    assert all(a < b for a, b in zip(layer.selection_cdf, layer.selection_cdf[1:]))
    assert layer.mu_attenuation() == layer.mu_t_total
    sc, _, _ = scene_desc(cfg)
    L0 = sc.layers[0]
    assert L0.n_species == 3 and L0.medium == -1
    for k in range(3):
        m = sc.media[L0.species[k]]
        assert m.cross_section == sig[k]
        assert L0.number_density[k] == layer.number_densities[k]
    assert sc.layers[1].n_species == 0 and sc.media[sc.layers[1].medium].cross_section > 0


def test_mixture_layer_validation_messages():
    hg = lm.MieMedium(lm.HenyeyGreensteinPhaseFunction(0.9), 0.5e-3, 1.59, 1.33, 0.633e-3)
    s = lm.Sample(1.33)
    with pytest.raises(ValueError, match="must not be empty"):
        s.add_mixture_layer([], [], 0.0, 1.0)
    with pytest.raises(ValueError, match="sizes differ"):
        s.add_mixture_layer([hg], [1.0, 2.0], 0.0, 1.0)
    with pytest.raises(NotImplementedError, match="scattering_cross_section"):
        s.add_mixture_layer([hg], [1.0], 0.0, 1.0)
    spec = W.mixture_cbs_small(10, 1)
    cfg, _, keep = W.build(lm, spec)
    with pytest.raises(ValueError, match="total mu_s must be positive"):
        lm.Sample(1.33).add_mixture_layer(cfg.sample.get_layer(0).species, [0.0, 0.0], 0.0, 1.0)
    with pytest.raises(ValueError, match="first layer must start at z = 0"):
        lm.Sample(1.33).add_mixture_layer(cfg.sample.get_layer(0).species, [1.0, 1.0], 0.5, 1.0)


@pytest.mark.parametrize("mutate,match", [
    (lambda c: c.sample.layers[0].medium.set_mean_free_path(0.0), "mean_free_path"),
    (lambda c: setattr(c.laser, "position", lm.Vec3(0, 0, -1.0)), "outside the sample"),
    (lambda c: setattr(c.laser, "wavelength", 0.0), "wavelength"),
])
def test_library_validates_scenes_before_touching_a_gpu(mutate, match):
    cfg, _, keep = W.build(lm, W.mie_cbs_small(10, 1))
    mutate(cfg)
    with pytest.raises(ValueError, match=match):
        Transport(cfg)


def test_hg_g_zero_is_rejected():
    spec = W.bilayer_hg(10, 1)
    spec["phases"][0]["g"] = 0.0
    cfg, _, keep = W.build(lm, spec)
    with pytest.raises(ValueError, match="Henyey-Greenstein"):
        Transport(cfg)


def test_sensor_shapes_and_filters_match_the_reference():
    ref = reference()
    spec = W.bilayer_rgd_mie(10, 1)
    spec["sensors"] = spec["sensors"][:2] + [
        {"kind": "planar_field", "z": 0.0, "len_x": 2.56, "len_y": 2.56, "dx": 0.01, "dy": 0.01}]
    c1, h1, k1 = W.build(lm, spec)
    c2, h2, k2 = W.build(ref, spec)
    for a, b in zip(h1, h2):
        for attr in ("N_theta", "N_phi", "N_t", "N_x", "N_y", "dtheta", "dphi", "dx", "dy", "dt",
                     "filter_theta_enabled", "filter_position_enabled", "filter_x_min",
                     "filter_x_max", "absorb_photons", "estimator_enabled", "id"):
            if hasattr(b, attr):
                assert getattr(a, attr) == getattr(b, attr), attr
    assert np.array(h1[0].S0_coh[0]).shape == np.array(h2[0].S0_coh[0]).shape
    assert len(h1[1].S0) == len(h2[1].S0)
    assert np.array(h1[2].Ex).shape == np.array(h2[2].Ex).shape


def test_postprocess_matches_the_reference_on_the_same_tallies():
    ref = reference()
    spec = W.bilayer_rgd_mie(10, 1)
    spec["sensors"][1].update(len_x=2.0, len_y=2.0, dx=0.1, dy=0.1, len_t=7.0, d_t=1.0)
    spec["sensors"] = spec["sensors"][:2]
    c2, h2, k2 = W.build(ref, spec, n_photons=3000)
    ref.run_simulation_parallel(c2)
    c1, h1, k1 = W.build(lm, spec)
    for a, b, s in zip(h1, h2, spec["sensors"]):
        a._tally[:] = W.tally_arrays(b, s["kind"]).ravel()
    p1 = lm.postprocess_farfield_cbs(h1[0], 3000)
    p2 = ref.postprocess_farfield_cbs(h2[0], 3000)
    np.testing.assert_allclose(np.array(p1.dOmega), np.array(p2.dOmega), rtol=1e-15)
    for t in range(len(p2.coherent)):
        for q in ("S0", "S1", "S2", "S3"):
            np.testing.assert_allclose(np.array(getattr(p1.coherent[t], q)),
                                       np.array(getattr(p2.coherent[t], q)), rtol=1e-14)
            np.testing.assert_allclose(np.array(getattr(p1.incoherent[t], q)),
                                       np.array(getattr(p2.incoherent[t], q)), rtol=1e-14)
    f1 = lm.postprocess_planar_fluence(h1[1], 3000)
    f2 = ref.postprocess_planar_fluence(h2[1], 3000)
    for q in ("S0", "S1", "S2", "S3"):
        for t in range(len(getattr(f2, q))):
            np.testing.assert_allclose(np.array(getattr(f1, q)[t]), np.array(getattr(f2, q)[t]),
                                       rtol=1e-14)


def test_add_detector_clones_like_the_reference():
    g = lm.SensorsGroup()
    d = lm.FarFieldCBSSensor(0.1, 2 * math.pi, 0.0, 1e-3, 2 * math.pi, 0.0)
    d.set_theta_limit(0.0, 0.1)
    h = g.add_detector(d)
    assert h is not d and h is g.detectors[0] and h.filter_theta_enabled
    d.set_phi_limit(0.0, 1.0)
    assert not h.filter_phi_enabled
