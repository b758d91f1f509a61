"""Failure detection on the host: a corrupt scene is refused before any device call.

The reference validates its configuration and throws std::invalid_argument
(validate_sim_config, src/simulation.cpp:95-103; Sample::add_layer and MixtureLayer,
src/sample.cpp:47-72,124), and a missing phase function ends the process
(src/medium.cpp:37-38,47-48,57-58).  lmc_create checks every
scene field first, returns LMC_ERR_INVALID with a message (ValueError in Python), and
only then touches the GPU.  So each fault below is injected into an otherwise valid C
scene and must be refused on a machine without a GPU.  The unmodified scene must pass
validation and fail only at the first CUDA call.  lmc_create_sweep names the faulty
scene, and lmc_run_noalloc refuses corrupt scenes and options the same way.
"""
import ctypes as C
import math

import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import _native as N
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.simulation import scene_desc
from tests.conftest import gpu_available

NAN, INF = math.nan, math.inf


def _scene(make=W.bilayer_rgd_mie):
    cfg, _, keep = W.build(lm, make(10, 1))
    sc, keep2, sensors = scene_desc(cfg)
    return sc, (cfg, keep, keep2)


def _set(obj, path, value):
    *head, last = path.split(".")
    for p in head:
        obj = obj[int(p)] if p.isdigit() else getattr(obj, p)
    if last.isdigit():
        obj[int(last)] = value
    else:
        setattr(obj, last, value)


FAULTS = [
    ("n_host", NAN, "host refractive index"),
    ("n_host", -1.33, "host refractive index"),
    ("media.0.mu_s", NAN, "medium coefficients"),
    ("media.1.mu_a", -0.01, "medium coefficients"),
    ("media.0.mean_free_path", 0.0, "mean_free_path"),
    ("media.1.mean_free_path", INF, "mean_free_path"),
    ("layers.0.z_min", 0.1, "first layer must start at z = 0"),
    ("layers.1.z_min", 0.6, "does not match previous z_max"),
    ("layers.0.z_max", -1.0, "z_max must be greater than z_min"),
    ("layers.1.medium", 7, "medium index out of range"),
    ("n_layers", 0, "layers"),
    ("n_media", 0, "media"),
    ("n_sensors", 9, "sensors"),
    ("laser.wavelength", 0.0, "wavelength"),
    ("laser.source", 9, "laser source"),
    ("laser.position.2", -5.0, "outside the sample"),
    ("sensors.0.kind", 42, "sensor kind"),
    ("sensors.0.dtheta", 0.0, "bin widths"),
    ("sensors.1.dx", -0.05, "pixel sizes"),
    ("sensors.1.len_t", 0.0, "len_t > 0"),
]


@pytest.mark.parametrize("path,value,message", FAULTS, ids=[f"{p}={v}" for p, v, _ in FAULTS])
def test_corrupt_scene_is_refused_before_the_gpu(path, value, message):
    sc, keep = _scene()
    _set(sc, path, value)
    h = C.c_void_p()
    with pytest.raises(ValueError, match=message):
        N.check(N.lib().lmc_create(C.byref(sc), C.byref(h)))
    assert not h.value


def test_phase_table_faults_are_refused():
    """A sampling table whose CDF decreases, or an HG g outside [-1, 1], is refused."""
    sc, keep = _scene()
    cdf = (C.c_double * sc.media[0].theta_n)()
    C.memmove(cdf, sc.media[0].theta_cdf, C.sizeof(cdf))
    cdf[5], cdf[6] = cdf[6], cdf[5] - 0.5
    sc.media[0].theta_cdf = C.cast(cdf, C.POINTER(C.c_double))
    h = C.c_void_p()
    with pytest.raises(ValueError, match="non-decreasing"):
        N.check(N.lib().lmc_create(C.byref(sc), C.byref(h)))
    sc2, keep2 = _scene(W.bilayer_hg)
    sc2.media[0].hg_g = 1.5
    with pytest.raises(ValueError, match="Henyey-Greenstein g"):
        N.check(N.lib().lmc_create(C.byref(sc2), C.byref(h)))


def test_sweep_names_the_faulty_scene():
    scs = [_scene() for _ in range(3)]
    arr = (N.SceneDesc * 3)(*[s for s, _ in scs])
    arr[2].media[0].mu_s = NAN
    h = C.c_void_p()
    with pytest.raises(ValueError, match="scene 2: medium coefficients"):
        N.check(N.lib().lmc_create_sweep(arr, 3, C.byref(h)))


@pytest.mark.parametrize("what,message", [("scene", "medium coefficients"),
                                           ("precision", "unknown precision"),
                                           ("max_events", "max_events"),
                                           ("reverse_paths", "track_reverse_paths")])
def test_noalloc_refuses_before_the_gpu(what, message):
    sc, keep = _scene()
    o = N.RunOpts()
    o.precision, o.max_events, o.track_reverse_paths = N.PRECISION["fp32"], 1000, 1
    if what == "scene":
        sc.media[0].mu_s = NAN
    elif what == "precision":
        o.precision = 7
    elif what == "max_events":
        o.max_events = -1
    else:
        o.track_reverse_paths = 0           # the scene has a FarFieldCBS grid
    with pytest.raises(ValueError, match=message):
        N.check(N.lib().lmc_run_noalloc(C.byref(sc), 1, 0, 1000, C.byref(o), None, None))


@pytest.mark.skipif(gpu_available(), reason="on a GPU machine the valid scene is created")
def test_valid_scene_passes_validation_and_stops_at_the_device():
    sc, keep = _scene()
    h = C.c_void_p()
    with pytest.raises(RuntimeError):
        N.check(N.lib().lmc_create(C.byref(sc), C.byref(h)))
    assert "CUDA" in N.last_error() or "cuda" in N.last_error()
