"""The reference-side binding (luminis_mc_b200.refbind) reads the reference's OWN objects.

A SimConfig built with the reference's Python API (its pybind module, built from its
sources under oracle/_ref) must reach the GPU as exactly the scene the package builds
from its mirror objects for the same workload: the C scene byte for byte, and every
sampling and amplitude table bit for bit.  The binding reads the phase functions'
private SamplingTables and the media's DataTables directly, so the GPU samples the
reference's own tables.  Errors follow the reference (ValueError for a config without
sample, laser or detector).  No GPU is needed: nothing here runs the transport.
"""
import ctypes as C
import sys

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import refbind
from luminis_mc_b200 import simulation as S
from luminis_mc_b200 import workloads as W
from oracle import pyoracle as O
from tests.golden.make_golden import (absorption_scenes, estimator_scenes, golden_scenes,
                                      mixture_scenes, statistics_scenes)


def reference():
    """Whichever build of the reference this process imported, else the pin build."""
    loaded = sys.modules.get("luminis_mc")
    if loaded is not None:
        return loaded
    try:
        return O.reference_module("pin")
    except ImportError as e:
        pytest.skip(str(e))


def _binding():
    try:
        return refbind.module()
    except ImportError as e:
        pytest.skip(str(e))


def _scenes():
    out = [W.bilayer_hg(1000, 3), W.mixture_bilayer(1000, 3), W.mie_long_paths(100, 3),
           W.mixture_cbs_small(100, 3)]
    out += golden_scenes() + statistics_scenes() + absorption_scenes() + mixture_scenes()
    out += estimator_scenes()
    for s in out:       # FarFieldFluence is this package's sensor: the reference has no class
        s["sensors"] = [x for x in s["sensors"] if x["kind"] != "farfield_fluence"]
    return out


def _tables(m):
    def arr(p, n):
        return np.ctypeslib.as_array(p, (n,)).copy() if n else np.zeros(0)
    return (arr(m.theta_values, m.theta_n), arr(m.theta_cdf, m.theta_n),
            arr(m.amp_s1, 2 * m.amp_n), arr(m.amp_s2, 2 * m.amp_n))


@pytest.mark.parametrize("spec", _scenes(), ids=lambda s: s["name"])
def test_scene_from_reference_objects_equals_the_package_scene(spec):
    ref = reference()
    _binding()
    ref.set_log_level(ref.LogLevel.off)
    cfg_r, _, keep_r = W.build(ref, spec)
    got, tables = refbind.describe(cfg_r)
    cfg_m, _, keep_m = W.build(lm, spec)
    want, keep, _ = S.scene_desc(cfg_m)
    assert got.n_media == want.n_media
    for i in range(want.n_media):
        for a, b in zip(_tables(want.media[i]), tables[i]):
            assert a.tobytes() == b.tobytes()
        m = want.media[i]
        m.theta_values = m.theta_cdf = m.amp_s1 = m.amp_s2 = None
    assert bytes(got) == bytes(want)


def test_binding_rejects_missing_pointers_like_the_reference():
    ref = reference()
    _binding()
    cfg, _, keep = W.build(ref, W.mie_cbs_small(10, 1))
    cfg.laser = None
    with pytest.raises(ValueError, match="laser"):
        refbind.run_simulation_parallel(cfg)
    cfg = ref.SimConfig()
    with pytest.raises(ValueError, match="sample"):
        refbind.describe(cfg)
    with pytest.raises(ValueError, match="precision"):
        refbind.run_simulation_parallel(cfg, precision="fp16")


def test_binding_refuses_photon_record_sensor():
    ref = reference()
    _binding()
    cfg, _, keep = W.build(ref, W.mie_cbs_small(10, 1))
    rec = cfg.detector.add_detector(ref.PhotonRecordSensor(0.0, True))
    with pytest.raises(NotImplementedError, match="PhotonRecordSensor"):
        refbind.describe(cfg)
