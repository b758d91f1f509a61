"""run_simulation_parallel for the reference's OWN objects.

A user of the reference keeps building the scene with its Python API
(``import luminis_mc``: Sample, media, phase functions, Laser, SensorsGroup, SimConfig,
python/python_module.cpp:114-673) and swaps one call::

    import luminis_mc                                  # the reference
    from luminis_mc_b200 import refbind
    refbind.run_simulation_parallel(config)            # instead of luminis_mc.run_...
    out = luminis_mc.postprocess_farfield_cbs(det, config.n_photons)   # unchanged

The photons are transported on the GPU and every sensor's tallies and hit count are
ADDED into the reference's own sensor objects, as the reference's
run_simulation_parallel merges its worker clones into them (src/simulation.cpp:233-243),
so the reference's postprocess_* and any code reading its arrays work unchanged.

The work is done by the compiled module ``lib/_lmc_refbind`` (refbind/lmc_refbind.cpp),
built against the reference's headers (``make -C luminis-mc_b200/refbind REF=...``).
It reads the reference's objects through its pybind11 type registry, so the
reference's ``luminis_mc`` must be imported first, built with the same compiler and
pybind11 version.
"""
from __future__ import annotations

import importlib.util
import os
import sysconfig

import numpy as np

from . import _native as N

_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
_mod = None


def module():
    """The compiled binding (ImportError if it was not built)."""
    global _mod
    if _mod is None:
        N.lib()                                           # libluminis_b200.so first (rpath)
        path = os.path.join(_LIB, "_lmc_refbind" + sysconfig.get_config_var("EXT_SUFFIX"))
        if not os.path.exists(path):
            raise ImportError(f"{path} is not built: make -C luminis-mc_b200/refbind REF=<reference>")
        spec = importlib.util.spec_from_file_location("_lmc_refbind", path)
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        _mod = m
    return _mod


def run_simulation_parallel(config, precision: str = "fp32") -> dict:
    """The reference's run_simulation_parallel(config) on the GPU (blocking; tallies and
    hits added into config.detector's sensors and config.absorption).  Raises ValueError
    as the reference does for a config without sample, laser or detector, and
    NotImplementedError for objects the GPU transport does not cover
    (PhotonRecordSensor).  Returns the run's counters."""
    return module().run_simulation_parallel(config, precision)


def describe(config):
    """The C scene (``_native.SceneDesc``, table pointers cleared) the binding builds from
    the reference's config, and per medium its (theta values, theta cdf, S1, S2) tables
    as float64 arrays (S1, S2 interleaved re, im)."""
    raw, tables = module().describe(config)
    sc = N.SceneDesc.from_buffer_copy(raw)
    return sc, [tuple(np.frombuffer(t, dtype=np.float64) for t in m) for m in tables]
