"""Persistence compatibility with the reference's HDF5 layout.

The reference persists sensors with `Experiment.save_sensor`
(python/luminis_mc/manager.py:814-868).  Its schema registry
(python/luminis_mc/schema.py:30-133) names the attributes written under
/sensors/<name>/meta and the arrays written under /sensors/<name>/data.  This package's
sensors carry the same class names, attributes and array layouts.  So a user who
switches the simulation to the GPU keeps the reference's own writer, and it writes the
same file.

The test runs that writer, unchanged, from the reference's source tree.  Its HDF5 groups
are a small in-memory stand-in, because h5py is absent from this image.  The writer runs
on two sets of sensors:
* the reference's own, after its own run (the `pin` build, its xoshiro256++ RNG);
* this package's, holding the oracle's tallies for the same scene, seed and RNG.  The
  oracle reproduces the `pin` build bit for bit there (tests/test_oracle_golden.py), and
  they are added into the sensors as `run_simulation_parallel` adds the GPU's.
Both must give the same tree: groups, attribute names and values, dataset names, shapes,
dtypes and contents.  The scenes cover the four sensor classes the reference has, with
time bins, theta limits and a direction filter.
"""
import importlib.util
import os
import subprocess
import sys
import types

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W
from oracle import pyoracle as O
from tests.golden.make_golden import golden_scenes, statistics_scenes

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.reference


class _Group:
    """The part of h5py's Group API that save_sensor uses, kept in memory."""

    def __init__(self):
        self.attrs = {}
        self.members = {}

    def require_group(self, name):
        return self.members.setdefault(name, _Group())

    def __contains__(self, name):
        return name in self.members

    def __delitem__(self, name):
        del self.members[name]

    def create_dataset(self, name, data=None, **_compression):
        self.members[name] = np.array(data)
        return self.members[name]


def _reference_source() -> str:
    """The reference's source tree: LUMINIS_REFERENCE_SRC, else oracle/Makefile's."""
    src = os.environ.get("LUMINIS_REFERENCE_SRC")
    if not src:
        src = subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "print-ref"],
                             check=True, capture_output=True, text=True).stdout.strip()
    return src


@pytest.fixture(scope="module")
def writer():
    """The reference's Experiment.save_sensor, loaded from its sources with the in-memory
    groups standing in for h5py (which it imports at module level)."""
    pkg_dir = os.path.join(_reference_source(), "python", "luminis_mc")
    if not os.path.exists(os.path.join(pkg_dir, "manager.py")):
        pytest.skip("the reference's Python sources are not on this machine")
    stub = types.ModuleType("h5py")
    stub.Group, stub.Dataset, stub.File = _Group, np.ndarray, _Group
    saved = sys.modules.get("h5py")
    sys.modules["h5py"] = stub
    name = "_luminis_reference_persistence"
    pkg = types.ModuleType(name)
    pkg.__path__ = [pkg_dir]
    sys.modules[name] = pkg
    try:
        for mod in ("schema", "records", "manager"):
            spec = importlib.util.spec_from_file_location(f"{name}.{mod}",
                                                          os.path.join(pkg_dir, f"{mod}.py"))
            m = importlib.util.module_from_spec(spec)
            sys.modules[spec.name] = m
            spec.loader.exec_module(m)
    finally:
        if saved is None:
            sys.modules.pop("h5py", None)
        else:
            sys.modules["h5py"] = saved
    manager = sys.modules[f"{name}.manager"]
    exp = manager.Experiment.__new__(manager.Experiment)   # no directory, no file
    exp.h5 = types.SimpleNamespace(flush=lambda: None)

    def save(sensor):
        root = _Group()
        exp.g_sensors = root
        exp.save_sensor(sensor, "sensor")
        return root.members["sensor"]
    return save


def _reference():
    try:
        return O.reference_module("pin")
    except ImportError as e:
        pytest.skip(str(e))


def _assert_same_tree(a, b, path):
    assert isinstance(a, _Group) and isinstance(b, _Group), path
    assert sorted(a.attrs) == sorted(b.attrs), f"{path}: attributes differ"
    for k in a.attrs:
        va, vb = a.attrs[k], b.attrs[k]
        assert type(va) is type(vb), f"{path}@{k}: {type(va).__name__} against {type(vb).__name__}"
        if isinstance(va, np.ndarray):
            np.testing.assert_array_equal(va, vb, err_msg=f"{path}@{k}")
        else:
            assert va == vb, f"{path}@{k}: {va!r} against {vb!r}"
    assert sorted(a.members) == sorted(b.members), f"{path}: members differ"
    for k, va in a.members.items():
        vb = b.members[k]
        if isinstance(va, _Group):
            _assert_same_tree(va, vb, f"{path}/{k}")
        else:
            assert va.shape == vb.shape and va.dtype == vb.dtype, f"{path}/{k}"
            np.testing.assert_array_equal(va, vb, err_msg=f"{path}/{k}")


SCENES = [s for s in golden_scenes() if s["name"] in ("bilayer_small", "mie_speckle_small")] + \
         [s for s in statistics_scenes() if s["name"] == "stats_bilayer"]


@pytest.mark.parametrize("spec", SCENES, ids=lambda s: s["name"])
def test_reference_writer_gives_the_same_tree(spec, writer):
    ref = _reference()
    ref.set_log_level(ref.LogLevel.off)
    n, seed = int(spec["n_photons"]), int(spec["seed"])
    cfg_r, hs_r, keep_r = W.build(ref, spec, n_threads=1)
    ref.run_simulation_parallel(cfg_r)
    cfg_p, hs_p, keep_p = W.build(lm, spec)
    res = O.Oracle(spec).run(n, seed, rng="xoshiro")
    for i, s in enumerate(hs_p):            # as run_simulation_parallel adds the GPU's
        s._tally += np.ravel(res.tallies[i])
        s.hits += int(res.hits[i])
    assert sum(s.hits for s in hs_r) > 0
    for i, (mine, theirs) in enumerate(zip(hs_p, hs_r)):
        assert type(mine).__name__ == type(theirs).__name__
        assert mine.hits == theirs.hits, f"sensor {i}: hits"
        _assert_same_tree(writer(mine), writer(theirs), f"{spec['name']}/sensor{i}")


def test_enums_are_stored_by_name(writer):
    """The sensor's direction filter is an enum in both packages, stored by its name."""
    s = lm.StatisticsSensor(0.0, False)
    s.set_direction_limit(lm.CrossingDirection.Backward)
    meta = writer(s).members["meta"].attrs
    assert meta["filter_direction"] == "Backward" and meta["filter_direction_enabled"] is True
