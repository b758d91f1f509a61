"""The bounds-checked build of the library (lib/libluminis_b200_checked.so, built with
`luminis-mc_b200/build.py --bounds-check`): its kernels check every inverse-CDF guide
bucket and node, every amplitude node and every tally cell before use, and a failed
check fails the run with LMC_ERR_KERNEL naming the sites.  On the test scenes (every
sensor kind, the Absorption recorder, estimator mode, both transport precisions) no
check fails, and the binary64 tallies equal the product build's.  The checked library
runs in a child process (LUMINIS_B200_LIB selects it), the product build in this one.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import _native as N
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.device import DeviceRun

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys, json, numpy as np
sys.path.insert(0, {repo!r}); sys.path.insert(0, {pkg!r})
import luminis_mc_b200 as lm
from luminis_mc_b200 import _native as N, workloads as W
from luminis_mc_b200.device import DeviceRun
from tests.test_gpu_bounds import scenes
assert N.LIB_PATH.endswith("_checked.so"), N.LIB_PATH
out = {{}}
for spec in scenes():
    for precision in ("fp64", "fp32"):
        cfg, _, keep = W.build(lm, spec)
        run = DeviceRun(cfg)
        st, _ = run.run(spec["n_photons"], spec["seed"], precision=precision)   # raises on a failed check
        if precision == "fp64":
            for i, t in enumerate(run.host_tallies()):
                out[spec["name"] + "/" + str(i)] = t
        run.close()
np.savez(sys.argv[1], **out)
"""


def scenes():
    from tests.golden.make_golden import (absorption_scenes, estimator_scenes, golden_scenes,
                                          statistics_scenes)
    return golden_scenes() + absorption_scenes() + statistics_scenes() + estimator_scenes()[:1]


def test_checked_build_runs_clean_and_agrees(cuda, tmp_path):
    assert os.path.exists(N.CHECKED_LIB_PATH), "build the checked library (build.py --bounds-check)"
    path = str(tmp_path / "checked.npz")
    env = dict(os.environ, LUMINIS_B200_LIB=N.CHECKED_LIB_PATH)
    code = CHILD.format(repo=REPO, pkg=os.path.join(REPO, "luminis-mc_b200"))
    r = subprocess.run([sys.executable, "-c", code, path], env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    got = dict(np.load(path))
    for spec in scenes():
        cfg, _, keep = W.build(lm, spec)
        run = DeviceRun(cfg)
        run.run(spec["n_photons"], spec["seed"], precision="fp64")
        for i, (t, s) in enumerate(zip(run.host_tallies(), spec["sensors"])):
            tol = 1e-6 if s["kind"] == "planar_field" else 1e-9
            g = got[spec["name"] + "/" + str(i)]
            np.testing.assert_allclose(g, t, rtol=tol, atol=tol * max(np.abs(t).max(), 1e-300),
                                       err_msg=f"{spec['name']} sensor {i}")
        run.close()
