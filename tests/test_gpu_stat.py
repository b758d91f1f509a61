"""Statistical parity on the GPU: the CUDA transport (Philox stream, FP32 and FP64)
agrees bin by bin with the UNMODIFIED reference driven by its own xoshiro256++
stream (tests/golden/stat_ref_*.npz: 16 replicas x 1e5 photons), including the
coherent (CBS) grids, at equal per-photon tally sigma.  Same bars as the CPU
statistical oracle test (tests/statcheck.py)."""
import os

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.device import DeviceRun
from tests import statcheck as S
from tests.golden.make_golden import stat_scenes

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
R, N = 16, 200_000


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("spec", stat_scenes(), ids=lambda s: s["name"])
def test_gpu_agrees_with_reference_rng(spec, precision, cuda):
    ref = np.load(os.path.join(HERE, "golden", f"stat_ref_{spec['name']}.npz"))
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    reps = []
    for r in range(R):
        run.zero()
        run.run(N, 9000 + r, precision=precision)
        reps.append([t.copy() for t in run.host_tallies()])
    run.close()
    for i, (m, v) in enumerate(S.moments(reps, N)):
        kind = spec["sensors"][i]["kind"]
        res = S.compare(m, v, R, N, ref[f"sensor{i}_mean"], ref[f"sensor{i}_var"],
                        int(ref["R"]), int(ref["N"]),
                        max_rse=None if kind == "planar_field" else 0.25)
        S.assert_agree(res, f"{spec['name']}/{kind}/{precision}")
