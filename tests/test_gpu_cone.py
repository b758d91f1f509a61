"""The CBS cone at the workloads' own resolution, statistically against the UNMODIFIED
reference driven by its own xoshiro256++ stream (tests/golden/cone_ref_*.npz: 16
replicas x 1e6 photons, written by `make_golden.py cone`).

Two detectors, each exactly as its workload defines it (FarFieldCBSSensor,
src/detector.cpp:1231-1310):
  * cone_mie: mie_cbs_small's 100 theta bins of 1 mrad to 0.1 rad, one phi bin,
    mu_a = 0.01/mm, linear polarisation;
  * cone_bilayer: bilayer_rgd_mie's 200 x 8 grid to 0.1 rad on the RGD-over-Mie slab,
    circular polarisation.

Checks, for the CUDA transport in FP32 and in FP64 (Philox stream, independent seeds):
  * every well-populated bin of the 8 Stokes grids, Welch t against the reference
    (tests/statcheck.py bars);
  * the enhancement eta = S0_coh / S0_incoh inside 5, 10 and 20 mrad of exact
    backscatter, one ratio per replica, Welch t against the reference's replicas;
  * the S0 coherent and incoherent theta profiles in 10 mrad rings.

Bars calibrated on the reference against itself (a second set of 16 replicas with
other seeds): on the 200 x 8 grid the largest |t| over 3263 populated bins was 5.06
(0.6 % beyond 3 sigma, mean t^2 1.13), on the 100-bin grid 3.1 over 367 bins (mean
t^2 0.94); the enhancement ratios and ring sums stayed within |t| <= 2.3.  Per-photon
weights are heavy-tailed, so the largest |t| of thousands of bins runs above a normal
variate's; the grid bar is 6.5 here.  The cone itself, ~lambda / (2 pi l*) ~ 0.1 mrad
wide for these media, is narrower than one bin, so eta over a ring is close to 1.
"""
import os

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.device import DeviceRun
from tests import statcheck as S
from tests.golden.make_golden import cone_profiles, cone_scenes

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
R, N = 16, 1_000_000
MAX_T_RING = 4.0         # |t| bar for each enhancement ratio and ring sum


def welch(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    se = np.sqrt(a.var(ddof=1) / a.size + b.var(ddof=1) / b.size)
    return float((a.mean() - b.mean()) / se)


def _gpu_replicas(spec, precision):
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    reps, coh, inc = [], [], []
    for r in range(R):
        run.zero()
        run.run(N, 9000 + r, precision=precision)
        t = [x.copy() for x in run.host_tallies()]
        reps.append(t)
        c, i = cone_profiles(t[0])
        coh.append(c)
        inc.append(i)
    run.close()
    return reps, np.stack(coh), np.stack(inc)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("spec", cone_scenes(), ids=lambda s: s["name"])
def test_cone_agrees_with_reference_rng(spec, precision, cuda):
    ref = np.load(os.path.join(HERE, "golden", f"cone_ref_{spec['name']}.npz"))
    reps, coh, inc = _gpu_replicas(spec, precision)
    what = f"{spec['name']}/{precision}"
    (m, v), = S.moments(reps, N)
    res = S.compare(m, v, R, N, ref["sensor0_mean"], ref["sensor0_var"], int(ref["R"]), int(ref["N"]))
    S.assert_agree(res, what + "/grid", max_abs_t=6.5, min_tested=100)

    d_theta = spec["sensors"][0]["d_theta"]
    for mrad in (5, 10, 20):
        k = int(round(mrad * 1e-3 / d_theta))
        eta_gpu = coh[:, :k].sum(axis=1) / inc[:, :k].sum(axis=1)
        eta_ref = ref["coh_theta"][:, :k].sum(axis=1) / ref["incoh_theta"][:, :k].sum(axis=1)
        t = welch(eta_gpu, eta_ref)
        assert abs(t) <= MAX_T_RING, f"{what}: eta within {mrad} mrad, t = {t:.2f} " \
                                     f"(gpu {eta_gpu.mean():.4f}, reference {eta_ref.mean():.4f})"
        assert eta_gpu.mean() < 2.05, f"{what}: eta = {eta_gpu.mean():.4f} within {mrad} mrad"

    ring = int(round(10e-3 / d_theta))
    for lo in range(0, coh.shape[1], ring):
        for name, g, r in (("coherent", coh, ref["coh_theta"]), ("incoherent", inc, ref["incoh_theta"])):
            t = welch(g[:, lo:lo + ring].sum(axis=1) / N, r[:, lo:lo + ring].sum(axis=1) / int(ref["N"]))
            assert abs(t) <= MAX_T_RING, f"{what}: S0 {name} ring {lo}..{lo + ring} bins, t = {t:.2f}"
