"""The tally kernel's modes (lmc_run_opts.tally_mode) give the same tallies.

GLOBAL adds every hit with global atomics.  WARP first combines the adds of a warp's
lanes that fall into one grid cell.  SHARED adds into block-private shared-memory
copies of the grids that fit and adds those into the tallies when each block ends.
In binary64 runs only the order of the binary64 additions differs between them, so
every mode must equal GLOBAL to 1e-12 of each sensor's largest entry.  In binary32
runs each hit's Stokes values are binary32 numbers, and the kernel of each mode may
contract that arithmetic into FMAs differently, so a hit's value can differ in its
last binary32 bit: 1e-9 of the largest entry there.  That is still 5e4 times below
what one lost or doubled hit changes (about 5e-5 of the largest PlanarFluence entry
at 2e5 photons).  Photon, event and hit counts must be equal.  The cases:
* bilayer_rgd_mie: FarFieldCBS 200x8 and FarFieldFluence 90x36 are privatised, and the
  time-resolved PlanarFluence 200x200x64 is too large, so it stays global.  FP32 and
  FP64.
* A coarse time-resolved copy of that scene, where all three grids are privatised.
  This covers slice 0 and the arrival-time slices.
* Likelihood-ratio runs with a radial profile.  The private grids sit after the
  radial outputs in shared memory.
* lmc_run_noalloc with SHARED against lmc_run with GLOBAL.
Sweeps accept GLOBAL and WARP and refuse SHARED.  lmc_autotune reports the mode it
picked.
"""
import copy
import ctypes as C

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import _native as N
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.adjoint import AdjointTransport
from luminis_mc_b200.device import DeviceRun
from luminis_mc_b200.sweep import SweepRun

pytestmark = pytest.mark.gpu

RTOL = 1e-12         # summation order of binary64 atomics, relative to a sensor's largest entry
RTOL_FP32 = 1e-9     # plus a last-bit binary32 difference per hit value
MODES = ("warp", "shared")


def _coarse_timed(n, seed):
    """bilayer_rgd_mie with coarse, time-resolved grids that all fit in shared memory."""
    spec = copy.deepcopy(W.bilayer_rgd_mie(n, seed))
    cbs, pf, fff = spec["sensors"]
    cbs.update(len_t=40.0, d_t=4.0, d_theta=0.01)
    pf.update(len_t=64.0, d_t=8.0, dx=1.0, dy=1.0)
    fff.update(len_t=40.0, d_t=4.0, d_theta=W.PI / 18, d_phi=W.PI / 9)
    return spec


def _run(cfg, n, seed, precision, mode, begin=0):
    run = DeviceRun(cfg)
    st, _ = run.run(n, seed, begin, precision=precision, tally_mode=mode)
    out = run.host_tallies()
    run.close()
    return out, st


def _same(got, want, gst, wst, tol=RTOL):
    for g, w in zip(got, want):
        np.testing.assert_allclose(g, w, rtol=0, atol=tol * max(np.abs(w).max(), 1e-300))
    for key in ("photons", "events", "detected", "escaped", "hits"):
        assert gst[key] == wst[key], key
    assert gst["error_flags"] == 0


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("make", [W.bilayer_rgd_mie, _coarse_timed], ids=["bilayer_rgd_mie", "coarse_timed"])
def test_modes_match_global(make, precision, cuda):
    cfg, _, keep = W.build(lm, make(200_000, 77))
    want, wst = _run(cfg, 200_000, 77, precision, "global", begin=1000)
    assert min(wst["hits"][:3]) > 0
    for mode in MODES:
        got, gst = _run(cfg, 200_000, 77, precision, mode, begin=1000)
        _same(got, want, gst, wst, RTOL_FP32 if precision == "fp32" else RTOL)


def test_shared_mode_over_several_batches(cuda):
    """SHARED equals GLOBAL over several hit-queue batches too: each batch's tally
    launch zeroes its blocks' private grids and adds them into the tallies again."""
    cfg, _, keep = W.build(lm, _coarse_timed(300_000, 5))
    want, wst = _run(cfg, 300_000, 5, "fp32", "global")
    run = DeviceRun(cfg)
    gst, _ = run.run(300_000, 5, precision="fp32", tally_mode="shared", batch_photons=70_000)
    got = run.host_tallies()
    run.close()
    _same(got, want, gst, wst, RTOL_FP32)


@pytest.mark.parametrize("mode", MODES)
def test_likelihood_ratio_outputs_unchanged(mode, cuda):
    cfg, _, keep = W.build(lm, W.bilayer_hg(100_000, 9))
    tr = AdjointTransport(cfg, radial_sensor=1, radial_bins=20, radial_max=5.0)
    out0, jac0, st0 = tr.run(100_000, 9, precision="fp64", tally_mode="global")
    t0 = tr.last_tallies.cpu().numpy()
    out1, jac1, st1 = tr.run(100_000, 9, precision="fp64", tally_mode=mode)
    t1 = tr.last_tallies.cpu().numpy()
    tr.close()
    for a, b in ((out1, out0), (jac1, jac0)):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        np.testing.assert_allclose(a, b, rtol=0, atol=RTOL * np.abs(b).max())
    np.testing.assert_allclose(t1, t0, rtol=0, atol=RTOL * np.abs(t0).max())
    assert st1["hits"] == st0["hits"] and st1["events"] == st0["events"]


def test_noalloc_shared_matches_lmc_run(cuda):
    import torch
    cfg, _, keep = W.build(lm, W.bilayer_rgd_mie(100_000, 31))
    want, wst = _run(cfg, 100_000, 31, "fp64", "global")
    run = DeviceRun(cfg)
    d = torch.zeros(max(run.transport.tally_size, 1), dtype=torch.float64, device=run.device)
    torch.cuda.synchronize()
    st = N.Stats()
    o = run.transport.opts(precision="fp64", tally_mode="shared")
    N.check(N.lib().lmc_run_noalloc(C.byref(run.transport.scene), 31, 0, 100_000, C.byref(o),
                                    C.c_void_p(d.data_ptr()), C.byref(st)))
    got = run.transport.split(d.cpu().numpy()[: run.transport.tally_size])
    run.close()
    _same(got, want, st.as_dict(), wst)


def test_sweep_modes(cuda):
    from tests.test_gpu_sweep import _specs
    specs = _specs()[:3]
    counts = [20000, 7000, 13000]
    sw = SweepRun([W.build(lm, s)[0] for s in specs])
    sw.set_photons(counts)
    sw.launch = {"tally_mode": N.TALLY_MODES["global"]}
    st0 = sw.run(3, precision="fp64")
    base = [sw.host_tallies(k) for k in range(3)]
    sw.zero()
    sw.launch = {"tally_mode": N.TALLY_MODES["warp"]}
    st1 = sw.run(3, precision="fp64")
    assert st1["photons"] == st0["photons"] and st1["events"] == st0["events"]
    for k in range(3):
        for a, b in zip(sw.host_tallies(k), base[k]):
            np.testing.assert_allclose(a, b, rtol=0, atol=RTOL * max(np.abs(b).max(), 1e-300))
    sw.launch = {"tally_mode": N.TALLY_MODES["shared"]}
    with pytest.raises(ValueError, match="single-scene"):
        sw.run(3, precision="fp64")
    r = sw.autotune(3, precision="fp32", sample_photons=20000)
    assert r["tally_mode"] in (N.TALLY_MODES["global"], N.TALLY_MODES["warp"])
    sw.close()


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_sweep_adjoint_warp_matches_global(precision, cuda):
    """A sweep with each scene's gradients (the path the bench's sweep arm takes when the
    autotuner picks warp-combined adds): outputs, Jacobians and tallies as with global
    atomics."""
    from tests.test_gpu_sweep import _specs
    specs = _specs()[:3]
    sw = SweepRun([W.build(lm, s)[0] for s in specs])
    sw.set_photons([15000, 6000, 9000])
    got = {}
    for mode in ("global", "warp"):
        sw.zero()
        sw.launch = {"tally_mode": N.TALLY_MODES[mode]}
        blocks, st = sw.run_adjoint(21, precision=precision)
        got[mode] = ([(o.cpu().numpy(), j.cpu().numpy()) for o, j in blocks],
                     [sw.host_tallies(k) for k in range(3)], st)
    sw.close()
    tol = RTOL_FP32 if precision == "fp32" else RTOL
    (b0, t0, s0), (b1, t1, s1) = got["global"], got["warp"]
    assert s1["events"] == s0["events"] and s1["photons"] == s0["photons"]
    for (o0, j0), (o1, j1) in zip(b0, b1):
        np.testing.assert_allclose(o1, o0, rtol=0, atol=tol * max(np.abs(o0).max(), 1e-300))
        np.testing.assert_allclose(j1, j0, rtol=0, atol=tol * max(np.abs(j0).max(), 1e-300))
    for a, b in zip(t1, t0):
        for x, y in zip(a, b):
            np.testing.assert_allclose(x, y, rtol=0, atol=tol * max(np.abs(y).max(), 1e-300))


def test_autotune_reports_a_mode(cuda):
    from luminis_mc_b200.simulation import Transport
    t = Transport(W.build(lm, W.bilayer_rgd_mie(0, 1))[0])
    r = t.autotune(1, precision="fp32", sample_photons=200_000)
    assert r["tally_mode"] in (1, 2, 3) and r["photons_per_s"] > 0
    t.close()


def test_bad_mode_is_refused(cuda):
    cfg, _, keep = W.build(lm, W.mie_cbs_small(1000, 1))
    run = DeviceRun(cfg)
    o = run.transport.opts(precision="fp32")
    o.tally_mode = 7
    with pytest.raises(ValueError, match="tally_mode"):
        N.check(N.lib().lmc_run(run.transport._h, 1, 0, 1000, C.byref(o),
                                C.c_void_p(run.tallies.data_ptr()), None))
    run.close()
