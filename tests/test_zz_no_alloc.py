"""lmc_run_noalloc, the allocation-free entry point, against lmc_run.

lmc_run_noalloc keeps its device scene, tables, counters and hit queue in one
static device array instead of allocating them.  Its results must equal those of
lmc_create + lmc_run on the same scene, seed and photon range within the GPU
parity tests' FP64 tolerance, on consecutive calls (the array keeps the previous
call's contents, so the second call checks that everything that must start at
zero does), and when a run needs several hit-queue batches.  The file is named
to be collected last, after the other GPU tests have used the device.
"""
import ctypes as C

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import _native as N
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.device import DeviceRun

pytestmark = pytest.mark.gpu

RTOL = 1e-9          # the FP64 tally tolerance of tests/test_gpu_parity.py


def _noalloc(run, n, seed, begin, precision, scene=None):
    """One lmc_run_noalloc call into fresh device tallies; returns (tallies, stats)."""
    import torch
    d = torch.zeros(max(run.transport.tally_size, 1), dtype=torch.float64, device=run.device)
    torch.cuda.synchronize()
    st = N.Stats()
    o = run.transport.opts(precision=precision)
    sc = run.transport.scene if scene is None else scene
    N.check(N.lib().lmc_run_noalloc(C.byref(sc), seed, begin, n, C.byref(o),
                                    C.c_void_p(d.data_ptr()), C.byref(st)))
    flat = d.cpu().numpy()[: run.transport.tally_size]
    return run.transport.split(flat), st.as_dict()


def _lmc_run(cfg, n, seed, begin, precision):
    run = DeviceRun(cfg)
    st, _ = run.run(n, seed, begin, precision=precision)
    out = run.host_tallies()
    run.close()
    return out, st


def _same(got, want, gst, wst):
    for g, w in zip(got, want):
        np.testing.assert_allclose(g, w, rtol=RTOL, atol=RTOL * max(np.abs(w).max(), 1e-300))
    for key in ("photons", "events", "detected", "escaped", "hits"):
        assert gst[key] == wst[key], key
    assert gst["error_flags"] == 0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("make", [W.mie_cbs_small, W.bilayer_rgd_mie, W.mixture_bilayer],
                         ids=["mie_cbs_small", "bilayer_rgd_mie", "mixture_bilayer"])
def test_noalloc_matches_lmc_run_twice(make, precision, cuda):
    spec = make(3000, 2024)
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    for n, seed, begin in ((3000, 2024, 0), (2500, 99, 7000)):
        got, gst = _noalloc(run, n, seed, begin, precision)
        want, wst = _lmc_run(cfg, n, seed, begin, precision)
        _same(got, want, gst, wst)
    run.close()


def test_noalloc_absorption_grid_matches_lmc_run(cuda):
    """The Absorption grid sits after the sensors in the caller's tally buffer."""
    from tests.golden.make_golden import absorption_scenes
    for spec in absorption_scenes():
        import torch
        cfg, _, keep = W.build(lm, spec)
        run = DeviceRun(cfg)
        d = run.transport
        buf = torch.zeros(max(d.tally_size, 1), dtype=torch.float64, device=run.device)
        st = N.Stats()
        o = d.opts(precision="fp64")
        N.check(N.lib().lmc_run_noalloc(C.byref(d.scene), 31, 100, 900, C.byref(o),
                                        C.c_void_p(buf.data_ptr()), C.byref(st)))
        flat = buf.cpu().numpy()[: d.tally_size]
        wst, _ = run.run(900, 31, 100, precision="fp64")
        _same(d.split(flat), run.host_tallies(), st.as_dict(), wst)
        ref = run.host_absorption()
        np.testing.assert_allclose(d.absorption_grid(flat), ref, rtol=RTOL,
                                   atol=RTOL * np.abs(ref).max())
        run.close()


def test_noalloc_statistics_sensors_match_lmc_run(cuda):
    """StatisticsSensor histograms (their bin tables sit in the array's table region),
    queued at z = 0 and tallied in the transport kernel inside the sample."""
    from tests.golden.make_golden import statistics_scenes
    for spec in statistics_scenes():
        cfg, _, keep = W.build(lm, spec)
        run = DeviceRun(cfg)
        for n, seed, begin in ((600, 5, 0), (500, 6, 900)):
            got, gst = _noalloc(run, n, seed, begin, "fp64")
            want, wst = _lmc_run(cfg, n, seed, begin, "fp64")
            _same(got, want, gst, wst)
        run.close()


def test_noalloc_several_queue_batches(cuda):
    """300k photons need several batches of the fixed-size hit queue."""
    spec = W.mie_cbs_small(300_000, 5)
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    got, gst = _noalloc(run, 300_000, 5, 0, "fp64")
    want, wst = _lmc_run(cfg, 300_000, 5, 0, "fp64")
    _same(got, want, gst, wst)
    run.close()


def test_noalloc_records_over_several_batches(cuda):
    """Per-photon records of a run split into batches (a batch_photons below the
    queue's own limit is honoured) equal lmc_run's one-batch records."""
    import torch
    spec = W.bilayer_rgd_mie(1500, 41)
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    _, want = run.run(1500, 41, 200, precision="fp64", records=True)
    from luminis_mc_b200.device import RECORD_DTYPE
    rec = torch.zeros(1500 * RECORD_DTYPE.itemsize, dtype=torch.uint8, device=run.device)
    d = torch.zeros(max(run.transport.tally_size, 1), dtype=torch.float64, device=run.device)
    torch.cuda.synchronize()
    o = run.transport.opts(precision="fp64", records_ptr=rec.data_ptr(), batch_photons=400)
    st = N.Stats()
    N.check(N.lib().lmc_run_noalloc(C.byref(run.transport.scene), 41, 200, 1500, C.byref(o),
                                    C.c_void_p(d.data_ptr()), C.byref(st)))
    got = rec.cpu().numpy().view(RECORD_DTYPE)
    assert got.tobytes() == want.tobytes()
    run.close()


def test_noalloc_rejects_tables_beyond_its_limit(cuda):
    """A scene whose tables exceed the static array's table region is refused with
    a message naming the size, and the next call still works."""
    spec = W.mie_cbs_small(1000, 3)
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg)
    big = N.SceneDesc.from_buffer_copy(run.transport.scene)   # the run's own scene stays intact
    n = 400_000                                      # 32 bytes per entry: > 8 MiB
    vals = np.linspace(0.0, np.pi, n)
    cdf = np.linspace(0.0, 1.0, n)
    m = big.media[0]
    m.theta_kind, m.theta_n = N.THETA_TABLE, n
    m.theta_values, m.theta_cdf = N.as_dptr(vals), N.as_dptr(cdf)
    with pytest.raises(ValueError, match="at most"):
        _noalloc(run, 1000, 3, 0, "fp64", scene=big)
    got, gst = _noalloc(run, 1000, 3, 0, "fp64")
    want, wst = _lmc_run(cfg, 1000, 3, 0, "fp64")
    _same(got, want, gst, wst)
    run.close()
