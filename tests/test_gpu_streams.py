"""Ordering of the library's device work with torch's.

`Transport.run_device(..., want_stats=False)` returns as soon as the run is enqueued.  In
the C ABI a NULL `lmc_run_opts.stream` selects the handle's own non-blocking stream, which
torch's default stream does not wait for: a torch reduction of the tallies issued right
after such a call read zeros.  The Python layer therefore maps its default (None) and
torch's default-stream handle 0 to the legacy default stream, on which torch's
default-stream work runs; a created stream is used as given.  Each case reads the tallies
with torch, without synchronising, right after the call, and must see the whole run.
"""
import pytest
import torch

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W
from luminis_mc_b200.simulation import Transport

pytestmark = pytest.mark.gpu

N_PHOTONS = 4_000_000


@pytest.mark.parametrize("stream", [None, 0, "created"])
def test_run_is_ordered_with_torch_work(stream, cuda):
    spec = W.bilayer_rgd_mie(N_PHOTONS, 1)
    cfg, _, keep = W.build(lm, spec)
    t = Transport(cfg)
    buf = torch.zeros(t.tally_size, dtype=torch.float64, device="cuda:0")
    t.run_device(buf.data_ptr(), N_PHOTONS, 1, 0, want_stats=True)   # reference sum, queue grown
    ref = float(buf.sum().item())
    assert ref > 0
    for _ in range(2):
        buf.zero_()
        torch.cuda.synchronize()
        if stream == "created":
            s = torch.cuda.Stream()
            t.run_device(buf.data_ptr(), N_PHOTONS, 1, 0, want_stats=False, stream=s.cuda_stream)
            with torch.cuda.stream(s):                  # the sum and its read-back on s
                got = float(buf.sum().item())
        else:
            t.run_device(buf.data_ptr(), N_PHOTONS, 1, 0, want_stats=False, stream=stream)
            got = float(buf.sum().item())          # torch's default stream, no synchronise
        # the tallies are sums of FP64 atomics: equal up to the order of the additions
        assert got == pytest.approx(ref, rel=1e-9), (stream, got, ref)
    torch.cuda.synchronize()
    t.close()
