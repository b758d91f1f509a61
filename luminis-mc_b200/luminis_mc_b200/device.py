"""Device-resident runs: tallies and per-photon records kept in GPU memory.

PyTorch is used here only as the allocator and stream provider (plumbing); the
transport itself is the C ABI's lmc_run.
"""
from __future__ import annotations

import numpy as np

from . import _native as N
from .simulation import SimConfig, Transport

RECORD_DTYPE = np.dtype(N.RECORD_FIELDS)


class DeviceRun:
    """A scene with a device tally buffer that accumulates over runs."""

    def __init__(self, config: SimConfig, device="cuda:0"):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        with torch.cuda.device(self.device):
            self.transport = Transport(config)
            self.tallies = torch.zeros(max(self.transport.tally_size, 1), dtype=torch.float64,
                                       device=self.device)

    def zero(self):
        self.tallies.zero_()

    def run(self, n_photons: int, seed: int, begin: int = 0, precision: str = "fp32",
            records: bool = False, want_stats: bool = True, **kw):
        """Transport photons [begin, begin + n_photons); returns (stats, records or None)."""
        torch = self.torch
        rec = None
        if records:
            rec = torch.zeros(n_photons * RECORD_DTYPE.itemsize, dtype=torch.uint8,
                              device=self.device)
        torch.cuda.synchronize(self.device)
        stats = self.transport.run_device(self.tallies.data_ptr(), n_photons, seed, begin,
                                          want_stats=want_stats or records, precision=precision,
                                          records_ptr=rec.data_ptr() if rec is not None else None,
                                          **kw)
        out = None
        if rec is not None:
            out = rec.cpu().numpy().view(RECORD_DTYPE)
        return stats, out

    def host_absorption(self):
        """The Absorption grid [n_t][n_r][n_z] of the device tallies (None without one)."""
        self.torch.cuda.synchronize(self.device)
        return self.transport.absorption_grid(self.tallies.cpu().numpy())

    def host_tallies(self):
        self.torch.cuda.synchronize(self.device)
        flat = self.tallies.cpu().numpy()[: self.transport.tally_size]
        return self.transport.split(flat)

    def close(self):
        self.transport.close()
