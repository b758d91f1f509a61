"""Parameter sweeps: many independent scenes transported in one launch.

The reference runs a sweep as one run_simulation_parallel call per scene. Here all
scenes share one persistent kernel (lmc_create_sweep / lmc_run_sweep): photons are
numbered across the scenes, scene s owning [P_s, P_s + n_s), and photon g draws the
stream of (seed, g). Scene s therefore gets exactly the tallies of a lone run of that
scene over photons [P_s, P_s + n_s), while short scenes no longer leave the GPU idle
between launches. A run enqueues only device work when no statistics are asked for,
so it can be captured in a CUDA graph and replayed.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .simulation import SimConfig, layout_shape, scene_desc


class SweepRun:
    """Scenes of several SimConfigs with one device tally buffer."""

    def __init__(self, configs: list[SimConfig], device="cuda:0"):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.configs = list(configs)
        n = len(self.configs)
        self._scenes = (N.SceneDesc * n)()
        self._keep = []
        self.sensors = []
        for k, cfg in enumerate(self.configs):
            sc, keep, sensors = scene_desc(cfg)
            self._scenes[k] = sc
            self._keep.append(keep)
            self.sensors.append(sensors)
        with torch.cuda.device(self.device):
            h = C.c_void_p()
            N.check(N.lib().lmc_create_sweep(self._scenes, n, C.byref(h)))
        self._h = h
        total = C.c_size_t()
        N.check(N.lib().lmc_sweep_layout(h, -1, 0, None, C.byref(total), None))
        self.tally_size = int(total.value)
        self.layout = []
        for k in range(n):
            rows = []
            for i in range(len(self.sensors[k])):
                off, cnt = C.c_size_t(), C.c_size_t()
                dims = (C.c_int * 4)()
                N.check(N.lib().lmc_sweep_layout(h, k, i, C.byref(off), C.byref(cnt), dims))
                rows.append((int(off.value), int(cnt.value), layout_shape(cnt, dims)))
            self.layout.append(rows)
        self.tallies = torch.zeros(max(self.tally_size, 1), dtype=torch.float64, device=self.device)
        self.n_scenes = n
        self.photons = None
        self.launch = {}                 # launch shape from autotune(), used by every run

    def set_photons(self, counts) -> None:
        """Photons per scene for the following runs."""
        c = np.ascontiguousarray(np.asarray(counts, dtype=np.uint64))
        assert c.size == self.n_scenes
        N.check(N.lib().lmc_sweep_set_photons(self._h, c.ctypes.data_as(C.POINTER(C.c_uint64))))
        self.photons = c.copy()

    def offsets(self) -> np.ndarray:
        """First photon index of every scene (P_s)."""
        return np.concatenate([[0], np.cumsum(self.photons)[:-1]]).astype(np.uint64)

    def opts(self, precision="fp32", stream=None, max_events=None) -> N.RunOpts:
        c = self.configs[0]
        o = N.RunOpts()
        o.precision = N.PRECISION[precision]
        o.max_events = int(c.MAX_EVENTS if max_events is None else max_events)
        o.track_reverse_paths = int(any(bool(cfg.track_reverse_paths) for cfg in self.configs))
        o.stream = N.launch_stream(stream)
        for key, value in self.launch.items():
            setattr(o, key, value)
        return o

    def autotune(self, seed: int, precision: str = "fp32", sample_photons: int = 10_000_000) -> dict:
        """Pick the launch shape (threads per block, blocks per SM, photons per batch) and
        the tally kernel's mode by timing candidates on a scaled-down copy of the sweep
        (lmc_autotune); later runs use them.  Returns the choice and its rate on the
        sample."""
        if self.photons is None:
            raise ValueError("set_photons() first")
        self.launch = {}
        r = N.TuneResult()
        N.check(N.lib().lmc_autotune(self._h, int(seed) & (2 ** 64 - 1),
                                     C.byref(self.opts(precision)), int(sample_photons),
                                     C.byref(r)))
        self.launch = {"block_size": r.block_size, "blocks_per_sm": r.blocks_per_sm,
                       "batch_photons": r.batch_photons, "tally_mode": r.tally_mode}
        return r.as_dict()

    def run(self, seed: int, precision: str = "fp32", stream=None, want_stats: bool = True):
        """Transport every scene's photons, adding into self.tallies; stats or {}."""
        if self.photons is None:
            raise ValueError("set_photons() first")
        o = self.opts(precision, stream)
        st = N.Stats()
        N.check(N.lib().lmc_run_sweep(self._h, int(seed) & (2 ** 64 - 1), C.byref(o),
                                      C.c_void_p(self.tallies.data_ptr()),
                                      C.byref(st) if want_stats else None))
        return st.as_dict() if want_stats else {}

    def adjoint_layout(self, radial_sensor: int = -1, radial_bins: int = 100,
                       radial_max: float = 5.0):
        """Options and per-scene blocks [(offset, n_out, n_params)] of the likelihood-ratio
        outputs (lmc_sweep_adjoint_layout), and the buffer's total size."""
        a = N.AdjointOpts(int(radial_sensor), int(radial_bins), float(radial_max))
        off, n, k = C.c_size_t(), C.c_size_t(), C.c_int()
        N.check(N.lib().lmc_sweep_adjoint_layout(self._h, C.byref(a), -1, C.byref(off),
                                                 C.byref(n), C.byref(k)))
        total = int(n.value)
        blocks = []
        for s in range(self.n_scenes):
            N.check(N.lib().lmc_sweep_adjoint_layout(self._h, C.byref(a), s, C.byref(off),
                                                     C.byref(n), C.byref(k)))
            blocks.append((int(off.value), int(n.value), int(k.value)))
        return a, blocks, total

    def run_adjoint(self, seed: int, precision: str = "fp32", adjoint=None, stream=None,
                    want_stats: bool = True, **layout):
        """Transport every scene's photons with likelihood-ratio outputs: adds the tallies
        into self.tallies and returns (per scene (outputs [n_out], jacobian [n_params, n_out])
        as sums over its photons, stats).  `adjoint`: a device buffer to add into instead."""
        if self.photons is None:
            raise ValueError("set_photons() first")
        torch = self.torch
        a, blocks, total = self.adjoint_layout(**layout)
        buf = adjoint if adjoint is not None else torch.zeros(max(total, 1), dtype=torch.float64,
                                                              device=self.device)
        o = self.opts(precision, stream)
        st = N.Stats()
        N.check(N.lib().lmc_run_sweep_adjoint(self._h, int(seed) & (2 ** 64 - 1), C.byref(o),
                                              C.byref(a), C.c_void_p(self.tallies.data_ptr()),
                                              C.c_void_p(buf.data_ptr()),
                                              C.byref(st) if want_stats else None))
        out = []
        for off, n, k in blocks:
            blk = buf[off:off + (1 + k) * n].view(1 + k, n)
            out.append((blk[0], blk[1:]))
        return out, (st.as_dict() if want_stats else {})

    def capture(self, seed: int, precision: str = "fp32"):
        """A CUDA graph of one run (after one uncaptured run of the same size has grown
        the hit queue): replay() adds another run's tallies."""
        torch = self.torch
        s = torch.cuda.Stream(device=self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
            self.run(seed, precision, stream=s.cuda_stream, want_stats=False)
        return g

    def zero(self):
        self.tallies.zero_()

    def host_tallies(self, scene: int):
        self.torch.cuda.synchronize(self.device)
        flat = self.tallies.cpu().numpy()
        return [flat[o:o + c].reshape(d) for (o, c, d) in self.layout[scene]]

    def host_absorption(self, scene: int):
        """Scene `scene`'s Absorption grid [n_t][n_r][n_z] (None without one)."""
        off, cnt = C.c_size_t(), C.c_size_t()
        dims = (C.c_int * 4)()
        N.check(N.lib().lmc_sweep_layout(self._h, scene, N.TALLY_ABSORPTION, C.byref(off),
                                         C.byref(cnt), dims))
        if not cnt.value:
            return None
        self.torch.cuda.synchronize(self.device)
        flat = self.tallies.cpu().numpy()
        return flat[off.value:off.value + cnt.value].reshape(tuple(dims[:3]))

    def hits(self) -> np.ndarray:
        """[n_scenes, n_sensors max] hit counts of the last run."""
        out = np.zeros(self.n_scenes * N.MAX_SENSORS, dtype=np.uint64)
        N.check(N.lib().lmc_sweep_hits(self._h, out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out.reshape(self.n_scenes, N.MAX_SENSORS)

    def close(self):
        if getattr(self, "_h", None):
            N.lib().lmc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
