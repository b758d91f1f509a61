"""run_simulation_parallel on the GPU, and the reference's post-processing.

``run_simulation_parallel(config)`` keeps the reference's contract
(python/python_module.cpp:664-673, src/simulation.cpp:105-249): it blocks, it
ADDS each sensor's contribution into the sensor objects owned by
``config.detector`` and increments their ``hits``, and it raises ValueError for
a config without sample, laser or detector.  The work runs in one CUDA kernel
through the C ABI (include/luminis_b200.h); there is no CPU fallback.
"""
from __future__ import annotations

import atexit
import ctypes as C
import hashlib
import math
import random
import threading

import numpy as np

from . import _native as N
from .core import (FarFieldCBSSensor, FarFieldFluenceSensor, HenyeyGreensteinPhaseFunction,
                   Matrix, MixtureLayer, PlanarFieldSensor, PlanarFluenceSensor,
                   StatisticsSensor, UniformPhaseFunction, _TablePhase,
                   solid_angle_bin)  # noqa: F401


class SimConfig:
    """Run configuration (include/luminis/core/simulation.hpp:67-90)."""

    def __init__(self):
        self.MAX_EVENTS = 1000
        self.batch_size = 0
        self.show_progress = True
        self.progress_interval_pct = 5
        self.seed = random.getrandbits(32)
        self.n_threads = 1
        self.n_photons = 0
        self.pin_threads_to_cores = False
        self.track_reverse_paths = False
        self.sample = None
        self.laser = None
        self.detector = None
        self.absorption = None


_last_stats: dict = {}


def last_run_stats() -> dict:
    """Counters of the most recent run: photons, events, steps (free flights),
    fates, draws, per-sensor hits, kernel_ms."""
    return dict(_last_stats)


def validate_sim_config(config: SimConfig) -> None:
    """src/simulation.cpp:95-103."""
    if config.sample is None:
        raise ValueError("SimConfig::sample must not be null")
    if config.laser is None:
        raise ValueError("SimConfig::laser must not be null")
    if config.detector is None:
        raise ValueError("SimConfig::detector must not be null")


def _medium_desc(d: N.MediumDesc, medium, keep: list) -> None:
    ph = medium.phase_function
    if ph is None:
        raise ValueError("ScatteringMedium: Phase function is not defined!")
    if isinstance(ph, HenyeyGreensteinPhaseFunction):
        d.theta_kind = N.THETA_HG
        d.hg_g = ph.g
    elif isinstance(ph, UniformPhaseFunction):
        d.theta_kind = N.THETA_UNIFORM
    elif isinstance(ph, _TablePhase):
        d.theta_kind = N.THETA_TABLE if ph._samples_theta else N.THETA_TABLE_COS
        values, cdf = ph._table()
        keep += [values, cdf]
        d.theta_n = values.size
        d.theta_values = N.as_dptr(values)
        d.theta_cdf = N.as_dptr(cdf)
    else:
        raise NotImplementedError(f"phase function {type(ph).__name__} has no GPU sampler")
    s1 = np.ascontiguousarray(medium._s1).view(np.float64)
    s2 = np.ascontiguousarray(medium._s2).view(np.float64)
    keep += [s1, s2]
    d.amp_n = medium._s1.size
    d.amp_dtheta = medium._dtheta
    d.amp_s1 = N.as_dptr(s1)
    d.amp_s2 = N.as_dptr(s2)
    d.mu_a = medium.mu_a
    d.mu_s = medium.mu_s
    d.mean_free_path = medium.mean_free_path
    try:
        d.cross_section = float(ph.scattering_cross_section())
    except NotImplementedError:
        d.cross_section = 0.0


def _sensor_desc(d: N.SensorDesc, s) -> None:
    d.kind = s._kind
    d.z = s.origin.z
    d.absorb = int(s.absorb_photons)
    d.estimator = int(s.estimator_enabled)
    d.f_theta = int(s.filter_theta_enabled)
    d.theta_min, d.theta_max = s.filter_theta_min, s.filter_theta_max
    d.f_phi = int(s.filter_phi_enabled)
    d.phi_min, d.phi_max = s.filter_phi_min, s.filter_phi_max
    d.f_pos = int(s.filter_position_enabled)
    d.x_min, d.x_max, d.y_min, d.y_max = (s.filter_x_min, s.filter_x_max, s.filter_y_min,
                                          s.filter_y_max)
    d.f_dir = int(s.filter_direction_enabled)
    d.direction = int(s.filter_direction)
    d.f_events = int(s.filter_events_enabled)
    d.events_min, d.events_max = s.filter_events_min, s.filter_events_max
    if isinstance(s, (FarFieldCBSSensor, FarFieldFluenceSensor)):
        d.theta_max_grid, d.phi_max_grid = s.theta_max, s.phi_max
        d.dtheta, d.dphi = s.dtheta, s.dphi
        d.len_t, d.dt = s.t_max, s.dt
        if isinstance(s, FarFieldCBSSensor) and s.phi_explicit:
            if s.estimator_enabled:
                raise NotImplementedError("estimator-mode FarFieldCBSSensor with explicit phi "
                                          "slices is not supported by the GPU transport")
            d.phi_max_grid = s.N_phi * s.dphi       # the explicit slices set the column count
        if isinstance(s, FarFieldCBSSensor):
            d.theta_pp_max = s.theta_pp_max
    elif isinstance(s, PlanarFluenceSensor):
        d.len_x, d.len_y, d.len_t = s.len_x, s.len_y, s.len_t
        d.dx, d.dy, d.dt = s.dx, s.dy, s.dt
    elif isinstance(s, StatisticsSensor):
        d.len_t, d.dt = s.t_max, s.dt
        q = d.stats
        bits = {"events": N.STAT_EVENTS, "theta": N.STAT_THETA, "phi": N.STAT_PHI,
                "depth": N.STAT_DEPTH, "time": N.STAT_TIME, "weight": N.STAT_WEIGHT}
        for name, bit in bits.items():
            if getattr(s, f"{name}_histogram_bins_set"):
                q.set |= bit
        q.n_events = s.max_events
        q.n_theta, q.theta_min, q.theta_max = s.n_bins_theta, s.min_theta, s.max_theta
        q.n_phi, q.phi_min, q.phi_max = s.n_bins_phi, s.min_phi, s.max_phi
        q.n_depth, q.depth_max = s.n_bins_depth, s.max_depth
        q.n_time, q.time_max = (s._time_bins if s.time_histogram_bins_set else 0), s.h_max_time
        q.n_weight, q.weight_max = s.n_bins_weight, s.max_weight
    else:
        d.len_x, d.len_y, d.dx, d.dy = s.len_x, s.len_y, s.dx, s.dy


def scene_desc(config: SimConfig):
    """Pack the config's Sample / Laser / SensorsGroup into the C scene.
    Returns (scene, keep-alive list, gpu sensors)."""
    validate_sim_config(config)
    sample, laser, group = config.sample, config.laser, config.detector
    sc = N.SceneDesc()
    keep: list = []
    sc.n_host = sample.refractive_index
    media: list = []
    if len(sample.layers) > N.MAX_LAYERS:
        raise ValueError(f"at most {N.MAX_LAYERS} layers")
    def medium_index(m):
        idx = next((k for k, x in enumerate(media) if x is m), None)
        if idx is None:
            if len(media) == N.MAX_MEDIA:
                raise ValueError(f"at most {N.MAX_MEDIA} distinct media")
            idx = len(media)
            media.append(m)
            _medium_desc(sc.media[idx], m, keep)
        return idx

    for i, layer in enumerate(sample.layers):
        sc.layers[i].z_min = layer.z_min
        sc.layers[i].z_max = layer.z_max
        if isinstance(layer, MixtureLayer):
            if len(layer.species) > N.MAX_SPECIES:
                raise NotImplementedError(f"a MixtureLayer of at most {N.MAX_SPECIES} species")
            sc.layers[i].medium = -1
            sc.layers[i].n_species = len(layer.species)
            for k, (sp, n) in enumerate(zip(layer.species, layer.number_densities)):
                sc.layers[i].species[k] = medium_index(sp)
                sc.layers[i].number_density[k] = n
        else:
            sc.layers[i].medium = medium_index(layer.medium)
    sc.n_layers = len(sample.layers)
    sc.n_media = len(media)
    L = sc.laser
    for dst, v in ((L.position, laser.position), (L.direction, laser.direction),
                   (L.local_m, laser.local_m), (L.local_n, laser.local_n)):
        dst[0], dst[1], dst[2] = v.x, v.y, v.z
    pm, pn = laser.polarization.m, laser.polarization.n
    L.jones[0], L.jones[1], L.jones[2], L.jones[3] = pm.real, pm.imag, pn.real, pn.imag
    L.wavelength = laser.wavelength
    L.sigma = laser.sigma
    L.source = int(laser.source_type)
    L.temporal = int(laser.temporal_profile)
    L.pulse_duration = laser.pulse_duration
    L.repetition_rate = laser.repetition_rate
    L.time_offset = laser.time_offset
    sensors = list(group.detectors)
    for s in sensors:
        if not s._gpu:
            raise NotImplementedError(f"{type(s).__name__} is not supported by the GPU transport")
    if len(sensors) > N.MAX_SENSORS:
        raise ValueError(f"at most {N.MAX_SENSORS} sensors")
    for i, s in enumerate(sensors):
        _sensor_desc(sc.sensors[i], s)
    sc.n_sensors = len(sensors)
    a = config.absorption
    if a is not None:
        A = sc.absorption
        A.enabled = 1
        A.radius, A.depth, A.d_r, A.d_z = a.radius, a.depth, a.d_r, a.d_z
        A.d_t, A.t_max = a.d_t, a.t_max
    return sc, keep, sensors


def layout_shape(count, dims) -> tuple:
    """Array shape of a tally-layout entry: the 4 dims, or a flat run of counts for a
    StatisticsSensor (dims {N_t, count, 0, 0})."""
    d = tuple(dims)
    return (int(getattr(count, "value", count)),) if d[2] == 0 and d[3] == 0 else d


class Transport:
    """A created scene (lmc_create) that can run many photon ranges.

    ``run_simulation_parallel`` uses one per call; benchmarks and tests keep one
    to run repeatedly (tallies stay on the device between ``run_device`` calls).
    """

    def __init__(self, config: SimConfig, desc=None):
        self.config = config
        self.scene, self._keep, self.sensors = scene_desc(config) if desc is None else desc
        h = C.c_void_p()
        N.check(N.lib().lmc_create(C.byref(self.scene), C.byref(h)))
        self._h = h
        total = C.c_size_t()
        N.check(N.lib().lmc_tally_layout(self._h, -1, None, C.byref(total), None))
        self.tally_size = int(total.value)
        self.layout = []
        for i in range(len(self.sensors)):
            off, cnt = C.c_size_t(), C.c_size_t()
            dims = (C.c_int * 4)()
            N.check(N.lib().lmc_tally_layout(self._h, i, C.byref(off), C.byref(cnt), dims))
            self.layout.append((int(off.value), int(cnt.value), layout_shape(cnt, dims)))
        off, cnt = C.c_size_t(), C.c_size_t()
        dims = (C.c_int * 4)()
        N.check(N.lib().lmc_tally_layout(self._h, N.TALLY_ABSORPTION, C.byref(off), C.byref(cnt),
                                         dims))
        # Absorption grid (offset, count, (n_t, n_r, n_z)) or None
        self.absorption_layout = ((int(off.value), int(cnt.value), tuple(dims[:3]))
                                  if cnt.value else None)

    def close(self):
        if getattr(self, "_h", None):
            N.lib().lmc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def opts(self, precision="fp32", max_events=None, track_reverse_paths=None, block_size=0,
             blocks_per_sm=0, records_ptr=None, stream=None, batch_photons=0,
             stream_format=0, host_tallies_zero=False, cbs_phase="fp64",
             stage_tables=False, no_replay=False, tally_mode="default") -> N.RunOpts:
        if precision not in N.PRECISION:
            raise ValueError("precision must be 'fp32' or 'fp64'")
        c = self.config
        o = N.RunOpts()
        o.precision = N.PRECISION[precision]
        o.max_events = int(c.MAX_EVENTS if max_events is None else max_events)
        o.track_reverse_paths = int(bool(c.track_reverse_paths if track_reverse_paths is None
                                         else track_reverse_paths))
        o.block_size = int(block_size)
        o.blocks_per_sm = int(blocks_per_sm)
        o.records = records_ptr
        o.stream = N.launch_stream(stream)
        o.batch_photons = int(batch_photons)
        o.stream_format = int(stream_format)
        o.host_tallies_zero = int(bool(host_tallies_zero))
        if cbs_phase not in ("fp64", "fp32"):
            raise ValueError("cbs_phase must be 'fp64' or 'fp32'")
        o.cbs_phase = 1 if cbs_phase == "fp32" else 0
        o.stage_tables = int(bool(stage_tables))
        o.no_replay = int(bool(no_replay))
        o.tally_mode = N.tally_mode_value(tally_mode)
        return o

    def run_host(self, tallies: np.ndarray, n_photons: int, seed: int, begin: int = 0,
                 **kw) -> dict:
        """lmc_run_host: tallies is a float64 host array of tally_size, accumulated."""
        assert tallies.dtype == np.float64 and tallies.size == self.tally_size
        st = N.Stats()
        o = self.opts(**kw)
        N.check(N.lib().lmc_run_host(self._h, int(seed) & (2 ** 64 - 1), int(begin),
                                     int(n_photons), C.byref(o), N.as_dptr(tallies),
                                     C.byref(st)))
        return st.as_dict()

    def run_device(self, d_tallies_ptr: int, n_photons: int, seed: int, begin: int = 0,
                   want_stats: bool = True, **kw) -> dict:
        """lmc_run on a caller-owned device buffer (e.g. a torch tensor's data_ptr())."""
        st = N.Stats()
        o = self.opts(**kw)
        N.check(N.lib().lmc_run(self._h, int(seed) & (2 ** 64 - 1), int(begin), int(n_photons),
                                C.byref(o), C.c_void_p(d_tallies_ptr),
                                C.byref(st) if want_stats else None))
        return st.as_dict() if want_stats else {}

    def autotune(self, seed: int, precision: str = "fp32", sample_photons: int = 4_000_000,
                 **kw) -> dict:
        """Launch shape (block_size, blocks_per_sm, batch_photons) and tally_mode that ran
        a sample of this scene fastest (lmc_autotune); pass them to run_device / run_host."""
        r = N.TuneResult()
        N.check(N.lib().lmc_autotune(self._h, int(seed) & (2 ** 64 - 1),
                                     C.byref(self.opts(precision=precision, **kw)),
                                     int(sample_photons), C.byref(r)))
        return r.as_dict()

    def split(self, tallies: np.ndarray):
        """Per-sensor views of a flat tally buffer, in the sensor layouts."""
        return [tallies[o:o + c].reshape(d) for (o, c, d) in self.layout]

    def absorption_grid(self, tallies: np.ndarray):
        """The Absorption grid [n_t][n_r][n_z] inside a flat tally buffer (or None)."""
        if self.absorption_layout is None:
            return None
        o, c, d = self.absorption_layout
        return tallies[o:o + c].reshape(d)


def run_simulation_parallel(config: SimConfig, *, precision: str = "fp32", block_size: int = 0,
                            blocks_per_sm: int = 0) -> None:
    """GPU drop-in for luminis_mc.run_simulation_parallel(config).

    Photon i draws the Philox stream (config.seed, i), so results do not depend
    on the launch shape (as the reference's do not depend on n_threads).
    ``n_threads``, ``batch_size``, ``pin_threads_to_cores`` and ``show_progress``
    are accepted and ignored.
    """
    global _last_stats
    validate_sim_config(config)
    desc = scene_desc(config)
    with _cache_lock:
        t = _cached_transport(config, desc)
        flat = np.empty(t.tally_size)       # overwritten: the device tallies start at zero
        stats = t.run_host(flat, int(config.n_photons), int(config.seed), 0,
                           precision=precision, block_size=block_size,
                           blocks_per_sm=blocks_per_sm, host_tallies_zero=True,
                           max_events=int(config.MAX_EVENTS),
                           track_reverse_paths=bool(config.track_reverse_paths))
    for i, (s, (off, cnt, _)) in enumerate(zip(desc[2], t.layout)):
        s._tally += flat[off:off + cnt]
        s.hits += stats["hits"][i]
    if config.absorption is not None:                     # src/simulation.cpp:237-242
        config.absorption._add(t.absorption_grid(flat))
    _last_stats = stats


# One created scene is kept between run_simulation_parallel calls: a call whose scene
# (every parameter and table) equals the previous call's reuses its device tables, hit
# queue and tally buffer instead of allocating and freeing them again.  It holds that
# device memory until a call with another scene, release_gpu_cache() or exit.
_cache_lock = threading.Lock()
_cache: list = []                    # [digest, Transport] of the last scene


def _scene_digest(desc) -> bytes:
    sc, keep, _ = desc
    h = hashlib.blake2b(bytes(sc), digest_size=32)
    for a in keep:
        if isinstance(a, np.ndarray):
            h.update(np.ascontiguousarray(a).view(np.uint8).tobytes())
    return h.digest()


def _cached_transport(config: SimConfig, desc) -> "Transport":
    digest = _scene_digest(desc)
    if _cache and _cache[0] == digest:
        return _cache[1]
    release_gpu_cache()
    t = Transport(config, desc)
    _cache[:] = [digest, t]
    return t


def release_gpu_cache() -> None:
    """Free the device memory run_simulation_parallel keeps for its last scene."""
    if _cache:
        _cache[1].close()
        _cache.clear()


atexit.register(release_gpu_cache)


# --------------------------------------------------------------------- post-processing
class StokesMatrixProcessed:
    def __init__(self, S0, S1, S2, S3):
        self.S0, self.S1, self.S2, self.S3 = S0, S1, S2, S3


class FarFieldCBSProcessed:
    def __init__(self, dOmega, coherent, incoherent):
        self.dOmega, self.coherent, self.incoherent = dOmega, coherent, incoherent


class PlanarFluenceProcessed:
    def __init__(self, S0, S1, S2, S3):
        self.S0, self.S1, self.S2, self.S3 = S0, S1, S2, S3


class PlanarFieldProcessed:
    def __init__(self, Ex, Ey):
        self.Ex, self.Ey = Ex, Ey


def postprocess_farfield_cbs(det, n_photons, normalize_per_solid_angle=True,
                             normalize_per_photon=True, eps=1e-30) -> FarFieldCBSProcessed:
    """Divide by N and by the theta band's solid angle (src/results.cpp:61-101)."""
    a = det._tally.reshape(det._shape())
    invN = 1.0 / float(n_photons) if (normalize_per_photon and n_photons > 0) else 1.0
    dOm = np.array([solid_angle_bin(i, det.dtheta, det.dphi) if normalize_per_solid_angle else 1.0
                    for i in range(det.N_theta)])
    invOm = np.where(dOm > eps, 1.0 / np.where(dOm > eps, dOm, 1.0), 0.0)
    norm = (invN * invOm)[:, None]
    dOmega = np.repeat(dOm[:, None], det.N_phi, axis=1).view(Matrix)
    coh, inc = [], []
    for t in range(det.N_t):
        coh.append(StokesMatrixProcessed(*[(a[q, t] * norm).view(Matrix) for q in range(4)]))
        inc.append(StokesMatrixProcessed(*[(a[4 + q, t] * norm).view(Matrix) for q in range(4)]))
    return FarFieldCBSProcessed(dOmega, coh, inc)


def postprocess_farfield_fluence(det, n_photons, normalize_per_solid_angle=True,
                                 normalize_per_photon=True, eps=1e-30) -> list:
    """Per time bin StokesMatrixProcessed, normalised like postprocess_farfield_cbs."""
    a = det._tally.reshape(det._shape())
    invN = 1.0 / float(n_photons) if (normalize_per_photon and n_photons > 0) else 1.0
    dOm = np.array([solid_angle_bin(i, det.dtheta, det.dphi) if normalize_per_solid_angle else 1.0
                    for i in range(det.N_theta)])
    invOm = np.where(dOm > eps, 1.0 / np.where(dOm > eps, dOm, 1.0), 0.0)
    norm = (invN * invOm)[:, None]
    return [StokesMatrixProcessed(*[(a[q, t] * norm).view(Matrix) for q in range(4)])
            for t in range(det.N_t)]


def postprocess_planar_fluence(det, n_photons, normalize_per_photon=True, normalize_per_area=True,
                               eps=1e-30) -> PlanarFluenceProcessed:
    """src/results.cpp:5-35."""
    a = det._tally.reshape(det._shape())
    invN = 1.0 / float(n_photons) if (normalize_per_photon and n_photons > 0) else 1.0
    area = det.dx * det.dy
    norm = invN * ((1.0 / area) if (normalize_per_area and area > eps) else 1.0)
    return PlanarFluenceProcessed(*[[(a[q, t] * norm).view(Matrix) for t in range(det.N_t)]
                                    for q in range(4)])


def postprocess_planar_field(det, n_photons, normalize_per_photon=True, normalize_per_area=True,
                             eps=1e-30) -> PlanarFieldProcessed:
    """src/results.cpp:37-58."""
    invN = 1.0 / float(n_photons) if (normalize_per_photon and n_photons > 0) else 1.0
    area = det.dx * det.dy
    norm = invN * ((1.0 / area) if (normalize_per_area and area > eps) else 1.0)
    return PlanarFieldProcessed(np.asarray(det.Ex) * norm, np.asarray(det.Ey) * norm)
