"""ctypes binding of the C oracle (oracle/lmc_oracle.h) -- TEST INFRASTRUCTURE.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module.  It turns a scene spec (the dict format of
``luminis_mc_b200.workloads``) into the oracle's ``lmc_o_scene`` and runs the
C restatement of the reference's transport over a photon range.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblmc_oracle.so")

MAXP, MAXM, MAXL, MAXS = 16, 16, 16, 8

PHASE_KIND = {"uniform": 0, "rayleigh": 1, "hg": 2, "rd": 3, "rdemc": 4, "draine": 5, "mie": 6}
MEDIUM_KIND = {"rgd": 0, "mie": 1}
SENSOR_KIND = {"farfield_cbs": 0, "planar_fluence": 1, "planar_field": 2, "farfield_fluence": 3,
               "statistics": 4}
STAT_BITS = {"events": 1, "theta": 2, "phi": 4, "depth": 8, "time": 16, "weight": 32}
RNG = {"xoshiro": 0, "philox_u53": 1, "philox_u24": 2}
SOURCE = {"point": 0, "uniform": 1, "gaussian": 2}
TEMPORAL = {"delta": 0, "gaussian": 1, "tophat": 2, "exponential": 3, "pulsetrain": 4, "cw": 5}
DIRECTION = {"forward": 0, "backward": 1, "both": 2}
FATE = {1: "detected", 2: "escaped", 3: "stack", 4: "roulette", 5: "cap"}


class Phase(C.Structure):
    _fields_ = [("kind", C.c_int), ("g", C.c_double), ("a", C.c_double),
                ("wavelength", C.c_double), ("radius", C.c_double), ("n_particle", C.c_double),
                ("n_medium", C.c_double), ("n_div", C.c_int), ("min_val", C.c_double),
                ("max_val", C.c_double)]


class Medium(C.Structure):
    _fields_ = [("kind", C.c_int), ("phase", C.c_int), ("radius", C.c_double),
                ("n_particle", C.c_double), ("n_medium", C.c_double), ("wavelength", C.c_double),
                ("mu_a", C.c_double), ("mu_s", C.c_double), ("mfp", C.c_double)]


MAX_SPECIES = 8


class Layer(C.Structure):
    _fields_ = [("medium", C.c_int), ("z_min", C.c_double), ("z_max", C.c_double),
                ("n_species", C.c_int), ("species", C.c_int * MAX_SPECIES),
                ("number_density", C.c_double * MAX_SPECIES)]


class Laser(C.Structure):
    _fields_ = [("position", C.c_double * 3), ("direction", C.c_double * 3),
                ("local_m", C.c_double * 3), ("local_n", C.c_double * 3), ("pol", C.c_double * 4),
                ("wavelength", C.c_double), ("sigma", C.c_double), ("source", C.c_int),
                ("temporal", C.c_int), ("pulse_duration", C.c_double),
                ("repetition_rate", C.c_double), ("time_offset", C.c_double)]


class Statistics(C.Structure):
    _fields_ = [("set", C.c_int), ("n_events", C.c_int),
                ("n_theta", C.c_int), ("theta_min", C.c_double), ("theta_max", C.c_double),
                ("n_phi", C.c_int), ("phi_min", C.c_double), ("phi_max", C.c_double),
                ("n_depth", C.c_int), ("depth_max", C.c_double),
                ("n_time", C.c_int), ("time_max", C.c_double),
                ("n_weight", C.c_int), ("weight_max", C.c_double)]


class Sensor(C.Structure):
    _fields_ = [("kind", C.c_int), ("z", C.c_double), ("absorb", C.c_int), ("estimator", C.c_int),
                ("f_theta", C.c_int), ("theta_min", C.c_double), ("theta_max", C.c_double),
                ("f_phi", C.c_int), ("phi_min", C.c_double), ("phi_max", C.c_double),
                ("f_pos", C.c_int), ("x_min", C.c_double), ("x_max", C.c_double),
                ("y_min", C.c_double), ("y_max", C.c_double),
                ("f_dir", C.c_int), ("direction", C.c_int),
                ("f_events", C.c_int), ("events_min", C.c_int), ("events_max", C.c_int),
                ("len_x", C.c_double), ("len_y", C.c_double), ("len_t", C.c_double),
                ("dx", C.c_double), ("dy", C.c_double), ("dt", C.c_double),
                ("theta_max_grid", C.c_double), ("phi_max_grid", C.c_double),
                ("dtheta", C.c_double), ("dphi", C.c_double), ("theta_pp_max", C.c_double),
                ("stats", Statistics)]


class AbsorptionGrid(C.Structure):
    _fields_ = [("enabled", C.c_int), ("radius", C.c_double), ("depth", C.c_double),
                ("d_r", C.c_double), ("d_z", C.c_double), ("d_t", C.c_double),
                ("t_max", C.c_double)]


class Scene(C.Structure):
    _fields_ = [("n_host", C.c_double), ("n_phase", C.c_int), ("phase", Phase * MAXP),
                ("n_media", C.c_int), ("media", Medium * MAXM), ("n_layers", C.c_int),
                ("layers", Layer * MAXL), ("laser", Laser), ("n_sensors", C.c_int),
                ("sensors", Sensor * MAXS), ("absorption", AbsorptionGrid)]


class Record(C.Structure):
    _fields_ = [("photon", C.c_uint64), ("events", C.c_uint32), ("draws", C.c_uint32),
                ("fate", C.c_int32), ("layer", C.c_int32), ("weight", C.c_double),
                ("opticalpath", C.c_double), ("penetration_depth", C.c_double),
                ("launch_time", C.c_double), ("pos", C.c_double * 3), ("dir", C.c_double * 3),
                ("m", C.c_double * 3), ("n", C.c_double * 3), ("E", C.c_double * 4),
                ("r1", C.c_double * 3), ("rn", C.c_double * 3), ("Er", C.c_double * 4),
                ("hit", C.c_double * 3), ("n_hits", C.c_int32), ("pad", C.c_int32)]


RECORD_DTYPE = np.dtype([("photon", "<u8"), ("events", "<u4"), ("draws", "<u4"), ("fate", "<i4"),
                         ("layer", "<i4"), ("weight", "<f8"), ("opticalpath", "<f8"),
                         ("penetration_depth", "<f8"), ("launch_time", "<f8"),
                         ("pos", "<f8", 3), ("dir", "<f8", 3), ("m", "<f8", 3), ("n", "<f8", 3),
                         ("E", "<f8", 4), ("r1", "<f8", 3), ("rn", "<f8", 3), ("Er", "<f8", 4),
                         ("hit", "<f8", 3), ("n_hits", "<i4"), ("pad", "<i4")])
assert RECORD_DTYPE.itemsize == C.sizeof(Record)


class Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in
                ("photons", "events", "steps", "detected", "escaped", "stack", "roulette", "cap",
                 "draws")]


class Adjoint(C.Structure):
    _fields_ = [("radial_sensor", C.c_int), ("radial_bins", C.c_int), ("radial_max", C.c_double)]


ADJ_PARAMS = ("mu_a", "mu_s", "mfp", "g")      # per medium, in this order


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run `make -C oracle restatement`)")
        L = C.CDLL(LIB_PATH)
        L.lmc_oracle_create.restype = C.c_void_p
        L.lmc_oracle_create.argtypes = [C.POINTER(Scene), C.c_char_p, C.c_int]
        L.lmc_oracle_destroy.argtypes = [C.c_void_p]
        L.lmc_oracle_sensor_shape.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                              C.POINTER(C.c_size_t)]
        L.lmc_oracle_run.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_int,
                                     C.c_int, C.c_int, C.POINTER(C.POINTER(C.c_double)),
                                     C.POINTER(C.c_uint64), C.c_void_p, C.POINTER(Stats)]
        L.lmc_oracle_adjoint_outputs.restype = C.c_size_t
        L.lmc_oracle_adjoint_outputs.argtypes = [C.c_void_p, C.POINTER(Adjoint)]
        L.lmc_oracle_run_adjoint.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64,
                                             C.c_int, C.c_int, C.c_int,
                                             C.POINTER(C.POINTER(C.c_double)),
                                             C.POINTER(C.c_uint64), C.POINTER(Adjoint),
                                             C.POINTER(C.c_double), C.POINTER(Stats)]
        L.lmc_oracle_phase_table.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                             C.POINTER(C.POINTER(C.c_double)),
                                             C.POINTER(C.POINTER(C.c_double))]
        L.lmc_oracle_amp_table.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                           C.POINTER(C.c_double),
                                           C.POINTER(C.POINTER(C.c_double)),
                                           C.POINTER(C.POINTER(C.c_double))]
        L.lmc_oracle_phase_sample_theta.restype = C.c_double
        L.lmc_oracle_phase_sample_theta.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.lmc_oracle_philox.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                        C.POINTER(C.c_uint32)]
        L.lmc_oracle_stream_uniform.restype = C.c_double
        L.lmc_oracle_stream_uniform.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_int]
        L.lmc_oracle_miev0_selftest.argtypes = [C.POINTER(C.c_double)]
        L.lmc_oracle_mie.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int,
                                     C.POINTER(C.c_double), C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _lib = L
    return _lib


def _vec(dst, v):
    for i, x in enumerate(v):
        dst[i] = float(x)


def scene_from_spec(spec: dict) -> Scene:
    """Translate a workload spec dict into the oracle's POD scene."""
    sc = Scene()
    sc.n_host = float(spec.get("n_host", 1.0))
    phases = spec["phases"]
    sc.n_phase = len(phases)
    for i, p in enumerate(phases):
        q = sc.phase[i]
        q.kind = PHASE_KIND[p["kind"]]
        q.g = float(p.get("g", 0.0))
        q.a = float(p.get("a", 0.0))
        q.wavelength = float(p.get("wavelength", 0.0))
        q.radius = float(p.get("radius", 0.0))
        q.n_particle = float(p.get("n_particle", 0.0))
        q.n_medium = float(p.get("n_medium", 1.0))
        q.n_div = int(p.get("nDiv", 0))
        q.min_val = float(p.get("min", 0.0))
        q.max_val = float(p.get("max", 0.0))
    media = spec["media"]
    sc.n_media = len(media)
    for i, m in enumerate(media):
        q = sc.media[i]
        q.kind = MEDIUM_KIND[m["kind"]]
        q.phase = int(m["phase"])
        q.radius = float(m["radius"])
        q.n_particle = float(m["n_particle"])
        q.n_medium = float(m["n_medium"])
        q.wavelength = float(m["wavelength"])
        q.mu_a = float(m["mu_a"])
        q.mu_s = float(m["mu_s"])
        q.mfp = float(m["mfp"])
    layers = spec["layers"]
    sc.n_layers = len(layers)
    for i, l in enumerate(layers):
        sc.layers[i].z_min = float(l["z_min"])
        sc.layers[i].z_max = float(l["z_max"])
        if "species" in l:                      # MixtureLayer
            sc.layers[i].medium = -1
            sc.layers[i].n_species = len(l["species"])
            for k, (m, n) in enumerate(zip(l["species"], l["densities"])):
                sc.layers[i].species[k] = int(m)
                sc.layers[i].number_density[k] = float(n)
        else:
            sc.layers[i].medium = int(l["medium"])
    L = spec["laser"]
    _vec(sc.laser.position, L.get("position", (0.0, 0.0, 1e-9)))
    _vec(sc.laser.direction, L.get("direction", (0.0, 0.0, 1.0)))
    _vec(sc.laser.local_m, L.get("local_m", (1.0, 0.0, 0.0)))
    _vec(sc.laser.local_n, L.get("local_n", (0.0, 1.0, 0.0)))
    m_state, n_state = complex(L["m"]), complex(L["n"])
    _vec(sc.laser.pol, (m_state.real, m_state.imag, n_state.real, n_state.imag))
    sc.laser.wavelength = float(L["wavelength"])
    sc.laser.sigma = float(L.get("sigma", 0.0))
    sc.laser.source = SOURCE[L.get("source", "point")]
    sc.laser.temporal = TEMPORAL[L.get("temporal", "delta")]
    sc.laser.pulse_duration = float(L.get("pulse_duration", 0.0))
    sc.laser.repetition_rate = float(L.get("repetition_rate", 0.0))
    sc.laser.time_offset = float(L.get("time_offset", 0.0))
    sensors = spec["sensors"]
    sc.n_sensors = len(sensors)
    for i, s in enumerate(sensors):
        q = sc.sensors[i]
        kind = s["kind"]
        q.kind = SENSOR_KIND[kind]
        q.estimator = int(bool(s.get("estimator", False)))
        if kind in ("farfield_cbs", "farfield_fluence"):
            q.z, q.absorb = 0.0, 1
            q.theta_max_grid = float(s["theta_max"])
            q.phi_max_grid = float(s["phi_max"])
            q.len_t = float(s.get("len_t", 0.0))
            q.dtheta = float(s["d_theta"])
            q.dphi = float(s["d_phi"])
            q.theta_pp_max = float(s.get("theta_pp_max", 0.0))
            q.dt = float(s.get("d_t", 0.0))
        elif kind == "statistics":
            q.z = float(s["z"])
            q.absorb = int(bool(s.get("absorb", False)))
            q.len_t, q.dt = float(s.get("len_t", 0.0)), float(s.get("d_t", 0.0))
            st = q.stats
            for key, bit in STAT_BITS.items():
                if key in s:
                    st.set |= bit
            if "events" in s:
                st.n_events = int(s["events"])
            if "theta" in s:
                lo, hi, nb = s["theta"]
                st.theta_min, st.theta_max, st.n_theta = float(lo), float(hi), int(nb)
            if "phi" in s:
                lo, hi, nb = s["phi"]
                st.phi_min, st.phi_max, st.n_phi = float(lo), float(hi), int(nb)
            if "depth" in s:
                st.depth_max, st.n_depth = float(s["depth"][0]), int(s["depth"][1])
            if "time" in s:
                st.time_max, st.n_time = float(s["time"][0]), int(s["time"][1])
            if "weight" in s:
                st.weight_max, st.n_weight = float(s["weight"][0]), int(s["weight"][1])
        else:
            q.z = float(s["z"])
            q.absorb = int(bool(s.get("absorb", True)))
            q.len_x, q.len_y = float(s["len_x"]), float(s["len_y"])
            q.dx, q.dy = float(s["dx"]), float(s["dy"])
            if kind == "planar_fluence":
                q.len_t, q.dt = float(s.get("len_t", 0.0)), float(s.get("d_t", 0.0))
            q.f_pos = 1
            q.x_min, q.x_max = -0.5 * q.len_x, 0.5 * q.len_x
            q.y_min, q.y_max = -0.5 * q.len_y, 0.5 * q.len_y
        if "theta_limit" in s:
            q.f_theta = 1
            q.theta_min, q.theta_max = map(float, s["theta_limit"])
        if "phi_limit" in s:
            q.f_phi = 1
            q.phi_min, q.phi_max = map(float, s["phi_limit"])
        if "position_limit" in s:
            q.f_pos = 1
            q.x_min, q.x_max, q.y_min, q.y_max = map(float, s["position_limit"])
        if "direction_limit" in s:
            q.f_dir = 1
            q.direction = DIRECTION[s["direction_limit"]]
        if "events_limit" in s:
            q.f_events = 1
            q.events_min, q.events_max = map(int, s["events_limit"])
    a = spec.get("absorption")
    if a is not None:
        sc.absorption.enabled = 1
        sc.absorption.radius, sc.absorption.depth = float(a["radius"]), float(a["depth"])
        sc.absorption.d_r, sc.absorption.d_z = float(a["d_r"]), float(a["d_z"])
        sc.absorption.d_t, sc.absorption.t_max = float(a.get("d_t", 0.0)), float(a.get("t_max", 0.0))
    return sc


@dataclass
class OracleResult:
    tallies: list          # one float64 ndarray per sensor, shaped per the layout
    hits: np.ndarray
    records: np.ndarray | None
    stats: dict
    absorption: np.ndarray | None = None   # [n_t][n_r][n_z] deposited weight


class Oracle:
    """One oracle scene (tables built from the spec's physical parameters)."""

    def __init__(self, spec: dict):
        self.spec = spec
        self._scene = scene_from_spec(spec)
        err = C.create_string_buffer(512)
        self._h = lib().lmc_oracle_create(C.byref(self._scene), err, 512)
        if not self._h:
            raise ValueError(f"oracle rejected the scene: {err.value.decode()}")
        self.shapes = []
        for s in range(self._scene.n_sensors):
            dims = (C.c_int * 4)()
            n = C.c_size_t()
            lib().lmc_oracle_sensor_shape(self._h, s, dims, C.byref(n))
            if self._scene.sensors[s].kind == SENSOR_KIND["statistics"]:
                self.shapes.append((int(n.value),))     # histograms one after another
            else:
                self.shapes.append(tuple(dims))
        self.absorption_shape = None
        if self._scene.absorption.enabled:
            dims = (C.c_int * 4)()
            n = C.c_size_t()
            lib().lmc_oracle_sensor_shape(self._h, self._scene.n_sensors, dims, C.byref(n))
            self.absorption_shape = tuple(dims[:3])

    def _buffers(self):
        """Zeroed tallies, the pointer array the C side fills (the Absorption grid
        after the sensors) and the grid (or None)."""
        tallies = [np.zeros(int(np.prod(s)), dtype=np.float64) for s in self.shapes]
        grid = (np.zeros(self.absorption_shape, dtype=np.float64)
                if self.absorption_shape is not None else None)
        ptrs = (C.POINTER(C.c_double) * (len(tallies) + 1))()
        for i, t in enumerate(tallies):
            ptrs[i] = t.ctypes.data_as(C.POINTER(C.c_double))
        if grid is not None:
            ptrs[len(tallies)] = grid.ctypes.data_as(C.POINTER(C.c_double))
        return tallies, ptrs, grid

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().lmc_oracle_destroy(h)
            self._h = None

    def run(self, n_photons: int, seed: int, begin: int = 0, rng: str = "philox_u53",
            max_events: int | None = None, track_reverse: bool | None = None,
            records: bool = False) -> OracleResult:
        max_events = int(self.spec.get("max_events", 1000) if max_events is None else max_events)
        if track_reverse is None:
            track_reverse = bool(self.spec.get("track_reverse_paths", True))
        tallies, ptrs, grid = self._buffers()
        hits = np.zeros(max(1, len(tallies)), dtype=np.uint64)
        rec = np.zeros(n_photons, dtype=RECORD_DTYPE) if records else None
        st = Stats()
        rc = lib().lmc_oracle_run(self._h, seed, begin, n_photons, RNG[rng], max_events,
                                  int(bool(track_reverse)), ptrs,
                                  hits.ctypes.data_as(C.POINTER(C.c_uint64)),
                                  rec.ctypes.data if rec is not None else None, C.byref(st))
        if rc != 0:
            raise ValueError(f"oracle run failed ({rc}): launch position outside the sample")
        stats = {n: int(getattr(st, n)) for n, _ in Stats._fields_}
        return OracleResult([t.reshape(s) for t, s in zip(tallies, self.shapes)],
                            hits[: len(tallies)], rec, stats, grid)

    def run_adjoint(self, n_photons: int, seed: int, radial_sensor: int = -1,
                    radial_bins: int = 100, radial_max: float = 5.0, begin: int = 0,
                    rng: str = "philox_u53", max_events: int | None = None,
                    track_reverse: bool | None = None):
        """Tallies plus the likelihood-ratio outputs: returns (OracleResult, out) with
        out[0] the outputs (radial total + profile, then S0 coherent / incoherent of
        each FarFieldCBS sensor) and out[1 + 4 m + j] their derivative with respect
        to parameter j = (mu_a, mu_s, mfp, g) of medium m."""
        max_events = int(self.spec.get("max_events", 1000) if max_events is None else max_events)
        if track_reverse is None:
            track_reverse = bool(self.spec.get("track_reverse_paths", True))
        a = Adjoint(radial_sensor, radial_bins, radial_max)
        n_out = lib().lmc_oracle_adjoint_outputs(self._h, C.byref(a))
        if n_out == 0:
            raise ValueError("no adjoint outputs (radial sensor must be a PlanarFluenceSensor)")
        K = 4 * self._scene.n_media
        out = np.zeros((1 + K, n_out), dtype=np.float64)
        tallies, ptrs, grid = self._buffers()
        hits = np.zeros(max(1, len(tallies)), dtype=np.uint64)
        st = Stats()
        rc = lib().lmc_oracle_run_adjoint(self._h, seed, begin, n_photons, RNG[rng], max_events,
                                          int(bool(track_reverse)), ptrs,
                                          hits.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(a),
                                          out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(st))
        if rc != 0:
            raise ValueError(f"oracle adjoint run failed ({rc})")
        stats = {n: int(getattr(st, n)) for n, _ in Stats._fields_}
        return OracleResult([t.reshape(s) for t, s in zip(tallies, self.shapes)],
                            hits[: len(tallies)], None, stats, grid), out

    def phase_table(self, medium: int):
        n = C.c_int()
        v = C.POINTER(C.c_double)()
        c = C.POINTER(C.c_double)()
        lib().lmc_oracle_phase_table(self._h, medium, C.byref(n), C.byref(v), C.byref(c))
        if n.value == 0:
            return None, None
        return (np.ctypeslib.as_array(v, (n.value,)).copy(),
                np.ctypeslib.as_array(c, (n.value,)).copy())

    def amp_table(self, medium: int):
        n = C.c_int()
        d = C.c_double()
        s1 = C.POINTER(C.c_double)()
        s2 = C.POINTER(C.c_double)()
        lib().lmc_oracle_amp_table(self._h, medium, C.byref(n), C.byref(d), C.byref(s1),
                                   C.byref(s2))
        a = np.ctypeslib.as_array(s1, (2 * n.value,)).copy().view(np.complex128)
        b = np.ctypeslib.as_array(s2, (2 * n.value,)).copy().view(np.complex128)
        return d.value, a, b

    def sample_theta(self, medium: int, u: float) -> float:
        return lib().lmc_oracle_phase_sample_theta(self._h, medium, float(u))


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().lmc_oracle_philox(c, k, o)
    return tuple(o)


def stream_uniform(seed: int, photon: int, draw: int, fmt: str = "u53") -> float:
    return lib().lmc_oracle_stream_uniform(seed, photon, draw, 0 if fmt == "u53" else 1)


def miev0_selftest() -> tuple[bool, float]:
    w = C.c_double()
    ok = lib().lmc_oracle_miev0_selftest(C.byref(w))
    return bool(ok), w.value


def mie(x: float, m: complex, mu: np.ndarray):
    """S1, S2 (complex arrays) and (qext, qsca, g) from the MIEV0 restatement."""
    mu = np.ascontiguousarray(mu, dtype=np.float64)
    n = mu.size
    s1 = np.zeros(2 * max(n, 1))
    s2 = np.zeros(2 * max(n, 1))
    qe, qs, g = C.c_double(), C.c_double(), C.c_double()
    dp = C.POINTER(C.c_double)
    lib().lmc_oracle_mie(float(x), float(m.real), float(m.imag), n, mu.ctypes.data_as(dp),
                         s1.ctypes.data_as(dp), s2.ctypes.data_as(dp), C.byref(qe), C.byref(qs),
                         C.byref(g))
    return (s1[: 2 * n].view(np.complex128), s2[: 2 * n].view(np.complex128),
            (qe.value, qs.value, g.value))


def reference_module(flavour: str = "pin"):
    """Import the reference's own pybind module built by oracle/Makefile
    (oracle/_ref/<flavour>/luminis_mc), or raise if it was not built."""
    import importlib
    import sys
    root = os.path.join(HERE, "_ref", flavour)
    if not os.path.isdir(os.path.join(root, "luminis_mc")):
        raise ImportError(f"reference flavour {flavour!r} not built under {root}")
    # the three flavours share a module name: only one may be imported per process
    loaded = sys.modules.get("luminis_mc")
    if loaded is not None:
        if os.path.dirname(os.path.dirname(loaded.__file__)) != root:
            raise ImportError("another reference flavour is already imported in this process")
        return loaded
    sys.path.insert(0, root)
    try:
        return importlib.import_module("luminis_mc")
    finally:
        sys.path.remove(root)


def unit_cbs_eta(t):
    """Enhancement factor S0_coh/S0_incoh of a FarFieldCBS tally (bin 0)."""
    with np.errstate(invalid="ignore", divide="ignore"):
        return t[0, 0] / t[4, 0]


__all__ = ["Oracle", "OracleResult", "scene_from_spec", "miev0_selftest", "mie",
           "reference_module", "RECORD_DTYPE", "FATE", "math"]
