"""ctypes view of the C ABI in include/luminis_b200.h (libluminis_b200.so).

The library is built in-tree by ``luminis-mc_b200/build.py``.  There is no
fallback: if the library is missing, every entry point that needs it raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# LUMINIS_B200_LIB names another build of the library, e.g. the bounds-checked
# lib/libluminis_b200_checked.so (luminis-mc_b200/build.py --bounds-check)
LIB_PATH = os.environ.get("LUMINIS_B200_LIB") or os.path.join(HERE, "lib", "libluminis_b200.so")
CHECKED_LIB_PATH = os.path.join(HERE, "lib", "libluminis_b200_checked.so")

MAX_LAYERS, MAX_MEDIA, MAX_SENSORS = 16, 16, 8
MAX_SPECIES, MAX_MIX_ENTRIES = 8, 32

LMC_OK, LMC_ERR_INVALID, LMC_ERR_CUDA, LMC_ERR_NOMEM, LMC_ERR_KERNEL, LMC_ERR_UNSUPPORTED = range(6)
THETA_TABLE, THETA_TABLE_COS, THETA_HG, THETA_UNIFORM = range(4)
(SENSOR_FARFIELD_CBS, SENSOR_PLANAR_FLUENCE, SENSOR_PLANAR_FIELD, SENSOR_FARFIELD_FLUENCE,
 SENSOR_STATISTICS) = range(5)
STAT_EVENTS, STAT_THETA, STAT_PHI, STAT_DEPTH, STAT_TIME, STAT_WEIGHT = 1, 2, 4, 8, 16, 32
PDF_RAYLEIGH, PDF_RD, PDF_RDEMC, PDF_DRAINE, PDF_MIE = 1, 3, 4, 5, 6
AMP_RGD, AMP_MIE = 0, 1
PRECISION = {"fp32": 0, "fp64": 1}
# lmc_tally_mode: how the hit-queue tally kernel adds into the sensor grids
TALLY_MODES = {"default": 0, "global": 1, "warp": 2, "shared": 3}


def tally_mode_value(mode) -> int:
    """lmc_tally_mode of a name in TALLY_MODES or of its integer value."""
    if isinstance(mode, str):
        if mode not in TALLY_MODES:
            raise ValueError(f"tally_mode must be one of {sorted(TALLY_MODES)}")
        return TALLY_MODES[mode]
    if int(mode) not in TALLY_MODES.values():
        raise ValueError(f"tally_mode must be one of {sorted(TALLY_MODES)}")
    return int(mode)

dptr = C.POINTER(C.c_double)


class MediumDesc(C.Structure):
    _fields_ = [("theta_kind", C.c_int), ("hg_g", C.c_double), ("theta_n", C.c_int),
                ("theta_values", dptr), ("theta_cdf", dptr), ("amp_n", C.c_int),
                ("amp_dtheta", C.c_double), ("amp_s1", dptr), ("amp_s2", dptr),
                ("mu_a", C.c_double), ("mu_s", C.c_double), ("mean_free_path", C.c_double),
                ("cross_section", C.c_double)]


class LayerDesc(C.Structure):
    _fields_ = [("z_min", C.c_double), ("z_max", C.c_double), ("medium", C.c_int),
                ("n_species", C.c_int), ("species", C.c_int * MAX_SPECIES),
                ("number_density", C.c_double * MAX_SPECIES)]


class LaserDesc(C.Structure):
    _fields_ = [("position", C.c_double * 3), ("direction", C.c_double * 3),
                ("local_m", C.c_double * 3), ("local_n", C.c_double * 3),
                ("jones", C.c_double * 4), ("wavelength", C.c_double), ("sigma", C.c_double),
                ("source", C.c_int), ("temporal", C.c_int), ("pulse_duration", C.c_double),
                ("repetition_rate", C.c_double), ("time_offset", C.c_double)]


class StatisticsDesc(C.Structure):
    _fields_ = [("set", C.c_int), ("n_events", C.c_int),
                ("n_theta", C.c_int), ("theta_min", C.c_double), ("theta_max", C.c_double),
                ("n_phi", C.c_int), ("phi_min", C.c_double), ("phi_max", C.c_double),
                ("n_depth", C.c_int), ("depth_max", C.c_double),
                ("n_time", C.c_int), ("time_max", C.c_double),
                ("n_weight", C.c_int), ("weight_max", C.c_double)]


class SensorDesc(C.Structure):
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
                ("stats", StatisticsDesc)]


class AbsorptionDesc(C.Structure):
    _fields_ = [("enabled", C.c_int), ("radius", C.c_double), ("depth", C.c_double),
                ("d_r", C.c_double), ("d_z", C.c_double), ("d_t", C.c_double),
                ("t_max", C.c_double)]


TALLY_ABSORPTION = -2


class SceneDesc(C.Structure):
    _fields_ = [("n_host", C.c_double), ("n_media", C.c_int), ("media", MediumDesc * MAX_MEDIA),
                ("n_layers", C.c_int), ("layers", LayerDesc * MAX_LAYERS), ("laser", LaserDesc),
                ("n_sensors", C.c_int), ("sensors", SensorDesc * MAX_SENSORS),
                ("absorption", AbsorptionDesc)]


class TuneResult(C.Structure):
    _fields_ = [("block_size", C.c_int), ("blocks_per_sm", C.c_int),
                ("batch_photons", C.c_uint64), ("photons_per_s", C.c_double),
                ("sample_photons", C.c_uint64), ("n_tried", C.c_int), ("tally_mode", C.c_int)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class RunOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("max_events", C.c_int), ("track_reverse_paths", C.c_int),
                ("block_size", C.c_int), ("blocks_per_sm", C.c_int), ("records", C.c_void_p),
                ("stream", C.c_void_p), ("batch_photons", C.c_uint64),
                ("stream_format", C.c_int), ("host_tallies_zero", C.c_int),
                ("cbs_phase", C.c_int), ("stage_tables", C.c_int), ("no_replay", C.c_int),
                ("tally_mode", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("photons", C.c_uint64), ("events", C.c_uint64), ("steps", C.c_uint64),
                ("detected", C.c_uint64), ("escaped", C.c_uint64), ("stack", C.c_uint64),
                ("roulette", C.c_uint64), ("cap", C.c_uint64), ("draws", C.c_uint64),
                ("hits", C.c_uint64 * MAX_SENSORS), ("error_flags", C.c_uint32),
                ("kernel_ms", C.c_float), ("transport_ms", C.c_float),
                ("transport_launches", C.c_uint32), ("replay_launches", C.c_uint32),
                ("replayed", C.c_uint64)]

    def as_dict(self) -> dict:
        d = {n: int(getattr(self, n)) for n in
             ("photons", "events", "steps", "detected", "escaped", "stack", "roulette", "cap",
              "draws", "error_flags")}
        d["hits"] = [int(x) for x in self.hits]
        d["kernel_ms"] = float(self.kernel_ms)
        d["transport_ms"] = float(self.transport_ms)
        d["transport_launches"] = int(self.transport_launches)
        d["replay_launches"] = int(self.replay_launches)
        d["replayed"] = int(self.replayed)
        return d


class AdjointOpts(C.Structure):
    _fields_ = [("radial_sensor", C.c_int), ("radial_bins", C.c_int), ("radial_max", C.c_double)]


class PhaseParams(C.Structure):
    _fields_ = [("kind", C.c_int), ("g", C.c_double), ("a", C.c_double),
                ("wavelength", C.c_double), ("radius", C.c_double), ("n_particle", C.c_double),
                ("n_medium", C.c_double)]


class MieSpecies(C.Structure):
    _fields_ = [("wavelength", C.c_double), ("radius", C.c_double), ("n_particle", C.c_double),
                ("n_medium", C.c_double)]


# Per-photon record (same layout as lmc_record).
RECORD_FIELDS = [("photon", "<u8"), ("events", "<u4"), ("draws", "<u4"), ("fate", "<i4"),
                 ("layer", "<i4"), ("weight", "<f8"), ("opticalpath", "<f8"),
                 ("penetration_depth", "<f8"), ("launch_time", "<f8"), ("pos", "<f8", 3),
                 ("dir", "<f8", 3), ("m", "<f8", 3), ("n", "<f8", 3), ("E", "<f8", 4),
                 ("r1", "<f8", 3), ("rn", "<f8", 3), ("Er", "<f8", 4), ("hit", "<f8", 3),
                 ("n_hits", "<i4"), ("pad", "<i4")]

# Every symbol the header declares (checked by the CPU test suite).
EXPORTED = ["lmc_create", "lmc_destroy", "lmc_tally_layout", "lmc_run", "lmc_run_host",
            "lmc_last_error", "lmc_mie", "lmc_sampling_table", "lmc_phase_cross_section",
            "lmc_amplitude_table", "lmc_probe_fp32_peak", "lmc_run_noalloc",
            "lmc_adjoint_layout", "lmc_run_adjoint", "lmc_adjoint_contract",
            "lmc_create_sweep", "lmc_sweep_layout", "lmc_sweep_set_photons", "lmc_run_sweep",
            "lmc_sweep_hits", "lmc_sweep_adjoint_layout", "lmc_run_sweep_adjoint",
            "lmc_autotune", "lmc_mie_tables"]

_lib = None


def lib_path() -> str:
    return LIB_PATH


def lib():
    """Load libluminis_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python luminis-mc_b200/build.py`"
                           " (there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.lmc_create.argtypes = [C.POINTER(SceneDesc), C.POINTER(vp)]
    L.lmc_create.restype = C.c_int
    L.lmc_destroy.argtypes = [vp]
    L.lmc_destroy.restype = None
    L.lmc_tally_layout.argtypes = [vp, C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                   C.POINTER(C.c_int)]
    L.lmc_tally_layout.restype = C.c_int
    L.lmc_run.argtypes = [vp, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(RunOpts), vp,
                          C.POINTER(Stats)]
    L.lmc_run.restype = C.c_int
    L.lmc_run_host.argtypes = [vp, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(RunOpts), dptr,
                               C.POINTER(Stats)]
    L.lmc_run_host.restype = C.c_int
    L.lmc_last_error.argtypes = [C.c_char_p, C.c_size_t]
    L.lmc_last_error.restype = C.c_size_t
    L.lmc_mie.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, dptr, dptr, dptr, dptr,
                          dptr, dptr]
    L.lmc_mie.restype = C.c_int
    L.lmc_sampling_table.argtypes = [C.POINTER(PhaseParams), C.c_int, C.c_double, C.c_double,
                                     dptr, dptr]
    L.lmc_sampling_table.restype = C.c_int
    L.lmc_phase_cross_section.argtypes = [C.POINTER(PhaseParams), dptr]
    L.lmc_phase_cross_section.restype = C.c_int
    L.lmc_amplitude_table.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.c_int, dptr, dptr]
    L.lmc_amplitude_table.restype = C.c_int
    L.lmc_mie_tables.argtypes = [C.POINTER(MieSpecies), C.c_int, C.c_int, C.c_double, C.c_double,
                                 C.c_int, dptr, dptr, dptr, dptr, dptr, dptr]
    L.lmc_mie_tables.restype = C.c_int
    L.lmc_probe_fp32_peak.argtypes = [C.c_int, dptr, dptr]
    L.lmc_probe_fp32_peak.restype = C.c_int
    L.lmc_run_noalloc.argtypes = [C.POINTER(SceneDesc), C.c_uint64, C.c_uint64, C.c_uint64,
                                  C.POINTER(RunOpts), vp, C.POINTER(Stats)]
    L.lmc_run_noalloc.restype = C.c_int
    L.lmc_adjoint_layout.argtypes = [vp, C.POINTER(AdjointOpts), C.POINTER(C.c_size_t),
                                     C.POINTER(C.c_int)]
    L.lmc_adjoint_layout.restype = C.c_int
    L.lmc_run_adjoint.argtypes = [vp, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(RunOpts),
                                  C.POINTER(AdjointOpts), vp, vp, C.POINTER(Stats)]
    L.lmc_run_adjoint.restype = C.c_int
    L.lmc_adjoint_contract.argtypes = [vp, vp, C.c_size_t, C.c_int, vp, vp]
    L.lmc_adjoint_contract.restype = C.c_int
    L.lmc_create_sweep.argtypes = [C.POINTER(SceneDesc), C.c_int, C.POINTER(vp)]
    L.lmc_create_sweep.restype = C.c_int
    L.lmc_sweep_layout.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_size_t),
                                   C.POINTER(C.c_size_t), C.POINTER(C.c_int)]
    L.lmc_sweep_layout.restype = C.c_int
    L.lmc_sweep_set_photons.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.lmc_sweep_set_photons.restype = C.c_int
    L.lmc_run_sweep.argtypes = [vp, C.c_uint64, C.POINTER(RunOpts), vp, C.POINTER(Stats)]
    L.lmc_run_sweep.restype = C.c_int
    L.lmc_sweep_adjoint_layout.argtypes = [vp, C.POINTER(AdjointOpts), C.c_int,
                                           C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                           C.POINTER(C.c_int)]
    L.lmc_sweep_adjoint_layout.restype = C.c_int
    L.lmc_run_sweep_adjoint.argtypes = [vp, C.c_uint64, C.POINTER(RunOpts), C.POINTER(AdjointOpts),
                                        vp, vp, C.POINTER(Stats)]
    L.lmc_run_sweep_adjoint.restype = C.c_int
    L.lmc_autotune.argtypes = [vp, C.c_uint64, C.POINTER(RunOpts), C.c_uint64,
                               C.POINTER(TuneResult)]
    L.lmc_autotune.restype = C.c_int
    L.lmc_sweep_hits.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.lmc_sweep_hits.restype = C.c_int
    _lib = L
    return L


def probe_fp32_peak(iters: int = 200000) -> tuple[float, float]:
    """(TFLOP/s, ms) of the FP32 FMA probe kernel on the current device."""
    t = C.c_double()
    ms = C.c_double()
    check(lib().lmc_probe_fp32_peak(int(iters), C.byref(t), C.byref(ms)))
    return t.value, ms.value


# cudaStreamLegacy: the legacy default stream, on which torch's default stream runs.  In
# lmc_run_opts.stream a NULL handle selects the lmc handle's own (non-blocking) stream, which
# torch's default-stream work does not wait for.
CUDA_STREAM_LEGACY = 1


def launch_stream(stream):
    """The cudaStream_t to put in lmc_run_opts.stream for a Python caller: a stream handle
    (torch's `Stream.cuda_stream`) as given; None, or torch's default-stream handle 0, the
    legacy default stream, so that the run is ordered with torch's default-stream work."""
    return CUDA_STREAM_LEGACY if not stream else stream


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().lmc_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status: int, what: str = "") -> None:
    """Map an lmc_status to the reference's Python exception types."""
    if status == LMC_OK:
        return
    msg = last_error() or what
    if status == LMC_ERR_INVALID:
        raise ValueError(msg)
    if status == LMC_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if status == LMC_ERR_NOMEM:
        raise MemoryError(msg)
    raise RuntimeError(msg)


def as_dptr(arr):
    return arr.ctypes.data_as(dptr)
