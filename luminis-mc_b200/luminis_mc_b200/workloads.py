"""Named workloads of the photon-propagation path, as plain scene specs.

A spec is a dict of the physical parameters the luminis-mc constructors take
(units: mm).  ``build(lm, spec)`` constructs the scene through any module that
exposes the luminis-mc Python API -- this package, or the reference's own
``luminis_mc`` -- so the same workload runs on both.

Workloads (synthetic media; no dataset is involved):
  * ``mie_cbs_small``      semi-infinite polystyrene-sphere Mie medium (r=0.5 um,
                           n 1.59/1.33, lambda 0.633 um), mu_s=10/mm, mu_a=0.01/mm,
                           linear pencil beam, one FarFieldCBSSensor 100 x 1.
  * ``bilayer_rgd_mie``    0.5 mm RGD layer (r=0.1 um, mu_s=20, mu_a=0.05) over the
                           Mie medium above, circular polarisation, FarFieldCBS
                           200 x 8, PlanarFluence 200 x 200 x 64 time bins over
                           10 x 10 mm, FarFieldFluence 90 x 36.
  * ``bilayer_hg``         the bilayer geometry with Henyey-Greenstein theta
                           sampling (g=0.8 top, 0.9 bottom).
  * ``mie_long_paths``     Mie r=1.0 um, mu_s=100/mm, mu_a=1e-4/mm, MAX_EVENTS
                           raised to 1e6, FarFieldCBS 400 bins to 0.02 rad and a
                           256 x 256 PlanarFieldSensor.
  * ``mixture_bilayer``    a three-species MixtureLayer slab over the Mie medium.
  * ``mixture_cbs_small``  a semi-infinite two-species MixtureLayer.
  * ``mie_sweep(i)``       one of 256 single-layer Mie media with seeded random
                           radius / mu_s / mu_a / photon count.
"""
from __future__ import annotations

import math

import numpy as np

LAMBDA = 0.633e-3          # mm
N_SPHERE = 1.59
N_WATER = 1.33
PI = math.pi


def _mie_phase(radius, n_div=1000):
    return {"kind": "mie", "wavelength": LAMBDA, "radius": radius, "n_particle": N_SPHERE,
            "n_medium": N_WATER, "nDiv": n_div, "min": 0.0, "max": PI}


def _medium(kind, phase, radius, mu_s, mu_a, mfp=None):
    return {"kind": kind, "phase": phase, "radius": radius, "n_particle": N_SPHERE,
            "n_medium": N_WATER, "wavelength": LAMBDA, "mu_s": mu_s, "mu_a": mu_a,
            "mfp": (1.0 / mu_s) if mfp is None else mfp}


def _laser(m, n):
    return {"m": m, "n": n, "wavelength": LAMBDA, "sigma": 0.0, "source": "point"}


LINEAR = (1.0 + 0j, 0j)
CIRCULAR = (1.0 / math.sqrt(2.0) + 0j, 1j / math.sqrt(2.0))


def mie_cbs_small(n_photons=1_000_000, seed=12345):
    """Single semi-infinite Mie layer with one far-field CBS detector."""
    return {
        "name": "mie_cbs_small", "n_host": N_WATER,
        "phases": [_mie_phase(0.5e-3)],
        "media": [_medium("mie", 0, 0.5e-3, 10.0, 0.01, 0.1)],
        "layers": [{"medium": 0, "z_min": 0.0, "z_max": math.inf}],
        "laser": _laser(*LINEAR),
        "sensors": [{"kind": "farfield_cbs", "theta_max": 0.1, "phi_max": 2 * PI, "len_t": 0.0,
                     "d_theta": 1e-3, "d_phi": 2 * PI, "d_t": 0.0, "theta_limit": (0.0, 0.1)}],
        "n_photons": n_photons, "seed": seed, "max_events": 1000, "track_reverse_paths": True,
    }


def bilayer_rgd_mie(n_photons=100_000_000, seed=12345):
    """RGD top slab over a semi-infinite Mie medium, three detectors at z=0."""
    return {
        "name": "bilayer_rgd_mie", "n_host": N_WATER,
        "phases": [{"kind": "rdemc", "wavelength": LAMBDA, "radius": 0.1e-3,
                    "n_particle": N_SPHERE, "n_medium": N_WATER, "nDiv": 1000,
                    "min": 0.0, "max": PI},
                   _mie_phase(0.5e-3)],
        "media": [_medium("rgd", 0, 0.1e-3, 20.0, 0.05, 0.05),
                  _medium("mie", 1, 0.5e-3, 10.0, 0.01, 0.1)],
        "layers": [{"medium": 0, "z_min": 0.0, "z_max": 0.5},
                   {"medium": 1, "z_min": 0.5, "z_max": math.inf}],
        "laser": _laser(*CIRCULAR),
        "sensors": [
            {"kind": "farfield_cbs", "theta_max": 0.1, "phi_max": 2 * PI, "len_t": 0.0,
             "d_theta": 5e-4, "d_phi": PI / 4, "d_t": 0.0, "theta_limit": (0.0, 0.1)},
            {"kind": "planar_fluence", "z": 0.0, "len_x": 10.0, "len_y": 10.0, "len_t": 63.0,
             "dx": 0.05, "dy": 0.05, "d_t": 1.0, "absorb": True},
            {"kind": "farfield_fluence", "theta_max": PI / 2, "phi_max": 2 * PI, "len_t": 0.0,
             "d_theta": PI / 180, "d_phi": PI / 18, "d_t": 0.0},
        ],
        "n_photons": n_photons, "seed": seed, "max_events": 1000, "track_reverse_paths": True,
    }


def bilayer_hg(n_photons=10_000_000, seed=12345):
    """Bilayer geometry with Henyey-Greenstein theta sampling in both layers."""
    spec = bilayer_rgd_mie(n_photons, seed)
    spec["name"] = "bilayer_hg"
    spec["phases"] = [{"kind": "hg", "g": 0.8}, {"kind": "hg", "g": 0.9}]
    return spec


def mie_long_paths(n_photons=100_000_000, seed=12345, circular=False):
    """Long photon paths (mu_s = 100/mm, mu_a = 1e-4/mm) with a speckle grid."""
    return {
        "name": "mie_long_paths" + ("_circular" if circular else "_linear"), "n_host": N_WATER,
        "phases": [_mie_phase(1.0e-3)],
        "media": [_medium("mie", 0, 1.0e-3, 100.0, 1e-4, 0.01)],
        "layers": [{"medium": 0, "z_min": 0.0, "z_max": math.inf}],
        "laser": _laser(*(CIRCULAR if circular else LINEAR)),
        "sensors": [
            {"kind": "farfield_cbs", "theta_max": 0.02, "phi_max": 2 * PI, "len_t": 0.0,
             "d_theta": 5e-5, "d_phi": 2 * PI, "d_t": 0.0, "theta_limit": (0.0, 0.02)},
            {"kind": "planar_field", "z": 0.0, "len_x": 2.56, "len_y": 2.56, "dx": 0.01,
             "dy": 0.01, "absorb": True},
        ],
        "n_photons": n_photons, "seed": seed, "max_events": 1_000_000,
        "track_reverse_paths": True,
    }


def mie_sweep_parameters(count=256, seed=2026):
    """Seeded draws of the sweep's media: radius [mm], mu_s, mu_a [1/mm], photons."""
    rng = np.random.default_rng(seed)
    radius = np.exp(rng.uniform(math.log(0.05e-3), math.log(2.0e-3), count))
    mu_s = rng.uniform(1.0, 50.0, count)
    mu_a = np.exp(rng.uniform(math.log(1e-4), math.log(0.1), count))
    photons = np.exp(rng.uniform(math.log(1e5), math.log(1e7), count)).astype(np.int64)
    return radius, mu_s, mu_a, photons


def mie_sweep(i, seed=12345, count=256):
    r, mu_s, mu_a, photons = mie_sweep_parameters(count)
    spec = mie_cbs_small(int(photons[i]), seed)
    spec["name"] = f"mie_sweep_{i}"
    spec["phases"] = [_mie_phase(float(r[i]))]
    spec["media"] = [_medium("mie", 0, float(r[i]), float(mu_s[i]), float(mu_a[i]))]
    return spec


def build_mie_sweep(lm, specs):
    """Configs of single-medium Mie sweep specs (``mie_sweep``) whose phase functions and
    media are built together by ``lm.mie_species`` (one GPU batch) instead of one by one."""
    keys = []
    for sp in specs:
        p, m = sp["phases"][0], sp["media"][0]
        if len(sp["phases"]) != 1 or len(sp["media"]) != 1 or p["kind"] != "mie" or m["kind"] != "mie":
            raise ValueError("build_mie_sweep takes single-medium Mie specs")
        if (p["wavelength"], p["radius"], p["n_particle"], p["n_medium"]) != (
                m["wavelength"], m["radius"], m["n_particle"], m["n_medium"]):
            raise ValueError("phase function and medium must describe the same particle")
        keys.append((p["nDiv"], p["min"], p["max"]))
    if len(set(keys)) > 1:
        raise ValueError("all phase tables of a batch share nDiv, minVal, maxVal")
    n_div, lo, hi = keys[0] if keys else (1000, 0.0, PI)
    pairs = lm.mie_species([(sp["phases"][0]["wavelength"], sp["phases"][0]["radius"],
                             sp["phases"][0]["n_particle"], sp["phases"][0]["n_medium"])
                            for sp in specs], n_div, lo, hi)
    return [build(lm, sp, prebuilt=([ph], [med]))[0] for sp, (ph, med) in zip(specs, pairs)]


def mixture_bilayer(n_photons=10_000_000, seed=12345):
    """A MixtureLayer of three co-located species -- polystyrene spheres r = 0.5 um
    (n = 3e6 /mm^3, mu_s_i ~ 6.1/mm) and r = 0.25 um (1.5e7 /mm^3, ~2.3/mm) and RGD
    spheres r = 0.1 um (2e9 /mm^3, ~4.6/mm), each with its own albedo -- in 0 <= z < 0.5
    mm over the semi-infinite Mie medium.  Circular polarisation; FarFieldCBS 200 x 8,
    PlanarFluence 100 x 100 x 32 time bins over 10 x 10 mm."""
    spec = bilayer_rgd_mie(n_photons, seed)
    spec["name"] = "mixture_bilayer"
    spec["phases"].append(_mie_phase(0.25e-3))
    spec["media"].append(_medium("mie", 2, 0.25e-3, 5.0, 0.2))
    spec["layers"] = [{"species": [1, 0, 2], "densities": [3.0e6, 2.0e9, 1.5e7],
                       "z_min": 0.0, "z_max": 0.5},
                      {"medium": 1, "z_min": 0.5, "z_max": math.inf}]
    spec["sensors"][1].update(dx=0.1, dy=0.1, len_t=31.0, d_t=1.0)
    spec["sensors"].pop(2)
    return spec


def mixture_cbs_small(n_photons=1_000_000, seed=12345):
    """A semi-infinite MixtureLayer of the r = 0.5 um Mie and r = 0.1 um RGD species
    (3e6 and 2e9 /mm^3), linear pencil beam, FarFieldCBS 100 x 1 and PlanarFluence."""
    spec = mie_cbs_small(n_photons, seed)
    spec["name"] = "mixture_cbs_small"
    spec["phases"].append({"kind": "rdemc", "wavelength": LAMBDA, "radius": 0.1e-3,
                           "n_particle": N_SPHERE, "n_medium": N_WATER, "nDiv": 1000,
                           "min": 0.0, "max": PI})
    spec["media"].append(_medium("rgd", 1, 0.1e-3, 20.0, 0.05, 0.05))
    spec["layers"] = [{"species": [0, 1], "densities": [3.0e6, 2.0e9],
                       "z_min": 0.0, "z_max": math.inf}]
    spec["sensors"].append({"kind": "planar_fluence", "z": 0.0, "len_x": 4.0, "len_y": 4.0,
                            "len_t": 0.0, "dx": 0.25, "dy": 0.25, "d_t": 0.0, "absorb": True})
    return spec


WORKLOADS = {"mie_cbs_small": mie_cbs_small, "bilayer_rgd_mie": bilayer_rgd_mie,
             "bilayer_hg": bilayer_hg, "mie_long_paths": mie_long_paths,
             "mixture_bilayer": mixture_bilayer, "mixture_cbs_small": mixture_cbs_small}


# --------------------------------------------------------------------------- builder
_PHASE_CTORS = {
    "uniform": lambda lm, p: lm.UniformPhaseFunction(),
    "rayleigh": lambda lm, p: lm.RayleighPhaseFunction(p["nDiv"], p["min"], p["max"]),
    "hg": lambda lm, p: lm.HenyeyGreensteinPhaseFunction(p["g"]),
    "rd": lambda lm, p: lm.RayleighDebyePhaseFunction(p["wavelength"], p["radius"], p["nDiv"],
                                                      p["min"], p["max"]),
    "rdemc": lambda lm, p: lm.RayleighDebyeEMCPhaseFunction(
        p["wavelength"], p["radius"], p["n_particle"], p["n_medium"], p["nDiv"], p["min"], p["max"]),
    "draine": lambda lm, p: lm.DrainePhaseFunction(p["g"], p["a"], p["nDiv"], p["min"], p["max"]),
    "mie": lambda lm, p: lm.MiePhaseFunction(p["wavelength"], p["radius"], p["n_particle"],
                                             p["n_medium"], p["nDiv"], p["min"], p["max"]),
}


def build(lm, spec, n_photons=None, seed=None, n_threads=None, prebuilt=None):
    """Build (config, sensor handles, keep-alive list) with the luminis-mc API of ``lm``.

    Sensors whose class ``lm`` does not define are skipped and reported as None.
    ``prebuilt`` = (phases, media objects) replaces the per-object constructors (the
    media's coefficients are still set from the spec).
    """
    keep = []
    phases = (list(prebuilt[0]) if prebuilt else
              [_PHASE_CTORS[p["kind"]](lm, p) for p in spec["phases"]])
    keep += phases
    media = []
    for j, m in enumerate(spec["media"]):
        if prebuilt:
            med = prebuilt[1][j]
        else:
            cls = lm.MieMedium if m["kind"] == "mie" else lm.RGDMedium
            med = cls(phases[m["phase"]], m["radius"], m["n_particle"], m["n_medium"],
                      m["wavelength"])
        med.set_scattering_coefficient(m["mu_s"])
        med.set_absorption_coefficient(m["mu_a"])
        med.set_mean_free_path(m["mfp"])
        media.append(med)
    keep += media
    sample = lm.Sample(spec.get("n_host", 1.0))
    for l in spec["layers"]:
        if "species" in l:
            sample.add_mixture_layer([media[i] for i in l["species"]],
                                     [float(n) for n in l["densities"]], l["z_min"], l["z_max"])
        else:
            sample.add_layer(media[l["medium"]], l["z_min"], l["z_max"])
    L = spec["laser"]
    source = {"point": lm.LaserSource.Point, "uniform": lm.LaserSource.Uniform,
              "gaussian": lm.LaserSource.Gaussian}[L.get("source", "point")]
    laser = lm.Laser(complex(L["m"]), complex(L["n"]), L["wavelength"], L.get("sigma", 0.0), source)
    if "position" in L:
        laser.position = lm.Vec3(*L["position"])
    group = lm.SensorsGroup()
    handles = []
    for s in spec["sensors"]:
        kind = s["kind"]
        if kind == "farfield_cbs":
            det = lm.FarFieldCBSSensor(s["theta_max"], s["phi_max"], s.get("len_t", 0.0),
                                       s["d_theta"], s["d_phi"], s.get("d_t", 0.0),
                                       s.get("estimator", False))
        elif kind == "planar_fluence":
            det = lm.PlanarFluenceSensor(s["z"], s["len_x"], s["len_y"], s.get("len_t", 0.0),
                                         s["dx"], s["dy"], s.get("d_t", 0.0),
                                         s.get("absorb", True), s.get("estimator", False))
        elif kind == "planar_field":
            det = lm.PlanarFieldSensor(s["z"], s["len_x"], s["len_y"], s["dx"], s["dy"],
                                       s.get("absorb", True), s.get("estimator", False))
        elif kind == "statistics":
            det = lm.StatisticsSensor(s["z"], s.get("absorb", False))
            if s.get("d_t", 0.0) > 0.0:
                det.set_time_resolution(s["len_t"], s["d_t"])
            if "events" in s:
                det.set_events_histogram_bins(int(s["events"]))
            if "theta" in s:
                det.set_theta_histogram_bins(*s["theta"])
            if "phi" in s:
                det.set_phi_histogram_bins(*s["phi"])
            if "depth" in s:
                det.set_depth_histogram_bins(*s["depth"])
            if "time" in s:
                det.set_time_histogram_bins(*s["time"])
            if "weight" in s:
                det.set_weight_histogram_bins(*s["weight"])
        elif kind == "farfield_fluence":
            if not hasattr(lm, "FarFieldFluenceSensor"):
                handles.append(None)
                continue
            det = lm.FarFieldFluenceSensor(s["theta_max"], s["phi_max"], s.get("len_t", 0.0),
                                           s["d_theta"], s["d_phi"], s.get("d_t", 0.0))
        else:
            raise ValueError(f"unknown sensor kind {kind!r}")
        if "theta_pp_max" in s:
            det.theta_pp_max = float(s["theta_pp_max"])
        if "theta_limit" in s:
            det.set_theta_limit(*s["theta_limit"])
        if "phi_limit" in s:
            det.set_phi_limit(*s["phi_limit"])
        if "position_limit" in s:
            det.set_position_limit(*s["position_limit"])
        if "events_limit" in s:
            det.set_events_limit(*s["events_limit"])
        if "direction_limit" in s:
            det.set_direction_limit({"forward": lm.CrossingDirection.Forward,
                                     "backward": lm.CrossingDirection.Backward,
                                     "both": lm.CrossingDirection.Both}[s["direction_limit"]])
        handles.append(group.add_detector(det))
    cfg = lm.SimConfig()
    cfg.n_photons = int(spec["n_photons"] if n_photons is None else n_photons)
    cfg.seed = int(spec["seed"] if seed is None else seed)
    cfg.MAX_EVENTS = int(spec.get("max_events", 1000))
    cfg.track_reverse_paths = bool(spec.get("track_reverse_paths", True))
    cfg.show_progress = False
    if n_threads is not None:
        cfg.n_threads = int(n_threads)
    cfg.sample = sample
    cfg.laser = laser
    cfg.detector = group
    keep += [sample, laser, group]
    a = spec.get("absorption")
    if a is not None:
        rec = lm.Absorption(a["radius"], a["depth"], a["d_r"], a["d_z"], a.get("d_t", 0.0),
                            a.get("t_max", 0.0))
        cfg.absorption = rec
        keep.append(rec)
    return cfg, handles, keep


def tally_arrays(lm_sensor, kind):
    """Copy a sensor's tallies into one float64 array in the oracle layout."""
    if kind == "farfield_cbs":
        grids = [lm_sensor.S0_coh, lm_sensor.S1_coh, lm_sensor.S2_coh, lm_sensor.S3_coh,
                 lm_sensor.S0_incoh, lm_sensor.S1_incoh, lm_sensor.S2_incoh, lm_sensor.S3_incoh]
        return np.stack([np.stack([np.array(m, copy=True) for m in g]) for g in grids])
    if kind in ("planar_fluence", "farfield_fluence"):
        grids = [lm_sensor.S0, lm_sensor.S1, lm_sensor.S2, lm_sensor.S3]
        return np.stack([np.stack([np.array(m, copy=True) for m in g]) for g in grids])
    if kind == "statistics":
        parts = []
        for name in ("events", "theta", "phi", "depth", "time", "weight"):
            if getattr(lm_sensor, f"{name}_histogram_bins_set"):
                parts.append(np.asarray(getattr(lm_sensor, f"{name}_histogram"),
                                        dtype=np.float64).ravel())
        return np.concatenate(parts) if parts else np.zeros(0)
    if kind == "planar_field":
        ex = np.array(lm_sensor.Ex, copy=True)
        ey = np.array(lm_sensor.Ey, copy=True)
        return np.stack([ex, ey]).view(np.float64).reshape(2, ex.shape[0], ex.shape[1], 2)
    raise ValueError(kind)
