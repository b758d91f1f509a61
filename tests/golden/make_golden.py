"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own Python API (its pybind module built from its sources by
oracle/Makefile into oracle/_ref) on small scenes and stores every sensor's
tallies and hit counts:

  ref_xoshiro_<scene>.npz  the unmodified reference, its own RNG, n_threads=1
                           ("pin" build: -O2 -ffp-contract=off)
  ref_philox_<scene>.npz   the reference with the Philox replay seam
                           (oracle/replay_rng.cpp), the stream the GPU draws
  ref_farfield_fluence_small.npz  the far-field fluence definition applied to the
                           reference's own PhotonRecordSensor records (replay build)
  stat_ref_<scene>.npz     R independent-seed replicas of the unmodified reference
                           (its own RNG): per-bin mean and variance of tally / N,
                           the statistical oracle for other random streams
  cone_ref_<scene>.npz     the same for the FarFieldCBS grids of the workloads, plus
                           every replica's theta profiles of S0 coherent / incoherent

    python tests/golden/make_golden.py        (needs oracle/_ref; run `make -C oracle ref`)
    python tests/golden/make_golden.py stat   (the replica fixtures only)
    python tests/golden/make_golden.py cone   (CBS cone replicas at the workloads' resolution)
    python tests/golden/make_golden.py farfield  (far-field fluence from reference records)
    python tests/golden/make_golden.py estimator (estimator-mode FarFieldCBS, Philox stream)
    python tests/golden/make_golden.py mixture   (MixtureLayer scenes, both streams)
    python tests/golden/make_golden.py absorption (Absorption recorder scenes, both streams)
    python tests/golden/make_golden.py statistics (StatisticsSensor scenes, both streams)

The fixtures pin the oracle (tests/test_oracle_golden.py) and the GPU path
(tests/test_gpu_golden.py) without the reference present at test time.
"""
import ctypes
import glob
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "luminis-mc_b200"))

from luminis_mc_b200 import workloads as W  # noqa: E402


def golden_scenes():
    """Small scenes covering every sensor type the reference has, both media, HG,
    interfaces, time bins, filters and circular/linear polarisation."""
    a = W.mie_cbs_small(2000, 20240)
    b = W.bilayer_rgd_mie(2000, 77)
    b["name"] = "bilayer_small"
    b["sensors"][1].update(len_x=4.0, len_y=4.0, dx=0.2, dy=0.2, len_t=15.0, d_t=1.0)
    b["sensors"].pop(2)           # FarFieldFluence has no reference class
    c = W.bilayer_hg(1500, 5)
    c["name"] = "bilayer_hg_small"
    c["sensors"][1].update(len_x=4.0, len_y=4.0, dx=0.25, dy=0.25, len_t=0.0, d_t=0.0)
    c["sensors"].pop(2)
    d = W.mie_long_paths(150, 9)
    d["name"] = "mie_speckle_small"
    d["max_events"] = 5000
    d["sensors"][1].update(len_x=0.64, len_y=0.64, dx=0.02, dy=0.02)
    return [a, b, c, d]


STAT_REPLICAS = 16
STAT_PHOTONS = 100_000


def stat_scenes():
    """Scenes with coarse detectors, so that a CPU reference run of R x 1e5 photons fills
    most bins: mu_a = 0.5/mm keeps paths short.  Every detector kind the reference has,
    both polarisations, an interface, time bins."""
    PI = W.PI
    cbs = {"kind": "farfield_cbs", "theta_max": 0.5, "phi_max": 2 * PI, "len_t": 0.0,
           "d_theta": 0.05, "d_phi": PI / 2, "d_t": 0.0, "theta_limit": (0.0, 0.5)}
    flu = {"kind": "planar_fluence", "z": 0.0, "len_x": 4.0, "len_y": 4.0, "len_t": 8.0,
           "dx": 0.5, "dy": 0.5, "d_t": 2.0, "absorb": True}
    a = W.mie_cbs_small(STAT_PHOTONS, 1)
    a["name"] = "stat_mie"
    a["media"][0].update(mu_a=0.5)
    a["sensors"] = [dict(cbs), dict(flu)]
    b = W.bilayer_rgd_mie(STAT_PHOTONS, 1)
    b["name"] = "stat_bilayer"
    b["media"][0].update(mu_a=0.5)
    b["media"][1].update(mu_a=0.5)
    b["sensors"] = [dict(cbs, len_t=6.0, d_t=3.0), dict(flu),
                    {"kind": "planar_field", "z": 0.0, "len_x": 1.6, "len_y": 1.6,
                     "dx": 0.2, "dy": 0.2, "absorb": True}]
    return [a, b]


def replica_moments(tallies_by_replica, n_photons):
    """Per-bin mean and sample variance (ddof=1) of tally / N over the replicas,
    one (mean, var) pair per sensor."""
    out = []
    for sensor in zip(*tallies_by_replica):
        x = np.stack([np.asarray(t, dtype=np.float64) / n_photons for t in sensor])
        out.append((x.mean(axis=0), x.var(axis=0, ddof=1)))
    return out


def run_stat_reference(scene_name):
    """R replicas of one stat scene with the reference's own RNG (pin build), in a
    fresh interpreter; returns {sensor<i>_mean, sensor<i>_var, R, N}."""
    code = f"""
import os, sys, numpy as np
sys.path.insert(0, {REPO!r}); sys.path.insert(0, {os.path.join(REPO, 'luminis-mc_b200')!r})
from tests.golden.make_golden import stat_scenes, replica_moments, STAT_REPLICAS, STAT_PHOTONS
from luminis_mc_b200 import workloads as W
from oracle import pyoracle as O
lm = O.reference_module("pin"); lm.set_log_level(lm.LogLevel.off)
spec = [s for s in stat_scenes() if s["name"] == {scene_name!r}][0]
reps = []
for r in range(STAT_REPLICAS):
    cfg, hs, keep = W.build(lm, spec, seed=1000 + r, n_threads=os.cpu_count())
    lm.run_simulation_parallel(cfg)
    reps.append([W.tally_arrays(h, s["kind"]) for h, s in zip(hs, spec["sensors"])])
out = {{"R": np.int64(STAT_REPLICAS), "N": np.int64(STAT_PHOTONS)}}
for i, (m, v) in enumerate(replica_moments(reps, STAT_PHOTONS)):
    out[f"sensor{{i}}_mean"] = m
    out[f"sensor{{i}}_var"] = v
np.savez_compressed(sys.argv[1], **out)
"""
    path = os.path.join(HERE, f"stat_ref_{scene_name}.npz")
    subprocess.run([sys.executable, "-c", code, path], check=True)
    return path


def stat_main():
    for spec in stat_scenes():
        print("wrote", run_stat_reference(spec["name"]))


CONE_REPLICAS = 16
CONE_PHOTONS = 1_000_000


def cone_scenes():
    """The CBS cone at the resolution the workloads use: the mie_cbs_small detector as
    written (100 theta bins of 1 mrad to 0.1 rad, one phi bin, mu_a = 0.01/mm) and the
    bilayer_rgd_mie FarFieldCBS grid (200 x 8 bins to 0.1 rad) alone on that geometry.
    1e6 photons per replica put tens of photons into the innermost 10 mrad, where the
    enhancement eta = S0_coh / S0_incoh peaks."""
    a = W.mie_cbs_small(CONE_PHOTONS, 1)
    a["name"] = "cone_mie"
    b = W.bilayer_rgd_mie(CONE_PHOTONS, 1)
    b["name"] = "cone_bilayer"
    b["sensors"] = [b["sensors"][0]]
    return [a, b]


def cone_profiles(tally):
    """S0 coherent and incoherent of a FarFieldCBS tally [8][N_t][N_theta][N_phi],
    time bin 0, summed over phi: two profiles over theta."""
    t = np.asarray(tally)
    return t[0, 0].sum(axis=-1), t[4, 0].sum(axis=-1)


def run_cone_reference(scene_name, seed0=1000, path=None):
    """R replicas of one cone scene with the reference's own RNG (pin build), in a fresh
    interpreter: per-bin moments of the full grid and every replica's theta profiles of
    S0 coherent / incoherent (for the enhancement near theta = 0)."""
    code = f"""
import os, sys, numpy as np
sys.path.insert(0, {REPO!r}); sys.path.insert(0, {os.path.join(REPO, 'luminis-mc_b200')!r})
from tests.golden.make_golden import (cone_scenes, cone_profiles, replica_moments,
                                      CONE_REPLICAS, CONE_PHOTONS)
from luminis_mc_b200 import workloads as W
from oracle import pyoracle as O
lm = O.reference_module("pin"); lm.set_log_level(lm.LogLevel.off)
spec = [s for s in cone_scenes() if s["name"] == {scene_name!r}][0]
reps, coh, inc = [], [], []
for r in range(CONE_REPLICAS):
    cfg, hs, keep = W.build(lm, spec, seed={seed0} + r, n_threads=os.cpu_count())
    lm.run_simulation_parallel(cfg)
    t = [W.tally_arrays(h, s["kind"]) for h, s in zip(hs, spec["sensors"])]
    reps.append(t)
    c, i = cone_profiles(t[0])
    coh.append(c)
    inc.append(i)
out = {{"R": np.int64(CONE_REPLICAS), "N": np.int64(CONE_PHOTONS),
       "coh_theta": np.stack(coh), "incoh_theta": np.stack(inc)}}
for i, (m, v) in enumerate(replica_moments(reps, CONE_PHOTONS)):
    out[f"sensor{{i}}_mean"] = m
    out[f"sensor{{i}}_var"] = v
np.savez_compressed(sys.argv[1], **out)
"""
    path = path or os.path.join(HERE, f"cone_ref_{scene_name}.npz")
    subprocess.run([sys.executable, "-c", code, path], check=True)
    return path


def cone_main():
    for spec in cone_scenes():
        print("wrote", run_cone_reference(spec["name"]))


def estimator_scenes():
    """Estimator-mode FarFieldCBS (the reference's last-flight CBS estimate at every
    scattering vertex): one semi-infinite Mie medium with the cfg-0 grid, and the
    two-layer slab with time bins, a 2-D angular grid and a theta cap, where the
    straight rays to the detector cross the interface."""
    a = W.mie_cbs_small(300, 31)
    a["name"] = "estimator_mie"
    a["media"][0].update(mu_a=0.2)
    a["sensors"] = [dict(a["sensors"][0], estimator=True)]
    b = W.bilayer_rgd_mie(200, 32)
    b["name"] = "estimator_bilayer"
    b["media"][0].update(mu_a=0.5)
    b["media"][1].update(mu_a=0.5)
    b["sensors"] = [{"kind": "farfield_cbs", "theta_max": 0.2, "phi_max": 2 * W.PI, "len_t": 12.0,
                     "d_theta": 0.01, "d_phi": W.PI / 2, "d_t": 2.0, "estimator": True,
                     "theta_pp_max": 0.15},
                    {"kind": "planar_fluence", "z": 0.0, "len_x": 4.0, "len_y": 4.0, "len_t": 0.0,
                     "dx": 0.5, "dy": 0.5, "d_t": 0.0, "absorb": True}]
    return [a, b]


def estimator_main():
    meta = {}
    for spec in estimator_scenes():
        name = spec["name"]
        np.savez_compressed(os.path.join(HERE, f"ref_philox_{name}.npz"),
                            **run_flavour("replay", name, fmt=0, source="estimator_scenes"))
        meta[name] = {"n_photons": spec["n_photons"], "seed": spec["seed"]}
    print("wrote", meta)


def mixture_scenes():
    """MixtureLayer scenes (species drawn per vertex, aggregate free paths and albedo):
    the three-species slab over the Mie medium (FarFieldCBS 200 x 8, PlanarFluence with
    time bins), the semi-infinite two-species mixture, and estimator-mode FarFieldCBS
    in that mixture (first-vertex layer albedo, later-vertex species albedo)."""
    a = W.mixture_bilayer(1500, 41)
    a["name"] = "mixture_bilayer_small"
    a["sensors"][1].update(len_x=4.0, len_y=4.0, dx=0.25, dy=0.25, len_t=15.0, d_t=1.0)
    b = W.mixture_cbs_small(2000, 42)
    c = W.mixture_cbs_small(250, 43)
    c["name"] = "estimator_mixture"
    c["media"][1].update(mu_a=0.5)
    c["sensors"] = [dict(c["sensors"][0], estimator=True, d_theta=2e-3, theta_max=0.1)]
    return [a, b, c]


def absorption_scenes():
    """Absorption recorder scenes: the two-layer slab with a time-resolved (r, z, t)
    grid whose depth ends inside the second layer, and the mixture slab with a
    time-integrated grid (deposits use the layer's aggregate albedo)."""
    a = W.bilayer_rgd_mie(1500, 51)
    a["name"] = "absorption_bilayer"
    a["media"][0].update(mu_a=2.0)
    a["media"][1].update(mu_a=0.5)
    a["sensors"] = [a["sensors"][0]]
    a["absorption"] = {"radius": 2.0, "depth": 1.5, "d_r": 0.1, "d_z": 0.05, "d_t": 2.0,
                       "t_max": 20.0}
    b = W.mixture_bilayer(1200, 52)
    b["name"] = "absorption_mixture"
    b["sensors"] = [b["sensors"][0]]
    b["absorption"] = {"radius": 3.0, "depth": 2.0, "d_r": 0.25, "d_z": 0.1}
    return [a, b]


def statistics_scenes():
    """StatisticsSensor scenes: on the two-layer slab a time-resolved sensor with all
    six histograms beside the FarFieldCBS sensor at z = 0, and a non-absorbing one
    inside the sample (z = 0.25, crossed any number of times, backward crossings
    only); on the Mie medium a sensor with theta and event filters."""
    a = W.bilayer_rgd_mie(1500, 61)
    a["name"] = "stats_bilayer"
    a["sensors"] = [a["sensors"][0],
                    {"kind": "statistics", "z": 0.0, "absorb": True, "len_t": 20.0, "d_t": 2.0,
                     "events": 200, "theta": (0.0, W.PI / 2, 30), "phi": (0.0, 2 * W.PI, 12),
                     "depth": (3.0, 30), "time": (30.0, 30), "weight": (1.0, 20)},
                    {"kind": "statistics", "z": 0.25, "absorb": False, "events": 60,
                     "depth": (2.0, 40), "direction_limit": "backward"}]
    b = W.mie_cbs_small(2500, 62)
    b["name"] = "stats_mie"
    b["sensors"] = [{"kind": "statistics", "z": 0.0, "absorb": True, "events": 100,
                     "theta": (0.0, 1.2, 24), "weight": (0.5, 25), "theta_limit": (0.1, 1.0),
                     "events_limit": (2, 80)}]
    return [a, b]


def statistics_main():
    meta = {}
    for spec in statistics_scenes():
        name = spec["name"]
        np.savez_compressed(os.path.join(HERE, f"ref_philox_{name}.npz"),
                            **run_flavour("replay", name, fmt=0, source="statistics_scenes"))
        np.savez_compressed(os.path.join(HERE, f"ref_xoshiro_{name}.npz"),
                            **run_flavour("pin", name, source="statistics_scenes"))
        meta[name] = {"n_photons": spec["n_photons"], "seed": spec["seed"]}
    print("wrote", meta)


def absorption_main():
    meta = {}
    for spec in absorption_scenes():
        name = spec["name"]
        np.savez_compressed(os.path.join(HERE, f"ref_philox_{name}.npz"),
                            **run_flavour("replay", name, fmt=0, source="absorption_scenes"))
        np.savez_compressed(os.path.join(HERE, f"ref_xoshiro_{name}.npz"),
                            **run_flavour("pin", name, source="absorption_scenes"))
        meta[name] = {"n_photons": spec["n_photons"], "seed": spec["seed"]}
    print("wrote", meta)


def mixture_main():
    meta = {}
    for spec in mixture_scenes():
        name = spec["name"]
        np.savez_compressed(os.path.join(HERE, f"ref_philox_{name}.npz"),
                            **run_flavour("replay", name, fmt=0, source="mixture_scenes"))
        if not name.startswith("estimator"):
            np.savez_compressed(os.path.join(HERE, f"ref_xoshiro_{name}.npz"),
                                **run_flavour("pin", name, source="mixture_scenes"))
        meta[name] = {"n_photons": spec["n_photons"], "seed": spec["seed"]}
    print("wrote", meta)


FF_GRID = {"theta_max": 1.5707963267948966, "phi_max": 2 * 3.141592653589793, "len_t": 20.0,
           "d_theta": 3.141592653589793 / 36, "d_phi": 2 * 3.141592653589793 / 12, "d_t": 2.0}


def farfield_scene():
    """bilayer_small with one absorbing sensor at z = 0: a FarFieldFluenceSensor for
    this library and the oracle, a PhotonRecordSensor for the reference (which has no
    far-field fluence class); the photon histories are the same."""
    spec = W.bilayer_rgd_mie(2000, 77)
    spec["name"] = "farfield_fluence_small"
    spec["sensors"] = [dict(FF_GRID, kind="farfield_fluence")]
    return spec


def bin_farfield_fluence(records, grid):
    """The far-field fluence definition applied to the reference's own photon records
    (PhotonRecordSensor at z = 0): forward-field Stokes of each exiting photon, lab
    frame projection E_x = E_m m_x + E_n n_x, E_y = E_m m_y + E_n n_y (the FarFieldCBS
    incoherent part with a zero reverse field), binned on theta = acos(-s_z),
    phi = atan2(s_y, s_x) in [0, 2 pi), time-integrated bin 0 plus bin
    floor(t / dt) + 1 of the arrival time."""
    import math
    n_t = 1 if grid["d_t"] == 0 else int(math.ceil(grid["len_t"] / grid["d_t"])) + 1
    n_th = int(math.ceil(grid["theta_max"] / grid["d_theta"]))
    n_ph = int(math.ceil(grid["phi_max"] / grid["d_phi"]))
    out = np.zeros((4, n_t, n_th, n_ph))
    for r in records:
        if grid["d_t"] > 0:
            a = r["arrival"]
            if a < 0 or a >= grid["len_t"]:
                continue
            ti = int(a / grid["d_t"]) + 1
            if ti >= n_t:
                continue
        else:
            ti = 0
        sx, sy, sz = r["dir"]
        theta = math.acos(-sz)
        phi = math.atan2(sy, sx)
        if phi < 0:
            phi += 2.0 * math.pi
        it, jp = int(theta / grid["d_theta"]), int(phi / grid["d_phi"])
        if not (0 <= it < n_th and 0 <= jp < n_ph):
            continue
        w = math.sqrt(r["weight"])
        em, en = r["Em"] * w, r["En"] * w
        ex = em * r["m"][0] + en * r["n"][0]
        ey = em * r["m"][1] + en * r["n"][1]
        v = (abs(ex) ** 2 + abs(ey) ** 2, abs(ex) ** 2 - abs(ey) ** 2,
             2.0 * (ex * ey.conjugate()).real, 2.0 * (ex * ey.conjugate()).imag)
        for t in ((0, ti) if ti >= 1 else (0,)):
            out[:, t, it, jp] += v
    return out


def run_farfield_reference():
    """The reference (replay build, Philox u53) with a PhotonRecordSensor at z = 0;
    returns its records as plain dicts."""
    code = f"""
import sys, glob, ctypes, pickle
sys.path.insert(0, {REPO!r}); sys.path.insert(0, {os.path.join(REPO, 'luminis-mc_b200')!r})
from tests.golden.make_golden import farfield_scene
from luminis_mc_b200 import workloads as W
from oracle import pyoracle as O
lm = O.reference_module("replay"); lm.set_log_level(lm.LogLevel.off)
so = ctypes.CDLL(glob.glob({os.path.join(REPO, 'oracle', '_ref', 'replay', 'luminis_mc', '_core*.so')!r})[0])
so.lmc_replay_set_format(0)
spec = farfield_scene()
spec["sensors"] = []
cfg, hs, keep = W.build(lm, spec, n_threads=1)
rec = cfg.detector.add_detector(lm.PhotonRecordSensor(0.0, True))
lm.run_simulation_parallel(cfg)
out = []
for r in rec.recorded_photons:
    d = r.direction; m = r.m; n = r.n; E = r.polarization_forward
    out.append(dict(arrival=r.arrival_time, weight=r.weight, dir=(d.x, d.y, d.z), m=(m.x, m.y, m.z),
                    n=(n.x, n.y, n.z), Em=complex(E.m), En=complex(E.n)))
pickle.dump(out, open(sys.argv[1], "wb"))
"""
    import pickle
    tmp = os.path.join(HERE, "_tmp_records.pkl")
    subprocess.run([sys.executable, "-c", code, tmp], check=True)
    recs = pickle.load(open(tmp, "rb"))
    os.unlink(tmp)
    return recs


def farfield_main():
    recs = run_farfield_reference()
    t = bin_farfield_fluence(recs, FF_GRID)
    path = os.path.join(HERE, "ref_farfield_fluence_small.npz")
    np.savez_compressed(path, sensor0=t, records=np.int64(len(recs)))
    print("wrote", path, len(recs), "records")


def run_flavour(flavour, scene_name, fmt=None, source="golden_scenes"):
    """Run one scene in a fresh interpreter (each reference flavour is a module
    named luminis_mc) and return {sensor index: tally, 'hits': [...]}."""
    code = f"""
import sys, json, glob, ctypes, numpy as np
sys.path.insert(0, {REPO!r}); sys.path.insert(0, {os.path.join(REPO, 'luminis-mc_b200')!r})
from tests.golden.make_golden import (golden_scenes, estimator_scenes, mixture_scenes,
                                     absorption_scenes, statistics_scenes)
from luminis_mc_b200 import workloads as W
from oracle import pyoracle as O
lm = O.reference_module({flavour!r}); lm.set_log_level(lm.LogLevel.off)
if {fmt is not None!r}:
    so = ctypes.CDLL(glob.glob({os.path.join(REPO, 'oracle', '_ref', flavour, 'luminis_mc', '_core*.so')!r})[0])
    so.lmc_replay_set_format({fmt if fmt is not None else 0})
spec = [s for s in {source}() if s["name"] == {scene_name!r}][0]
cfg, hs, keep = W.build(lm, spec, n_threads=1)
lm.run_simulation_parallel(cfg)
out = {{}}
for i, (h, s) in enumerate(zip(hs, spec["sensors"])):
    out[f"sensor{{i}}"] = W.tally_arrays(h, s["kind"])
out["hits"] = np.array([h.hits for h in hs], dtype=np.int64)
if cfg.absorption is not None:
    out["absorption"] = np.stack([np.array(m, copy=True) for m in cfg.absorption.time_slices])
np.savez(sys.argv[1], **out)
"""
    tmp = os.path.join(HERE, f"_tmp_{flavour}_{scene_name}.npz")
    subprocess.run([sys.executable, "-c", code, tmp], check=True)
    data = dict(np.load(tmp))
    os.unlink(tmp)
    return data


def main():
    meta = {}
    for spec in golden_scenes():
        name = spec["name"]
        np.savez_compressed(os.path.join(HERE, f"ref_xoshiro_{name}.npz"),
                            **run_flavour("pin", name))
        np.savez_compressed(os.path.join(HERE, f"ref_philox_{name}.npz"),
                            **run_flavour("replay", name, fmt=0))
        meta[name] = {"n_photons": spec["n_photons"], "seed": spec["seed"],
                      "max_events": spec["max_events"],
                      "sensors": [s["kind"] for s in spec["sensors"]]}
    with open(os.path.join(HERE, "golden_meta.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "reference_builds": "oracle/_ref/pin (own RNG), oracle/_ref/replay (Philox u53)",
                   "scenes": meta}, f, indent=1)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "stat":
        stat_main()
    elif len(sys.argv) > 1 and sys.argv[1] == "cone":
        cone_main()
    elif len(sys.argv) > 1 and sys.argv[1] == "farfield":
        farfield_main()
    elif len(sys.argv) > 1 and sys.argv[1] == "estimator":
        estimator_main()
    elif len(sys.argv) > 1 and sys.argv[1] == "mixture":
        mixture_main()
    elif len(sys.argv) > 1 and sys.argv[1] == "absorption":
        absorption_main()
    elif len(sys.argv) > 1 and sys.argv[1] == "statistics":
        statistics_main()
    else:
        main()
