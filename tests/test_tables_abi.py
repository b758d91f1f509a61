"""Host side of the product on CPU: set-up physics against the oracle, and the C
ABI (every declared symbol exported, struct layouts identical to ctypes')."""
import ctypes as C
import math
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import _native as N
from luminis_mc_b200 import workloads as W
from oracle import pyoracle as O

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "luminis_b200.h")


def test_library_exports_every_declared_symbol():
    decl = re.findall(r"LMC_API\s+[\w\s\*]+?\b(lmc_\w+)\s*\(", open(HEADER).read())
    assert decl and set(decl) == set(N.EXPORTED)
    L = N.lib()
    for name in decl:
        assert hasattr(L, name), name


def test_checked_library_exports_the_same_symbols():
    """The bounds-checked debug build (build.py --bounds-check) is a drop-in for the
    product library: it loads and exports every declared entry point."""
    import ctypes
    assert os.path.exists(N.CHECKED_LIB_PATH), "build the checked library (build.py --bounds-check)"
    L = ctypes.CDLL(N.CHECKED_LIB_PATH)
    for name in N.EXPORTED:
        assert hasattr(L, name), name


def test_struct_layouts_match_ctypes():
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "luminis_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(lmc_scene),
         sizeof(lmc_medium_desc), sizeof(lmc_sensor_desc), sizeof(lmc_laser_desc),
         sizeof(lmc_run_opts), sizeof(lmc_stats), sizeof(lmc_record), offsetof(lmc_scene, sensors),
         offsetof(lmc_run_opts, batch_photons), sizeof(lmc_mie_species),
         offsetof(lmc_run_opts, tally_mode), sizeof(lmc_tune_result),
         offsetof(lmc_tune_result, tally_mode));
  printf("%d %d %d %d\n", LMC_TALLY_DEFAULT, LMC_TALLY_GLOBAL, LMC_TALLY_WARP, LMC_TALLY_SHARED);
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        lines = subprocess.run([exe], capture_output=True, text=True).stdout.splitlines()
    got = list(map(int, lines[0].split()))
    want = [C.sizeof(N.SceneDesc), C.sizeof(N.MediumDesc), C.sizeof(N.SensorDesc),
            C.sizeof(N.LaserDesc), C.sizeof(N.RunOpts), C.sizeof(N.Stats),
            np.dtype(N.RECORD_FIELDS).itemsize, N.SceneDesc.sensors.offset,
            N.RunOpts.batch_photons.offset, C.sizeof(N.MieSpecies),
            N.RunOpts.tally_mode.offset, C.sizeof(N.TuneResult), N.TuneResult.tally_mode.offset]
    assert got == want
    # lmc_tally_mode values, as the Python layer names them
    assert list(map(int, lines[1].split())) == [N.TALLY_MODES[k] for k in
                                                 ("default", "global", "warp", "shared")]


def test_tally_mode_names():
    """Run options take a tally mode by name or value; anything else is a ValueError
    before any call into the library."""
    assert N.tally_mode_value("shared") == 3 and N.tally_mode_value(2) == 2
    for bad in ("atomic", 4, -1):
        with pytest.raises(ValueError, match="tally_mode"):
            N.tally_mode_value(bad)


PHASES = [
    {"kind": "mie", "wavelength": 0.633e-3, "radius": 0.5e-3, "n_particle": 1.59, "n_medium": 1.33,
     "nDiv": 1000, "min": 0.0, "max": math.pi},
    {"kind": "mie", "wavelength": 0.514e-3, "radius": 2.0e-3, "n_particle": 1.59, "n_medium": 1.33,
     "nDiv": 10000, "min": 0.0, "max": math.pi},
    {"kind": "rdemc", "wavelength": 0.633e-3, "radius": 0.1e-3, "n_particle": 1.59,
     "n_medium": 1.33, "nDiv": 1000, "min": 0.0, "max": math.pi},
    {"kind": "rd", "wavelength": 0.633e-3, "radius": 0.2e-3, "nDiv": 500, "min": 0.0, "max": math.pi},
    {"kind": "rayleigh", "nDiv": 400, "min": -1.0, "max": 1.0},
    {"kind": "draine", "g": 0.7, "a": 0.5, "nDiv": 400, "min": -1.0, "max": 1.0},
    # odd nDiv: SamplingTable::initialize (src/table.cpp:23-41) writes and reads pdf[nDiv]
    # one past its nDiv-element vector; for odd nDiv that overwrites glibc's next chunk
    # header and the reference aborts in free() before it returns.  The tables here are
    # sized nDiv + 1 and follow the reference's arithmetic (the oracle's restatement); the
    # reference itself returns them for even nDiv only.
    {"kind": "mie", "wavelength": 0.633e-3, "radius": 0.5e-3, "n_particle": 1.59, "n_medium": 1.33,
     "nDiv": 999, "min": 0.0, "max": math.pi},
    {"kind": "rayleigh", "nDiv": 401, "min": -1.0, "max": 1.0},
]


@pytest.mark.parametrize("phase", PHASES, ids=lambda p: f"{p['kind']}-{p['nDiv']}")
def test_sampling_tables_bit_identical_to_oracle(phase):
    spec = W.mie_cbs_small(10, 1)
    spec["phases"] = [phase]
    spec["media"][0]["kind"] = "rgd" if phase["kind"] != "mie" else "mie"
    cfg, _, keep = W.build(lm, spec)
    v, c = cfg.sample.layers[0].medium.phase_function._table()
    ov, oc = O.Oracle(spec).phase_table(0)
    np.testing.assert_array_equal(v, ov)
    np.testing.assert_array_equal(c, oc)
    ph = cfg.sample.layers[0].medium.phase_function
    o = O.Oracle(spec)
    for u in np.linspace(1e-6, 1 - 1e-6, 97):
        assert ph.sample_theta(u) == pytest.approx(o.sample_theta(0, u), rel=1e-13, abs=1e-13)


@pytest.mark.parametrize("kind,radius", [("mie", 0.05e-3), ("mie", 0.5e-3), ("mie", 2.0e-3),
                                         ("rgd", 0.1e-3), ("rgd", 0.035e-3)])
def test_amplitude_tables_bit_identical_to_oracle(kind, radius):
    spec = W.mie_cbs_small(10, 1)
    spec["media"][0].update(kind=kind, radius=radius)
    cfg, _, keep = W.build(lm, spec)
    m = cfg.sample.layers[0].medium
    d, s1, s2 = O.Oracle(spec).amp_table(0)
    assert d == m._dtheta
    np.testing.assert_array_equal(s1, m._s1)
    np.testing.assert_array_equal(s2, m._s2)
    for th in np.linspace(0, math.pi, 31):
        S = m.scattering_matrix(th, 0.0)
        i = min(int(th / d), s1.size - 2)
        assert abs(S[1, 1]) <= np.abs(s1).max() * 1.0001 + 1e-30


def test_mie_matches_oracle_restatement():
    mu = np.cos(np.linspace(0, math.pi, 101))
    for x, m in [(4.96, 1.59 / 1.33), (0.05, 1.3), (20.0, 1.33), (10.0, 1.5 - 0.1j)]:
        s1, s2, (qe, qs, g) = lm.core._mie_at(x, complex(m), mu)
        o1, o2, (oe, os_, og) = O.mie(x, complex(m), mu)
        np.testing.assert_allclose(s1, o1, rtol=0, atol=1e-13 * np.abs(o1).max())
        np.testing.assert_allclose(s2, o2, rtol=0, atol=1e-13 * np.abs(o2).max())
        assert qe == pytest.approx(oe, rel=1e-13) and qs == pytest.approx(os_, rel=1e-13)
        assert g == pytest.approx(og, rel=1e-12)


def test_hg_half_angle_form_matches_reference_inverse_cdf():
    """The binary32 kernel samples HG through 1 -/+ cos(theta) (no cancellation);
    in exact arithmetic it is the reference's closed form (src/phase.cpp:108-115)."""
    for g in (0.8, 0.9, -0.5, 0.3):
        for u in np.linspace(1e-4, 1 - 1e-4, 41):
            d = 1 - g + 2 * g * u
            frac = (1 - g * g) / d
            ref = math.acos(max(-1.0, min(1.0, (1 + g * g - frac * frac) / (2 * g))))
            omc = (1 - g) * (1 - u) * (1 - g + frac) / d
            opc = (1 + g) * u * (1 + g + frac) / d
            assert 2 * math.atan2(math.sqrt(omc), math.sqrt(opc)) == pytest.approx(ref, abs=1e-7)


def test_mie_tables_rejects_bad_arguments_before_any_device_work():
    """lmc_mie_tables validates its arguments on the host (no GPU needed to refuse)."""
    sp = (N.MieSpecies * 1)(N.MieSpecies(0.633e-3, 0.5e-3, 1.59, 1.33))
    v, c, s = np.zeros(11), np.zeros(11), np.zeros(1)
    a, b = np.zeros(20), np.zeros(20)
    L = N.lib()
    assert L.lmc_mie_tables(sp, 1, 0, 0.0, 1.0, 10, N.as_dptr(v), N.as_dptr(c), N.as_dptr(s),
                            N.as_dptr(a), N.as_dptr(b), None) == N.LMC_ERR_INVALID
    assert L.lmc_mie_tables(sp, 1, 10, 1.0, 1.0, 10, N.as_dptr(v), N.as_dptr(c), N.as_dptr(s),
                            N.as_dptr(a), N.as_dptr(b), None) == N.LMC_ERR_INVALID
    assert L.lmc_mie_tables(sp, 1, 10, 0.0, 1.0, 1, None, None, None,
                            N.as_dptr(a), N.as_dptr(b), None) == N.LMC_ERR_INVALID
    assert L.lmc_mie_tables(sp, 1, 10, 0.0, 1.0, 10, N.as_dptr(v), None, N.as_dptr(s),
                            None, None, None) == N.LMC_ERR_INVALID
    bad = (N.MieSpecies * 1)(N.MieSpecies(0.0, 0.5e-3, 1.59, 1.33))
    assert L.lmc_mie_tables(bad, 1, 10, 0.0, 1.0, 10, N.as_dptr(v), N.as_dptr(c), N.as_dptr(s),
                            N.as_dptr(a), N.as_dptr(b), None) == N.LMC_ERR_INVALID
    assert "wavelength" in N.last_error()
    with pytest.raises(ValueError):
        lm.mie_species([(0.633e-3, 0.5e-3, 1.59, 1.33)], 0)


def test_build_mie_sweep_refuses_other_specs():
    """workloads.build_mie_sweep batches single-medium Mie specs only, on one node grid."""
    spec = W.mie_sweep(0)
    other = W.bilayer_rgd_mie(10, 1)
    with pytest.raises(ValueError, match="single-medium Mie"):
        W.build_mie_sweep(lm, [spec, other])
    grid = W.mie_sweep(1)
    grid["phases"][0]["nDiv"] = 500
    with pytest.raises(ValueError, match="nDiv"):
        W.build_mie_sweep(lm, [spec, grid])
    mismatch = W.mie_sweep(2)
    mismatch["media"][0]["radius"] *= 2
    with pytest.raises(ValueError, match="same particle"):
        W.build_mie_sweep(lm, [mismatch])


def test_python_default_stream_maps_to_the_legacy_stream():
    """A NULL lmc_run_opts.stream selects the handle's own non-blocking stream; the Python
    layer passes the legacy default stream for None and for torch's default-stream handle 0
    (so runs are ordered with torch's default-stream work) and other handles as given."""
    assert N.launch_stream(None) == N.CUDA_STREAM_LEGACY == 1
    assert N.launch_stream(0) == N.CUDA_STREAM_LEGACY
    assert N.launch_stream(12345) == 12345
