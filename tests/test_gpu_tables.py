"""Batched Mie set-up tables on the GPU (lmc_mie_tables, ``luminis_mc_b200.mie_species``).

Every table -- the MiePhaseFunction's sampling nodes and CDF and its scattering cross
section (src/phase.cpp:244-304, src/table.cpp:6-48), the MieMedium's S1 / S2 amplitude
tables (src/medium.cpp:160-236) -- must equal bit for bit the per-species host
construction, which the CPU suite pins against the reference's MIEV0 tables.  Species
cover the 256-medium sweep's size range (x up to ~26), the small-particle limit,
m < 1 (the log-derivative by downward recurrence) and other node grids.  A scene built
from batched tables transports to the same tallies as the one built species by species.
"""
import math

import numpy as np
import pytest

import luminis_mc_b200 as lm
from luminis_mc_b200 import workloads as W

pytestmark = pytest.mark.gpu

LAMBDA, N_SPHERE, N_WATER = 0.633e-3, 1.59, 1.33


def _species():
    r, _, _, _ = W.mie_sweep_parameters()
    out = [(LAMBDA, float(x), N_SPHERE, N_WATER) for x in r[:24]]
    out += [(LAMBDA, 0.005e-3, N_SPHERE, N_WATER),      # small-particle limit (x < 0.1)
            (LAMBDA, 0.012e-3, N_SPHERE, N_WATER),      # just above it
            (0.514e-3, 0.8e-3, 1.0, N_WATER),           # air bubble: m < 1
            (0.405e-3, 2.0e-3, 2.4, 1.0),               # high index in air, x ~ 31
            (LAMBDA, 2.0e-3, N_SPHERE, N_WATER)]        # largest sweep radius
    return out


def _assert_same(pairs, species, n_div, lo, hi):
    for (ph, med), (wl, r, n_p, n_m) in zip(pairs, species):
        ref_ph = lm.MiePhaseFunction(wl, r, n_p, n_m, n_div, lo, hi)
        ref_med = lm.MieMedium(ref_ph, r, n_p, n_m, wl)
        np.testing.assert_array_equal(ph._values, ref_ph._values)
        np.testing.assert_array_equal(ph._cdf, ref_ph._cdf, err_msg=f"cdf r={r}")
        assert ph.scattering_cross_section() == ref_ph.scattering_cross_section()
        np.testing.assert_array_equal(med._s1, ref_med._s1, err_msg=f"S1 r={r}")
        np.testing.assert_array_equal(med._s2, ref_med._s2, err_msg=f"S2 r={r}")
        assert med._dtheta == ref_med._dtheta
        for u in (1e-6, 0.3, 0.9, 1 - 1e-9):
            assert ph.sample_theta(u) == ref_ph.sample_theta(u)


def test_batched_tables_equal_per_species_construction(cuda):
    species = _species()
    pairs = lm.mie_species(species, 1000, 0.0, math.pi)
    assert len(pairs) == len(species)
    _assert_same(pairs, species, 1000, 0.0, math.pi)


def test_batched_tables_on_another_node_grid(cuda):
    species = _species()[::5]
    pairs = lm.mie_species(species, 357, 0.1, 3.0)
    _assert_same(pairs, species, 357, 0.1, 3.0)


def test_empty_batch_and_argument_errors(cuda):
    assert lm.mie_species([]) == []
    with pytest.raises(ValueError):
        lm.mie_species([(LAMBDA, 0.5e-3, N_SPHERE, N_WATER)], 0)
    with pytest.raises(ValueError):
        lm.mie_species([(LAMBDA, 0.5e-3, N_SPHERE, N_WATER)], 100, 1.0, 1.0)
    with pytest.raises(ValueError, match="not finite"):      # no scattering: CDF not finite
        lm.mie_species([(LAMBDA, 0.0, N_SPHERE, N_WATER)])
    with pytest.raises(ValueError, match="not finite"):
        lm.MiePhaseFunction(LAMBDA, 0.0, N_SPHERE, N_WATER, 1000, 0.0, math.pi)


def test_scene_from_batched_tables_transports_identically(cuda):
    specs = [W.mie_sweep(i, seed=77) for i in (3, 40, 101)]
    for sp in specs:
        sp["n_photons"] = 2000
    batched = W.build_mie_sweep(lm, specs)
    for sp, cfg_b in zip(specs, batched):
        cfg_h, hs_h, keep = W.build(lm, sp)
        lm.run_simulation_parallel(cfg_h, precision="fp64")
        lm.run_simulation_parallel(cfg_b, precision="fp64")
        for h, b in zip(cfg_h.detector.detectors, cfg_b.detector.detectors):
            np.testing.assert_array_equal(np.asarray(b._tally), np.asarray(h._tally))
            assert b.hits == h.hits
    lm.release_gpu_cache()
