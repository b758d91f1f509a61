"""The oracle pinned against the reference: MIEV0's built-in known answers, an
independent Mie series, the Philox known-answer vectors, and the golden tallies
the reference itself produced (tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest
from scipy import special

from oracle import philox_ref_kat as KAT  # noqa: F401  (import check only)
from oracle import pyoracle as O
from tests.golden.make_golden import golden_scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_miev0_selftest_known_answers():
    """TESTMI (src/mie/MIEV0noP.f:1182-1300): x=10, m=1.5-0.1i, 140 deg at 1e-4."""
    ok, worst = O.miev0_selftest()
    assert ok and worst < 1e-4


def mie_scipy(x, m, mu):
    """Bohren-Huffman series with scipy's spherical Bessel functions (independent).
    Bohren-Huffman use exp(-i w t); MIEV0 uses exp(+i w t), so its amplitudes are the
    complex conjugates of these."""
    nmax = int(x + 4 * x ** (1 / 3) + 2) + 10
    n = np.arange(1, nmax + 1)
    mx = m * x
    jx, yx = special.spherical_jn(n, x), special.spherical_yn(n, x)
    jmx = special.spherical_jn(n, mx)
    djx = special.spherical_jn(n, x, derivative=True)
    dyx = special.spherical_yn(n, x, derivative=True)
    djmx = special.spherical_jn(n, mx, derivative=True)
    psi, dpsi = x * jx, jx + x * djx
    xi, dxi = x * (jx + 1j * yx), (jx + 1j * yx) + x * (djx + 1j * dyx)
    psim, dpsim = mx * jmx, jmx + mx * djmx
    a = (m * psim * dpsi - psi * dpsim) / (m * psim * dxi - xi * dpsim)
    b = (psim * dpsi - m * psi * dpsim) / (psim * dxi - m * xi * dpsim)
    s1 = np.zeros(mu.size, complex)
    s2 = np.zeros(mu.size, complex)
    for i, u in enumerate(mu):
        pi = np.zeros(nmax + 1)
        tau = np.zeros(nmax + 1)
        pi[1] = 1.0
        tau[1] = u
        if nmax > 1:
            pi[2] = 3 * u
            tau[2] = 2 * u * pi[2] - 3
        for k in range(3, nmax + 1):
            pi[k] = ((2 * k - 1) * u * pi[k - 1] - k * pi[k - 2]) / (k - 1)
            tau[k] = k * u * pi[k] - (k + 1) * pi[k - 1]
        c = (2 * n + 1) / (n * (n + 1))
        s1[i] = np.sum(c * (a * pi[1:] + b * tau[1:]))
        s2[i] = np.sum(c * (a * tau[1:] + b * pi[1:]))
    return np.conj(s1), np.conj(s2)


@pytest.mark.parametrize("x,m", [(4.96, 1.59 / 1.33), (6.6, 1.59 / 1.33), (0.5, 1.2),
                                 (26.0, 1.19), (10.0, 1.5)])
def test_mie_restatement_matches_independent_series(x, m):
    mu = np.cos(np.linspace(0, np.pi, 37))
    s1, s2, _ = O.mie(x, complex(m, 0.0), mu)
    r1, r2 = mie_scipy(x, m, mu)
    scale = max(np.abs(r1).max(), np.abs(r2).max())
    # MIEV0 stops the series after x + 4 x^(1/3) + 1 terms (MIEV0noP.f:177-189);
    # at x = 0.5 that is 4 terms and leaves ~3e-9 of truncation, which the
    # reference inherits, so the bound is 1e-8 rather than round-off.
    assert np.abs(s1 - r1).max() < 1e-8 * scale
    assert np.abs(s2 - r2).max() < 1e-8 * scale


def _golden(kind, name):
    return dict(np.load(os.path.join(GOLDEN, f"ref_{kind}_{name}.npz")))


@pytest.mark.parametrize("spec", golden_scenes(), ids=lambda s: s["name"])
def test_oracle_reproduces_reference_tallies_bit_for_bit(spec):
    """The C restatement with the reference's own xoshiro streams gives the
    reference's tallies exactly (both built with -ffp-contract=off, 1 thread)."""
    g = _golden("xoshiro", spec["name"])
    res = O.Oracle(spec).run(spec["n_photons"], spec["seed"], rng="xoshiro")
    for i, t in enumerate(res.tallies):
        np.testing.assert_array_equal(t, g[f"sensor{i}"])
    np.testing.assert_array_equal(res.hits.astype(np.int64), g["hits"])


@pytest.mark.parametrize("spec", golden_scenes(), ids=lambda s: s["name"])
def test_oracle_reproduces_reference_on_philox_stream(spec):
    """The unmodified reference drawing the GPU's Philox stream through the replay
    seam (oracle/replay_rng.cpp) equals the oracle's Philox mode."""
    g = _golden("philox", spec["name"])
    res = O.Oracle(spec).run(spec["n_photons"], spec["seed"], rng="philox_u53")
    for i, t in enumerate(res.tallies):
        np.testing.assert_array_equal(t, g[f"sensor{i}"])
    np.testing.assert_array_equal(res.hits.astype(np.int64), g["hits"])


def test_golden_meta_lists_every_fixture():
    meta = json.load(open(os.path.join(GOLDEN, "golden_meta.json")))
    for name in meta["scenes"]:
        for kind in ("xoshiro", "philox"):
            assert os.path.exists(os.path.join(GOLDEN, f"ref_{kind}_{name}.npz"))


def test_philox_known_answers():
    from oracle.philox_ref_kat import KAT
    for ctr, key, out in KAT:
        assert O.philox(ctr, key) == out


def test_stream_contract():
    """u53: odd multiples of 2^-53 from the 64-bit words; u24: odd multiples of
    2^-24 from each 32-bit word; never 0 or 1 (include/luminis_b200.h)."""
    x = O.philox((0, 0, 7, 0), (123, 0))
    w0 = (x[1] << 32) | x[0]
    w1 = (x[3] << 32) | x[2]
    assert O.stream_uniform(123, 7, 0, "u53") == (2 * (w0 >> 12) + 1) * 2.0 ** -53
    assert O.stream_uniform(123, 7, 1, "u53") == (2 * (w1 >> 12) + 1) * 2.0 ** -53
    for j in range(4):
        assert O.stream_uniform(123, 7, j, "u24") == (2 * (x[j] >> 9) + 1) * 2.0 ** -24
    u = [O.stream_uniform(5, p, d, "u24") for p in range(50) for d in range(40)]
    assert 0.0 < min(u) and max(u) < 1.0


def test_farfield_fluence_pinned_by_reference_records():
    """The reference has no far-field fluence class: its definition (forward-field
    Stokes binned on exit angles) applied to the reference's own PhotonRecordSensor
    records on the Philox stream (tests/golden/ref_farfield_fluence_small.npz) equals
    the oracle's FarFieldFluence tally of the same photons."""
    from tests.golden.make_golden import farfield_scene
    spec = farfield_scene()
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden",
                               "ref_farfield_fluence_small.npz"))["sensor0"]
    got = O.Oracle(spec).run(spec["n_photons"], spec["seed"], rng="philox_u53").tallies[0]
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("name", ["estimator_mie", "estimator_bilayer"])
def test_oracle_estimator_reproduces_reference(name):
    """Estimator-mode FarFieldCBS (the last-flight CBS estimate at every vertex): the
    oracle's tallies and hit counts equal the reference's on the Philox stream
    (tests/golden/ref_philox_estimator_*.npz, made by the replay build)."""
    from tests.golden.make_golden import estimator_scenes
    spec = [s for s in estimator_scenes() if s["name"] == name][0]
    g = np.load(os.path.join(GOLDEN, f"ref_philox_{name}.npz"))
    res = O.Oracle(spec).run(spec["n_photons"], spec["seed"], rng="philox_u53")
    for i, t in enumerate(res.tallies):
        ref = g[f"sensor{i}"]
        np.testing.assert_allclose(t, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
        assert res.hits[i] == g["hits"][i]
