"""Statistical comparison of two Monte Carlo tallies from independent random streams.

Each side is summarised per bin by the mean and the sample variance of tally / N
over R independent-seed replicas, as the reference's own convergence studies do
(results/study_estimator_vs_analog/study_estimator_vs_analog__PCIR.py:126-140).
Two runs of the same analog estimator then agree bin by bin: Welch's
t = (m_a - m_b) / sqrt(v_a / R_a + v_b / R_b) is close to standard normal, and the
per-photon variances v * N (the tally sigma at equal photon count) are equal.

Bins are tested where both sides are well populated (relative standard error of
the mean below `max_rse` on each side); sparse bins have skewed, discrete
replica distributions for which the normal approximation does not hold.
"""
from __future__ import annotations

import numpy as np


def moments(tallies_by_replica, n_photons):
    """[(mean, var)] per sensor from R replicas' tally lists (var with ddof=1)."""
    out = []
    for sensor in zip(*tallies_by_replica):
        x = np.stack([np.asarray(t, dtype=np.float64) / n_photons for t in sensor])
        out.append((x.mean(axis=0), x.var(axis=0, ddof=1)))
    return out


def compare(a_mean, a_var, a_R, a_N, b_mean, b_var, b_R, b_N, max_rse=0.25):
    """Welch t per well-populated bin and the per-photon variance ratio there.
    max_rse=None tests every bin that scored on both sides: for signed, zero-mean
    quantities (speckle fields) whose bins are all crossed by many photons."""
    a_mean, a_var = np.ravel(a_mean), np.ravel(a_var)
    b_mean, b_var = np.ravel(b_mean), np.ravel(b_var)
    se_a = np.sqrt(a_var / a_R)
    se_b = np.sqrt(b_var / b_R)
    with np.errstate(divide="ignore", invalid="ignore"):
        rse_a = se_a / np.abs(a_mean)
        rse_b = se_b / np.abs(b_mean)
        ok = (a_var > 0) & (b_var > 0)
        if max_rse is not None:
            ok &= (rse_a < max_rse) & (rse_b < max_rse)
        t = (a_mean - b_mean) / np.sqrt(se_a ** 2 + se_b ** 2)
        ratio = (a_var * a_N) / (b_var * b_N)
    # bins where neither side ever scored must be zero on both
    both_silent = (a_var == 0) & (b_var == 0)
    return {
        "t": t[ok],
        "var_ratio": ratio[ok],
        "n_tested": int(ok.sum()),
        "n_bins": int(a_mean.size),
        "silent_mismatch": int(np.sum(both_silent & (a_mean != b_mean))),
    }


def assert_agree(res, what, max_abs_t=6.0, max_frac_over_3=0.05, t2_range=(0.6, 1.8),
                 var_ratio_range=(0.8, 1.25), min_tested=20):
    """Bars: no |t| above max_abs_t, at most max_frac_over_3 of bins beyond 3 sigma,
    mean t^2 in t2_range, median per-photon variance ratio in var_ratio_range (equal
    tally sigma at equal N).  For a normal t these would be 0.27 % and 1; the bars are
    wider because the variances are estimated from 16 replicas (Student tails,
    E[t^2] ~ 1.1), the population cut favours bins whose variance came out low, and
    the 8 Stokes grids of one angular bin see the same photons, so their t values
    move together.  Calibrated on independent seed sets of the oracle against the
    reference (mean t^2 0.83-1.50, max |t| <= 4.8, <= 3.2 % beyond 3 sigma)."""
    t = res["t"]
    assert res["n_tested"] >= min_tested, f"{what}: only {res['n_tested']} bins populated"
    assert res["silent_mismatch"] == 0, f"{what}: bins scored on one side only"
    worst = float(np.max(np.abs(t)))
    frac = float(np.mean(np.abs(t) > 3.0))
    t2 = float(np.mean(t ** 2))
    vr = float(np.median(res["var_ratio"]))
    assert worst <= max_abs_t, f"{what}: max |t| = {worst:.2f} over {res['n_tested']} bins"
    assert frac <= max_frac_over_3, f"{what}: {100 * frac:.2f}% of bins beyond 3 sigma"
    assert t2_range[0] <= t2 <= t2_range[1], f"{what}: mean t^2 = {t2:.3f}"
    assert var_ratio_range[0] <= vr <= var_ratio_range[1], \
        f"{what}: median per-photon variance ratio {vr:.3f}"
    return {"max_abs_t": worst, "frac_over_3": frac, "mean_t2": t2, "median_var_ratio": vr,
            "n_tested": res["n_tested"], "n_bins": res["n_bins"]}
