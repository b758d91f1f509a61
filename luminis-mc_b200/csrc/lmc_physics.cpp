// lmc_physics.cpp -- set-up-time physics of the photon-propagation path (host).
//
// Everything the reference computes when a PhaseFunction or ScatteringMedium is
// constructed: Mie coefficients and amplitudes (Wiscombe's MIEV0 method, the
// reference's src/mie/MIEV0noP.f), the phase functions' PDFs and their
// inverse-CDF SamplingTables (src/phase.cpp, src/table.cpp:6-48) and the
// amplitude DataTables of RGDMedium / MieMedium (src/medium.cpp:77-236).
//
// The Mie series here is organised as two passes -- coefficients a_n, b_n for a
// size parameter once, then the angular sums for any number of cosines -- which
// gives the same numbers as the reference's per-node calls (each call repeats
// the identical coefficient recurrence).  The recurrences, the term count and
// the up/down choice for the log-derivative follow Wiscombe's published method
// (NCAR TN-140, eqs. R16-R50), which MIEV0 implements.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "luminis_b200.h"
#include "lmc_internal.h"

namespace {

using cd = std::complex<double>;

struct MieCoefficients {
  int ntrm = 0;
  bool small = false;                    // two-term small-particle limit (R40-R42)
  std::vector<cd> an, bn;                // 1-based, an[0] unused
  double qext = 0, qsca = 0, gqsc = 0;
  cd small_a1, small_a2, small_b1;       // small-particle limit coefficients (x^3 missing)
  double small_rtmp = 0;
  bool conj_out = false;
};

// Lentz continued fraction for the log-derivative A_N(z), 1/z = zinv (R25-R35).
cd lentz_a(int n, cd zinv, bool *ok)
{
  const double eps1 = 1.e-2, eps2 = 1.e-8;
  cd value = double(n + 1) * zinv;
  int sign = -1;
  int k = 2 * n + 3;
  cd ak = double(sign * k) * zinv;
  cd den = ak;
  cd num = den + 1.0 / value;
  for (int it = 1; it <= 10000; ++it) {
    sign = -sign;
    k += 2;
    ak = double(sign * k) * zinv;
    if (std::abs(num / ak) <= eps1 || std::abs(den / ak) <= eps1) {
      const cd ntn = ak * num + 1.0;
      const cd dtd = ak * den + 1.0;
      value = (ntn / dtd) * value;
      sign = -sign;
      k += 2;
      ak = double(sign * k) * zinv;
      num = ak + num / ntn;
      den = ak + den / dtd;
      ++it;
      continue;
    }
    const cd capt = num / den;
    value = capt * value;
    if (std::fabs(capt.real() - 1.0) < eps2 && std::fabs(capt.imag()) < eps2) {
      *ok = true;
      return value;
    }
    num = ak + 1.0 / num;
    den = ak + 1.0 / den;
  }
  *ok = false;
  return value;
}

bool mie_coefficients(double x, cd m_in, bool any_angles, MieCoefficients &c)
{
  cd m = m_in;
  c.conj_out = m_in.imag() > 0.0;
  if (m.imag() > 0.0)
    m = std::conj(m);
  const double mre = m.real();
  const double mim = -m.imag();
  const bool noabs = mim <= 1e-8;

  if (x * std::max(1.0, std::abs(m)) <= 0.1) {                   // small-particle limit
    c.small = true;
    const cd m2 = m * m;
    const cd ct = cd(0., 2. / 3.) * (m2 - 1.0);
    const double x2 = x * x, x3 = x2 * x, x4 = x2 * x2;
    c.small_a1 = ct * (1. - 0.1 * x2 + (m2 / 350. + 1. / 280.) * x4) /
                 (m2 + 2. + (1. - 0.7 * m2) * x2 - (m2 * m2 / 175. - 0.275 * m2 + 0.25) * x4 +
                  x3 * ct * (1. - 0.1 * x2));
    c.small_b1 = (x2 / 30.) * ct * (1. + (m2 / 35. - 1. / 14.) * x2) / (1. - (m2 / 15. - 1. / 6.) * x2);
    c.small_a2 = (0.1 * x2) * ct * (1. - x2 / 14.) / (2. * m2 + 3. - (m2 / 7. - 0.5) * x2);
    const double five3 = 5. / 3.;
    c.qsca = (6. * x4) * (std::norm(c.small_a1) + std::norm(c.small_b1) + five3 * std::norm(c.small_a2));
    c.qext = (mim > 1e-8) ? 6. * x * (c.small_a1 + c.small_b1 + five3 * c.small_a2).real() : c.qsca;
    c.gqsc = (6. * x4) * (c.small_a1 * std::conj(c.small_a2 + c.small_b1)).real();
    c.small_rtmp = 1.5 * x3;
    return true;
  }

  int ntrm;
  if (x <= 8.0)
    ntrm = int(x + 4. * std::pow(x, 1. / 3.) + 1.);
  else if (x < 4200.)
    ntrm = int(x + 4.05 * std::pow(x, 1. / 3.) + 2.);
  else
    ntrm = int(x + 4. * std::pow(x, 1. / 3.) + 2.);
  if (ntrm + 1 > 10100)
    return false;
  c.ntrm = ntrm;

  // log-derivative A_n(m x), n = 1..ntrm (R20-R23, choice R47-R48)
  std::vector<double> ra(ntrm + 1, 0.0);
  std::vector<cd> ca(ntrm + 1, 0.0);
  bool down;
  if (mre < 1.0 || mre > 10.0 || mim > 10.0) {
    down = true;
  } else if (any_angles) {
    down = !(mim * x < 3.9 + mre * (-10.8 + 13.78 * mre));
  } else {
    down = !(mim * x < -8.0 + mre * mre * (26.22 + mre * (-0.4474 + mre * mre * mre *
                                                                     (0.00204 - 0.000175 * mre))));
  }
  const cd zinv = 1.0 / (m * x);
  const double rezinv = 1.0 / (mre * x);
  if (down) {
    bool ok = false;
    const cd top = lentz_a(ntrm, zinv, &ok);
    if (!ok)
      return false;
    if (noabs) {
      ra[ntrm] = top.real();
      for (int n = ntrm; n >= 2; --n)
        ra[n - 1] = (n * rezinv) - 1.0 / ((n * rezinv) + ra[n]);
    } else {
      ca[ntrm] = top;
      for (int n = ntrm; n >= 2; --n)
        ca[n - 1] = (double(n) * zinv) - 1.0 / ((double(n) * zinv) + ca[n]);
    }
  } else if (noabs) {
    const double s = std::sin(mre * x);
    ra[1] = -rezinv + s / (s * rezinv - std::cos(mre * x));
    for (int n = 2; n <= ntrm; ++n)
      ra[n] = -(n * rezinv) + 1.0 / ((n * rezinv) - ra[n - 1]);
  } else {
    const cd e = std::exp(cd(0., -2.) * m * x);
    ca[1] = -zinv + (1. - e) / (zinv * (1. - e) - cd(0., 1.) * (1. + e));
    for (int n = 2; n <= ntrm; ++n)
      ca[n] = -(double(n) * zinv) + 1.0 / ((double(n) * zinv) - ca[n - 1]);
  }

  // Riccati-Bessel upward recurrence (R17, R19) and the coefficients (R16)
  const double xinv = 1.0 / x;
  double psi_prev = std::sin(x);
  const double chi_prev = std::cos(x);
  double psi = psi_prev * xinv - chi_prev;
  const double chi = chi_prev * xinv + psi_prev;
  cd zeta_prev(psi_prev, chi_prev), zeta(psi, chi);
  const cd minv = 1.0 / m;
  const double mreinv = 1.0 / mre;
  c.an.assign(ntrm + 1, 0.0);
  c.bn.assign(ntrm + 1, 0.0);
  double qs = 0.0, gq = 0.0;
  cd sf = 0.0;
  cd a_prev = 0.0, b_prev = 0.0;
  for (int n = 1; n <= ntrm; ++n) {
    const double fn = n;
    const double twonp1 = 2 * n + 1;
    cd a, b;
    if (noabs) {
      a = ((mreinv * ra[n] + (fn * xinv)) * psi - psi_prev) /
          ((mreinv * ra[n] + (fn * xinv)) * zeta - zeta_prev);
      b = ((mre * ra[n] + (fn * xinv)) * psi - psi_prev) /
          ((mre * ra[n] + (fn * xinv)) * zeta - zeta_prev);
    } else {
      a = ((minv * ca[n] + (fn * xinv)) * psi - psi_prev) /
          ((minv * ca[n] + (fn * xinv)) * zeta - zeta_prev);
      b = ((m * ca[n] + (fn * xinv)) * psi - psi_prev) / ((m * ca[n] + (fn * xinv)) * zeta - zeta_prev);
      qs = qs + twonp1 * (std::norm(a) + std::norm(b));
    }
    sf = sf + twonp1 * (a + b);
    gq = gq + (fn - 1.0 / fn) * (a_prev * std::conj(a) + b_prev * std::conj(b)).real() +
         (twonp1 / (fn * (n + 1))) * (a * std::conj(b)).real();
    c.an[n] = a;
    c.bn[n] = b;
    a_prev = a;
    b_prev = b;
    const cd znext = (twonp1 * xinv) * zeta - zeta_prev;
    zeta_prev = zeta;
    zeta = znext;
    psi_prev = psi;
    psi = zeta.real();
  }
  c.qext = 2. / (x * x) * sf.real();
  c.qsca = noabs ? c.qext : 2. / (x * x) * qs;
  c.gqsc = 4. / (x * x) * gq;
  return true;
}

// S1, S2 at cosine mu from precomputed coefficients (R10-R11, R37-R39).
void mie_amplitudes(const MieCoefficients &c, double mu, cd &s1, cd &s2)
{
  if (c.small) {
    const double five3 = 5. / 3.;
    s1 = c.small_rtmp * (c.small_a1 + (c.small_b1 + five3 * c.small_a2) * mu);
    s2 = c.small_rtmp * (c.small_b1 + c.small_a1 * mu + five3 * c.small_a2 * (2. * mu * mu - 1.));
  } else {
    double pi_prev = 0.0, pi_n = 1.0;
    cd sp = 0.0, sm = 0.0;
    for (int n = 1; n <= c.ntrm; ++n) {
      const double fn = n;
      const double coeff = (2 * n + 1) / (fn * (n + 1));
      const cd ap = coeff * (c.an[n] + c.bn[n]);
      const cd bp = coeff * (c.an[n] - c.bn[n]);
      const double r = (mu * pi_n) - pi_prev;
      const double tau = fn * r - pi_prev;
      sp = sp + ap * (pi_n + tau);
      sm = sm + bp * (pi_n - tau);
      pi_prev = pi_n;
      pi_n = (mu * pi_n) + (1.0 + 1.0 / fn) * r;
    }
    s1 = 0.5 * (sp + sm);
    s2 = 0.5 * (sp - sm);
  }
  if (c.conj_out) {
    s1 = std::conj(s1);
    s2 = std::conj(s2);
  }
}

double form_factor(double theta, double k, double radius)       // src/phase.cpp:10-20
{
  if (std::fabs(theta) == 0.0)
    return 1.0;
  const double u = 2.0 * k * radius * std::sin(theta / 2.0);
  return 3 * (std::sin(u) - u * std::cos(u)) / std::pow(u, 3);
}

// RD-EMC scattering efficiency by composite Simpson over [0, pi], N = 100000
// (src/phase.cpp:168-195).
double rdemc_cross_section(const lmc_phase_params &p)
{
  const double k = 2 * M_PI * p.n_medium / p.wavelength;
  const double r = p.radius;
  const double x = r * k;
  const double V = 4 * M_PI * std::pow(r, 3) / 3.0;
  const double a = (std::pow(k, 6) * std::pow((p.n_particle / p.n_medium - 1.0), 2) * V * V) /
                   (4 * std::pow(M_PI, 2));
  const double c = a / std::pow(x, 2);
  const int N = 100000;
  const double h = M_PI / N;
  auto f = [&](double t) {
    const double F = form_factor(t, k, r);
    const double ct = std::cos(t);
    return F * F * std::sin(t) * (1.0 + ct * ct);
  };
  double sum = f(0.0) + f(M_PI);
  for (int i = 1; i < N; i += 2)
    sum += 4.0 * f(i * h);
  for (int i = 2; i < N; i += 2)
    sum += 2.0 * f(i * h);
  return c * (sum * h / 3.0) * (M_PI * std::pow(r, 2));
}

}  // namespace

bool lmc::mie_series(double x, double m_re, double m_im, MieSeries &out)
{
  MieCoefficients c;
  if (!mie_coefficients(x, cd(m_re, m_im), true, c))
    return false;
  out.conj_out = c.conj_out;
  out.qsca = c.qsca;
  if (c.small) {
    out.ntrm = 0;
    out.small_rtmp = c.small_rtmp;
    out.small_a1 = c.small_a1;
    out.small_a2 = c.small_a2;
    out.small_b1 = c.small_b1;
    return true;
  }
  out.ntrm = c.ntrm;
  out.ap.resize(c.ntrm);
  out.bp.resize(c.ntrm);
  for (int n = 1; n <= c.ntrm; ++n) {           // as in mie_amplitudes
    const double fn = n;
    const double coeff = (2 * n + 1) / (fn * (n + 1));
    out.ap[n - 1] = coeff * (c.an[n] + c.bn[n]);
    out.bp[n - 1] = coeff * (c.an[n] - c.bn[n]);
  }
  return true;
}

extern "C" {

lmc_status lmc_mie(double x, double m_re, double m_im, int n, const double *mu, double *s1,
                   double *s2, double *qext, double *qsca, double *g)
{
  if (!(x >= 0.0) || !(m_re > 0.0) || n < 0 || (n > 0 && (!mu || !s1 || !s2)))
    return lmc::fail(LMC_ERR_INVALID, "lmc_mie: invalid arguments");
  MieCoefficients c;
  if (!mie_coefficients(x, cd(m_re, m_im), true, c))
    return lmc::fail(LMC_ERR_INVALID, "lmc_mie: series did not converge or needs too many terms");
  for (int i = 0; i < n; ++i) {
    cd a, b;
    mie_amplitudes(c, mu[i], a, b);
    s1[2 * i] = a.real();
    s1[2 * i + 1] = a.imag();
    s2[2 * i] = b.real();
    s2[2 * i + 1] = b.imag();
  }
  if (qext) *qext = c.qext;
  if (qsca) *qsca = c.qsca;
  if (g) *g = c.gqsc / c.qsca;
  return LMC_OK;
}

lmc_status lmc_phase_cross_section(const lmc_phase_params *p, double *sigma_s)
{
  if (!p || !sigma_s)
    return lmc::fail(LMC_ERR_INVALID, "lmc_phase_cross_section: null argument");
  if (p->kind == LMC_PDF_RDEMC) {
    *sigma_s = rdemc_cross_section(*p);
    return LMC_OK;
  }
  if (p->kind == LMC_PDF_MIE) {                                   // src/phase.cpp:270-284
    const double k = 2 * M_PI * p->n_medium / p->wavelength;
    MieCoefficients c;
    if (!mie_coefficients(p->radius * k, cd(p->n_particle / p->n_medium, 0.0), true, c))
      return lmc::fail(LMC_ERR_INVALID, "Mie series failed");
    *sigma_s = c.qsca * (M_PI * std::pow(p->radius, 2));
    return LMC_OK;
  }
  return lmc::fail(LMC_ERR_UNSUPPORTED,
                   "scattering_cross_section is not implemented for this phase function");
}

lmc_status lmc_sampling_table(const lmc_phase_params *p, int n_div, double min_val,
                              double max_val, double *values, double *cdf)
{
  if (!p || !values || !cdf)
    return lmc::fail(LMC_ERR_INVALID, "lmc_sampling_table: null argument");
  if (n_div <= 0)
    return lmc::fail(LMC_ERR_INVALID, "nDiv must be greater than 0");
  if (min_val >= max_val)
    return lmc::fail(LMC_ERR_INVALID, "minVal must be less than maxVal");
  std::vector<double> pdf(size_t(n_div) + 1);
  double k = 0.0, sigma = 0.0;
  MieCoefficients mc;
  switch (p->kind) {
  case LMC_PDF_RAYLEIGH:
  case LMC_PDF_DRAINE:
    break;
  case LMC_PDF_RD:
    k = 2 * M_PI / p->wavelength;
    break;
  case LMC_PDF_RDEMC:
    k = 2 * M_PI * p->n_medium / p->wavelength;
    sigma = rdemc_cross_section(*p);
    break;
  case LMC_PDF_MIE:
    k = 2 * M_PI * p->n_medium / p->wavelength;
    if (!mie_coefficients(k * p->radius, cd(p->n_particle / p->n_medium, 0.0), true, mc))
      return lmc::fail(LMC_ERR_INVALID, "Mie series failed");
    sigma = mc.qsca * (M_PI * std::pow(p->radius, 2));
    break;
  default:
    return lmc::fail(LMC_ERR_INVALID, "lmc_sampling_table: unknown pdf kind");
  }
  auto pdf_at = [&](double x) -> double {
    switch (p->kind) {
    case LMC_PDF_RAYLEIGH:                                        // src/phase.cpp:96-98
      return 0.375 * (1.0 + x * x);
    case LMC_PDF_RD: {                                            // src/phase.cpp:138-142
      const double F = form_factor(x, k, p->radius);
      return (1.0 / (4.0 * M_PI)) * std::pow(F, 2);
    }
    case LMC_PDF_RDEMC: {                                         // src/phase.cpp:202-214
      const double m1 = (p->n_particle / p->n_medium) - 1.0;
      const double v = (4.0 / 3.0) * M_PI * std::pow(p->radius, 3);
      const double F = form_factor(x, k, p->radius);
      const double rho = (std::pow(k, 4) / (4.0 * M_PI * sigma)) * m1 * m1 * v * v * F * F *
                         (1.0 + std::cos(x) * std::cos(x));
      return rho * std::sin(x);
    }
    case LMC_PDF_DRAINE: {                                        // src/phase.cpp:236-240
      const double g = p->g, a = p->a;
      const double hg = (1.0 - g * g) / std::pow(1.0 + g * g - 2.0 * g * x, 1.5);
      const double dr = (1.0 + a * x * x) / (3 + a * (1 + 2 * g * g));
      return (1.0 / 4.0 * M_PI) * hg * dr;
    }
    default: {                                                    // Mie, src/phase.cpp:286-304
      double mu = std::cos(x);
      mu = std::min(1.0, std::max(-1.0, mu));
      cd s1, s2;
      mie_amplitudes(mc, mu, s1, s2);
      return (M_PI / (k * k * sigma)) * (std::norm(s1) + std::norm(s2)) * std::sin(x);
    }
    }
  };
  // rectangle-rule CDF normalised to end at 1 (src/table.cpp:19-47)
  const double step = (max_val - min_val) / n_div;
  double sum = 0.0;
  for (int i = 0; i <= n_div; ++i) {
    values[i] = min_val + i * step;
    pdf[i] = pdf_at(values[i]);
    sum += pdf[i] * step;
  }
  for (int i = 0; i <= n_div; ++i)
    pdf[i] /= sum;
  cdf[0] = pdf[0] * step;
  for (int i = 1; i <= n_div; ++i)
    cdf[i] = cdf[i - 1] + pdf[i] * step;
  const double last = cdf[n_div];
  for (int i = 0; i <= n_div; ++i)
    cdf[i] /= last;
  for (int i = 0; i <= n_div; ++i)
    if (!std::isfinite(cdf[i]))
      return lmc::fail(LMC_ERR_INVALID, "phase-function CDF is not finite");
  return LMC_OK;
}

lmc_status lmc_amplitude_table(int kind, double radius, double n_particle, double n_medium,
                               double wavelength, int n, double *s1, double *s2)
{
  if (n < 2 || !s1 || !s2 || !(wavelength > 0.0) || !(n_medium > 0.0))
    return lmc::fail(LMC_ERR_INVALID, "lmc_amplitude_table: invalid arguments");
  const double dtheta = M_PI / double(n - 1);
  if (kind == LMC_AMP_RGD) {                                      // src/medium.cpp:77-120
    const double k = 2 * M_PI * n_medium / wavelength;
    const double volume = 4.0 * M_PI * (radius * radius * radius) / 3.0;
    const double pref = -1.0 * (k * k * k) * ((n_particle / n_medium) - 1.0) * volume / (2.0 * M_PI);
    for (int i = 0; i < n; ++i) {
      const double theta = double(i) * dtheta;
      const double F = form_factor(theta, k, radius);
      s1[2 * i] = 0.0;
      s1[2 * i + 1] = pref * F;
      s2[2 * i] = 0.0;
      s2[2 * i + 1] = pref * F * std::cos(theta);
    }
    return LMC_OK;
  }
  if (kind == LMC_AMP_MIE) {                                      // src/medium.cpp:160-236
    MieCoefficients c;
    if (!mie_coefficients(2 * M_PI * radius / wavelength, cd(n_particle / n_medium, 0.0), true, c))
      return lmc::fail(LMC_ERR_INVALID, "Mie series failed");
    for (int i = 0; i < n; ++i) {
      cd a, b;
      mie_amplitudes(c, std::cos(double(i) * dtheta), a, b);
      s1[2 * i] = a.real();
      s1[2 * i + 1] = a.imag();
      s2[2 * i] = b.real();
      s2[2 * i + 1] = b.imag();
    }
    return LMC_OK;
  }
  return lmc::fail(LMC_ERR_INVALID, "lmc_amplitude_table: unknown medium kind");
}

}  // extern "C"
