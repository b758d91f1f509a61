/*
 * oracle/miev0.c -- TEST INFRASTRUCTURE (the oracle), never product code.
 *
 * C99 restatement of Wiscombe's MIEV0 (NoPMOM variant) as shipped by the
 * reference in src/mie/MIEV0noP.f, exporting the same Fortran-ABI symbol
 * `miev0_` that the reference's C++ wrapper src/mie/dmiev.cpp binds
 * (declaration: include/luminis/mie/dmiev.h:106).  The reference compiles the
 * Fortran with -fdefault-real-8 (CMakeLists.txt:38-39), so every REAL is a
 * C double and every COMPLEX a `double complex` here.  gfortran is absent in
 * this image, so this file is what lets the reference link (oracle/Makefile).
 *
 * Routines restated (file:line in src/mie/MIEV0noP.f):
 *   MIEV0  :2-510    series summation, S+/S- angular sums, efficiencies
 *   CKINMI :512-606  input checks
 *   BIGA   :608-745  log-derivative A_n (up/down recurrence choice, R47/R48)
 *   CONFRA :747-880  Lentz continued fraction for A_NTRM
 *   SMALL2 :1069-1180 small-particle limit, general refractive index
 *   TESTMI :1182-1330 built-in known-answer self-test (x=10, m=1.5-0.1i, 140 deg)
 * Not restated: the perfectly-conducting branch (PERFCT=.TRUE., SMALL1),
 * because every caller in the reference (src/mie/dmiev.cpp:9,28,52,71)
 * passes PERFCT=0; a non-zero PERFCT aborts with a message.
 *
 * The self-test runs on the first call exactly as the Fortran does (PASS1,
 * MIEV0noP.f:125-131,491-500) and aborts the process on a mismatch above
 * ACCUR = 1e-4.
 */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

typedef double complex cplx;

#define MIE_MAXTRM 10100   /* MIEV0noP.f:90 */
#define MIE_MAXANG 360001  /* MIEV0noP.f:86 */

static double sqc(cplx z) { return creal(z) * creal(z) + cimag(z) * cimag(z); }

static void mie_fatal(const char *msg)
{
  fprintf(stderr, "\n ****** ERROR *****  %s\n\n", msg);
  abort();
}

/* CONFRA, MIEV0noP.f:747-880: A_N(1/zinv) by the Lentz method. */
static cplx confra(int n, cplx zinv)
{
  const double eps1 = 1.e-2, eps2 = 1.e-8;
  const int maxit = 10000;
  cplx conf = (double)(n + 1) * zinv;             /* R25a */
  int mm = -1;
  int kk = 2 * n + 3;
  cplx cak = (double)(mm * kk) * zinv;            /* R25b, k=2 */
  cplx cdenom = cak;
  cplx cnumer = cdenom + 1.0 / conf;
  int kount = 1;
  for (;;) {
    kount++;
    if (kount > maxit)
      mie_fatal("ConFra--Iteration failed to converge");
    mm = -mm;
    kk += 2;
    cak = (double)(mm * kk) * zinv;               /* R25b */
    if (cabs(cnumer / cak) <= eps1 || cabs(cdenom / cak) <= eps1) {
      /* ill-conditioned: stride two terms (R32-R35) */
      cplx cntn = cak * cnumer + 1.0;
      cplx cdtd = cak * cdenom + 1.0;
      conf = (cntn / cdtd) * conf;
      mm = -mm;
      kk += 2;
      cak = (double)(mm * kk) * zinv;
      cnumer = cak + cnumer / cntn;
      cdenom = cak + cdenom / cdtd;
      kount++;
      continue;
    }
    cplx capt = cnumer / cdenom;                  /* R27 */
    conf = capt * conf;                           /* R26 */
    if (fabs(creal(capt) - 1.0) >= eps2 || fabs(cimag(capt)) >= eps2) {
      cnumer = cak + 1.0 / cnumer;                /* R30 */
      cdenom = cak + 1.0 / cdenom;
      continue;
    }
    return conf;
  }
}

/* BIGA, MIEV0noP.f:608-745: logarithmic derivatives A_1..A_ntrm (1-based). */
static void biga(cplx cior, double xx, int ntrm, int noabs, int yesang,
                 double *rbiga, cplx *cbiga)
{
  const double mre = creal(cior);
  const double mim = fabs(cimag(cior));
  int down;
  if (mre < 1.0 || mre > 10.0 || mim > 10.0) {
    down = 1;
  } else if (yesang) {
    const double f2 = 3.9 + mre * (-10.8 + 13.78 * mre);                 /* R47b */
    down = !(mim * xx < f2);                                              /* R48 */
  } else {
    const double f1 = -8.0 + mre * mre * (26.22 + mre * (-0.4474 + mre * mre * mre *
                                                          (0.00204 - 0.000175 * mre)));  /* R47c */
    down = !(mim * xx < f1);
  }
  const cplx zinv = 1.0 / (cior * xx);
  const double rezinv = 1.0 / (mre * xx);
  if (down) {
    const cplx ctmp = confra(ntrm, zinv);
    if (noabs) {                                  /* R23 */
      rbiga[ntrm] = creal(ctmp);
      for (int n = ntrm; n >= 2; --n)
        rbiga[n - 1] = (n * rezinv) - 1.0 / ((n * rezinv) + rbiga[n]);
    } else {
      cbiga[ntrm] = ctmp;
      for (int n = ntrm; n >= 2; --n)
        cbiga[n - 1] = ((double)n * zinv) - 1.0 / (((double)n * zinv) + cbiga[n]);
    }
  } else {
    if (noabs) {                                  /* R20, R21 */
      const double rtmp = sin(mre * xx);
      rbiga[1] = -rezinv + rtmp / (rtmp * rezinv - cos(mre * xx));
      for (int n = 2; n <= ntrm; ++n)
        rbiga[n] = -(n * rezinv) + 1.0 / ((n * rezinv) - rbiga[n - 1]);
    } else {                                      /* R20, R22 */
      const cplx ctmp = cexp(-2.0 * I * cior * xx);
      cbiga[1] = -zinv + (1.0 - ctmp) / (zinv * (1.0 - ctmp) - I * (1.0 + ctmp));
      for (int n = 2; n <= ntrm; ++n)
        cbiga[n] = -((double)n * zinv) + 1.0 / (((double)n * zinv) - cbiga[n - 1]);
    }
  }
}

/* SMALL2, MIEV0noP.f:1069-1180: two-term small-particle limit. */
static void small2(double xx, cplx cior, int calcqe, int numang, const double *xmu,
                   double *qext, double *qsca, double *gqsc, cplx *sforw, cplx *sback,
                   cplx *s1, cplx *s2, cplx *tforw, cplx *tback)
{
  const double twothr = 2. / 3., fivthr = 5. / 3.;
  const cplx ciorsq = cior * cior;
  const cplx ctmp = (I * twothr) * (ciorsq - 1.0);
  const double x2 = xx * xx, x3 = x2 * xx, x4 = x2 * x2;
  cplx a1 = ctmp * (1. - 0.1 * x2 + (ciorsq / 350. + 1. / 280.) * x4) /
            (ciorsq + 2. + (1. - 0.7 * ciorsq) * x2 -
             (ciorsq * ciorsq / 175. - 0.275 * ciorsq + 0.25) * x4 +
             x3 * ctmp * (1. - 0.1 * x2));                                /* R42a */
  cplx b1 = (x2 / 30.) * ctmp * (1. + (ciorsq / 35. - 1. / 14.) * x2) /
            (1. - (ciorsq / 15. - 1. / 6.) * x2);                         /* R42b */
  cplx a2 = (0.1 * x2) * ctmp * (1. - x2 / 14.) /
            (2. * ciorsq + 3. - (ciorsq / 7. - 0.5) * x2);                /* R42c */
  *qsca = (6. * x4) * (sqc(a1) + sqc(b1) + fivthr * sqc(a2));           /* R40a */
  *qext = *qsca;
  if (calcqe)
    *qext = 6. * xx * creal(a1 + b1 + fivthr * a2);                       /* R40b */
  *gqsc = (6. * x4) * creal(a1 * conj(a2 + b1));                          /* R40c */
  const double rtmp = 1.5 * x3;
  *sforw = rtmp * (a1 + b1 + fivthr * a2);
  *sback = rtmp * (a1 - b1 - fivthr * a2);
  tforw[0] = rtmp * (b1 - fivthr * a2);
  tforw[1] = rtmp * (a1 + 2. * fivthr * a2);
  tback[0] = tforw[0];
  tback[1] = rtmp * (a1 - 2. * fivthr * a2);
  for (int j = 0; j < numang; ++j) {                                      /* R40d,e */
    s1[j] = rtmp * (a1 + (b1 + fivthr * a2) * xmu[j]);
    s2[j] = rtmp * (b1 + a1 * xmu[j] + fivthr * a2 * (2. * xmu[j] * xmu[j] - 1.));
  }
}

/* CKINMI, MIEV0noP.f:512-606. */
static void ckinmi(int numang, double xx, int perfct, cplx crefin, int nmom, int anyang,
                   const double *xmu)
{
  int inperr = 0;
  if (numang > MIE_MAXANG) { fprintf(stderr, " ****** ERROR *****  MaxAng too small\n"); inperr = 1; }
  if (numang < 0) { fprintf(stderr, " ****  Input variable NUMANG out of range\n"); inperr = 1; }
  if (xx < 0.) { fprintf(stderr, " ****  Input variable XX out of range\n"); inperr = 1; }
  if (!perfct && creal(crefin) <= 0.) { fprintf(stderr, " ****  Input variable CREFIN out of range\n"); inperr = 1; }
  if (nmom != 0) {
    fprintf(stderr, " ****  Input variable NMOM out of range\n For nonzero NMOM, use complete version of MIEV0\n");
    inperr = 1;
  }
  if (anyang) {
    for (int i = 0; i < numang; ++i)
      if (xmu[i] < -1.00001 || xmu[i] > 1.00001) { fprintf(stderr, " ****  Input variable XMU out of range\n"); inperr = 1; }
  } else {
    for (int i = 0; i < (numang + 1) / 2; ++i)
      if (xmu[i] < -0.00001 || xmu[i] > 1.00001) { fprintf(stderr, " ****  Input variable XMU out of range\n"); inperr = 1; }
  }
  if (inperr)
    mie_fatal("MIEV0--INPUT ERROR(S).  Aborting...");
  if (xx > 20000.0 || creal(crefin) > 10.0 || fabs(cimag(crefin)) > 10.0)
    fprintf(stderr, "\n ****** WARNING *****  MIEV0--XX or CREFIN outside tested range\n\n");
}

/* One MIEV0 evaluation without the first-call self-test (MIEV0noP.f:133-488). */
static void miev0_core(double xx, cplx crefin, int perfct, double mimcut, int anyang,
                       int numang, const double *xmu, int nmom,
                       double *qext, double *qsca, double *gqsc, cplx *sforw, cplx *sback,
                       cplx *s1, cplx *s2, cplx *tforw, cplx *tback, double *spike)
{
  ckinmi(numang, xx, perfct, crefin, nmom, anyang, xmu);
  if (perfct)
    mie_fatal("MIEV0--perfectly conducting spheres are not restated (no caller uses them)");

  cplx cior = crefin;
  if (cimag(cior) > 0.0)
    cior = conj(cior);
  const double mre = creal(cior);
  const double mim = -cimag(cior);
  const int noabs = mim <= mimcut;
  const cplx ciorv = 1.0 / cior;
  const double riorv = 1.0 / mre;

  if (xx * fmax(1.0, cabs(cior)) <= 0.1) {
    small2(xx, cior, mim > mimcut, numang, xmu, qext, qsca, gqsc, sforw, sback, s1, s2,
           tforw, tback);
    *spike = 1.0;
    goto conjugate;
  }

  {
    const int nangd2 = (numang + 1) / 2;
    const int yesang = numang > 0;
    int ntrm;                                         /* R50, truncation to INTEGER */
    if (xx <= 8.0)
      ntrm = (int)(xx + 4. * pow(xx, 1. / 3.) + 1.);
    else if (xx < 4200.)
      ntrm = (int)(xx + 4.05 * pow(xx, 1. / 3.) + 2.);
    else
      ntrm = (int)(xx + 4. * pow(xx, 1. / 3.) + 2.);
    if (ntrm + 1 > MIE_MAXTRM)
      mie_fatal("MIEV0--PARAMETER MaxTrm TOO SMALL");

    double *rbiga = (double *)calloc((size_t)ntrm + 1, sizeof(double));
    cplx *cbiga = (cplx *)calloc((size_t)ntrm + 1, sizeof(cplx));
    const int nang = anyang ? numang : nangd2;
    double *pin = (double *)malloc(sizeof(double) * (size_t)(nang > 0 ? nang : 1));
    double *pinm1 = (double *)malloc(sizeof(double) * (size_t)(nang > 0 ? nang : 1));
    cplx *sp = (cplx *)malloc(sizeof(cplx) * (size_t)(nang > 0 ? nang : 1));
    cplx *sm = (cplx *)malloc(sizeof(cplx) * (size_t)(nang > 0 ? nang : 1));
    cplx *sps = (cplx *)malloc(sizeof(cplx) * (size_t)(nang > 0 ? nang : 1));
    cplx *sms = (cplx *)malloc(sizeof(cplx) * (size_t)(nang > 0 ? nang : 1));
    if (!rbiga || !cbiga || !pin || !pinm1 || !sp || !sm || !sps || !sms)
      mie_fatal("MIEV0--out of memory");

    biga(cior, xx, ntrm, noabs, yesang, rbiga, cbiga);

    /* R19: Riccati-Bessel psi, chi, zeta of orders 0 and 1 */
    const double xinv = 1.0 / xx;
    double psinm1 = sin(xx);
    double chinm1 = cos(xx);
    double psin = psinm1 * xinv - chinm1;
    double chin = chinm1 * xinv + psinm1;
    cplx zetnm1 = psinm1 + I * chinm1;
    cplx zetn = psin + I * chin;
    cplx anm1 = 0.0, bnm1 = 0.0;
    for (int j = 0; j < nang; ++j) {                  /* R39 */
      pinm1[j] = 0.0;
      pin[j] = 1.0;
      sp[j] = 0.0;
      sm[j] = 0.0;
      sps[j] = 0.0;
      sms[j] = 0.0;
    }
    double qs = 0.0, gq = 0.0;
    cplx sf = 0.0, sb = 0.0, csum1 = 0.0, csum2 = 0.0;
    double mm = +1.0;
    double spk = 1.0;
    cplx cdenan = 0.0, cdenbn = 0.0;

    for (int n = 1; n <= ntrm; ++n) {
      const double fn = n;
      const double rn = 1.0 / fn;
      const double np1dn = 1.0 + rn;
      const double twonp1 = 2 * n + 1;
      const double coeff = twonp1 / (fn * (n + 1));
      const double tcoef = twonp1 * (fn * (n + 1));
      cplx an, bn;
      if (noabs) {                                    /* R16, no absorption */
        cdenan = (riorv * rbiga[n] + (fn * xinv)) * zetn - zetnm1;
        an = ((riorv * rbiga[n] + (fn * xinv)) * psin - psinm1) / cdenan;
        cdenbn = (mre * rbiga[n] + (fn * xinv)) * zetn - zetnm1;
        bn = ((mre * rbiga[n] + (fn * xinv)) * psin - psinm1) / cdenbn;
      } else {                                        /* R16, absorbing */
        cdenan = (ciorv * cbiga[n] + (fn * xinv)) * zetn - zetnm1;
        cdenbn = (cior * cbiga[n] + (fn * xinv)) * zetn - zetnm1;
        an = ((ciorv * cbiga[n] + (fn * xinv)) * psin - psinm1) / cdenan;
        bn = ((cior * cbiga[n] + (fn * xinv)) * psin - psinm1) / cdenbn;
        qs = qs + twonp1 * (sqc(an) + sqc(bn));      /* R7 */
      }
      if (n > xx) {                                   /* resonance spikes, R/B.9-10 */
        const double denan = cabs(cdenan);
        const double denbn = cabs(cdenbn);
        const double ratio = denan / denbn;
        if (ratio <= 0.2 || ratio >= 5.0)
          spk = fmin(spk, fmin(denan, denbn));
      }
      sf = sf + twonp1 * (an + bn);                   /* R/B.2 */
      csum1 = csum1 + tcoef * (an - bn);              /* R/B.5,6 */
      sb = sb + (mm * twonp1) * (an - bn);            /* R/B.1 */
      csum2 = csum2 + (mm * tcoef) * (an + bn);       /* R/B.7,8 */
      gq = gq + (fn - rn) * creal(anm1 * conj(an) + bnm1 * conj(bn)) +
           coeff * creal(an * conj(bn));              /* R8 */
      if (yesang) {
        const cplx anp = coeff * (an + bn);           /* R10 */
        const cplx bnp = coeff * (an - bn);
        if (anyang) {
          for (int j = 0; j < numang; ++j) {
            const double rtmp = (xmu[j] * pin[j]) - pinm1[j];   /* R37b */
            const double taun = fn * rtmp - pinm1[j];           /* R38b */
            sp[j] = sp[j] + anp * (pin[j] + taun);
            sm[j] = sm[j] + bnp * (pin[j] - taun);
            pinm1[j] = pin[j];
            pin[j] = (xmu[j] * pin[j]) + np1dn * rtmp;          /* R37c */
          }
        } else {
          const cplx anpm = mm * anp;
          const cplx bnpm = mm * bnp;
          for (int j = 0; j < nangd2; ++j) {
            const double rtmp = (xmu[j] * pin[j]) - pinm1[j];
            const double taun = fn * rtmp - pinm1[j];
            sp[j] = sp[j] + anp * (pin[j] + taun);
            sms[j] = sms[j] + bnpm * (pin[j] + taun);
            sm[j] = sm[j] + bnp * (pin[j] - taun);
            sps[j] = sps[j] + anpm * (pin[j] - taun);
            pinm1[j] = pin[j];
            pin[j] = (xmu[j] * pin[j]) + np1dn * rtmp;
          }
        }
      }
      mm = -mm;
      anm1 = an;
      bnm1 = bn;
      const cplx zet = (twonp1 * xinv) * zetn - zetnm1;  /* R17 */
      zetnm1 = zetn;
      zetn = zet;
      psinm1 = psin;
      psin = creal(zetn);
    }

    *qext = 2. / (xx * xx) * creal(sf);               /* R6 */
    *qsca = noabs ? *qext : 2. / (xx * xx) * qs;
    *gqsc = 4. / (xx * xx) * gq;
    sf = 0.5 * sf;
    sb = 0.5 * sb;
    *sforw = sf;
    *sback = sb;
    tforw[0] = 0.5 * sf - 0.125 * csum1;
    tforw[1] = 0.5 * sf + 0.125 * csum1;
    tback[0] = -0.5 * sb + 0.125 * csum2;
    tback[1] = 0.5 * sb + 0.125 * csum2;
    *spike = spk;
    if (yesang) {                                     /* R11 */
      if (anyang) {
        for (int j = 0; j < numang; ++j) {
          s1[j] = 0.5 * (sp[j] + sm[j]);
          s2[j] = 0.5 * (sp[j] - sm[j]);
        }
      } else {
        for (int j = 0; j < nangd2; ++j) {
          s1[j] = 0.5 * (sp[j] + sm[j]);
          s2[j] = 0.5 * (sp[j] - sm[j]);
        }
        for (int j = 0; j < nangd2; ++j) {
          s1[numang - 1 - j] = 0.5 * (sps[j] + sms[j]);
          s2[numang - 1 - j] = 0.5 * (sps[j] - sms[j]);
        }
      }
    }
    free(rbiga); free(cbiga); free(pin); free(pinm1); free(sp); free(sm); free(sps); free(sms);
  }

conjugate:
  if (cimag(crefin) > 0.0) {                          /* MIEV0noP.f:459-478 */
    *sforw = conj(*sforw);
    *sback = conj(*sback);
    for (int i = 0; i < 2; ++i) {
      tforw[i] = conj(tforw[i]);
      tback[i] = conj(tback[i]);
    }
    for (int j = 0; j < numang; ++j) {
      s1[j] = conj(s1[j]);
      s2[j] = conj(s2[j]);
    }
  }
}

/* TESTMI, MIEV0noP.f:1182-1330: known answers for x=10, m=1.5-0.1i, mu=-0.7660444. */
int lmc_oracle_miev0_selftest(double *worst_rel_err)
{
  const double accur = 1.e-4;
  const double testqe = 2.459791, testqs = 1.235144, testgq = 1.139235;
  const cplx testsf = 61.49476 - 3.177994 * I, testsb = 1.493434 + 0.2963657 * I;
  const cplx tests1 = -0.1548380 - 1.128972 * I, tests2 = 0.05669755 + 0.5425681 * I;
  const cplx testtf[2] = {12.95238 - 136.6436 * I, 48.54238 + 133.4656 * I};
  const cplx testtb[2] = {41.88414 - 15.57833 * I, 43.37758 - 15.28196 * I};
  double xmu = -0.7660444;
  double qext, qsca, gqsc, spike;
  cplx sforw, sback, s1, s2, tforw[2], tback[2];
  miev0_core(10.0, 1.5 - 0.1 * I, 0, 0.0, 1, 1, &xmu, 0, &qext, &qsca, &gqsc, &sforw,
             &sback, &s1, &s2, tforw, tback, &spike);
  double worst = 0.0;
  int ok = 1;
#define LMC_CHECK(calc, exact)                                   \
  do {                                                           \
    const double e_ = fabs(((calc) - (exact)) / (exact));        \
    if (e_ > worst) worst = e_;                                  \
    if (e_ > accur) ok = 0;                                      \
  } while (0)
  LMC_CHECK(qext, testqe);
  LMC_CHECK(qsca, testqs);
  LMC_CHECK(gqsc, testgq);
  LMC_CHECK(creal(sforw), creal(testsf)); LMC_CHECK(cimag(sforw), cimag(testsf));
  LMC_CHECK(creal(sback), creal(testsb)); LMC_CHECK(cimag(sback), cimag(testsb));
  LMC_CHECK(creal(s1), creal(tests1));    LMC_CHECK(cimag(s1), cimag(tests1));
  LMC_CHECK(creal(s2), creal(tests2));    LMC_CHECK(cimag(s2), cimag(tests2));
  for (int n = 0; n < 2; ++n) {
    LMC_CHECK(creal(tforw[n]), creal(testtf[n])); LMC_CHECK(cimag(tforw[n]), cimag(testtf[n]));
    LMC_CHECK(creal(tback[n]), creal(testtb[n])); LMC_CHECK(cimag(tback[n]), cimag(testtb[n]));
  }
#undef LMC_CHECK
  if (worst_rel_err)
    *worst_rel_err = worst;
  return ok;
}

/* Fortran-ABI entry point bound by src/mie/dmiev.cpp (dmiev.h:106).  LOGICAL
 * arguments are 4-byte ints; PMOM, IPOLZN and MOMDIM are unused (NoPMOM). */
void miev0_(double *XX, cplx *CREFIN, int *PERFCT, double *MIMCUT, int *ANYANG, int *NUMANG,
            double *XMU, int *NMOM, int *IPOLZN, int *MOMDIM, int *PRNT, double *QEXT,
            double *QSCA, double *GQSC, double *PMOM, cplx *SFORW, cplx *SBACK, cplx *S1,
            cplx *S2, cplx *TFORW, cplx *TBACK, double *SPIKE)
{
  static int pass1 = 1;
  (void)IPOLZN; (void)MOMDIM; (void)PMOM; (void)PRNT;
  if (pass1) {
    double worst = 0.0;
    if (!lmc_oracle_miev0_selftest(&worst))
      mie_fatal("MIEV0 -- Self-test failed");
    pass1 = 0;
  }
  miev0_core(*XX, *CREFIN, *PERFCT, *MIMCUT, *ANYANG, *NUMANG, XMU, *NMOM, QEXT, QSCA, GQSC,
             SFORW, SBACK, S1, S2, TFORW, TBACK, SPIKE);
}
