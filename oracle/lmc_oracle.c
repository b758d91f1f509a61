/*
 * oracle/lmc_oracle.c -- TEST INFRASTRUCTURE (the oracle), never product code.
 *
 * Plain-C restatement of the reference's photon-propagation path.  Every
 * function cites the reference file:line it follows.  The expressions keep the
 * reference's operand order so that, compiled with -ffp-contract=off like the
 * `pin` build of the reference (oracle/Makefile), both produce the same bits.
 * std::complex<double> arithmetic maps onto C99 `double complex`; std::norm is
 * re*re + im*im (what libstdc++ evaluates at -O2 here).
 *
 * Out of scope (rejected at create time): MixtureLayer, PhotonRecord/Statistics
 * sensors, the Absorption recorder.  Planar sensors in estimator mode record nothing, as in
 * the reference (their process_estimation bodies are empty,
 * src/detector.cpp:571-700,844-846).
 */
#include "lmc_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "philox_ref.h"

typedef double complex cplx;

void miev0_(double *XX, cplx *CREFIN, int *PERFCT, double *MIMCUT, int *ANYANG, int *NUMANG,
            double *XMU, int *NMOM, int *IPOLZN, int *MOMDIM, int *PRNT, double *QEXT,
            double *QSCA, double *GQSC, double *PMOM, cplx *SFORW, cplx *SBACK, cplx *S1,
            cplx *S2, cplx *TFORW, cplx *TBACK, double *SPIKE);

/* ---------------------------------------------------------------- small math
 * include/luminis/math/vec.hpp:48-80, src/vec.cpp:10-32, src/utils.cpp:25-82 */
typedef struct { double x, y, z; } v3;

static v3 v3make(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static v3 v3add(v3 a, v3 b) { return v3make(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 v3sub(v3 a, v3 b) { return v3make(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 v3scale(v3 a, double s) { return v3make(a.x * s, a.y * s, a.z * s); }
static double v3dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }   /* vec.cpp:10 */
static double v3norm(v3 a) { return sqrt(v3dot(a, a)); }                       /* vec.cpp:28 */
static v3 v3cross(v3 a, v3 b)                                                    /* vec.cpp:14-26 */
{
  v3 r;
  r.x = a.y * b.z - a.z * b.y;
  r.y = a.z * b.x - a.x * b.z;
  r.z = a.x * b.y - a.y * b.x;
  const double nf = v3norm(r);
  if (nf > 0.0) {
    const double inv = 1.0 / nf;
    r = v3scale(r, inv);
  }
  return r;
}
static double clamp_pm1(double x) { return x > 1.0 ? 1.0 : (x < -1.0 ? -1.0 : x); }  /* utils.cpp:25 */
static v3 safe_unit(v3 v, v3 fallback)                                          /* utils.cpp:39-50 */
{
  const double eps = 1e-20;
  const double n2 = v3dot(v, v);
  if (n2 < eps) {
    const double f2 = v3dot(fallback, fallback);
    if (f2 < eps)
      return v3make(1, 0, 0);
    return v3scale(fallback, 1.0 / sqrt(f2));
  }
  return v3scale(v, 1.0 / sqrt(n2));
}
static double cnrm(cplx z) { return creal(z) * creal(z) + cimag(z) * cimag(z); }

/* 3x3 frame: rows m, n, s (photon.hpp:117) */
typedef struct { double a[3][3]; } m3;
static v3 m3row(const m3 *P, int r) { return v3make(P->a[r][0], P->a[r][1], P->a[r][2]); }

/* rot2 (utils.cpp:53-61): real 2x2 stored as doubles; the reference's complex
 * entries have zero imaginary parts, so S*R and R*E reduce exactly to scaled
 * complex numbers. */
typedef struct { double r00, r01, r10, r11; } rot2_t;
static rot2_t rot2(v3 m_to, v3 n_to, v3 m_from, v3 n_from)
{
  rot2_t R = {v3dot(m_to, m_from), v3dot(m_to, n_from), v3dot(n_to, m_from), v3dot(n_to, n_from)};
  return R;
}

/* ------------------------------------------------------------------- RNG */
typedef struct {
  int kind;
  uint64_t s[4];
  uint64_t seed, photon, draw;
} orng;

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t mix_seed(uint64_t base, uint64_t tid)        /* src/rng.cpp:5-10 */
{
  uint64_t z = base + 0x9E3779B97F4A7C15ULL * (tid + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

static void orng_seed_photon(orng *r, uint64_t seed, uint64_t photon)  /* rng.hpp:59-68 */
{
  r->seed = seed;
  r->photon = photon;
  r->draw = 0;
  if (r->kind == LMC_O_RNG_XOSHIRO) {
    uint64_t z = mix_seed(seed, photon);
    for (int i = 0; i < 4; ++i) {
      z += 0x9E3779B97F4A7C15ULL;
      uint64_t x = z;
      x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
      x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
      r->s[i] = x ^ (x >> 31);
    }
  }
}

static double orng_uniform(orng *r)
{
  const uint64_t d = r->draw++;
  if (r->kind == LMC_O_RNG_XOSHIRO) {                         /* rng.hpp:75-85, rng.cpp:12-16 */
    uint64_t *s = r->s;
    const uint64_t result = rotl64(s[0] + s[3], 23) + s[0];
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return (double)(result >> 11) * 0x1.0p-53;
  }
  return lmc_ref_stream_uniform(r->seed, r->photon, d,
                                r->kind == LMC_O_RNG_PHILOX_U24 ? LMC_STREAM_U24 : LMC_STREAM_U53);
}

static double orng_normal(orng *r, double mean, double stddev) /* src/rng.cpp:18-27 */
{
  double u1 = orng_uniform(r);
  while (u1 <= 0.0)
    u1 = orng_uniform(r);
  const double u2 = orng_uniform(r);
  const double z0 = sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
  return z0 * stddev + mean;
}

/* ---------------------------------------------------------------- tables */
typedef struct { int n; double *values, *cdf; } stable;        /* SamplingTable */
typedef struct { int n; double x_min, dx, inv_dx; cplx *y; } dtable;  /* DataTable (uniform) */

typedef double (*pdf_fn)(const void *ctx, double x);

/* SamplingTable::initialize, src/table.cpp:6-48 (pdf sized nDiv+1 here; the
 * reference's vector of nDiv is written one past its end at :29). */
static int stable_init(stable *t, pdf_fn f, const void *ctx, int nDiv, double minVal, double maxVal)
{
  if (nDiv <= 0 || minVal >= maxVal)
    return -1;
  const double step = (maxVal - minVal) / nDiv;
  t->n = nDiv + 1;
  t->values = (double *)malloc(sizeof(double) * (size_t)t->n);
  t->cdf = (double *)malloc(sizeof(double) * (size_t)t->n);
  double *pdf = (double *)malloc(sizeof(double) * (size_t)t->n);
  double sum = 0.0;
  for (int i = 0; i < nDiv + 1; i++) {
    t->values[i] = minVal + i * step;
    pdf[i] = f(ctx, t->values[i]);
    sum += pdf[i] * step;
  }
  for (int i = 0; i < nDiv + 1; i++)
    pdf[i] /= sum;
  t->cdf[0] = pdf[0] * step;
  for (int i = 1; i < nDiv + 1; i++)
    t->cdf[i] = t->cdf[i - 1] + pdf[i] * step;
  for (int i = 0; i < nDiv + 1; i++)
    t->cdf[i] /= t->cdf[nDiv];
  free(pdf);
  return 0;
}

static double stable_sample(const stable *t, double u)        /* src/table.cpp:50-66 */
{
  int lo = 0, hi = t->n;                                       /* std::lower_bound */
  while (lo < hi) {
    const int mid = lo + (hi - lo) / 2;
    if (t->cdf[mid] < u)
      lo = mid + 1;
    else
      hi = mid;
  }
  const int index = lo;
  if (index == 0)
    return t->values[0];
  if (index >= t->n)
    return t->values[t->n - 1];
  const double tt = (u - t->cdf[index - 1]) / (t->cdf[index] - t->cdf[index - 1]);
  return t->values[index - 1] + tt * (t->values[index] - t->values[index - 1]);
}

static void dtable_init_uniform(dtable *t, double x_min, double dx, const cplx *y, int n)
{                                                              /* src/table.cpp:78-98 */
  t->n = n;
  t->x_min = x_min;
  t->dx = dx;
  t->inv_dx = 1.0 / dx;
  t->y = (cplx *)malloc(sizeof(cplx) * (size_t)n);
  memcpy(t->y, y, sizeof(cplx) * (size_t)n);
}

static cplx dtable_sample(const dtable *t, double x)           /* src/table.cpp:100-118 */
{
  const double pos = (x - t->x_min) * t->inv_dx;
  if (pos <= 0.0)
    return t->y[0];
  const int last = t->n - 1;
  if (pos >= (double)last)
    return t->y[last];
  const size_t i = (size_t)pos;
  const double tt = pos - (double)i;
  return t->y[i] + tt * (t->y[i + 1] - t->y[i]);
}

/* ---------------------------------------------------- Mie wrappers (dmiev.cpp) */
static void amiev(double xx, cplx crefin, double mu, cplx *s1, cplx *s2)  /* dmiev.cpp:6-21 */
{
  int PERFCT = 0, ANYANG = 1, NUMANG = 1, NMOM = 0, IPOLZN = 0, MOMDIM = 1, PRNT[2] = {0, 0};
  double MIMCUT = 1e-8, QEXT, QSCA, GQSC, PMOM, SPIKE;
  cplx SFORW, SBACK, TFORW[2], TBACK[2];
  miev0_(&xx, &crefin, &PERFCT, &MIMCUT, &ANYANG, &NUMANG, &mu, &NMOM, &IPOLZN, &MOMDIM, PRNT,
         &QEXT, &QSCA, &GQSC, &PMOM, &SFORW, &SBACK, s1, s2, TFORW, TBACK, &SPIKE);
}

static void miev_many(double xx, cplx crefin, int numang, double *mu, cplx *s1, cplx *s2)
{                                                              /* dmiev.cpp:45-57 */
  int PERFCT = 0, ANYANG = 1, NMOM = 0, IPOLZN = 0, MOMDIM = 1, PRNT[2] = {0, 0};
  double MIMCUT = 1e-8, QEXT, QSCA, GQSC, PMOM, SPIKE;
  cplx SFORW, SBACK, TFORW[2], TBACK[2];
  miev0_(&xx, &crefin, &PERFCT, &MIMCUT, &ANYANG, &numang, mu, &NMOM, &IPOLZN, &MOMDIM, PRNT,
         &QEXT, &QSCA, &GQSC, &PMOM, &SFORW, &SBACK, s1, s2, TFORW, TBACK, &SPIKE);
}

static void mievinfo(double xx, cplx crefin, double *qext, double *qsca, double *g)
{                                                              /* dmiev.cpp:60-76 */
  int PERFCT = 0, ANYANG = 1, NUMANG = 1, NMOM = 0, IPOLZN = 0, MOMDIM = 1, PRNT[2] = {0, 0};
  double MIMCUT = 1e-8, XMU = 0, gqsc, PMOM, SPIKE;
  cplx SFORW, SBACK, S1, S2, TFORW[2], TBACK[2];
  miev0_(&xx, &crefin, &PERFCT, &MIMCUT, &ANYANG, &NUMANG, &XMU, &NMOM, &IPOLZN, &MOMDIM, PRNT,
         qext, qsca, &gqsc, &PMOM, &SFORW, &SBACK, &S1, &S2, TFORW, TBACK, &SPIKE);
  *g = gqsc / (*qsca);
}

void lmc_oracle_mie(double x, double m_re, double m_im, int n, const double *mu, double *s1,
                    double *s2, double *qext, double *qsca, double *g)
{
  cplx m = CMPLX(m_re, m_im);
  if (n > 0) {
    double *mm = (double *)malloc(sizeof(double) * (size_t)n);
    cplx *a = (cplx *)malloc(sizeof(cplx) * (size_t)n), *b = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    memcpy(mm, mu, sizeof(double) * (size_t)n);
    miev_many(x, m, n, mm, a, b);
    for (int i = 0; i < n; ++i) {
      s1[2 * i] = creal(a[i]); s1[2 * i + 1] = cimag(a[i]);
      s2[2 * i] = creal(b[i]); s2[2 * i + 1] = cimag(b[i]);
    }
    free(mm); free(a); free(b);
  }
  double qe, qs, gg;
  mievinfo(x, m, &qe, &qs, &gg);
  if (qext) *qext = qe;
  if (qsca) *qsca = qs;
  if (g) *g = gg;
}

/* --------------------------------------------------------- phase functions */
static double form_factor(double theta, double k, double radius)   /* src/phase.cpp:10-20 */
{
  if (fabs(theta) == 0.0)
    return 1.0;
  const double u = 2.0 * k * radius * sin(theta / 2.0);
  const double numerator = 3 * (sin(u) - u * cos(u));
  const double denominator = pow(u, 3);
  return numerator / denominator;
}

typedef struct {
  lmc_o_phase p;
  int samples_theta;      /* table holds theta (RD, RD-EMC, Mie) or cos theta (Rayleigh, Draine) */
  double k, sigma_s;      /* RD/RD-EMC/Mie wave number in the medium, cross section */
  cplx m;
  stable table;
} ophase;

static double pdf_rayleigh(const void *c, double x) { (void)c; return 0.375 * (1.0 + x * x); }  /* :96-98 */

static double pdf_rd(const void *c, double x)                  /* src/phase.cpp:138-142 */
{
  const ophase *ph = (const ophase *)c;
  const double F = form_factor(x, ph->k, ph->p.radius);
  const double a = 1.0 / (4.0 * M_PI);
  return a * pow(F, 2);
}

static double rdemc_qsca(const ophase *ph)                     /* src/phase.cpp:168-195 */
{
  const double radius = ph->p.radius, k = ph->k;
  const double x = radius * k;
  const double V = 4 * M_PI * pow(radius, 3) / 3.0;
  const double a = (pow(k, 6) * pow((ph->p.n_particle / ph->p.n_medium - 1.0), 2) * V * V) /
                   (4 * pow(M_PI, 2));
  const double c = a / pow(x, 2);
  const int N = 100000;
  const double h = M_PI / N;
#define LMC_RDEMC_INTEGRAND(th) \
  (form_factor((th), k, radius) * form_factor((th), k, radius) * sin(th) * (1.0 + cos(th) * cos(th)))
  double sum = LMC_RDEMC_INTEGRAND(0.0) + LMC_RDEMC_INTEGRAND(M_PI);
  for (int i = 1; i < N; i += 2)
    sum += 4.0 * LMC_RDEMC_INTEGRAND(i * h);
  for (int i = 2; i < N; i += 2)
    sum += 2.0 * LMC_RDEMC_INTEGRAND(i * h);
#undef LMC_RDEMC_INTEGRAND
  const double integral = sum * h / 3.0;
  return c * integral;
}

static double pdf_rdemc(const void *c, double x)               /* src/phase.cpp:202-214 */
{
  const ophase *ph = (const ophase *)c;
  const double k = ph->k;
  const double kkkk = pow(k, 4);
  const double m_1 = (ph->p.n_particle / ph->p.n_medium) - 1.0;
  const double v = (4.0 / 3.0) * M_PI * pow(ph->p.radius, 3);
  const double F = form_factor(x, k, ph->p.radius);
  const double intensity = (kkkk / (4.0 * M_PI * ph->sigma_s)) * m_1 * m_1 * v * v * F * F *
                           (1.0 + cos(x) * cos(x));
  return intensity * sin(x);
}

static double pdf_draine(const void *c, double x)              /* src/phase.cpp:236-240 */
{
  const ophase *ph = (const ophase *)c;
  const double g = ph->p.g, a = ph->p.a;
  const double hgTerm = (1.0 - g * g) / pow(1.0 + g * g - 2.0 * g * x, 1.5);
  const double draineTerm = (1.0 + a * x * x) / (3 + a * (1 + 2 * g * g));
  return (1.0 / 4.0 * M_PI) * hgTerm * draineTerm;
}

static double pdf_mie(const void *c, double x)                 /* src/phase.cpp:286-304 */
{
  const ophase *ph = (const ophase *)c;
  cplx s1, s2;
  double mu = cos(x);
  if (mu > 1.0) mu = 1.0;
  if (mu < -1.0) mu = -1.0;
  const double sizep = ph->k * ph->p.radius;
  amiev(sizep, ph->m, mu, &s1, &s2);
  const double intensity = (M_PI / (ph->k * ph->k * ph->sigma_s)) * (cnrm(s1) + cnrm(s2));
  return intensity * sin(x);
}

static int ophase_init(ophase *ph, const lmc_o_phase *p)
{
  memset(ph, 0, sizeof(*ph));
  ph->p = *p;
  switch (p->kind) {
  case LMC_O_PHASE_UNIFORM:
  case LMC_O_PHASE_HG:
    return 0;
  case LMC_O_PHASE_RAYLEIGH:                                   /* :87-89 */
    ph->samples_theta = 0;
    return stable_init(&ph->table, pdf_rayleigh, ph, p->n_div, p->min_val, p->max_val);
  case LMC_O_PHASE_RD:                                         /* :119-131 */
    ph->samples_theta = 1;
    ph->k = 2 * M_PI / p->wavelength;
    return stable_init(&ph->table, pdf_rd, ph, p->n_div, p->min_val, p->max_val);
  case LMC_O_PHASE_RDEMC:                                      /* :146-161, :196-200 */
    ph->samples_theta = 1;
    ph->k = 2 * M_PI * p->n_medium / p->wavelength;
    ph->sigma_s = rdemc_qsca(ph) * (M_PI * pow(p->radius, 2));
    return stable_init(&ph->table, pdf_rdemc, ph, p->n_div, p->min_val, p->max_val);
  case LMC_O_PHASE_DRAINE:                                     /* :218-229 */
    ph->samples_theta = 0;
    return stable_init(&ph->table, pdf_draine, ph, p->n_div, p->min_val, p->max_val);
  case LMC_O_PHASE_MIE: {                                      /* :244-260, :270-284 */
    ph->samples_theta = 1;
    ph->k = 2 * M_PI * p->n_medium / p->wavelength;
    ph->m = CMPLX(p->n_particle / p->n_medium, 0.0);
    double qext, qsca, g;
    mievinfo(p->radius * ph->k, ph->m, &qext, &qsca, &g);
    ph->sigma_s = qsca * (M_PI * pow(p->radius, 2));
    return stable_init(&ph->table, pdf_mie, ph, p->n_div, p->min_val, p->max_val);
  }
  default:
    return -1;
  }
}

static double ophase_sample_theta(const ophase *ph, double x)
{
  switch (ph->p.kind) {
  case LMC_O_PHASE_UNIFORM:                                    /* :78-83 */
    return acos(2.0 * x - 1.0);
  case LMC_O_PHASE_HG: {                                       /* :108-115 */
    const double g = ph->p.g;
    const double gg = g * g;
    const double frac = (1.0 - gg) / (1.0 - g + 2.0 * g * x);
    return acos((1.0 + gg - frac * frac) / (2.0 * g));
  }
  default:
    if (ph->samples_theta)
      return stable_sample(&ph->table, x);
    return acos(stable_sample(&ph->table, x));
  }
}

/* ------------------------------------------------------------------ media */
typedef struct {
  lmc_o_medium p;
  double mu_t;          /* mu_a + mu_s (src/medium.cpp:61-71) */
  double I_norm;        /* int_0^pi (|S11|^2 + |S22|^2) sin(theta) dtheta (estimator) */
  dtable S1, S2;
  int phase;
} omedium;

static int omedium_init(omedium *md, const lmc_o_medium *p)
{
  memset(md, 0, sizeof(*md));
  md->p = *p;
  md->phase = p->phase;
  md->mu_t = p->mu_a + p->mu_s;
  if (p->kind == LMC_O_MEDIUM_RGD) {                           /* src/medium.cpp:77-120 */
    const double k = 2 * M_PI * p->n_medium / p->wavelength;
    const double kkk = k * k * k;
    const double volume = 4.0 * M_PI * (p->radius * p->radius * p->radius) / 3.0;
    const double mm = (p->n_particle / p->n_medium) - 1.0;
    const double pref = -1.0 * kkk * mm * volume / (2.0 * M_PI);
    const int n = 2000;
    const double dtheta = M_PI / (double)(n - 1);
    cplx *s1 = (cplx *)malloc(sizeof(cplx) * n), *s2 = (cplx *)malloc(sizeof(cplx) * n);
    for (int i = 0; i < n; ++i) {
      const double theta = (double)i * dtheta;
      const double F = form_factor(theta, k, p->radius);
      s1[i] = CMPLX(0.0, pref * F);
      s2[i] = CMPLX(0.0, pref * F * cos(theta));
    }
    dtable_init_uniform(&md->S1, 0.0, dtheta, s1, n);
    dtable_init_uniform(&md->S2, 0.0, dtheta, s2, n);
    free(s1); free(s2);
    return 0;
  }
  if (p->kind == LMC_O_MEDIUM_MIE) {                           /* src/medium.cpp:160-236 */
    const cplx m = CMPLX(p->n_particle / p->n_medium, 0);
    const int n = 1000;
    const double x = 2 * M_PI * p->radius / p->wavelength;
    const double dtheta = M_PI / (double)(n - 1);
    double *mu = (double *)malloc(sizeof(double) * n);
    cplx *s1 = (cplx *)malloc(sizeof(cplx) * n), *s2 = (cplx *)malloc(sizeof(cplx) * n);
    for (int i = 0; i < n; ++i)
      mu[i] = cos((double)i * dtheta);
    miev_many(x, m, n, mu, s1, s2);
    dtable_init_uniform(&md->S1, 0.0, dtheta, s1, n);
    dtable_init_uniform(&md->S2, 0.0, dtheta, s2, n);
    free(mu); free(s1); free(s2);
    return 0;
  }
  return -1;
}

/* scattering_matrix (src/medium.cpp:138-148, :181-190): diag(S2, S1). */
static void omedium_smatrix(const omedium *md, double theta, cplx *s2, cplx *s1)
{
  *s1 = dtable_sample(&md->S1, theta);
  *s2 = dtable_sample(&md->S2, theta);
}

/* ----------------------------------------------------------------- sensors */
typedef struct {
  lmc_o_sensor p;
  int key;                        /* index of the z-plane group */
  double cos_min, cos_max;        /* set_theta_limit cache (src/detector.cpp:334-343) */
  int N_t, N_x, N_y, N_theta, N_phi;
  size_t n_doubles;
  /* STATISTICS: bin widths (src/detector.cpp:1836-1888) and histogram offsets */
  double st_dtheta, st_dphi, st_ddepth, st_dtime, st_dweight;
  size_t st_off[6];
} osensor;

/* A layer's transport coefficients (Layer::mu_attenuation/mu_scattering/mu_absorption,
 * sample_free_path): the wrapped medium's for a HomogeneousLayer, the aggregates of
 * MixtureLayer's constructor (src/sample.cpp:41-88) for a mixture. */
typedef struct {
  double mu_s, mu_a, mu_t, mfp;
  int n_species;                  /* 0: HomogeneousLayer (no species draw) */
  int species[LMC_O_MAX_SPECIES];
  double mu_s_i[LMC_O_MAX_SPECIES], cdf[LMC_O_MAX_SPECIES];
} olayer;

struct lmc_o_handle {
  lmc_o_scene scene;
  double light_speed;             /* 1 / n_host (src/sample.cpp:110-111) */
  ophase phase[LMC_O_MAX_PHASE];
  omedium media[LMC_O_MAX_MEDIA];
  olayer layer[LMC_O_MAX_LAYERS];
  double interfaces[LMC_O_MAX_LAYERS];
  int n_interfaces;
  osensor sensors[LMC_O_MAX_SENSORS];
  double plane_z[LMC_O_MAX_SENSORS]; /* z_layers keys, ascending */
  int n_planes;
  int abs_nt, abs_nr, abs_nz;       /* Absorption grid shape (src/absortion.cpp:13-32) */
};

static int osensor_init(lmc_o_handle *h, osensor *s, const lmc_o_sensor *p, char *err, int err_len)
{
  memset(s, 0, sizeof(*s));
  s->p = *p;
  /* Sensor ctor (src/detector.cpp:314-332): estimator only at z == 0 */
  if (p->z != 0.0 && p->estimator)
    s->p.estimator = 0;
  if (p->f_theta) {
    const double c1 = cos(p->theta_min), c2 = cos(p->theta_max);
    s->cos_min = fmin(c1, c2);
    s->cos_max = fmax(c1, c2);
  }
  switch (p->kind) {
  case LMC_O_SENSOR_FARFIELD_CBS:                               /* :851-875 */
  case LMC_O_SENSOR_FARFIELD_FLUENCE:
    s->p.z = 0.0;                 /* Sensor(0.0, true, estimator): always z=0, absorbing */
    s->p.absorb = 1;
    s->N_t = (p->dt == 0) ? 1 : (int)ceil(p->len_t / p->dt) + 1;
    s->N_theta = (int)ceil(p->theta_max_grid / p->dtheta);
    s->N_phi = (int)ceil(p->phi_max_grid / p->dphi);
    s->n_doubles = (size_t)(p->kind == LMC_O_SENSOR_FARFIELD_CBS ? 8 : 4) * s->N_t * s->N_theta * s->N_phi;
    break;
  case LMC_O_SENSOR_PLANAR_FLUENCE:                             /* :704-735 */
    s->N_t = (p->dt == 0) ? 1 : (int)ceil(p->len_t / p->dt) + 1;
    s->N_x = (int)ceil(p->len_x / p->dx);
    s->N_y = (int)ceil(p->len_y / p->dy);
    s->n_doubles = (size_t)4 * s->N_t * s->N_x * s->N_y;
    break;
  case LMC_O_SENSOR_PLANAR_FIELD:                               /* :490-506 */
    s->N_x = (int)ceil(p->len_x / p->dx);
    s->N_y = (int)ceil(p->len_y / p->dy);
    s->n_doubles = (size_t)4 * s->N_x * s->N_y;
    break;
  case LMC_O_SENSOR_STATISTICS: {                               /* :1571-1579, :1802-1888 */
    const lmc_o_statistics *q = &p->stats;
    s->p.estimator = 0;
    s->N_t = (p->dt <= 0.0) ? 1 : (int)ceil(p->len_t / p->dt) + 1;
    if (p->dt <= 0.0)
      s->p.dt = 0.0;
    if (q->n_events < 0 || q->n_theta < 0 || q->n_phi < 0 || q->n_depth < 0 || q->n_time < 0 ||
        q->n_weight < 0) {
      snprintf(err, (size_t)err_len, "StatisticsSensor: histogram sizes must be non-negative");
      return -1;
    }
    const int set = q->set;
    const size_t nt = (size_t)s->N_t;
    size_t n = 0;
    s->st_off[0] = n; n += (set & LMC_O_STAT_EVENTS) ? nt * (size_t)q->n_events : 0;
    s->st_off[1] = n; n += (set & LMC_O_STAT_THETA) ? nt * (size_t)q->n_theta : 0;
    s->st_off[2] = n; n += (set & LMC_O_STAT_PHI) ? nt * (size_t)q->n_phi : 0;
    s->st_off[3] = n; n += (set & LMC_O_STAT_DEPTH) ? nt * (size_t)q->n_depth : 0;
    s->st_off[4] = n; n += (set & LMC_O_STAT_TIME) ? (size_t)q->n_time : 0;
    s->st_off[5] = n; n += (set & LMC_O_STAT_WEIGHT) ? (size_t)q->n_weight : 0;
    s->n_doubles = n;
    s->st_dtheta = (q->theta_max - q->theta_min) / q->n_theta;
    s->st_dphi = (q->phi_max - q->phi_min) / q->n_phi;
    s->st_ddepth = q->depth_max / q->n_depth;
    s->st_dtime = q->time_max / q->n_time;
    s->st_dweight = q->weight_max / q->n_weight;
    break;
  }
  default:
    snprintf(err, (size_t)err_len, "unknown sensor kind %d", p->kind);
    return -1;
  }
  (void)h;
  return 0;
}

/* ------------------------------------------------------------------ photon */
typedef struct {
  v3 prev_pos, pos;
  unsigned events;
  double penetration_depth;
  int alive;
  double k, opticalpath, optical_path, launch_time, velocity, weight;
  int current_layer;
  int active_medium, first_medium, last_medium;
  m3 P;                                   /* P_local */
  cplx Em, En;                            /* polarization */
  cplx Erm, Ern;                          /* polarization_reverse */
  cplx E0m, E0n;                          /* initial_polarization */
  m3 P0, P1, Pn1, Pn;
  v3 r1, rn;
  cplx Traw[4], Traw_buf[4];              /* matrix_T_raw(_buffer), row-major 2x2 */
  int has_T_prev;
  int fate;
  v3 hit;
  int n_hits;
} ophoton;

/* Sample (src/sample.cpp:221-288) */
static int layer_index_at(const lmc_o_handle *h, double z)
{
  const int nl = h->scene.n_layers;
  if (nl == 0) return nl;
  if (z < 0.0) return nl;
  const double top = h->scene.layers[nl - 1].z_max;
  if (!isinf(top) && z >= top) return nl;
  int idx = 0;                                                 /* upper_bound */
  while (idx < h->n_interfaces && !(z < h->interfaces[idx]))
    idx++;
  return idx < nl ? idx : nl;
}

static int find_next_interface(const lmc_o_handle *h, double zc, double zt, double *out)
{                                                              /* :237-266 */
  if (h->n_interfaces == 0)
    return 0;
  if (zt > zc) {
    int i = 0;                                                 /* upper_bound(zc) */
    while (i < h->n_interfaces && !(zc < h->interfaces[i]))
      i++;
    if (i < h->n_interfaces && h->interfaces[i] <= zt) {
      *out = h->interfaces[i];
      return 1;
    }
  } else if (zt < zc) {
    int i = 0;                                                 /* lower_bound(zc) */
    while (i < h->n_interfaces && h->interfaces[i] < zc)
      i++;
    if (i != 0) {
      --i;
      if (h->interfaces[i] >= zt) {
        *out = h->interfaces[i];
        return 1;
      }
    }
  }
  return 0;
}

static int is_inside(const lmc_o_handle *h, v3 p)             /* :268-288 */
{
  const int nl = h->scene.n_layers;
  if (nl == 0) return 0;
  if (isnan(p.x) || isnan(p.y) || isnan(p.z)) return 0;
  if (isinf(p.x) || isinf(p.y) || isinf(p.z)) return 0;
  if (p.z < 0.0) return 0;
  const double top = h->scene.layers[nl - 1].z_max;
  if (!isinf(top) && p.z >= top) return 0;
  return 1;
}

static const olayer *layer_at(const lmc_o_handle *h, int layer)
{
  return &h->layer[layer];
}

/* MixtureLayer constructor (src/sample.cpp:41-88): mu_s_i = n_i sigma_s_i, the
 * absorption that keeps each species' albedo, mu_t, mfp = 1 / mu_s_total and the
 * selection CDF over mu_s_i (last entry exactly 1).  A HomogeneousLayer takes its
 * medium's coefficients (include/luminis/core/sample.hpp:142-144). */
static int olayer_init(const lmc_o_handle *h, const lmc_o_layer *p, olayer *L, char *err, int err_len)
{
  memset(L, 0, sizeof(*L));
  if (p->n_species <= 0) {
    const omedium *m = &h->media[p->medium];
    L->mu_s = m->p.mu_s;
    L->mu_a = m->p.mu_a;
    L->mu_t = m->mu_t;
    L->mfp = m->p.mfp;
    return 0;
  }
  if (p->n_species > LMC_O_MAX_SPECIES) {
    snprintf(err, (size_t)err_len, "MixtureLayer: too many species");
    return -1;
  }
  L->n_species = p->n_species;
  double mu_s_total = 0.0, mu_a_total = 0.0;
  for (int i = 0; i < p->n_species; ++i) {
    const int mi = p->species[i];
    if (mi < 0 || mi >= h->scene.n_media) {
      snprintf(err, (size_t)err_len, "MixtureLayer: species pointer must not be null.");
      return -1;
    }
    const omedium *sp = &h->media[mi];
    const ophase *ph = &h->phase[sp->phase];
    if (ph->p.kind != LMC_O_PHASE_MIE && ph->p.kind != LMC_O_PHASE_RDEMC) {
      /* PhaseFunction::scattering_cross_section exits for other phase functions */
      snprintf(err, (size_t)err_len, "PhaseFunction::scattering_cross_section: Not implemented");
      return -1;
    }
    const double mu_s = p->number_density[i] * ph->sigma_s;
    L->species[i] = mi;
    L->mu_s_i[i] = mu_s;
    mu_s_total += mu_s;
    if (sp->p.mu_s > 0.0)
      mu_a_total += mu_s * (sp->p.mu_a / sp->p.mu_s);
  }
  if (mu_s_total <= 0.0) {
    snprintf(err, (size_t)err_len, "MixtureLayer: total mu_s must be positive");
    return -1;
  }
  L->mu_s = mu_s_total;
  L->mu_a = mu_a_total;
  L->mu_t = mu_s_total + mu_a_total;
  L->mfp = 1.0 / mu_s_total;
  double acc = 0.0;
  for (int i = 0; i < p->n_species; ++i) {
    acc += L->mu_s_i[i] / mu_s_total;
    L->cdf[i] = acc;
  }
  L->cdf[p->n_species - 1] = 1.0;
  return 0;
}

/* Layer::select_scatter_medium: the lone medium without a draw (HomogeneousLayer),
 * or lower_bound of one uniform on the selection CDF (src/sample.cpp:96-104). */
static int select_scatter_medium(const lmc_o_handle *h, int layer, orng *rng)
{
  const olayer *L = &h->layer[layer];
  if (L->n_species == 0)
    return h->scene.layers[layer].medium;
  const double u = orng_uniform(rng);
  int idx = 0;
  while (idx < L->n_species && L->cdf[idx] < u)
    idx++;
  if (idx >= L->n_species)
    idx = L->n_species - 1;
  return L->species[idx];
}

/* Sensor::check_conditions, src/detector.cpp:374-417 */
static int check_conditions(const osensor *s, v3 hit, v3 dir, int crossing_dir, int events)
{
  const lmc_o_sensor *p = &s->p;
  if (p->f_dir && p->direction != 2 && p->direction != crossing_dir)
    return 0;
  if (p->f_events && (events < p->events_min || events > p->events_max))
    return 0;
  if (p->f_theta) {
    const double costtheta = -1 * dir.z;
    if (costtheta < s->cos_min || costtheta > s->cos_max)
      return 0;
  }
  if (p->f_phi) {
    double phi = atan2(dir.y, dir.x);
    if (phi < 0)
      phi += 2.0 * M_PI;
    if (phi < p->phi_min || phi > p->phi_max)
      return 0;
  }
  if (p->f_pos) {
    if (hit.x < p->x_min || hit.x > p->x_max) return 0;
    if (hit.y < p->y_min || hit.y > p->y_max) return 0;
  }
  return 1;
}

typedef struct {
  v3 point;
  cplx phase;
  int crossing_dir;
  double opticalpath_at_hit;
} ointeraction;

/* ------------------------------------------------------------ adjoint (LR)
 * Score of a photon history: d/d(param) of log(path density x weight), summed
 * over its free flights, albedo factors and HG angle draws.  Free flight from
 * medium a: tau ~ Exp(1), step = mfp_a tau, and at each interface the remaining
 * distance is rescaled by mu_t_old / mu_t_new (src/simulation.cpp:318-382), so the
 * optical depth O = sum_i d_i mu_t_i of a flight is Exp(mean m_a = mfp_a mu_t_a).
 * A flight ending in a scatter in medium c has log density
 * log mu_t_c - log m_a - O / m_a; a flight cut by a sensor hit after depth O has
 * log survival -O / m_a.  Parameters per medium: (mu_a, mu_s, mfp, g). */
#define OADJ_K (4 * LMC_O_MAX_MEDIA)
typedef struct {
  const lmc_o_adjoint *a;
  double *out;
  size_t n_out, radial_off, cbs_off[LMC_O_MAX_SENSORS];
  int K;
  double score[OADJ_K];       /* running score of the photon (completed segments)  */
  double hit_score[OADJ_K];   /* score of the current sensor crossing              */
  int fl_a, fl_cross, seg_med;
  double fl_m, fl_O, seg_len;
  const osensor *sensors0;    /* h->sensors, to tell sensors apart */
} oadj;

static __thread oadj *t_adj;

static void oadj_flight_start(const lmc_o_handle *h, int med)
{
  oadj *A = t_adj;
  A->fl_a = med;
  A->fl_m = h->media[med].p.mfp * h->media[med].mu_t;
  A->fl_O = 0.0;
  A->fl_cross = 0;
}

/* a segment of length d in medium `med` ended at an interface */
static void oadj_segment_done(const lmc_o_handle *h, int med, double d)
{
  oadj *A = t_adj;
  A->score[4 * med + 0] -= d / A->fl_m;
  A->score[4 * med + 1] -= d / A->fl_m;
  A->fl_O += d * h->media[med].mu_t;
  A->fl_cross = 1;
}

/* the flight ended in a scatter in medium c after a last segment of length d */
static void oadj_flight_scatter(const lmc_o_handle *h, int c, double d)
{
  oadj *A = t_adj;
  const int a = A->fl_a;
  const double mfp_a = h->media[a].p.mfp;
  if (!A->fl_cross) {
    A->score[4 * a + 2] += (d / mfp_a - 1.0) / mfp_a;
    return;
  }
  const double mt_a = h->media[a].mu_t, mt_c = h->media[c].mu_t;
  A->score[4 * c + 0] -= d / A->fl_m;
  A->score[4 * c + 1] -= d / A->fl_m;
  const double O = A->fl_O + d * mt_c;
  A->score[4 * c + 0] += 1.0 / mt_c;
  A->score[4 * c + 1] += 1.0 / mt_c;
  A->score[4 * a + 0] += O / (A->fl_m * mt_a) - 1.0 / mt_a;
  A->score[4 * a + 1] += O / (A->fl_m * mt_a) - 1.0 / mt_a;
  A->score[4 * a + 2] += O / (mfp_a * A->fl_m) - 1.0 / mfp_a;
}

/* score of a crossing at fraction t of the current segment */
static void oadj_hit(const lmc_o_handle *h, double t)
{
  oadj *A = t_adj;
  memcpy(A->hit_score, A->score, sizeof(double) * (size_t)A->K);
  const double d = t * A->seg_len;
  const int a = A->fl_a;
  const double mfp_a = h->media[a].p.mfp;
  if (!A->fl_cross) {
    A->hit_score[4 * a + 2] += (d / mfp_a) / mfp_a;
    return;
  }
  const int sm = A->seg_med;
  A->hit_score[4 * sm + 0] -= d / A->fl_m;
  A->hit_score[4 * sm + 1] -= d / A->fl_m;
  const double O = A->fl_O + d * h->media[sm].mu_t;
  A->hit_score[4 * a + 0] += O / (A->fl_m * h->media[a].mu_t);
  A->hit_score[4 * a + 1] += O / (A->fl_m * h->media[a].mu_t);
  A->hit_score[4 * a + 2] += O / (mfp_a * A->fl_m);
}

/* a scatter in medium c with sampled cos(theta): albedo and HG terms */
static void oadj_scatter(const lmc_o_handle *h, const ophase *ph, int c, double cos_theta)
{
  oadj *A = t_adj;
  const omedium *m = &h->media[c];
  if (m->mu_t > 0) {
    A->score[4 * c + 0] += -1.0 / m->mu_t;
    A->score[4 * c + 1] += 1.0 / m->p.mu_s - 1.0 / m->mu_t;
  }
  if (ph->p.kind == LMC_O_PHASE_HG) {
    const double g = ph->p.g;
    A->score[4 * c + 3] += -2.0 * g / (1.0 - g * g) - 3.0 * (g - cos_theta) / (1.0 + g * g - 2.0 * g * cos_theta);
  }
}

static void oadj_add(size_t idx, double v)
{
  oadj *A = t_adj;
  A->out[idx] += v;
  for (int k = 0; k < A->K; ++k)
    A->out[(size_t)(1 + k) * A->n_out + idx] += v * A->hit_score[k];
}

static int time_bin(const osensor *s, double arrival)         /* src/detector.cpp:1182-1190 */
{
  if (s->p.dt <= 0)
    return 0;
  if (arrival < 0 || arrival >= s->p.len_t)
    return -1;
  const int idx = (int)(arrival / s->p.dt) + 1;
  return (idx < s->N_t) ? idx : -1;
}

static void project_to_lab(cplx Em, cplx En, const m3 *P, cplx *Ex, cplx *Ey)  /* :1048-1053 */
{
  *Ex = Em * P->a[0][0] + En * P->a[1][0];
  *Ey = Em * P->a[0][1] + En * P->a[1][1];
}

/* FarFieldCBSSensor::accumulate_stokes, src/detector.cpp:1194-1226 */
static void accumulate_stokes(const osensor *s, double *tally, int it, int jp, int t_idx, cplx Efx,
                              cplx Efy, cplx Erx, cplx Ery)
{
  const cplx Ex = Efx + Erx;
  const cplx Ey = Efy + Ery;
  const double S0c = cnrm(Ex) + cnrm(Ey);
  const double S1c = cnrm(Ex) - cnrm(Ey);
  const double S2c = 2.0 * creal(Ex * conj(Ey));
  const double S3c = 2.0 * cimag(Ex * conj(Ey));
  const double S0i = cnrm(Efx) + cnrm(Efy) + cnrm(Erx) + cnrm(Ery);
  const double S1i = cnrm(Efx) - cnrm(Efy) + cnrm(Erx) - cnrm(Ery);
  const double S2i = 2.0 * (creal(Efx * conj(Efy)) + creal(Erx * conj(Ery)));
  const double S3i = 2.0 * (cimag(Efx * conj(Efy)) + cimag(Erx * conj(Ery)));
  const double v[8] = {S0c, S1c, S2c, S3c, S0i, S1i, S2i, S3i};
  const size_t plane = (size_t)s->N_t * s->N_theta * s->N_phi;
  for (int pass = 0; pass < 2; ++pass) {
    const int t = pass == 0 ? 0 : t_idx;
    if (pass == 1 && t_idx < 1)
      break;
    const size_t off = ((size_t)t * s->N_theta + it) * s->N_phi + jp;
    for (int q = 0; q < 8; ++q)
      tally[q * plane + off] += v[q];
  }
}

/* Stages A+B of the reverse path, src/detector.cpp:1080-1118. */
static void reverse_field_prefix(const lmc_o_handle *h, const m3 *P0, const m3 *Pnm1,
                                 const cplx *Traw, int med_n, cplx Ein_m, cplx Ein_n, cplx *Eo_m,
                                 cplx *Eo_n)
{
  const v3 s0 = m3row(P0, 2), snm1 = m3row(Pnm1, 2);
  const v3 m0 = m3row(P0, 0), n0 = m3row(P0, 1);
  const v3 mnm1 = m3row(Pnm1, 0), nnm1 = m3row(Pnm1, 1);
  const v3 s_in_a = s0;
  const v3 s_out_a = v3scale(snm1, -1.0);
  const double th_a = acos(clamp_pm1(v3dot(s_in_a, s_out_a)));
  cplx Sa2, Sa1;
  omedium_smatrix(&h->media[med_n], th_a, &Sa2, &Sa1);
  const v3 nprime = safe_unit(v3cross(s_in_a, s_out_a), n0);
  const v3 mprime_in = safe_unit(v3cross(nprime, s_in_a), m0);
  const v3 mprime_out = safe_unit(v3cross(nprime, s_out_a), mnm1);
  /* SR_a = S_a * rot2(mprime_in, nprime, m0, n0); E = SR_a * Ein */
  const rot2_t R = rot2(mprime_in, nprime, m0, n0);
  const cplx SR00 = Sa2 * R.r00, SR01 = Sa2 * R.r01, SR10 = Sa1 * R.r10, SR11 = Sa1 * R.r11;
  cplx Em = SR00 * Ein_m + SR01 * Ein_n;
  cplx En = SR10 * Ein_m + SR11 * Ein_n;
  /* R(phi_n'): -> (m_{n-1}, -n_{n-1}) */
  const rot2_t R2 = rot2(mnm1, v3scale(nnm1, -1.0), mprime_out, nprime);
  cplx tm = R2.r00 * Em + R2.r01 * En;
  cplx tn = R2.r10 * Em + R2.r11 * En;
  /* Stage B: E <- Q T^T Q E, Q = diag(1, -1) */
  tn = -tn;
  Em = Traw[0] * tm + Traw[2] * tn;       /* Tt = transpose(T_raw) */
  En = Traw[1] * tm + Traw[3] * tn;
  *Eo_m = Em;
  *Eo_n = -En;
}

/* Stage C + normalisation, src/detector.cpp:1125-1161. */
static void reverse_field_suffix(const lmc_o_handle *h, const m3 *P1, const m3 *Pn, int med_1,
                                 cplx Ep_m, cplx Ep_n, cplx *Eo_m, cplx *Eo_n)
{
  const v3 s1 = m3row(P1, 2), sn = m3row(Pn, 2);
  const v3 m1 = m3row(P1, 0), n1 = m3row(P1, 1);
  const v3 mn = m3row(Pn, 0), nn = m3row(Pn, 1);
  const v3 s_in_c = v3scale(s1, -1.0);
  const v3 s_out_c = sn;
  const double th_c = acos(clamp_pm1(v3dot(s_in_c, s_out_c)));
  cplx Sc2, Sc1;
  omedium_smatrix(&h->media[med_1], th_c, &Sc2, &Sc1);
  const v3 npp = safe_unit(v3cross(s_in_c, s_out_c), v3scale(n1, -1.0));
  const v3 mpp_in = safe_unit(v3cross(npp, s_in_c), m1);
  const v3 mpp_out = safe_unit(v3cross(npp, s_out_c), mn);
  const rot2_t R = rot2(mpp_in, npp, m1, v3scale(n1, -1.0));
  const cplx SR00 = Sc2 * R.r00, SR01 = Sc2 * R.r01, SR10 = Sc1 * R.r10, SR11 = Sc1 * R.r11;
  const cplx Em = SR00 * Ep_m + SR01 * Ep_n;
  const cplx En = SR10 * Ep_m + SR11 * Ep_n;
  const rot2_t R2 = rot2(mn, nn, mpp_out, npp);
  cplx fm = R2.r00 * Em + R2.r01 * En;
  cplx fn = R2.r10 * Em + R2.r11 * En;
  const double nrm = sqrt(cnrm(fm) + cnrm(fn));
  if (nrm > 1e-300) {
    fm = fm / nrm;
    fn = fn / nrm;
  } else {
    fm = 0;
    fn = 0;
  }
  *Eo_m = fm;
  *Eo_n = fn;
}

/* adjoint outputs of a FarFieldCBS hit: S0 coherent and incoherent, the bins
 * accumulate_stokes fills */
static void oadj_cbs(const lmc_o_handle *h, const osensor *s, int it, int jp, int t_idx, cplx Efx,
                     cplx Efy, cplx Erx, cplx Ery)
{
  const size_t si = (size_t)(s - h->sensors);
  const cplx Ex = Efx + Erx, Ey = Efy + Ery;
  const double S0c = cnrm(Ex) + cnrm(Ey);
  const double S0i = cnrm(Efx) + cnrm(Efy) + cnrm(Erx) + cnrm(Ery);
  const size_t plane = (size_t)s->N_t * s->N_theta * s->N_phi;
  for (int pass = 0; pass < 2; ++pass) {
    const int t = pass == 0 ? 0 : t_idx;
    if (pass == 1 && t_idx < 1)
      break;
    const size_t off = t_adj->cbs_off[si] + ((size_t)t * s->N_theta + it) * s->N_phi + jp;
    oadj_add(off, S0c);
    oadj_add(off + plane, S0i);
  }
}

/* FarFieldCBSSensor::process_hit, src/detector.cpp:1231-1310; the far-field
 * fluence sensor uses the same binning with the reverse field set to zero. */
static void process_hit_farfield(const lmc_o_handle *h, const osensor *s, double *tally, ophoton *ph,
                                 const ointeraction *info, uint64_t *hits)
{
  const int t_idx = time_bin(s, ph->launch_time + info->opticalpath_at_hit / ph->velocity);
  if (t_idx < 0)
    return;
  const m3 *P = &ph->P;
  const v3 s_out = m3row(P, 2);
  const double theta = acos(-s_out.z);
  double phi = atan2(s_out.y, s_out.x);
  if (phi < 0)
    phi += 2.0 * M_PI;
  const int it = (int)(theta / s->p.dtheta);
  const int jp = (int)(phi / s->p.dphi);
  if (it < 0 || it >= s->N_theta || jp < 0 || jp >= s->N_phi)
    return;
  if (s->p.kind == LMC_O_SENSOR_FARFIELD_FLUENCE || ph->events < 2) {
    const double w_sqrt = sqrt(ph->weight);
    const cplx Efm = ph->Em * info->phase * w_sqrt;
    const cplx Efn = ph->En * info->phase * w_sqrt;
    cplx Efx, Efy;
    project_to_lab(Efm, Efn, P, &Efx, &Efy);
    if (s->p.kind == LMC_O_SENSOR_FARFIELD_FLUENCE) {
      const double v[4] = {cnrm(Efx) + cnrm(Efy), cnrm(Efx) - cnrm(Efy),
                           2.0 * creal(Efx * conj(Efy)), 2.0 * cimag(Efx * conj(Efy))};
      const size_t plane = (size_t)s->N_t * s->N_theta * s->N_phi;
      for (int pass = 0; pass < 2; ++pass) {
        const int t = pass == 0 ? 0 : t_idx;
        if (pass == 1 && t_idx < 1)
          break;
        const size_t off = ((size_t)t * s->N_theta + it) * s->N_phi + jp;
        for (int q = 0; q < 4; ++q)
          tally[q * plane + off] += v[q];
      }
    } else {
      accumulate_stokes(s, tally, it, jp, t_idx, Efx, Efy, 0.0, 0.0);
      if (t_adj)
        oadj_cbs(h, s, it, jp, t_idx, Efx, Efy, 0.0, 0.0);
    }
    *hits += 1;
    return;
  }
  cplx pm, pn, Erm, Ern;
  reverse_field_prefix(h, &ph->P0, &ph->Pn1, ph->Traw, ph->last_medium, ph->E0m, ph->E0n, &pm, &pn);
  reverse_field_suffix(h, &ph->P1, &ph->Pn, ph->first_medium, pm, pn, &Erm, &Ern);
  ph->Erm = Erm;
  ph->Ern = Ern;
  const v3 s_in = m3row(&ph->P0, 2);
  const v3 qb = v3scale(v3add(s_out, s_in), ph->k);
  const cplx path_phase = cexp(CMPLX(0.0, v3dot(qb, v3sub(ph->rn, ph->r1))));
  const cplx amp = info->phase * sqrt(ph->weight);
  const cplx Efm = ph->Em * amp, Efn = ph->En * amp;
  const cplx Ermm = Erm * amp * path_phase, Ernn = Ern * amp * path_phase;
  cplx Efx, Efy, Erx, Ery;
  project_to_lab(Efm, Efn, P, &Efx, &Efy);
  project_to_lab(Ermm, Ernn, P, &Erx, &Ery);
  accumulate_stokes(s, tally, it, jp, t_idx, Efx, Efy, Erx, Ery);
  if (t_adj)
    oadj_cbs(h, s, it, jp, t_idx, Efx, Efy, Erx, Ery);
  *hits += 1;
}

/* PlanarFluenceSensor::process_hit, src/detector.cpp:780-841 */
static void process_hit_fluence(const osensor *s, double *tally, const ophoton *ph,
                                const ointeraction *info, uint64_t *hits)
{
  const lmc_o_sensor *p = &s->p;
  int t_idx = -1;
  if (p->dt > 0) {
    const double arrival = ph->launch_time + (info->opticalpath_at_hit / ph->velocity);
    if (arrival < 0 || arrival >= p->len_t)
      return;
    t_idx = (int)(arrival / p->dt) + 1;
    if (t_idx >= s->N_t)
      return;
  }
  const int x_idx = (int)((info->point.x + 0.5 * p->len_x) / p->dx);
  const int y_idx = (int)((info->point.y + 0.5 * p->len_y) / p->dy);
  if (x_idx < 0 || x_idx >= s->N_x || y_idx < 0 || y_idx >= s->N_y)
    return;
  const double w_sqrt = sqrt(ph->weight);
  const cplx Em = ph->Em * info->phase * w_sqrt;
  const cplx En = ph->En * info->phase * w_sqrt;
  const cplx Edx = (Em * ph->P.a[0][0] + En * ph->P.a[1][0]) * -1.0;
  const cplx Edy = (Em * ph->P.a[0][1] + En * ph->P.a[1][1]);
  const double v[4] = {cnrm(Edx) + cnrm(Edy), cnrm(Edx) - cnrm(Edy), 2.0 * creal(Edx * conj(Edy)),
                       2.0 * cimag(Edx * conj(Edy))};
  const size_t plane = (size_t)s->N_t * s->N_x * s->N_y;
  if (p->dt > 0) {
    const size_t off = ((size_t)t_idx * s->N_x + x_idx) * s->N_y + y_idx;
    for (int q = 0; q < 4; ++q)
      tally[q * plane + off] += v[q];
  }
  const size_t off0 = (size_t)x_idx * s->N_y + y_idx;
  for (int q = 0; q < 4; ++q)
    tally[q * plane + off0] += v[q];
  if (t_adj && (int)(s - t_adj->sensors0) == t_adj->a->radial_sensor) {
    const size_t r0 = t_adj->radial_off;
    oadj_add(r0, v[0]);
    const double r = sqrt(info->point.x * info->point.x + info->point.y * info->point.y);
    if (r < t_adj->a->radial_max) {
      const int ir = (int)(r / (t_adj->a->radial_max / t_adj->a->radial_bins));
      if (ir >= 0 && ir < t_adj->a->radial_bins)
        oadj_add(r0 + 1 + (size_t)ir, v[0]);
    }
  }
  *hits += 1;
}

/* PlanarFieldSensor::process_hit, src/detector.cpp:546-568 */
static void process_hit_field(const osensor *s, double *tally, const ophoton *ph,
                              const ointeraction *info, uint64_t *hits)
{
  const lmc_o_sensor *p = &s->p;
  const int x_idx = (int)((info->point.x + 0.5 * p->len_x) / p->dx);
  const int y_idx = (int)((info->point.y + 0.5 * p->len_y) / p->dy);
  if (x_idx < 0 || x_idx >= s->N_x || y_idx < 0 || y_idx >= s->N_y)
    return;
  const double w_sqrt = sqrt(ph->weight);
  const cplx Ex = (ph->Em * ph->P.a[0][0] + ph->En * ph->P.a[1][0]) * info->phase * w_sqrt;
  const cplx Ey = (ph->Em * ph->P.a[0][1] + ph->En * ph->P.a[1][1]) * info->phase * w_sqrt;
  const size_t plane = (size_t)s->N_x * s->N_y * 2;
  const size_t off = ((size_t)x_idx * s->N_y + y_idx) * 2;
  tally[off] += creal(Ex);
  tally[off + 1] += cimag(Ex);
  tally[plane + off] += creal(Ey);
  tally[plane + off + 1] += cimag(Ey);
  *hits += 1;
}

/* ------------------------------------------------- last-flight CBS estimator */
/* I_norm = int_0^pi (|S11|^2 + |S22|^2) sin(theta) dtheta, midpoint rule with 2048
 * points (src/detector.cpp:106-118). */
static double compute_I_norm(const omedium *md)
{
  const int n = 2048;
  double acc = 0.0;
  const double dth = M_PI / n;
  for (int i = 0; i < n; i++) {
    const double th = (i + 0.5) * dth;
    cplx S2, S1;
    omedium_smatrix(md, th, &S2, &S1);
    acc += (cnrm(S1) + cnrm(S2)) * sin(th);
  }
  return acc * dth;
}

/* Optical depth along a straight ray, layer by layer (src/detector.cpp:52-102). */
static double optical_depth_to_detector(const lmc_o_handle *h, v3 start, v3 dir, double L_total)
{
  double tau = 0.0, traveled = 0.0;
  v3 p = start;
  int layer = layer_index_at(h, p.z);
  if (layer >= h->scene.n_layers)
    return 0.0;
  if (h->scene.n_layers == 1)
    return layer_at(h, layer)->mu_t * L_total;
  const double dz = dir.z;
  while (traveled < L_total - 1e-15) {
    const double remaining = L_total - traveled;
    const double mu = layer_at(h, layer)->mu_t;
    double seg = remaining;
    if (fabs(dz) > 1e-15) {
      double zi;
      if (find_next_interface(h, p.z, p.z + dz * remaining, &zi)) {
        const double sd = (zi - p.z) / dz;
        if (sd > 1e-15 && sd < remaining)
          seg = sd;
      }
    }
    tau += mu * seg;
    p.x += dir.x * seg;
    p.y += dir.y * seg;
    p.z += dir.z * seg;
    traveled += seg;
    if (seg >= remaining - 1e-15)
      break;
    const double nudge = (dz > 0) ? 1e-12 : -1e-12;
    const int next = layer_index_at(h, p.z + nudge);
    if (next >= h->scene.n_layers)
      break;
    layer = next;
  }
  return tau;
}

/* phase_F (src/detector.cpp:1012-1024) */
static double phase_F(cplx S2, cplx S1, double cos_phi, double sin_phi, cplx Em, cplx En)
{
  const double s22 = cnrm(S2), s11 = cnrm(S1);
  const double Emm = cnrm(Em), Enn = cnrm(En);
  const double c2 = cos_phi * cos_phi, s2 = sin_phi * sin_phi;
  return Emm * (s22 * c2 + s11 * s2) + Enn * (s22 * s2 + s11 * c2) +
         2.0 * creal(Em * conj(En)) * (s22 - s11) * sin_phi * cos_phi;
}

/* scatter_frame (src/detector.cpp:1027-1045): A(theta, phi) P */
static m3 scatter_frame(const m3 *P, double theta, double cos_phi, double sin_phi)
{
  const double ct = cos(theta), st = sin(theta);
  const double A[3][3] = {{ct * cos_phi, ct * sin_phi, -st}, {-sin_phi, cos_phi, 0}, {st * cos_phi, st * sin_phi, ct}};
  m3 out;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = 0.0;
      for (int k = 0; k < 3; ++k)
        acc += A[i][k] * P->a[k][j];
      out.a[i][j] = acc;
    }
  return out;
}

/* apply_scatter_normalized (src/detector.cpp:121-160): (S R(phi)) E / sqrt(F) */
static void apply_scatter_normalized(cplx S2, cplx S1, double cos_phi, double sin_phi, cplx Em, cplx En,
                                     cplx *Om, cplx *On)
{
  const cplx T00 = S2 * cos_phi, T01 = S2 * sin_phi, T10 = S1 * -sin_phi, T11 = S1 * cos_phi;
  const double F = phase_F(S2, S1, cos_phi, sin_phi, Em, En);
  if (F < 1e-300) {
    *Om = 0.0;
    *On = 0.0;
    return;
  }
  const double inv = 1.0 / sqrt(F);
  *Om = inv * (T00 * Em + T01 * En);
  *On = inv * (T10 * Em + T11 * En);
}

/* FarFieldCBSSensor::process_estimation (src/detector.cpp:1315-1566): at every
 * scattering vertex, before the scatter is sampled, the photon is forced toward
 * the centre of every angular bin (theta, phi) of the grid; the bin receives the
 * weight w mu_s/mu_t x transmittance x p(Omega) dOmega with p = F / (pi I_norm),
 * its forward field and, from the second vertex on, its reverse (CBS) field. */
static void estimate_farfield_cbs(const lmc_o_handle *h, const osensor *s, double *tally,
                                  const ophoton *ph, int med_idx, uint64_t *hits)
{
  const lmc_o_sensor *p = &s->p;
  if (p->f_events && ((int)ph->events < p->events_min || (int)ph->events > p->events_max))
    return;
  const omedium *med = &h->media[med_idx];
  const double I_norm = med->I_norm;
  if (I_norm < 1e-300)
    return;
  const v3 e1 = m3row(&ph->P0, 0), e2 = m3row(&ph->P0, 1), s_in = m3row(&ph->P0, 2);
  const v3 e3 = v3scale(s_in, -1.0);
  const m3 *Pcur = &ph->P;
  const v3 m_cur = m3row(Pcur, 0), n_cur = m3row(Pcur, 1), s_cur = m3row(Pcur, 2);
  /* first vertex: the layer's aggregate albedo (src/detector.cpp:1378); later
   * vertices: the selected species' own (:1472).  Equal for a HomogeneousLayer. */
  const olayer *SL = layer_at(h, ph->current_layer);
  const double w_scatter = ph->weight * (ph->events == 0 ? SL->mu_s / SL->mu_t : med->p.mu_s / med->mu_t);
  if (w_scatter < 1e-300)
    return;
  const double th_cap = (p->theta_pp_max > 0.0) ? fmin(p->theta_pp_max, p->theta_max_grid) : p->theta_max_grid;
  int i_max = (int)(th_cap / p->dtheta);
  if (i_max > s->N_theta)
    i_max = s->N_theta;
  const int multi = ph->events >= 1;
  cplx pre_m = 0.0, pre_n = 0.0;
  if (multi) {
    cplx Tmid[4] = {ph->Traw[0], ph->Traw[1], ph->Traw[2], ph->Traw[3]};
    if (ph->events >= 2 && ph->has_T_prev) {
      const cplx *A = ph->Traw_buf, *B = ph->Traw;
      Tmid[0] = A[0] * B[0] + A[1] * B[2];
      Tmid[1] = A[0] * B[1] + A[1] * B[3];
      Tmid[2] = A[2] * B[0] + A[3] * B[2];
      Tmid[3] = A[2] * B[1] + A[3] * B[3];
    }
    reverse_field_prefix(h, &ph->P0, Pcur, Tmid, med_idx, ph->E0m, ph->E0n, &pre_m, &pre_n);
  }
  for (int it = 0; it < i_max; ++it) {
    const double th_det = (it + 0.5) * p->dtheta;
    const double c_th = cos(th_det), s_th = sin(th_det);
    const double dOmega_band = cos(it * p->dtheta) - cos((it + 1) * p->dtheta);
    for (int jp = 0; jp < s->N_phi; ++jp) {
      const double ph_det = (jp + 0.5) * p->dphi;
      const double c_ph = cos(ph_det), s_ph = sin(ph_det);
      const v3 s_out = v3add(v3add(v3scale(e1, s_th * c_ph), v3scale(e2, s_th * s_ph)), v3scale(e3, c_th));
      /* intersect_plane with the sensor plane z = 0, normal +z (src/detector.cpp:35-47) */
      const double denom = s_out.z;
      if (fabs(denom) < 1e-14)
        continue;
      const double L = (-ph->pos.z) / denom;
      if (L <= 0.0)
        continue;
      const double Tr = exp(-optical_depth_to_detector(h, ph->pos, s_out, L));
      if (Tr < 1e-20)
        continue;
      const v3 pv = v3cross(s_cur, s_out);
      const double pn = v3norm(pv);
      if (pn < 1e-12)
        continue;
      const v3 p_hat = v3scale(pv, 1.0 / pn);
      const double sin_phi = -v3dot(m_cur, p_hat);
      const double cos_phi = v3dot(n_cur, p_hat);
      const double th_scat = acos(clamp_pm1(v3dot(s_cur, s_out)));
      cplx S2, S1;
      omedium_smatrix(med, th_scat, &S2, &S1);
      const double F = phase_F(S2, S1, cos_phi, sin_phi, ph->Em, ph->En);
      if (F < 1e-300)
        continue;
      const double prob_bin = (F / (M_PI * I_norm)) * (dOmega_band * p->dphi);
      const double w_bin = w_scatter * Tr * prob_bin;
      if (w_bin < 1e-300)
        continue;
      const cplx amp = sqrt(w_bin) * cexp(CMPLX(0.0, ph->k * L));
      const m3 P_exit = scatter_frame(Pcur, th_scat, cos_phi, sin_phi);
      cplx Efm, Efn;
      apply_scatter_normalized(S2, S1, cos_phi, sin_phi, ph->Em, ph->En, &Efm, &Efn);
      const int t_idx = time_bin(s, ph->launch_time + (ph->opticalpath + L) / ph->velocity);
      if (t_idx < 0)
        continue;
      cplx Efx, Efy, Erx = 0.0, Ery = 0.0;
      project_to_lab(Efm * amp, Efn * amp, &P_exit, &Efx, &Efy);
      if (multi) {
        cplx Erm, Ern;
        reverse_field_suffix(h, &ph->P1, &P_exit, ph->first_medium, pre_m, pre_n, &Erm, &Ern);
        const v3 qb = v3scale(v3add(s_out, s_in), ph->k);
        const cplx path_phase = cexp(CMPLX(0.0, v3dot(qb, v3sub(ph->pos, ph->r1))));
        project_to_lab(Erm * amp * path_phase, Ern * amp * path_phase, &P_exit, &Erx, &Ery);
      }
      accumulate_stokes(s, tally, it, jp, t_idx, Efx, Efy, Erx, Ery);
    }
  }
  *hits += 1;
}

/* StatisticsSensor::process_hit (src/detector.cpp:1720-1800): one count per active
 * histogram, in bin 0 of its time axis and in the arrival-time window.  Bins that
 * would fall past a histogram's end through rounding are skipped. */
static void process_hit_statistics(const osensor *s, double *tally, const ophoton *ph,
                                   const ointeraction *info, uint64_t *hits)
{
  const lmc_o_statistics *q = &s->p.stats;
  const double arrival_time = ph->launch_time + (info->opticalpath_at_hit / ph->velocity);
  int t_idx = -1;
  if (s->N_t > 1 && s->p.dt > 0.0 && arrival_time >= 0.0 && arrival_time < s->p.len_t) {
    t_idx = (int)(arrival_time / s->p.dt) + 1;
    if (t_idx >= s->N_t)
      t_idx = -1;
  }
#define DEPOSIT(off, nb, idx)                                                         \
  do {                                                                                \
    if ((idx) >= 0 && (idx) < (nb)) {                                                 \
      tally[(off) + (size_t)(idx)] += 1.0;                                            \
      if (t_idx >= 1 && t_idx < s->N_t)                                               \
        tally[(off) + (size_t)t_idx * (size_t)(nb) + (size_t)(idx)] += 1.0;           \
    }                                                                                 \
  } while (0)
  if (q->set & LMC_O_STAT_EVENTS) {
    const int events = (int)ph->events;
    if (events >= 0 && events < q->n_events)
      DEPOSIT(s->st_off[0], q->n_events, events);
  }
  if (q->set & LMC_O_STAT_THETA) {
    const double theta = acos(-ph->P.a[2][2]);
    if (theta >= q->theta_min && theta < q->theta_max)
      DEPOSIT(s->st_off[1], q->n_theta, (int)((theta - q->theta_min) / s->st_dtheta));
  }
  if (q->set & LMC_O_STAT_PHI) {
    double phi = atan2(ph->P.a[2][1], ph->P.a[2][0]);
    if (phi < 0)
      phi += 2.0 * M_PI;
    if (phi >= q->phi_min && phi < q->phi_max)
      DEPOSIT(s->st_off[2], q->n_phi, (int)((phi - q->phi_min) / s->st_dphi));
  }
  if (q->set & LMC_O_STAT_DEPTH) {
    const double depth = ph->penetration_depth;
    if (depth >= 0 && depth < q->depth_max)
      DEPOSIT(s->st_off[3], q->n_depth, (int)(depth / s->st_ddepth));
  }
#undef DEPOSIT
  if (q->set & LMC_O_STAT_TIME) {
    const double fi = arrival_time / s->st_dtime;
    if (fi >= 1.0 && fi < (double)q->n_time)
      tally[s->st_off[4] + (size_t)fi] += 1.0;
  }
  if (q->set & LMC_O_STAT_WEIGHT) {
    const double weight = ph->weight;
    if (weight >= 0 && weight < q->weight_max) {
      const int idx = (int)(weight / s->st_dweight);
      if (idx < q->n_weight)
        tally[s->st_off[5] + (size_t)idx] += 1.0;
    }
  }
  *hits += 1;
}

/* SensorsGroup::record_hit, src/detector.cpp:178-270 */
static int record_hit(const lmc_o_handle *h, ophoton *ph, double **tallies, uint64_t *hits)
{
  int killed = 0;
  const double z1 = ph->prev_pos.z, z2 = ph->pos.z;
  if (fabs(z2 - z1) < 1e-12)
    return 0;
  const int crossing_dir = (z2 > z1) ? 0 : 1;
  const double z_min = fmin(z1, z2), z_max = fmax(z1, z2);
  for (int g = 0; g < h->n_planes; ++g) {
    const double z_plane = h->plane_z[g];
    if (!(z_plane >= z_min && z_plane <= z_max))
      continue;
    const v3 xn = ph->prev_pos, xf = ph->pos;
    const v3 d = v3sub(xf, xn);
    const v3 normal = v3make(0, 0, 1);
    const double denom = v3dot(d, normal);
    const double t = v3dot(v3sub(v3make(0, 0, z_plane), xn), normal) / denom;
    const v3 hit = v3add(xn, v3scale(d, t));
    if (t_adj)
      oadj_hit(h, t);
    const double correction = v3norm(v3sub(hit, xf));
    const double n_local = 1.0 / h->light_speed;
    double optical_path_correction = ph->optical_path;
    double opticalpath_at_hit = ph->opticalpath;
    if (correction > 0) {
      optical_path_correction -= correction * n_local;
      opticalpath_at_hit -= correction;
    }
    ointeraction info;
    info.point = hit;
    info.phase = cexp(CMPLX(0.0, ph->k * optical_path_correction));
    info.crossing_dir = crossing_dir;
    info.opticalpath_at_hit = opticalpath_at_hit;
    for (int si = 0; si < h->scene.n_sensors; ++si) {
      const osensor *s = &h->sensors[si];
      if (s->key != g || s->p.estimator)
        continue;
      const v3 direction = m3row(&ph->P, 2);
      if (!check_conditions(s, hit, direction, crossing_dir, (int)ph->events))
        continue;
      const uint64_t before = hits[si];
      if (s->p.kind == LMC_O_SENSOR_FARFIELD_CBS || s->p.kind == LMC_O_SENSOR_FARFIELD_FLUENCE)
        process_hit_farfield(h, s, tallies[si], ph, &info, &hits[si]);
      else if (s->p.kind == LMC_O_SENSOR_PLANAR_FLUENCE)
        process_hit_fluence(s, tallies[si], ph, &info, &hits[si]);
      else if (s->p.kind == LMC_O_SENSOR_PLANAR_FIELD)
        process_hit_field(s, tallies[si], ph, &info, &hits[si]);
      else if (s->p.kind == LMC_O_SENSOR_STATISTICS)
        process_hit_statistics(s, tallies[si], ph, &info, &hits[si]);
      if (hits[si] != before) {
        ph->hit = hit;
        ph->n_hits++;
      }
      if (s->p.absorb)
        killed = 1;
    }
  }
  return killed;
}

/* Laser::emit_photon + the driver's per-photon set-up (src/laser.cpp:77-99,
 * :42-75, :11-28; src/photon.cpp:24-53; src/simulation.cpp:197-201). */
static void emit_photon(const lmc_o_handle *h, orng *rng, ophoton *ph)
{
  const lmc_o_laser *L = &h->scene.laser;
  memset(ph, 0, sizeof(*ph));
  v3 c = v3make(L->position[0], L->position[1], L->position[2]);
  v3 pos = c;
  if (L->source == 1) {
    const double theta = orng_uniform(rng) * 2.0 * M_PI;
    const double r = sqrt(orng_uniform(rng)) * L->sigma;
    pos = v3make(c.x + r * cos(theta), c.y + r * sin(theta), c.z);
  } else if (L->source == 2) {
    const double x = orng_normal(rng, c.x, L->sigma);
    const double y = orng_normal(rng, c.y, L->sigma);
    pos = v3make(x, y, c.z);
  }
  ph->pos = pos;
  ph->prev_pos = pos;
  ph->k = 2.0 * M_PI / L->wavelength;
  for (int j = 0; j < 3; ++j) {
    ph->P.a[0][j] = L->local_m[j];
    ph->P.a[1][j] = L->local_n[j];
    ph->P.a[2][j] = L->direction[j];
  }
  ph->Em = CMPLX(L->pol[0], L->pol[1]);
  ph->En = CMPLX(L->pol[2], L->pol[3]);
  const double PS_TO_NS = 1e-3;
  const double FWHM_TO_SIGMA = 1.0 / (2.0 * sqrt(2.0 * log(2.0)));
  const double t0 = L->time_offset * PS_TO_NS;
  double t = t0;
  switch (L->temporal) {
  case 1: t = orng_normal(rng, t0, L->pulse_duration * FWHM_TO_SIGMA * PS_TO_NS); break;
  case 2: t = t0 + (orng_uniform(rng) - 0.5) * L->pulse_duration * PS_TO_NS; break;
  case 3: t = t0 - log(orng_uniform(rng)) * L->pulse_duration * PS_TO_NS; break;
  case 4: t = (L->repetition_rate <= 0.0) ? t0 : t0 + orng_uniform(rng) * (1e9 / L->repetition_rate); break;
  case 5: t = (L->pulse_duration <= 0.0) ? t0 : t0 + orng_uniform(rng) * L->pulse_duration * PS_TO_NS; break;
  default: break;
  }
  ph->launch_time = t;
  ph->velocity = 1.0;
  ph->weight = 1.0;
  ph->alive = 1;
  ph->current_layer = layer_index_at(h, ph->pos.z);
}

/* Absorption::record_absorption (src/absortion.cpp:54-91): the deposit at the
 * photon's position in slice 0 and, time-resolved, in the slice of its arrival time. */
static void record_absorption(const lmc_o_handle *h, const ophoton *ph, double d_weight, double *grid)
{
  const lmc_o_absorption *A = &h->scene.absorption;
  const double r = sqrt(ph->pos.x * ph->pos.x + ph->pos.y * ph->pos.y);
  const double z = ph->pos.z;
  if (r > A->radius || z < 0.0 || z > A->depth)
    return;
  const double fr = floor(r / A->d_r), fz = floor(z / A->d_z);
  if (fr >= (double)h->abs_nr || fz >= (double)h->abs_nz)
    return;
  const size_t cell = (size_t)fr * (size_t)h->abs_nz + (size_t)fz;
  grid[cell] += d_weight;
  if (A->d_t > 0.0) {
    const double time = ph->launch_time + (ph->opticalpath / ph->velocity);
    const double fk = floor(time / A->d_t) + 1.0;
    if (fk >= 1.0 && fk < (double)h->abs_nt)
      grid[(size_t)fk * (size_t)h->abs_nr * (size_t)h->abs_nz + cell] += d_weight;
  }
}

/* run_photon, src/simulation.cpp:255-617 */
static void run_photon(const lmc_o_handle *h, ophoton *ph, orng *rng, int track, int max_events,
                       double **tallies, uint64_t *hits, lmc_o_stats *st)
{
  ph->r1 = ph->pos;
  ph->rn = ph->pos;
  ph->P0 = ph->P;
  ph->P1 = ph->P;
  ph->Pn1 = ph->P;
  ph->Pn = ph->P;
  ph->E0m = ph->Em;
  ph->E0n = ph->En;
  ph->Traw[0] = 1; ph->Traw[1] = 0; ph->Traw[2] = 0; ph->Traw[3] = 1;
  ph->Traw_buf[0] = 1; ph->Traw_buf[1] = 0; ph->Traw_buf[2] = 0; ph->Traw_buf[3] = 1;
  ph->has_T_prev = 0;
  ph->active_medium = ph->first_medium = ph->last_medium = -1;
  const double n_step = 1.0 / h->light_speed;
  if (t_adj)
    memset(t_adj->score, 0, sizeof(t_adj->score));

  while (ph->alive) {
    const olayer *cur = layer_at(h, ph->current_layer);
    double step = -1 * cur->mfp * log(orng_uniform(rng));        /* medium.cpp:123-126, sample.cpp:90-94 */
    if (t_adj)
      oadj_flight_start(h, h->scene.layers[ph->current_layer].medium);
    st->steps++;
    const double dir_x = ph->P.a[2][0], dir_y = ph->P.a[2][1], dir_z = ph->P.a[2][2];
    double new_z = ph->pos.z + dir_z * step;
    double z_iface;
    int found = find_next_interface(h, ph->pos.z, new_z, &z_iface);   /* :318-382 */
    while (found) {
      const double dz_total = dir_z * step;
      if (fabs(dz_total) < 1e-15)
        break;
      const double t = (z_iface - ph->pos.z) / dz_total;
      if (t < 0.0 || t > 1.0)
        break;
      const double step_to_iface = step * t;
      const double remaining_optical = (step - step_to_iface) * layer_at(h, ph->current_layer)->mu_t;
      ph->opticalpath += step_to_iface;
      ph->optical_path += n_step * step_to_iface;
      ph->prev_pos = ph->pos;
      ph->pos.x += dir_x * step_to_iface;
      ph->pos.y += dir_y * step_to_iface;
      const double nudge = (dir_z > 0) ? 1e-12 : -1e-12;
      ph->pos.z = z_iface + nudge;
      if (t_adj) {
        t_adj->seg_med = h->scene.layers[ph->current_layer].medium;
        t_adj->seg_len = step_to_iface;
      }
      if (record_hit(h, ph, tallies, hits)) {
        ph->alive = 0;
        ph->fate = LMC_O_FATE_DETECTED;
        break;
      }
      if (t_adj)
        oadj_segment_done(h, h->scene.layers[ph->current_layer].medium, step_to_iface);
      const int new_layer = layer_index_at(h, ph->pos.z);
      if (new_layer >= h->scene.n_layers) {
        ph->alive = 0;
        ph->fate = LMC_O_FATE_STACK;
        break;
      }
      ph->current_layer = new_layer;
      const double new_mu_t = layer_at(h, ph->current_layer)->mu_t;
      if (new_mu_t > 0)
        step = remaining_optical / new_mu_t;
      else
        step = remaining_optical;
      new_z = ph->pos.z + dir_z * step;
      found = find_next_interface(h, ph->pos.z, new_z, &z_iface);
    }
    if (!ph->alive)
      break;

    ph->opticalpath += step;                                    /* :389-400 */
    ph->optical_path += n_step * step;
    ph->prev_pos = ph->pos;
    ph->pos.x += dir_x * step;
    ph->pos.y += dir_y * step;
    ph->pos.z += dir_z * step;
    if (ph->pos.z > ph->penetration_depth)
      ph->penetration_depth = ph->pos.z;
    const int last_seg_med = h->scene.layers[ph->current_layer].medium;
    if (t_adj) {
      t_adj->seg_med = last_seg_med;
      t_adj->seg_len = step;
    }

    if (record_hit(h, ph, tallies, hits)) {                     /* :403-408 */
      ph->alive = 0;
      ph->fate = LMC_O_FATE_DETECTED;
      break;
    }
    if (!is_inside(h, ph->pos)) {                               /* :411-416 */
      ph->alive = 0;
      ph->fate = LMC_O_FATE_ESCAPED;
      break;
    }
    ph->current_layer = layer_index_at(h, ph->pos.z);
    const int scatter_layer = ph->current_layer;
    const int med_idx = select_scatter_medium(h, scatter_layer, rng);  /* :419-426 */
    const omedium *sm = &h->media[med_idx];
    ph->active_medium = med_idx;
    for (int si = 0; si < h->scene.n_sensors; ++si) {             /* :419-426 run_estimators */
      const osensor *es = &h->sensors[si];
      if (es->p.estimator && es->p.kind == LMC_O_SENSOR_FARFIELD_CBS)
        estimate_farfield_cbs(h, es, tallies[si], ph, med_idx, &hits[si]);
    }
    if (t_adj)
      oadj_flight_scatter(h, last_seg_med, step);

    const double theta = ophase_sample_theta(&h->phase[sm->phase], orng_uniform(rng));  /* :429 */
    cplx S2, S1;
    omedium_smatrix(sm, theta, &S2, &S1);                       /* :430 */
    double phi;
    {                                                           /* phase.cpp:27-49 */
      const double s2sq = cnrm(S2), s1sq = cnrm(S1);
      const double e1sq = cnrm(ph->Em), e2sq = cnrm(ph->En);
      const double e12 = creal(ph->Em * conj(ph->En));
      const double a = s2sq * e1sq + s1sq * e2sq;
      const double b = s1sq * e1sq + s2sq * e2sq;
      const double c = 2.0 * (s2sq - s1sq) * e12;
      const double diff = (a - b);
      const double Fmax = 0.5 * (a + b) + 0.5 * sqrt(diff * diff + c * c);
      for (;;) {
        const double phi_try = 2.0 * M_PI * orng_uniform(rng);
        const double cp = cos(phi_try), sp = sin(phi_try);
        const double F = a * cp * cp + b * sp * sp + c * cp * sp;
        const double Fclamped = fmax(F, 0.0);
        if (orng_uniform(rng) * Fmax <= Fclamped) {
          phi = phi_try;
          break;
        }
      }
    }
    const double cos_theta = cos(theta), sin_theta = sin(theta);     /* :438-453 */
    const double cos_phi = cos(phi), sin_phi = sin(phi);
    if (t_adj)
      oadj_scatter(h, &h->phase[sm->phase], med_idx, cos_theta);
    {
      double A[3][3] = {{cos_theta * cos_phi, cos_theta * sin_phi, -sin_theta},
                        {-sin_phi, cos_phi, 0},
                        {sin_theta * cos_phi, sin_theta * sin_phi, cos_theta}};
      m3 np;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double acc = 0.0;
          for (int k = 0; k < 3; ++k)
            acc += A[i][k] * ph->P.a[k][j];
          np.a[i][j] = acc;
        }
      ph->P = np;
    }
    {                                                           /* :456-492 */
      cplx T00 = S2 * cos_phi, T01 = S2 * sin_phi, T10 = S1 * -sin_phi, T11 = S1 * cos_phi;
      const cplx Em = ph->Em, En = ph->En;
      const double Emm = cnrm(Em), Enn = cnrm(En);
      const double s22 = cnrm(S2), s11 = cnrm(S1);
      const double pow_cos_phi = cos_phi * cos_phi, pow_sin_phi = sin_phi * sin_phi;
      const double F = Emm * (s22 * pow_cos_phi + s11 * pow_sin_phi) +
                       Enn * (s22 * pow_sin_phi + s11 * pow_cos_phi) +
                       2.0 * creal(Em * conj(En)) * (s22 - s11) * sin_phi * cos_phi;
      const double F_inv_sqrt = 1.0 / sqrt(F);
      T00 = T00 * F_inv_sqrt; T01 = T01 * F_inv_sqrt; T10 = T10 * F_inv_sqrt; T11 = T11 * F_inv_sqrt;
      ph->Em = (T00 * Em + T01 * En);
      ph->En = (T10 * Em + T11 * En);

      if (track) {                                              /* :495-568 */
        const cplx Tr[4] = {S2 * cos_phi, S2 * sin_phi, -S1 * sin_phi, S1 * cos_phi};
        const unsigned evt = ph->events + 1;
        if (evt == 1) {
          ph->r1 = ph->pos;
          ph->first_medium = ph->active_medium;
          ph->P1 = ph->P;
        }
        ph->rn = ph->pos;
        ph->last_medium = ph->active_medium;
        ph->Pn1 = ph->Pn;
        ph->Pn = ph->P;
        if (evt >= 2) {
          if (!ph->has_T_prev) {
            for (int q = 0; q < 4; ++q)
              ph->Traw_buf[q] = Tr[q];
            ph->has_T_prev = 1;
          } else {
            const cplx *A = ph->Traw_buf, *B = ph->Traw;
            cplx t[4];
            t[0] = A[0] * B[0] + A[1] * B[2];
            t[1] = A[0] * B[1] + A[1] * B[3];
            t[2] = A[2] * B[0] + A[3] * B[2];
            t[3] = A[2] * B[1] + A[3] * B[3];
            const double frob = sqrt(cnrm(t[0]) + cnrm(t[1]) + cnrm(t[2]) + cnrm(t[3]));
            if (frob > 1e-300)
              for (int q = 0; q < 4; ++q)
                t[q] = t[q] / frob;
            for (int q = 0; q < 4; ++q) {
              ph->Traw[q] = t[q];
              ph->Traw_buf[q] = Tr[q];
            }
          }
        }
      }
    }
    ph->events++;                                               /* :578-587 */
    st->events++;
    const olayer *SL = layer_at(h, scatter_layer);             /* the layer's aggregate albedo */
    const double layer_mu_t = SL->mu_t;
    double d_weight = 1.0;
    if (layer_mu_t > 0) {
      const double absorption_prob = SL->mu_a / layer_mu_t;
      const double scattering_prob = SL->mu_s / layer_mu_t;
      d_weight = ph->weight * absorption_prob;
      ph->weight *= scattering_prob;
    }
    if (h->scene.absorption.enabled)                            /* :589-592 */
      record_absorption(h, ph, d_weight, tallies[h->scene.n_sensors]);
    if (ph->weight < 1e-4) {                                    /* :596-607 */
      if (orng_uniform(rng) < 0.1) {
        ph->weight /= 0.1;
      } else {
        ph->alive = 0;
        ph->fate = LMC_O_FATE_ROULETTE;
        break;
      }
    }
    if ((int)ph->events > max_events) {                         /* :609-613 */
      ph->alive = 0;
      ph->fate = LMC_O_FATE_EVENT_CAP;
      break;
    }
  }
}

/* --------------------------------------------------------------- public API */
lmc_o_handle *lmc_oracle_create(const lmc_o_scene *scene, char *err, int err_len)
{
  char dummy[8];
  if (!err) { err = dummy; err_len = (int)sizeof(dummy); }
  err[0] = 0;
  if (scene->n_layers < 1 || scene->n_layers > LMC_O_MAX_LAYERS || scene->n_media > LMC_O_MAX_MEDIA ||
      scene->n_phase > LMC_O_MAX_PHASE || scene->n_sensors > LMC_O_MAX_SENSORS) {
    snprintf(err, (size_t)err_len, "scene sizes out of range");
    return NULL;
  }
  lmc_o_handle *h = (lmc_o_handle *)calloc(1, sizeof(lmc_o_handle));
  h->scene = *scene;
  h->light_speed = 1.0 / scene->n_host;
  for (int i = 0; i < scene->n_phase; ++i)
    if (ophase_init(&h->phase[i], &scene->phase[i]) != 0) {
      snprintf(err, (size_t)err_len, "phase function %d: bad parameters", i);
      lmc_oracle_destroy(h);
      return NULL;
    }
  for (int i = 0; i < scene->n_media; ++i) {
    if (omedium_init(&h->media[i], &scene->media[i]) != 0) {
      snprintf(err, (size_t)err_len, "medium %d: bad parameters", i);
      lmc_oracle_destroy(h);
      return NULL;
    }
    h->media[i].I_norm = compute_I_norm(&h->media[i]);
  }
  for (int l = 0; l < scene->n_layers; ++l) {
    const lmc_o_layer *L = &scene->layers[l];
    if (L->n_species <= 0 && (L->medium < 0 || L->medium >= scene->n_media)) {
      snprintf(err, (size_t)err_len, "Sample::add_layer: medium pointer must not be null.");
      lmc_oracle_destroy(h);
      return NULL;
    }
    if (olayer_init(h, L, &h->layer[l], err, err_len) != 0) {
      lmc_oracle_destroy(h);
      return NULL;
    }
  }
  for (int l = 1; l < scene->n_layers; ++l)                     /* sample.cpp:155-158 */
    h->interfaces[h->n_interfaces++] = scene->layers[l].z_min;
  if (scene->absorption.enabled) {                             /* absortion.cpp:13-32 */
    const lmc_o_absorption *A = &scene->absorption;
    if (!(A->d_r > 0.0) || !(A->d_z > 0.0) || !(A->radius >= 0.0) || !(A->depth >= 0.0) ||
        !(A->d_t >= 0.0) || (A->d_t > 0.0 && !(A->t_max >= 0.0)) ||
        A->radius / A->d_r > 1e7 || A->depth / A->d_z > 1e7 ||
        (A->d_t > 0.0 && A->t_max / A->d_t > 1e6)) {
      snprintf(err, (size_t)err_len, "Absorption: bin widths must be positive and the grid bounded");
      lmc_oracle_destroy(h);
      return NULL;
    }
    h->abs_nt = (A->d_t > 0.0) ? (int)ceil(A->t_max / A->d_t) + 1 : 1;
    h->abs_nr = (int)(A->radius / A->d_r) + 1;
    h->abs_nz = (int)(A->depth / A->d_z) + 1;
  }
  /* z_layers (detector.hpp:46-48, detector.cpp:166-176): a key per plane within 1e-9 */
  for (int si = 0; si < scene->n_sensors; ++si) {
    if (osensor_init(h, &h->sensors[si], &scene->sensors[si], err, err_len) != 0) {
      lmc_oracle_destroy(h);
      return NULL;
    }
    const double z = h->sensors[si].p.z;
    int g = -1;
    for (int k = 0; k < h->n_planes; ++k)
      if (!(h->plane_z[k] < z - 1e-9) && !(z < h->plane_z[k] - 1e-9))
        g = k;
    if (g < 0) {
      int pos = h->n_planes;
      while (pos > 0 && h->plane_z[pos - 1] > z) {
        h->plane_z[pos] = h->plane_z[pos - 1];
        for (int q = 0; q < si; ++q)
          if (h->sensors[q].key == pos - 1)
            h->sensors[q].key = pos;
        pos--;
      }
      h->plane_z[pos] = z;
      h->n_planes++;
      g = pos;
    }
    h->sensors[si].key = g;
  }
  return h;
}

void lmc_oracle_destroy(lmc_o_handle *h)
{
  if (!h)
    return;
  for (int i = 0; i < LMC_O_MAX_PHASE; ++i) {
    free(h->phase[i].table.values);
    free(h->phase[i].table.cdf);
  }
  for (int i = 0; i < LMC_O_MAX_MEDIA; ++i) {
    free(h->media[i].S1.y);
    free(h->media[i].S2.y);
  }
  free(h);
}

int lmc_oracle_sensor_shape(const lmc_o_handle *h, int sensor, int dims[4], size_t *n_doubles)
{
  if (sensor == h->scene.n_sensors && h->scene.absorption.enabled) {
    dims[0] = h->abs_nt; dims[1] = h->abs_nr; dims[2] = h->abs_nz; dims[3] = 1;
    *n_doubles = (size_t)h->abs_nt * (size_t)h->abs_nr * (size_t)h->abs_nz;
    return 0;
  }
  if (sensor < 0 || sensor >= h->scene.n_sensors)
    return -1;
  const osensor *s = &h->sensors[sensor];
  switch (s->p.kind) {
  case LMC_O_SENSOR_FARFIELD_CBS:
    dims[0] = 8; dims[1] = s->N_t; dims[2] = s->N_theta; dims[3] = s->N_phi; break;
  case LMC_O_SENSOR_FARFIELD_FLUENCE:
    dims[0] = 4; dims[1] = s->N_t; dims[2] = s->N_theta; dims[3] = s->N_phi; break;
  case LMC_O_SENSOR_PLANAR_FLUENCE:
    dims[0] = 4; dims[1] = s->N_t; dims[2] = s->N_x; dims[3] = s->N_y; break;
  case LMC_O_SENSOR_STATISTICS:
    dims[0] = s->N_t; dims[1] = (int)s->n_doubles; dims[2] = 0; dims[3] = 0; break;
  default:
    dims[0] = 2; dims[1] = s->N_x; dims[2] = s->N_y; dims[3] = 2; break;
  }
  *n_doubles = s->n_doubles;
  return 0;
}

int lmc_oracle_run(lmc_o_handle *h, uint64_t seed, uint64_t begin, uint64_t count, int rng_kind,
                   int max_events, int track_reverse, double **tallies, uint64_t *hits,
                   lmc_o_record *records, lmc_o_stats *stats)
{
  lmc_o_stats local;
  memset(&local, 0, sizeof(local));
  orng rng;
  memset(&rng, 0, sizeof(rng));
  rng.kind = rng_kind;
  for (uint64_t i = begin; i < begin + count; ++i) {
    orng_seed_photon(&rng, seed, i);
    ophoton ph;
    emit_photon(h, &rng, &ph);
    if (ph.current_layer >= h->scene.n_layers)
      return -2;   /* the reference throws std::out_of_range from Sample::get_layer */
    run_photon(h, &ph, &rng, track_reverse, max_events, tallies, hits, &local);
    local.photons++;
    local.draws += rng.draw;
    switch (ph.fate) {
    case LMC_O_FATE_DETECTED: local.detected++; break;
    case LMC_O_FATE_ESCAPED: local.escaped++; break;
    case LMC_O_FATE_STACK: local.stack++; break;
    case LMC_O_FATE_ROULETTE: local.roulette++; break;
    default: local.cap++; break;
    }
    if (records) {
      lmc_o_record *r = &records[i - begin];
      memset(r, 0, sizeof(*r));
      r->photon = i;
      r->events = ph.events;
      r->draws = (uint32_t)rng.draw;
      r->fate = ph.fate;
      r->layer = ph.current_layer;
      r->weight = ph.weight;
      r->opticalpath = ph.opticalpath;
      r->penetration_depth = ph.penetration_depth;
      r->launch_time = ph.launch_time;
      r->pos[0] = ph.pos.x; r->pos[1] = ph.pos.y; r->pos[2] = ph.pos.z;
      for (int j = 0; j < 3; ++j) {
        r->m[j] = ph.P.a[0][j];
        r->n[j] = ph.P.a[1][j];
        r->dir[j] = ph.P.a[2][j];
      }
      r->E[0] = creal(ph.Em); r->E[1] = cimag(ph.Em); r->E[2] = creal(ph.En); r->E[3] = cimag(ph.En);
      r->r1[0] = ph.r1.x; r->r1[1] = ph.r1.y; r->r1[2] = ph.r1.z;
      r->rn[0] = ph.rn.x; r->rn[1] = ph.rn.y; r->rn[2] = ph.rn.z;
      r->Er[0] = creal(ph.Erm); r->Er[1] = cimag(ph.Erm); r->Er[2] = creal(ph.Ern); r->Er[3] = cimag(ph.Ern);
      r->hit[0] = ph.hit.x; r->hit[1] = ph.hit.y; r->hit[2] = ph.hit.z;
      r->n_hits = ph.n_hits;
    }
  }
  if (stats) {
    stats->photons += local.photons; stats->events += local.events; stats->steps += local.steps;
    stats->detected += local.detected; stats->escaped += local.escaped; stats->stack += local.stack;
    stats->roulette += local.roulette; stats->cap += local.cap; stats->draws += local.draws;
  }
  return 0;
}

static int oadj_layout(const lmc_o_handle *h, const lmc_o_adjoint *a, oadj *A)
{
  memset(A, 0, sizeof(*A));
  A->a = a;
  A->K = 4 * h->scene.n_media;
  A->sensors0 = h->sensors;
  size_t n = 0;
  if (a->radial_sensor >= 0) {
    if (a->radial_sensor >= h->scene.n_sensors ||
        h->sensors[a->radial_sensor].p.kind != LMC_O_SENSOR_PLANAR_FLUENCE ||
        a->radial_bins < 1 || !(a->radial_max > 0))
      return -1;
    A->radial_off = 0;
    n = 1 + (size_t)a->radial_bins;
  }
  for (int si = 0; si < h->scene.n_sensors; ++si) {
    const osensor *s = &h->sensors[si];
    if (s->p.kind != LMC_O_SENSOR_FARFIELD_CBS)
      continue;
    A->cbs_off[si] = n;
    n += 2 * (size_t)s->N_t * s->N_theta * s->N_phi;
  }
  A->n_out = n;
  return 0;
}

size_t lmc_oracle_adjoint_outputs(const lmc_o_handle *h, const lmc_o_adjoint *a)
{
  oadj A;
  return oadj_layout(h, a, &A) == 0 ? A.n_out : 0;
}

int lmc_oracle_run_adjoint(lmc_o_handle *h, uint64_t seed, uint64_t begin, uint64_t count, int rng,
                           int max_events, int track_reverse, double **tallies, uint64_t *hits,
                           const lmc_o_adjoint *a, double *out, lmc_o_stats *stats)
{
  oadj A;
  for (int l = 0; l < h->scene.n_layers; ++l)
    if (h->layer[l].n_species > 0)
      return -3;                  /* the likelihood-ratio scores model HomogeneousLayers only */
  if (oadj_layout(h, a, &A) != 0)
    return -3;
  A.out = out;
  t_adj = &A;
  const int rc = lmc_oracle_run(h, seed, begin, count, rng, max_events, track_reverse, tallies, hits,
                                NULL, stats);
  t_adj = NULL;
  return rc;
}

int lmc_oracle_phase_table(const lmc_o_handle *h, int medium, int *n, const double **values,
                           const double **cdf)
{
  if (medium < 0 || medium >= h->scene.n_media)
    return -1;
  const ophase *ph = &h->phase[h->media[medium].phase];
  *n = ph->table.n;
  *values = ph->table.values;
  *cdf = ph->table.cdf;
  return 0;
}

int lmc_oracle_amp_table(const lmc_o_handle *h, int medium, int *n, double *dtheta,
                         const double **s1, const double **s2)
{
  if (medium < 0 || medium >= h->scene.n_media)
    return -1;
  const omedium *md = &h->media[medium];
  *n = md->S1.n;
  *dtheta = md->S1.dx;
  *s1 = (const double *)md->S1.y;
  *s2 = (const double *)md->S2.y;
  return 0;
}

double lmc_oracle_phase_sample_theta(const lmc_o_handle *h, int medium, double u)
{
  return ophase_sample_theta(&h->phase[h->media[medium].phase], u);
}

void lmc_oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
  lmc_ref_philox4x32_10(ctr, key, out);
}

double lmc_oracle_stream_uniform(uint64_t seed, uint64_t photon, uint64_t draw, int format)
{
  return lmc_ref_stream_uniform(seed, photon, draw, format);
}
