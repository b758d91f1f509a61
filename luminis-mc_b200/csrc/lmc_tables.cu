// lmc_tables.cu -- batched set-up tables of Mie species on the GPU (lmc_mie_tables).
//
// A sweep over many Mie media spends its set-up time in the Mie angular sums: every
// species needs S1, S2 at the 1000 amplitude nodes of its MieMedium and at the
// n_div + 1 nodes of its MiePhaseFunction's PDF, each a sum over ~x + 4 x^(1/3) terms.
// Here one thread evaluates one (species, node) pair; the O(terms) coefficient
// recurrence of each species stays on the host (lmc::mie_series), and so do the node
// cosines and sines, which all species share.  The GPU side uses only explicitly rounded
// binary64 add / subtract / multiply / divide in the order the host builder uses them
// (no fused multiply-add), so every table equals the per-species host construction bit
// for bit.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <mutex>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "lmc_internal.h"
#include "luminis_b200.h"

namespace lmc {
namespace tables {

// One coefficient set: a species' amplitude series (x = 2 pi r / lambda) or its phase
// series (x = k r, k = 2 pi n_m / lambda).
struct SeriesDesc {
  int ntrm;              // 0: small-particle limit
  int conj_out;
  long long off;         // first ap / bp entry
  double rtmp;
  double2 a1, a2, b1;
  double fac;            // pi / (k^2 sigma): PDF prefactor (phase series only)
};

__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

// S1, S2 at cosine mu (the host's mie_amplitudes, R10-R11 and R37-R42 of Wiscombe's method).
__device__ void amplitudes(const SeriesDesc &s, const double2 *__restrict__ ap,
                           const double2 *__restrict__ bp, double mu, double2 &s1, double2 &s2)
{
  if (s.ntrm == 0) {
    const double five3 = 5. / 3.;
    const double2 f = make_double2(mul(five3, s.a2.x), mul(five3, s.a2.y));
    const double2 t = make_double2(mul(add(s.b1.x, f.x), mu), mul(add(s.b1.y, f.y), mu));
    s1 = make_double2(mul(s.rtmp, add(s.a1.x, t.x)), mul(s.rtmp, add(s.a1.y, t.y)));
    const double q = sub(mul(mul(2., mu), mu), 1.);
    const double2 u = make_double2(add(s.b1.x, mul(s.a1.x, mu)), add(s.b1.y, mul(s.a1.y, mu)));
    s2 = make_double2(mul(s.rtmp, add(u.x, mul(f.x, q))), mul(s.rtmp, add(u.y, mul(f.y, q))));
  } else {
    double pi_prev = 0.0, pi_n = 1.0;
    double spr = 0.0, spi = 0.0, smr = 0.0, smi = 0.0;
    for (int n = 1; n <= s.ntrm; ++n) {
      const double fn = n;
      const double2 a = ap[n - 1], b = bp[n - 1];
      const double r = sub(mul(mu, pi_n), pi_prev);
      const double tau = sub(mul(fn, r), pi_prev);
      const double pp = add(pi_n, tau), pm = sub(pi_n, tau);
      spr = add(spr, mul(a.x, pp));
      spi = add(spi, mul(a.y, pp));
      smr = add(smr, mul(b.x, pm));
      smi = add(smi, mul(b.y, pm));
      pi_prev = pi_n;
      pi_n = add(mul(mu, pi_n), mul(add(1.0, dvd(1.0, fn)), r));
    }
    s1 = make_double2(mul(0.5, add(spr, smr)), mul(0.5, add(spi, smi)));
    s2 = make_double2(mul(0.5, sub(spr, smr)), mul(0.5, sub(spi, smi)));
  }
  if (s.conj_out) {
    s1.y = -s1.y;
    s2.y = -s2.y;
  }
}

// Grid (node blocks, species): nodes [0, n_amp) are amplitude-table nodes, the next
// n_pdf are PDF nodes (written into the cdf buffer, turned into the CDF by cdf_kernel).
__global__ void sums_kernel(const SeriesDesc *__restrict__ series, const double2 *__restrict__ ap,
                            const double2 *__restrict__ bp, int n_species, int n_amp, int n_pdf,
                            const double *__restrict__ mu_amp, const double *__restrict__ mu_pdf,
                            const double *__restrict__ sin_pdf, double2 *__restrict__ s1_out,
                            double2 *__restrict__ s2_out, double *__restrict__ pdf_out)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_amp + n_pdf)
    return;
  for (int sp = blockIdx.y; sp < n_species; sp += gridDim.y) {
    double2 s1, s2;
    if (j < n_amp) {
      const SeriesDesc s = series[2 * sp];
      amplitudes(s, ap + s.off, bp + s.off, mu_amp[j], s1, s2);
      s1_out[size_t(sp) * n_amp + j] = s1;
      s2_out[size_t(sp) * n_amp + j] = s2;
    } else {
      const int k = j - n_amp;
      const SeriesDesc s = series[2 * sp + 1];
      amplitudes(s, ap + s.off, bp + s.off, mu_pdf[k], s1, s2);
      const double norm = add(add(mul(s1.x, s1.x), mul(s1.y, s1.y)),
                              add(mul(s2.x, s2.x), mul(s2.y, s2.y)));
      pdf_out[size_t(sp) * n_pdf + k] = mul(mul(s.fac, norm), sin_pdf[k]);
    }
  }
}

// Rectangle-rule CDF of each species' PDF row, normalised to end at 1, in place
// (src/table.cpp:19-47); one thread per species, the host builder's order of sums.
__global__ void cdf_kernel(double *__restrict__ rows, int n_species, int n_pdf, double step,
                           int *__restrict__ nonfinite)
{
  const int sp = blockIdx.x * blockDim.x + threadIdx.x;
  if (sp >= n_species)
    return;
  double *row = rows + size_t(sp) * n_pdf;
  double sum = 0.0;
  for (int i = 0; i < n_pdf; ++i)
    sum = add(sum, mul(row[i], step));
  double prev = 0.0;
  for (int i = 0; i < n_pdf; ++i) {
    const double p = dvd(row[i], sum);
    prev = i == 0 ? mul(p, step) : add(prev, mul(p, step));
    row[i] = prev;
  }
  const double last = row[n_pdf - 1];
  bool bad = false;
  for (int i = 0; i < n_pdf; ++i) {
    const double c = dvd(row[i], last);
    row[i] = c;
    bad |= !isfinite(c);
  }
  if (bad)
    atomicExch(nonfinite, 1);
}

// One work buffer per device, kept between calls (a sweep's 256 species need ~12 MB);
// allocating and freeing it per call cost more than the whole computation.
std::mutex g_arena_mutex;
std::vector<std::pair<void *, size_t>> g_arena;        // per device ordinal

lmc_status arena(size_t bytes, unsigned char **out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return fail(LMC_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (g_arena.size() <= size_t(dev))
    g_arena.resize(size_t(dev) + 1, {nullptr, 0});
  auto &a = g_arena[dev];
  if (a.second < bytes) {
    cudaFree(a.first);
    a = {nullptr, 0};
    e = cudaMalloc(&a.first, bytes);
    if (e != cudaSuccess)
      return fail(e == cudaErrorMemoryAllocation ? LMC_ERR_NOMEM : LMC_ERR_CUDA,
                  std::string("lmc_mie_tables work buffer: ") + cudaGetErrorString(e));
    a.second = bytes;
  }
  *out = static_cast<unsigned char *>(a.first);
  return LMC_OK;
}

}  // namespace tables
}  // namespace lmc

#define LMC_TCUDA(call)                                                                     \
  do {                                                                                      \
    const cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                                  \
      return lmc::fail(LMC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
  } while (0)

extern "C" {

LMC_API lmc_status lmc_mie_tables(const lmc_mie_species *species, int n, int n_div,
                                  double min_val, double max_val, int n_amp, double *values,
                                  double *cdf, double *sigma, double *s1, double *s2,
                                  double *timing_ms)
{
  using namespace lmc;
  using namespace lmc::tables;
  NvtxRange range("lmc_mie_tables: batched Mie set-up tables");
  const bool want_pdf = values || cdf || sigma;
  const bool want_amp = (s1 || s2) && n_amp != 0;
  if (n < 0 || (n > 0 && !species))
    return fail(LMC_ERR_INVALID, "lmc_mie_tables: invalid species list");
  if (want_pdf && (!values || !cdf || !sigma))
    return fail(LMC_ERR_INVALID, "lmc_mie_tables: values, cdf and sigma go together");
  if (want_pdf && n_div <= 0)
    return fail(LMC_ERR_INVALID, "nDiv must be greater than 0");
  if (want_pdf && !(min_val < max_val))
    return fail(LMC_ERR_INVALID, "minVal must be less than maxVal");
  if (want_amp && (!s1 || !s2 || n_amp < 2))
    return fail(LMC_ERR_INVALID, "lmc_mie_tables: s1 and s2 go together, n_amp >= 2");
  const int n_pdf = want_pdf ? n_div + 1 : 0;
  const int n_nodes_amp = want_amp ? n_amp : 0;
  using clock = std::chrono::steady_clock;
  auto ms_since = [](clock::time_point t) {
    return std::chrono::duration<double, std::milli>(clock::now() - t).count();
  };
  double timing[4] = {0.0, 0.0, 0.0, 0.0};      // series, upload, kernels, read-back
  auto report = [&] {
    if (timing_ms)
      for (int i = 0; i < 4; ++i)
        timing_ms[i] = timing[i];
  };
  clock::time_point t0 = clock::now();

  // host side: node tables shared by all species (as lmc_sampling_table and
  // lmc_amplitude_table compute them), then each species' two coefficient series
  std::vector<double> mu_amp(n_nodes_amp), mu_pdf(n_pdf), sin_pdf(n_pdf);
  if (want_amp) {
    const double dtheta = M_PI / double(n_amp - 1);
    for (int i = 0; i < n_amp; ++i)
      mu_amp[i] = std::cos(double(i) * dtheta);
  }
  const double step = want_pdf ? (max_val - min_val) / n_div : 0.0;
  for (int i = 0; i < n_pdf; ++i) {
    values[i] = min_val + i * step;
    mu_pdf[i] = std::min(1.0, std::max(-1.0, std::cos(values[i])));
    sin_pdf[i] = std::sin(values[i]);
  }
  std::vector<SeriesDesc> desc(2 * size_t(n));
  std::vector<double2> ap, bp;
  auto append = [&](const MieSeries &m, SeriesDesc &d) {
    d.ntrm = m.ntrm;
    d.conj_out = m.conj_out;
    d.off = (long long)ap.size();
    d.rtmp = m.small_rtmp;
    d.a1 = make_double2(m.small_a1.real(), m.small_a1.imag());
    d.a2 = make_double2(m.small_a2.real(), m.small_a2.imag());
    d.b1 = make_double2(m.small_b1.real(), m.small_b1.imag());
    d.fac = 0.0;
    for (int k = 0; k < m.ntrm; ++k) {
      ap.push_back(make_double2(m.ap[k].real(), m.ap[k].imag()));
      bp.push_back(make_double2(m.bp[k].real(), m.bp[k].imag()));
    }
  };
  for (int i = 0; i < n; ++i) {
    const lmc_mie_species &q = species[i];
    if (!(q.wavelength > 0.0) || !(q.n_medium > 0.0) || !(q.radius >= 0.0) || !(q.n_particle > 0.0))
      return fail(LMC_ERR_INVALID, "lmc_mie_tables: species " + std::to_string(i) +
                                       " needs wavelength, n_medium, n_particle > 0, radius >= 0");
    MieSeries m;
    if (want_amp) {                                       // src/medium.cpp:160-236
      if (!mie_series(2 * M_PI * q.radius / q.wavelength, q.n_particle / q.n_medium, 0.0, m))
        return fail(LMC_ERR_INVALID, "Mie series failed");
      append(m, desc[2 * size_t(i)]);
    }
    if (want_pdf) {                                       // src/phase.cpp:270-304
      const double k = 2 * M_PI * q.n_medium / q.wavelength;
      if (!mie_series(k * q.radius, q.n_particle / q.n_medium, 0.0, m))
        return fail(LMC_ERR_INVALID, "Mie series failed");
      append(m, desc[2 * size_t(i) + 1]);
      sigma[i] = m.qsca * (M_PI * std::pow(q.radius, 2));
      desc[2 * size_t(i) + 1].fac = M_PI / (k * k * sigma[i]);
    }
  }
  timing[0] = ms_since(t0);
  if (n == 0 || (!want_pdf && !want_amp)) {
    report();
    return LMC_OK;
  }
  t0 = clock::now();

  // device side: one allocation for every input and output
  const size_t b_desc = desc.size() * sizeof(SeriesDesc);
  const size_t b_coef = std::max<size_t>(ap.size(), 1) * sizeof(double2);
  const size_t b_nodes = (size_t(n_nodes_amp) + 2 * size_t(n_pdf)) * sizeof(double);
  const size_t b_amp = size_t(n) * n_nodes_amp * sizeof(double2);
  const size_t b_pdf = size_t(n) * n_pdf * sizeof(double);
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t o_coef = up(b_desc), o_bp = o_coef + up(b_coef), o_nodes = o_bp + up(b_coef);
  const size_t o_s1 = o_nodes + up(b_nodes), o_s2 = o_s1 + up(b_amp), o_pdf = o_s2 + up(b_amp);
  const size_t o_flag = o_pdf + up(b_pdf), total = o_flag + 256;
  std::lock_guard<std::mutex> lock(g_arena_mutex);
  unsigned char *base = nullptr;
  const lmc_status ar = arena(total, &base);
  if (ar != LMC_OK)
    return ar;
  auto at = [&](size_t off) { return base + off; };
  double *d_nodes = reinterpret_cast<double *>(at(o_nodes));
  LMC_TCUDA(cudaMemcpy(at(0), desc.data(), b_desc, cudaMemcpyHostToDevice));
  if (!ap.empty()) {
    LMC_TCUDA(cudaMemcpy(at(o_coef), ap.data(), ap.size() * sizeof(double2), cudaMemcpyHostToDevice));
    LMC_TCUDA(cudaMemcpy(at(o_bp), bp.data(), bp.size() * sizeof(double2), cudaMemcpyHostToDevice));
  }
  if (n_nodes_amp)
    LMC_TCUDA(cudaMemcpy(d_nodes, mu_amp.data(), n_nodes_amp * sizeof(double), cudaMemcpyHostToDevice));
  if (n_pdf) {
    LMC_TCUDA(cudaMemcpy(d_nodes + n_nodes_amp, mu_pdf.data(), n_pdf * sizeof(double),
                         cudaMemcpyHostToDevice));
    LMC_TCUDA(cudaMemcpy(d_nodes + n_nodes_amp + n_pdf, sin_pdf.data(), n_pdf * sizeof(double),
                         cudaMemcpyHostToDevice));
  }
  LMC_TCUDA(cudaMemset(at(o_flag), 0, sizeof(int)));
  timing[1] = ms_since(t0);
  cudaEvent_t ev[2] = {nullptr, nullptr};
  struct EventPair {
    cudaEvent_t *e;
    ~EventPair() { for (int i = 0; i < 2; ++i) if (e[i]) cudaEventDestroy(e[i]); }
  } ev_guard{ev};
  LMC_TCUDA(cudaEventCreate(&ev[0]));
  LMC_TCUDA(cudaEventCreate(&ev[1]));
  LMC_TCUDA(cudaEventRecord(ev[0]));
  constexpr int kThreads = 128;
  const dim3 grid((n_nodes_amp + n_pdf + kThreads - 1) / kThreads, std::min(n, 65535));
  sums_kernel<<<grid, kThreads>>>(
      reinterpret_cast<const SeriesDesc *>(at(0)), reinterpret_cast<const double2 *>(at(o_coef)),
      reinterpret_cast<const double2 *>(at(o_bp)), n, n_nodes_amp, n_pdf, d_nodes,
      d_nodes + n_nodes_amp, d_nodes + n_nodes_amp + n_pdf, reinterpret_cast<double2 *>(at(o_s1)),
      reinterpret_cast<double2 *>(at(o_s2)), reinterpret_cast<double *>(at(o_pdf)));
  LMC_TCUDA(cudaGetLastError());
  if (n_pdf) {
    cdf_kernel<<<(n + kThreads - 1) / kThreads, kThreads>>>(
        reinterpret_cast<double *>(at(o_pdf)), n, n_pdf, step, reinterpret_cast<int *>(at(o_flag)));
    LMC_TCUDA(cudaGetLastError());
  }
  LMC_TCUDA(cudaEventRecord(ev[1]));
  LMC_TCUDA(cudaEventSynchronize(ev[1]));
  float kernel_ms = 0.f;
  LMC_TCUDA(cudaEventElapsedTime(&kernel_ms, ev[0], ev[1]));
  timing[2] = kernel_ms;
  t0 = clock::now();
  int nonfinite = 0;
  if (n_pdf)
    LMC_TCUDA(cudaMemcpy(&nonfinite, at(o_flag), sizeof(int), cudaMemcpyDeviceToHost));
  if (nonfinite)
    return fail(LMC_ERR_INVALID, "phase-function CDF is not finite");
  for (auto [dst, off, bytes] : {std::make_tuple(cdf, o_pdf, b_pdf), std::make_tuple(s1, o_s1, b_amp),
                                  std::make_tuple(s2, o_s2, b_amp)}) {
    if (!bytes)
      continue;
    const lmc_status rb = read_back(dst, reinterpret_cast<const double *>(at(off)), bytes, nullptr);
    if (rb != LMC_OK)
      return rb;
  }
  timing[3] = ms_since(t0);
  report();
  return LMC_OK;
}

}  // extern "C"
