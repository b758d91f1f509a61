// lmc_transport.cu -- host side of the photon-propagation library: scene
// validation and upload (lmc_create), launches (lmc_run, lmc_run_host), tally
// layout and errors.  The kernel itself is in lmc_kernel.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "lmc_device.cuh"
#include "lmc_internal.h"
#include "lmc_kernel.cuh"
#include "luminis_b200.h"

namespace lmc {

std::string &last_error()
{
  thread_local std::string s;
  return s;
}

// ============================================================== host side ==
namespace {

struct CudaCheck {
  cudaError_t e;
};

#define LMC_CUDA(call)                                                                      \
  do {                                                                                      \
    const cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                                  \
      return fail(LMC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));        \
  } while (0)

// Bounds-checked builds: the sites whose index checks failed during the run on `stream`
// (the flag word is cleared for the next run).  Product builds have no checks: LMC_OK.
lmc_status bounds_status(cudaStream_t stream)
{
#ifdef LMC_BOUNDS_CHECK
  unsigned failed = 0;
  LMC_CUDA(cudaMemcpyFromSymbolAsync(&failed, dev::g_bounds_failed, sizeof failed, 0,
                                     cudaMemcpyDeviceToHost, stream));
  LMC_CUDA(cudaStreamSynchronize(stream));
  if (failed) {
    const unsigned zero = 0;
    LMC_CUDA(cudaMemcpyToSymbol(dev::g_bounds_failed, &zero, sizeof zero));
    char msg[96];
    std::snprintf(msg, sizeof msg, "bounds check failed at sites 0x%x (lmc::dev::BoundSite bits)", failed);
    return fail(LMC_ERR_KERNEL, msg);
  }
#else
  (void)stream;
#endif
  return LMC_OK;
}

}  // namespace

}  // namespace lmc

struct lmc_handle {
  lmc::dev::Scene scene;                 // host copy (device table pointers inside)
  lmc::dev::Scene *d_scene = nullptr;
  lmc::dev::Scratch *d_scratch = nullptr;
  void *d_arena = nullptr;
  size_t arena_bytes = 0;
  size_t tally_doubles = 0;
  size_t sensor_off[LMC_MAX_SENSORS] = {};
  size_t sensor_count[LMC_MAX_SENSORS] = {};
  int sensor_dims[LMC_MAX_SENSORS][4] = {};
  size_t abs_off = 0, abs_count = 0;     // Absorption grid (LMC_TALLY_ABSORPTION)
  int abs_dims[4] = {};
  int n_sensors = 0;
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> kev;          // per transport launch: start, end
  double *d_host_tally = nullptr;        // staging for lmc_run_host
  size_t host_tally_cap = 0;
  void *d_queue = nullptr;               // hit queue (queued mode), grown on demand
  size_t queue_bytes = 0;
  unsigned cbs_mask = 0;                 // sensors that need the CBS fields of a hit
  bool queued = false;                   // every sensor plane at z <= 0: queued kernel pair
  int max_planes = 0;                    // most sensor planes of any scene
  bool has_est = false;                  // an estimator-mode FarFieldCBS sensor
  // sweep handles (lmc_create_sweep): n_scenes scenes in one device array
  bool sweep = false;
  int n_scenes = 1;
  struct SceneLayout {
    size_t tally_base = 0;
    int n_sensors = 0;
    size_t off[LMC_MAX_SENSORS] = {}, count[LMC_MAX_SENSORS] = {};
    int dims[LMC_MAX_SENSORS][4] = {};
    size_t abs_off = 0, abs_count = 0;
    int abs_dims[4] = {};
  };
  std::vector<lmc::dev::Scene> scenes;   // host copies (device table pointers inside)
  std::vector<SceneLayout> layouts;
  unsigned long long *d_prefix = nullptr;      // n_scenes + 1 photon offsets
  unsigned long long *d_sweep_hits = nullptr;  // n_scenes x LMC_MAX_SENSORS, last run
  unsigned long long total_photons = 0;        // photons of one sweep run
  std::vector<uint64_t> sweep_counts;          // photons per scene (host copy)
  std::vector<lmc::dev::AdjScene> adj_scenes;  // sweep likelihood-ratio layouts (last run)
  void *d_adj_scenes = nullptr;
  size_t adj_scenes_bytes = 0;
};

namespace lmc {
namespace {

bool finite(double x) { return std::isfinite(x); }

// Host lower_bound (first i with cdf[i] >= key), same predicate as the kernel.
template <typename T> int lower_bound_idx(const std::vector<T> &cdf, T key)
{
  int lo = 0, hi = (int)cdf.size();
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (cdf[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

lmc_status validate(const lmc_scene *s)
{
  if (!s)
    return fail(LMC_ERR_INVALID, "scene must not be null");
  if (s->n_layers < 1 || s->n_layers > LMC_MAX_LAYERS)
    return fail(LMC_ERR_INVALID, "the sample needs 1.." + std::to_string(LMC_MAX_LAYERS) + " layers");
  if (s->n_media < 1 || s->n_media > LMC_MAX_MEDIA)
    return fail(LMC_ERR_INVALID, "the sample needs 1.." + std::to_string(LMC_MAX_MEDIA) + " media");
  if (s->n_sensors < 0 || s->n_sensors > LMC_MAX_SENSORS)
    return fail(LMC_ERR_INVALID, "at most " + std::to_string(LMC_MAX_SENSORS) + " sensors");
  if (!(s->n_host > 0.0) || !finite(s->n_host))
    return fail(LMC_ERR_INVALID, "host refractive index must be positive and finite");
  int mix_entries = 0;
  for (int l = 0; l < s->n_layers; ++l) {                  // src/sample.cpp:120-140
    const lmc_layer_desc &L = s->layers[l];
    if (L.n_species < 0 || L.n_species > LMC_MAX_SPECIES)
      return fail(LMC_ERR_INVALID, "a MixtureLayer holds 1.." + std::to_string(LMC_MAX_SPECIES) + " species");
    if (L.n_species == 0 && (L.medium < 0 || L.medium >= s->n_media))
      return fail(LMC_ERR_INVALID, "layer medium index out of range");
    if (L.n_species > 0) {                                 // src/sample.cpp:41-82
      mix_entries += L.n_species;
      if (mix_entries > LMC_MAX_MIX_ENTRIES)
        return fail(LMC_ERR_UNSUPPORTED, "at most " + std::to_string(LMC_MAX_MIX_ENTRIES) +
                                             " species over all MixtureLayers of a scene");
      double mu_s_total = 0.0;
      for (int i = 0; i < L.n_species; ++i) {
        const int m = L.species[i];
        if (m < 0 || m >= s->n_media)
          return fail(LMC_ERR_INVALID, "MixtureLayer: species pointer must not be null.");
        const double sig = s->media[m].cross_section;
        if (!(sig > 0.0) || !finite(sig))
          return fail(LMC_ERR_INVALID, "PhaseFunction::scattering_cross_section: Not implemented "
                                       "for this phase function.");
        if (!finite(L.number_density[i]))
          return fail(LMC_ERR_INVALID, "MixtureLayer: number densities must be finite");
        mu_s_total += L.number_density[i] * sig;
      }
      if (!(mu_s_total > 0.0) || !finite(mu_s_total))
        return fail(LMC_ERR_INVALID, "MixtureLayer: total mu_s must be positive (check number "
                                     "densities and that the species' phase functions expose a "
                                     "scattering cross-section).");
    }
    if (!(L.z_max > L.z_min))
      return fail(LMC_ERR_INVALID, "Sample::add_layer: z_max must be greater than z_min.");
    if (l == 0 && L.z_min != 0.0)
      return fail(LMC_ERR_INVALID, "Sample::add_layer: first layer must start at z = 0.");
    if (l > 0 && L.z_min != s->layers[l - 1].z_max)
      return fail(LMC_ERR_INVALID, "Sample::add_layer: layer z_min does not match previous z_max.");
    if (l < s->n_layers - 1 && std::isinf(L.z_max))
      return fail(LMC_ERR_INVALID, "Sample::add_layer: cannot add a layer after an infinite top layer.");
  }
  for (int i = 0; i < s->n_media; ++i) {
    const lmc_medium_desc &M = s->media[i];
    if (!finite(M.mu_a) || !finite(M.mu_s) || M.mu_a < 0 || M.mu_s < 0)
      return fail(LMC_ERR_INVALID, "medium coefficients must be finite and non-negative");
    if (!(M.mean_free_path > 0.0) || !finite(M.mean_free_path))
      return fail(LMC_ERR_INVALID, "medium mean_free_path must be set (set_mean_free_path) and positive");
    if (M.theta_kind == LMC_THETA_TABLE || M.theta_kind == LMC_THETA_TABLE_COS) {
      if (M.theta_n < 2 || !M.theta_values || !M.theta_cdf)
        return fail(LMC_ERR_INVALID, "phase-function sampling table missing");
      for (int k = 1; k < M.theta_n; ++k)                    // std::lower_bound needs order
        if (!(M.theta_cdf[k] >= M.theta_cdf[k - 1]))
          return fail(LMC_ERR_INVALID, "phase-function CDF must be non-decreasing");
      if (M.theta_cdf[M.theta_n - 1] != 1.0 || !(M.theta_cdf[0] >= 0.0))
        return fail(LMC_ERR_INVALID, "phase-function CDF must lie in [0, 1] and end at 1");
    } else if (M.theta_kind == LMC_THETA_HG) {
      if (!(M.hg_g != 0.0) || !(M.hg_g >= -1.0 && M.hg_g <= 1.0))
        return fail(LMC_ERR_INVALID, "Henyey-Greenstein g must be in [-1, 1] and non-zero");
    } else if (M.theta_kind != LMC_THETA_UNIFORM) {
      return fail(LMC_ERR_INVALID, "unknown theta sampling kind");
    }
    if (M.amp_n < 2 || !M.amp_s1 || !M.amp_s2 || !(M.amp_dtheta > 0.0))
      return fail(LMC_ERR_INVALID, "medium amplitude table missing");
  }
  if (s->absorption.enabled) {                               // src/absortion.cpp:13-32
    const lmc_absorption_desc &A = s->absorption;
    if (!(A.d_r > 0.0) || !(A.d_z > 0.0) || !finite(A.d_r) || !finite(A.d_z))
      return fail(LMC_ERR_INVALID, "Absorption: d_r and d_z must be positive");
    if (!(A.radius >= 0.0) || !(A.depth >= 0.0) || !finite(A.radius) || !finite(A.depth))
      return fail(LMC_ERR_INVALID, "Absorption: radius and depth must be finite and non-negative");
    if (!(A.d_t >= 0.0) || !finite(A.d_t) || (A.d_t > 0.0 && (!(A.t_max >= 0.0) || !finite(A.t_max))))
      return fail(LMC_ERR_INVALID, "Absorption: d_t and t_max must be finite and non-negative");
    const double cells = (std::floor(A.radius / A.d_r) + 1.0) * (std::floor(A.depth / A.d_z) + 1.0) *
                         (A.d_t > 0.0 ? std::ceil(A.t_max / A.d_t) + 1.0 : 1.0);
    if (!(cells <= 1.0e9))
      return fail(LMC_ERR_INVALID, "Absorption: the grid exceeds 1e9 cells");
  }
  const lmc_laser_desc &L = s->laser;
  if (!(L.wavelength > 0.0))
    return fail(LMC_ERR_INVALID, "laser wavelength must be positive");
  if (L.source < 0 || L.source > 2 || L.temporal < 0 || L.temporal > 5)
    return fail(LMC_ERR_INVALID, "unknown laser source or temporal profile");
  const double z = L.position[2];
  const double top = s->layers[s->n_layers - 1].z_max;
  if (!(z >= 0.0) || (!std::isinf(top) && z >= top))
    return fail(LMC_ERR_INVALID, "laser position lies outside the sample (the reference throws "
                                 "std::out_of_range from Sample::get_layer)");
  for (int i = 0; i < s->n_sensors; ++i) {
    const lmc_sensor_desc &S = s->sensors[i];
    if (S.kind < 0 || S.kind > 4)
      return fail(LMC_ERR_INVALID, "unknown sensor kind");
    if (S.kind == LMC_SENSOR_STATISTICS) {                 // src/detector.cpp:1802-1888
      const lmc_statistics_desc &q = S.stats;
      if (q.n_events < 0 || q.n_theta < 0 || q.n_phi < 0 || q.n_depth < 0 || q.n_time < 0 ||
          q.n_weight < 0)
        return fail(LMC_ERR_INVALID, "StatisticsSensor: histogram sizes must be non-negative");
      if (!finite(S.len_t) || !finite(S.dt))
        return fail(LMC_ERR_INVALID, "StatisticsSensor: time resolution must be finite");
      if (S.dt > 0 && S.len_t / S.dt > 1e6)
        return fail(LMC_ERR_INVALID, "StatisticsSensor: at most 1e6 time windows");
      continue;
    }
    if (S.kind == LMC_SENSOR_FARFIELD_CBS || S.kind == LMC_SENSOR_FARFIELD_FLUENCE) {
      if (!(S.dtheta > 0) || !(S.dphi > 0) || !(S.theta_max_grid > 0) || !(S.phi_max_grid > 0))
        return fail(LMC_ERR_INVALID, "far-field sensor bin widths and extents must be positive");
    } else if (!(S.dx > 0) || !(S.dy > 0) || !(S.len_x > 0) || !(S.len_y > 0)) {
      return fail(LMC_ERR_INVALID, "planar sensor pixel sizes and extents must be positive");
    }
    if (S.dt < 0 || (S.dt > 0 && !(S.len_t > 0)))
      return fail(LMC_ERR_INVALID, "sensor time axis must have len_t > 0 when dt > 0");
  }
  return LMC_OK;
}

void fill_sensor(const lmc_sensor_desc &S, dev::Sensor &d, size_t &count, int dims[4])
{
  std::memset(&d, 0, sizeof(d));
  d.kind = S.kind;
  d.absorb = S.absorb;
  d.estimator = S.estimator;
  // Sensor::Sensor forces the estimator off away from z = 0 (src/detector.cpp:323-331)
  if (S.z != 0.0 && S.estimator)
    d.estimator = 0;
  d.f_theta = S.f_theta;
  if (S.f_theta) {                                          // src/detector.cpp:334-343
    const double c1 = std::cos(S.theta_min), c2 = std::cos(S.theta_max);
    d.cos_min = std::min(c1, c2);
    d.cos_max = std::max(c1, c2);
  }
  d.f_phi = S.f_phi; d.phi_min = S.phi_min; d.phi_max = S.phi_max;
  d.f_pos = S.f_pos; d.x_min = S.x_min; d.x_max = S.x_max; d.y_min = S.y_min; d.y_max = S.y_max;
  d.f_dir = S.f_dir; d.direction = S.direction;
  d.f_events = S.f_events; d.events_min = S.events_min; d.events_max = S.events_max;
  d.len_x = S.len_x; d.len_y = S.len_y; d.len_t = S.len_t; d.dx = S.dx; d.dy = S.dy; d.dt = S.dt;
  d.dtheta = S.dtheta; d.dphi = S.dphi;
  if (S.kind == LMC_SENSOR_FARFIELD_CBS || S.kind == LMC_SENSOR_FARFIELD_FLUENCE) {
    d.absorb = 1;                                           // Sensor(0.0, true, ...)
    d.N_t = (S.dt == 0) ? 1 : (int)std::ceil(S.len_t / S.dt) + 1;
    d.N_theta = (int)std::ceil(S.theta_max_grid / S.dtheta);
    d.N_phi = (int)std::ceil(S.phi_max_grid / S.dphi);
    const int planes = S.kind == LMC_SENSOR_FARFIELD_CBS ? 8 : 4;
    d.plane_stride = (unsigned long long)d.N_t * d.N_theta * d.N_phi;
    count = (size_t)planes * d.plane_stride;
    dims[0] = planes; dims[1] = d.N_t; dims[2] = d.N_theta; dims[3] = d.N_phi;
  } else if (S.kind == LMC_SENSOR_STATISTICS) {
    d.estimator = 0;                                        // Sensor(z, absorb, false)
    d.N_t = (S.dt <= 0.0) ? 1 : (int)std::ceil(S.len_t / S.dt) + 1;   // :1802-1817
    if (S.dt <= 0.0)
      d.dt = 0.0;
    const lmc_statistics_desc &q = S.stats;
    const size_t nt = (size_t)d.N_t;
    size_t n = 0;
    n += (q.set & LMC_STAT_EVENTS) ? nt * (size_t)q.n_events : 0;
    n += (q.set & LMC_STAT_THETA) ? nt * (size_t)q.n_theta : 0;
    n += (q.set & LMC_STAT_PHI) ? nt * (size_t)q.n_phi : 0;
    n += (q.set & LMC_STAT_DEPTH) ? nt * (size_t)q.n_depth : 0;
    n += (q.set & LMC_STAT_TIME) ? (size_t)q.n_time : 0;
    n += (q.set & LMC_STAT_WEIGHT) ? (size_t)q.n_weight : 0;
    count = n;
    dims[0] = d.N_t; dims[1] = (int)n; dims[2] = 0; dims[3] = 0;
  } else if (S.kind == LMC_SENSOR_PLANAR_FLUENCE) {
    d.N_t = (S.dt == 0) ? 1 : (int)std::ceil(S.len_t / S.dt) + 1;
    d.N_x = (int)std::ceil(S.len_x / S.dx);
    d.N_y = (int)std::ceil(S.len_y / S.dy);
    d.plane_stride = (unsigned long long)d.N_t * d.N_x * d.N_y;
    count = 4 * (size_t)d.plane_stride;
    dims[0] = 4; dims[1] = d.N_t; dims[2] = d.N_x; dims[3] = d.N_y;
  } else {
    d.N_x = (int)std::ceil(S.len_x / S.dx);
    d.N_y = (int)std::ceil(S.len_y / S.dy);
    d.plane_stride = (unsigned long long)d.N_x * d.N_y * 2;
    count = 2 * (size_t)d.plane_stride;
    dims[0] = 2; dims[1] = d.N_x; dims[2] = d.N_y; dims[3] = 2;
  }
}

}  // namespace
}  // namespace lmc

using lmc::fail;

namespace lmc {
namespace {

// Host half of a scene: the device Scene (table pointers patched later), its
// sensor layout and its tables appended to a shared arena.
struct MedOff { size_t tvd, tcd, tcs, gd, ad, af; };
struct SceneBuild {
  dev::Scene sc;
  size_t tally_doubles = 0;
  size_t sensor_off[LMC_MAX_SENSORS] = {};
  size_t sensor_count[LMC_MAX_SENSORS] = {};
  int sensor_dims[LMC_MAX_SENSORS][4] = {};
  size_t abs_off = 0, abs_count = 0;
  int abs_dims[4] = {};
  unsigned cbs_mask = 0;
  bool queued = false;
  bool has_est = false;                  // an estimator-mode FarFieldCBS sensor
  size_t est_off[LMC_MAX_SENSORS] = {};  // its bin table in the arena
  size_t stat_off[LMC_MAX_SENSORS] = {}; // StatisticsSensor histograms in the arena
  MedOff mo[LMC_MAX_MEDIA] = {};
};

// A StatisticsSensor's histogram parameters (src/detector.cpp:1836-1888: bin widths
// (max - min) / n) and the offsets of the histograms present, in layout order.
dev::StatHist stat_hist(const lmc_sensor_desc &S, int N_t)
{
  dev::StatHist h;
  std::memset(&h, 0, sizeof(h));
  const lmc_statistics_desc &q = S.stats;
  h.set = q.set;
  h.n_events = q.n_events;
  h.n_theta = q.n_theta;
  h.n_phi = q.n_phi;
  h.n_depth = q.n_depth;
  h.n_time = q.n_time;
  h.n_weight = q.n_weight;
  h.theta_min = q.theta_min; h.theta_max = q.theta_max;
  h.phi_min = q.phi_min; h.phi_max = q.phi_max;
  h.depth_max = q.depth_max;
  h.weight_max = q.weight_max;
  h.dtheta = (q.theta_max - q.theta_min) / q.n_theta;
  h.dphi = (q.phi_max - q.phi_min) / q.n_phi;
  h.ddepth = q.depth_max / q.n_depth;
  h.dtime = q.time_max / q.n_time;
  h.dweight = q.weight_max / q.n_weight;
  const unsigned long long nt = (unsigned long long)N_t;
  unsigned long long o = 0;
  h.off[0] = o; o += (q.set & LMC_STAT_EVENTS) ? nt * q.n_events : 0;
  h.off[1] = o; o += (q.set & LMC_STAT_THETA) ? nt * q.n_theta : 0;
  h.off[2] = o; o += (q.set & LMC_STAT_PHI) ? nt * q.n_phi : 0;
  h.off[3] = o; o += (q.set & LMC_STAT_DEPTH) ? nt * q.n_depth : 0;
  h.off[4] = o; o += (q.set & LMC_STAT_TIME) ? (unsigned long long)q.n_time : 0;
  h.off[5] = o;
  return h;
}

// int_0^pi (|S1|^2 + |S2|^2) sin(theta) dtheta over the medium's amplitude table,
// midpoint rule with 2048 points (src/detector.cpp:106-118); the table lookup is
// DataTable's clamped lerp (src/table.cpp:100-118).
double medium_I_norm(const lmc_medium_desc &M)
{
  const int n = 2048;
  const double inv_dx = 1.0 / M.amp_dtheta;
  const int last = M.amp_n - 1;
  double acc = 0.0;
  const double dth = M_PI / n;
  for (int i = 0; i < n; i++) {
    const double th = (i + 0.5) * dth;
    const double pos = th * inv_dx;
    double v[4];                                // s1.re, s1.im, s2.re, s2.im
    if (pos <= 0.0 || pos >= (double)last) {
      const int k = pos <= 0.0 ? 0 : last;
      v[0] = M.amp_s1[2 * k]; v[1] = M.amp_s1[2 * k + 1];
      v[2] = M.amp_s2[2 * k]; v[3] = M.amp_s2[2 * k + 1];
    } else {
      const int k = (int)pos;
      const double t = pos - (double)k;
      const double *a1 = M.amp_s1 + 2 * k, *a2 = M.amp_s2 + 2 * k;
      v[0] = a1[0] + t * (a1[2] - a1[0]); v[1] = a1[1] + t * (a1[3] - a1[1]);
      v[2] = a2[0] + t * (a2[2] - a2[0]); v[3] = a2[1] + t * (a2[3] - a2[1]);
    }
    acc += ((v[0] * v[0] + v[1] * v[1]) + (v[2] * v[2] + v[3] * v[3])) * std::sin(th);
  }
  return acc * dth;
}

// Layers, interfaces and MixtureLayer tables of the device scene.  A HomogeneousLayer
// takes its medium's coefficients (include/luminis/core/sample.hpp:142-144); a
// MixtureLayer the aggregates of its constructor (src/sample.cpp:55-88): mu_s_i =
// n_i sigma_i, absorption keeping each species' albedo, mu_t, mfp = 1 / mu_s and the
// normalised CDF over mu_s_i whose last entry is exactly 1.
void fill_layers(const lmc_scene *s, dev::Scene &sc)
{
  int mix = 0;
  for (int l = 0; l < s->n_layers; ++l) {
    const lmc_layer_desc &in = s->layers[l];
    dev::Layer &d = sc.layers[l];
    d.z_min = in.z_min;
    d.z_max = in.z_max;
    double mu_a = 0.0;
    if (in.n_species == 0) {
      const lmc_medium_desc &M = s->media[in.medium];
      d.medium = in.medium;
      mu_a = M.mu_a;
      d.mu_s = M.mu_s;
      d.mu_t = M.mu_a + M.mu_s;                             // src/medium.cpp:61-71
      d.mfp = M.mean_free_path;
    } else {
      double mu_s_i[LMC_MAX_SPECIES];
      double mu_s_total = 0.0, mu_a_total = 0.0;
      for (int i = 0; i < in.n_species; ++i) {
        const lmc_medium_desc &M = s->media[in.species[i]];
        mu_s_i[i] = in.number_density[i] * M.cross_section;
        mu_s_total += mu_s_i[i];
        if (M.mu_s > 0.0)
          mu_a_total += mu_s_i[i] * (M.mu_a / M.mu_s);
      }
      d.medium = in.species[0];
      d.n_species = in.n_species;
      d.mix_begin = mix;
      d.flags |= dev::kLayerMixture;
      mu_a = mu_a_total;
      d.mu_s = mu_s_total;
      d.mu_t = mu_s_total + mu_a_total;
      d.mfp = 1.0 / mu_s_total;
      double acc = 0.0;
      for (int i = 0; i < in.n_species; ++i) {
        acc += mu_s_i[i] / mu_s_total;
        sc.mix_cdf[mix + i] = acc;
        sc.mix_species[mix + i] = in.species[i];
      }
      sc.mix_cdf[mix + in.n_species - 1] = 1.0;
      mix += in.n_species;
    }
    d.albedo = d.mu_t > 0 ? d.mu_s / d.mu_t : 1.0;          // src/simulation.cpp:578-587
    d.absorb_prob = d.mu_t > 0 ? mu_a / d.mu_t : 0.0;
    d.mu_t_f = (float)d.mu_t;
    d.mfp_f = (float)d.mfp;
    if (l > 0) {
      sc.interfaces[sc.n_interfaces] = in.z_min;
      sc.interfaces_f[sc.n_interfaces] = (float)in.z_min;
      sc.n_interfaces++;
    }
  }
}

// The Absorption grid's shape and its place after the sensors (`off` doubles into the
// scene's tallies, which start at tally_base); advances off.
void fill_absorption(const lmc_scene *s, dev::Scene &sc, size_t tally_base, size_t &off,
                     size_t &count, int dims[4])
{
  count = 0;
  dims[0] = dims[1] = dims[2] = dims[3] = 0;
  std::memset(&sc.absorb, 0, sizeof(sc.absorb));
  const lmc_absorption_desc &A = s->absorption;
  if (!A.enabled)
    return;
  dev::AbsorbGrid &g = sc.absorb;
  g.on = 1;
  for (int l = 0; l < sc.n_layers; ++l)
    sc.layers[l].flags |= dev::kLayerAbsorb;
  g.n_t = (A.d_t > 0.0) ? (int)std::ceil(A.t_max / A.d_t) + 1 : 1;   // src/absortion.cpp:16-25
  g.n_r = (int)(A.radius / A.d_r) + 1;
  g.n_z = (int)(A.depth / A.d_z) + 1;
  g.radius = A.radius;
  g.depth = A.depth;
  g.d_r = A.d_r;
  g.d_z = A.d_z;
  g.d_t = A.d_t;
  g.radius_f = (float)A.radius;
  g.depth_f = (float)A.depth;
  g.inv_dr_f = (float)(1.0 / A.d_r);
  g.inv_dz_f = (float)(1.0 / A.d_z);
  g.off = tally_base + off;
  count = (size_t)g.n_t * (size_t)g.n_r * (size_t)g.n_z;
  dims[0] = g.n_t; dims[1] = g.n_r; dims[2] = g.n_z; dims[3] = 1;
  off += count;
}

// The parts of a device scene that need no table memory, shared by lmc_create and
// lmc_run_noalloc: counts, layers, laser, sensors with their planes and tally offsets,
// the Absorption grid, the sensor masks and every medium's scalar fields (the table
// pointers stay null).  Sensor i's tallies start at tally_base + sensor_off[i]; returns
// the scene's tally doubles (sensors, then the Absorption grid at *abs_off).
size_t fill_scene_head(const lmc_scene *s, size_t tally_base, dev::Scene &sc, size_t *sensor_off,
                       size_t *sensor_count, int (*sensor_dims)[4], size_t *abs_off,
                       size_t *abs_count, int *abs_dims)
{
  std::memset(&sc, 0, sizeof(sc));
  sc.n_layers = s->n_layers;
  sc.n_media = s->n_media;
  sc.n_sensors = s->n_sensors;
  sc.top = s->layers[s->n_layers - 1].z_max;
  sc.top_is_inf = std::isinf(sc.top) ? 1 : 0;
  sc.top_f = (float)sc.top;
  sc.n_step = 1.0 / (1.0 / s->n_host);                      // src/simulation.cpp:343,390
  fill_layers(s, sc);
  const lmc_laser_desc &L = s->laser;
  for (int j = 0; j < 3; ++j) {
    sc.laser.pos[j] = L.position[j];
    sc.laser.dir[j] = L.direction[j];
    sc.laser.m[j] = L.local_m[j];
    sc.laser.n[j] = L.local_n[j];
  }
  for (int j = 0; j < 4; ++j)
    sc.laser.E[j] = L.jones[j];
  sc.laser.k = 2.0 * M_PI / L.wavelength;                   // src/photon.cpp:39
  sc.laser.sigma = L.sigma;
  sc.laser.source = L.source;
  sc.laser.temporal = L.temporal;
  sc.laser.pulse_duration = L.pulse_duration;
  sc.laser.repetition_rate = L.repetition_rate;
  sc.laser.time_offset = L.time_offset;

  // sensor planes: one key per z within 1e-9 (DoubleComparator, detector.hpp:46-48)
  double planes[LMC_MAX_SENSORS];
  int n_planes = 0;
  size_t off = 0;
  for (int i = 0; i < s->n_sensors; ++i) {
    const lmc_sensor_desc &S = s->sensors[i];
    dev::Sensor &d = sc.sensors[i];
    size_t count = 0;
    fill_sensor(S, d, count, sensor_dims[i]);
    const double z = (S.kind == LMC_SENSOR_FARFIELD_CBS || S.kind == LMC_SENSOR_FARFIELD_FLUENCE) ? 0.0 : S.z;
    if (S.kind == LMC_SENSOR_PLANAR_FIELD && !d.estimator)
      sc.need_phase = 1;
    int g = -1;
    for (int k = 0; k < n_planes; ++k)
      if (!(planes[k] < z - 1e-9) && !(z < planes[k] - 1e-9))
        g = k;
    if (g < 0) {
      planes[n_planes] = z;
      g = n_planes++;
    }
    d.plane = g;
    d.tally_off = tally_base + off;
    sensor_off[i] = off;
    sensor_count[i] = count;
    off += count;
  }
  // planes in ascending z, ties in insertion order (record_hit walks the map in key
  // order)
  int rank[LMC_MAX_SENSORS];
  for (int k = 0; k < n_planes; ++k) {
    int r = 0;
    for (int q = 0; q < n_planes; ++q)
      r += (planes[q] < planes[k] || (planes[q] == planes[k] && q < k)) ? 1 : 0;
    rank[k] = r;
    sc.plane_z[r] = planes[k];
    sc.plane_z_f[r] = (float)planes[k];
  }
  for (int i = 0; i < s->n_sensors; ++i)
    sc.sensors[i].plane = rank[sc.sensors[i].plane];
  sc.n_planes = n_planes;
  *abs_off = off;
  fill_absorption(s, sc, tally_base, off, *abs_count, abs_dims);
  for (int i = 0; i < s->n_sensors; ++i) {
    if (s->sensors[i].kind == LMC_SENSOR_FARFIELD_CBS)
      sc.cbs_mask |= 1u << i;
    if (s->sensors[i].kind == LMC_SENSOR_STATISTICS)
      sc.stat_mask |= 1u << i;
  }
  for (int i = 0; i < s->n_media; ++i) {
    const lmc_medium_desc &M = s->media[i];
    dev::Medium &d = sc.media[i];
    d.theta_kind = M.theta_kind;
    d.hg_g = M.hg_g;
    d.hg_g_f = (float)M.hg_g;
    d.mu_t = M.mu_a + M.mu_s;                               // src/medium.cpp:61-71
    d.mfp = M.mean_free_path;
    d.mu_t_f = (float)d.mu_t;
    d.mfp_f = (float)d.mfp;
    d.amp_n = M.amp_n;
    d.amp_inv_dx = 1.0 / M.amp_dtheta;
    d.amp_inv_dx_f = (float)d.amp_inv_dx;
    d.mu_s = M.mu_s;
    d.mu_s_f = (float)M.mu_s;
    d.I_norm = medium_I_norm(M);
    if (M.theta_kind == LMC_THETA_TABLE || M.theta_kind == LMC_THETA_TABLE_COS)
      d.theta_n = M.theta_n;
  }
  return off;
}

// A photon below z = 0 has left the sample, so a plane at z <= 0 is crossed at most
// once per photon: hits fit a queue of (photons x planes) entries and are tallied by a
// second kernel.  Planes inside the sample may be crossed any number of times; such
// scenes tally inside the transport kernel.
bool scene_queued(const dev::Scene &sc)
{
  return sc.n_planes == 0 || sc.plane_z[sc.n_planes - 1] <= 0.0;
}

// tally_base: offset (doubles) of this scene's first sensor in the tally buffer.
void build_scene(const lmc_scene *s, size_t tally_base, std::vector<unsigned char> &arena, SceneBuild &b)
{
  dev::Scene &sc = b.sc;
  b.tally_doubles = fill_scene_head(s, tally_base, sc, b.sensor_off, b.sensor_count, b.sensor_dims,
                                    &b.abs_off, &b.abs_count, b.abs_dims);
  b.queued = scene_queued(sc);
  b.cbs_mask = sc.cbs_mask;
  const lmc_laser_desc &L = s->laser;

  // table arena: per medium double/float theta tables, guide tables, amplitudes
  auto put = [&](const void *src, size_t bytes) -> size_t {
    const size_t o = (arena.size() + 255) & ~size_t(255);
    arena.resize(o + bytes);
    std::memcpy(arena.data() + o, src, bytes);
    return o;
  };
  for (int i = 0; i < s->n_media; ++i) {
    const lmc_medium_desc &M = s->media[i];
    MedOff &o = b.mo[i];
    o = MedOff{0, 0, 0, 0, 0, 0};
    if (M.theta_kind == LMC_THETA_TABLE || M.theta_kind == LMC_THETA_TABLE_COS) {
      const int n = M.theta_n;
      std::vector<double> vd(M.theta_values, M.theta_values + n), cd(M.theta_cdf, M.theta_cdf + n);
      std::vector<double2> cs(n);
      for (int k = 0; k < n; ++k) {
        const double dc = k ? cd[k] - cd[k - 1] : 0.0;
        cs[k] = make_double2(cd[k], dc > 0.0 ? (vd[k] - vd[k - 1]) / dc : 0.0);
      }
      std::vector<int> gd(dev::kGuideBuckets + 1);
      for (int j = 0; j <= dev::kGuideBuckets; ++j)
        gd[j] = std::min(lower_bound_idx(cd, (double)j / dev::kGuideBuckets), n - 1);
      o.tvd = put(vd.data(), n * sizeof(double));
      o.tcd = put(cd.data(), n * sizeof(double));
      o.tcs = put(cs.data(), n * sizeof(double2));
      o.gd = put(gd.data(), gd.size() * sizeof(int));
    }
    std::vector<double4> ad(M.amp_n);
    std::vector<float4> af(M.amp_n);
    for (int k = 0; k < M.amp_n; ++k) {
      ad[k] = make_double4(M.amp_s1[2 * k], M.amp_s1[2 * k + 1], M.amp_s2[2 * k], M.amp_s2[2 * k + 1]);
      af[k] = make_float4((float)ad[k].x, (float)ad[k].y, (float)ad[k].z, (float)ad[k].w);
    }
    o.ad = put(ad.data(), ad.size() * sizeof(double4));
    o.af = put(af.data(), af.size() * sizeof(float4));
  }
  // Estimator-mode FarFieldCBS: the bin directions of the estimated grid around the
  // backscatter axis -s_in of the launch frame, with their solid angles
  // (src/detector.cpp:886-904, :1476-1498), evaluated once here.
  for (int i = 0; i < s->n_sensors; ++i) {
    const lmc_sensor_desc &S = s->sensors[i];
    dev::Sensor &d = sc.sensors[i];
    if (S.kind != LMC_SENSOR_FARFIELD_CBS || !d.estimator)
      continue;
    const double th_cap = (S.theta_pp_max > 0.0) ? std::min(S.theta_pp_max, S.theta_max_grid)
                                                 : S.theta_max_grid;
    const int i_max = std::min(d.N_theta, (int)(th_cap / S.dtheta));
    const double *e1 = L.local_m, *e2 = L.local_n, *s_in = L.direction;
    std::vector<double4> bins;
    for (int it = 0; it < i_max; ++it) {
      const double th_det = (it + 0.5) * S.dtheta;
      const double c_th = std::cos(th_det), s_th = std::sin(th_det);
      const double dOmega_band = std::cos(it * S.dtheta) - std::cos((it + 1) * S.dtheta);
      for (int jp = 0; jp < d.N_phi; ++jp) {
        const double ph_det = (jp + 0.5) * S.dphi;
        const double c_ph = std::cos(ph_det), s_ph = std::sin(ph_det);
        double so[3];
        for (int k = 0; k < 3; ++k)
          so[k] = (e1[k] * (s_th * c_ph) + e2[k] * (s_th * s_ph)) + (s_in[k] * -1.0) * c_th;
        bins.push_back(make_double4(so[0], so[1], so[2], dOmega_band * S.dphi));
      }
    }
    d.est_n = (int)bins.size();
    // binary32 copy for binary32 transport, after the binary64 table: per bin
    // (s_out, dOmega dphi) and the CBS wave vector q = k (s_out + s_in), formed here in
    // binary64 (s_out + s_in cancels near back-scatter)
    const size_t nb = bins.size();
    bins.resize(nb + nb);                                    // 2 float4 = 1 double4 per bin
    float4 *bf = reinterpret_cast<float4 *>(bins.data() + nb);
    for (size_t k = 0; k < nb; ++k) {
      const double4 q = bins[k];
      bf[2 * k] = make_float4((float)q.x, (float)q.y, (float)q.z, (float)q.w);
      bf[2 * k + 1] = make_float4((float)((q.x + s_in[0]) * sc.laser.k), (float)((q.y + s_in[1]) * sc.laser.k),
                                  (float)((q.z + s_in[2]) * sc.laser.k), 0.0f);
    }
    b.est_off[i] = bins.empty() ? 0 : put(bins.data(), bins.size() * sizeof(double4));
    b.has_est = true;
  }
  for (int i = 0; i < s->n_sensors; ++i)
    if (s->sensors[i].kind == LMC_SENSOR_STATISTICS) {
      const dev::StatHist hh = stat_hist(s->sensors[i], sc.sensors[i].N_t);
      b.stat_off[i] = put(&hh, sizeof(hh));
    }
}

// Device table pointers of a built scene, given the device copy of the arena.
void patch_tables(SceneBuild &b, unsigned char *base)
{
  for (int i = 0; i < b.sc.n_media; ++i) {
    dev::Medium &d = b.sc.media[i];
    const MedOff &o = b.mo[i];
    if (d.theta_n) {
      d.th_val_d = reinterpret_cast<const double *>(base + o.tvd);
      d.th_cdf_d = reinterpret_cast<const double *>(base + o.tcd);
      d.th_cs = reinterpret_cast<const double2 *>(base + o.tcs);
      d.guide_d = reinterpret_cast<const int *>(base + o.gd);
    }
    d.amp_d = reinterpret_cast<const double4 *>(base + o.ad);
    d.amp_f = reinterpret_cast<const float4 *>(base + o.af);
  }
  for (int i = 0; i < b.sc.n_sensors; ++i) {
    if (b.sc.sensors[i].est_n > 0)
      b.sc.sensors[i].est_bins = reinterpret_cast<const double4 *>(base + b.est_off[i]);
    if (b.sc.sensors[i].kind == LMC_SENSOR_STATISTICS)
      b.sc.sensors[i].stat = reinterpret_cast<const dev::StatHist *>(base + b.stat_off[i]);
  }
}

// Device allocations shared by lmc_create and lmc_create_sweep: arena, scenes,
// scratch, stream and events.
cudaError_t alloc_handle(lmc_handle *h, const std::vector<unsigned char> &arena, size_t n_scenes)
{
  h->arena_bytes = arena.size();
  cudaError_t e = cudaMalloc(&h->d_arena, std::max<size_t>(h->arena_bytes, 256));
  if (e == cudaSuccess)
    e = cudaMemcpy(h->d_arena, arena.data(), arena.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMalloc(&h->d_scene, n_scenes * sizeof(dev::Scene));
  if (e == cudaSuccess)
    e = cudaMalloc(&h->d_scratch, sizeof(dev::Scratch));
  if (e == cudaSuccess)
    e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess)
    e = cudaEventCreate(&h->ev0);
  if (e == cudaSuccess)
    e = cudaEventCreate(&h->ev1);
  return e;
}

}  // namespace
}  // namespace lmc

extern "C" {

size_t lmc_last_error(char *buf, size_t len)
{
  const std::string &e = lmc::last_error();
  if (buf && len) {
    const size_t n = std::min(len - 1, e.size());
    std::memcpy(buf, e.data(), n);
    buf[n] = 0;
  }
  return e.size();
}

lmc_status lmc_create(const lmc_scene *s, lmc_handle **out)
{
  using namespace lmc;
  NvtxRange range("lmc_create: scene set-up and upload");
  if (!out)
    return fail(LMC_ERR_INVALID, "out must not be null");
  *out = nullptr;
  const lmc_status v = validate(s);
  if (v != LMC_OK)
    return v;
  int device = 0;
  LMC_CUDA(cudaGetDevice(&device));
  lmc_handle *h = new lmc_handle();
  h->device = device;
  LMC_CUDA(cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device));
  std::vector<unsigned char> arena;
  SceneBuild b;
  build_scene(s, 0, arena, b);
  h->n_sensors = s->n_sensors;
  h->tally_doubles = b.tally_doubles;
  h->queued = b.queued;
  h->cbs_mask = b.cbs_mask;
  h->max_planes = b.sc.n_planes;
  h->has_est = b.has_est;
  h->abs_off = b.abs_off;
  h->abs_count = b.abs_count;
  for (int k = 0; k < 4; ++k)
    h->abs_dims[k] = b.abs_dims[k];
  for (int i = 0; i < LMC_MAX_SENSORS; ++i) {
    h->sensor_off[i] = b.sensor_off[i];
    h->sensor_count[i] = b.sensor_count[i];
    for (int k = 0; k < 4; ++k)
      h->sensor_dims[i][k] = b.sensor_dims[i][k];
  }
  cudaError_t e = alloc_handle(h, arena, 1);
  if (e == cudaSuccess) {
    patch_tables(b, static_cast<unsigned char *>(h->d_arena));
    h->scene = b.sc;
    e = cudaMemcpy(h->d_scene, &h->scene, sizeof(h->scene), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    lmc_destroy(h);
    return fail(LMC_ERR_CUDA, std::string("lmc_create: ") + cudaGetErrorString(e));
  }
  *out = h;
  return LMC_OK;
}

void lmc_destroy(lmc_handle *h)
{
  if (!h)
    return;
  if (h->stream)
    cudaStreamSynchronize(h->stream);
  cudaFree(h->d_arena);
  cudaFree(h->d_scene);
  cudaFree(h->d_scratch);
  cudaFree(h->d_host_tally);
  cudaFree(h->d_queue);
  cudaFree(h->d_prefix);
  cudaFree(h->d_sweep_hits);
  cudaFree(h->d_adj_scenes);
  for (cudaEvent_t e : h->kev)
    cudaEventDestroy(e);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

lmc_status lmc_tally_layout(const lmc_handle *h, int sensor, size_t *offset, size_t *count, int dims[4])
{
  if (!h)
    return fail(LMC_ERR_INVALID, "handle must not be null");
  if (sensor == -1) {
    if (offset) *offset = 0;
    if (count) *count = h->tally_doubles;
    return LMC_OK;
  }
  if (sensor == LMC_TALLY_ABSORPTION) {
    if (offset) *offset = h->abs_off;
    if (count) *count = h->abs_count;
    if (dims)
      for (int k = 0; k < 4; ++k)
        dims[k] = h->abs_dims[k];
    return LMC_OK;
  }
  if (sensor < 0 || sensor >= h->n_sensors)
    return fail(LMC_ERR_INVALID, "sensor index out of range");
  if (offset) *offset = h->sensor_off[sensor];
  if (count) *count = h->sensor_count[sensor];
  if (dims)
    for (int k = 0; k < 4; ++k)
      dims[k] = h->sensor_dims[sensor][k];
  return LMC_OK;
}

// Layout of the likelihood-ratio outputs of one scene (lmc_adjoint_layout, and each
// scene of lmc_sweep_adjoint_layout).
static lmc_status scene_adjoint_layout(const lmc::dev::Scene &sc, const lmc_adjoint_opts *a,
                                       size_t *n_out, unsigned long long cbs_off[LMC_MAX_SENSORS])
{
  using namespace lmc;
  if (sc.n_media > dev::kAdjMaxMedia)
    return fail(LMC_ERR_UNSUPPORTED, "likelihood-ratio outputs support at most 4 media");
  for (int l = 0; l < sc.n_layers; ++l)
    if (sc.layers[l].n_species > 0)
      return fail(LMC_ERR_UNSUPPORTED, "likelihood-ratio outputs model HomogeneousLayers only");
  for (int i = 0; i < sc.n_media; ++i) {
    const dev::Medium &m = sc.media[i];
    if (!(m.mu_t > 0) || !(m.mu_s > 0))
      return fail(LMC_ERR_INVALID, "likelihood-ratio outputs need mu_s > 0 in every medium");
  }
  size_t n = 0;
  if (a->radial_sensor >= 0) {
    if (a->radial_sensor >= sc.n_sensors || sc.sensors[a->radial_sensor].kind != LMC_SENSOR_PLANAR_FLUENCE)
      return fail(LMC_ERR_INVALID, "radial_sensor must be a PlanarFluenceSensor");
    if (a->radial_bins < 1 || a->radial_bins > dev::kAdjMaxRadialBins || !(a->radial_max > 0))
      return fail(LMC_ERR_INVALID, "radial_bins must be in [1, 512] and radial_max > 0");
    n = 1 + (size_t)a->radial_bins;
  }
  for (int i = 0; i < LMC_MAX_SENSORS; ++i)
    cbs_off[i] = 0;
  for (int i = 0; i < sc.n_sensors; ++i) {
    const dev::Sensor &s = sc.sensors[i];
    if (s.kind != LMC_SENSOR_FARFIELD_CBS)
      continue;
    cbs_off[i] = n;
    n += 2 * (size_t)s.N_t * s.N_theta * s.N_phi;
  }
  if (n == 0)
    return fail(LMC_ERR_INVALID, "no likelihood-ratio outputs: no radial sensor and no FarFieldCBSSensor");
  *n_out = n;
  return LMC_OK;
}

// Layout of the likelihood-ratio outputs of a handle (lmc_adjoint_layout).
static lmc_status adjoint_layout(const lmc_handle *h, const lmc_adjoint_opts *a, size_t *n_out,
                                 unsigned long long cbs_off[LMC_MAX_SENSORS])
{
  using namespace lmc;
  if (!h || !a)
    return fail(LMC_ERR_INVALID, "handle and adjoint options must not be null");
  if (h->sweep)
    return fail(LMC_ERR_INVALID, "a sweep handle lays its outputs out with lmc_sweep_adjoint_layout");
  if (!h->queued)
    return fail(LMC_ERR_UNSUPPORTED, "likelihood-ratio outputs need every sensor plane at z <= 0");
  return scene_adjoint_layout(h->scene, a, n_out, cbs_off);
}

// Per-scene blocks of a sweep's likelihood-ratio outputs, one after another; the
// total size (doubles) and the largest parameter count.
static lmc_status sweep_adjoint_layout(const lmc_handle *h, const lmc_adjoint_opts *a,
                                       std::vector<lmc::dev::AdjScene> &out, size_t *total, int *max_K)
{
  using namespace lmc;
  if (!h || !a)
    return fail(LMC_ERR_INVALID, "handle and adjoint options must not be null");
  if (!h->sweep)
    return fail(LMC_ERR_INVALID, "not a sweep handle");
  out.assign(h->n_scenes, dev::AdjScene{});
  size_t off = 0;
  int kmax = 0;
  for (int k = 0; k < h->n_scenes; ++k) {
    dev::AdjScene &A = out[k];
    size_t n = 0;
    const lmc_status st = scene_adjoint_layout(h->scenes[k], a, &n, A.cbs_off);
    if (st != LMC_OK)
      return fail(st, "scene " + std::to_string(k) + ": " + last_error());
    A.out_off = off;
    A.n_out = n;
    A.K = 4 * h->scenes[k].n_media;
    A.radial_sensor = a->radial_sensor;
    A.radial_bins = a->radial_bins;
    A.radial_max = a->radial_max;
    off += (size_t)(1 + A.K) * n;
    kmax = std::max(kmax, A.K);
  }
  *total = off;
  *max_K = kmax;
  return LMC_OK;
}

}  // extern "C"

// The transport and tally kernels of a run.  `extras`: a scene has a MixtureLayer or an
// Absorption recorder (the variants with their code; the others leave it out).
using KernelFn = void (*)(const lmc::dev::Scene *, lmc::dev::RunParams);

template <bool E>
static KernelFn pick_transport_e(bool fp32, bool queued, bool wide, bool adj, bool sw, bool est)
{
  using namespace lmc::dev;
  if (est)
    return fp32 ? transport_kernel<float, true, 2, false, false, true, E>
                : transport_kernel<double, true, 2, false, false, true, E>;
  if (sw && adj)
    return fp32 ? transport_kernel<float, true, 3, true, true> : transport_kernel<double, true, 1, true, true>;
  if (sw)
    return fp32 ? transport_kernel<float, true, 3, false, true, false, E>
                : transport_kernel<double, true, 2, false, true, false, E>;
  if (adj)
    return fp32 ? transport_kernel<float, true, 3, true> : transport_kernel<double, true, 1, true>;
  if (fp32)
    return queued ? (wide ? transport_kernel<float, true, 4, false, false, false, E>
                           : transport_kernel<float, true, 2, false, false, false, E>)
                  : transport_kernel<float, false, 1, false, false, false, E>;
  return queued ? transport_kernel<double, true, 2, false, false, false, E>
                : transport_kernel<double, false, 1, false, false, false, E>;
}

static KernelFn pick_transport(bool fp32, bool queued, bool wide, bool adj, bool sw, bool est, bool extras)
{
  return extras ? pick_transport_e<true>(fp32, queued, wide, adj, sw, est)
                : pick_transport_e<false>(fp32, queued, wide, adj, sw, est);
}

template <int kT>
static KernelFn pick_tally_t(bool fp32, bool adj, bool sw)
{
  using namespace lmc::dev;
  if (sw) {
    constexpr int kS = kT == kTallyShared ? kTallyGlobal : kT;   // (refused by tally_setup)
    return adj ? (fp32 ? tally_kernel<float, true, true, kS> : tally_kernel<double, true, true, kS>)
               : (fp32 ? tally_kernel<float, false, true, kS> : tally_kernel<double, false, true, kS>);
  }
  return adj ? (fp32 ? tally_kernel<float, true, false, kT> : tally_kernel<double, true, false, kT>)
             : (fp32 ? tally_kernel<float, false, false, kT> : tally_kernel<double, false, false, kT>);
}

// kt: the device tally mode (dev::kTallyGlobal, kTallyWarp, kTallyShared).
static KernelFn pick_tally(bool fp32, bool adj, bool sw, int kt = lmc::dev::kTallyGlobal)
{
  using namespace lmc::dev;
  if (kt == kTallyWarp)
    return pick_tally_t<kTallyWarp>(fp32, adj, sw);
  if (kt == kTallyShared)
    return pick_tally_t<kTallyShared>(fp32, adj, sw);
  return pick_tally_t<kTallyGlobal>(fp32, adj, sw);
}

// The hit-queue tally kernel of a run under lmc_run_opts.tally_mode `mode`: the kernel,
// its dynamic shared memory (dyn_tally: what it needs before the private grids) and
// its grid.  LMC_TALLY_SHARED gives private copies to the direct-hit PlanarFluence,
// FarFieldCBS and FarFieldFluence grids, smallest first, while they fit in the shared
// memory a block may have beside the kernel's static arrays; their offsets go to rp.
// Without any grid that fits the mode adds like LMC_TALLY_GLOBAL (and says so in kt).
struct TallyLaunch {
  KernelFn fn;
  size_t dyn;
  int grid_per_sm;                       // blocks per SM of the tally grid
  int kt;                                // device mode used
};

static lmc_status tally_setup(int mode, bool sw, bool fp32, bool adj, const lmc::dev::Scene &sc,
                              const size_t *sensor_count, int device, size_t dyn_tally,
                              lmc::dev::RunParams &rp, TallyLaunch &out)
{
  using namespace lmc;
  if (mode < LMC_TALLY_DEFAULT || mode > LMC_TALLY_SHARED)
    return fail(LMC_ERR_INVALID, "tally_mode must be an lmc_tally_mode");
  if (mode == LMC_TALLY_SHARED && sw)
    return fail(LMC_ERR_INVALID, "tally_mode LMC_TALLY_SHARED needs a single-scene handle");
  for (int i = 0; i < LMC_MAX_SENSORS; ++i) {
    rp.tally_smem[i] = -1;
    rp.tally_smem_n[i] = 0;
  }
  rp.tally_smem_doubles = 0;
  int kt = mode == LMC_TALLY_WARP ? dev::kTallyWarp
         : mode == LMC_TALLY_SHARED ? dev::kTallyShared : dev::kTallyGlobal;
  out.dyn = dyn_tally;
  out.grid_per_sm = 8;
  if (kt == dev::kTallyShared) {
    const KernelFn fn = pick_tally(fp32, adj, sw, kt);
    int optin = 0;
    LMC_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    cudaFuncAttributes fa;
    LMC_CUDA(cudaFuncGetAttributes(&fa, (const void *)fn));
    const size_t room = (size_t)optin > fa.sharedSizeBytes + dyn_tally
                            ? ((size_t)optin - fa.sharedSizeBytes - dyn_tally) / sizeof(double) : 0;
    int order[LMC_MAX_SENSORS], n = 0;
    for (int i = 0; i < sc.n_sensors; ++i) {
      const dev::Sensor &s = sc.sensors[i];
      const bool direct = s.kind == LMC_SENSOR_PLANAR_FLUENCE || s.kind == LMC_SENSOR_FARFIELD_FLUENCE ||
                          (s.kind == LMC_SENSOR_FARFIELD_CBS && !s.estimator);
      if (direct && sensor_count[i] > 0)
        order[n++] = i;
    }
    std::stable_sort(order, order + n, [&](int a, int b) { return sensor_count[a] < sensor_count[b]; });
    size_t used = 0;
    for (int k = 0; k < n; ++k) {
      const size_t c = sensor_count[order[k]];
      if (used + c > room)
        break;
      rp.tally_smem[order[k]] = (int)used;
      rp.tally_smem_n[order[k]] = (int)c;
      used += c;
    }
    rp.tally_smem_doubles = (int)used;
    if (used == 0) {
      kt = dev::kTallyGlobal;
    } else {
      out.dyn = dyn_tally + used * sizeof(double);
      LMC_CUDA(cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)out.dyn));
      int per = 0;
      LMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)fn, dev::kBlock, out.dyn));
      if (per < 1)
        return fail(LMC_ERR_CUDA, "tally kernel with private grids does not fit on an SM");
      out.grid_per_sm = per;            // one pass of resident blocks: each adds its grids once
    }
  }
  out.kt = kt;
  out.fn = pick_tally(fp32, adj, sw, kt);
  if (out.dyn > 0 && kt != dev::kTallyShared)
    LMC_CUDA(cudaFuncSetAttribute((const void *)out.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)out.dyn));
  return LMC_OK;
}

static KernelFn pick_replay(bool fp32, bool sw, bool extras)
{
  using namespace lmc::dev;
  if (extras)
    return fp32 ? (sw ? cbs_replay_kernel<float, true, true> : cbs_replay_kernel<float, false, true>)
                : (sw ? cbs_replay_kernel<double, true, true> : cbs_replay_kernel<double, false, true>);
  return fp32 ? (sw ? cbs_replay_kernel<float, true> : cbs_replay_kernel<float, false>)
              : (sw ? cbs_replay_kernel<double, true> : cbs_replay_kernel<double, false>);
}

// Whether any of a scene's layers draws species or records absorption.
static bool scene_extras(const lmc::dev::Scene &sc)
{
  for (int l = 0; l < sc.n_layers; ++l)
    if (sc.layers[l].flags & (lmc::dev::kLayerMixture | lmc::dev::kLayerAbsorb))
      return true;
  return false;
}

extern "C" {

// lmc_run and lmc_run_adjoint (adj == nullptr: plain run).
static lmc_status run_impl(lmc_handle *h, uint64_t seed, uint64_t photon_begin, uint64_t n_photons,
                           const lmc_run_opts *opts, const lmc_adjoint_opts *adj, double *d_adj,
                           double *d_tallies, lmc_stats *stats)
{
  using namespace lmc;
  if (!h || !opts)
    return fail(LMC_ERR_INVALID, "handle and options must not be null");
  NvtxRange range("lmc_run: transport and tally launches");
  if (h->tally_doubles && !d_tallies)
    return fail(LMC_ERR_INVALID, "device tally buffer must not be null");
  if (opts->precision != LMC_PRECISION_FP32 && opts->precision != LMC_PRECISION_FP64)
    return fail(LMC_ERR_INVALID, "unknown precision");
  if (opts->max_events < 0)
    return fail(LMC_ERR_INVALID, "max_events must be non-negative");
  const bool sw = h->sweep;
  const bool est = h->has_est;
  if (est && (adj || !h->queued))
    return fail(LMC_ERR_UNSUPPORTED, "estimator-mode FarFieldCBS runs need every sensor plane at "
                                     "z <= 0 and no likelihood-ratio outputs");
  for (int k = 0; k < h->n_scenes; ++k) {
    const dev::Scene &scn = sw ? h->scenes[k] : h->scene;
    for (int i = 0; i < scn.n_sensors; ++i)
      if (scn.sensors[i].kind == LMC_SENSOR_FARFIELD_CBS && !opts->track_reverse_paths)
        return fail(LMC_ERR_INVALID, "FarFieldCBSSensor needs track_reverse_paths (the reference "
                                     "dereferences null species pointers without it)");
  }
  LMC_CUDA(cudaSetDevice(h->device));
  cudaStream_t stream = opts->stream ? static_cast<cudaStream_t>(opts->stream) : h->stream;
  LMC_CUDA(cudaMemsetAsync(h->d_scratch, 0, sizeof(dev::Scratch), stream));
  if (sw)
    LMC_CUDA(cudaMemsetAsync(h->d_sweep_hits, 0,
                             sizeof(unsigned long long) * h->n_scenes * LMC_MAX_SENSORS, stream));
  dev::RunParams rp;
  std::memset(&rp, 0, sizeof(rp));
  rp.key0 = (uint32_t)seed;
  rp.key1 = (uint32_t)(seed >> 32);
  rp.max_events = opts->max_events;
  rp.track_reverse = opts->track_reverse_paths ? 1 : 0;
  rp.tallies = d_tallies;
  rp.records = static_cast<lmc_record *>(opts->records);
  rp.scratch = h->d_scratch;
  rp.cbs_mask = h->cbs_mask;
  const bool fp32 = opts->precision == LMC_PRECISION_FP32;
  if (opts->stream_format != 0 && opts->stream_format != 1)
    return fail(LMC_ERR_INVALID, "stream_format must be 0 or 1");
  rp.stream_u24 = (!fp32 && opts->stream_format == 1) ? 1 : 0;
  if (opts->cbs_phase != 0 && opts->cbs_phase != 1)
    return fail(LMC_ERR_INVALID, "cbs_phase must be 0 (binary64) or 1 (binary32)");
  rp.cbs_phase_f32 = opts->cbs_phase;
  if (sw) {
    rp.n_scenes = h->n_scenes;
    rp.sweep_prefix = h->d_prefix;
    rp.sweep_hits = h->d_sweep_hits;
  }
  const int block = opts->block_size > 0 ? opts->block_size : dev::kBlock;
  if (block % 32 != 0 || block > dev::kBlock)
    return fail(LMC_ERR_INVALID, "block_size must be a multiple of 32 and at most 256");
  const size_t rbytes = fp32 ? sizeof(float) : sizeof(double);
  size_t dyn_transport = fp32 ? dev::side_bytes<float>() : dev::side_bytes<double>();
  size_t dyn_tally = 0;
  // estimator-mode grids: each block accumulates its vertices' estimates in a shared
  // copy of the grid (one flush of non-zero cells per block), as long as they fit
  for (int i = 0; i < LMC_MAX_SENSORS; ++i)
    rp.est_smem[i] = -1;
  size_t est_block_doubles = 0;          // the grids' shared copies, one per block
  if (est) {
    constexpr size_t kEstSmemDoubles = (40u << 10) / sizeof(double);
    size_t used = 0;
    for (int i = 0; i < h->scene.n_sensors; ++i) {
      const dev::Sensor &S = h->scene.sensors[i];
      if (S.kind != LMC_SENSOR_FARFIELD_CBS || !S.estimator || S.est_n == 0)
        continue;
      const size_t n = h->sensor_count[i];
      if (used + n > kEstSmemDoubles)
        continue;
      rp.est_smem[i] = (int)used;
      used += n;
    }
    est_block_doubles = used;
    rp.est_smem_doubles = (int)used;
    rp.est_warp_doubles = (int)used;
  }
  if (adj && sw) {
    size_t total = 0;
    int kmax = 0;
    std::vector<dev::AdjScene> lay;
    const lmc_status ls = sweep_adjoint_layout(h, adj, lay, &total, &kmax);
    if (ls != LMC_OK)
      return ls;
    if (!d_adj)
      return fail(LMC_ERR_INVALID, "device adjoint buffer must not be null");
    // upload the layouts only when they change (synchronously), so that a run with
    // the layouts of the previous one enqueues device work only and can be captured
    const size_t bytes = sizeof(dev::AdjScene) * lay.size();
    if (!h->d_adj_scenes || h->adj_scenes.size() != lay.size() ||
        std::memcmp(h->adj_scenes.data(), lay.data(), bytes) != 0) {
      if (h->adj_scenes_bytes < bytes) {
        cudaFree(h->d_adj_scenes);
        h->d_adj_scenes = nullptr;
        h->adj_scenes_bytes = 0;
        const cudaError_t e = cudaMalloc(&h->d_adj_scenes, bytes);
        if (e != cudaSuccess)
          return fail(LMC_ERR_NOMEM, std::string("sweep adjoint layout: ") + cudaGetErrorString(e));
        h->adj_scenes_bytes = bytes;
      }
      LMC_CUDA(cudaMemcpy(h->d_adj_scenes, lay.data(), bytes, cudaMemcpyHostToDevice));
      h->adj_scenes = lay;
    }
    rp.adj_scenes = static_cast<const dev::AdjScene *>(h->d_adj_scenes);
    rp.adj_out = d_adj;
    rp.adj_n_out = total;
    rp.adj_K = kmax;
    rp.adj_radial_sensor = -1;           // per scene in adj_scenes, added globally
  } else if (adj) {
    size_t n_out = 0;
    const lmc_status ls = adjoint_layout(h, adj, &n_out, rp.adj_cbs_off);
    if (ls != LMC_OK)
      return ls;
    if (!d_adj)
      return fail(LMC_ERR_INVALID, "device adjoint buffer must not be null");
    rp.adj_out = d_adj;
    rp.adj_n_out = n_out;
    rp.adj_K = 4 * h->scene.n_media;
    rp.adj_radial_sensor = adj->radial_sensor;
    rp.adj_radial_bins = adj->radial_bins;
    rp.adj_radial_max = adj->radial_max;
    if (adj->radial_sensor >= 0)
      dyn_tally = (size_t)(1 + rp.adj_K) * (adj->radial_bins + 1) * sizeof(double);
  }
  // binary32 queued transport: a 4-block (<=64 registers, the default) and a
  // 2-block (<=128 registers) variant; blocks_per_sm == 1 or 2 selects the latter
  const bool wide = fp32 && h->queued && !adj && (opts->blocks_per_sm == 0 || opts->blocks_per_sm >= 3);
  bool extras = false;
  for (int k = 0; k < h->n_scenes; ++k)
    extras = extras || scene_extras(sw ? h->scenes[k] : h->scene);
  if (adj && extras)                     // (MixtureLayers are refused by the layout already)
    return fail(LMC_ERR_UNSUPPORTED, "likelihood-ratio runs do not record an Absorption grid");
  const KernelFn tk = pick_transport(fp32, h->queued, wide, adj != nullptr, sw, est, extras);
  TallyLaunch tl{};
  if (h->queued && h->tally_doubles > 0) {
    const lmc_status st = tally_setup(opts->tally_mode, sw, fp32, adj != nullptr,
                                      sw ? h->scenes[0] : h->scene, h->sensor_count, h->device,
                                      (adj && !sw) ? dyn_tally : 0, rp, tl);
    if (st != LMC_OK)
      return st;
  }
  // CBS replay: queued runs without an estimator or records keep no reverse-path
  // history in the transport; the replay kernel rebuilds it for the hits that
  // FarFieldCBS grids read (likelihood-ratio scores are carried apart from it)
  bool any_cbs = false;
  for (int k = 0; k < h->n_scenes; ++k)
    any_cbs = any_cbs || (sw ? h->scenes[k] : h->scene).cbs_mask != 0;
  const bool replay = h->queued && !est && !opts->records && !opts->no_replay &&
                      opts->track_reverse_paths && any_cbs;
  rp.cbs_replay = replay ? 1 : 0;
  if (replay) {                          // no history: the ring and first species only
    rp.track_reverse = 0;
    dyn_transport = fp32 ? dev::side_slim_bytes<float>() : dev::side_slim_bytes<double>();
  }
  // the likelihood-ratio scores (or the estimated grids below) follow the Side arrays
  rp.side_off = (unsigned)dyn_transport;
  if (adj)
    dyn_transport += (size_t)rp.adj_K * dev::kBlock * rbytes;
  const KernelFn tr = replay ? pick_replay(fp32, sw, extras) : nullptr;
  const size_t dyn_replay = fp32 ? dev::side_bytes<float>() : dev::side_bytes<double>();
  int replay_grid = 0;
  if (replay) {
    LMC_CUDA(cudaFuncSetAttribute((const void *)tr, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)dyn_replay));
    int per = 0;
    LMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)tr, dev::kBlock, dyn_replay));
    replay_grid = h->sm_count * std::max(per, 1);
  }
  if (est_block_doubles) {
    // one copy of the estimated grids per warp (plain adds) when that keeps as many
    // blocks per SM as one shared copy per block (shared atomics); else the latter
    const size_t shared_one = dyn_transport + est_block_doubles * sizeof(double);
    const size_t per_warp = dyn_transport + (size_t)(block / 32) * est_block_doubles * sizeof(double);
    // the largest dynamic shared memory a block of this kernel may ask for
    int optin = 0;
    LMC_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
    cudaFuncAttributes fa;
    LMC_CUDA(cudaFuncGetAttributes(&fa, (const void *)tk));
    const size_t dyn_max = (size_t)optin > fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
    int occ_one = 0, occ_warp = 0;
    if (per_warp <= dyn_max) {
      LMC_CUDA(cudaFuncSetAttribute((const void *)tk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)std::max(shared_one, per_warp)));
      LMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_one, (const void *)tk, block, shared_one));
      LMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_warp, (const void *)tk, block, per_warp));
    }
    rp.est_per_warp = (per_warp <= dyn_max && occ_warp >= occ_one && occ_warp > 0) ? 1 : 0;
    rp.est_smem_doubles = (int)(rp.est_per_warp ? (block / 32) * est_block_doubles : est_block_doubles);
    dyn_transport += (size_t)rp.est_smem_doubles * sizeof(double);
  }
  if (opts->stage_tables && fp32 && !sw) {
    // every medium's binary32 amplitude table in the block's shared memory, after the
    // other dynamic arrays -- as long as that keeps the blocks per SM
    size_t bytes = 0;
    for (int m = 0; m < h->scene.n_media; ++m)
      bytes += (size_t)h->scene.media[m].amp_n * sizeof(float4);
    const size_t off = (dyn_transport + 15) & ~size_t(15);
    int optin = 0;
    LMC_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
    cudaFuncAttributes fa;
    LMC_CUDA(cudaFuncGetAttributes(&fa, (const void *)tk));
    int occ0 = 0, occ1 = 0;
    if (off + bytes + fa.sharedSizeBytes <= (size_t)optin) {
      LMC_CUDA(cudaFuncSetAttribute((const void *)tk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(off + bytes)));
      LMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ0, (const void *)tk, block, dyn_transport));
      LMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ1, (const void *)tk, block, off + bytes));
    }
    if (bytes > 0 && occ1 >= occ0 && occ1 > 0) {
      rp.stage_bytes = (unsigned)bytes;
      rp.stage_off = (unsigned)off;
      dyn_transport = off + bytes;
    }
  }
  LMC_CUDA(cudaFuncSetAttribute((const void *)tk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dyn_transport));
  int per_sm = 0;
  LMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)tk, block, dyn_transport));
  if (opts->blocks_per_sm > 0)
    per_sm = std::min(per_sm, opts->blocks_per_sm);
  per_sm = std::max(per_sm, 1);

  // batches: the whole range at once inline; queue-sized batches when queued
  unsigned long long batch = n_photons;
  if (h->queued && n_photons > 0) {
    batch = opts->batch_photons ? opts->batch_photons : (32ull << 20);   // ~110 B of queue per photon
    batch = std::min<unsigned long long>(batch, n_photons);
    const unsigned long long planes = std::max(1, h->max_planes);
    const unsigned long long cap = batch * planes + batch / 16 + 1024;
    const size_t need = (size_t)cap * (dev::kQU32Fields * 4 + dev::kQF64Fields * 8 +
                                       (dev::kQRFields + (size_t)rp.adj_K) * rbytes) +
                        (replay ? (size_t)cap * sizeof(uint32_t) : 0) + 4 * 256;
    if (h->queue_bytes < need) {
      cudaFree(h->d_queue);
      h->d_queue = nullptr;
      h->queue_bytes = 0;
      const cudaError_t e = cudaMalloc(&h->d_queue, need);
      if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? LMC_ERR_NOMEM : LMC_ERR_CUDA,
                    std::string("hit queue allocation: ") + cudaGetErrorString(e));
      h->queue_bytes = need;
    }
    unsigned char *q = static_cast<unsigned char *>(h->d_queue);
    auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
    rp.queue.cap = cap;
    rp.queue.u32 = reinterpret_cast<uint32_t *>(q);
    size_t o = align((size_t)cap * dev::kQU32Fields * 4);
    rp.queue.f64 = reinterpret_cast<double *>(q + o);
    o += align((size_t)cap * dev::kQF64Fields * 8);
    rp.queue.r = q + o;
    o += align((size_t)cap * (dev::kQRFields + (size_t)rp.adj_K) * rbytes);
    rp.replay_list = replay ? reinterpret_cast<uint32_t *>(q + o) : nullptr;
  }
  if (stats && n_photons > 0) {           // one event pair per transport launch
    const size_t need_ev = 2 * (size_t)((n_photons + batch - 1) / batch);
    while (h->kev.size() < need_ev) {
      cudaEvent_t e = nullptr;
      LMC_CUDA(cudaEventCreate(&e));
      h->kev.push_back(e);
    }
  }
  LMC_CUDA(cudaEventRecord(h->ev0, stream));
  lmc_record *const records = static_cast<lmc_record *>(opts->records);
  for (unsigned long long done = 0; done < n_photons; done += batch) {
    const unsigned long long nb = std::min(batch, n_photons - done);
    rp.photon_begin = photon_begin + done;
    rp.n_photons = nb;
    rp.records = records ? records + done : nullptr;   // the kernels index from photon_begin
    // reset the work counters (transport, replay) and the queue fills of this batch
    LMC_CUDA(cudaMemsetAsync(h->d_scratch, 0, 4 * sizeof(unsigned long long), stream));
    const int grid = (int)std::max<unsigned long long>(
        1ull, std::min<unsigned long long>((unsigned long long)h->sm_count * per_sm,
                                           (nb + block - 1) / block));
    const size_t pair = 2 * (size_t)(done / batch);
    if (stats)
      LMC_CUDA(cudaEventRecord(h->kev[pair], stream));
    tk<<<grid, block, dyn_transport, stream>>>(h->d_scene, rp);
    LMC_CUDA(cudaGetLastError());
    if (replay) {                        // part of the transport (timed with it)
      tr<<<replay_grid, dev::kBlock, dyn_replay, stream>>>(h->d_scene, rp);
      LMC_CUDA(cudaGetLastError());
    }
    if (stats)
      LMC_CUDA(cudaEventRecord(h->kev[pair + 1], stream));
    if (h->queued && h->tally_doubles > 0) {
      const int tgrid = (int)std::max<unsigned long long>(
          1ull, std::min<unsigned long long>((unsigned long long)h->sm_count * tl.grid_per_sm,
                                             (rp.queue.cap + dev::kBlock - 1) / dev::kBlock));
      tl.fn<<<tgrid, dev::kBlock, tl.dyn, stream>>>(h->d_scene, rp);
      LMC_CUDA(cudaGetLastError());
    }
  }
  LMC_CUDA(cudaEventRecord(h->ev1, stream));
  if (stats) {
    dev::Scratch sc;
    LMC_CUDA(cudaMemcpyAsync(&sc, h->d_scratch, sizeof(sc), cudaMemcpyDeviceToHost, stream));
    LMC_CUDA(cudaStreamSynchronize(stream));
    std::memset(stats, 0, sizeof(*stats));
    stats->photons = sc.photons; stats->events = sc.events; stats->steps = sc.steps;
    stats->detected = sc.detected; stats->escaped = sc.escaped; stats->stack = sc.stack;
    stats->roulette = sc.roulette; stats->cap = sc.cap; stats->draws = sc.draws;
    for (int i = 0; i < LMC_MAX_SENSORS; ++i)
      stats->hits[i] = sc.hits[i];
    stats->error_flags = sc.error_flags;
    float ms = 0.f;
    LMC_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    stats->kernel_ms = ms;
    const size_t launches = batch ? (size_t)((n_photons + batch - 1) / batch) : 0;
    double tms = 0.0;
    for (size_t b = 0; b < launches; ++b) {
      float d = 0.f;
      LMC_CUDA(cudaEventElapsedTime(&d, h->kev[2 * b], h->kev[2 * b + 1]));
      tms += d;
    }
    stats->transport_ms = (float)tms;
    stats->transport_launches = (uint32_t)launches;
    stats->replay_launches = replay ? (uint32_t)launches : 0u;
    stats->replayed = sc.replayed;
    if (sc.error_flags)
      return fail(LMC_ERR_KERNEL, "transport kernel raised error flags " + std::to_string(sc.error_flags));
  }
  return bounds_status(stream);
}

lmc_status lmc_run(lmc_handle *h, uint64_t seed, uint64_t photon_begin, uint64_t n_photons,
                   const lmc_run_opts *opts, double *d_tallies, lmc_stats *stats)
{
  if (h && h->sweep)
    return lmc::fail(LMC_ERR_INVALID, "a sweep handle runs through lmc_run_sweep");
  return run_impl(h, seed, photon_begin, n_photons, opts, nullptr, nullptr, d_tallies, stats);
}

lmc_status lmc_create_sweep(const lmc_scene *scenes, int n_scenes, lmc_handle **out)
{
  using namespace lmc;
  NvtxRange range("lmc_create_sweep: scene set-up and upload");
  if (!out || !scenes)
    return fail(LMC_ERR_INVALID, "scenes and out must not be null");
  *out = nullptr;
  if (n_scenes < 1 || n_scenes > LMC_MAX_SWEEP_SCENES)
    return fail(LMC_ERR_INVALID, "n_scenes must be in [1, " + std::to_string(LMC_MAX_SWEEP_SCENES) + "]");
  for (int k = 0; k < n_scenes; ++k) {
    const lmc_status v = validate(scenes + k);
    if (v != LMC_OK)
      return fail(v, "scene " + std::to_string(k) + ": " + last_error());
  }
  int device = 0;
  LMC_CUDA(cudaGetDevice(&device));
  lmc_handle *h = new lmc_handle();
  h->device = device;
  h->sweep = true;
  h->n_scenes = n_scenes;
  LMC_CUDA(cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device));
  std::vector<unsigned char> arena;
  std::vector<SceneBuild> builds(n_scenes);
  h->layouts.resize(n_scenes);
  size_t tally = 0;
  h->queued = true;
  for (int k = 0; k < n_scenes; ++k) {
    build_scene(scenes + k, tally, arena, builds[k]);
    if (!builds[k].queued || builds[k].has_est) {
      delete h;
      return fail(LMC_ERR_UNSUPPORTED, "scene " + std::to_string(k) +
                                           ": a sweep needs every sensor plane at z <= 0 and "
                                           "no estimator-mode sensor");
    }
    lmc_handle::SceneLayout &L = h->layouts[k];
    L.tally_base = tally;
    L.n_sensors = scenes[k].n_sensors;
    for (int i = 0; i < LMC_MAX_SENSORS; ++i) {
      L.off[i] = tally + builds[k].sensor_off[i];
      L.count[i] = builds[k].sensor_count[i];
      for (int j = 0; j < 4; ++j)
        L.dims[i][j] = builds[k].sensor_dims[i][j];
    }
    L.abs_off = tally + builds[k].abs_off;
    L.abs_count = builds[k].abs_count;
    for (int j = 0; j < 4; ++j)
      L.abs_dims[j] = builds[k].abs_dims[j];
    h->max_planes = std::max(h->max_planes, builds[k].sc.n_planes);
    tally += builds[k].tally_doubles;
  }
  h->tally_doubles = tally;
  h->n_sensors = scenes[0].n_sensors;
  for (int i = 0; i < LMC_MAX_SENSORS; ++i) {
    h->sensor_off[i] = h->layouts[0].off[i];
    h->sensor_count[i] = h->layouts[0].count[i];
  }
  cudaError_t e = alloc_handle(h, arena, (size_t)n_scenes);
  if (e == cudaSuccess)
    e = cudaMalloc(&h->d_prefix, sizeof(unsigned long long) * (n_scenes + 1));
  if (e == cudaSuccess)
    e = cudaMalloc(&h->d_sweep_hits, sizeof(unsigned long long) * n_scenes * LMC_MAX_SENSORS);
  if (e == cudaSuccess) {
    h->scenes.resize(n_scenes);
    for (int k = 0; k < n_scenes; ++k) {
      patch_tables(builds[k], static_cast<unsigned char *>(h->d_arena));
      h->scenes[k] = builds[k].sc;
    }
    h->scene = h->scenes[0];
    e = cudaMemcpy(h->d_scene, h->scenes.data(), sizeof(dev::Scene) * n_scenes, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) {
    std::vector<unsigned long long> zero(n_scenes + 1, 0ull);
    e = cudaMemcpy(h->d_prefix, zero.data(), sizeof(unsigned long long) * (n_scenes + 1),
                   cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    lmc_destroy(h);
    return fail(LMC_ERR_CUDA, std::string("lmc_create_sweep: ") + cudaGetErrorString(e));
  }
  *out = h;
  return LMC_OK;
}

lmc_status lmc_sweep_layout(const lmc_handle *h, int scene, int sensor, size_t *offset,
                            size_t *count, int dims[4])
{
  using namespace lmc;
  if (!h || !h->sweep)
    return fail(LMC_ERR_INVALID, "not a sweep handle");
  if (scene == -1) {
    if (count)
      *count = h->tally_doubles;
    return LMC_OK;
  }
  if (scene < 0 || scene >= h->n_scenes)
    return fail(LMC_ERR_INVALID, "scene out of range");
  const lmc_handle::SceneLayout &L = h->layouts[scene];
  if (sensor == LMC_TALLY_ABSORPTION) {
    if (offset) *offset = L.abs_off;
    if (count) *count = L.abs_count;
    if (dims)
      for (int k = 0; k < 4; ++k)
        dims[k] = L.abs_dims[k];
    return LMC_OK;
  }
  if (sensor < 0 || sensor >= L.n_sensors)
    return fail(LMC_ERR_INVALID, "sensor out of range");
  if (offset)
    *offset = L.off[sensor];
  if (count)
    *count = L.count[sensor];
  if (dims)
    for (int k = 0; k < 4; ++k)
      dims[k] = L.dims[sensor][k];
  return LMC_OK;
}

lmc_status lmc_sweep_set_photons(lmc_handle *h, const uint64_t *n_photons)
{
  using namespace lmc;
  if (!h || !h->sweep || !n_photons)
    return fail(LMC_ERR_INVALID, "sweep handle and photon counts must not be null");
  std::vector<unsigned long long> prefix(h->n_scenes + 1, 0ull);
  for (int k = 0; k < h->n_scenes; ++k)
    prefix[k + 1] = prefix[k] + n_photons[k];
  LMC_CUDA(cudaSetDevice(h->device));
  LMC_CUDA(cudaStreamSynchronize(h->stream));
  LMC_CUDA(cudaMemcpy(h->d_prefix, prefix.data(), sizeof(unsigned long long) * (h->n_scenes + 1),
                      cudaMemcpyHostToDevice));
  h->total_photons = prefix[h->n_scenes];
  h->sweep_counts.assign(n_photons, n_photons + h->n_scenes);
  return LMC_OK;
}

lmc_status lmc_autotune(lmc_handle *h, uint64_t seed, const lmc_run_opts *opts, uint64_t sample_photons,
                        lmc_tune_result *out)
{
  using namespace lmc;
  if (!h || !opts || !out)
    return fail(LMC_ERR_INVALID, "handle, options and result must not be null");
  if (sample_photons == 0)
    return fail(LMC_ERR_INVALID, "sample_photons must be positive");
  if (h->sweep && h->sweep_counts.empty())
    return fail(LMC_ERR_INVALID, "lmc_sweep_set_photons() first");
  LMC_CUDA(cudaSetDevice(h->device));
  // the sample: photons [0, sample) of a single scene; for a sweep every scene's count
  // scaled to a total of about sample_photons (at least one photon each), restored after
  const std::vector<uint64_t> counts = h->sweep_counts;
  unsigned long long n_sample = sample_photons;
  if (h->sweep) {
    const double f = std::min(1.0, (double)sample_photons / (double)std::max<uint64_t>(1, h->total_photons));
    std::vector<uint64_t> scaled(counts.size());
    for (size_t k = 0; k < counts.size(); ++k)
      scaled[k] = counts[k] ? std::max<uint64_t>(1, (uint64_t)std::llround((double)counts[k] * f)) : 0;
    const lmc_status st = lmc_sweep_set_photons(h, scaled.data());
    if (st != LMC_OK)
      return st;
    n_sample = h->total_photons;
  }
  double *d_t = nullptr;
  cudaError_t e = cudaMalloc(&d_t, std::max<size_t>(h->tally_doubles, 1) * sizeof(double));
  if (e != cudaSuccess) {
    if (h->sweep)
      lmc_sweep_set_photons(h, counts.data());
    return fail(LMC_ERR_NOMEM, std::string("lmc_autotune: ") + cudaGetErrorString(e));
  }
  // candidates: threads per block x resident blocks per SM (the grid, hence photons per
  // thread of the persistent kernel) x photons per hit-queue batch
  const int blocks[] = {256, 128};
  const int per_sm[] = {0, 2, 1};
  const unsigned long long batches[] = {32ull << 20, 8ull << 20};
  lmc_tune_result best;
  std::memset(&best, 0, sizeof(best));
  lmc_status result = LMC_OK;
  int tried = 0;
  for (int b : blocks)
    for (int p : per_sm)
      for (unsigned long long q : batches) {
        if (q != batches[0] && (!h->queued || n_sample <= batches[1]))
          continue;                              // the batch size only matters past it
        lmc_run_opts o = *opts;
        o.block_size = b;
        o.blocks_per_sm = p;
        o.batch_photons = q;
        o.records = nullptr;
        lmc_stats st;
        double ms = 0.0;
        for (int rep = 0; rep < 2 && result == LMC_OK; ++rep) {   // warm-up, then timed
          result = run_impl(h, seed, 0, n_sample, &o, nullptr, nullptr, d_t, &st);
          ms = st.kernel_ms;
        }
        if (result != LMC_OK)
          break;
        ++tried;
        const double rate = ms > 0 ? (double)n_sample / (ms * 1e-3) : 0.0;
        if (rate > best.photons_per_s) {
          best.block_size = b;
          best.blocks_per_sm = p;
          best.batch_photons = q;
          best.photons_per_s = rate;
        }
      }
  // the tally kernel's mode at that shape (hit-queue runs; a sweep's scenes share no
  // private grid, so it has two modes)
  best.tally_mode = opts->tally_mode;
  if (result == LMC_OK && h->queued && h->tally_doubles > 0) {
    const int modes[] = {LMC_TALLY_GLOBAL, LMC_TALLY_WARP, LMC_TALLY_SHARED};
    double best_rate = 0.0;
    for (int m : modes) {
      if (m == LMC_TALLY_SHARED && h->sweep)
        continue;
      lmc_run_opts o = *opts;
      o.block_size = best.block_size;
      o.blocks_per_sm = best.blocks_per_sm;
      o.batch_photons = best.batch_photons;
      o.tally_mode = m;
      o.records = nullptr;
      lmc_stats st;
      double ms = 0.0;
      for (int rep = 0; rep < 2 && result == LMC_OK; ++rep) {
        result = run_impl(h, seed, 0, n_sample, &o, nullptr, nullptr, d_t, &st);
        ms = st.kernel_ms;
      }
      if (result != LMC_OK)
        break;
      ++tried;
      const double rate = ms > 0 ? (double)n_sample / (ms * 1e-3) : 0.0;
      if (rate > best_rate) {
        best_rate = rate;
        best.tally_mode = m;
        best.photons_per_s = rate;
      }
    }
  }
  cudaFree(d_t);
  if (h->sweep) {
    const lmc_status st = lmc_sweep_set_photons(h, counts.data());
    if (result == LMC_OK)
      result = st;
  }
  if (result != LMC_OK)
    return result;
  best.n_tried = tried;
  best.sample_photons = n_sample;
  *out = best;
  return LMC_OK;
}

lmc_status lmc_run_sweep(lmc_handle *h, uint64_t seed, const lmc_run_opts *opts, double *d_tallies,
                         lmc_stats *stats)
{
  if (!h || !h->sweep)
    return lmc::fail(LMC_ERR_INVALID, "not a sweep handle");
  return run_impl(h, seed, 0, h->total_photons, opts, nullptr, nullptr, d_tallies, stats);
}

lmc_status lmc_sweep_adjoint_layout(const lmc_handle *h, const lmc_adjoint_opts *a, int scene,
                                    size_t *offset, size_t *n_out, int *n_params)
{
  using namespace lmc;
  std::vector<dev::AdjScene> lay;
  size_t total = 0;
  int kmax = 0;
  const lmc_status st = sweep_adjoint_layout(h, a, lay, &total, &kmax);
  if (st != LMC_OK)
    return st;
  if (scene == -1) {
    if (offset) *offset = 0;
    if (n_out) *n_out = total;
    if (n_params) *n_params = kmax;
    return LMC_OK;
  }
  if (scene < 0 || scene >= h->n_scenes)
    return fail(LMC_ERR_INVALID, "scene out of range");
  if (offset) *offset = lay[scene].out_off;
  if (n_out) *n_out = lay[scene].n_out;
  if (n_params) *n_params = lay[scene].K;
  return LMC_OK;
}

lmc_status lmc_run_sweep_adjoint(lmc_handle *h, uint64_t seed, const lmc_run_opts *opts,
                                 const lmc_adjoint_opts *a, double *d_tallies, double *d_adjoint,
                                 lmc_stats *stats)
{
  if (!h || !h->sweep)
    return lmc::fail(LMC_ERR_INVALID, "not a sweep handle");
  if (!a)
    return lmc::fail(LMC_ERR_INVALID, "adjoint options must not be null");
  return run_impl(h, seed, 0, h->total_photons, opts, a, d_adjoint, d_tallies, stats);
}

lmc_status lmc_sweep_hits(lmc_handle *h, uint64_t *hits)
{
  using namespace lmc;
  if (!h || !h->sweep || !hits)
    return fail(LMC_ERR_INVALID, "sweep handle and output must not be null");
  LMC_CUDA(cudaSetDevice(h->device));
  LMC_CUDA(cudaDeviceSynchronize());
  LMC_CUDA(cudaMemcpy(hits, h->d_sweep_hits, sizeof(unsigned long long) * h->n_scenes * LMC_MAX_SENSORS,
                      cudaMemcpyDeviceToHost));
  return LMC_OK;
}

lmc_status lmc_adjoint_layout(const lmc_handle *h, const lmc_adjoint_opts *a, size_t *n_out,
                              int *n_params)
{
  unsigned long long off[LMC_MAX_SENSORS];
  size_t n = 0;
  const lmc_status st = adjoint_layout(h, a, &n, off);
  if (st != LMC_OK)
    return st;
  if (n_out)
    *n_out = n;
  if (n_params)
    *n_params = 4 * h->scene.n_media;
  return LMC_OK;
}

lmc_status lmc_run_adjoint(lmc_handle *h, uint64_t seed, uint64_t photon_begin, uint64_t n_photons,
                           const lmc_run_opts *opts, const lmc_adjoint_opts *adj, double *d_tallies,
                           double *d_adjoint, lmc_stats *stats)
{
  if (!adj)
    return lmc::fail(LMC_ERR_INVALID, "adjoint options must not be null");
  return run_impl(h, seed, photon_begin, n_photons, opts, adj, d_adjoint, d_tallies, stats);
}

lmc_status lmc_adjoint_contract(const double *d_adjoint, const double *d_grad_out, size_t n_out,
                                int n_params, double *d_grad_params, void *stream)
{
  using namespace lmc;
  if (!d_adjoint || !d_grad_out || !d_grad_params || n_out == 0 || n_params < 1)
    return fail(LMC_ERR_INVALID, "lmc_adjoint_contract: null buffer or empty sizes");
  dev::adjoint_contract_kernel<<<n_params, dev::kBlock, 0, static_cast<cudaStream_t>(stream)>>>(
      d_adjoint, d_grad_out, n_out, d_grad_params);
  LMC_CUDA(cudaGetLastError());
  return LMC_OK;
}

}  // extern "C"

namespace lmc {
namespace {

// lmc_run_host reads its tallies back through two pinned 16 MiB halves shared by every
// handle of the process (allocated on first use, kept until exit): the copy engine fills
// one half while host threads move the other into the caller's pageable buffer.
constexpr size_t kStageBytes = size_t(16) << 20;
std::mutex g_stage_mutex;
unsigned char *g_stage = nullptr;

struct StageEvents {
  cudaEvent_t e[2] = {nullptr, nullptr};
  cudaError_t create()
  {
    for (cudaEvent_t &x : e) {
      const cudaError_t r = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
      if (r != cudaSuccess)
        return r;
    }
    return cudaSuccess;
  }
  ~StageEvents()
  {
    for (cudaEvent_t x : e)
      if (x)
        cudaEventDestroy(x);
  }
};

// memcpy split over up to 8 host threads (2 MiB or more each).
void parallel_copy(unsigned char *dst, const unsigned char *src, size_t bytes)
{
  constexpr size_t kMinPart = size_t(2) << 20;
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t n = std::min<size_t>(std::min<size_t>(hw, 8), (bytes + kMinPart - 1) / kMinPart);
  if (n <= 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  const size_t part = ((bytes + n - 1) / n + 63) & ~size_t(63);
  std::vector<std::thread> pool;
  for (size_t i = 1; i < n && i * part < bytes; ++i)
    pool.emplace_back([=] { std::memcpy(dst + i * part, src + i * part, std::min(part, bytes - i * part)); });
  std::memcpy(dst, src, std::min(part, bytes));
  for (std::thread &t : pool)
    t.join();
}

}  // namespace

// Device tallies -> caller's host buffer, chunk by chunk through the pinned halves.
lmc_status read_back(double *h_dst, const double *d_src, size_t bytes, void *stream_ptr)
{
  NvtxRange range("lmc tallies: device to host read-back");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  std::lock_guard<std::mutex> lock(g_stage_mutex);
  if (!g_stage)
    LMC_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&g_stage), 2 * kStageBytes, cudaHostAllocPortable));
  StageEvents ev;
  LMC_CUDA(ev.create());
  const unsigned char *src = reinterpret_cast<const unsigned char *>(d_src);
  unsigned char *dst = reinterpret_cast<unsigned char *>(h_dst);
  const size_t n_chunks = (bytes + kStageBytes - 1) / kStageBytes;
  auto chunk_len = [&](size_t k) { return std::min(kStageBytes, bytes - k * kStageBytes); };
  auto issue = [&](size_t k) {
    cudaError_t e = cudaMemcpyAsync(g_stage + (k & 1) * kStageBytes, src + k * kStageBytes,
                                    chunk_len(k), cudaMemcpyDeviceToHost, stream);
    return e == cudaSuccess ? cudaEventRecord(ev.e[k & 1], stream) : e;
  };
  LMC_CUDA(issue(0));
  for (size_t k = 0; k < n_chunks; ++k) {
    LMC_CUDA(cudaEventSynchronize(ev.e[k & 1]));
    if (k + 1 < n_chunks)           // the other half was emptied in the previous iteration
      LMC_CUDA(issue(k + 1));
    parallel_copy(dst + k * kStageBytes, g_stage + (k & 1) * kStageBytes, chunk_len(k));
  }
  return LMC_OK;
}

}  // namespace lmc

extern "C" {

lmc_status lmc_run_host(lmc_handle *h, uint64_t seed, uint64_t photon_begin, uint64_t n_photons,
                        const lmc_run_opts *opts, double *h_tallies, lmc_stats *stats)
{
  using namespace lmc;
  NvtxRange range("lmc_run_host");
  if (!h)
    return fail(LMC_ERR_INVALID, "handle must not be null");
  if (h->tally_doubles && !h_tallies)
    return fail(LMC_ERR_INVALID, "host tally buffer must not be null");
  LMC_CUDA(cudaSetDevice(h->device));
  const size_t bytes = h->tally_doubles * sizeof(double);
  if (h->host_tally_cap < bytes) {
    cudaFree(h->d_host_tally);
    h->d_host_tally = nullptr;
    h->host_tally_cap = 0;
    LMC_CUDA(cudaMalloc(&h->d_host_tally, std::max<size_t>(bytes, 8)));
    h->host_tally_cap = bytes;
  }
  cudaStream_t stream = opts && opts->stream ? static_cast<cudaStream_t>(opts->stream) : h->stream;
  if (bytes && opts && opts->host_tallies_zero)
    LMC_CUDA(cudaMemsetAsync(h->d_host_tally, 0, bytes, stream));
  else if (bytes)
    LMC_CUDA(cudaMemcpyAsync(h->d_host_tally, h_tallies, bytes, cudaMemcpyHostToDevice, stream));
  lmc_stats local;
  const lmc_status st = lmc_run(h, seed, photon_begin, n_photons, opts, h->d_host_tally,
                                stats ? stats : &local);
  if (st != LMC_OK)
    return st;
  if (bytes) {
    const lmc_status rb = read_back(h_tallies, h->d_host_tally, bytes, static_cast<void *>(stream));
    if (rb != LMC_OK)
      return rb;
  }
  LMC_CUDA(cudaStreamSynchronize(stream));
  return LMC_OK;
}

}  // extern "C"

// ======================================================== allocation-free path ==
// lmc_run_noalloc: the transport for callers that cannot allocate device memory.
// Everything the kernels need beyond the caller's inputs and outputs -- the
// device scene, the derived tables, the run counters and the hit queue -- lives
// in one file-scope __device__ array.  The CUDA runtime reserves it on every GPU
// that loads this library, until the process exits.
namespace lmc {
namespace {

constexpr size_t kNoAllocBytes = size_t(64) << 20;          // 64 MiB per GPU
constexpr size_t kNaSceneOff = 0;                           // dev::Scene
constexpr size_t kNaCountersOff = 8192;                     // dev::Scratch
constexpr size_t kNaTablesOff = 16384;                      // copied + derived tables
constexpr size_t kNaTablesBytes = size_t(8) << 20;
constexpr size_t kNaQueueOff = kNaTablesOff + kNaTablesBytes;   // hit queue: the rest
static_assert(sizeof(dev::Scene) <= kNaCountersOff - kNaSceneOff, "scene region too small");
static_assert(sizeof(dev::Scratch) <= kNaTablesOff - kNaCountersOff, "counter region too small");

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mutex;
unsigned char *g_noalloc_base[256] = {};                      // per device ordinal

// Device address of g_noalloc_scratch on the current device (looked up once per
// device; host code cannot use the symbol itself as a device pointer).
lmc_status noalloc_base(int device, unsigned char **out)
{
  if (device < 0 || device >= 256)
    return fail(LMC_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_base[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(LMC_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") +
                                    cudaGetErrorString(e));
    g_noalloc_base[device] = static_cast<unsigned char *>(p);
  }
  *out = g_noalloc_base[device];
  return LMC_OK;
}

// Guide, (cdf, slope) and interleaved amplitude tables from the copied base tables,
// the same values lmc_create computes on the host.
struct DeriveArgs {
  const double *vals, *cdf;
  int n;
  double2 *cs;
  int *guide;
  const double *s1, *s2;
  int amp_n;
  double4 *amp_d;
  float4 *amp_f;
};

__global__ void derive_tables(DeriveArgs a)
{
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    const double dc = i ? a.cdf[i] - a.cdf[i - 1] : 0.0;
    a.cs[i] = make_double2(a.cdf[i], dc > 0.0 ? (a.vals[i] - a.vals[i - 1]) / dc : 0.0);
  }
  if (a.n > 0)
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j <= dev::kGuideBuckets; j += stride) {
      const double key = (double)j / dev::kGuideBuckets;
      int lo = 0, hi = a.n;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a.cdf[mid] < key)
          lo = mid + 1;
        else
          hi = mid;
      }
      a.guide[j] = lo < a.n - 1 ? lo : a.n - 1;
    }
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.amp_n; k += stride) {
    const double4 v = make_double4(a.s1[2 * k], a.s1[2 * k + 1], a.s2[2 * k], a.s2[2 * k + 1]);
    a.amp_d[k] = v;
    a.amp_f[k] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)v.w);
  }
}

}  // namespace
}  // namespace lmc

extern "C" lmc_status lmc_run_noalloc(const lmc_scene *s, uint64_t seed, uint64_t photon_begin,
                                      uint64_t n_photons, const lmc_run_opts *opts,
                                      double *d_tallies, lmc_stats *stats)
{
  using namespace lmc;
  if (!opts)
    return fail(LMC_ERR_INVALID, "options must not be null");
  NvtxRange range("lmc_run_noalloc");
  const lmc_status v = validate(s);
  if (v != LMC_OK)
    return v;
  for (int i = 0; i < s->n_sensors; ++i)
    if (s->sensors[i].kind == LMC_SENSOR_FARFIELD_CBS && s->sensors[i].estimator && s->sensors[i].z == 0.0)
      return fail(LMC_ERR_UNSUPPORTED, "lmc_run_noalloc: estimator-mode FarFieldCBS is not available here");
  if (opts->precision != LMC_PRECISION_FP32 && opts->precision != LMC_PRECISION_FP64)
    return fail(LMC_ERR_INVALID, "unknown precision");
  if (opts->max_events < 0)
    return fail(LMC_ERR_INVALID, "max_events must be non-negative");
  for (int i = 0; i < s->n_sensors; ++i)
    if (s->sensors[i].kind == LMC_SENSOR_FARFIELD_CBS && !opts->track_reverse_paths)
      return fail(LMC_ERR_INVALID, "FarFieldCBSSensor needs track_reverse_paths (the reference "
                                   "dereferences null species pointers without it)");
  int device = 0, sm_count = 0;
  LMC_CUDA(cudaGetDevice(&device));
  LMC_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device));
  unsigned char *base = nullptr;
  const lmc_status b = noalloc_base(device, &base);
  if (b != LMC_OK)
    return b;
  cudaStream_t stream = static_cast<cudaStream_t>(opts->stream);

  // ---- device scene, built on the stack (no device allocation): the same fields as
  // lmc_create's, tables patched in below
  dev::Scene sc;
  size_t sensor_off[LMC_MAX_SENSORS], sensor_count[LMC_MAX_SENSORS], abs_off = 0, abs_count = 0;
  int sensor_dims[LMC_MAX_SENSORS][4], abs_dims[4];
  const size_t tally_doubles = fill_scene_head(s, 0, sc, sensor_off, sensor_count, sensor_dims,
                                               &abs_off, &abs_count, abs_dims);
  const bool queued = scene_queued(sc);
  const int n_planes = sc.n_planes;
  const unsigned cbs_mask = sc.cbs_mask;
  if (tally_doubles && !d_tallies)
    return fail(LMC_ERR_INVALID, "device tally buffer must not be null");

  // ---- tables: base arrays copied in, derived arrays computed on the device
  auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
  size_t toff = 0;
  struct MediumSpan { size_t vals, cdf, cs, guide, s1, s2, amp_d, amp_f; };
  MediumSpan span[LMC_MAX_MEDIA];
  for (int i = 0; i < s->n_media; ++i) {
    const lmc_medium_desc &M = s->media[i];
    const size_t nt = (M.theta_kind == LMC_THETA_TABLE || M.theta_kind == LMC_THETA_TABLE_COS)
                          ? (size_t)M.theta_n : 0;
    MediumSpan &p = span[i];
    p.vals = toff; toff = align(toff + nt * sizeof(double));
    p.cdf = toff; toff = align(toff + nt * sizeof(double));
    p.cs = toff; toff = align(toff + nt * sizeof(double2));
    p.guide = toff; toff = align(toff + (nt ? (dev::kGuideBuckets + 1) * sizeof(int) : 0));
    p.s1 = toff; toff = align(toff + (size_t)M.amp_n * 2 * sizeof(double));
    p.s2 = toff; toff = align(toff + (size_t)M.amp_n * 2 * sizeof(double));
    p.amp_d = toff; toff = align(toff + (size_t)M.amp_n * sizeof(double4));
    p.amp_f = toff; toff = align(toff + (size_t)M.amp_n * sizeof(float4));
  }
  dev::StatHist stat[LMC_MAX_SENSORS];                       // StatisticsSensor histograms
  size_t stat_toff[LMC_MAX_SENSORS] = {};
  for (int i = 0; i < s->n_sensors; ++i)
    if (s->sensors[i].kind == LMC_SENSOR_STATISTICS) {
      stat[i] = stat_hist(s->sensors[i], sc.sensors[i].N_t);
      stat_toff[i] = toff;
      toff = align(toff + sizeof(dev::StatHist));
    }
  if (toff > kNaTablesBytes)
    return fail(LMC_ERR_INVALID, "lmc_run_noalloc: the scene's tables need " + std::to_string(toff) +
                                     " bytes of device memory; this entry point holds at most " +
                                     std::to_string(kNaTablesBytes) + " (use lmc_create/lmc_run)");
  unsigned char *tb = base + kNaTablesOff;
  for (int i = 0; i < s->n_media; ++i) {
    const lmc_medium_desc &M = s->media[i];
    const MediumSpan &p = span[i];
    dev::Medium &d = sc.media[i];
    const int nt = d.theta_n;
    DeriveArgs a;
    std::memset(&a, 0, sizeof(a));
    if (nt) {
      d.th_val_d = reinterpret_cast<const double *>(tb + p.vals);
      d.th_cdf_d = reinterpret_cast<const double *>(tb + p.cdf);
      d.th_cs = reinterpret_cast<const double2 *>(tb + p.cs);
      d.guide_d = reinterpret_cast<const int *>(tb + p.guide);
      LMC_CUDA(cudaMemcpyAsync(tb + p.vals, M.theta_values, nt * sizeof(double),
                               cudaMemcpyHostToDevice, stream));
      LMC_CUDA(cudaMemcpyAsync(tb + p.cdf, M.theta_cdf, nt * sizeof(double),
                               cudaMemcpyHostToDevice, stream));
      a.vals = d.th_val_d;
      a.cdf = d.th_cdf_d;
      a.n = nt;
      a.cs = reinterpret_cast<double2 *>(tb + p.cs);
      a.guide = reinterpret_cast<int *>(tb + p.guide);
    }
    d.amp_d = reinterpret_cast<const double4 *>(tb + p.amp_d);
    d.amp_f = reinterpret_cast<const float4 *>(tb + p.amp_f);
    LMC_CUDA(cudaMemcpyAsync(tb + p.s1, M.amp_s1, (size_t)M.amp_n * 2 * sizeof(double),
                             cudaMemcpyHostToDevice, stream));
    LMC_CUDA(cudaMemcpyAsync(tb + p.s2, M.amp_s2, (size_t)M.amp_n * 2 * sizeof(double),
                             cudaMemcpyHostToDevice, stream));
    a.s1 = reinterpret_cast<const double *>(tb + p.s1);
    a.s2 = reinterpret_cast<const double *>(tb + p.s2);
    a.amp_n = M.amp_n;
    a.amp_d = reinterpret_cast<double4 *>(tb + p.amp_d);
    a.amp_f = reinterpret_cast<float4 *>(tb + p.amp_f);
    derive_tables<<<64, 256, 0, stream>>>(a);
    LMC_CUDA(cudaGetLastError());
  }
  for (int i = 0; i < s->n_sensors; ++i)
    if (s->sensors[i].kind == LMC_SENSOR_STATISTICS) {
      sc.sensors[i].stat = reinterpret_cast<const dev::StatHist *>(tb + stat_toff[i]);
      LMC_CUDA(cudaMemcpyAsync(tb + stat_toff[i], &stat[i], sizeof(dev::StatHist),
                               cudaMemcpyHostToDevice, stream));
    }
  dev::Scene *d_scene = reinterpret_cast<dev::Scene *>(base + kNaSceneOff);
  dev::Scratch *d_counters = reinterpret_cast<dev::Scratch *>(base + kNaCountersOff);
  LMC_CUDA(cudaMemcpyAsync(d_scene, &sc, sizeof(sc), cudaMemcpyHostToDevice, stream));
  // the array keeps the previous call's contents: counters must start at zero
  LMC_CUDA(cudaMemsetAsync(d_counters, 0, sizeof(dev::Scratch), stream));

  // ---- launches: the same kernels and batch loop as lmc_run, queue in the array
  dev::RunParams rp;
  std::memset(&rp, 0, sizeof(rp));
  rp.key0 = (uint32_t)seed;
  rp.key1 = (uint32_t)(seed >> 32);
  rp.max_events = opts->max_events;
  rp.track_reverse = opts->track_reverse_paths ? 1 : 0;
  rp.tallies = d_tallies;
  rp.records = static_cast<lmc_record *>(opts->records);
  rp.scratch = d_counters;
  rp.cbs_mask = cbs_mask;
  const bool fp32 = opts->precision == LMC_PRECISION_FP32;
  if (opts->stream_format != 0 && opts->stream_format != 1)
    return fail(LMC_ERR_INVALID, "stream_format must be 0 or 1");
  rp.stream_u24 = (!fp32 && opts->stream_format == 1) ? 1 : 0;
  const int block = opts->block_size > 0 ? opts->block_size : dev::kBlock;
  if (block % 32 != 0 || block > dev::kBlock)
    return fail(LMC_ERR_INVALID, "block_size must be a multiple of 32 and at most 256");
  // the kernels lmc_run picks for the same scene and options
  const bool wide = fp32 && queued && (opts->blocks_per_sm == 0 || opts->blocks_per_sm >= 3);
  const KernelFn tk = pick_transport(fp32, queued, wide, false, false, false, scene_extras(sc));
  TallyLaunch tl{};
  if (queued && s->n_sensors > 0) {
    const lmc_status st = tally_setup(opts->tally_mode, false, fp32, false, sc, sensor_count, device,
                                      0, rp, tl);
    if (st != LMC_OK)
      return st;
  }
  const size_t dyn_transport = fp32 ? dev::side_bytes<float>() : dev::side_bytes<double>();
  rp.side_off = (unsigned)dyn_transport;
  LMC_CUDA(cudaFuncSetAttribute((const void *)tk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dyn_transport));
  int per_sm = 0;
  LMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)tk, block, dyn_transport));
  if (opts->blocks_per_sm > 0)
    per_sm = std::min(per_sm, opts->blocks_per_sm);
  per_sm = std::max(per_sm, 1);
  unsigned long long batch = n_photons;
  if (queued && n_photons > 0) {
    const size_t entry = dev::kQU32Fields * 4 + dev::kQF64Fields * 8 +
                         dev::kQRFields * (fp32 ? sizeof(float) : sizeof(double));
    const unsigned long long cap = (kNoAllocBytes - kNaQueueOff - 3 * 256) / entry;
    const unsigned long long planes_n = std::max(1, n_planes);
    // cap = batch * planes + batch / 16 + 1024, as in lmc_run; a smaller batch_photons
    // of the options is honoured
    batch = std::min<unsigned long long>(n_photons, ((cap - 1024) * 16) / (16 * planes_n + 1));
    if (opts->batch_photons)
      batch = std::min<unsigned long long>(batch, opts->batch_photons);
    if (batch == 0)
      return fail(LMC_ERR_INVALID, "lmc_run_noalloc: too many sensor planes for the hit queue");
    unsigned char *q = base + kNaQueueOff;
    rp.queue.cap = cap;
    rp.queue.u32 = reinterpret_cast<uint32_t *>(q);
    size_t o = align((size_t)cap * dev::kQU32Fields * 4);
    rp.queue.f64 = reinterpret_cast<double *>(q + o);
    o += align((size_t)cap * dev::kQF64Fields * 8);
    rp.queue.r = q + o;
  }
  lmc_record *const records = static_cast<lmc_record *>(opts->records);
  for (unsigned long long done = 0; done < n_photons; done += batch) {
    const unsigned long long nb = std::min(batch, n_photons - done);
    rp.photon_begin = photon_begin + done;
    rp.n_photons = nb;
    rp.records = records ? records + done : nullptr;   // the kernels index from photon_begin
    LMC_CUDA(cudaMemsetAsync(d_counters, 0, 4 * sizeof(unsigned long long), stream));
    const int grid = (int)std::max<unsigned long long>(
        1ull, std::min<unsigned long long>((unsigned long long)sm_count * per_sm, (nb + block - 1) / block));
    tk<<<grid, block, dyn_transport, stream>>>(d_scene, rp);
    LMC_CUDA(cudaGetLastError());
    if (queued && s->n_sensors > 0) {
      const int tgrid = (int)std::max<unsigned long long>(
          1ull, std::min<unsigned long long>((unsigned long long)sm_count * tl.grid_per_sm,
                                             (rp.queue.cap + dev::kBlock - 1) / dev::kBlock));
      tl.fn<<<tgrid, dev::kBlock, tl.dyn, stream>>>(d_scene, rp);
      LMC_CUDA(cudaGetLastError());
    }
  }
  dev::Scratch c;
  LMC_CUDA(cudaMemcpyAsync(&c, d_counters, sizeof(c), cudaMemcpyDeviceToHost, stream));
  LMC_CUDA(cudaStreamSynchronize(stream));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->photons = c.photons; stats->events = c.events; stats->steps = c.steps;
    stats->detected = c.detected; stats->escaped = c.escaped; stats->stack = c.stack;
    stats->roulette = c.roulette; stats->cap = c.cap; stats->draws = c.draws;
    for (int i = 0; i < LMC_MAX_SENSORS; ++i)
      stats->hits[i] = c.hits[i];
    stats->error_flags = c.error_flags;
    stats->kernel_ms = 0.f;                  // not timed: timing events would be allocations
  }
  if (c.error_flags)
    return fail(LMC_ERR_KERNEL, "transport kernel raised error flags " + std::to_string(c.error_flags));
  return bounds_status(stream);
}
